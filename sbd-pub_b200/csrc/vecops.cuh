// Davidson vector-kernel interfaces (see vecops.cu).
#pragma once

#include "tpb_common.cuh"

namespace sbdtpb {

constexpr int kVecThreads = 256;
constexpr int kMaxSub = 16;            // largest Davidson subspace handled by the fused kernels
constexpr int kMaxVec = kMaxSub + 3;   // values reduced per pass

template <typename T>
struct VecPtrs {
  const T *p[kMaxVec];
};

struct CoefArray {
  double v[kMaxSub];
};

template <typename T>
struct ResidualArgs {
  VecPtrs<T> C, HC;   // stored subspace vectors S_k and sigma(S_k); true C_k = f_k S_k
  double u[kMaxSub];  // Ritz coefficients already multiplied by the scale factors f_k
  int m;              // subspace size
  double e_shifted;   // Ritz value of (H - shift)
  double e0;          // Ritz value of H
  const double *hii;  // FP64 diagonal (FP64 vectors)
  const float *hii32; // H_ii - H_00 in FP32 (FP32 vectors; used with e_shifted = E - H_00)
  T *W;               // Ritz vector out (may be null)
  T *t;               // preconditioned correction out (may be null: W only)
};

int vec_blocks(sbd_tpb_handle *h);
template <typename T>
int residual_step(sbd_tpb_handle *h, const ResidualArgs<T> &a, size_t n, double *out);
template <typename T>
int cgs_update(sbd_tpb_handle *h, const T *const *C, int m, const double *o, T *t, size_t n,
               int want_dots, double *out);
template <typename T>
int scale_vec(sbd_tpb_handle *h, T *x, double a, size_t n);
// t <- (t + t^T)/2 over the square (alpha = beta strings) determinant matrix; tt = new t.t
template <typename T>
int symmetrize(sbd_tpb_handle *h, T *t, double *tt);
// x <- x + x^T over the square determinant matrix (in place, no reduction)
template <typename T>
int sym_add(sbd_tpb_handle *h, T *x);

// The same passes without a host round trip: each reduces into slots of a small device array
// (kScalarSlots doubles), read back together by fetch_scalars (one stream synchronisation).
// cgs_update_async takes the overlaps from device slots ov_slot.. (o_k = coef[k] * overlap_k).
constexpr int kScalarSlots = 64;
template <typename T>
int residual_step_async(sbd_tpb_handle *h, const ResidualArgs<T> &a, size_t n, int slot);
template <typename T>
int symmetrize_async(sbd_tpb_handle *h, T *t, int slot);
template <typename T>
int cgs_update_async(sbd_tpb_handle *h, const T *const *C, int m, const double *coef, int ov_slot, T *t,
                     size_t n, int want_dots, int slot);
const double *fetch_scalars(sbd_tpb_handle *h, int count);
template <typename S, typename D>
int convert_vec(sbd_tpb_handle *h, const S *x, D *y, size_t n);
template <typename T>
int axpby(sbd_tpb_handle *h, const T *x, T *y, double a, double b, size_t n);

}  // namespace sbdtpb
