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
  // when set, u, e_shifted and e0 = e_shifted + shift are read from the device Rayleigh-Ritz
  // result instead (rr_solve: u_dev[k], e_dev[0])
  const double *u_dev = nullptr, *e_dev = nullptr;
  double shift = 0.0;
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
// Exchange-symmetric subspace (every S_k and sigma(S_k) exactly symmetric): the residual pass with
// the projection of t folded in, reading one tile of each 32 x 32 tile pair (no W; slots as
// residual_step_async: W.W, r.r, S_k.t, t.t), and a Gram-Schmidt round the same way (slots: t.t,
// S_k.t with want_dots; t0_slot >= 0 makes it the device-decided second round of
// cgs_second_round_async).
template <typename T>
int residual_sym_async(sbd_tpb_handle *h, const ResidualArgs<T> &a, int slot);
// the reference's seeded random start values (reference order and sign convention, not normalised)
int random_start_vector(sbd_tpb_handle *h, double *x, size_t n, unsigned long long seed);
// the last step of a cycle (W out, no correction) on an exchange-symmetric subspace, tile pairs
template <typename T>
int residual_w_sym_async(sbd_tpb_handle *h, const ResidualArgs<T> &a, int slot);
template <typename T>
int cgs_sym_async(sbd_tpb_handle *h, const T *const *C, int m, const double *coef, int ov_slot, T *t,
                  int want_dots, int slot, int t0_slot = -1, int tt_slot = -1);
// the same, and S_k . x_new (k < m, S_k exactly symmetric) into scalar slots slot..
template <typename T>
int sym_add_dots(sbd_tpb_handle *h, T *x, const T *const *S, int m, int slot);
// x <- (x + x^T) / 2 (the exchange projection), S_k . x_new into slots slot .. slot+m-1 and x_new . x_new
// into slot+m, in one tile-pair pass
template <typename T>
int symmetrize_dots(sbd_tpb_handle *h, T *x, const T *const *S, int m, int slot);

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

// Device Rayleigh-Ritz of the Davidson subspace (replaces the host dsyev of tpb/davidson.h:
// 770-780).  The projected matrix lives in h->d_rr (kMaxSub x kMaxSub, column-major): rr_solve
// sets its column/row ib to f_k f_ib ov_k (ov = the overlaps S_k . sigma(S_ib) in device slots
// ov_slot..), solves the leading (ib+1) x (ib+1) eigenproblem with a cyclic Jacobi method
// (eigenvalues sorted ascending), and leaves u_k = U_k0 f_k at rr_u(h), the eigenvalues at
// rr_e(h) and the lowest four in slots eig_slot.. (for the host's convergence and print lines).
struct ScaleArray {
  double v[kMaxSub];
};
int rr_solve(sbd_tpb_handle *h, int ib, const ScaleArray &f, int ov_slot, int eig_slot);
const double *rr_u(sbd_tpb_handle *h);
const double *rr_e(sbd_tpb_handle *h);
// multi_dot into device slots (no host round trip): slot + j = X_j . y
template <typename T>
int multi_dot_async(sbd_tpb_handle *h, const T *const *X, int k, const T *y, size_t n, int slot);
// second Gram-Schmidt round, run only where the first cancelled more than half of |t|^2: t -=
// sum_k coef_k ov_k C_k when slot tt_slot < 0.5 * slot t0_slot (both device values); the new
// t.t goes to slot `slot`, or 0 there when the round is skipped
template <typename T>
int cgs_second_round_async(sbd_tpb_handle *h, const T *const *C, int m, const double *coef, int ov_slot, T *t,
                           size_t n, int t0_slot, int tt_slot, int slot);
template <typename S, typename D>
int convert_vec(sbd_tpb_handle *h, const S *x, D *y, size_t n);
template <typename T>
int axpby(sbd_tpb_handle *h, const T *x, T *y, double a, double b, size_t n);

}  // namespace sbdtpb
