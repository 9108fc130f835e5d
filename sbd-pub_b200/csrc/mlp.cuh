// Learned Davidson preconditioner: internal interfaces (kernels and training in mlp.cu).
#pragma once

#include <vector>

#include "tpb_common.cuh"

namespace sbdtpb {

constexpr int kMlpHidden = SBD_TPB_MLP_HIDDEN;   // width of both hidden layers
constexpr int kMlpFeat = SBD_TPB_MLP_FEATURES;   // input width (K of the first layer)
constexpr int kMlpWin = 24;                      // orbitals per spin around the Fermi level
constexpr float kMlpBound = 0.5f;                // correction factor 1 + 0.5 tanh(y) in (0.5, 1.5)

// Steps of a Davidson run kept for training (FP32 copies, separated convention).  Step k: the
// diagonal correction d_k = r_k / (E_k - H_ii), E_k, |r_k| and the indices of its orthonormal
// basis vectors C_j = scale_j * vec_j (a cycle's start vector, then the Gram-Schmidt images of
// the corrections actually added).  The run may use the learned correction, so pairs can be
// collected along the learned solver's own trajectory.
struct DavRecord {
  std::vector<float *> d;
  std::vector<double> e0, rnorm;
  std::vector<std::vector<int>> basis;  // per step: indices into vec/scale
  std::vector<const float *> vec;       // basis vectors (owned through owned)
  std::vector<double> scale;
  std::vector<float *> owned;
  int max_steps = 64;
  DavRecord() = default;
  DavRecord(const DavRecord &) = delete;
  DavRecord &operator=(const DavRecord &) = delete;
  ~DavRecord() {
    for (float *p : owned) cudaFree(p);
  }
};

// FP64 Davidson with recording (diagonal correction, or the learned one when learned is given);
// Psi (device, n doubles) receives the normalised final vector, energy the last Ritz value.
int davidson_record(sbd_tpb_handle *h, const sbd_tpb_params *p, DavRecord *rec, double *Psi,
                    double *energy, sbd_tpb_precond *learned);

// Most determinants the network corrects per application; beyond it only the entries with
// |d_i| >= |d| / sqrt(budget) are corrected (the others keep the diagonal correction).
constexpr size_t kMlpBudget = (size_t)1 << 22;

// t[i] <- t[i] * (1 + y_i) in place, t holding the diagonal correction of Ritz value e0 and
// residual norm rnorm (tt = t.t, 0 = correct every entry) on the handle's stream.
template <typename T>
int precond_apply(sbd_tpb_handle *h, sbd_tpb_precond *p, T *t, double e0, double rnorm, double tt);

// Occupation window of one string: bit q = occupation of orbital nel - 12 + q (1 below orbital 0).
__host__ __device__ inline uint32_t occ_window(uint64_t s, int nel) {
  uint32_t w = 0;
  for (int q = 0; q < kMlpWin; q++) {
    const int p = nel - kMlpWin / 2 + q;
    const uint32_t bit = p < 0 ? 1u : (p >= 64 ? 0u : (uint32_t)((s >> p) & 1ull));
    w |= bit << q;
  }
  return w;
}

}  // namespace sbdtpb
