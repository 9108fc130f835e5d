// Lanczos for the lowest root (--method 2): the reference's matrix-free Lanczos
// (tpb/lanczos.h:167-320; dispatched from tpb/sbdiag.h:404-411), on the same sigma as Davidson.
//
// Per outer iteration, from the current W:
//   C_0 = W, HC = 0
//   step k: HC += H C_k; alpha_k = <C_k, HC>; lowest eigenvalues of the (k+1)x(k+1) tridiagonal
//   T; stop when the lowest moved by less than eps; otherwise r = HC - alpha_k C_k,
//   beta_k = |r|, C_{k+1} = r / beta_k, HC = -beta_k C_k (so the next sigma completes the
//   three-term recurrence); end the iteration early when beta_k < eps.
//   W = sum_k u_k C_k with u the lowest eigenvector of T.
// There is no reorthogonalisation, as in the reference.  Unlike the reference, W is renormalised
// after each outer iteration (see below); with orthonormal Krylov vectors its norm is 1 anyway.
// The vectors stay in HBM (FP64, separated convention); each step is one accumulating sigma plus
// two fused vector passes and a dot, with two host reads (alpha, beta^2).  T is tridiagonal, so its eigenvalues come from Sturm-sequence
// bisection and the lowest eigenvector from inverse iteration with a pivoted tridiagonal
// factorisation, instead of the reference's dense LAPACK dsyev on the same matrix (same
// eigenvalues; the eigenvector's sign is fixed here by u_0 >= 0, where dsyev leaves it to the
// implementation, so W may come out with the opposite global sign).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <limits>
#include <vector>

#include "tpb_common.cuh"
#include "vecops.cuh"

namespace sbdtpb {
namespace {

constexpr int kLzThreads = 256;

// ---- host: symmetric tridiagonal T (diagonal a[0..n), off-diagonal b[0..n-1)) ---------------

// number of eigenvalues of T below x (signs of the LDL^T pivots of T - x I)
int sturm_below(const std::vector<double> &a, const std::vector<double> &b, int n, double x) {
  const double tiny = std::numeric_limits<double>::min();
  int c = 0;
  double d = 1.0;
  for (int i = 0; i < n; i++) {
    d = (a[i] - x) - (i ? b[i - 1] * b[i - 1] / d : 0.0);
    if (d == 0.0) d = -tiny;
    if (d < 0.0) c++;
  }
  return c;
}

// k-th smallest eigenvalue (0-based) by bisection inside the Gershgorin interval
double tridiag_eigenvalue(const std::vector<double> &a, const std::vector<double> &b, int n, int k) {
  double lo = a[0], hi = a[0];
  for (int i = 0; i < n; i++) {
    const double r = (i ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(b[i]) : 0.0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  const double eps = std::numeric_limits<double>::epsilon();
  for (int it = 0; it < 2000 && hi - lo > 2.0 * eps * (std::fabs(lo) + std::fabs(hi)) + 1e-300; it++) {
    const double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    if (sturm_below(a, b, n, mid) > k) hi = mid;
    else lo = mid;
  }
  return 0.5 * (lo + hi);
}

// eigenvector of T for eigenvalue s: inverse iteration, T - s I factorised with partial pivoting
// (row interchanges give a second super-diagonal), three solves from a vector of ones
void tridiag_eigenvector(const std::vector<double> &a, const std::vector<double> &b, int n, double s,
                         std::vector<double> &x) {
  x.assign(n, 1.0);
  if (n == 1) return;
  double scale = 0.0;
  for (int i = 0; i < n; i++) scale = std::max(scale, std::fabs(a[i]) + (i + 1 < n ? std::fabs(b[i]) : 0.0));
  const double tiny = std::numeric_limits<double>::epsilon() * std::max(scale, 1e-300);
  std::vector<double> dl(n - 1), d(n), du(n - 1), du2(n, 0.0);
  std::vector<char> swapped(n, 0);
  for (int i = 0; i < n; i++) d[i] = a[i] - s;
  for (int i = 0; i + 1 < n; i++) dl[i] = du[i] = b[i];
  for (int i = 0; i + 1 < n; i++) {
    if (std::fabs(d[i]) >= std::fabs(dl[i])) {
      if (d[i] == 0.0) d[i] = tiny;
      const double l = dl[i] / d[i];
      dl[i] = l;
      d[i + 1] -= l * du[i];
    } else {
      swapped[i] = 1;
      const double l = d[i] / dl[i];
      d[i] = dl[i];
      dl[i] = l;
      const double t = du[i];
      du[i] = d[i + 1];
      d[i + 1] = t - l * d[i + 1];
      if (i + 2 < n) {
        du2[i] = du[i + 1];
        du[i + 1] = -l * du[i + 1];
      }
    }
  }
  if (d[n - 1] == 0.0) d[n - 1] = tiny;
  for (int rep = 0; rep < 3; rep++) {
    for (int i = 0; i + 1 < n; i++) {
      if (!swapped[i]) {
        x[i + 1] -= dl[i] * x[i];
      } else {
        const double t = x[i];
        x[i] = x[i + 1];
        x[i + 1] = t - dl[i] * x[i + 1];
      }
    }
    x[n - 1] /= d[n - 1];
    x[n - 2] = (x[n - 2] - du[n - 2] * x[n - 1]) / d[n - 2];
    for (int i = n - 3; i >= 0; i--) x[i] = (x[i] - du[i] * x[i + 1] - du2[i] * x[i + 2]) / d[i];
    double nrm = 0.0;
    for (int i = 0; i < n; i++) nrm += x[i] * x[i];
    nrm = std::sqrt(nrm);
    if (!(nrm > 0.0) || !std::isfinite(nrm)) break;
    for (int i = 0; i < n; i++) x[i] /= nrm;
  }
  if (x[0] < 0.0)
    for (int i = 0; i < n; i++) x[i] = -x[i];
}

// ---- device passes ---------------------------------------------------------------------------

// HC <- HC - alpha C; partials[block] = sum of the new HC^2 over the block's elements (fixed
// element-to-block assignment, so the host's in-order sum of the partials is deterministic)
__global__ void __launch_bounds__(kLzThreads) lz_residual_kernel(const double *__restrict__ C,
                                                                 double *__restrict__ HC, double alpha,
                                                                 size_t n, double *__restrict__ partials) {
  __shared__ double red[kLzThreads / 32];
  double acc = 0.0;
  const size_t n2 = n / 2;
  const double2 *C2 = reinterpret_cast<const double2 *>(C);
  double2 *H2 = reinterpret_cast<double2 *>(HC);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n2; i += (size_t)gridDim.x * blockDim.x) {
    const double2 c = C2[i];
    double2 r = H2[i];
    r.x -= alpha * c.x;
    r.y -= alpha * c.y;
    H2[i] = r;
    acc += r.x * r.x + r.y * r.y;
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const double r = HC[n - 1] - alpha * C[n - 1];
    HC[n - 1] = r;
    acc += r * r;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kLzThreads / 32; w++) s += red[w];
    partials[blockIdx.x] = s;
  }
}

// Cnext <- HC / beta; HC <- -beta C
__global__ void __launch_bounds__(kLzThreads) lz_advance_kernel(const double *__restrict__ C,
                                                                double *__restrict__ HC,
                                                                double *__restrict__ Cnext, double beta,
                                                                size_t n) {
  const double inv = 1.0 / beta;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    Cnext[i] = HC[i] * inv;
    HC[i] = -beta * C[i];
  }
}

// W <- u C (first term of the Ritz vector)
__global__ void lz_scale_set_kernel(const double *__restrict__ C, double *__restrict__ W, double u, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    W[i] = u * C[i];
}

}  // namespace

int lanczos_run(sbd_tpb_handle *h, const sbd_tpb_params *p, const double *W0, sbd_tpb_result *res) {
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "lanczos: tables not built");
  if (p->max_nb < 1 || p->max_nb > 4096) return fail(SBD_TPB_ERR_INVALID, "lanczos: --block must be in [1, 4096]");
  if (p->max_it < 1) return fail(SBD_TPB_ERR_INVALID, "lanczos: --iteration must be >= 1");
  if (p->precision != SBD_TPB_FP64)
    return fail(SBD_TPB_ERR_INVALID, "lanczos: runs in FP64 only (--precision fp64)");
  const size_t n = h->ndet();
  const int nb = p->max_nb;
  const auto t0 = std::chrono::steady_clock::now();
  const int blocks = vec_blocks(h);
  TPB_CHECK(ensure_partials(h, blocks));

  DevVec<double> W, HC;
  std::vector<DevVec<double>> C(nb);
  TPB_CHECK(W.get(h, n));
  TPB_CHECK(HC.get(h, n));
  for (int k = 0; k < nb; k++) TPB_CHECK(C[k].get(h, n));

  // start: the stored vector (reference convention in, separated inside), the first determinant
  // (BasisInitVector with init 0, tpb/davidson.h:134-137; no normalisation, as in the reference) or
  // the seeded random vector, normalised (init 1, tpb/davidson.h:138-141)
  if (W0) {
    TPB_CUDA(cudaMemcpyAsync(W.p, W0, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    TPB_CHECK(reorder_sign_apply_f64(h, W.p, W.p));
  } else if (p->init == 1) {
    TPB_CHECK(random_start_vector(h, W.p, n, p->seed));
    TPB_CHECK(reorder_sign_apply_f64(h, W.p, W.p));
    const double *wp[1] = {W.p};
    double nrm = 0.0;
    TPB_CHECK(multi_dot<double>(h, wp, 1, W.p, n, &nrm));
    if (!(nrm > 0.0)) return fail(SBD_TPB_ERR_INVALID, "initial vector is zero");
    TPB_CHECK(scale_vec<double>(h, W.p, 1.0 / std::sqrt(nrm), n));
  } else {
    TPB_CUDA(cudaMemsetAsync(W.p, 0, sizeof(double) * n, h->stream));
    const double one = 1.0;
    TPB_CUDA(cudaMemcpyAsync(W.p, &one, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  }

  std::vector<double> alpha(nb, 0.0), beta(nb, 0.0), part(blocks), u;
  int nsig = 0, conv = 0;
  for (int it = 0; it < p->max_it; it++) {
    TPB_CUDA(cudaMemcpyAsync(C[0].p, W.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
    TPB_CUDA(cudaMemsetAsync(HC.p, 0, sizeof(double) * n, h->stream));
    int m = 0;
    double E_old = 1.0e+8;
    bool stop = false;
    for (int ib = 0; ib < nb; ib++) {
      m++;
      TPB_CHECK(sigma_sep<double>(h, C[ib].p, HC.p, 1));
      nsig++;
      const double *cp[1] = {C[ib].p};
      TPB_CHECK(multi_dot<double>(h, cp, 1, HC.p, n, &alpha[ib]));
      const int ne = std::min(m, 4);
      double E[4];
      for (int k = 0; k < ne; k++) E[k] = tridiag_eigenvalue(alpha, beta, m, k);
      if (std::fabs(E[0] - E_old) < p->eps) {
        stop = true;
        break;
      }
      E_old = E[0];
      if (ib + 1 == nb) break;
      lz_residual_kernel<<<blocks, kLzThreads, 0, h->stream>>>(C[ib].p, HC.p, alpha[ib], n, h->d_partials);
      TPB_LAUNCHED(h);
      TPB_CUDA(cudaMemcpyAsync(part.data(), h->d_partials, sizeof(double) * blocks, cudaMemcpyDeviceToHost,
                               h->stream));
      TPB_CUDA(cudaStreamSynchronize(h->stream));
      double bb = 0.0;
      for (int b = 0; b < blocks; b++) bb += part[b];
      beta[ib] = std::sqrt(bb);
      if (p->verbose) {
        std::printf(" Lanczos iteration %d, step %d: (A,B)=(%.16g,%.16g):", it, ib, alpha[ib], beta[ib]);
        for (int k = 0; k < ne; k++) std::printf(" %.16g", E[k]);
        std::printf("\n");
        std::fflush(stdout);
      }
      if (std::fabs(beta[ib]) < p->eps) break;
      lz_advance_kernel<<<blocks, kLzThreads, 0, h->stream>>>(C[ib].p, HC.p, C[ib + 1].p, beta[ib], n);
      TPB_LAUNCHED(h);
    }
    // Ritz vector of the lowest eigenvalue of the m x m tridiagonal
    const double lam = tridiag_eigenvalue(alpha, beta, m, 0);
    tridiag_eigenvector(alpha, beta, m, lam, u);
    lz_scale_set_kernel<<<blocks, kLzThreads, 0, h->stream>>>(C[0].p, W.p, u[0], n);
    TPB_LAUNCHED(h);
    for (int k = 1; k < m; k++) TPB_CHECK(axpby<double>(h, C[k].p, W.p, u[k], 1.0, n));
    // renormalised restart: without reorthogonalisation the Krylov vectors lose orthogonality once
    // the lowest Ritz value converges, and the norm of sum_k u_k C_k drifts from 1; restarting from
    // such a W biases the next alpha_0 = <W|H|W> and the drift grows at every restart
    double ww = 0.0;
    const double *wp[1] = {W.p};
    TPB_CHECK(multi_dot<double>(h, wp, 1, W.p, n, &ww));
    if (!(ww > 0.0)) return fail(SBD_TPB_ERR_NOT_CONVERGED, "lanczos: the Ritz vector vanished");
    TPB_CHECK(scale_vec<double>(h, W.p, 1.0 / std::sqrt(ww), n));
    if (stop) {
      conv = 1;
      break;
    }
  }
  // the Krylov vectors go back to the pool before the final sigma and the RDMs
  C.clear();
  HC.release();
  return solve_finish(h, W.p, res, t0, nsig, conv, -1.0);
}

}  // namespace sbdtpb
