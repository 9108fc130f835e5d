// Davidson driver (host side of the loop; kernels in vecops.cu and sigma.cu).
//
// Follows the reference's block Davidson for the lowest root (tpb/davidson.h:667-930,
// basic/davidson_thrust.h:85-373): subspace C_0..C_k with HC_k = H C_k, Rayleigh-Ritz on the
// (k+1)x(k+1) projection, W = sum U_k0 C_k, R = E0 W - H W, convergence when |R| < eps, diagonal
// correction t = R / (E0 - H_ii) with the 1e-12 regularisation, Gram-Schmidt against the subspace,
// restart from W after max_nb steps, and the max_time guard.  The small eigenproblem is solved on
// the host with a cyclic Jacobi method, eigenvalues sorted ascending (the reference calls LAPACK
// dsyev, framework/hp_numeric.h:500-520, which also returns them ascending).
//
// Vectors live in HBM in the separated sign convention.  The FP64 path keeps everything in
// double.  The mixed path stores C/HC/W/t in FP32, computes sigma of (H - s) with s = H_00 so the
// FP32 entries carry residual-sized values, keeps all dot products and the Rayleigh-Ritz in FP64,
// and finishes with one FP64 sigma on the converged vector for the reported energy and residual.
// Both orthogonalise with two rounds of classical Gram-Schmidt (as stable as the reference's
// modified Gram-Schmidt, tpb/davidson.h:871-879, with two fused passes instead of k+1).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <vector>

#include "tpb_common.cuh"
#include "vecops.cuh"

namespace sbdtpb {
namespace {

// Cyclic Jacobi eigen-solver; A is n x n column-major with leading dimension lda (only the
// leading n x n block is read).  On return V holds eigenvectors (columns), E eigenvalues sorted
// ascending.
void jacobi_eigen(int n, const double *A, int lda, std::vector<double> &E, std::vector<double> &V) {
  std::vector<double> M((size_t)n * n);
  V.assign((size_t)n * n, 0.0);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) M[i + (size_t)n * j] = A[i + (size_t)lda * j];
  for (int i = 0; i < n; i++) V[i + (size_t)n * i] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, diag = 0.0;
    for (int j = 0; j < n; j++) {
      diag += M[j + (size_t)n * j] * M[j + (size_t)n * j];
      for (int i = 0; i < j; i++) off += M[i + (size_t)n * j] * M[i + (size_t)n * j];
    }
    if (off <= 1e-32 * (diag + 1e-300)) break;
    for (int p = 0; p < n; p++) {
      for (int q = p + 1; q < n; q++) {
        const double apq = M[p + (size_t)n * q];
        if (std::fabs(apq) < 1e-300) continue;
        const double app = M[p + (size_t)n * p], aqq = M[q + (size_t)n * q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; k++) {
          const double mkp = M[k + (size_t)n * p], mkq = M[k + (size_t)n * q];
          M[k + (size_t)n * p] = c * mkp - s * mkq;
          M[k + (size_t)n * q] = s * mkp + c * mkq;
        }
        for (int k = 0; k < n; k++) {
          const double mpk = M[p + (size_t)n * k], mqk = M[q + (size_t)n * k];
          M[p + (size_t)n * k] = c * mpk - s * mqk;
          M[q + (size_t)n * k] = s * mpk + c * mqk;
        }
        for (int k = 0; k < n; k++) {
          const double vkp = V[k + (size_t)n * p], vkq = V[k + (size_t)n * q];
          V[k + (size_t)n * p] = c * vkp - s * vkq;
          V[k + (size_t)n * q] = s * vkp + c * vkq;
        }
      }
    }
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; i++) ord[i] = i;
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++)
      if (M[ord[j] + (size_t)n * ord[j]] < M[ord[i] + (size_t)n * ord[i]]) std::swap(ord[i], ord[j]);
  std::vector<double> Vs((size_t)n * n);
  E.resize(n);
  for (int k = 0; k < n; k++) {
    E[k] = M[ord[k] + (size_t)n * ord[k]];
    for (int i = 0; i < n; i++) Vs[i + (size_t)n * k] = V[i + (size_t)n * ord[k]];
  }
  V.swap(Vs);
}

template <typename T>
struct DevVec {
  T *p = nullptr;
  ~DevVec() {
    if (p) cudaFree(p);
  }
};

template <typename T>
int run_typed(sbd_tpb_handle *h, const sbd_tpb_params *prm, const double *W0, double shift,
              int cgs_rounds, sbd_tpb_result *res, std::vector<double> &Wout_sep,
              double *resid_out, int *nsigma_out, int *converged_out) {
  const size_t n = h->ndet();
  const int nb = prm->max_nb;
  const int max_it = prm->max_it;
  std::vector<DevVec<T>> C(nb), HC(nb);
  DevVec<T> Wv, tv;
  for (int k = 0; k < nb; k++) {
    TPB_CUDA(cudaMalloc(&C[k].p, sizeof(T) * n));
    TPB_CUDA(cudaMalloc(&HC[k].p, sizeof(T) * n));
  }
  TPB_CUDA(cudaMalloc(&Wv.p, sizeof(T) * n));
  TPB_CUDA(cudaMalloc(&tv.p, sizeof(T) * n));

  // initial vector (separated convention)
  {
    DevVec<double> w64;
    TPB_CUDA(cudaMalloc(&w64.p, sizeof(double) * n));
    if (W0) {
      TPB_CUDA(cudaMemcpyAsync(w64.p, W0, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
      TPB_CHECK(reorder_sign_apply_f64(h, w64.p, w64.p));
    } else {
      // --init 0: the first determinant, i.e. the HF string when it is the smallest
      // (tpb/davidson.h:134-137)
      TPB_CUDA(cudaMemsetAsync(w64.p, 0, sizeof(double) * n, h->stream));
      const double one = 1.0;
      TPB_CUDA(cudaMemcpyAsync(w64.p, &one, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    }
    if (std::is_same<T, double>::value) {
      TPB_CUDA(cudaMemcpyAsync(C[0].p, w64.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
    } else {
      TPB_CHECK((convert_vec<double, T>(h, w64.p, C[0].p, n)));
    }
    double nrm = 0.0;
    const T *cp[1] = {C[0].p};
    TPB_CHECK(multi_dot<T>(h, cp, 1, C[0].p, n, &nrm));
    if (!(nrm > 0.0)) return fail(SBD_TPB_ERR_INVALID, "initial vector is zero");
    TPB_CHECK(scale_vec<T>(h, C[0].p, 1.0 / std::sqrt(nrm), n));
  }

  std::vector<double> Hs((size_t)nb * nb, 0.0), E, U;
  std::vector<double> out(kMaxVec + 2);
  std::vector<double> step_times;
  double norm_R = 0.0, ww = 1.0;
  int nsigma = 0;
  bool converged = false, stop = false;
  const auto t_start = std::chrono::steady_clock::now();

  for (int it = 0; it < max_it && !stop; it++) {
    if (it > 0) {
      // restart from the normalised Ritz vector (tpb/davidson.h:918-922)
      TPB_CUDA(cudaMemcpyAsync(C[0].p, Wv.p, sizeof(T) * n, cudaMemcpyDeviceToDevice, h->stream));
      TPB_CHECK(scale_vec<T>(h, C[0].p, 1.0 / std::sqrt(ww), n));
    }
    for (int ib = 0; ib < nb; ib++) {
      const auto s0 = std::chrono::steady_clock::now();
      TPB_CHECK(sigma_sep_shift<T>(h, C[ib].p, HC[ib].p, 0, shift));
      nsigma++;
      std::vector<const T *> cp(ib + 1);
      for (int k = 0; k <= ib; k++) cp[k] = C[k].p;
      TPB_CHECK(multi_dot<T>(h, cp.data(), ib + 1, HC[ib].p, n, out.data()));
      for (int k = 0; k <= ib; k++) {
        Hs[k + (size_t)nb * ib] = out[k];
        Hs[ib + (size_t)nb * k] = out[k];
      }
      jacobi_eigen(ib + 1, Hs.data(), nb, E, U);
      ResidualArgs<T> ra;
      for (int k = 0; k < kMaxVec; k++) {
        ra.C.p[k] = k <= ib ? C[k].p : nullptr;
        ra.HC.p[k] = k <= ib ? HC[k].p : nullptr;
      }
      for (int k = 0; k < kMaxSub; k++) ra.u[k] = k <= ib ? U[k] : 0.0;
      ra.m = ib + 1;
      ra.e_shifted = E[0];
      ra.e0 = E[0] + shift;
      ra.hii = h->d_hii;
      ra.W = Wv.p;
      T *tnext = (ib < nb - 1) ? C[ib + 1].p : tv.p;
      ra.t = tnext;
      TPB_CHECK(residual_step<T>(h, ra, n, out.data()));
      ww = out[0];
      norm_R = std::sqrt(out[1] / ww);
      if (prm->verbose) {
        std::printf(" Davidson iteration %d.%d (tol=%.16g):", it, ib, norm_R);
        for (int p = 0; p < std::min(ib + 1, 4); p++) std::printf(" %.16g", E[p] + shift);
        std::printf("\n");
        std::fflush(stdout);
      }
      if (norm_R < prm->eps) {
        converged = true;
        stop = true;
        break;
      }
      if (ib < nb - 1) {
        std::vector<double> olap(out.begin() + 2, out.begin() + 2 + ib + 1);
        double tt = 0.0;
        for (int round = 0; round < cgs_rounds; round++) {
          const bool more = round + 1 < cgs_rounds;
          TPB_CHECK(cgs_update<T>(h, cp.data(), ib + 1, olap.data(), tnext, n, more ? 1 : 0,
                                  out.data()));
          tt = out[0];
          if (more) olap.assign(out.begin() + 1, out.begin() + 1 + ib + 1);
        }
        if (!(tt > 0.0)) {
          // the correction lies in the subspace: nothing left to add
          stop = true;
          break;
        }
        TPB_CHECK(scale_vec<T>(h, tnext, 1.0 / std::sqrt(tt), n));
      }
      // max_time guard (tpb/davidson.h:887-913): stop when the next step would overrun
      TPB_CUDA(cudaStreamSynchronize(h->stream));
      const auto s1 = std::chrono::steady_clock::now();
      step_times.push_back(std::chrono::duration<double>(s1 - s0).count());
      double avg = 0.0;
      for (double x : step_times) avg += x;
      avg /= step_times.size();
      const double elapsed = std::chrono::duration<double>(s1 - t_start).count();
      if (elapsed + avg > prm->max_time) {
        std::fprintf(stderr, "halting iterations due to max_time limit\n");
        stop = true;
        break;
      }
    }
  }
  // W = Ritz vector of the last step, normalised, promoted to FP64
  Wout_sep.resize(n);
  {
    DevVec<double> w64;
    TPB_CUDA(cudaMalloc(&w64.p, sizeof(double) * n));
    if (std::is_same<T, double>::value) {
      TPB_CUDA(cudaMemcpyAsync(w64.p, Wv.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
    } else {
      TPB_CHECK((convert_vec<T, double>(h, Wv.p, w64.p, n)));
    }
    double nrm = 0.0;
    const double *wp[1] = {w64.p};
    TPB_CHECK(multi_dot<double>(h, wp, 1, w64.p, n, &nrm));
    TPB_CHECK(scale_vec<double>(h, w64.p, 1.0 / std::sqrt(nrm), n));
    TPB_CUDA(cudaMemcpyAsync(Wout_sep.data(), w64.p, sizeof(double) * n, cudaMemcpyDeviceToHost,
                             h->stream));
    TPB_CUDA(cudaStreamSynchronize(h->stream));
  }
  *resid_out = norm_R;
  *nsigma_out = nsigma;
  *converged_out = converged ? 1 : 0;
  (void)res;
  return SBD_TPB_OK;
}

}  // namespace

int davidson_run(sbd_tpb_handle *h, const sbd_tpb_params *p, const double *W0,
                 sbd_tpb_result *res) {
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "davidson: tables not built");
  if (p->max_nb < 1 || p->max_nb > kMaxSub)
    return fail(SBD_TPB_ERR_INVALID, "davidson: --block must be in [1, 16]");
  if (p->max_it < 1) return fail(SBD_TPB_ERR_INVALID, "davidson: --iteration must be >= 1");
  const size_t n = h->ndet();
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<double> Wsep;
  double resid = 0.0;
  int nsig = 0, conv = 0;
  if (p->precision == SBD_TPB_MIXED) {
    double h00 = 0.0;
    TPB_CUDA(cudaMemcpy(&h00, h->d_hii, sizeof(double), cudaMemcpyDeviceToHost));
    TPB_CHECK(run_typed<float>(h, p, W0, h00, 2, res, Wsep, &resid, &nsig, &conv));
  } else {
    TPB_CHECK(run_typed<double>(h, p, W0, 0.0, 2, res, Wsep, &resid, &nsig, &conv));
  }
  // final FP64 sigma: energy <W|H|W> (tpb/sbdiag.h:431-469) and the FP64 residual |HW - E W|
  double *dW = nullptr, *dHW = nullptr;
  TPB_CUDA(cudaMalloc(&dW, sizeof(double) * n));
  TPB_CUDA(cudaMalloc(&dHW, sizeof(double) * n));
  int rc = SBD_TPB_OK;
  double E = 0.0, rr = 0.0;
  do {
    if (cudaMemcpyAsync(dW, Wsep.data(), sizeof(double) * n, cudaMemcpyHostToDevice, h->stream) !=
        cudaSuccess) {
      rc = fail(SBD_TPB_ERR_CUDA, "davidson: upload of W failed");
      break;
    }
    if ((rc = sigma_sep<double>(h, dW, dHW, 0)) != SBD_TPB_OK) break;
    const double *wp[1] = {dW};
    if ((rc = multi_dot<double>(h, wp, 1, dHW, n, &E)) != SBD_TPB_OK) break;
    if ((rc = axpby<double>(h, dW, dHW, -E, 1.0, n)) != SBD_TPB_OK) break;
    const double *hp[1] = {dHW};
    if ((rc = multi_dot<double>(h, hp, 1, dHW, n, &rr)) != SBD_TPB_OK) break;
    if (res->ci_vector) {
      if ((rc = reorder_sign_apply_f64(h, dW, dHW)) != SBD_TPB_OK) break;
      if (cudaMemcpyAsync(res->ci_vector, dHW, sizeof(double) * n, cudaMemcpyDeviceToHost,
                          h->stream) != cudaSuccess) {
        rc = fail(SBD_TPB_ERR_CUDA, "davidson: download of W failed");
        break;
      }
    }
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
      rc = fail(SBD_TPB_ERR_CUDA, "davidson: stream failed");
      break;
    }
    if (res->density || res->one_rdm || res->two_rdm) {
      if ((rc = rdm_sep(h, dW, res->one_rdm, res->two_rdm, res->density)) != SBD_TPB_OK) break;
    }
  } while (0);
  cudaFree(dW);
  cudaFree(dHW);
  TPB_CHECK(rc);
  res->energy = E;
  res->residual = (p->precision == SBD_TPB_MIXED) ? std::sqrt(rr) : resid;
  res->iterations = nsig;
  res->converged = conv;
  res->seconds_davidson = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return conv ? SBD_TPB_OK : SBD_TPB_ERR_NOT_CONVERGED;
}

}  // namespace sbdtpb
