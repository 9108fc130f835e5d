// Davidson driver (host side of the loop; kernels in vecops.cu and sigma.cu).
//
// Follows the reference's block Davidson for the lowest root (tpb/davidson.h:667-930,
// basic/davidson_thrust.h:85-373): subspace C_0..C_k with HC_k = H C_k, Rayleigh-Ritz on the
// (k+1)x(k+1) projection, W = sum U_k0 C_k, R = E0 W - H W, convergence when |R| < eps, diagonal
// correction t = R / (E0 - H_ii) with the 1e-12 regularisation, Gram-Schmidt against the subspace,
// restart from W after max_nb steps, and the max_time guard.  The small eigenproblem is solved on
// the device (rr_solve: the projected matrix kept in HBM, cyclic Jacobi on one warp, eigenvalues
// sorted ascending; the reference calls LAPACK dsyev on the host, framework/hp_numeric.h:500-520,
// which also returns them ascending), so a step synchronises with the host once, to read its
// scalars for the convergence test.
//
// Vectors live in HBM in the separated sign convention.  The FP64 path keeps everything in
// double.  The mixed path stores C/HC/W/t in FP32, computes sigma of (H - s) with s = H_00 so the
// FP32 entries carry residual-sized values, keeps all dot products and the Rayleigh-Ritz in FP64,
// and finishes with one FP64 sigma on the converged vector for the reported energy and residual.
// With a learned preconditioner attached, the first four restart cycles alternate between the
// diagonal and the learned correction and later cycles use the learned one only if its cycles
// lowered the residual more than 10% faster per step; inside a learned cycle a step whose residual
// did not drop is followed by a diagonal step.  Both precisions orthogonalise with classical Gram-Schmidt, repeated once
// when the first round cancels more than half of |t|^2 (as stable as the reference's modified
// Gram-Schmidt, tpb/davidson.h:871-879, with one or two fused passes instead of k+1).  The
// converged vector stays in HBM for the final sigma and the RDMs; it crosses to the host only when
// the caller asks for it.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <vector>

#include "mlp.cuh"
#include "tpb_common.cuh"
#include "vecops.cuh"

namespace sbdtpb {
namespace {

// Reduction slots of one Davidson step (device array of kScalarSlots doubles read back together):
// [0, ib+4) residual pass (W.W, r.r, S_k.t, t.t), 20 t.t after the symmetric projection,
// [24, 24+ib+2) first Gram-Schmidt round (t.t, S_k.t), 41 t.t after the second round (0 when the
// device skipped it), [44, 44+ib+1) overlaps S_k . sigma(S_ib), [60, 64) the lowest Ritz values.
constexpr int kSymSlot = 20, kCgsSlot = 24, kCgs2Slot = 41, kOvSlot = 44, kEigSlot = 60;

// alpha <-> beta exchange symmetry (C = C^T): the HF start lies in the symmetric sector and H
// preserves it, so corrections are projected back onto it (and, with symmetry 2, the random start
// is projected onto it first); every vector of such a run is exactly symmetric
bool symmetric_run(const sbd_tpb_handle *h, const sbd_tpb_params *prm, const double *W0) {
  return !W0 && h->astr == h->bstr && (prm->symmetry == 2 || (prm->symmetry == 1 && prm->init == 0));
}

template <typename T>
int run_typed(sbd_tpb_handle *h, const sbd_tpb_params *prm, const double *W0, double shift,
              double *dWout, double *resid_out, int *nsigma_out, int *converged_out, DavRecord *rec,
              sbd_tpb_precond *learned, double *energy_out, int *learned_steps, int *fallback_steps) {
  const size_t n = h->ndet();
  const int nb = prm->max_nb;
  const int max_it = prm->max_it;
  std::vector<DevVec<T>> S(nb), HS(nb);
  DevVec<T> Wv;
  for (int k = 0; k < nb; k++) {
    TPB_CHECK(S[k].get(h, n));
    TPB_CHECK(HS[k].get(h, n));
  }
  TPB_CHECK(Wv.get(h, n));

  // Subspace vectors are stored unnormalised: the basis vector is C_k = f_k S_k and
  // H C_k = f_k sigma(S_k), so normalising costs no pass over the vector.
  std::vector<double> f(nb, 1.0);

  // initial vector (separated convention), staged through dWout
  {
    if (W0) {
      TPB_CUDA(cudaMemcpyAsync(dWout, W0, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
      TPB_CHECK(reorder_sign_apply_f64(h, dWout, dWout));
    } else if (prm->init == 1) {
      // --init 1: the reference's seeded random vector (tpb/davidson.h:138-141); its normalisation
      // is the scale factor f_0 below.  With symmetry 2 it is projected onto the exchange-symmetric
      // sector first (in the separated convention, (x + x^T) / 2).
      TPB_CHECK(random_start_vector(h, dWout, n, prm->seed));
      TPB_CHECK(reorder_sign_apply_f64(h, dWout, dWout));
      if (prm->symmetry == 2 && h->astr == h->bstr) {
        double tt = 0.0;
        TPB_CHECK(symmetrize<double>(h, dWout, &tt));
      }
    } else {
      // --init 0: the first determinant, i.e. the HF string when it is the smallest
      // (tpb/davidson.h:134-137)
      TPB_CUDA(cudaMemsetAsync(dWout, 0, sizeof(double) * n, h->stream));
      const double one = 1.0;
      TPB_CUDA(cudaMemcpyAsync(dWout, &one, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    }
    if (std::is_same<T, double>::value) {
      TPB_CUDA(cudaMemcpyAsync(S[0].p, dWout, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
    } else {
      TPB_CHECK((convert_vec<double, T>(h, dWout, S[0].p, n)));
    }
    double nrm = 0.0;
    const T *cp[1] = {S[0].p};
    TPB_CHECK(multi_dot<T>(h, cp, 1, S[0].p, n, &nrm));
    if (!(nrm > 0.0)) return fail(SBD_TPB_ERR_INVALID, "initial vector is zero");
    f[0] = 1.0 / std::sqrt(nrm);
  }

  std::vector<double> out(kMaxVec + 2), dots(kMaxVec + 2);
  std::vector<double> step_times;
  double norm_R = 0.0, ww = 1.0;
  int nsigma = 0, m_last = 0;
  bool converged = false, stop = false, w_current = false;
  const bool sym = symmetric_run(h, prm, W0);
  ResidualArgs<T> ra;
  double energy = 0.0, prev_norm = 0.0;
  bool prev_learned = false;
  int nlearned = 0, nfallback = 0;
  // Which correction a cycle uses: the first four cycles alternate learned / diagonal, then every
  // cycle uses the one whose cycles lowered log|r| faster per step (ties: diagonal).
  double rate_sum[2] = {0.0, 0.0};  // [0] diagonal, [1] learned
  int rate_cnt[2] = {0, 0};
  int cycle_mode = 0, cycle_steps = 0;
  double cycle_r0 = 0.0;
  std::vector<int> rec_cycle;  // basis indices of the current cycle (recording)
  const auto t_start = std::chrono::steady_clock::now();

  for (int it = 0; it < max_it && !stop; it++) {
    if (it > 0) {
      // restart from the normalised Ritz vector (tpb/davidson.h:918-922): W becomes S_0
      std::swap(S[0].p, Wv.p);
      f[0] = 1.0 / std::sqrt(ww);
      w_current = false;
    }
    if (learned) {
      if (it < 4) {
        // diagonal first: convergence slows as it proceeds, so the learned cycles (later in each
        // pair) are measured at a disadvantage and must really be faster to be kept
        cycle_mode = (it % 2 == 0) ? 0 : 1;
      } else {
        const double rl = rate_cnt[1] ? rate_sum[1] / rate_cnt[1] : 0.0;
        const double rd = rate_cnt[0] ? rate_sum[0] / rate_cnt[0] : 0.0;
        cycle_mode = rl > 1.1 * rd ? 1 : 0;
      }
    }
    cycle_steps = 0;
    for (int ib = 0; ib < nb; ib++) {
      const auto s0 = std::chrono::steady_clock::now();
      std::vector<const T *> cp(ib + 1);
      for (int k = 0; k <= ib; k++) cp[k] = S[k].p;
      // S_ib is exactly exchange-symmetric under the projection (every correction is projected,
      // every other operation is elementwise), so its sigma takes the one-pass symmetric form,
      // whose transpose-add also forms the new column S_k . sigma(S_ib) of the projected matrix
      if (sym) {
        TPB_CHECK(sigma_sep_sym<T>(h, S[ib].p, HS[ib].p, shift, cp.data(), ib + 1, kOvSlot));
      } else {
        TPB_CHECK(sigma_sep_shift<T>(h, S[ib].p, HS[ib].p, 0, shift));
        TPB_CHECK(multi_dot_async<T>(h, cp.data(), ib + 1, HS[ib].p, n, kOvSlot));
      }
      nsigma++;
      // the Rayleigh-Ritz solve stays on the device; the residual kernel reads the Ritz
      // coefficients from there
      ScaleArray fa;
      for (int k = 0; k < kMaxSub; k++) fa.v[k] = k <= ib ? f[k] : 0.0;
      TPB_CHECK(rr_solve(h, ib, fa, kOvSlot, kEigSlot));
      for (int k = 0; k < kMaxVec; k++) {
        ra.C.p[k] = k <= ib ? S[k].p : nullptr;
        ra.HC.p[k] = k <= ib ? HS[k].p : nullptr;
      }
      ra.u_dev = rr_u(h);
      ra.e_dev = rr_e(h);
      ra.shift = shift;
      ra.m = ib + 1;
      // FP32 vectors: the correction's denominator from H_ii - H_00 in FP32 (half the bytes of the
      // FP64 diagonal; its 1e-7 relative rounding is far below what a preconditioner needs)
      ra.hii = h->d_hii;
      ra.hii32 = std::is_same<T, float>::value ? h->d_hii32 : nullptr;
      // W is needed for the restart after the last step of a cycle; otherwise it is formed
      // only once, when the loop stops.  The last step of a cycle needs no correction.
      const bool last = ib == nb - 1;
      ra.W = last ? Wv.p : nullptr;
      T *tnext = last ? nullptr : S[ib + 1].p;
      ra.t = tnext;
      // Fast path: residual, symmetric projection and both Gram-Schmidt rounds (the second one
      // decided on the device) go back to back, and the step's scalars come back with its one
      // synchronisation.  If this step turns out converged, the extra work on t is discarded.
      const bool fast = !rec && !last && !(learned && cycle_mode == 1);
      // a step of a learned cycle in the exchange-symmetric sector: the tile-pair residual now, the
      // learned correction (or not) and the tile-pair Gram-Schmidt after the convergence test
      const bool lsym = sym && !rec && !last && learned && cycle_mode == 1;
      double t0_fast = 0.0, tt_fast = 0.0;
      std::vector<double> coef(ib + 1);
      for (int k = 0; k <= ib; k++) coef[k] = f[k] * f[k];
      if (lsym) {
        TPB_CHECK(residual_sym_async<T>(h, ra, 0));
      } else if (fast && sym) {
        // exchange-symmetric subspace: residual with the projection of t folded in and both
        // Gram-Schmidt rounds in tile-pair form (half the subspace bytes of the general passes)
        TPB_CHECK(residual_sym_async<T>(h, ra, 0));
        TPB_CHECK(cgs_sym_async<T>(h, cp.data(), ib + 1, coef.data(), 2, tnext, 1, kCgsSlot));
        TPB_CHECK(cgs_sym_async<T>(h, cp.data(), ib + 1, coef.data(), kCgsSlot + 1, tnext, 0, kCgs2Slot,
                                   2 + ib + 1, kCgsSlot));
      } else if (sym && last) {
        TPB_CHECK(residual_w_sym_async<T>(h, ra, 0));
      } else {
        TPB_CHECK(residual_step_async<T>(h, ra, n, 0));
        if (fast) {
          if (sym) TPB_CHECK(symmetrize_async<T>(h, tnext, kSymSlot));
          const int t0_slot = sym ? kSymSlot : 2 + ib + 1;
          TPB_CHECK(cgs_update_async<T>(h, cp.data(), ib + 1, coef.data(), 2, tnext, n, 1, kCgsSlot));
          TPB_CHECK(cgs_second_round_async<T>(h, cp.data(), ib + 1, coef.data(), kCgsSlot + 1, tnext, n, t0_slot,
                                              kCgsSlot, kCgs2Slot));
        }
      }
      const double *sc = fetch_scalars(h, kScalarSlots);
      if (!sc) return SBD_TPB_ERR_CUDA;
      for (int k = 0; k < ib + 4; k++) out[k] = sc[k];  // W.W, r.r, S_k.t, t.t
      if (fast) {
        // t.t after the projection: from the symmetrize pass, or (tile-pair residual, or no
        // projection) from the residual pass itself
        t0_fast = sym && !(fast && sym) ? sc[kSymSlot] : sc[2 + ib + 1];
        const double tt1 = sc[kCgsSlot];
        tt_fast = tt1 < 0.5 * t0_fast ? sc[kCgs2Slot] : tt1;
      }
      double eig[4];
      for (int p = 0; p < 4; p++) eig[p] = sc[kEigSlot + p] + shift;
      w_current = last;
      m_last = ib + 1;
      ww = out[0];
      norm_R = std::sqrt(out[1] / ww);
      energy = eig[0];
      bool recording = false;
      if (rec && !last && (int)rec->d.size() < rec->max_steps) {
        // keep d_k, E_k, |r_k| and the step's basis for training pairs (dperp after Gram-Schmidt)
        recording = true;
        if (ib == 0) {
          float *c0 = nullptr;
          TPB_CUDA(cudaMalloc(&c0, sizeof(float) * n));
          rec->owned.push_back(c0);
          TPB_CHECK((convert_vec<T, float>(h, S[0].p, c0, n)));
          rec->vec.push_back(c0);
          rec->scale.push_back(f[0]);
          rec_cycle.assign(1, (int)rec->vec.size() - 1);
        }
        float *dk = nullptr;
        TPB_CUDA(cudaMalloc(&dk, sizeof(float) * n));
        rec->owned.push_back(dk);
        rec->d.push_back(dk);
        TPB_CHECK((convert_vec<T, float>(h, tnext, dk, n)));
        rec->e0.push_back(energy);
        rec->rnorm.push_back(std::sqrt(out[1]));
        rec->basis.push_back(rec_cycle);
      }
      // learned correction: used unless the previous step was a learned one that did not lower
      // the residual, in which case this step falls back to the diagonal correction
      if (ib == 0) cycle_r0 = norm_R;
      cycle_steps++;
      if (learned && (last || norm_R < prm->eps) && cycle_steps > 1 && cycle_r0 > 0.0 && norm_R > 0.0) {
        // the cycle's rate of residual reduction, for the choice of the next cycles' correction
        rate_sum[cycle_mode] += std::log(cycle_r0 / norm_R) / (cycle_steps - 1);
        rate_cnt[cycle_mode]++;
      }
      bool use_learned = false;
      if (learned && cycle_mode == 1 && !last) {
        const bool failed = ib > 0 && prev_learned && !(norm_R < prev_norm);
        use_learned = !failed;
        if (failed) nfallback++;
      }
      prev_learned = use_learned;
      prev_norm = norm_R;
      if (prm->verbose) {
        std::printf(" Davidson iteration %d.%d (tol=%.16g):", it, ib, norm_R);
        for (int p = 0; p < std::min(ib + 1, 4); p++) std::printf(" %.16g", eig[p]);
        std::printf("\n");
        std::fflush(stdout);
      }
      if (norm_R < prm->eps) {
        converged = true;
        stop = true;
        break;
      }
      if (lsym) {
        // t is t_sym (slots 2.. hold S_k.t, 2+ib+1 t.t).  The learned factor depends on the spatial
        // occupation and on H_ii, which is exchange-symmetric only up to rounding, and above the
        // inference budget it corrects a capped subset of entries; so the corrected t is projected
        // again and its overlaps with the subspace recomputed for the Gram-Schmidt rounds
        const int t0_slot = 2 + ib + 1;
        if (use_learned) {
          TPB_CHECK(precond_apply<T>(h, learned, tnext, energy, std::sqrt(out[1]), out[2 + ib + 1]));
          TPB_CHECK(symmetrize_dots<T>(h, tnext, cp.data(), ib + 1, 2));
          nlearned++;
        }
        TPB_CHECK(cgs_sym_async<T>(h, cp.data(), ib + 1, coef.data(), 2, tnext, 1, kCgsSlot));
        TPB_CHECK(cgs_sym_async<T>(h, cp.data(), ib + 1, coef.data(), kCgsSlot + 1, tnext, 0, kCgs2Slot,
                                   t0_slot, kCgsSlot));
        const double *sc2 = fetch_scalars(h, kScalarSlots);
        if (!sc2) return SBD_TPB_ERR_CUDA;
        t0_fast = sc2[t0_slot];
        const double tt1 = sc2[kCgsSlot];
        tt_fast = tt1 < 0.5 * t0_fast ? sc2[kCgs2Slot] : tt1;
      }
      if (use_learned && !lsym)
        TPB_CHECK(precond_apply<T>(h, learned, tnext, energy, std::sqrt(out[1]), out[2 + ib + 1]));
      if (sym && !last && !fast && !lsym) {
        // the S_k are exactly symmetric, so S_k.t is unchanged by the projection; only t.t is
        TPB_CHECK(symmetrize<T>(h, tnext, &out[2 + ib + 1]));
      }
      if (use_learned && !lsym) {
        // overlaps S_k.t and t.t of the learned correction for the Gram-Schmidt below
        std::vector<const T *> xp(ib + 2);
        for (int k = 0; k <= ib; k++) xp[k] = S[k].p;
        xp[ib + 1] = tnext;
        TPB_CHECK(multi_dot<T>(h, xp.data(), ib + 2, tnext, n, dots.data()));
        for (int k = 0; k <= ib + 1; k++) out[2 + k] = dots[k];
        nlearned++;
      }
      if (!last) {
        // classical Gram-Schmidt against C_0..C_ib: t -= sum_k (C_k.t) C_k = sum_k f_k^2 (S_k.t) S_k.
        // A second round runs only when the first cancelled more than half of |t|^2 ("twice is
        // enough": after a round that keeps |t|^2 >= 1/2 of its input, t is orthogonal to the
        // subspace to working precision).
        double t0 = t0_fast, tt = tt_fast;
        std::vector<double> o(ib + 1);
        if (!fast && !lsym) {  // (the fast and learned-cycle symmetric paths ran both rounds on the device)
          t0 = out[2 + ib + 1];
          for (int k = 0; k <= ib; k++) o[k] = f[k] * f[k] * out[2 + k];
          TPB_CHECK(cgs_update<T>(h, cp.data(), ib + 1, o.data(), tnext, n, 1, dots.data()));
          tt = dots[0];
          if (tt < 0.5 * t0) {
            for (int k = 0; k <= ib; k++) o[k] = f[k] * f[k] * dots[1 + k];
            TPB_CHECK(cgs_update<T>(h, cp.data(), ib + 1, o.data(), tnext, n, 0, dots.data()));
            tt = dots[0];
          }
        }
        if (!(tt > 0.0)) {
          // the correction lies in the subspace: nothing left to add
          stop = true;
          break;
        }
        f[ib + 1] = 1.0 / std::sqrt(tt);
        if (recording) {
          float *dp = nullptr;
          TPB_CUDA(cudaMalloc(&dp, sizeof(float) * n));
          rec->owned.push_back(dp);
          TPB_CHECK((convert_vec<T, float>(h, tnext, dp, n)));
          rec->vec.push_back(dp);
          rec->scale.push_back(f[ib + 1]);
          rec_cycle.push_back((int)rec->vec.size() - 1);
        }
      }
      // max_time guard (tpb/davidson.h:887-913): stop when the next step would overrun (after the
      // fast path the stream is already idle)
      if (!fast && !lsym) TPB_CUDA(cudaStreamSynchronize(h->stream));
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
  if (!w_current) {
    // form W = sum_k u_k S_k of the last step (no correction)
    ra.W = Wv.p;
    ra.t = nullptr;
    ra.m = m_last;
    if (sym) {
      TPB_CHECK(residual_w_sym_async<T>(h, ra, 0));
      const double *sc = fetch_scalars(h, kScalarSlots);
      if (!sc) return SBD_TPB_ERR_CUDA;
      ww = sc[0];
    } else {
      TPB_CHECK(residual_step<T>(h, ra, n, out.data()));
      ww = out[0];
    }
  }
  // W normalised and promoted to FP64 into dWout
  if (std::is_same<T, double>::value) {
    TPB_CUDA(cudaMemcpyAsync(dWout, Wv.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
  } else {
    TPB_CHECK((convert_vec<T, double>(h, Wv.p, dWout, n)));
  }
  double nrm = 0.0;
  const double *wp[1] = {dWout};
  TPB_CHECK(multi_dot<double>(h, wp, 1, dWout, n, &nrm));
  TPB_CHECK(scale_vec<double>(h, dWout, 1.0 / std::sqrt(nrm), n));
  *resid_out = norm_R;
  *nsigma_out = nsigma;
  *converged_out = converged ? 1 : 0;
  if (energy_out) *energy_out = energy;
  if (learned_steps) *learned_steps = nlearned;
  if (fallback_steps) *fallback_steps = nfallback;
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
  double resid = 0.0;
  int nsig = 0, conv = 0;
  sbd_tpb_precond *learned = nullptr;
  if (p->preconditioner == SBD_TPB_PRECOND_LEARNED) {
    learned = h->precond;
    if (!learned)
      return fail(SBD_TPB_ERR_STATE, "davidson: learned preconditioner requested but none attached "
                                     "(sbd_tpb_set_preconditioner)");
  } else if (p->preconditioner != SBD_TPB_PRECOND_DIAGONAL) {
    return fail(SBD_TPB_ERR_INVALID, "davidson: unknown preconditioner");
  }
  int nl = 0, nf = 0;
  DevVec<double> dW;
  TPB_CHECK(dW.get(h, n));
  if (p->precision == SBD_TPB_MIXED) {
    double h00 = 0.0;
    TPB_CUDA(cudaMemcpy(&h00, h->d_hii, sizeof(double), cudaMemcpyDeviceToHost));
    TPB_CHECK(run_typed<float>(h, p, W0, h00, dW.p, &resid, &nsig, &conv, nullptr, learned, nullptr, &nl, &nf));
  } else {
    TPB_CHECK(run_typed<double>(h, p, W0, 0.0, dW.p, &resid, &nsig, &conv, nullptr, learned, nullptr, &nl, &nf));
  }
  res->learned_steps = nl;
  res->fallback_steps = nf;
  return solve_finish(h, dW.p, res, t0, nsig, conv, p->precision == SBD_TPB_MIXED ? -1.0 : resid,
                      symmetric_run(h, p, W0));
}

int solve_finish(sbd_tpb_handle *h, double *dW, sbd_tpb_result *res,
                 std::chrono::steady_clock::time_point t0, int nsig, int conv, double resid, bool sym_w) {
  const size_t n = h->ndet();
  // final FP64 sigma: energy <W|H|W> (tpb/sbdiag.h:431-469) and the FP64 residual |HW - E W|;
  // the one-pass symmetric form when W is exactly exchange-symmetric
  DevVec<double> dHW;
  TPB_CHECK(dHW.get(h, n));
  double E = 0.0, rr = 0.0;
  if (sym_w) {
    TPB_CHECK(sigma_sep_sym<double>(h, dW, dHW.p, 0.0));
  } else {
    TPB_CHECK(sigma_sep<double>(h, dW, dHW.p, 0));
  }
  const double *wp[1] = {dW};
  TPB_CHECK(multi_dot<double>(h, wp, 1, dHW.p, n, &E));
  TPB_CHECK(axpby<double>(h, dW, dHW.p, -E, 1.0, n));
  const double *hp[1] = {dHW.p};
  TPB_CHECK(multi_dot<double>(h, hp, 1, dHW.p, n, &rr));
  if (res->ci_vector) {
    TPB_CHECK(reorder_sign_apply_f64(h, dW, dHW.p));
    TPB_CUDA(cudaMemcpyAsync(res->ci_vector, dHW.p, sizeof(double) * n, cudaMemcpyDeviceToHost,
                             h->stream));
  }
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  if (res->density || res->one_rdm || res->two_rdm) {
    if (res->one_rdm || res->two_rdm) pool_clear(h);  // the 2-RDM passes need their own N-vectors
    TPB_CHECK(rdm_sep(h, dW, res->one_rdm, res->two_rdm, res->density));
  }
  // carry-over strings of the final vector (tpb/sbdiag.h:690-736); a short caller buffer is
  // reported after the rest of the result is filled
  int co_rc = SBD_TPB_OK;
  if (res->carryover && res->carryover->type != SBD_TPB_CARRYOVER_NONE) {
    co_rc = carryover_device(h, dW, res->carryover);
    if (co_rc != SBD_TPB_OK && co_rc != SBD_TPB_ERR_CAPACITY) return co_rc;
  }
  res->energy = E;
  res->residual = resid < 0.0 ? std::sqrt(rr) : resid;
  res->iterations = nsig;
  res->converged = conv;
  res->seconds_davidson = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (co_rc != SBD_TPB_OK) return co_rc;
  return conv ? SBD_TPB_OK : SBD_TPB_ERR_NOT_CONVERGED;
}

int pool_get(sbd_tpb_handle *h, size_t bytes, void **out) {
  *out = nullptr;
  size_t best = h->vec_pool.size();
  for (size_t i = 0; i < h->vec_pool.size(); i++) {
    const size_t b = h->vec_pool[i].second;
    if (b >= bytes && b <= 2 * bytes && (best == h->vec_pool.size() || b < h->vec_pool[best].second)) best = i;
  }
  if (best < h->vec_pool.size()) {
    *out = h->vec_pool[best].first;
    h->vec_pool.erase(h->vec_pool.begin() + best);
    return SBD_TPB_OK;
  }
  if (cudaMalloc(out, bytes) == cudaSuccess) return SBD_TPB_OK;
  cudaGetLastError();
  pool_clear(h);
  TPB_CUDA(cudaMalloc(out, bytes));
  return SBD_TPB_OK;
}

void pool_put(sbd_tpb_handle *h, void *p, size_t bytes) {
  if (p) h->vec_pool.emplace_back(p, bytes);
}

void pool_clear(sbd_tpb_handle *h) {
  for (auto &b : h->vec_pool) cudaFree(b.first);
  h->vec_pool.clear();
}

int davidson_record(sbd_tpb_handle *h, const sbd_tpb_params *p, DavRecord *rec, double *Psi,
                    double *energy, sbd_tpb_precond *learned) {
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "davidson: tables not built");
  if (p->max_nb < 2 || p->max_nb > kMaxSub)
    return fail(SBD_TPB_ERR_INVALID, "davidson: --block must be in [2, 16] for recording");
  if (p->max_it < 1) return fail(SBD_TPB_ERR_INVALID, "davidson: --iteration must be >= 1");
  double resid = 0.0;
  int nsig = 0, conv = 0;
  return run_typed<double>(h, p, nullptr, 0.0, Psi, &resid, &nsig, &conv, rec, learned, energy, nullptr,
                           nullptr);
}

}  // namespace sbdtpb
