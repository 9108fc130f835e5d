// Integrals, per-string data, the diagonal and the sigma programs.
//
// Integral setup follows SetupIntegrals (basic/makeintegrals.h:123-174): the packed 8-fold store
// (basic/integrals.h:64-107) is unpacked once into a dense (pq|rs) table so kernels index it
// directly.  The diagonal uses the separable form of ZeroExcite (basic/determinants.h:434-457):
//   H_ii = I0 + E(Ia) + E(Ib) + sum_{p in Ia, q in Ib} (pp|qq),
//   E(I) = sum_{p in I} h_pp + sum_{p<q in I} [(pp|qq) - (pq|qp)].
// The sigma programs turn each excitation-table entry into its separated-convention matrix
// element (see tpb_common.cuh): for a same-spin single cr -> an on bra string I,
//   sgn * [h_{an,cr} + sum_{j in I} ((an cr|jj) - (an j|j cr))]   (+ the other-spin Coulomb term
//   sgn * sum_{k in other} (an cr|kk), added inside the sigma kernels),
// sgn = (-1)^{|I ∩ (min(cr,an), max(cr,an))|}, as OneExcite (determinants.h:459-481) restricted to
// one spin; for a double, the TwoExcite sign rule (determinants.h:483-501) on the one-spin string
// and value (an0 cr0|an1 cr1) - (an0 cr1|an1 cr0).
#include <algorithm>
#include <cmath>

#include "tpb_common.cuh"

namespace sbdtpb {
namespace {

inline size_t packed_index(int I, int J, int K, int L_) {
  const int mij = std::max(I, J), nij = std::min(I, J);
  const int mkl = std::max(K, L_), nkl = std::min(K, L_);
  const size_t ij = (size_t)mij * (mij + 1) / 2 + nij;
  const size_t kl = (size_t)mkl * (mkl + 1) / 2 + nkl;
  const size_t a = std::max(ij, kl), b = std::min(ij, kl);
  return a * (a + 1) / 2 + b;
}

template <typename T>
void free_dev(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

__global__ void diag_kernel(const uint64_t *__restrict__ astr, const uint64_t *__restrict__ bstr,
                            const double *__restrict__ Ea, const double *__restrict__ Eb,
                            const double *__restrict__ uJ, int L, uint32_t na, uint32_t nb,
                            double I0, double *__restrict__ hii) {
  const size_t n = (size_t)na * nb;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t ia = (uint32_t)(i / nb), ib = (uint32_t)(i - (size_t)ia * nb);
    uint64_t b = bstr[ib];
    const double *u = uJ + (size_t)ia * L;
    double x = 0.0;
    while (b) {
      const int q = lowest_bit(b);
      x += u[q];
      b &= b - 1;
    }
    hii[i] = I0 + Ea[ia] + Eb[ib] + x;
  }
}

__global__ void diag32_kernel(const double *__restrict__ hii, size_t n, double h00,
                              float *__restrict__ hii32) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    hii32[i] = (float)(hii[i] - h00);
}

// Values of the sigma program, aligned entry by entry with the excitation tables.
__global__ void single_values_kernel(const uint64_t *__restrict__ str, uint32_t n, int L,
                                     const uint32_t *__restrict__ off,
                                     const uint32_t *__restrict__ lab,
                                     const double *__restrict__ eri, const double *__restrict__ h1,
                                     double *__restrict__ val, float *__restrict__ valf,
                                     int32_t *__restrict__ pairsgn) {
  const uint32_t row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const uint64_t I = str[row];
  const size_t L2 = (size_t)L * L;
  for (uint32_t e = off[row] + lane; e < off[row + 1]; e += 32) {
    const uint32_t lb = lab[e];
    const int cr = lb & 0xff, an = (lb >> 8) & 0xff;
    const int lo = min(cr, an), hi = max(cr, an);
    const double sgn = (__popcll(I & open_mask(lo, hi)) & 1) ? -1.0 : 1.0;
    double v = h1[(size_t)an * L + cr];
    uint64_t occ = I;
    while (occ) {
      const int j = lowest_bit(occ);
      v += eri[((size_t)an * L + cr) * L2 + (size_t)j * L + j] -
           eri[((size_t)an * L + j) * L2 + (size_t)j * L + cr];
      occ &= occ - 1;
    }
    val[e] = sgn * v;
    valf[e] = (float)(sgn * v);
    pairsgn[e] = (sgn < 0 ? -1 : 1) * (an * L + cr + 1);
  }
}

__global__ void double_values_kernel(const uint64_t *__restrict__ str, uint32_t n, int L,
                                     const uint32_t *__restrict__ off,
                                     const uint32_t *__restrict__ lab,
                                     const double *__restrict__ eri, double *__restrict__ val,
                                     float *__restrict__ valf) {
  const uint32_t row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const uint64_t I = str[row];
  const size_t L2 = (size_t)L * L;
  for (uint32_t e = off[row] + lane; e < off[row + 1]; e += 32) {
    const uint32_t lb = lab[e];
    const int I0 = lb & 0xff, J0 = (lb >> 8) & 0xff, A0 = (lb >> 16) & 0xff, B0 = (lb >> 24) & 0xff;
    int par = __popcll(I & open_mask(min(I0, A0), max(I0, A0))) +
              __popcll(I & open_mask(min(J0, B0), max(J0, B0)));
    if (A0 > J0 || B0 < I0) par += 1;
    const double sgn = (par & 1) ? -1.0 : 1.0;
    const double v = eri[((size_t)A0 * L + I0) * L2 + (size_t)B0 * L + J0] -
                     eri[((size_t)A0 * L + J0) * L2 + (size_t)B0 * L + I0];
    val[e] = sgn * v;
    valf[e] = (float)(sgn * v);
  }
}

void free_prog(SigmaProg &p) {
  free_dev(p.jtab);
  free_dev(p.pmap);
  free_dev(p.s_val);
  free_dev(p.s_valf);
  free_dev(p.s_pair);
  free_dev(p.d_val);
  free_dev(p.d_valf);
  p = SigmaProg();
}

int build_prog(sbd_tpb_handle *h, const uint64_t *d_str, uint32_t n, const ExTable &ts,
               const ExTable &td, const double *h1dev, SigmaProg &p) {
  free_prog(p);
  const size_t ms = ts.nnz ? ts.nnz : 1, md = td.nnz ? td.nnz : 1;
  TPB_CUDA(cudaMalloc(&p.s_val, sizeof(double) * ms));
  TPB_CUDA(cudaMalloc(&p.s_valf, sizeof(float) * ms));
  TPB_CUDA(cudaMalloc(&p.s_pair, sizeof(int32_t) * ms));
  TPB_CUDA(cudaMalloc(&p.d_val, sizeof(double) * md));
  TPB_CUDA(cudaMalloc(&p.d_valf, sizeof(float) * md));
  const unsigned grid = (n + 7) / 8;
  single_values_kernel<<<grid, 256, 0, h->stream>>>(d_str, n, h->L, ts.off, ts.lab, h->d_eri, h1dev,
                                                   p.s_val, p.s_valf, p.s_pair);
  TPB_LAUNCHED(h);
  double_values_kernel<<<grid, 256, 0, h->stream>>>(d_str, n, h->L, td.off, td.lab, h->d_eri,
                                                   p.d_val, p.d_valf);
  TPB_LAUNCHED(h);
  p.s = &ts;
  p.d = &td;
  return SBD_TPB_OK;
}

// J[i][c] = sum over the orbitals k of col_str[c], ascending, of vd[pair(i)][k]
__global__ void coulomb_table_kernel(const uint64_t *__restrict__ col_str, size_t ncols,
                                     const int32_t *__restrict__ pairs, uint32_t npair, int L,
                                     const double *__restrict__ vd, double *__restrict__ J) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)npair * ncols) return;
  const uint32_t i = (uint32_t)(t / ncols);
  const size_t c = t - (size_t)i * ncols;
  const double *vrow = vd + (size_t)pairs[i] * L;
  double o = 0.0;
  for (uint64_t m = col_str[c]; m; m &= m - 1) o += __ldg(&vrow[lowest_bit(m)]);
  J[t] = o;
}

}  // namespace

int build_coulomb_table(sbd_tpb_handle *h, SigmaProg &p, const uint64_t *col_str, size_t ncols) {
  if (p.jtab_tried || !p.s || p.s->nnz == 0) return SBD_TPB_OK;
  p.jtab_tried = true;
  const int L2 = h->L * h->L;
  std::vector<int32_t> sp(p.s->nnz), pmap(L2, -1), pairs;
  TPB_CUDA(cudaMemcpy(sp.data(), p.s_pair, sizeof(int32_t) * sp.size(), cudaMemcpyDeviceToHost));
  for (int32_t ps : sp) {
    const int pr = (ps > 0 ? ps : -ps) - 1;
    if (pmap[pr] < 0) {
      pmap[pr] = (int32_t)pairs.size();
      pairs.push_back(pr);
    }
  }
  // the table is an optimisation: above 1/16 of the free device memory (or if it cannot be
  // allocated) the singles keep the loop over the column string's orbitals
  const size_t bytes = sizeof(double) * pairs.size() * ncols;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || bytes > free_b / 16) {
    cudaGetLastError();
    return SBD_TPB_OK;
  }
  if (cudaMalloc(&p.jtab, bytes) != cudaSuccess) {
    cudaGetLastError();
    p.jtab = nullptr;
    return SBD_TPB_OK;
  }
  int32_t *d_pairs = nullptr;
  TPB_CUDA(cudaMalloc(&p.pmap, sizeof(int32_t) * L2));
  TPB_CUDA(cudaMalloc(&d_pairs, sizeof(int32_t) * pairs.size()));
  TPB_CUDA(cudaMemcpy(p.pmap, pmap.data(), sizeof(int32_t) * L2, cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(d_pairs, pairs.data(), sizeof(int32_t) * pairs.size(), cudaMemcpyHostToDevice));
  p.npair = (uint32_t)pairs.size();
  const size_t tot = pairs.size() * ncols;
  coulomb_table_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, h->stream>>>(col_str, ncols, d_pairs, p.npair,
                                                                             h->L, h->d_vd, p.jtab);
  TPB_LAUNCHED(h);
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  cudaFree(d_pairs);
  return SBD_TPB_OK;
}

void free_device_problem(sbd_tpb_handle *h) {
  free_dev(h->d_eri);
  free_dev(h->d_vd);
  free_dev(h->d_J);
  free_dev(h->d_astr);
  free_dev(h->d_bstr);
  free_dev(h->d_apar);
  free_dev(h->d_Ea);
  free_dev(h->d_Eb);
  free_dev(h->d_uJ);
  free_dev(h->d_hii);
  free_dev(h->d_hii32);
  for (ExTable *t : {&h->ta_s, &h->ta_d, &h->tb_s, &h->tb_d}) {
    free_dev(t->off);
    free_dev(t->ket);
    free_dev(t->lab);
    *t = ExTable();
  }
  free_prog(h->pa);
  free_prog(h->pb);
  free_dev(h->ab.pq_of_label);
  free_dev(h->ab.rs_of_label);
  free_dev(h->ab.a_label);
  free_dev(h->ab.b_label);
  free_dev(h->ab.V);
  free_dev(h->ab.Vf);
  free_dev(h->ab.Vhi);
  free_dev(h->ab.Vlo);
  free_dev(h->ab.err);
  h->ab = ABDense();
  pool_clear(h);
  free_dev(h->d_partials);
  h->partials_cap = 0;
  free_dev(h->d_scal);
  if (h->h_scal) cudaFreeHost(h->h_scal);
  h->h_scal = nullptr;
  free_dev(h->d_tmp64);
  free_dev(h->d_tmp64b);
  free_dev(h->d_tmp32);
  free_dev(h->d_tmp32b);
  if (h->d_ab_work) cudaFree(h->d_ab_work);
  h->d_ab_work = nullptr;
  h->ab_work_bytes = 0;
  if (h->d_ct) cudaFree(h->d_ct);
  h->d_ct = nullptr;
  h->ct_bytes = 0;
  free_dev(h->d_mlp_idx);
  free_dev(h->d_kx_a);
  free_dev(h->d_kx_b);
  free_dev(h->d_occw_a);
  free_dev(h->d_occw_b);
  free_dev(h->d_ab_rows);
  free_dev(h->d_ab_colp);
  free_dev(h->d_ab_bsp);
  free_dev(h->d_ab_kets);
  h->ab_nkets = 0;
  h->ab_nrows = h->ab_ncols = h->ab_max_k = 0;
  h->ab_nchunks = 1;
  h->ab_chunk = 0;
  h->ab_dense = false;
  h->blk_for = nullptr;
  h->have_tables = false;
}

int upload_hamiltonian(sbd_tpb_handle *h) {
  const int L = h->L;
  const size_t L2 = (size_t)L * L;
  std::vector<double> eri(L2 * L2), vd(L2 * L), J(L2), h1full(L2);
  for (int p = 0; p < L; p++)
    for (int q = 0; q < L; q++)
      for (int r = 0; r < L; r++)
        for (int s = 0; s < L; s++)
          eri[((size_t)p * L + q) * L2 + (size_t)r * L + s] = h->eri_packed[packed_index(p, q, r, s)];
  for (size_t pq = 0; pq < L2; pq++)
    for (int k = 0; k < L; k++) vd[pq * L + k] = eri[pq * L2 + (size_t)k * L + k];
  for (int p = 0; p < L; p++)
    for (int q = 0; q < L; q++) J[(size_t)p * L + q] = eri[((size_t)p * L + p) * L2 + (size_t)q * L + q];
  free_dev(h->d_eri);
  free_dev(h->d_vd);
  free_dev(h->d_J);
  TPB_CUDA(cudaMalloc(&h->d_eri, sizeof(double) * eri.size()));
  TPB_CUDA(cudaMalloc(&h->d_vd, sizeof(double) * vd.size()));
  TPB_CUDA(cudaMalloc(&h->d_J, sizeof(double) * (J.size() + L2)));
  TPB_CUDA(cudaMemcpy(h->d_eri, eri.data(), sizeof(double) * eri.size(), cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(h->d_vd, vd.data(), sizeof(double) * vd.size(), cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(h->d_J, J.data(), sizeof(double) * J.size(), cudaMemcpyHostToDevice));
  // the one-electron matrix rides behind J
  TPB_CUDA(cudaMemcpy(h->d_J + L2, h->h1.data(), sizeof(double) * L2, cudaMemcpyHostToDevice));
  return SBD_TPB_OK;
}

static void string_energies(const sbd_tpb_handle *h, const std::vector<uint64_t> &s,
                            std::vector<double> &E) {
  const int L = h->L;
  E.resize(s.size());
  for (size_t i = 0; i < s.size(); i++) {
    double e = 0.0;
    for (int p = 0; p < L; p++) {
      if (!((s[i] >> p) & 1)) continue;
      e += h->h1[(size_t)p * L + p];
      for (int q = p + 1; q < L; q++) {
        if (!((s[i] >> q) & 1)) continue;
        e += h->eri_packed[packed_index(p, p, q, q)] - h->eri_packed[packed_index(p, q, q, p)];
      }
    }
    E[i] = e;
  }
}

int build_string_data(sbd_tpb_handle *h) {
  const size_t na = h->astr.size(), nb = h->bstr.size();
  const int L = h->L;
  for (uint64_t **p : {&h->d_astr, &h->d_bstr, &h->d_apar}) free_dev(*p);
  for (double **p : {&h->d_Ea, &h->d_Eb, &h->d_uJ}) free_dev(*p);
  std::vector<double> Ea, Eb, uJ(na * L, 0.0);
  std::vector<uint64_t> apar(na);
  string_energies(h, h->astr, Ea);
  string_energies(h, h->bstr, Eb);
  for (size_t i = 0; i < na; i++) {
    apar[i] = above_parity_mask(h->astr[i]);
    for (int p = 0; p < L; p++) {
      if (!((h->astr[i] >> p) & 1)) continue;
      for (int q = 0; q < L; q++) uJ[i * L + q] += h->eri_packed[packed_index(p, p, q, q)];
    }
  }
  TPB_CUDA(cudaMalloc(&h->d_astr, sizeof(uint64_t) * na));
  TPB_CUDA(cudaMalloc(&h->d_bstr, sizeof(uint64_t) * nb));
  TPB_CUDA(cudaMalloc(&h->d_apar, sizeof(uint64_t) * na));
  TPB_CUDA(cudaMalloc(&h->d_Ea, sizeof(double) * na));
  TPB_CUDA(cudaMalloc(&h->d_Eb, sizeof(double) * nb));
  TPB_CUDA(cudaMalloc(&h->d_uJ, sizeof(double) * na * L));
  TPB_CUDA(cudaMemcpy(h->d_astr, h->astr.data(), sizeof(uint64_t) * na, cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(h->d_bstr, h->bstr.data(), sizeof(uint64_t) * nb, cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(h->d_apar, apar.data(), sizeof(uint64_t) * na, cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(h->d_Ea, Ea.data(), sizeof(double) * na, cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(h->d_Eb, Eb.data(), sizeof(double) * nb, cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(h->d_uJ, uJ.data(), sizeof(double) * na * L, cudaMemcpyHostToDevice));
  return SBD_TPB_OK;
}

int compute_diagonal(sbd_tpb_handle *h) {
  const size_t n = h->ndet();
  free_dev(h->d_hii);
  TPB_CUDA(cudaMalloc(&h->d_hii, sizeof(double) * n));
  const int grid = h->num_sms * 8;
  diag_kernel<<<grid, 256, 0, h->stream>>>(h->d_astr, h->d_bstr, h->d_Ea, h->d_Eb, h->d_uJ, h->L,
                                          (uint32_t)h->astr.size(), (uint32_t)h->bstr.size(),
                                          h->I0, h->d_hii);
  TPB_LAUNCHED(h);
  TPB_CUDA(cudaMemcpyAsync(&h->h00, h->d_hii, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  free_dev(h->d_hii32);
  TPB_CUDA(cudaMalloc(&h->d_hii32, sizeof(float) * n));
  diag32_kernel<<<grid, 256, 0, h->stream>>>(h->d_hii, n, h->h00, h->d_hii32);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

int build_sigma_programs(sbd_tpb_handle *h) {
  // the one-electron matrix is stored on the device right behind J
  const double *h1dev = h->d_J + (size_t)h->L * h->L;
  TPB_CHECK(build_prog(h, h->d_astr, (uint32_t)h->astr.size(), h->ta_s, h->ta_d, h1dev, h->pa));
  TPB_CHECK(build_prog(h, h->d_bstr, (uint32_t)h->bstr.size(), h->tb_s, h->tb_d, h1dev, h->pb));
  return SBD_TPB_OK;
}

}  // namespace sbdtpb
