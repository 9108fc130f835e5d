// sigma = H*C on the GPU (separated sign convention; see tpb_common.cuh).
//
// Replaces MultTPBThrust::run (tpb/mult_thrust.h:1172-1582) and sbd::mult (tpb/mult.h:625-881).
// Where the reference launches one thread per (connection, determinant) and adds into sigma with
// FP64 atomics, every sigma element here has exactly one owner, so results are deterministic:
//
//   row kernel    one CTA per alpha row Ia.  C[Ia, :] is staged in shared memory; for each
//                 beta column Ib the owner thread adds the diagonal, the beta singles/doubles
//                 (gathered from the staged row) and the alpha-single x beta-single terms
//                 (sa * sb * (pq|rs) * C[Ja, Jb]); it writes sigma[Ia, Ib] once.
//   slab kernel   one CTA per (alpha row Ia, 512-column slab).  Adds the alpha singles/doubles
//                 sum_Ja H_a(Ia, Ja) C[Ja, slab].  Blocks are ordered slab-major so the CTAs in
//                 flight share one column slab of C, which stays resident in L2 while every row
//                 gathers from it.
//
// The alpha-beta term of FCI-like problems (dense singles) goes through the gather -> dense
// (pq|rs) contraction -> scatter path in ab_dense.cu instead of the direct loop.
#include <algorithm>

#include "tpb_common.cuh"

namespace sbdtpb {
namespace {

constexpr int kRowThreads = 512;
constexpr int kSlabThreads = 256;

template <typename T>
__device__ __forceinline__ T val_of(const double *v, const float *vf, uint32_t e);
template <>
__device__ __forceinline__ double val_of<double>(const double *v, const float *, uint32_t e) {
  return __ldg(&v[e]);
}
template <>
__device__ __forceinline__ float val_of<float>(const double *, const float *vf, uint32_t e) {
  return __ldg(&vf[e]);
}

struct RowArgs {
  const uint64_t *astr, *bstr;
  const uint32_t *bs_off, *bs_ket;  // beta singles
  const double *bs_val;
  const float *bs_valf;
  const int32_t *bs_pair;
  const uint32_t *bd_off, *bd_ket;  // beta doubles
  const double *bd_val;
  const float *bd_valf;
  const uint32_t *as_off, *as_ket;  // alpha singles (alpha-beta term)
  const int32_t *as_pair;
  const double *hii, *vd, *eri;
  int L;
  uint32_t na, nb;
  double shift;
  int accumulate;
  int do_ab;   // 1: alpha-single x beta-single terms by direct gather here
  int max_as;  // longest alpha-singles row (shared-memory staging)
};

// Row kernel: a CTA owns R consecutive alpha rows; G lanes cooperate on one beta column Ib,
// reading its table entries coalesced and gathering C[Ia, Jb] from the rows staged in shared
// memory; the G partial sums meet in a shuffle reduction and one lane writes sigma[Ia, Ib].
// Shared memory: [crow: R x nb T][uA: R x L^2 double][asng: R x max_as int2][nas: R int]
template <typename T, int G, int R, bool kSmemRow>
__global__ void __launch_bounds__(kRowThreads)
    sigma_row_kernel(RowArgs a, const T *__restrict__ C, T *__restrict__ sigma) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t nb = a.nb;
  const int L = a.L;
  const int L2 = L * L;
  const uint32_t row0 = blockIdx.x * R;
  const size_t row_bytes = ((size_t)nb * sizeof(T) + 15) & ~(size_t)15;
  T *crow = reinterpret_cast<T *>(smem);
  size_t off = kSmemRow ? R * row_bytes : 0;
  double *uA = reinterpret_cast<double *>(smem + off);
  off += (size_t)R * L2 * sizeof(double);
  int2 *asng = reinterpret_cast<int2 *>(smem + off);
  off += (size_t)R * a.max_as * sizeof(int2);
  int *nas = reinterpret_cast<int *>(smem + off);

  int nrows = 0;
#pragma unroll
  for (int r = 0; r < R; r++)
    if (row0 + r < a.na) nrows = r + 1;
  if (threadIdx.x < R) nas[threadIdx.x] = 0;
#pragma unroll
  for (int r = 0; r < R; r++) {
    if (r >= nrows) break;
    const uint32_t ia = row0 + r;
    if (kSmemRow) {
      const T *src = C + (size_t)ia * nb;
      T *dst = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(crow) + r * row_bytes);
      for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) dst[j] = src[j];
    }
    // other-spin Coulomb term of beta singles: uA[r][pair] = sum_{k in Ia} (pair|kk)
    const uint64_t Ia = a.astr[ia];
    for (int pq = threadIdx.x; pq < L2; pq += blockDim.x) {
      double sacc = 0.0;
      uint64_t occ = Ia;
      while (occ) {
        sacc += a.vd[(size_t)pq * L + lowest_bit(occ)];
        occ &= occ - 1;
      }
      uA[r * L2 + pq] = sacc;
    }
    if (a.do_ab) {
      const uint32_t e0 = a.as_off[ia], e1 = a.as_off[ia + 1];
      for (uint32_t e = e0 + threadIdx.x; e < e1; e += blockDim.x)
        asng[r * a.max_as + (e - e0)] = make_int2((int)a.as_ket[e], a.as_pair[e]);
      if (threadIdx.x == 0) nas[r] = (int)(e1 - e0);
    }
  }
  __syncthreads();

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int sub = lane % G, grp = lane / G;
  constexpr int GPW = 32 / G;
  for (uint32_t base = (uint32_t)warp * GPW; base < nb; base += (uint32_t)nwarps * GPW) {
    const uint32_t ib = base + grp;
    const bool valid = ib < nb;
    T acc[R];
#pragma unroll
    for (int r = 0; r < R; r++) acc[r] = T(0);
    if (valid) {
      const uint32_t d0 = __ldg(&a.bd_off[ib]), d1 = __ldg(&a.bd_off[ib + 1]);
      for (uint32_t e = d0 + sub; e < d1; e += G) {
        const uint32_t jb = __ldg(&a.bd_ket[e]);
        const T v = val_of<T>(a.bd_val, a.bd_valf, e);
#pragma unroll
        for (int r = 0; r < R; r++) {
          const T c = kSmemRow ? reinterpret_cast<const T *>(reinterpret_cast<const unsigned char *>(crow) + r * row_bytes)[jb]
                               : C[(size_t)(row0 + r) * nb + jb];
          if (r < nrows) acc[r] += v * c;
        }
      }
      const uint32_t s0 = __ldg(&a.bs_off[ib]), s1 = __ldg(&a.bs_off[ib + 1]);
      for (uint32_t e = s0 + sub; e < s1; e += G) {
        const uint32_t jb = __ldg(&a.bs_ket[e]);
        const double v = (double)val_of<T>(a.bs_val, a.bs_valf, e);
        const int32_t ps = __ldg(&a.bs_pair[e]);
        const int pr = (ps > 0 ? ps : -ps) - 1;
        const double sb = ps > 0 ? 1.0 : -1.0;
#pragma unroll
        for (int r = 0; r < R; r++) {
          if (r >= nrows) break;
          const T c = kSmemRow ? reinterpret_cast<const T *>(reinterpret_cast<const unsigned char *>(crow) + r * row_bytes)[jb]
                               : C[(size_t)(row0 + r) * nb + jb];
          double x = (v + sb * uA[r * L2 + pr]) * (double)c;
          // alpha single (Ja, pq, sa) x this beta single (Jb, rs, sb): sa sb (pq|rs) C[Ja, Jb]
          const int n_as = nas[r];
          for (int k = 0; k < n_as; k++) {
            const int2 as = asng[r * a.max_as + k];
            const int pq = (as.y > 0 ? as.y : -as.y) - 1;
            const double g = __ldg(&a.eri[(size_t)pq * L2 + pr]);
            const double cj = (double)C[(size_t)as.x * nb + jb];
            x += sb * (as.y > 0 ? g : -g) * cj;
          }
          acc[r] += (T)x;
        }
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1)
#pragma unroll
      for (int r = 0; r < R; r++) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
    if (valid && sub == 0) {
#pragma unroll
      for (int r = 0; r < R; r++) {
        if (r >= nrows) break;
        const size_t bra = (size_t)(row0 + r) * nb + ib;
        const T cself = kSmemRow ? reinterpret_cast<const T *>(reinterpret_cast<const unsigned char *>(crow) + r * row_bytes)[ib]
                                 : C[bra];
        double x = (double)acc[r] + (a.hii[bra] - a.shift) * (double)cself;
        if (a.accumulate) x += (double)sigma[bra];
        sigma[bra] = (T)x;
      }
    }
  }
}

struct SlabArgs {
  const uint64_t *bstr;
  const uint32_t *as_off, *as_ket;
  const double *as_val;
  const float *as_valf;
  const int32_t *as_pair;
  const uint32_t *ad_off, *ad_ket;
  const double *ad_val;
  const float *ad_valf;
  const double *vd;
  int L;
  uint32_t na, nb;
};

// Alpha slab kernel: CTA = (alpha row Ia, column slab of kSlabThreads*CPT columns), blocks
// ordered slab-major so the CTAs in flight gather from one L2-resident slab of C.
template <typename T, int CPT>
__global__ void __launch_bounds__(kSlabThreads)
    sigma_alpha_slab_kernel(SlabArgs a, const T *__restrict__ C, T *__restrict__ sigma) {
  const uint32_t ia = blockIdx.x % a.na;
  const uint32_t slab = blockIdx.x / a.na;
  const uint32_t nb = a.nb;
  const int L = a.L;
  constexpr uint32_t W = kSlabThreads * CPT;
  uint32_t col[CPT];
  bool ok[CPT];
  T acc[CPT];
#pragma unroll
  for (int k = 0; k < CPT; k++) {
    col[k] = slab * W + k * kSlabThreads + threadIdx.x;
    ok[k] = col[k] < nb;
    acc[k] = T(0);
  }
  const uint32_t d0 = __ldg(&a.ad_off[ia]), d1 = __ldg(&a.ad_off[ia + 1]);
#pragma unroll 4
  for (uint32_t e = d0; e < d1; e++) {
    const uint32_t ja = __ldg(&a.ad_ket[e]);
    const T v = val_of<T>(a.ad_val, a.ad_valf, e);
    const T *crow = C + (size_t)ja * nb;
#pragma unroll
    for (int k = 0; k < CPT; k++)
      if (ok[k]) acc[k] += v * __ldg(&crow[col[k]]);
  }
  const uint32_t s0 = __ldg(&a.as_off[ia]), s1 = __ldg(&a.as_off[ia + 1]);
  if (s1 > s0) {
    uint64_t bcol[CPT];
#pragma unroll
    for (int k = 0; k < CPT; k++) bcol[k] = ok[k] ? __ldg(&a.bstr[col[k]]) : 0ull;
    for (uint32_t e = s0; e < s1; e++) {
      const uint32_t ja = __ldg(&a.as_ket[e]);
      const double v = (double)val_of<T>(a.as_val, a.as_valf, e);
      const int32_t ps = __ldg(&a.as_pair[e]);
      const int pr = (ps > 0 ? ps : -ps) - 1;
      const double *vrow = a.vd + (size_t)pr * L;
      const T *crow = C + (size_t)ja * nb;
#pragma unroll
      for (int k = 0; k < CPT; k++) {
        if (!ok[k]) continue;
        uint64_t occ = bcol[k];
        double o = 0.0;
        while (occ) {
          o += __ldg(&vrow[lowest_bit(occ)]);
          occ &= occ - 1;
        }
        acc[k] += (T)((v + (ps > 0 ? o : -o)) * (double)__ldg(&crow[col[k]]));
      }
    }
  }
  T *srow = sigma + (size_t)ia * nb;
#pragma unroll
  for (int k = 0; k < CPT; k++)
    if (ok[k]) srow[col[k]] += acc[k];
}

__global__ void reorder_sign_kernel_f64(const uint64_t *__restrict__ apar,
                                        const uint64_t *__restrict__ bstr, uint32_t nb, size_t n,
                                        const double *__restrict__ x, double *__restrict__ y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t ia = i / nb, ib = i - ia * nb;
    const double v = x[i];
    y[i] = (__popcll(apar[ia] & bstr[ib]) & 1) ? -v : v;
  }
}

__global__ void reorder_sign_kernel_f32(const uint64_t *__restrict__ apar,
                                        const uint64_t *__restrict__ bstr, uint32_t nb, size_t n,
                                        const float *__restrict__ x, float *__restrict__ y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t ia = i / nb, ib = i - ia * nb;
    const float v = x[i];
    y[i] = (__popcll(apar[ia] & bstr[ib]) & 1) ? -v : v;
  }
}

}  // namespace

int reorder_sign_apply_f64(sbd_tpb_handle *h, const double *x, double *y) {
  reorder_sign_kernel_f64<<<h->num_sms * 8, 256, 0, h->stream>>>(
      h->d_apar, h->d_bstr, (uint32_t)h->bstr.size(), h->ndet(), x, y);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

int reorder_sign_apply_f32(sbd_tpb_handle *h, const float *x, float *y) {
  reorder_sign_kernel_f32<<<h->num_sms * 8, 256, 0, h->stream>>>(
      h->d_apar, h->d_bstr, (uint32_t)h->bstr.size(), h->ndet(), x, y);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

template <typename T, int G, int R, bool kSmemRow>
int launch_row(sbd_tpb_handle *h, const RowArgs &ra, const T *C, T *sigma, size_t smem) {
  auto kern = sigma_row_kernel<T, G, R, kSmemRow>;
  TPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const unsigned grid = (unsigned)((ra.na + R - 1) / R);
  kern<<<grid, kRowThreads, smem, h->stream>>>(ra, C, sigma);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

template <typename T, int G>
int launch_row_r(sbd_tpb_handle *h, const RowArgs &ra, const T *C, T *sigma) {
  const size_t row_bytes = ((size_t)ra.nb * sizeof(T) + 15) & ~(size_t)15;
  const size_t per_row_fixed = (size_t)ra.L * ra.L * sizeof(double) + (size_t)ra.max_as * sizeof(int2);
  const size_t tail = 2 * sizeof(int) + 16;
  // two rows per CTA when both fit: every beta table entry read from L2 then serves both rows
  if (2 * (row_bytes + per_row_fixed) + tail <= h->smem_optin && ra.na >= 2 * (uint32_t)h->num_sms)
    return launch_row<T, G, 2, true>(h, ra, C, sigma, 2 * (row_bytes + per_row_fixed) + tail);
  if (row_bytes + per_row_fixed + tail <= h->smem_optin)
    return launch_row<T, G, 1, true>(h, ra, C, sigma, row_bytes + per_row_fixed + tail);
  if (per_row_fixed + tail > h->smem_optin)
    return fail(SBD_TPB_ERR_INVALID, "sigma: alpha-single staging exceeds shared memory");
  return launch_row<T, G, 1, false>(h, ra, C, sigma, per_row_fixed + tail);
}

template <typename T, int CPT>
int launch_slab(sbd_tpb_handle *h, const SlabArgs &sa, const T *C, T *sigma) {
  const size_t W = (size_t)kSlabThreads * CPT;
  const size_t nslab = (sa.nb + W - 1) / W;
  const size_t blocks = nslab * sa.na;
  if (blocks > 0x7fffffffull) return fail(SBD_TPB_ERR_INVALID, "sigma: grid too large");
  sigma_alpha_slab_kernel<T, CPT><<<(unsigned)blocks, kSlabThreads, 0, h->stream>>>(sa, C, sigma);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

template <typename T>
int sigma_sep_shift(sbd_tpb_handle *h, const T *C, T *sigma, int accumulate, double shift) {
  const uint32_t na = (uint32_t)h->astr.size(), nb = (uint32_t)h->bstr.size();
  const bool dense_ab = h->ab.enabled;
  RowArgs ra;
  ra.astr = h->d_astr;
  ra.bstr = h->d_bstr;
  ra.bs_off = h->tb_s.off;
  ra.bs_ket = h->tb_s.ket;
  ra.bs_val = h->pb.s_val;
  ra.bs_valf = h->pb.s_valf;
  ra.bs_pair = h->pb.s_pair;
  ra.bd_off = h->tb_d.off;
  ra.bd_ket = h->tb_d.ket;
  ra.bd_val = h->pb.d_val;
  ra.bd_valf = h->pb.d_valf;
  ra.as_off = h->ta_s.off;
  ra.as_ket = h->ta_s.ket;
  ra.as_pair = h->pa.s_pair;
  ra.hii = h->d_hii;
  ra.vd = h->d_vd;
  ra.eri = h->d_eri;
  ra.L = h->L;
  ra.na = na;
  ra.nb = nb;
  ra.shift = shift;
  ra.accumulate = accumulate;
  ra.do_ab = dense_ab ? 0 : 1;
  ra.max_as = dense_ab ? 0 : (int)h->ta_s.max_row;

  // lanes per beta column from the mean beta row length (singles + doubles)
  const double mean_row = (double)(h->tb_s.nnz + h->tb_d.nnz) / nb;
  TPB_CUDA(cudaEventRecord(h->ev0, h->stream));
  if (mean_row >= 24) TPB_CHECK((launch_row_r<T, 32>(h, ra, C, sigma)));
  else if (mean_row >= 12) TPB_CHECK((launch_row_r<T, 16>(h, ra, C, sigma)));
  else if (mean_row >= 6) TPB_CHECK((launch_row_r<T, 8>(h, ra, C, sigma)));
  else TPB_CHECK((launch_row_r<T, 4>(h, ra, C, sigma)));
  TPB_CUDA(cudaEventRecord(h->ev_k[0], h->stream));
  h->sigma_kernels = 1;
  if (h->ta_s.nnz + h->ta_d.nnz > 0) {
    SlabArgs sa;
    sa.bstr = h->d_bstr;
    sa.as_off = h->ta_s.off;
    sa.as_ket = h->ta_s.ket;
    sa.as_val = h->pa.s_val;
    sa.as_valf = h->pa.s_valf;
    sa.as_pair = h->pa.s_pair;
    sa.ad_off = h->ta_d.off;
    sa.ad_ket = h->ta_d.ket;
    sa.ad_val = h->pa.d_val;
    sa.ad_valf = h->pa.d_valf;
    sa.vd = h->d_vd;
    sa.L = h->L;
    sa.na = na;
    sa.nb = nb;
    // slab width: keep na x slab bytes (the L2 working set) near 64 MB
    const double slab_bytes = 64.0e6 / na;
    const int cpt_max = std::max(1, (int)(slab_bytes / (kSlabThreads * sizeof(T))));
    if (cpt_max >= 8 && nb >= 8u * kSlabThreads) TPB_CHECK((launch_slab<T, 8>(h, sa, C, sigma)));
    else if (cpt_max >= 4 && nb >= 4u * kSlabThreads) TPB_CHECK((launch_slab<T, 4>(h, sa, C, sigma)));
    else if (cpt_max >= 2 && nb >= 2u * kSlabThreads) TPB_CHECK((launch_slab<T, 2>(h, sa, C, sigma)));
    else TPB_CHECK((launch_slab<T, 1>(h, sa, C, sigma)));
    TPB_CUDA(cudaEventRecord(h->ev_k[1], h->stream));
    h->sigma_kernels = 2;
  }
  if (dense_ab) TPB_CHECK(ab_dense_apply<T>(h, C, sigma));
  TPB_CUDA(cudaEventRecord(h->ev1, h->stream));
  return SBD_TPB_OK;
}

template <typename T>
int sigma_sep(sbd_tpb_handle *h, const T *C, T *sigma, int accumulate) {
  return sigma_sep_shift<T>(h, C, sigma, accumulate, 0.0);
}

template int sigma_sep<double>(sbd_tpb_handle *, const double *, double *, int);
template int sigma_sep<float>(sbd_tpb_handle *, const float *, float *, int);
template int sigma_sep_shift<double>(sbd_tpb_handle *, const double *, double *, int, double);
template int sigma_sep_shift<float>(sbd_tpb_handle *, const float *, float *, int, double);

}  // namespace sbdtpb
