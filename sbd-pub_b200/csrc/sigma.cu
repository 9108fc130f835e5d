// sigma = H*C on the GPU (separated sign convention; see tpb_common.cuh).
//
// Replaces MultTPBThrust::run (tpb/mult_thrust.h:1172-1582) and sbd::mult (tpb/mult.h:625-881).
// Where the reference launches one thread per (connection, determinant) and adds into sigma with
// FP64 atomics, every sigma element here has exactly one owner, so results are deterministic:
//
//   alpha pass    sigma[Ia, Ib] = (H_ii - shift) C[Ia, Ib] + sum_Ja H_a(Ia, Ja) C[Ja, Ib]
//                 (+ the alpha-single x beta-single terms sa sb (pq|rs) C[Ja, Jb] when the
//                 singles are sparse), gathering rows Ja of C from an L2-resident column slab;
//                 the same CTA writes its own tile of C transposed into C^T.
//   beta pass     sigma[Ia, Ib] += sum_Jb H_b(Ib, Jb) C^T[Jb, Ia], the same kernel on C^T, its
//                 result transposed back through shared memory with coalesced writes.
// Both passes are the alpha-string "row SpMM" on a row-major operand, which is what makes every
// gather a 128-byte coalesced row segment.
//
// The alpha-beta term of FCI-like problems (dense singles) goes through the gather -> dense
// (pq|rs) contraction -> scatter path in ab_dense.cu instead of the direct loop.
#include <algorithm>

#include "tpb_common.cuh"

namespace sbdtpb {
namespace {

constexpr int kBlkRows = 32;     // bra rows per CTA
constexpr int kBlkThreads = 128;

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

struct BlockArgs {
  // sigma program of the bra spin (rows of X)
  const uint32_t *s_off, *s_ket;
  const double *s_val;
  const float *s_valf;
  const int32_t *s_pair;
  const uint32_t *d_off, *d_ket;
  const double *d_val;
  const float *d_valf;
  const uint64_t *col_str;  // strings of the column spin (other-spin Coulomb term of singles)
  const double *vd;         // (pq|kk) [L*L][L]
  int L;
  uint32_t nrows, ncols;    // X is nrows x ncols, row-major
  // alpha pass only: on-the-fly diagonal, alpha-single x beta-single terms
  double core_shift;        // I0 - shift
  const double *Ea, *Eb, *uJ;
  int accumulate;
  int do_ab;
  const uint32_t *bs_off, *bs_ket;
  const int32_t *bs_pair;
  const double *eri;
};

// One kernel, two passes.  A CTA owns 32 consecutive bra strings (rows of X) and a slab of
// kBlkThreads*CPT columns; blocks run slab-major so the CTAs in flight gather from one slab of X
// that stays in L2.  For each of its rows a thread accumulates sum_ket H(row, ket) X[ket, col]
// over its CPT columns.
//   alpha pass (kAlpha): X = C.  Adds the diagonal (computed from per-string energies) and the
//     alpha-single x beta-single terms, writes sigma[Ia, Ib] once, and writes the CTA's own
//     32 x slab tile of C transposed into XT (C^T) through shared memory.
//   beta pass: X = C^T.  The 32 x slab tile of results goes through shared memory and is added
//     into sigma[Ia, Ib0..Ib0+31] with 128-byte coalesced read-modify-writes.
template <typename T, int CPT, bool kAlpha>
__global__ void __launch_bounds__(kBlkThreads)
    sigma_block_kernel(BlockArgs a, const T *__restrict__ X, T *__restrict__ out, T *__restrict__ XT) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int W = kBlkThreads * CPT;
  T(*tile)[W + 1] = reinterpret_cast<T(*)[W + 1]>(smem_raw);
  const uint32_t nrb = (a.nrows + kBlkRows - 1) / kBlkRows;
  const uint32_t rb = blockIdx.x % nrb, slab = blockIdx.x / nrb;
  const uint32_t r0 = rb * kBlkRows, c0 = slab * W;
  const uint32_t ncols = a.ncols;
  const int L = a.L, L2 = L * L;
  const int nr = (int)min((uint32_t)kBlkRows, a.nrows - r0);
  uint32_t col[CPT];
  bool ok[CPT];
  uint64_t cstr[CPT];
  double ecol[CPT];
#pragma unroll
  for (int k = 0; k < CPT; k++) {
    col[k] = c0 + threadIdx.x + k * kBlkThreads;
    ok[k] = col[k] < ncols;
    cstr[k] = ok[k] ? __ldg(&a.col_str[col[k]]) : 0ull;
    ecol[k] = (kAlpha && ok[k]) ? __ldg(&a.Eb[col[k]]) : 0.0;
  }
  for (int r = 0; r < nr; r++) {
    const uint32_t row = r0 + r;
    T acc[CPT];
#pragma unroll
    for (int k = 0; k < CPT; k++) acc[k] = T(0);
    const uint32_t d0 = __ldg(&a.d_off[row]), d1 = __ldg(&a.d_off[row + 1]);
#pragma unroll 4
    for (uint32_t e = d0; e < d1; e++) {
      const uint32_t ket = __ldg(&a.d_ket[e]);
      const T v = val_of<T>(a.d_val, a.d_valf, e);
      const T *xr = X + (size_t)ket * ncols;
#pragma unroll
      for (int k = 0; k < CPT; k++)
        if (ok[k]) acc[k] += v * __ldg(&xr[col[k]]);
    }
    const uint32_t s0 = __ldg(&a.s_off[row]), s1 = __ldg(&a.s_off[row + 1]);
    for (uint32_t e = s0; e < s1; e++) {
      const uint32_t ket = __ldg(&a.s_ket[e]);
      const double v = (double)val_of<T>(a.s_val, a.s_valf, e);
      const int32_t ps = __ldg(&a.s_pair[e]);
      const int pr = (ps > 0 ? ps : -ps) - 1;
      const double sg = ps > 0 ? 1.0 : -1.0;
      const double *vrow = a.vd + (size_t)pr * L;
      const T *xr = X + (size_t)ket * ncols;
#pragma unroll
      for (int k = 0; k < CPT; k++) {
        if (!ok[k]) continue;
        uint64_t occ = cstr[k];
        double o = 0.0;
        while (occ) {
          o += __ldg(&vrow[lowest_bit(occ)]);
          occ &= occ - 1;
        }
        double x = (v + sg * o) * (double)__ldg(&xr[col[k]]);
        if (kAlpha && a.do_ab) {
          // this alpha single (ket = Ja, pair pr, sign sg) x every beta single of column Ib
          for (uint32_t f = __ldg(&a.bs_off[col[k]]); f < __ldg(&a.bs_off[col[k] + 1]); f++) {
            const int32_t pb = __ldg(&a.bs_pair[f]);
            const int rs = (pb > 0 ? pb : -pb) - 1;
            const double g = __ldg(&a.eri[(size_t)pr * L2 + rs]);
            const double cj = (double)__ldg(&xr[__ldg(&a.bs_ket[f])]);
            x += (pb > 0 ? g : -g) * cj * sg;
          }
        }
        acc[k] += (T)x;
      }
    }
    if (kAlpha) {
      const double erow = a.core_shift + __ldg(&a.Ea[row]);
      const double *urow = a.uJ + (size_t)row * L;
#pragma unroll
      for (int k = 0; k < CPT; k++) {
        if (!ok[k]) continue;
        const size_t idx = (size_t)row * ncols + col[k];
        const T own = __ldg(&X[idx]);
        tile[r][threadIdx.x + k * kBlkThreads] = own;
        // H_ii - shift = I0 + E(Ia) + E(Ib) + sum_{q in Ib} uJ[Ia][q] - shift
        uint64_t occ = cstr[k];
        double hd = erow + ecol[k];
        while (occ) {
          hd += __ldg(&urow[lowest_bit(occ)]);
          occ &= occ - 1;
        }
        double res = (double)acc[k] + hd * (double)own;
        if (a.accumulate) res += (double)out[idx];
        out[idx] = (T)res;
      }
    } else {
#pragma unroll
      for (int k = 0; k < CPT; k++) tile[r][threadIdx.x + k * kBlkThreads] = acc[k];
    }
  }
  __syncthreads();
  // transposed write-out: lane = row within the block, one warp per column
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t ccount = min((uint32_t)W, ncols - c0);
  for (uint32_t c = warp; c < ccount; c += kBlkThreads / 32) {
    if (lane >= nr) continue;
    const size_t o = (size_t)(c0 + c) * a.nrows + r0 + lane;
    if (kAlpha) XT[o] = tile[lane][c];
    else out[o] += tile[lane][c];
  }
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

template <typename T, int CPT, bool kAlpha>
int launch_block(sbd_tpb_handle *h, const BlockArgs &ba, const T *X, T *out, T *XT) {
  constexpr int W = kBlkThreads * CPT;
  const size_t nrb = (ba.nrows + kBlkRows - 1) / kBlkRows, nslab = (ba.ncols + W - 1) / W;
  const size_t blocks = nrb * nslab;
  if (blocks > 0x7fffffffull) return fail(SBD_TPB_ERR_INVALID, "sigma: grid too large");
  const size_t smem = sizeof(T) * kBlkRows * (W + 1);
  auto kern = sigma_block_kernel<T, CPT, kAlpha>;
  TPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)blocks, kBlkThreads, smem, h->stream>>>(ba, X, out, XT);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

template <typename T>
int sigma_sep_shift(sbd_tpb_handle *h, const T *C, T *sigma, int accumulate, double shift) {
  const uint32_t na = (uint32_t)h->astr.size(), nb = (uint32_t)h->bstr.size();
  const bool dense_ab = h->ab.enabled;
  const size_t n = h->ndet();
  if (h->ct_bytes < n * sizeof(T)) {
    if (h->d_ct) cudaFree(h->d_ct);
    h->d_ct = nullptr;
    h->ct_bytes = 0;
    TPB_CUDA(cudaMalloc(&h->d_ct, n * sizeof(double)));
    h->ct_bytes = n * sizeof(double);
  }
  T *CT = reinterpret_cast<T *>(h->d_ct);
  constexpr int CPT = sizeof(T) == 4 ? 4 : 2;

  BlockArgs ba{};
  ba.s_off = h->ta_s.off;
  ba.s_ket = h->ta_s.ket;
  ba.s_val = h->pa.s_val;
  ba.s_valf = h->pa.s_valf;
  ba.s_pair = h->pa.s_pair;
  ba.d_off = h->ta_d.off;
  ba.d_ket = h->ta_d.ket;
  ba.d_val = h->pa.d_val;
  ba.d_valf = h->pa.d_valf;
  ba.col_str = h->d_bstr;
  ba.vd = h->d_vd;
  ba.L = h->L;
  ba.nrows = na;
  ba.ncols = nb;
  ba.core_shift = h->I0 - shift;
  ba.Ea = h->d_Ea;
  ba.Eb = h->d_Eb;
  ba.uJ = h->d_uJ;
  ba.accumulate = accumulate;
  ba.do_ab = dense_ab ? 0 : 1;
  ba.bs_off = h->tb_s.off;
  ba.bs_ket = h->tb_s.ket;
  ba.bs_pair = h->pb.s_pair;
  ba.eri = h->d_eri;
  TPB_CUDA(cudaEventRecord(h->ev0, h->stream));
  TPB_CHECK((launch_block<T, CPT, true>(h, ba, C, sigma, CT)));
  TPB_CUDA(cudaEventRecord(h->ev_k[0], h->stream));

  BlockArgs bb{};
  bb.s_off = h->tb_s.off;
  bb.s_ket = h->tb_s.ket;
  bb.s_val = h->pb.s_val;
  bb.s_valf = h->pb.s_valf;
  bb.s_pair = h->pb.s_pair;
  bb.d_off = h->tb_d.off;
  bb.d_ket = h->tb_d.ket;
  bb.d_val = h->pb.d_val;
  bb.d_valf = h->pb.d_valf;
  bb.col_str = h->d_astr;
  bb.vd = h->d_vd;
  bb.L = h->L;
  bb.nrows = nb;
  bb.ncols = na;
  TPB_CHECK((launch_block<T, CPT, false>(h, bb, CT, sigma, nullptr)));
  TPB_CUDA(cudaEventRecord(h->ev_k[1], h->stream));
  h->sigma_kernels = 2;
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
