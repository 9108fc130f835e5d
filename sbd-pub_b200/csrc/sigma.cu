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
constexpr int kSlabCols = 2;  // columns per thread
constexpr int kSlabWidth = kSlabThreads * kSlabCols;

template <typename T>
__device__ __forceinline__ T val_of(const double *v, const float *vf, uint32_t e);
template <>
__device__ __forceinline__ double val_of<double>(const double *v, const float *, uint32_t e) {
  return v[e];
}
template <>
__device__ __forceinline__ float val_of<float>(const double *, const float *vf, uint32_t e) {
  return vf[e];
}

struct RowArgs {
  const uint64_t *astr, *bstr;
  const uint32_t *b_off, *b_ket;
  const double *b_val;
  const float *b_valf;
  const int32_t *b_pair;
  const uint32_t *a_off, *a_ket;
  const int32_t *a_pair;
  const double *hii, *vd, *eri;
  int L;
  uint32_t na, nb;
  double shift;
  int accumulate;
  int do_ab;  // 1: direct alpha-beta loop here; 0: handled elsewhere
};

// Dynamic shared memory: [crow: nb T, 16B aligned][uA: L*L double][asng: max_sing int2]
template <typename T, bool kSmemRow>
__global__ void __launch_bounds__(kRowThreads)
    sigma_row_kernel(RowArgs a, const T *__restrict__ C, T *__restrict__ sigma) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t ia = blockIdx.x;
  const uint32_t nb = a.nb;
  const int L = a.L;
  const size_t L2 = (size_t)L * L;
  size_t off = 0;
  T *crow = reinterpret_cast<T *>(smem);
  if (kSmemRow) off = ((size_t)nb * sizeof(T) + 15) & ~(size_t)15;
  double *uA = reinterpret_cast<double *>(smem + off);
  off += L2 * sizeof(double);
  int2 *asng = reinterpret_cast<int2 *>(smem + off);

  const T *Crow_g = C + (size_t)ia * nb;
  if (kSmemRow) {
    for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) crow[j] = Crow_g[j];
  }
  // other-spin Coulomb term of beta singles: uA[pair] = sum_{k in Ia} (pair|kk)
  const uint64_t Ia = a.astr[ia];
  for (uint32_t pq = threadIdx.x; pq < L2; pq += blockDim.x) {
    double s = 0.0;
    uint64_t occ = Ia;
    while (occ) {
      s += a.vd[(size_t)pq * L + lowest_bit(occ)];
      occ &= occ - 1;
    }
    uA[pq] = s;
  }
  // alpha singles of this row (singles come first in the program row)
  const uint32_t a0 = a.a_off[ia], a1 = a.a_off[ia + 1];
  __shared__ int n_asng;
  if (threadIdx.x == 0) n_asng = 0;
  __syncthreads();
  if (a.do_ab) {
    for (uint32_t e = a0 + threadIdx.x; e < a1; e += blockDim.x) {
      const int32_t ps = a.a_pair[e];
      if (ps != 0) asng[e - a0] = make_int2((int)a.a_ket[e], ps);
      if (ps != 0) atomicMax(&n_asng, (int)(e - a0 + 1));
    }
  }
  __syncthreads();
  const int nas = n_asng;

  for (uint32_t ib = threadIdx.x; ib < nb; ib += blockDim.x) {
    const size_t bra = (size_t)ia * nb + ib;
    const T cself = kSmemRow ? crow[ib] : Crow_g[ib];
    double acc = (a.hii[bra] - a.shift) * (double)cself;
    const uint32_t e0 = a.b_off[ib], e1 = a.b_off[ib + 1];
    for (uint32_t e = e0; e < e1; e++) {
      const uint32_t jb = a.b_ket[e];
      double v = (double)val_of<T>(a.b_val, a.b_valf, e);
      const int32_t ps = a.b_pair[e];
      if (ps != 0) {
        const int pr = (ps > 0 ? ps : -ps) - 1;
        v += (ps > 0 ? uA[pr] : -uA[pr]);
        if (nas > 0) {
          // alpha single (Ja, pq, sa) x this beta single (Jb, rs, sb)
          const double sb = ps > 0 ? 1.0 : -1.0;
          double x = 0.0;
          for (int k = 0; k < nas; k++) {
            const int2 as = asng[k];
            const int pq = (as.y > 0 ? as.y : -as.y) - 1;
            const double g = a.eri[(size_t)pq * L2 + pr];
            const double cj = (double)C[(size_t)as.x * nb + jb];
            x += (as.y > 0 ? g : -g) * cj;
          }
          acc += sb * x;
        }
      }
      acc += v * (double)(kSmemRow ? crow[jb] : Crow_g[jb]);
    }
    if (a.accumulate) acc += (double)sigma[bra];
    sigma[bra] = (T)acc;
  }
}

struct SlabArgs {
  const uint64_t *bstr;
  const uint32_t *a_off, *a_ket;
  const double *a_val;
  const float *a_valf;
  const int32_t *a_pair;
  const double *vd;
  int L;
  uint32_t na, nb;
};

template <typename T>
__global__ void __launch_bounds__(kSlabThreads)
    sigma_alpha_slab_kernel(SlabArgs a, const T *__restrict__ C, T *__restrict__ sigma) {
  const uint32_t ia = blockIdx.x % a.na;
  const uint32_t slab = blockIdx.x / a.na;
  const uint32_t nb = a.nb;
  const int L = a.L;
  uint32_t col[kSlabCols];
  bool ok[kSlabCols];
  double acc[kSlabCols];
#pragma unroll
  for (int k = 0; k < kSlabCols; k++) {
    col[k] = slab * kSlabWidth + k * kSlabThreads + threadIdx.x;
    ok[k] = col[k] < nb;
    acc[k] = 0.0;
  }
  const uint32_t e0 = a.a_off[ia], e1 = a.a_off[ia + 1];
  for (uint32_t e = e0; e < e1; e++) {
    const uint32_t ja = __ldg(&a.a_ket[e]);
    const double v = (double)val_of<T>(a.a_val, a.a_valf, e);
    const int32_t ps = __ldg(&a.a_pair[e]);
    const T *crow = C + (size_t)ja * nb;
    if (ps == 0) {
#pragma unroll
      for (int k = 0; k < kSlabCols; k++)
        if (ok[k]) acc[k] += v * (double)crow[col[k]];
    } else {
      const int pr = (ps > 0 ? ps : -ps) - 1;
      const double *vrow = a.vd + (size_t)pr * L;
#pragma unroll
      for (int k = 0; k < kSlabCols; k++) {
        if (!ok[k]) continue;
        uint64_t occ = __ldg(&a.bstr[col[k]]);
        double o = 0.0;
        while (occ) {
          o += __ldg(&vrow[lowest_bit(occ)]);
          occ &= occ - 1;
        }
        acc[k] += (v + (ps > 0 ? o : -o)) * (double)crow[col[k]];
      }
    }
  }
  T *srow = sigma + (size_t)ia * nb;
#pragma unroll
  for (int k = 0; k < kSlabCols; k++)
    if (ok[k]) srow[col[k]] = (T)((double)srow[col[k]] + acc[k]);
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

template <typename T>
int sigma_sep_shift(sbd_tpb_handle *h, const T *C, T *sigma, int accumulate, double shift) {
  const uint32_t na = (uint32_t)h->astr.size(), nb = (uint32_t)h->bstr.size();
  const int L = h->L;
  const uint32_t max_sing = h->ta_s.max_row;
  const bool dense_ab = h->ab.enabled;

  RowArgs ra;
  ra.astr = h->d_astr;
  ra.bstr = h->d_bstr;
  ra.b_off = h->pb.off;
  ra.b_ket = h->pb.ket;
  ra.b_val = h->pb.val;
  ra.b_valf = h->pb.valf;
  ra.b_pair = h->pb.pairsgn;
  ra.a_off = h->pa.off;
  ra.a_ket = h->pa.ket;
  ra.a_pair = h->pa.pairsgn;
  ra.hii = h->d_hii;
  ra.vd = h->d_vd;
  ra.eri = h->d_eri;
  ra.L = L;
  ra.na = na;
  ra.nb = nb;
  ra.shift = shift;
  ra.accumulate = accumulate;
  ra.do_ab = dense_ab ? 0 : 1;

  const size_t row_bytes = ((size_t)nb * sizeof(T) + 15) & ~(size_t)15;
  const size_t fixed = (size_t)L * L * sizeof(double) + (size_t)std::max<uint32_t>(max_sing, 1) * sizeof(int2);
  const bool smem_row = row_bytes + fixed <= h->smem_optin;
  const size_t smem = (smem_row ? row_bytes : 0) + fixed;
  if (smem > h->smem_optin) return fail(SBD_TPB_ERR_INVALID, "sigma: shared-memory staging too large");

  TPB_CUDA(cudaEventRecord(h->ev0, h->stream));
  if (smem_row) {
    TPB_CUDA(cudaFuncSetAttribute(sigma_row_kernel<T, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    sigma_row_kernel<T, true><<<na, kRowThreads, smem, h->stream>>>(ra, C, sigma);
  } else {
    TPB_CUDA(cudaFuncSetAttribute(sigma_row_kernel<T, false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    sigma_row_kernel<T, false><<<na, kRowThreads, smem, h->stream>>>(ra, C, sigma);
  }
  TPB_LAUNCHED(h);
  TPB_CUDA(cudaEventRecord(h->ev_k[0], h->stream));
  h->sigma_kernels = 1;
  if (h->pa.nnz > 0) {
    SlabArgs sa;
    sa.bstr = h->d_bstr;
    sa.a_off = h->pa.off;
    sa.a_ket = h->pa.ket;
    sa.a_val = h->pa.val;
    sa.a_valf = h->pa.valf;
    sa.a_pair = h->pa.pairsgn;
    sa.vd = h->d_vd;
    sa.L = L;
    sa.na = na;
    sa.nb = nb;
    const size_t nslab = (nb + kSlabWidth - 1) / kSlabWidth;
    const size_t blocks = nslab * na;
    if (blocks > 0x7fffffffull) return fail(SBD_TPB_ERR_INVALID, "sigma: grid too large");
    sigma_alpha_slab_kernel<T><<<(unsigned)blocks, kSlabThreads, 0, h->stream>>>(sa, C, sigma);
    TPB_LAUNCHED(h);
    TPB_CUDA(cudaEventRecord(h->ev_k[1], h->stream));
    h->sigma_kernels = 2;
  }
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
