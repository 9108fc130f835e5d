// Spin-resolved 1- and 2-RDMs of the converged vector.
//
// Replaces Correlation (tpb/correlation.h:378-664, with Zero/One/TwoDiffCorrelation of
// basic/correlation.h:16-231) and MultTPBThrust::correlation (tpb/correlation_thrust.h:504-731).
// The reference adds every (bra, ket) contribution into the L^4 arrays with FP64 atomics (GPU)
// or per-thread private copies (CPU).  Here each contribution class is first contracted over the
// index it does not carry, on the GPU, into a short per-pair list; the host then places those
// sums into the reference layouts:
//   onebody[s][p + L q]          = <c+_{p s} c_{q s}>
//   twobody[s + 2t][p + L q + L^2 r + L^3 u] = <c+_{p s} c+_{q t} c_{u t} c_{r s}>
// (the layout the reference app contracts with (pr|qs), apps/.../main.cc:264-317).
//   diagonal      rho_a[Ia] = sum_Ib W^2, rho_b[Ib] = sum_Ia W^2, M[p][q] = sum W^2 n_p(Ia) n_q(Ib)
//   alpha pairs   T0(Ia,Ja) = sum_Ib W[Ia,Ib] W[Ja,Ib]  (+ per beta orbital q for singles)
//   beta pairs    the same on the transposed vector
//   alpha x beta  X(e, rs) = sum_{beta singles with label rs} s_b W[Ia,Ib] W[Ja,Jb]
// Signs are those of the separated convention, in which the vector W also lives, so the RDMs
// equal the reference's.  Same-spin blocks are the physical <c+ c+ c c> above; the opposite-spin
// blocks of alpha-single x beta-single pairs follow the reference's placement rule, which puts
// a pair's value in the [s+2t] block chosen by the spin-orbital ordering of its four indices
// (basic/correlation.h:191-231), so the spin-resolved arrays match it entry by entry.
#include <algorithm>
#include <cstring>
#include <vector>

#include "tpb_common.cuh"

namespace sbdtpb {
namespace {

constexpr int kRdmThreads = 256;

__device__ __forceinline__ double block_sum(double x, double *red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  __syncthreads();
  if (lane == 0) red[wid] = x;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
  return s;  // valid in thread 0
}

// rho_a[Ia] = sum_Ib W^2 and Y[Ia][q] = sum_{Ib : q in Ib} W^2; one CTA per alpha row.  Each warp
// takes 32 beta columns at a time: the orbitals every lane's string holds get the warp's total
// once, the others (held by some lanes only) one warp sum each; lane 0 adds them into its warp's
// own row of shared memory, and the warps' rows are added in warp order, so the sums are the same
// on every run (no floating-point atomics).
__global__ void __launch_bounds__(kRdmThreads)
    rdm_row_kernel(const double *__restrict__ W, const uint64_t *__restrict__ bstr, uint32_t nb, int L,
                   double *__restrict__ rho_a, double *__restrict__ Y) {
  __shared__ double mq[kRdmThreads / 32][64];
  __shared__ double red[32];
  const uint32_t ia = blockIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < (kRdmThreads / 32) * 64; i += blockDim.x) (&mq[0][0])[i] = 0.0;
  __syncthreads();
  double s = 0.0;
  const uint32_t nbp = (nb + 31) & ~31u;  // every lane of a warp runs the same iterations
  for (uint32_t ib = threadIdx.x; ib < nbp; ib += blockDim.x) {
    const bool in = ib < nb;
    const double w = in ? W[(size_t)ia * nb + ib] : 0.0;
    const double w2 = __dmul_rn(w, w);  // rounded product (never fused): rdm_rowsum_kernel repeats it
    const uint64_t occ = in ? bstr[ib] : 0ull;
    s += w2;
    const unsigned lo = (unsigned)occ, hi = (unsigned)(occ >> 32);
    const uint64_t all = ((uint64_t)__reduce_and_sync(0xffffffffu, hi) << 32) | __reduce_and_sync(0xffffffffu, lo);
    const uint64_t any = ((uint64_t)__reduce_or_sync(0xffffffffu, hi) << 32) | __reduce_or_sync(0xffffffffu, lo);
    double tot = w2;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    uint64_t some = any & ~all;
    while (some) {
      const int q = lowest_bit(some);
      double v = ((occ >> q) & 1) ? w2 : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) mq[wid][q] += v;
      some &= some - 1;
    }
    if (lane == 0) {
      uint64_t a = all;
      while (a) {
        mq[wid][lowest_bit(a)] += tot;
        a &= a - 1;
      }
    }
  }
  const double t = block_sum(s, red);
  if (threadIdx.x == 0) rho_a[ia] = t;
  __syncthreads();
  for (int q = threadIdx.x; q < L; q += blockDim.x) {
    double v = 0.0;
    for (int w = 0; w < kRdmThreads / 32; w++) v += mq[w][q];
    Y[(size_t)ia * L + q] = v;
  }
}

// rho_a[Ia] = sum_Ib W[Ia, Ib]^2 alone (orbital occupations need no pair sums): the same
// per-thread order and block sum as rdm_row_kernel's rho_a, so the occupations repeat bit for bit
__global__ void __launch_bounds__(kRdmThreads)
    rdm_rowsum_kernel(const double *__restrict__ W, uint32_t nb, double *__restrict__ rho_a) {
  __shared__ double red[32];
  const uint32_t ia = blockIdx.x;
  double s = 0.0;
  const uint32_t nbp = (nb + 31) & ~31u;
  for (uint32_t ib = threadIdx.x; ib < nbp; ib += blockDim.x) {
    const double w = ib < nb ? W[(size_t)ia * nb + ib] : 0.0;
    s += __dmul_rn(w, w);
  }
  const double t = block_sum(s, red);
  if (threadIdx.x == 0) rho_a[ia] = t;
}

// Mpart[c][p*L + q] = sum over alpha rows Ia of chunk c with p in Ia of Y[Ia][q]
__global__ void rdm_pq_kernel(const double *__restrict__ Y, const uint64_t *__restrict__ astr, uint32_t na, int L,
                              uint32_t rows_per_chunk, double *__restrict__ Mpart) {
  const int pq = blockIdx.x * blockDim.x + threadIdx.x;
  if (pq >= L * L) return;
  const int p = pq / L, q = pq - p * L;
  const uint32_t r0 = blockIdx.y * rows_per_chunk, r1 = min(na, r0 + rows_per_chunk);
  double v = 0.0;
  for (uint32_t r = r0; r < r1; r++)
    if ((astr[r] >> p) & 1) v += Y[(size_t)r * L + q];
  Mpart[(size_t)blockIdx.y * L * L + pq] = v;
}

// column sums of W^2 over a chunk of rows: part[chunk][col]
__global__ void rdm_colsum_kernel(const double *__restrict__ W, uint32_t na, uint32_t nb,
                                  uint32_t rows_per_chunk, double *__restrict__ part) {
  const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= nb) return;
  const uint32_t r0 = blockIdx.y * rows_per_chunk;
  const uint32_t r1 = min(na, r0 + rows_per_chunk);
  double s = 0.0;
  for (uint32_t r = r0; r < r1; r++) {
    const double w = W[(size_t)r * nb + col];
    s += w * w;
  }
  part[(size_t)blockIdx.y * nb + col] = s;
}

// rho_b[col] = sum of the chunk partials in chunk order
__global__ void rdm_chunk_sum_kernel(const double *__restrict__ part, uint32_t nchunks, uint32_t n,
                                     double *__restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (uint32_t c = 0; c < nchunks; c++) s += part[(size_t)c * n + i];
  out[i] = s;
}

// T0[e] = sum_c X[bra,c] X[ket,c]; Tq[e][q] = same restricted to columns whose other-spin string
// holds q (only when Tq != null).  One CTA per bra row of the CSR table; its entries go kPairE at a
// time, so each pass over the columns reads the bra row once for kPairE ket rows.  The per-orbital
// sums take the warp trick of rdm_row_kernel (orbitals held by all 32 columns of a warp get the
// warp total, the others one warp sum each, lane 0 adds into its warp's row of shared memory), and
// every sum has a fixed order, so the results repeat bit for bit.
constexpr int kPairE = 4;

__global__ void __launch_bounds__(kRdmThreads)
    rdm_pair_kernel(const double *__restrict__ X, uint32_t ncol, const uint32_t *__restrict__ off,
                    const uint32_t *__restrict__ ket, const uint64_t *__restrict__ other, int L,
                    double *__restrict__ T0, double *__restrict__ Tq) {
  constexpr int NW = kRdmThreads / 32;
  __shared__ double red[NW][kPairE];
  __shared__ double acc[kPairE][NW][64];
  const uint32_t row = blockIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const double *xr = X + (size_t)row * ncol;
  const uint32_t ncp = (ncol + 31) & ~31u;  // every lane of a warp runs the same iterations
  for (uint32_t e0 = off[row]; e0 < off[row + 1]; e0 += kPairE) {
    const int ne = (int)min((uint32_t)kPairE, off[row + 1] - e0);
    const double *xk[kPairE];
#pragma unroll
    for (int k = 0; k < kPairE; k++) xk[k] = X + (size_t)ket[e0 + (k < ne ? k : 0)] * ncol;
    if (Tq) {
      for (int i = threadIdx.x; i < kPairE * NW * 64; i += blockDim.x) (&acc[0][0][0])[i] = 0.0;
      __syncthreads();
    }
    double sum[kPairE];
#pragma unroll
    for (int k = 0; k < kPairE; k++) sum[k] = 0.0;
    for (uint32_t c = threadIdx.x; c < ncp; c += blockDim.x) {
      const bool in = c < ncol;
      const double b = in ? xr[c] : 0.0;
      double x[kPairE];
#pragma unroll
      for (int k = 0; k < kPairE; k++) {
        x[k] = (in && k < ne) ? b * xk[k][c] : 0.0;
        sum[k] += x[k];
      }
      if (Tq) {
        const uint64_t occ = in ? other[c] : 0ull;
        const unsigned lo = (unsigned)occ, hi = (unsigned)(occ >> 32);
        const uint64_t all =
            ((uint64_t)__reduce_and_sync(0xffffffffu, hi) << 32) | __reduce_and_sync(0xffffffffu, lo);
        const uint64_t any =
            ((uint64_t)__reduce_or_sync(0xffffffffu, hi) << 32) | __reduce_or_sync(0xffffffffu, lo);
#pragma unroll
        for (int k = 0; k < kPairE; k++) {
          if (k >= ne) break;
          double tot = x[k];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
          uint64_t some = any & ~all;
          while (some) {
            const int q = lowest_bit(some);
            double v = ((occ >> q) & 1) ? x[k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) acc[k][wid][q] += v;
            some &= some - 1;
          }
          if (lane == 0) {
            uint64_t a = all;
            while (a) {
              acc[k][wid][lowest_bit(a)] += tot;
              a &= a - 1;
            }
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kPairE; k++) {
      double v = sum[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[wid][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < ne) {
      double t = 0.0;
      for (int w = 0; w < NW; w++) t += red[w][threadIdx.x];
      T0[e0 + threadIdx.x] = t;
    }
    if (Tq) {
      for (int i = threadIdx.x; i < ne * L; i += blockDim.x) {
        const int k = i / L, q = i - k * L;
        double t = 0.0;
        for (int w = 0; w < NW; w++) t += acc[k][w][q];
        Tq[(size_t)(e0 + k) * L + q] = t;
      }
    }
    __syncthreads();
  }
}

__global__ void transpose_kernel(const double *__restrict__ A, double *__restrict__ B,
                                 uint32_t rows, uint32_t cols) {
  __shared__ double tile[32][33];
  const uint32_t bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const uint32_t r = by + k, c = bx + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = A[(size_t)r * cols + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const uint32_t c = bx + k, r = by + threadIdx.x;
    if (r < rows && c < cols) B[(size_t)c * rows + r] = tile[threadIdx.x][k];
  }
}

// X[e][rs] for one alpha single e = (ia, ja) per CTA; beta singles given flat.
__global__ void __launch_bounds__(kRdmThreads)
    rdm_mixed_kernel(const double *__restrict__ W, uint32_t nb, const uint32_t *__restrict__ a_bra,
                     const uint32_t *__restrict__ a_ket, const uint32_t *__restrict__ b_bra,
                     const uint32_t *__restrict__ b_ket, const int32_t *__restrict__ b_lab,
                     uint32_t nbp, int L2, double *__restrict__ X) {
  extern __shared__ double accs[];
  const uint32_t e = blockIdx.x;
  for (int i = threadIdx.x; i < L2; i += blockDim.x) accs[i] = 0.0;
  __syncthreads();
  const double *wa = W + (size_t)a_bra[e] * nb;
  const double *wj = W + (size_t)a_ket[e] * nb;
  for (uint32_t k = threadIdx.x; k < nbp; k += blockDim.x) {
    const int32_t lab = b_lab[k];
    const double x = wa[b_bra[k]] * wj[b_ket[k]];
    atomicAdd(&accs[(lab > 0 ? lab : -lab) - 1], lab > 0 ? x : -x);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < L2; i += blockDim.x) X[(size_t)e * L2 + i] = accs[i];
}

struct HostTable {
  std::vector<uint32_t> off, ket, lab;
};

int fetch(sbd_tpb_handle *h, const ExTable &t, size_t n, HostTable &o) {
  o.off.resize(n + 1);
  o.ket.resize(t.nnz);
  o.lab.resize(t.nnz);
  TPB_CUDA(cudaMemcpy(o.off.data(), t.off, sizeof(uint32_t) * (n + 1), cudaMemcpyDeviceToHost));
  if (t.nnz) {
    TPB_CUDA(cudaMemcpy(o.ket.data(), t.ket, sizeof(uint32_t) * t.nnz, cudaMemcpyDeviceToHost));
    TPB_CUDA(cudaMemcpy(o.lab.data(), t.lab, sizeof(uint32_t) * t.nnz, cudaMemcpyDeviceToHost));
  }
  return SBD_TPB_OK;
}

inline int popc(uint64_t x) { return __builtin_popcountll(x); }
inline double single_sign(uint64_t I, int cr, int an) {
  const int lo = std::min(cr, an), hi = std::max(cr, an);
  return (popc(I & open_mask(lo, hi)) & 1) ? -1.0 : 1.0;
}
inline double double_sign(uint64_t I, int i0, int j0, int a0, int b0) {
  int par = popc(I & open_mask(std::min(i0, a0), std::max(i0, a0))) +
            popc(I & open_mask(std::min(j0, b0), std::max(j0, b0)));
  if (a0 > j0 || b0 < i0) par++;
  return (par & 1) ? -1.0 : 1.0;
}

struct Rdm {
  int L;
  size_t L2, L4;
  std::vector<double> one, two;
  Rdm(int L_) : L(L_), L2((size_t)L_ * L_), L4((size_t)L_ * L_ * L_ * L_), one(2 * L2, 0.0), two(4 * L4, 0.0) {}
  double &g(int s, int p, int q) { return one[s * L2 + p + (size_t)L * q]; }
  double &G(int s, int t, int p, int q, int r, int u) {
    return two[(s + 2 * t) * L4 + p + (size_t)L * q + L2 * r + L2 * L * u];
  }
  // <c+_{cr s} c+_{j t} c_{j t} c_{an s}> = x for j != cr, an (both pair orders, exchange if s==t)
  void single_with_number(int s, int cr, int an, int t, int j, double x) {
    G(s, t, cr, j, an, j) += x;
    G(t, s, j, cr, j, an) += x;
    if (s == t) {
      G(s, s, cr, j, j, an) -= x;
      G(s, s, j, cr, an, j) -= x;
    }
  }
};

}  // namespace

int rdm_sep(sbd_tpb_handle *h, const double *W, double *one, double *two, double *density) {
  const uint32_t na = (uint32_t)h->astr.size(), nb = (uint32_t)h->bstr.size();
  const int L = h->L;
  const size_t n = h->ndet();
  constexpr uint32_t kChunk = 1024;
  const uint32_t nca = (na + kChunk - 1) / kChunk;
  if (!one && !two) {
    // orbital occupations only: the string weights rho (row and column sums of W^2), summed over
    // each string's orbitals in the order the full pass below adds them
    if (!density) return SBD_TPB_OK;
    double *d_rho = nullptr, *d_cp = nullptr;
    TPB_CUDA(cudaMalloc(&d_rho, sizeof(double) * ((size_t)na + nb)));
    TPB_CUDA(cudaMalloc(&d_cp, sizeof(double) * (size_t)nca * nb));
    rdm_rowsum_kernel<<<na, kRdmThreads, 0, h->stream>>>(W, nb, d_rho);
    TPB_LAUNCHED(h);
    dim3 gridc((nb + 255) / 256, nca);
    rdm_colsum_kernel<<<gridc, 256, 0, h->stream>>>(W, na, nb, kChunk, d_cp);
    TPB_LAUNCHED(h);
    rdm_chunk_sum_kernel<<<(nb + 255) / 256, 256, 0, h->stream>>>(d_cp, nca, nb, d_rho + na);
    TPB_LAUNCHED(h);
    std::vector<double> rho((size_t)na + nb);
    const cudaError_t e1 = cudaMemcpyAsync(rho.data(), d_rho, sizeof(double) * rho.size(), cudaMemcpyDeviceToHost,
                                           h->stream);
    const cudaError_t e2 = e1 == cudaSuccess ? cudaStreamSynchronize(h->stream) : e1;
    cudaFree(d_rho);
    cudaFree(d_cp);
    if (e2 != cudaSuccess) return fail(SBD_TPB_ERR_CUDA, std::string("occupations: ") + cudaGetErrorString(e2));
    std::vector<double> occ(2 * (size_t)L, 0.0);
    auto add = [&](int s, const std::vector<uint64_t> &str, const double *r) {
      for (size_t i = 0; i < str.size(); i++)
        for (int p = 0; p < L; p++)
          if ((str[i] >> p) & 1) occ[2 * p + s] += r[i];
    };
    add(0, h->astr, rho.data());
    add(1, h->bstr, rho.data() + na);
    std::memcpy(density, occ.data(), sizeof(double) * occ.size());
    return SBD_TPB_OK;
  }
  Rdm R(L);
  // ---- diagonal part (deterministic: fixed summation order throughout)
  double *d_rho_a = nullptr, *d_rho_b = nullptr, *d_Y = nullptr, *d_Mp = nullptr, *d_cp = nullptr;
  TPB_CUDA(cudaMalloc(&d_rho_a, sizeof(double) * na));
  TPB_CUDA(cudaMalloc(&d_rho_b, sizeof(double) * nb));
  TPB_CUDA(cudaMalloc(&d_Y, sizeof(double) * (size_t)na * L));
  TPB_CUDA(cudaMalloc(&d_Mp, sizeof(double) * (size_t)nca * L * L));
  TPB_CUDA(cudaMalloc(&d_cp, sizeof(double) * (size_t)nca * nb));
  rdm_row_kernel<<<na, kRdmThreads, 0, h->stream>>>(W, h->d_bstr, nb, L, d_rho_a, d_Y);
  TPB_LAUNCHED(h);
  {
    dim3 grid((L * L + 127) / 128, nca);
    rdm_pq_kernel<<<grid, 128, 0, h->stream>>>(d_Y, h->d_astr, na, L, kChunk, d_Mp);
    TPB_LAUNCHED(h);
    dim3 gridc((nb + 255) / 256, nca);
    rdm_colsum_kernel<<<gridc, 256, 0, h->stream>>>(W, na, nb, kChunk, d_cp);
    TPB_LAUNCHED(h);
    rdm_chunk_sum_kernel<<<(nb + 255) / 256, 256, 0, h->stream>>>(d_cp, nca, nb, d_rho_b);
    TPB_LAUNCHED(h);
  }
  std::vector<double> rho_a(na), rho_b(nb), Mp((size_t)nca * L * L), M((size_t)L * L, 0.0);
  TPB_CUDA(cudaMemcpyAsync(rho_a.data(), d_rho_a, sizeof(double) * na, cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaMemcpyAsync(rho_b.data(), d_rho_b, sizeof(double) * nb, cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaMemcpyAsync(Mp.data(), d_Mp, sizeof(double) * Mp.size(), cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  for (uint32_t c = 0; c < nca; c++)
    for (size_t k = 0; k < M.size(); k++) M[k] += Mp[(size_t)c * L * L + k];
  cudaFree(d_rho_a);
  cudaFree(d_rho_b);
  cudaFree(d_Y);
  cudaFree(d_Mp);
  cudaFree(d_cp);
  auto diag_same = [&](int s, const std::vector<uint64_t> &str, const std::vector<double> &rho) {
    for (size_t i = 0; i < str.size(); i++) {
      const double w2 = rho[i];
      for (int p = 0; p < L; p++) {
        if (!((str[i] >> p) & 1)) continue;
        R.g(s, p, p) += w2;
        for (int q = 0; q < L; q++) {
          if (q == p || !((str[i] >> q) & 1)) continue;
          R.G(s, s, p, q, p, q) += w2;   // n_p n_q
          R.G(s, s, p, q, q, p) -= w2;   // exchange
        }
      }
    }
  };
  diag_same(0, h->astr, rho_a);
  diag_same(1, h->bstr, rho_b);
  for (int p = 0; p < L; p++)
    for (int q = 0; q < L; q++) {
      const double m = M[(size_t)p * L + q];
      R.G(0, 1, p, q, p, q) += m;
      R.G(1, 0, q, p, q, p) += m;
    }

  if (one || two) {
    HostTable as, ad, bs, bd;
    TPB_CHECK(fetch(h, h->ta_s, na, as));
    TPB_CHECK(fetch(h, h->ta_d, na, ad));
    TPB_CHECK(fetch(h, h->tb_s, nb, bs));
    TPB_CHECK(fetch(h, h->tb_d, nb, bd));
    double *d_WT = nullptr, *d_T0 = nullptr, *d_Tq = nullptr;
    const size_t maxp = std::max({h->ta_s.nnz, h->ta_d.nnz, h->tb_s.nnz, h->tb_d.nnz, (size_t)1});
    TPB_CUDA(cudaMalloc(&d_WT, sizeof(double) * n));
    TPB_CUDA(cudaMalloc(&d_T0, sizeof(double) * maxp));
    TPB_CUDA(cudaMalloc(&d_Tq, sizeof(double) * maxp * L));
    {
      dim3 grid((nb + 31) / 32, (na + 31) / 32), block(32, 8);
      transpose_kernel<<<grid, block, 0, h->stream>>>(W, d_WT, na, nb);
      TPB_LAUNCHED(h);
    }
    std::vector<double> T0, Tq;
    // same-spin pairs; s = 0 alpha (rows of W), 1 beta (rows of W^T)
    auto run_pairs = [&](int s, const double *X, uint32_t nrow, uint32_t ncol, const ExTable &t,
                         const HostTable &ht, const uint64_t *d_other, bool single) -> int {
      if (t.nnz == 0) return SBD_TPB_OK;
      rdm_pair_kernel<<<nrow, kRdmThreads, 0, h->stream>>>(X, ncol, t.off, t.ket, d_other, L, d_T0,
                                                         single ? d_Tq : nullptr);
      TPB_LAUNCHED(h);
      T0.resize(t.nnz);
      TPB_CUDA(cudaMemcpyAsync(T0.data(), d_T0, sizeof(double) * t.nnz, cudaMemcpyDeviceToHost, h->stream));
      if (single) {
        Tq.resize(t.nnz * L);
        TPB_CUDA(cudaMemcpyAsync(Tq.data(), d_Tq, sizeof(double) * t.nnz * L, cudaMemcpyDeviceToHost, h->stream));
      }
      TPB_CUDA(cudaStreamSynchronize(h->stream));
      const std::vector<uint64_t> &str = s == 0 ? h->astr : h->bstr;
      const int o = 1 - s;
      for (uint32_t i = 0; i < nrow; i++) {
        const uint64_t I = str[i];
        for (uint32_t e = ht.off[i]; e < ht.off[i + 1]; e++) {
          const uint32_t lab = ht.lab[e];
          if (single) {
            const int cr = lab & 0xff, an = (lab >> 8) & 0xff;
            const double x = single_sign(I, cr, an) * T0[e];
            R.g(s, cr, an) += x;
            uint64_t occ = I & ~(1ull << cr);
            while (occ) {
              const int j = __builtin_ctzll(occ);
              R.single_with_number(s, cr, an, s, j, x);
              occ &= occ - 1;
            }
            const double sg = single_sign(I, cr, an);
            for (int j = 0; j < L; j++) {
              const double y = sg * Tq[(size_t)e * L + j];
              if (y != 0.0) R.single_with_number(s, cr, an, o, j, y);
            }
          } else {
            const int i0 = lab & 0xff, j0 = (lab >> 8) & 0xff, a0 = (lab >> 16) & 0xff,
                      b0 = (lab >> 24) & 0xff;
            const double x = double_sign(I, i0, j0, a0, b0) * T0[e];
            // <c+_{i0} c+_{j0} c_{b0} c_{a0}> = sign, and the three reorderings
            R.G(s, s, i0, j0, a0, b0) += x;
            R.G(s, s, j0, i0, b0, a0) += x;
            R.G(s, s, i0, j0, b0, a0) -= x;
            R.G(s, s, j0, i0, a0, b0) -= x;
          }
        }
      }
      return SBD_TPB_OK;
    };
    int rc = SBD_TPB_OK;
    if ((rc = run_pairs(0, W, na, nb, h->ta_s, as, h->d_bstr, true)) == SBD_TPB_OK &&
        (rc = run_pairs(0, W, na, nb, h->ta_d, ad, h->d_bstr, false)) == SBD_TPB_OK &&
        (rc = run_pairs(1, d_WT, nb, na, h->tb_s, bs, h->d_astr, true)) == SBD_TPB_OK &&
        (rc = run_pairs(1, d_WT, nb, na, h->tb_d, bd, h->d_astr, false)) == SBD_TPB_OK) {
    }
    cudaFree(d_WT);
    cudaFree(d_T0);
    cudaFree(d_Tq);
    TPB_CHECK(rc);

    // alpha single x beta single
    if (h->ta_s.nnz && h->tb_s.nnz) {
      const int L2 = L * L;
      std::vector<uint32_t> abra(h->ta_s.nnz), bbra(h->tb_s.nnz);
      std::vector<int32_t> blab(h->tb_s.nnz);
      for (uint32_t i = 0; i < na; i++)
        for (uint32_t e = as.off[i]; e < as.off[i + 1]; e++) abra[e] = i;
      for (uint32_t i = 0; i < nb; i++)
        for (uint32_t e = bs.off[i]; e < bs.off[i + 1]; e++) {
          bbra[e] = i;
          const int cr = bs.lab[e] & 0xff, an = (bs.lab[e] >> 8) & 0xff;
          const int rs = cr * L + an + 1;
          blab[e] = single_sign(h->bstr[i], cr, an) > 0 ? rs : -rs;
        }
      uint32_t *d_abra = nullptr, *d_bbra = nullptr;
      int32_t *d_blab = nullptr;
      double *d_X = nullptr;
      TPB_CUDA(cudaMalloc(&d_abra, sizeof(uint32_t) * abra.size()));
      TPB_CUDA(cudaMalloc(&d_bbra, sizeof(uint32_t) * bbra.size()));
      TPB_CUDA(cudaMalloc(&d_blab, sizeof(int32_t) * blab.size()));
      TPB_CUDA(cudaMalloc(&d_X, sizeof(double) * h->ta_s.nnz * L2));
      TPB_CUDA(cudaMemcpy(d_abra, abra.data(), sizeof(uint32_t) * abra.size(), cudaMemcpyHostToDevice));
      TPB_CUDA(cudaMemcpy(d_bbra, bbra.data(), sizeof(uint32_t) * bbra.size(), cudaMemcpyHostToDevice));
      TPB_CUDA(cudaMemcpy(d_blab, blab.data(), sizeof(int32_t) * blab.size(), cudaMemcpyHostToDevice));
      rdm_mixed_kernel<<<(unsigned)h->ta_s.nnz, kRdmThreads, sizeof(double) * L2, h->stream>>>(
          W, nb, d_abra, h->ta_s.ket, d_bbra, h->tb_s.ket, d_blab, (uint32_t)h->tb_s.nnz, L2, d_X);
      TPB_LAUNCHED(h);
      std::vector<double> X(h->ta_s.nnz * (size_t)L2);
      TPB_CUDA(cudaMemcpyAsync(X.data(), d_X, sizeof(double) * X.size(), cudaMemcpyDeviceToHost, h->stream));
      TPB_CUDA(cudaStreamSynchronize(h->stream));
      cudaFree(d_abra);
      cudaFree(d_bbra);
      cudaFree(d_blab);
      cudaFree(d_X);
      for (uint32_t i = 0; i < na; i++)
        for (uint32_t e = as.off[i]; e < as.off[i + 1]; e++) {
          const int cra = as.lab[e] & 0xff, ana = (as.lab[e] >> 8) & 0xff;
          const double sa = single_sign(h->astr[i], cra, ana);
          const double *xr = X.data() + (size_t)e * L2;
          for (int rs = 0; rs < L2; rs++) {
            if (xr[rs] == 0.0) continue;
            const int crb = rs / L, anb = rs % L;
            const double x = sa * xr[rs];
            // placement of TwoDiffCorrelation for an alpha-single x beta-single pair
            // (basic/correlation.h:191-231): spin-orbitals ordered I<J (bra), A<B (ket); the
            // value is the separated-convention sign sa*sb times W_bra W_ket in either branch
            const int i = 2 * cra, j = 2 * crb + 1, a = 2 * ana, b = 2 * anb + 1;
            const int I = std::min(i, j), J = std::max(i, j), A = std::min(a, b), B = std::max(a, b);
            const int oi = I / 2, si = I % 2, oj = J / 2, sj = J % 2, oa = A / 2, sa_ = A % 2,
                      ob = B / 2;
            if (si == sa_) {
              R.G(si, sj, oa, ob, oi, oj) += x;
              R.G(sj, si, ob, oa, oj, oi) += x;
            } else {
              R.G(si, sj, oa, ob, oj, oi) += x;
              R.G(sj, si, ob, oa, oi, oj) += x;
            }
          }
        }
    }
  }
  if (one) std::memcpy(one, R.one.data(), sizeof(double) * R.one.size());
  if (two) std::memcpy(two, R.two.data(), sizeof(double) * R.two.size());
  if (density)
    for (int p = 0; p < L; p++) {
      density[2 * p] = R.g(0, p, p);
      density[2 * p + 1] = R.g(1, p, p);
    }
  return SBD_TPB_OK;
}

}  // namespace sbdtpb
