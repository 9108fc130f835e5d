// Carry-over strings of a CI vector: the step after the solver in the sample-based loop
// (tpb/sbdiag.h:690-736).
//
//   type 1  dominant strings: per-string weights w_a[Ia] = sum_Ib W^2, w_b[Ib] = sum_Ia W^2
//           (DiagonalAdet/BdetReducedDensityMatrix, tpb/rdmat.h:11-61, 138-188), strings by
//           descending weight, kept up to the running weight 1 - threshold or the first
//           floor(ratio * n) (CarryOverAdet/Bdet, tpb/rdmat.h:63-135, 190-262);
//   type 2  type 1 followed by every single excitation of the kept strings, sorted and unique
//           (SinglesExtendHalfdets, tpb/extend.h:186-320);
//   type 3  the strings of determinants with W^2 > threshold and their singles, sorted and
//           unique, with the total weight of those determinants (tpb/extend.h:13-177).
//
// One pass over W in HBM gives both spins' weights (or counts): CTAs own contiguous row bands,
// a thread owns two columns of a 512-column chunk and walks the band's rows, so a warp reads
// 256 contiguous bytes per load; row sums go through warp shuffles into per-warp slots in shared
// memory, column sums into one partial row per CTA that a second kernel adds up.  Every sum is
// taken in a fixed order, so results do not change from run to run.  Sorting, scans and
// compaction of the (small) per-string arrays use CUB.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "tpb_common.cuh"

namespace sbdtpb {
namespace {

constexpr int kCoThreads = 256;
constexpr int kCoWarps = kCoThreads / 32;
constexpr int kCoChunk = 2 * kCoThreads;  // columns per chunk
constexpr int kCoBand = 256;              // most rows a CTA holds row partials for at once

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ uint32_t warp_sum(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// COUNT = false: row and column sums of W^2.  COUNT = true: row and column counts of entries with
// W^2 > cutoff and the sum of those entries.  CTA b owns rows [r0, r1) of W (na x nb, row-major)
// and writes its column partials to colw/colc[b][nb] and, for COUNT, its total to tot[b].
template <bool COUNT>
__global__ void __launch_bounds__(kCoThreads) string_weights_kernel(const double *__restrict__ W,
                                                                    size_t na, size_t nb, int nbands,
                                                                    double cutoff, double *__restrict__ roww,
                                                                    uint32_t *__restrict__ rowc,
                                                                    double *__restrict__ colw,
                                                                    uint32_t *__restrict__ colc,
                                                                    double *__restrict__ tot) {
  __shared__ double sw[kCoBand][kCoWarps];
  __shared__ uint32_t sc[kCoBand][kCoWarps];
  __shared__ double stot[kCoWarps];
  const int b = blockIdx.x;
  const size_t r0 = na * (size_t)b / nbands, r1 = na * (size_t)(b + 1) / nbands;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double my_tot = 0.0;
  for (size_t s0 = r0; s0 < r1; s0 += kCoBand) {
    const int nr = (int)std::min<size_t>(kCoBand, r1 - s0);
    for (int i = threadIdx.x; i < nr * kCoWarps; i += kCoThreads) {
      (&sw[0][0])[i] = 0.0;
      (&sc[0][0])[i] = 0u;
    }
    __syncthreads();
    for (size_t c0 = 0; c0 < nb; c0 += kCoChunk) {
      const size_t ca = c0 + threadIdx.x, cb = ca + kCoThreads;
      const bool va = ca < nb, vb = cb < nb;
      double wa = 0.0, wb = 0.0;
      uint32_t na_ = 0, nb_ = 0;
      const double *row = W + s0 * nb;
      int r = 0;
      // four rows per step: eight independent loads in flight per thread
      for (; r + 4 <= nr; r += 4) {
        double x[4], y[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const double *p = row + (size_t)(r + u) * nb;
          x[u] = va ? __ldcs(p + ca) : 0.0;
          y[u] = vb ? __ldcs(p + cb) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const double xa = x[u] * x[u], xb = y[u] * y[u];
          if (COUNT) {
            const uint32_t ka = (va && xa > cutoff) ? 1u : 0u, kb = (vb && xb > cutoff) ? 1u : 0u;
            na_ += ka;
            nb_ += kb;
            if (ka) my_tot += xa;
            if (kb) my_tot += xb;
            const uint32_t rc = warp_sum(ka + kb);
            if (lane == 0) sc[r + u][warp] += rc;
          } else {
            wa += xa;
            wb += xb;
            const double rs = warp_sum(xa + xb);
            if (lane == 0) sw[r + u][warp] += rs;
          }
        }
      }
      for (; r < nr; r++) {
        const double *p = row + (size_t)r * nb;
        const double x = va ? __ldcs(p + ca) : 0.0, y = vb ? __ldcs(p + cb) : 0.0;
        const double xa = x * x, xb = y * y;
        if (COUNT) {
          const uint32_t ka = (va && xa > cutoff) ? 1u : 0u, kb = (vb && xb > cutoff) ? 1u : 0u;
          na_ += ka;
          nb_ += kb;
          if (ka) my_tot += xa;
          if (kb) my_tot += xb;
          const uint32_t rc = warp_sum(ka + kb);
          if (lane == 0) sc[r][warp] += rc;
        } else {
          wa += xa;
          wb += xb;
          const double rs = warp_sum(xa + xb);
          if (lane == 0) sw[r][warp] += rs;
        }
      }
      // column partials of this CTA: the first row band writes, later bands add (same CTA, in order)
      const bool first = s0 == r0;
      if (COUNT) {
        uint32_t *pc = colc + (size_t)b * nb;
        if (va) pc[ca] = first ? na_ : pc[ca] + na_;
        if (vb) pc[cb] = first ? nb_ : pc[cb] + nb_;
      } else {
        double *pw = colw + (size_t)b * nb;
        if (va) pw[ca] = first ? wa : pw[ca] + wa;
        if (vb) pw[cb] = first ? wb : pw[cb] + wb;
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nr; i += kCoThreads) {
      if (COUNT) {
        uint32_t c = 0;
#pragma unroll
        for (int w = 0; w < kCoWarps; w++) c += sc[i][w];
        rowc[s0 + i] = c;
      } else {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kCoWarps; w++) s += sw[i][w];
        roww[s0 + i] = s;
      }
    }
    __syncthreads();
  }
  if (COUNT) {
    my_tot = warp_sum(my_tot);
    if (lane == 0) stot[warp] = my_tot;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kCoWarps; w++) t += stot[w];
      tot[b] = t;
    }
  }
}

// column j: sum of the nbands CTA partials.  A CTA covers 32 columns with 8 band groups; thread
// (g, j) adds bands g, g+8, ... into four accumulators (four independent loads in flight), the
// groups are then added in group order, so the result is the same on every run.  Block 0 also
// adds the per-CTA totals the same way.
template <bool COUNT>
__global__ void __launch_bounds__(256) column_reduce_kernel(size_t nb, int nbands, const double *__restrict__ colw,
                                                            const uint32_t *__restrict__ colc,
                                                            const double *__restrict__ tot, double *__restrict__ wb,
                                                            uint32_t *__restrict__ cb, double *__restrict__ total) {
  __shared__ double sv[8][33];
  __shared__ uint32_t sn[8][33];
  const int cx = threadIdx.x & 31, g = threadIdx.x >> 5;
  const size_t j = (size_t)blockIdx.x * 32 + cx;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  uint32_t c[4] = {0u, 0u, 0u, 0u};
  if (j < nb) {
    int b = g;
    for (; b + 24 < nbands; b += 32) {
#pragma unroll
      for (int u = 0; u < 4; u++) {
        if (COUNT) c[u] += colc[(size_t)(b + 8 * u) * nb + j];
        else s[u] += colw[(size_t)(b + 8 * u) * nb + j];
      }
    }
    for (; b < nbands; b += 8) {
      if (COUNT) c[0] += colc[(size_t)b * nb + j];
      else s[0] += colw[(size_t)b * nb + j];
    }
  }
  sv[g][cx] = (s[0] + s[1]) + (s[2] + s[3]);
  sn[g][cx] = (c[0] + c[1]) + (c[2] + c[3]);
  __syncthreads();
  if (g == 0 && j < nb) {
    if (COUNT) {
      uint32_t t = 0;
      for (int k = 0; k < 8; k++) t += sn[k][cx];
      cb[j] = t;
    } else {
      double t = 0.0;
      for (int k = 0; k < 8; k++) t += sv[k][cx];
      wb[j] = t;
    }
  }
  if (COUNT && blockIdx.x == 0) {
    __syncthreads();
    double t = 0.0;
    for (int b = threadIdx.x; b < nbands; b += 256) t += tot[b];
    sv[g][cx] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0;
      for (int k = 0; k < 8; k++)
        for (int x = 0; x < 32; x++) a += sv[k][x];
      *total = a;
    }
  }
}

// sort keys: weights are >= 0, so the bit pattern is monotone and its complement sorts by
// descending weight; the stable radix sort keeps equal weights in ascending string order
__global__ void weight_keys_kernel(const double *__restrict__ w, size_t n, uint64_t *__restrict__ key,
                                   uint32_t *__restrict__ idx) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    key[i] = ~(uint64_t)__double_as_longlong(w[i]);
    idx[i] = (uint32_t)i;
  }
}

__global__ void weights_from_keys_kernel(const uint64_t *__restrict__ key, size_t n, double *__restrict__ w) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) w[i] = __longlong_as_double((long long)~key[i]);
}

// kept strings: ratio > 0 -> floor(ratio * n); else 1 + #(running weight <= 1 - threshold),
// at most n (running sums are non-decreasing, so a binary search finds the count)
__global__ void kept_count_kernel(const double *__restrict__ S, size_t n, double ratio, double threshold,
                                  unsigned long long *__restrict__ kept, double *__restrict__ truncated) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (ratio > 0.0) {
    size_t k = (size_t)(ratio * (double)n);
    if (k > n) k = n;
    *kept = k;
    *truncated = 1.0 - (k ? S[k - 1] : 0.0);
    return;
  }
  const double target = 1.0 - threshold;
  size_t lo = 0, hi = n;  // first index with S > target
  while (lo < hi) {
    const size_t mid = (lo + hi) >> 1;
    if (S[mid] <= target) lo = mid + 1;
    else hi = mid;
  }
  *kept = lo + 1 < n ? lo + 1 : n;
  *truncated = 0.0;
}

__global__ void gather_strings_kernel(const uint64_t *__restrict__ str, const uint32_t *__restrict__ order,
                                      size_t n, uint64_t *__restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = str[order[i]];
}

__global__ void flag_counts_kernel(const uint32_t *__restrict__ c, size_t n, uint8_t *__restrict__ f) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) f[i] = c[i] > 0 ? 1 : 0;
}

// position of the k-th (0-based) set bit of x
__device__ __forceinline__ int nth_set_bit(uint64_t x, int k) {
  const uint32_t lo = (uint32_t)x;
  const int nlo = __popc(lo);
  if (k < nlo) return __fns(lo, 0, k + 1);
  return 32 + __fns((uint32_t)(x >> 32), 0, k - nlo + 1);
}

// string i and its singles: slot 0 = the string, slot 1 + j*(L-e) + k = closed orbital j
// (ascending) moved to open orbital k (ascending), as single_from_hdet (basic/excitation.h:9-29)
__global__ void singles_extend_kernel(const uint64_t *__restrict__ s, size_t n, int L, int e,
                                      uint64_t *__restrict__ out) {
  const size_t per = 1 + (size_t)e * (L - e);
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * per) return;
  const size_t i = t / per;
  const int r = (int)(t - i * per);
  const uint64_t x = s[i];
  if (r == 0) {
    out[t] = x;
    return;
  }
  const int j = (r - 1) / (L - e), k = (r - 1) - j * (L - e);
  const uint64_t full = (L == 64) ? ~0ull : ((1ull << L) - 1ull);
  const int pc = nth_set_bit(x, j), po = nth_set_bit(~x & full, k);
  out[t] = (x & ~(1ull << pc)) | (1ull << po);
}

inline unsigned grid_for(size_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// device buffers from the handle's pool, returned to it on scope exit (repeated calls of the same
// size allocate nothing)
struct Scratch {
  sbd_tpb_handle *h;
  std::vector<std::pair<void *, size_t>> got;
  explicit Scratch(sbd_tpb_handle *hh) : h(hh) {}
  ~Scratch() {
    for (auto &g : got) pool_put(h, g.first, g.second);
  }
  template <typename T>
  int get(T **out, size_t count) {
    *out = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    void *p = nullptr;
    TPB_CHECK(pool_get(h, bytes, &p));
    got.emplace_back(p, bytes);
    *out = (T *)p;
    return SBD_TPB_OK;
  }
};

// per-string weights (COUNT = false) or counts above the cutoff and their total (COUNT = true)
template <bool COUNT>
int string_weights(sbd_tpb_handle *h, const double *dW, double cutoff, Scratch &sc, double *wa, double *wb,
                   uint32_t *ca, uint32_t *cb, double *total) {
  const size_t na = h->astr.size(), nb = h->bstr.size();
  // six CTAs of 256 threads fit an SM (40 registers a thread): one full wave
  const int nbands = (int)std::max<size_t>(1, std::min<size_t>(na, (size_t)h->num_sms * 6));
  double *colw = nullptr, *tot = nullptr;
  uint32_t *colc = nullptr;
  if (COUNT) {
    TPB_CHECK(sc.get(&colc, (size_t)nbands * nb));
    TPB_CHECK(sc.get(&tot, (size_t)nbands));
  } else {
    TPB_CHECK(sc.get(&colw, (size_t)nbands * nb));
  }
  // timed from here: the scratch above is allocated before the first event
  TPB_CUDA(cudaEventRecord(h->ev_co[0], h->stream));
  string_weights_kernel<COUNT><<<nbands, kCoThreads, 0, h->stream>>>(dW, na, nb, nbands, cutoff, wa, ca, colw,
                                                                      colc, tot);
  TPB_LAUNCHED(h);
  column_reduce_kernel<COUNT><<<grid_for(nb, 32), 256, 0, h->stream>>>(nb, nbands, colw, colc, tot, wb, cb,
                                                                        total);
  TPB_LAUNCHED(h);
  TPB_CUDA(cudaEventRecord(h->ev_co[1], h->stream));
  return SBD_TPB_OK;
}

// dominant strings of one spin: order by descending weight, kept count, truncated weight
int select_dominant(sbd_tpb_handle *h, const double *w, const uint64_t *dstr, size_t n, double ratio,
                    double threshold, Scratch &sc, uint64_t **kept_str, size_t *kept, double *truncated) {
  uint64_t *key = nullptr, *key_s = nullptr, *out = nullptr;
  uint32_t *idx = nullptr, *idx_s = nullptr;
  double *ws = nullptr, *S = nullptr, *dtr = nullptr;
  unsigned long long *dk = nullptr;
  TPB_CHECK(sc.get(&key, n));
  TPB_CHECK(sc.get(&key_s, n));
  TPB_CHECK(sc.get(&idx, n));
  TPB_CHECK(sc.get(&idx_s, n));
  TPB_CHECK(sc.get(&ws, n));
  TPB_CHECK(sc.get(&S, n));
  TPB_CHECK(sc.get(&dk, 1));
  TPB_CHECK(sc.get(&dtr, 1));
  TPB_CHECK(sc.get(&out, n));
  weight_keys_kernel<<<grid_for(n, 256), 256, 0, h->stream>>>(w, n, key, idx);
  TPB_LAUNCHED(h);
  size_t tmp_bytes = 0, scan_bytes = 0;
  TPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key, key_s, idx, idx_s, (int)n, 0, 64, h->stream));
  TPB_CUDA(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, ws, S, (int)n, h->stream));
  void *tmp = nullptr;
  TPB_CHECK(sc.get((uint8_t **)&tmp, std::max(tmp_bytes, scan_bytes)));
  TPB_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, key, key_s, idx, idx_s, (int)n, 0, 64, h->stream));
  weights_from_keys_kernel<<<grid_for(n, 256), 256, 0, h->stream>>>(key_s, n, ws);
  TPB_LAUNCHED(h);
  TPB_CUDA(cub::DeviceScan::InclusiveSum(tmp, scan_bytes, ws, S, (int)n, h->stream));
  kept_count_kernel<<<1, 32, 0, h->stream>>>(S, n, ratio, threshold, dk, dtr);
  TPB_LAUNCHED(h);
  gather_strings_kernel<<<grid_for(n, 256), 256, 0, h->stream>>>(dstr, idx_s, n, out);
  TPB_LAUNCHED(h);
  unsigned long long k = 0;
  TPB_CUDA(cudaMemcpyAsync(&k, dk, sizeof(k), cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaMemcpyAsync(truncated, dtr, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  *kept = (size_t)k;
  *kept_str = out;
  return SBD_TPB_OK;
}

// s (device, n strings of e electrons) and their singles, sorted ascending and unique
int singles_extend(sbd_tpb_handle *h, const uint64_t *s, size_t n, int e, Scratch &sc, uint64_t **res,
                   size_t *count) {
  const int L = h->L;
  const size_t m = n * (1 + (size_t)e * (L - e));
  if (m > (size_t)INT32_MAX) return fail(SBD_TPB_ERR_INVALID, "carry-over: too many extended strings");
  *res = nullptr;
  *count = 0;
  if (m == 0) return SBD_TPB_OK;
  uint64_t *cand = nullptr, *sorted = nullptr, *uniq = nullptr;
  int *dnum = nullptr;
  TPB_CHECK(sc.get(&cand, m));
  TPB_CHECK(sc.get(&sorted, m));
  TPB_CHECK(sc.get(&uniq, m));
  TPB_CHECK(sc.get(&dnum, 1));
  singles_extend_kernel<<<grid_for(m, 256), 256, 0, h->stream>>>(s, n, L, e, cand);
  TPB_LAUNCHED(h);
  size_t b1 = 0, b2 = 0;
  TPB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, b1, cand, sorted, (int)m, 0, L, h->stream));
  TPB_CUDA(cub::DeviceSelect::Unique(nullptr, b2, sorted, uniq, dnum, (int)m, h->stream));
  void *tmp = nullptr;
  TPB_CHECK(sc.get((uint8_t **)&tmp, std::max(b1, b2)));
  TPB_CUDA(cub::DeviceRadixSort::SortKeys(tmp, b1, cand, sorted, (int)m, 0, L, h->stream));
  TPB_CUDA(cub::DeviceSelect::Unique(tmp, b2, sorted, uniq, dnum, (int)m, h->stream));
  int u = 0;
  TPB_CUDA(cudaMemcpyAsync(&u, dnum, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  *res = uniq;
  *count = (size_t)u;
  return SBD_TPB_OK;
}

// strings whose count is > 0, in string order
int select_counted(sbd_tpb_handle *h, const uint32_t *c, const uint64_t *dstr, size_t n, Scratch &sc,
                   uint64_t **res, size_t *count) {
  uint8_t *f = nullptr;
  uint64_t *out = nullptr;
  int *dnum = nullptr;
  TPB_CHECK(sc.get(&f, n));
  TPB_CHECK(sc.get(&out, n));
  TPB_CHECK(sc.get(&dnum, 1));
  flag_counts_kernel<<<grid_for(n, 256), 256, 0, h->stream>>>(c, n, f);
  TPB_LAUNCHED(h);
  size_t b = 0;
  TPB_CUDA(cub::DeviceSelect::Flagged(nullptr, b, dstr, f, out, dnum, (int)n, h->stream));
  void *tmp = nullptr;
  TPB_CHECK(sc.get((uint8_t **)&tmp, b));
  TPB_CUDA(cub::DeviceSelect::Flagged(tmp, b, dstr, f, out, dnum, (int)n, h->stream));
  int u = 0;
  TPB_CUDA(cudaMemcpyAsync(&u, dnum, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  *res = out;
  *count = (size_t)u;
  return SBD_TPB_OK;
}

// copies n device strings into the caller's buffer when it holds them all
int deliver(sbd_tpb_handle *h, const uint64_t *d, size_t n, uint64_t *buf, size_t cap, size_t *count,
            bool *short_buf) {
  *count = n;
  if (!buf || cap < n) {
    *short_buf = true;
    return SBD_TPB_OK;
  }
  if (n) TPB_CUDA(cudaMemcpyAsync(buf, d, n * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
  return SBD_TPB_OK;
}

}  // namespace

int carryover_device(sbd_tpb_handle *h, const double *dW, sbd_tpb_carryover *co) {
  if (co->type < 1 || co->type > 3) return fail(SBD_TPB_ERR_INVALID, "carry-over: type must be 1, 2 or 3");
  if (!(co->ratio >= 0.0) || !std::isfinite(co->threshold))
    return fail(SBD_TPB_ERR_INVALID, "carry-over: ratio must be >= 0 and the threshold finite");
  const size_t na = h->astr.size(), nb = h->bstr.size();
  if (na > (size_t)INT32_MAX || nb > (size_t)INT32_MAX)
    return fail(SBD_TPB_ERR_INVALID, "carry-over: more than 2^31 strings of one spin");
  const auto t0 = std::chrono::steady_clock::now();
  Scratch sc(h);
  co->truncated_a = co->truncated_b = 0.0;
  co->total_weight = 0.0;
  uint64_t *ra = nullptr, *rb = nullptr;
  size_t nra = 0, nrb = 0;
  if (co->type == 1 || co->type == 2) {
    double *wa = nullptr, *wb = nullptr;
    TPB_CHECK(sc.get(&wa, na));
    TPB_CHECK(sc.get(&wb, nb));
    TPB_CHECK(string_weights<false>(h, dW, 0.0, sc, wa, wb, nullptr, nullptr, nullptr));
    TPB_CHECK(select_dominant(h, wa, h->d_astr, na, co->ratio, co->threshold, sc, &ra, &nra, &co->truncated_a));
    TPB_CHECK(select_dominant(h, wb, h->d_bstr, nb, co->ratio, co->threshold, sc, &rb, &nrb, &co->truncated_b));
  } else {
    uint32_t *ca = nullptr, *cb = nullptr;
    double *tot = nullptr;
    TPB_CHECK(sc.get(&ca, na));
    TPB_CHECK(sc.get(&cb, nb));
    TPB_CHECK(sc.get(&tot, 1));
    TPB_CHECK(string_weights<true>(h, dW, co->threshold, sc, nullptr, nullptr, ca, cb, tot));
    TPB_CUDA(cudaMemcpyAsync(&co->total_weight, tot, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TPB_CHECK(select_counted(h, ca, h->d_astr, na, sc, &ra, &nra));
    TPB_CHECK(select_counted(h, cb, h->d_bstr, nb, sc, &rb, &nrb));
  }
  if (co->type == 2 || co->type == 3) {
    uint64_t *xa = nullptr, *xb = nullptr;
    size_t nxa = 0, nxb = 0;
    TPB_CHECK(singles_extend(h, ra, nra, h->n_alpha, sc, &xa, &nxa));
    TPB_CHECK(singles_extend(h, rb, nrb, h->n_beta, sc, &xb, &nxb));
    ra = xa, nra = nxa, rb = xb, nrb = nxb;
  }
  bool short_buf = false;
  TPB_CHECK(deliver(h, ra, nra, co->astr, co->acap, &co->na, &short_buf));
  TPB_CHECK(deliver(h, rb, nrb, co->bstr, co->bcap, &co->nb, &short_buf));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  TPB_CUDA(cudaEventElapsedTime(&h->last_carryover_ms[0], h->ev_co[0], h->ev_co[1]));
  h->last_carryover_ms[1] =
      (float)(1e3 * std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
  if (short_buf)
    return fail(SBD_TPB_ERR_CAPACITY, "carry-over: output buffer missing or too small (counts returned in na/nb)");
  return SBD_TPB_OK;
}

}  // namespace sbdtpb
