// Excitation tables on the GPU.
//
// Replaces the host-side GenerateExcitation of the reference (tpb/helper.h:185-323): for every
// bra string, the ket strings at XOR-popcount 2 (singles) or 4 (doubles), ket index ascending,
// with labels cr = bra \ ket and an = ket \ bra ascending (OrbitalDifference,
// basic/determinants.h:386-432).  One warp owns one bra string and sweeps all ket strings 32 at
// a time; a warp ballot assigns output slots so the ket order of the reference is kept exactly.
// Two passes: count (both kinds at once), exclusive scan, fill.
#include <cstdio>

#include "tpb_common.cuh"

namespace sbdtpb {
namespace {

constexpr int kWarpsPerBlock = 8;

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    ex_count_kernel(const uint64_t *__restrict__ s, uint32_t n, uint64_t mask,
                    uint32_t *__restrict__ cnt_s, uint32_t *__restrict__ cnt_d) {
  const uint32_t warp = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const uint64_t bra = s[warp];
  uint32_t cs = 0, cd = 0;
  for (uint32_t j = lane; j < n; j += 32) {
    const int d = __popcll((bra ^ __ldg(&s[j])) & mask);
    cs += (d == 2);
    cd += (d == 4);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cs += __shfl_xor_sync(0xffffffffu, cs, o);
    cd += __shfl_xor_sync(0xffffffffu, cd, o);
  }
  if (lane == 0) {
    cnt_s[warp] = cs;
    cnt_d[warp] = cd;
  }
}

// Exclusive scan of n counts into off[0..n] (off[n] = total) by one block; the totals of this
// path are at most a few million, so a single pass over chunks is enough.  Overflow of the
// 32-bit total is reported through *overflow.
__global__ void __launch_bounds__(1024)
    scan_kernel(const uint32_t *__restrict__ cnt, uint32_t n, uint32_t *__restrict__ off,
                int *__restrict__ overflow) {
  __shared__ unsigned long long warp_sums[32];
  __shared__ unsigned long long carry;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < n; base += 1024) {
    const uint32_t i = base + tid;
    unsigned long long v = (i < n) ? cnt[i] : 0ull;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
      unsigned long long w = warp_sums[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    const unsigned long long before = carry + (wid ? warp_sums[wid - 1] : 0ull) + x - v;
    if (i < n) {
      off[i] = (uint32_t)before;
      if (before > 0xffffffffull) *overflow = 1;
    }
    __syncthreads();
    if (tid == 1023) carry = before + v;
    __syncthreads();
  }
  if (tid == 0) {
    off[n] = (uint32_t)carry;
    if (carry > 0xffffffffull) *overflow = 1;
  }
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    ex_fill_kernel(const uint64_t *__restrict__ s, uint32_t n, uint64_t mask,
                   const uint32_t *__restrict__ off_s, uint32_t *__restrict__ ket_s,
                   uint32_t *__restrict__ lab_s, const uint32_t *__restrict__ off_d,
                   uint32_t *__restrict__ ket_d, uint32_t *__restrict__ lab_d) {
  const uint32_t warp = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const uint64_t bra = s[warp] & mask;
  uint32_t ws = off_s[warp], wd = off_d[warp];
  const uint32_t lt = (1u << lane) - 1u;
  for (uint32_t base = 0; base < n; base += 32) {
    const uint32_t j = base + lane;
    const uint64_t ket = (j < n) ? (__ldg(&s[j]) & mask) : bra;
    const int d = __popcll(bra ^ ket);
    const uint32_t bs = __ballot_sync(0xffffffffu, d == 2);
    const uint32_t bd = __ballot_sync(0xffffffffu, d == 4);
    const uint64_t cr = bra & ~ket, an = ket & ~bra;
    if (d == 2) {
      const uint32_t pos = ws + __popc(bs & lt);
      ket_s[pos] = j;
      lab_s[pos] = (uint32_t)lowest_bit(cr) | ((uint32_t)lowest_bit(an) << 8);
    } else if (d == 4) {
      const uint32_t pos = wd + __popc(bd & lt);
      ket_d[pos] = j;
      lab_d[pos] = (uint32_t)lowest_bit(cr) | ((uint32_t)highest_bit(cr) << 8) |
                   ((uint32_t)lowest_bit(an) << 16) | ((uint32_t)highest_bit(an) << 24);
    }
    ws += __popc(bs);
    wd += __popc(bd);
  }
}

void free_table(ExTable &t) {
  cudaFree(t.off);
  cudaFree(t.ket);
  cudaFree(t.lab);
  t = ExTable();
}

int build_spin(sbd_tpb_handle *h, const uint64_t *d_s, uint32_t n, ExTable &ts, ExTable &td) {
  free_table(ts);
  free_table(td);
  const uint64_t mask = h->L >= 64 ? ~0ull : ((1ull << h->L) - 1ull);
  uint32_t *cnt = nullptr;
  int *d_over = nullptr;
  TPB_CUDA(cudaMallocAsync(&cnt, sizeof(uint32_t) * 2 * (size_t)(n + 1), h->stream));
  TPB_CUDA(cudaMallocAsync(&d_over, sizeof(int), h->stream));
  TPB_CUDA(cudaMemsetAsync(d_over, 0, sizeof(int), h->stream));
  TPB_CUDA(cudaMallocAsync(&ts.off, sizeof(uint32_t) * (n + 1), h->stream));
  TPB_CUDA(cudaMallocAsync(&td.off, sizeof(uint32_t) * (n + 1), h->stream));
  const unsigned grid = (n + kWarpsPerBlock - 1) / kWarpsPerBlock;
  ex_count_kernel<<<grid, kWarpsPerBlock * 32, 0, h->stream>>>(d_s, n, mask, cnt, cnt + n + 1);
  TPB_LAUNCHED(h);
  scan_kernel<<<1, 1024, 0, h->stream>>>(cnt, n, ts.off, d_over);
  TPB_LAUNCHED(h);
  scan_kernel<<<1, 1024, 0, h->stream>>>(cnt + n + 1, n, td.off, d_over);
  TPB_LAUNCHED(h);
  uint32_t tot[2];
  int over = 0;
  TPB_CUDA(cudaMemcpyAsync(&tot[0], ts.off + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaMemcpyAsync(&tot[1], td.off + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaMemcpyAsync(&over, d_over, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  cudaFreeAsync(cnt, h->stream);
  cudaFreeAsync(d_over, h->stream);
  if (over) return fail(SBD_TPB_ERR_INVALID, "excitation table exceeds 2^32 entries");
  ts.nnz = tot[0];
  td.nnz = tot[1];
  TPB_CUDA(cudaMallocAsync(&ts.ket, sizeof(uint32_t) * (ts.nnz ? ts.nnz : 1), h->stream));
  TPB_CUDA(cudaMallocAsync(&ts.lab, sizeof(uint32_t) * (ts.nnz ? ts.nnz : 1), h->stream));
  TPB_CUDA(cudaMallocAsync(&td.ket, sizeof(uint32_t) * (td.nnz ? td.nnz : 1), h->stream));
  TPB_CUDA(cudaMallocAsync(&td.lab, sizeof(uint32_t) * (td.nnz ? td.nnz : 1), h->stream));
  ex_fill_kernel<<<grid, kWarpsPerBlock * 32, 0, h->stream>>>(d_s, n, mask, ts.off, ts.ket, ts.lab,
                                                               td.off, td.ket, td.lab);
  TPB_LAUNCHED(h);
  // longest rows, for the sigma kernels' shared-memory staging
  std::vector<uint32_t> o(n + 1);
  for (ExTable *t : {&ts, &td}) {
    TPB_CUDA(cudaMemcpyAsync(o.data(), t->off, sizeof(uint32_t) * (n + 1), cudaMemcpyDeviceToHost,
                             h->stream));
    TPB_CUDA(cudaStreamSynchronize(h->stream));
    uint32_t mx = 0;
    for (uint32_t i = 0; i < n; i++) mx = o[i + 1] - o[i] > mx ? o[i + 1] - o[i] : mx;
    t->max_row = mx;
  }
  return SBD_TPB_OK;
}

}  // namespace

int build_excitation_tables(sbd_tpb_handle *h) {
  TPB_CHECK(build_spin(h, h->d_astr, (uint32_t)h->astr.size(), h->ta_s, h->ta_d));
  TPB_CHECK(build_spin(h, h->d_bstr, (uint32_t)h->bstr.size(), h->tb_s, h->tb_d));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  return SBD_TPB_OK;
}

int copy_table_reference_layout(sbd_tpb_handle *h, int kind, uint64_t *off, uint64_t *ket,
                                int32_t *cran) {
  const ExTable *t = nullptr;
  size_t n = 0;
  int spin = 0, per = 2;
  switch (kind) {
    case SBD_TPB_SINGLES_ALPHA: t = &h->ta_s; n = h->astr.size(); break;
    case SBD_TPB_DOUBLES_ALPHA: t = &h->ta_d; n = h->astr.size(); per = 4; break;
    case SBD_TPB_SINGLES_BETA: t = &h->tb_s; n = h->bstr.size(); spin = 1; break;
    case SBD_TPB_DOUBLES_BETA: t = &h->tb_d; n = h->bstr.size(); spin = 1; per = 4; break;
    default: return fail(SBD_TPB_ERR_INVALID, "unknown table kind");
  }
  std::vector<uint32_t> o(n + 1), k(t->nnz), l(t->nnz);
  TPB_CUDA(cudaMemcpyAsync(o.data(), t->off, sizeof(uint32_t) * (n + 1), cudaMemcpyDeviceToHost, h->stream));
  if (t->nnz) {
    TPB_CUDA(cudaMemcpyAsync(k.data(), t->ket, sizeof(uint32_t) * t->nnz, cudaMemcpyDeviceToHost, h->stream));
    TPB_CUDA(cudaMemcpyAsync(l.data(), t->lab, sizeof(uint32_t) * t->nnz, cudaMemcpyDeviceToHost, h->stream));
  }
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  // TaskHelpers layout: CrAn = 2*orbital + spin (tpb/helper.h:242-243, 271-274, 287-288, 314-317)
  if (off)
    for (size_t i = 0; i <= n; i++) off[i] = o[i];
  for (size_t e = 0; e < t->nnz; e++) {
    if (ket) ket[e] = k[e];
    if (cran) {
      for (int q = 0; q < per; q++) cran[per * e + q] = 2 * (int32_t)((l[e] >> (8 * q)) & 0xff) + spin;
    }
  }
  return SBD_TPB_OK;
}

}  // namespace sbdtpb
