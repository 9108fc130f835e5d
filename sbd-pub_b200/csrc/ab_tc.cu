// Split-BF16 tcgen05 contraction for the dense alpha-beta path of the FP32 (mixed) sigma.
//
//   E[n][j] = sum_k V[n][k] D[j][k],  D ~ Dhi + Dlo,  V ~ Vhi + Vlo  (BF16 parts)
//   E ~ Dhi.Vhi + Dhi.Vlo + Dlo.Vhi   with FP32 accumulation in tensor memory.
//
// One persistent CTA per SM (128 threads).  The V operand (alpha labels x beta labels) stays in
// shared memory for the whole kernel; for each 128-row tile of D one thread issues a 1-D bulk
// copy (cp.async.bulk, completion on an mbarrier) of the hi and lo parts -- the gather kernel
// already wrote each tile in the canonical K-major, no-swizzle layout tcgen05.mma reads (8x8
// core matrices of 128 B; k-groups 2 KB apart) -- then issues 3 x Kp/16 tcgen05.mma
// (cta_group::1, kind::f16, M=128, N<=256 per instruction) into an FP32 accumulator in TMEM and
// commits to a second mbarrier; the four warps read their 32 accumulator lanes back with
// tcgen05.ld and store E label-major (coalesced along the determinant index).  Every mbarrier
// wait is bounded; on timeout the kernel records an error code, waits (bounded) for copies in
// flight, releases its TMEM and returns, and the host reports the failure.
#include <cuda_bf16.h>

#include <algorithm>
#include <string>
#include <vector>

#include "ab_tc.cuh"
#include "tc_util.cuh"

namespace sbdtpb {
namespace {

using namespace tc;

__host__ __device__ __forceinline__ size_t tiled_off(size_t j, int k, int Kp) { return a_off(j, k, Kp); }
__host__ __device__ __forceinline__ size_t tiled_off_b(int n, int k, int Np) { return b_off(n, (size_t)k, Np); }

// Shared memory: [Bhi Np*Kp][Blo Np*Kp][Ahi 128*Kp][Alo 128*Kp] (bf16) | mbar_load | mbar_mma |
// tmem base | status
__global__ void __launch_bounds__(128, 1)
    ab_tc_kernel(const __nv_bfloat16 *__restrict__ Ahi, const __nv_bfloat16 *__restrict__ Alo,
                 const __nv_bfloat16 *__restrict__ Bhi, const __nv_bfloat16 *__restrict__ Blo,
                 float *__restrict__ E, int Kp, int Np, int npq, size_t M, size_t ntiles,
                 int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const uint32_t b_bytes = (uint32_t)Np * Kp * 2, a_bytes = 128u * Kp * 2;
  unsigned char *sBhi = smem, *sBlo = smem + b_bytes, *sAhi = smem + 2 * b_bytes,
                *sAlo = smem + 2 * b_bytes + a_bytes;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * b_bytes + 2 * a_bytes);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2);
  volatile int *status = reinterpret_cast<volatile int *>(tmem_slot + 1);
  const uint32_t bar_load = smem_addr(&bars[0]), bar_mma = smem_addr(&bars[1]);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t ncols = 32;
  while ((int)ncols < Np) ncols <<= 1;

  if (threadIdx.x == 0) {
    mbar_init(bar_load, 1);
    mbar_init(bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    *status = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // idesc: D F32 (bits 4-5 = 1), A/B BF16 (bits 7-9, 10-12 = 1), K-major A/B, M = 128 (bits 24-28)
  uint32_t load_phase = 0, mma_phase = 0;
  if (threadIdx.x == 0) {
    mbar_expect_tx(bar_load, 2 * b_bytes);
    bulk_g2s(smem_addr(sBhi), Bhi, b_bytes, bar_load);
    bulk_g2s(smem_addr(sBlo), Blo, b_bytes, bar_load);
    if (!mbar_wait(bar_load, load_phase)) {
      atomicExch(err, 1);
      *status = 1;
      mbar_wait(bar_load, load_phase);  // bounded second wait for the copies in flight
    }
    load_phase ^= 1;
  }
  __syncthreads();

  const int NG = Np >> 3;
  for (size_t tile = blockIdx.x; tile < ntiles && *status == 0; tile += gridDim.x) {
    if (threadIdx.x == 0) {
      const size_t off = tile * (size_t)128 * Kp;
      mbar_expect_tx(bar_load, 2 * a_bytes);
      bulk_g2s(smem_addr(sAhi), Ahi + off, a_bytes, bar_load);
      bulk_g2s(smem_addr(sAlo), Alo + off, a_bytes, bar_load);
      bool ok = mbar_wait(bar_load, load_phase);
      load_phase ^= 1;
      if (!ok) {
        atomicExch(err, 2);
        *status = 1;
        mbar_wait(bar_load, load_phase ^ 1);
      } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_addr(sAhi), a1 = smem_addr(sAlo);
        const uint32_t b0 = smem_addr(sBhi), b1 = smem_addr(sBlo);
        for (int c = 0; c * 256 < Np; c++) {
          const int nc = min(256, Np - c * 256);
          const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nc >> 3) << 17) |
                                 ((uint32_t)(128 >> 4) << 24);
          const uint32_t td = tmem + (uint32_t)(c * 256);
          for (int s = 0; s < Kp / 16; s++) {
            const uint32_t aoff = (uint32_t)(2 * s) * 2048u;
            const uint32_t boff = (uint32_t)((2 * s) * NG + 32 * c) * 128u;
            const uint64_t dah = make_desc(a0 + aoff, 2048u, 128u);
            const uint64_t dal = make_desc(a1 + aoff, 2048u, 128u);
            const uint64_t dbh = make_desc(b0 + boff, (uint32_t)NG * 128u, 128u);
            const uint64_t dbl = make_desc(b1 + boff, (uint32_t)NG * 128u, 128u);
            mma_bf16(td, dah, dbh, idesc, s > 0 ? 1u : 0u);
            mma_bf16(td, dah, dbl, idesc, 1u);
            mma_bf16(td, dal, dbh, idesc, 1u);
          }
        }
        mma_commit(bar_mma);
        ok = mbar_wait(bar_mma, mma_phase);
        mma_phase ^= 1;
        if (!ok) {
          atomicExch(err, 3);
          *status = 1;
        }
      }
    }
    __syncthreads();
    if (*status != 0) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const size_t j = tile * 128 + (size_t)warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    for (int col = 0; col < Np; col += 16) {
      float v[16];
      tmem_ld16(trow + (uint32_t)col, v);
      if (j < M) {
#pragma unroll
        for (int i = 0; i < 16; i++)
          if (col + i < npq) E[(size_t)(col + i) * M + j] = v[i];
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

// Fused gather -> contraction: the A tiles are built in shared memory straight from C instead of
// being gathered to HBM first.  Warp roles of a persistent CTA (288 threads, one per SM):
//   warps 0-3  producers: thread r builds row r of the 128-row tile of determinants j = (Ja, Ib)
//              in stage s -- zeroes it, then writes the split-BF16 s_b C[Ja, Jb] of every beta
//              single Ib -> Jb (label rs) at column rs -- then fences the writes for the tensor
//              core's proxy and arrives on full[s];
//   warp 8     the MMA issuer: waits for full[s] and a free accumulator, issues 3 x Kp/16
//              tcgen05.mma into it, commits to empty[s] (stage reusable) and acc_full[a];
//   warps 4-7  the epilogue: wait acc_full[a], read their 32 TMEM lanes with tcgen05.ld, store E
//              label-major, arrive on acc_empty[a].
// NA A stages (2 when they fit beside the resident V operand, else 1) and two TMEM accumulators,
// so the gather of tile t+1, the MMAs of tile t and the write-out of tile t-1 overlap.  The MMA
// sequence and the hi/lo split are those of the unfused path, so E is the same.  Every wait is
// bounded; an expired one records a code, stops the CTA's loops, and the MMA warp drains its
// tensor-core work before TMEM is released.
constexpr int kFusedThreads = 288;

__global__ void __launch_bounds__(kFusedThreads, 1)
    ab_tc_fused_kernel(const float *__restrict__ C, uint32_t nb, const uint32_t *__restrict__ b_off,
                       const uint32_t *__restrict__ b_ket, const int32_t *__restrict__ b_label,
                       const __nv_bfloat16 *__restrict__ Bhi, const __nv_bfloat16 *__restrict__ Blo,
                       float *__restrict__ E, int Kp, int Np, int npq, size_t M, size_t ntiles, int NA,
                       int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const uint32_t b_bytes = (uint32_t)Np * Kp * 2, a_bytes = 128u * Kp * 2;
  unsigned char *sBhi = smem, *sBlo = smem + b_bytes, *sA = smem + 2 * b_bytes;  // stage s: hi, lo
  uint64_t *bars = reinterpret_cast<uint64_t *>(sA + (size_t)NA * 2 * a_bytes);
  // bars: [0,2) full, [2,4) empty, [4,6) acc_full, [6,8) acc_empty, 8 B loaded, 9 drain
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 10);
  volatile int *status = reinterpret_cast<volatile int *>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t ncols = 32;
  while ((int)ncols < Np) ncols <<= 1;
  auto bar = [&](int i) { return smem_addr(&bars[i]); };
  auto fail_with = [&](int code) {
    atomicExch(err, code);
    *status = 1;
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < 2; s++) {
      mbar_init(bar(s), 128);
      mbar_init(bar(2 + s), 1);
      mbar_init(bar(4 + s), 1);
      mbar_init(bar(6 + s), 128);
    }
    mbar_init(bar(8), 1);
    mbar_init(bar(9), 1);
    fence_mbar_init();
    *status = 0;
  }
  if (warp == 8) tmem_alloc(smem_addr(tmem_slot), 2 * ncols);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  if (warp < 4) {
    // ---------------- producers: build A tiles from C ----------------
    const int r = threadIdx.x;
    uint32_t it = 0;
    for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
      if (*status) break;
      const int s = (int)(it % (uint32_t)NA);
      const uint32_t ph = (it / (uint32_t)NA) & 1u;
      if (!mbar_wait(bar(2 + s), ph ^ 1u)) {
        fail_with(11);
        break;
      }
      unsigned char *hi = sA + (size_t)s * 2 * a_bytes, *lo = hi + a_bytes;
      // row r of the canonical K-major layout: 16 bytes in each k-group's core matrix r/8
      for (int g = 0; g < Kp / 8; g++) {
        const uint32_t o = (uint32_t)((g * 16 + (r >> 3)) << 7) + ((r & 7) << 4);
        *reinterpret_cast<uint4 *>(hi + o) = make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4 *>(lo + o) = make_uint4(0, 0, 0, 0);
      }
      const size_t j = tile * 128 + r;
      if (j < M) {
        const uint32_t ja = (uint32_t)(j / nb), ib = (uint32_t)(j - (size_t)ja * nb);
        const float *crow = C + (size_t)ja * nb;
        const uint32_t e1 = __ldg(&b_off[ib + 1]);
#pragma unroll 4
        for (uint32_t e = __ldg(&b_off[ib]); e < e1; e++) {
          const int32_t lab = __ldg(&b_label[e]);
          float x = __ldg(&crow[__ldg(&b_ket[e])]);
          if (lab < 0) x = -x;
          const __nv_bfloat16 xh = __float2bfloat16_rn(x);
          const __nv_bfloat16 xl = __float2bfloat16_rn(x - __bfloat162float(xh));
          const int k = (lab > 0 ? lab : -lab) - 1;
          const uint32_t o = (uint32_t)((((k >> 3) * 16 + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
          *reinterpret_cast<__nv_bfloat16 *>(hi + o) = xh;
          *reinterpret_cast<__nv_bfloat16 *>(lo + o) = xl;
        }
      }
      fence_proxy_async();
      mbar_arrive(bar(s));
    }
  } else if (warp < 8) {
    // ---------------- epilogue: TMEM -> E (label-major) ----------------
    const int q = threadIdx.x - 128, ew = q >> 5;
    uint32_t tc = 0;
    for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, tc++) {
      if (*status) break;
      const int a = (int)(tc & 1u);
      const uint32_t aph = (tc >> 1) & 1u;
      if (!mbar_wait(bar(4 + a), aph)) {
        fail_with(12);
        break;
      }
      fence_after_sync();
      const size_t j = tile * 128 + q;
      const uint32_t trow = tmem + (uint32_t)(a * (int)ncols) + ((uint32_t)(ew * 32) << 16);
      // the next 16 columns load from TMEM while this 16 go out to E
      uint32_t ra[16], rb[16];
      tmem_ld16_issue(trow, ra);
      tmem_ld_wait16(ra);
      for (int col = 0; col < Np; col += 16) {
        const bool more = col + 16 < Np;
        if (more) tmem_ld16_issue(trow + (uint32_t)(col + 16), rb);
        if (j < M) {
#pragma unroll
          for (int i = 0; i < 16; i++)
            if (col + i < npq) E[(size_t)(col + i) * M + j] = __uint_as_float(ra[i]);
        }
        if (more) {
          tmem_ld_wait16(rb);
#pragma unroll
          for (int i = 0; i < 16; i++) ra[i] = rb[i];
        }
      }
      fence_before_sync();
      mbar_arrive(bar(6 + a));
    }
  } else if (lane == 0) {
    // ---------------- MMA issuer ----------------
    mbar_expect_tx(bar(8), 2 * b_bytes);
    bulk_g2s(smem_addr(sBhi), Bhi, b_bytes, bar(8));
    bulk_g2s(smem_addr(sBlo), Blo, b_bytes, bar(8));
    bool ok = mbar_wait(bar(8), 0);
    if (!ok) {
      fail_with(13);
      mbar_wait(bar(8), 0);  // bounded second wait for the copies in flight
    }
    const int NG = Np >> 3;
    const uint32_t b0 = smem_addr(sBhi), b1 = smem_addr(sBlo);
    uint32_t it = 0;
    for (size_t tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x, it++) {
      if (*status) break;
      const int a = (int)(it & 1u);
      const uint32_t aph = (it >> 1) & 1u;
      const int s = (int)(it % (uint32_t)NA);
      const uint32_t ph = (it / (uint32_t)NA) & 1u;
      if (!mbar_wait(bar(6 + a), aph ^ 1u)) {
        fail_with(14);
        break;
      }
      if (!mbar_wait(bar(s), ph)) {
        fail_with(15);
        break;
      }
      fence_after_sync();
      const uint32_t a0 = smem_addr(sA + (size_t)s * 2 * a_bytes), a1 = a0 + a_bytes;
      for (int c = 0; c * 256 < Np; c++) {
        const int nc = min(256, Np - c * 256);
        const uint32_t idesc = idesc_bf16(nc);
        const uint32_t td = tmem + (uint32_t)(a * (int)ncols) + (uint32_t)(c * 256);
        for (int k16 = 0; k16 < Kp / 16; k16++) {
          const uint32_t aoff = (uint32_t)(2 * k16) * 2048u;
          const uint32_t boff = (uint32_t)((2 * k16) * NG + 32 * c) * 128u;
          const uint64_t dah = make_desc(a0 + aoff, 2048u, 128u);
          const uint64_t dal = make_desc(a1 + aoff, 2048u, 128u);
          const uint64_t dbh = make_desc(b0 + boff, (uint32_t)NG * 128u, 128u);
          const uint64_t dbl = make_desc(b1 + boff, (uint32_t)NG * 128u, 128u);
          mma_bf16(td, dah, dbh, idesc, k16 > 0 ? 1u : 0u);
          mma_bf16(td, dah, dbl, idesc, 1u);
          mma_bf16(td, dal, dbh, idesc, 1u);
        }
      }
      mma_commit(bar(2 + s));
      mma_commit(bar(4 + a));
    }
    // drain: every tensor-core operation this thread issued has completed before TMEM goes
    mma_commit(bar(9));
    if (!mbar_wait(bar(9), 0)) fail_with(16);
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 8) tmem_dealloc(tmem, 2 * ncols);
}

__global__ void ab_tc_gather_kernel(const float *__restrict__ C, uint32_t na, uint32_t nb,
                                    const uint32_t *__restrict__ b_off, const uint32_t *__restrict__ b_ket,
                                    const int32_t *__restrict__ b_label, int Kp,
                                    __nv_bfloat16 *__restrict__ Dhi, __nv_bfloat16 *__restrict__ Dlo) {
  const size_t total = (size_t)na * nb;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < total;
       j += (size_t)gridDim.x * blockDim.x) {
    const uint32_t ja = (uint32_t)(j / nb), ib = (uint32_t)(j - (size_t)ja * nb);
    const float *crow = C + (size_t)ja * nb;
    for (uint32_t e = b_off[ib]; e < b_off[ib + 1]; e++) {
      const int32_t lab = b_label[e];
      float x = crow[b_ket[e]];
      if (lab < 0) x = -x;
      const __nv_bfloat16 hi = __float2bfloat16_rn(x);
      const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
      const size_t o = tiled_off(j, (lab > 0 ? lab : -lab) - 1, Kp);
      Dhi[o] = hi;
      Dlo[o] = lo;
    }
  }
}

size_t fused_smem(int Kp, int Np, int na) {
  return (size_t)2 * Np * Kp * 2 + (size_t)na * 2 * 128 * Kp * 2 + 10 * 8 + 16;
}

}  // namespace

int ab_tc_setup(sbd_tpb_handle *h) {
  ABDense &ab = h->ab;
  ab.tc_ready = false;
  const int Kp = (ab.nrs + 15) / 16 * 16, Np = (ab.npq + 15) / 16 * 16;
  const size_t smem = (size_t)2 * Np * Kp * 2 + (size_t)2 * 128 * Kp * 2 + 64;
  if (Np > 512 || smem > h->smem_optin) return SBD_TPB_OK;  // CUDA-core contraction instead
  ab.Kp = Kp;
  ab.Np = Np;
  std::vector<double> V((size_t)ab.npq * ab.nrs);
  TPB_CUDA(cudaMemcpy(V.data(), ab.V, sizeof(double) * V.size(), cudaMemcpyDeviceToHost));
  std::vector<__nv_bfloat16> hi((size_t)Np * Kp, __float2bfloat16(0.f)), lo = hi;
  for (int n = 0; n < ab.npq; n++)
    for (int k = 0; k < ab.nrs; k++) {
      const float x = (float)V[(size_t)n * ab.nrs + k];
      const __nv_bfloat16 xh = __float2bfloat16_rn(x);
      hi[tiled_off_b(n, k, Np)] = xh;
      lo[tiled_off_b(n, k, Np)] = __float2bfloat16_rn(x - __bfloat162float(xh));
    }
  TPB_CUDA(cudaMalloc(&ab.Vhi, sizeof(uint16_t) * hi.size()));
  TPB_CUDA(cudaMalloc(&ab.Vlo, sizeof(uint16_t) * lo.size()));
  TPB_CUDA(cudaMemcpy(ab.Vhi, hi.data(), sizeof(uint16_t) * hi.size(), cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(ab.Vlo, lo.data(), sizeof(uint16_t) * lo.size(), cudaMemcpyHostToDevice));
  if (!ab.err) TPB_CUDA(cudaMalloc(&ab.err, sizeof(int)));
  TPB_CUDA(cudaMemset(ab.err, 0, sizeof(int)));
  TPB_CUDA(cudaFuncSetAttribute(ab_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // fused gather + contraction: two accumulators of up to 256 columns, V resident, one or two A stages
  ab.tc_fused_stages = 0;
  if (Np <= 256) {
    for (int na = 2; na >= 1; na--) {
      const size_t fs = fused_smem(Kp, Np, na);
      if (fs <= h->smem_optin) {
        TPB_CUDA(cudaFuncSetAttribute(ab_tc_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fs));
        ab.tc_fused_stages = na;
        break;
      }
    }
  }
  ab.tc_ready = true;
  return SBD_TPB_OK;
}

size_t ab_tc_work_bytes(sbd_tpb_handle *h) {
  const ABDense &ab = h->ab;
  const size_t M = h->ndet(), Mp = (M + 127) / 128 * 128;
  return Mp * ab.Kp * 2 * sizeof(uint16_t) + M * (size_t)ab.npq * sizeof(float);
}

size_t ab_tc_fused_work_bytes(sbd_tpb_handle *h) { return h->ndet() * (size_t)h->ab.npq * sizeof(float); }

int ab_tc_fused(sbd_tpb_handle *h, const float *C, float *E, size_t M) {
  ABDense &ab = h->ab;
  const size_t ntiles = (M + 127) / 128;
  const size_t smem = fused_smem(ab.Kp, ab.Np, ab.tc_fused_stages);
  const unsigned grid = (unsigned)std::min<size_t>(ntiles, (size_t)h->num_sms);
  ab_tc_fused_kernel<<<grid, kFusedThreads, smem, h->stream>>>(
      C, (uint32_t)h->bstr.size(), h->tb_s.off, h->tb_s.ket, ab.b_label,
      reinterpret_cast<const __nv_bfloat16 *>(ab.Vhi), reinterpret_cast<const __nv_bfloat16 *>(ab.Vlo), E, ab.Kp,
      ab.Np, ab.npq, M, ntiles, ab.tc_fused_stages, ab.err);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

int ab_tc_gather(sbd_tpb_handle *h, const float *C, size_t M) {
  ABDense &ab = h->ab;
  const size_t Mp = (M + 127) / 128 * 128;
  __nv_bfloat16 *Dhi = reinterpret_cast<__nv_bfloat16 *>(h->d_ab_work);
  __nv_bfloat16 *Dlo = Dhi + Mp * ab.Kp;
  TPB_CUDA(cudaMemsetAsync(Dhi, 0, sizeof(uint16_t) * Mp * ab.Kp * 2, h->stream));
  ab_tc_gather_kernel<<<h->num_sms * 8, 256, 0, h->stream>>>(
      C, (uint32_t)h->astr.size(), (uint32_t)h->bstr.size(), h->tb_s.off, h->tb_s.ket, ab.b_label,
      ab.Kp, Dhi, Dlo);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

int ab_tc_gemm(sbd_tpb_handle *h, const float *, float *E, size_t M) {
  ABDense &ab = h->ab;
  const size_t Mp = (M + 127) / 128 * 128, ntiles = Mp / 128;
  const __nv_bfloat16 *Dhi = reinterpret_cast<const __nv_bfloat16 *>(h->d_ab_work);
  const __nv_bfloat16 *Dlo = Dhi + Mp * ab.Kp;
  const size_t smem = (size_t)2 * ab.Np * ab.Kp * 2 + (size_t)2 * 128 * ab.Kp * 2 + 64;
  const unsigned grid = (unsigned)std::min<size_t>(ntiles, (size_t)h->num_sms);
  ab_tc_kernel<<<grid, 128, smem, h->stream>>>(Dhi, Dlo, reinterpret_cast<const __nv_bfloat16 *>(ab.Vhi),
                                               reinterpret_cast<const __nv_bfloat16 *>(ab.Vlo), E,
                                               ab.Kp, ab.Np, ab.npq, M, ntiles, ab.err);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

int ab_tc_check(sbd_tpb_handle *h) {
  if (!h->ab.err) return SBD_TPB_OK;
  int e = 0;
  TPB_CUDA(cudaMemcpy(&e, h->ab.err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    cudaMemset(h->ab.err, 0, sizeof(int));
    return fail(SBD_TPB_ERR_CUDA, "alpha-beta tensor-core kernel: bounded wait expired (code " +
                                      std::to_string(e) + ")");
  }
  return SBD_TPB_OK;
}

}  // namespace sbdtpb
