// Learned Davidson preconditioner: BF16 tensor-core MLP, its training and the fused inference
// kernel used inside the Davidson loop.
//
// The reference has no learned part; its correction is t = r / (E0 - H_ii)
// (tpb/davidson.h:858-868).  Here a network predicts a per-determinant factor on top of it,
// t_i = d_i (1 + y_i), so w3 = b3 = 0 reproduces the diagonal correction exactly and a trained
// network can only redirect the search vector; the Rayleigh quotient and residual in FP64 still
// decide convergence.
//
//   x (64)  -> Z1 = W1 x + b1 (256) -> GELU -> Z2 = W2 A1 + b2 (256) -> GELU -> y = w3.A2 + b3
//
// Kernels:
//   tc_gemm_kernel     D = A B^T with tcgen05.mma (BF16 operands staged by 1-D bulk copies in
//                      64-wide K chunks, double buffered, FP32 accumulator in TMEM); split-K
//                      partials for the weight gradients.  Every GEMM of training uses it.
//   mlp_infer_kernel   persistent, one CTA per SM: W1 and W2 stay in shared memory; per tile of
//                      128 determinants it builds the features in shared memory, runs layer 1
//                      and layer 2 on the tensor cores with GELU epilogues from TMEM, and writes
//                      t = d (1 + y) in place.
//   the elementwise kernels of the backward pass, Adam, and the sampling of training pairs.
// All mbarrier waits are bounded; an expired wait sets an error code that the host reports.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "mlp.cuh"
#include "tc_util.cuh"
#include "tpb_common.cuh"

using bf16 = __nv_bfloat16;

namespace sbdtpb {
namespace {

using namespace tc;

constexpr int H = kMlpHidden, F = kMlpFeat;
constexpr size_t oW1 = 0, ob1 = oW1 + (size_t)H * F, oW2 = ob1 + H, ob2 = oW2 + (size_t)H * H,
                 ow3 = ob2 + H, ob3 = ow3 + H, kParams = ob3 + 1;
static_assert(kParams == SBD_TPB_MLP_PARAMS, "parameter count");
constexpr int kChunk = 64;  // K chunk of the GEMM pipeline

// ---------------------------------------------------------------- activation and features
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// GELU, tanh form (Hendrycks & Gimpel): 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))
__device__ __forceinline__ float gelu(float z) {
  const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
  return 0.5f * z * (1.f + tanh_fast(u));
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
  const float th = tanh_fast(u);
  return 0.5f * (1.f + th) + 0.5f * z * (1.f - th * th) * 0.7978845608028654f * (1.f + 0.134145f * z * z);
}

// Features depend only on a determinant's spatial occupation (which orbitals are empty, singly or
// doubly occupied), never on which singly occupied orbitals carry alpha and which beta.  Every
// determinant of a spin-coupled set then gets the same factor 1 + y, so the learned correction
// (1 + Y) D r commutes with S^2 wherever the diagonal one D r does, and cannot steer the solver to a
// state of another spin than the diagonal correction's: the energy feature is the spin-free diagonal
// E_J = H_ii + sum of the same-spin exchange integrals of both strings (Coulomb terms only), and
// the residual-entry input is held at zero (r_i differs within a spin-coupled set).
__device__ __forceinline__ void cont_features(double hdJ, double e0, float &fe, float &fr) {
  fe = asinhf((float)(hdJ - e0)) * 0.25f;
  fr = 0.f;
}

// 8 consecutive features k0..k0+7 of one row as BF16: [fe, fr, doubly occupied window (24),
// singly occupied window (24), 14 zeros]
__device__ __forceinline__ uint4 feature_group(int g, float fe, float fr, uint32_t oa, uint32_t ob) {
  union {
    bf16 h[8];
    uint4 u;
  } o;
  const uint32_t dbl = oa & ob, sgl = oa ^ ob;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int k = g * 8 + i;
    float x = 0.f;
    if (k == 0) x = fe;
    else if (k == 1) x = fr;
    else if (k < 2 + kMlpWin) x = (float)((dbl >> (k - 2)) & 1u);
    else if (k < 2 + 2 * kMlpWin) x = (float)((sgl >> (k - 2 - kMlpWin)) & 1u);
    o.h[i] = __float2bfloat16_rn(x);
  }
  return o.u;
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// ---------------------------------------------------------------- GEMM: D = A . B^T
// A: M x Kp (tiles of 128 rows), B: Np x Kp, both in the tc_util.cuh operand layouts; grid
// (M/128, splits); split s covers K chunks [s*kper, (s+1)*kper) and writes D + s*M*Np (FP32,
// row-major M x Np).
__global__ void __launch_bounds__(128, 1)
    tc_gemm_kernel(const bf16 *__restrict__ A, const bf16 *__restrict__ B, float *__restrict__ D, int Kp,
                   int Np, int kper, int M, int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const uint32_t a_chunk = 128u * kChunk * 2, b_chunk = (uint32_t)Np * kChunk * 2;
  unsigned char *sA[2] = {smem, smem + a_chunk + b_chunk};
  unsigned char *sB[2] = {smem + a_chunk, smem + 2 * a_chunk + b_chunk};
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * (a_chunk + b_chunk));  // load[2], mma[2]
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 4);
  volatile int *status = reinterpret_cast<volatile int *>(tslot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mt = blockIdx.x, split = blockIdx.y;
  const int c0 = split * kper, c1 = min(c0 + kper, Kp / kChunk);
  uint32_t ncols = 32;
  while ((int)ncols < Np) ncols <<= 1;

  if (threadIdx.x == 0) {
    for (int i = 0; i < 4; i++) mbar_init(smem_addr(&bars[i]), 1);
    fence_mbar_init();
    *status = 0;
  }
  if (warp == 0) tmem_alloc(smem_addr(tslot), ncols);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;

  if (threadIdx.x == 0) {
    const bf16 *Abase = A + (size_t)mt * 128 * Kp;
    uint32_t lph[2] = {0, 0}, mph[2] = {0, 0};
    bool lpend[2] = {false, false}, mpend[2] = {false, false};
    int code = 0;
    auto issue_load = [&](int c, int s) {
      const uint32_t bar = smem_addr(&bars[s]);
      mbar_expect_tx(bar, a_chunk + b_chunk);
      bulk_g2s(smem_addr(sA[s]), Abase + (size_t)c * 128 * kChunk, a_chunk, bar);
      bulk_g2s(smem_addr(sB[s]), B + (size_t)c * Np * kChunk, b_chunk, bar);
      lpend[s] = true;
    };
    const int NG = Np >> 3;
    const uint32_t idesc = idesc_bf16(Np);
    if (c0 < c1) issue_load(c0, 0);
    for (int c = c0; c < c1 && code == 0; c++) {
      const int s = (c - c0) & 1;
      if (c + 1 < c1) {
        const int s2 = s ^ 1;
        if (mpend[s2]) {  // the stage is free once the MMAs that read it completed
          if (!mbar_wait(smem_addr(&bars[2 + s2]), mph[s2])) {
            code = 1;
            break;
          }
          mph[s2] ^= 1;
          mpend[s2] = false;
        }
        issue_load(c + 1, s2);
      }
      if (!mbar_wait(smem_addr(&bars[s]), lph[s])) {
        code = 2;
        break;
      }
      lph[s] ^= 1;
      lpend[s] = false;
      fence_after_sync();
      const uint32_t a0 = smem_addr(sA[s]), b0 = smem_addr(sB[s]);
#pragma unroll
      for (int k = 0; k < kChunk / 16; k++) {
        const uint64_t ad = make_desc(a0 + (uint32_t)k * 4096u, 2048u, 128u);
        const uint64_t bd = make_desc(b0 + (uint32_t)(k * 2 * NG) * 128u, (uint32_t)NG * 128u, 128u);
        mma_bf16(tmem, ad, bd, idesc, (c > c0 || k > 0) ? 1u : 0u);
      }
      mma_commit(smem_addr(&bars[2 + s]));
      mpend[s] = true;
    }
    // drain (bounded): copies and MMAs still in flight must finish before the CTA exits
    for (int s = 0; s < 2; s++) {
      if (lpend[s] && !mbar_wait(smem_addr(&bars[s]), lph[s]) && code == 0) code = 3;
      if (mpend[s] && !mbar_wait(smem_addr(&bars[2 + s]), mph[s]) && code == 0) code = 4;
    }
    if (code) {
      atomicExch(err, 100 + code);
      *status = 1;
    }
  }
  __syncthreads();
  if (*status == 0) {
    fence_after_sync();
    const int row = warp * 32 + lane;
    float *drow = D + ((size_t)split * M + (size_t)mt * 128 + row) * Np;
    for (int col = 0; col < Np; col += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col, v);
      float4 *o = reinterpret_cast<float4 *>(drow + col);
#pragma unroll
      for (int i = 0; i < 4; i++) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------- training kernels
struct SampleView {
  const float *fe, *fr, *a, *b, *w;
  const uint32_t *oa, *ob;
};

// Batch rows r < nB: sample idx[base + r] (or base + r) when base + r < navail, else a zero row
// of weight 0.  xraw (n x 64, FP32) replaces the sample set when given.
__global__ void pack_batch_kernel(SampleView s, const float *__restrict__ xraw, const uint32_t *__restrict__ idx,
                                  size_t base, size_t navail, int nB, bf16 *__restrict__ Xa,
                                  bf16 *__restrict__ XbT, float *__restrict__ av, float *__restrict__ bv,
                                  float *__restrict__ wv) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nB) return;
  const bool have = base + r < navail;
  const size_t j = have ? (idx ? (size_t)idx[base + r] : base + r) : 0;
  float A = 0.f, Bv = 0.f, W = 0.f;
  if (have) {
    A = s.a[j];
    Bv = s.b[j];
    W = s.w[j];
  }
  for (int g = 0; g < F / 8; g++) {
    union {
      bf16 h[8];
      uint4 u;
    } o;
    if (!have) {
      o.u = make_uint4(0, 0, 0, 0);
    } else if (xraw) {
#pragma unroll
      for (int i = 0; i < 8; i++) o.h[i] = __float2bfloat16_rn(xraw[j * F + g * 8 + i]);
    } else {
      o.u = feature_group(g, s.fe[j], s.fr[j], s.oa[j], s.ob[j]);
    }
    *reinterpret_cast<uint4 *>(Xa + a_off((size_t)r, g * 8, F)) = o.u;
#pragma unroll
    for (int i = 0; i < 8; i++) XbT[b_off(g * 8 + i, (size_t)r, F)] = o.h[i];
  }
  av[r] = A;
  bv[r] = Bv;
  wv[r] = W;
}

// Z1 += b1 (kept for the backward pass); A1 = gelu(Z1) as the A operand of layer 2 and as the
// B operand (hidden x batch) of the W2 gradient
__global__ void act1_kernel(float *__restrict__ Z, const float *__restrict__ P, int nB, bf16 *__restrict__ A1a,
                            bf16 *__restrict__ A1bT) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)nB * H) return;
  const int s = (int)(idx / H), j = (int)(idx % H);
  const float z = Z[idx] + P[ob1 + j];
  Z[idx] = z;
  const bf16 a = __float2bfloat16_rn(gelu(z));
  A1a[a_off((size_t)s, j, H)] = a;
  A1bT[b_off(j, (size_t)s, H)] = a;
}

// One warp per sample: layer-2 activation, output, loss and dL/dZ2.
__global__ void head_kernel(const float *__restrict__ Z2, const float *__restrict__ P, const float *__restrict__ av,
                            const float *__restrict__ bv, const float *__restrict__ wv, int nB, float inv_n,
                            float *__restrict__ G2, float *__restrict__ A2, float *__restrict__ gy,
                            float *__restrict__ lossv, float *__restrict__ yout, bf16 *__restrict__ G2a,
                            bf16 *__restrict__ G2Ta) {
  const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (s >= nB) return;
  float z[H / 32], a2[H / 32], part = 0.f;
#pragma unroll
  for (int c = 0; c < H / 32; c++) {
    const int j = lane + 32 * c;
    z[c] = Z2[(size_t)s * H + j] + P[ob2 + j];
    a2[c] = gelu(z[c]);
    part += a2[c] * P[ow3 + j];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  // bounded factor 1 + c tanh(y): the correction keeps d's sign and at most scales it by 1 +- c
  const float th = tanhf(part + P[ob3]);
  const float y = kMlpBound * th;
  const float A = av[s], Bv = bv[s], W = wv[s];
  const float e = A * (1.f + y) - Bv;
  const float g = W * A * e * inv_n * kMlpBound * (1.f - th * th);
  if (lane == 0) {
    gy[s] = g;
    lossv[s] = 0.5f * W * e * e * inv_n;
    yout[s] = y;
  }
#pragma unroll
  for (int c = 0; c < H / 32; c++) {
    const int j = lane + 32 * c;
    const float g2 = g * P[ow3 + j] * gelu_grad(z[c]);
    G2[(size_t)s * H + j] = g2;
    A2[(size_t)s * H + j] = a2[c];
    const bf16 gb = __float2bfloat16_rn(g2);
    G2a[a_off((size_t)s, j, H)] = gb;
    G2Ta[a_off((size_t)j, s, nB)] = gb;
  }
}

// gradients of b2, w3, b3 and the loss (fixed-order sums over the batch)
__global__ void head_sums_kernel(const float *__restrict__ G2, const float *__restrict__ A2,
                                 const float *__restrict__ gy, const float *__restrict__ lossv, int nB,
                                 float *__restrict__ grad, double *__restrict__ loss) {
  const int j = threadIdx.x;
  double sb = 0.0, sw = 0.0;
  for (int s = 0; s < nB; s++) {
    sb += G2[(size_t)s * H + j];
    sw += (double)gy[s] * A2[(size_t)s * H + j];
  }
  grad[ob2 + j] = (float)sb;
  grad[ow3 + j] = (float)sw;
  if (j == 0) {
    double g = 0.0, l = 0.0;
    for (int s = 0; s < nB; s++) {
      g += gy[s];
      l += lossv[s];
    }
    grad[ob3] = (float)g;
    *loss = l;
  }
}

// G1 = dA1 * gelu'(Z1) (in place) and as the A operand (hidden x batch) of the W1 gradient
__global__ void act1_bwd_kernel(float *__restrict__ dA1, const float *__restrict__ Z1, int nB,
                                bf16 *__restrict__ G1Ta) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)nB * H) return;
  const int s = (int)(idx / H), j = (int)(idx % H);
  const float g = dA1[idx] * gelu_grad(Z1[idx]);
  dA1[idx] = g;
  G1Ta[a_off((size_t)j, s, nB)] = __float2bfloat16_rn(g);
}

__global__ void colsum_kernel(const float *__restrict__ G, int nB, float *__restrict__ out) {
  const int j = threadIdx.x;
  double s = 0.0;
  for (int r = 0; r < nB; r++) s += G[(size_t)r * H + j];
  out[j] = (float)s;
}

__global__ void reduce_split_kernel(const float *__restrict__ Dp, int splits, size_t mn, float *__restrict__ out) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= mn) return;
  float s = 0.f;
  for (int k = 0; k < splits; k++) s += Dp[(size_t)k * mn + i];
  out[i] = s;
}

__global__ void adam_kernel(float *__restrict__ P, const float *__restrict__ G, float *__restrict__ m,
                            float *__restrict__ v, size_t n, float lr, float c1, float c2) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = G[i];
  const float mi = 0.9f * m[i] + 0.1f * g, vi = 0.999f * v[i] + 0.001f * g * g;
  m[i] = mi;
  v[i] = vi;
  P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

// BF16 operand copies of the weights: W1 (N = hidden, K = feature), W2 (N = out, K = in) and
// W2^T (N = in, K = out) for the layer-1 activation gradient
__global__ void pack_weights_kernel(const float *__restrict__ P, bf16 *__restrict__ W1p, bf16 *__restrict__ W2p,
                                    bf16 *__restrict__ W2Tp) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < H * H) {
    const int o = idx / H, i = idx % H;
    const bf16 w = __float2bfloat16_rn(P[oW2 + idx]);
    W2p[b_off(o, (size_t)i, H)] = w;
    W2Tp[b_off(i, (size_t)o, H)] = w;
  }
  if (idx < H * F) {
    const int o = idx / F, k = idx % F;
    W1p[b_off(o, (size_t)k, H)] = __float2bfloat16_rn(P[oW1 + idx]);
  }
}

// ---------------------------------------------------------------- fused inference
constexpr int kInfThreads = 256;
constexpr uint32_t kSmW1 = (uint32_t)H * F * 2;           // 32 KB
constexpr uint32_t kSmW2 = (uint32_t)H * H * 2;           // 128 KB
constexpr uint32_t kSmA = 128u * H * 2;                   // 64 KB (the feature tile uses 16 KB)
constexpr uint32_t kSmPart = 128 * 4, kSmD = 128 * 8;
constexpr uint32_t kSmInfer = kSmW1 + kSmW2 + kSmA + kSmPart + kSmD + 64;

struct InferArgs {
  const double *hii;
  const double *kxa, *kxb;  // same-spin exchange sums of the alpha / beta strings
  double e0;
  const uint32_t *occ_a, *occ_b;
  uint32_t nb;
  const uint32_t *idx;  // determinants to correct (null: all of 0 .. count-1)
  size_t count;
  const bf16 *W1p, *W2p;
  const float *P;
  int *err;
};

template <typename T>
__global__ void __launch_bounds__(kInfThreads, 1) mlp_infer_kernel(InferArgs a, T *__restrict__ t) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sW1 = smem, *sW2 = smem + kSmW1, *sA = smem + kSmW1 + kSmW2;
  float *part = reinterpret_cast<float *>(sA + kSmA);
  double *dsh = reinterpret_cast<double *>(sA + kSmA + kSmPart);
  uint64_t *bars = reinterpret_cast<uint64_t *>(sA + kSmA + kSmPart + kSmD);  // load, mma
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2);
  volatile int *status = reinterpret_cast<volatile int *>(tslot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = warp & 3, half = warp >> 2;
  const uint32_t bar_load = smem_addr(&bars[0]), bar_mma = smem_addr(&bars[1]);

  if (threadIdx.x == 0) {
    mbar_init(bar_load, 1);
    mbar_init(bar_mma, 1);
    fence_mbar_init();
    *status = 0;
  }
  if (warp == 0) tmem_alloc(smem_addr(tslot), 256);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  uint32_t mma_phase = 0;

  if (threadIdx.x == 0) {
    mbar_expect_tx(bar_load, kSmW1 + kSmW2);
    bulk_g2s(smem_addr(sW1), a.W1p, kSmW1, bar_load);
    bulk_g2s(smem_addr(sW2), a.W2p, kSmW2, bar_load);
    if (!mbar_wait(bar_load, 0)) {
      atomicExch(a.err, 201);
      *status = 1;
      mbar_wait(bar_load, 0);  // bounded second wait for the copies in flight
    }
  }
  __syncthreads();

  const size_t ntiles = (a.count + 127) / 128;
  const int row = quad * 32 + lane;  // TMEM lane of this thread in the epilogues
  const uint32_t trow = tmem + ((uint32_t)(quad * 32) << 16);
  for (size_t tile = blockIdx.x; tile < ntiles && *status == 0; tile += gridDim.x) {
    // features of the tile's 128 determinants (threads 0..127, one row each)
    if (threadIdx.x < 128) {
      const int r = threadIdx.x;
      const size_t kk = tile * 128 + r;
      const bool live = kk < a.count;
      const size_t i = live ? (a.idx ? (size_t)__ldg(&a.idx[kk]) : kk) : 0;
      float fe = 0.f, fr = 0.f;
      uint32_t oa = 0, ob = 0;
      double d = 0.0;
      if (live) {
        d = (double)t[i];
        const size_t ia = i / a.nb, ib = i - ia * a.nb;
        cont_features(__ldg(&a.hii[i]) + __ldg(&a.kxa[ia]) + __ldg(&a.kxb[ib]), a.e0, fe, fr);
        oa = __ldg(&a.occ_a[ia]);
        ob = __ldg(&a.occ_b[ib]);
      }
      dsh[r] = d;
#pragma unroll
      for (int g = 0; g < F / 8; g++) {
        const uint4 u = live ? feature_group(g, fe, fr, oa, ob) : make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4 *>(sA + a_off((size_t)r, g * 8, F) * 2) = u;
      }
      fence_proxy_async();
    }
    __syncthreads();
    // layer 1: [128 x 64] . W1^T -> TMEM columns 0..255
    if (threadIdx.x == 0) {
      fence_after_sync();
      const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sW1);
#pragma unroll
      for (int k = 0; k < F / 16; k++)
        mma_bf16(tmem, make_desc(a0 + (uint32_t)k * 4096u, 2048u, 128u),
                 make_desc(b0 + (uint32_t)k * 2 * (H / 8) * 128u, (H / 8) * 128u, 128u), idesc_bf16(H),
                 k > 0 ? 1u : 0u);
      mma_commit(bar_mma);
      if (!mbar_wait(bar_mma, mma_phase)) {
        atomicExch(a.err, 202);
        *status = 1;
        mbar_wait(bar_mma, mma_phase);
      }
      mma_phase ^= 1;
    }
    __syncthreads();
    if (*status) break;
    fence_after_sync();
    // epilogue 1: A1 = gelu(Z1 + b1) as BF16 into the A tile (the features are consumed)
    for (int c = 0; c < 8; c++) {
      const int col = half * 128 + c * 16;
      float v[16];
      tmem_ld16(trow + (uint32_t)col, v);
      union {
        bf16 h[16];
        uint4 u[2];
      } o;
#pragma unroll
      for (int i = 0; i < 16; i++) o.h[i] = __float2bfloat16_rn(gelu(v[i] + __ldg(&a.P[ob1 + col + i])));
      *reinterpret_cast<uint4 *>(sA + a_off((size_t)row, col, H) * 2) = o.u[0];
      *reinterpret_cast<uint4 *>(sA + a_off((size_t)row, col + 8, H) * 2) = o.u[1];
    }
    fence_before_sync();
    fence_proxy_async();
    __syncthreads();
    // layer 2: [128 x 256] . W2^T -> TMEM columns 0..255
    if (threadIdx.x == 0) {
      fence_after_sync();
      const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sW2);
#pragma unroll 4
      for (int k = 0; k < H / 16; k++)
        mma_bf16(tmem, make_desc(a0 + (uint32_t)k * 4096u, 2048u, 128u),
                 make_desc(b0 + (uint32_t)k * 2 * (H / 8) * 128u, (H / 8) * 128u, 128u), idesc_bf16(H),
                 k > 0 ? 1u : 0u);
      mma_commit(bar_mma);
      if (!mbar_wait(bar_mma, mma_phase)) {
        atomicExch(a.err, 203);
        *status = 1;
        mbar_wait(bar_mma, mma_phase);
      }
      mma_phase ^= 1;
    }
    __syncthreads();
    if (*status) break;
    fence_after_sync();
    // epilogue 2: y = w3 . gelu(Z2 + b2) + b3, t = d (1 + y)
    float acc = 0.f;
    for (int c = 0; c < 8; c++) {
      const int col = half * 128 + c * 16;
      float v[16];
      tmem_ld16(trow + (uint32_t)col, v);
#pragma unroll
      for (int i = 0; i < 16; i++)
        acc += gelu(v[i] + __ldg(&a.P[ob2 + col + i])) * __ldg(&a.P[ow3 + col + i]);
    }
    if (half == 1) part[row] = acc;
    fence_before_sync();
    __syncthreads();
    if (half == 0) {
      const size_t kk = tile * 128 + row;
      if (kk < a.count) {
        const size_t i = a.idx ? (size_t)__ldg(&a.idx[kk]) : kk;
        const float y = kMlpBound * tanhf(acc + part[row] + __ldg(&a.P[ob3]));
        t[i] = (T)(dsh[row] * (1.0 + (double)y));
      }
    }
    __syncthreads();
  }
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 256);
}

// Determinants whose diagonal correction is at least theta in magnitude, compacted into idx (order
// arbitrary: every corrected entry depends only on itself).  With theta = |d| / sqrt(cap) at most
// cap entries qualify (sum of d_i^2 over them is at most |d|^2); the counter guards the rest.
template <typename T>
__global__ void select_kernel(const T *__restrict__ d, size_t n, double theta, uint32_t *__restrict__ idx,
                              uint32_t cap, unsigned long long *__restrict__ count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if (fabs((double)d[i]) >= theta) {
      const unsigned long long pos = atomicAdd(count, 1ull);
      if (pos < cap) idx[pos] = (uint32_t)i;
    }
  }
}

// ---------------------------------------------------------------- training pairs
// A recorded step gives, per determinant i,
//   a_i = d_i / |d|,   b_i = (d_i - (Pd)_i + alpha (P Psi)_i) / |d|,
// with P = 1 - sum_j C_j C_j^T the projector out of the step's subspace, Pd = d - sum_j hd_j vec_j
// and P Psi = Psi - sum_j g_j vec_j, and alpha = (Pd . Psi) / |P Psi|^2 the scale that best fits
// P Psi to Pd.  Only the part of a correction outside the subspace moves the Ritz vector, so b
// keeps d's in-subspace part (the network need not change it) and replaces its outside part by the
// exact direction: (a - b) = (Pd - alpha P Psi) / |d| is the diagonal correction's error, and the
// network is trained to shrink it.
constexpr int kMaxBasis = 16;

struct PairArgs {
  const float *d;
  const double *Psi;
  const float *C[kMaxBasis];  // basis vectors (unnormalised)
  double g[kMaxBasis];        // P Psi = Psi - sum_j g_j C_j
  double hd[kMaxBasis];       // P d   = d   - sum_j hd_j C_j
  int m;
  double inv_dn, alpha, c;    // 1/|d|, fit scale, sampling scale p = min(1, c (|a| + |b|))
  double e0;
  uint64_t seed;
};

__device__ __forceinline__ void pair_proj(const PairArgs &k, size_t i, double &d, double &pd, double &pp) {
  d = k.d[i];
  pd = d;
  pp = k.Psi[i];
  for (int j = 0; j < k.m; j++) {
    const double c = k.C[j][i];
    pd -= k.hd[j] * c;
    pp -= k.g[j] * c;
  }
}

__device__ __forceinline__ void pair_ab(const PairArgs &k, size_t i, double &A, double &B) {
  double d, pd, pp;
  pair_proj(k, i, d, pd, pp);
  A = d * k.inv_dn;
  B = (d - pd + k.alpha * pp) * k.inv_dn;
}

// dots of the basis vectors against Psi (dsrc null) or against d: partials[j * nblk + b]
__global__ void basis_dots_kernel(PairArgs k, const double *__restrict__ Psi, const float *__restrict__ dsrc,
                                  size_t n, int nv, double *__restrict__ partials) {
  double s[kMaxBasis];
  for (int j = 0; j < kMaxBasis; j++) s[j] = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double p = dsrc ? (double)dsrc[i] : Psi[i];
    for (int j = 0; j < nv; j++) s[j] += (double)k.C[j][i] * p;
  }
  __shared__ double red[kMaxBasis][8];
  for (int j = 0; j < nv; j++) {
    double v = s[j];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[j][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < nv) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[threadIdx.x][w];
    partials[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = v;
  }
}

// partials[0..3][b]: d.d, Pd.Pd, Pd.Psi, sum |a| + |b| (the last with k's coefficients)
__global__ void pair_sums_kernel(PairArgs k, size_t n, int with_ab, double *__restrict__ partials) {
  double s[4] = {0, 0, 0, 0};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double d, pd, pp;
    pair_proj(k, i, d, pd, pp);
    s[0] += d * d;
    s[1] += pd * pd;
    s[2] += pd * k.Psi[i];
    if (with_ab) {
      const double A = d * k.inv_dn, B = (d - pd + k.alpha * pp) * k.inv_dn;
      s[3] += fabs(A) + fabs(B);
    }
  }
  __shared__ double red[4][8];
  for (int j = 0; j < 4; j++) {
    double v = s[j];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[j][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[threadIdx.x][w];
    partials[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = v;
  }
}

__global__ void sum_partials_kernel(const double *__restrict__ partials, int nblocks, int nvals,
                                    double *__restrict__ out) {
  if (threadIdx.x >= nvals) return;
  double v = 0.0;
  for (int b = 0; b < nblocks; b++) v += partials[(size_t)threadIdx.x * nblocks + b];
  out[threadIdx.x] = v;
}

__device__ __forceinline__ bool pair_keep(const PairArgs &k, size_t i, double A, double B, double &p) {
  p = fmin(1.0, k.c * (fabs(A) + fabs(B)));
  const double u = (double)(splitmix64(k.seed ^ (uint64_t)i) >> 11) * (1.0 / 9007199254740992.0);
  return u < p;
}

// pass 1: keep flags and per-block counts over contiguous chunks
__global__ void pair_flag_kernel(PairArgs k, size_t n, size_t chunk, uint8_t *__restrict__ flags,
                                 uint32_t *__restrict__ counts) {
  __shared__ uint32_t cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  const size_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
  uint32_t mine = 0;
  for (size_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double A, B, p;
    pair_ab(k, i, A, B);
    const bool keep = pair_keep(k, i, A, B, p);
    flags[i] = keep ? 1 : 0;
    mine += keep;
  }
  atomicAdd(&cnt, mine);
  __syncthreads();
  if (threadIdx.x == 0) counts[blockIdx.x] = cnt;
}

struct SampleOut {
  float *fe, *fr, *a, *b, *w;
  uint32_t *oa, *ob;
};

// pass 2: write the kept pairs in index order (block offsets from the host scan)
__global__ void pair_write_kernel(PairArgs k, const double *__restrict__ hii, const double *__restrict__ kxa,
                                  const double *__restrict__ kxb, const uint32_t *__restrict__ occ_a,
                                  const uint32_t *__restrict__ occ_b, uint32_t nb, size_t n, size_t chunk,
                                  const uint8_t *__restrict__ flags, const uint64_t *__restrict__ offsets,
                                  SampleOut o) {
  __shared__ uint32_t wsum[32];
  __shared__ uint64_t running;
  if (threadIdx.x == 0) running = offsets[blockIdx.x];
  __syncthreads();
  const size_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (size_t base = lo; base < hi; base += blockDim.x) {
    const size_t i = base + threadIdx.x;
    const bool keep = i < hi && flags[i];
    const uint32_t m = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) wsum[wid] = __popc(m);
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (int w = 0; w < nw; w++) {
      if (w < wid) before += wsum[w];
      total += wsum[w];
    }
    if (keep) {
      const uint64_t pos = running + before + __popc(m & ((1u << lane) - 1u));
      double A, B, p;
      pair_ab(k, i, A, B);
      pair_keep(k, i, A, B, p);
      float fe, fr;
      const size_t ia = i / nb, ib = i - ia * nb;
      cont_features(hii[i] + kxa[ia] + kxb[ib], k.e0, fe, fr);
      o.fe[pos] = fe;
      o.fr[pos] = fr;
      o.oa[pos] = occ_a[ia];
      o.ob[pos] = occ_b[ib];
      o.a[pos] = (float)A;
      o.b[pos] = (float)B;
      o.w[pos] = (float)(1.0 / p);
    }
    __syncthreads();
    if (threadIdx.x == 0) running += total;
    __syncthreads();
  }
}

template <typename T>
void free_dev(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

}  // namespace
}  // namespace sbdtpb

// ==================================================================== host object
struct sbd_tpb_precond {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  uint64_t seed = 0;
  float *P = nullptr, *G = nullptr, *m = nullptr, *v = nullptr;  // params, grads, Adam moments
  int adam_t = 0;
  bf16 *W1p = nullptr, *W2p = nullptr, *W2Tp = nullptr;
  int *err = nullptr;
  struct Set {
    float *fe = nullptr, *fr = nullptr, *a = nullptr, *b = nullptr, *w = nullptr;
    uint32_t *oa = nullptr, *ob = nullptr;
    size_t n = 0, cap = 0;
  } set[2];
  // batch work buffers (sized for cap_batch rows)
  int cap_batch = 0;
  bf16 *Xa = nullptr, *XbT = nullptr, *A1a = nullptr, *A1bT = nullptr, *G2a = nullptr, *G2Ta = nullptr,
       *G1Ta = nullptr;
  float *Z1 = nullptr, *Z2 = nullptr, *G2 = nullptr, *A2 = nullptr, *dA1 = nullptr;
  float *av = nullptr, *bv = nullptr, *wv = nullptr, *gy = nullptr, *lossv = nullptr, *yv = nullptr;
  float *Dp = nullptr;  // split-K partials
  size_t dp_cap = 0;
  double *dloss = nullptr;
  uint64_t steps_seen = 0;  // recorded Davidson steps turned into pairs (sampling seeds)
  float *xraw = nullptr;
  size_t xraw_cap = 0;
  ~sbd_tpb_precond();
};

namespace sbdtpb {
namespace {

void free_set(sbd_tpb_precond::Set &s) {
  free_dev(s.fe);
  free_dev(s.fr);
  free_dev(s.a);
  free_dev(s.b);
  free_dev(s.w);
  free_dev(s.oa);
  free_dev(s.ob);
  s.n = s.cap = 0;
}

void free_batch(sbd_tpb_precond *p) {
  free_dev(p->Xa);
  free_dev(p->XbT);
  free_dev(p->A1a);
  free_dev(p->A1bT);
  free_dev(p->G2a);
  free_dev(p->G2Ta);
  free_dev(p->G1Ta);
  free_dev(p->Z1);
  free_dev(p->Z2);
  free_dev(p->G2);
  free_dev(p->A2);
  free_dev(p->dA1);
  free_dev(p->av);
  free_dev(p->bv);
  free_dev(p->wv);
  free_dev(p->gy);
  free_dev(p->lossv);
  free_dev(p->yv);
  p->cap_batch = 0;
}

int check_err(sbd_tpb_precond *p, const char *what) {
  int e = 0;
  TPB_CUDA(cudaMemcpyAsync(&e, p->err, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  TPB_CUDA(cudaStreamSynchronize(p->stream));
  if (e) {
    cudaMemsetAsync(p->err, 0, sizeof(int), p->stream);
    return fail(SBD_TPB_ERR_CUDA, std::string(what) + ": tensor-core kernel wait expired (code " +
                                      std::to_string(e) + ")");
  }
  return SBD_TPB_OK;
}

int ensure_batch(sbd_tpb_precond *p, int nB) {
  if (p->cap_batch >= nB) return SBD_TPB_OK;
  free_batch(p);
  const size_t b = (size_t)nB;
  TPB_CUDA(cudaMalloc(&p->Xa, b * F * 2));
  TPB_CUDA(cudaMalloc(&p->XbT, b * F * 2));
  TPB_CUDA(cudaMalloc(&p->A1a, b * H * 2));
  TPB_CUDA(cudaMalloc(&p->A1bT, b * H * 2));
  TPB_CUDA(cudaMalloc(&p->G2a, b * H * 2));
  TPB_CUDA(cudaMalloc(&p->G2Ta, b * H * 2));
  TPB_CUDA(cudaMalloc(&p->G1Ta, b * H * 2));
  TPB_CUDA(cudaMalloc(&p->Z1, b * H * 4));
  TPB_CUDA(cudaMalloc(&p->Z2, b * H * 4));
  TPB_CUDA(cudaMalloc(&p->G2, b * H * 4));
  TPB_CUDA(cudaMalloc(&p->A2, b * H * 4));
  TPB_CUDA(cudaMalloc(&p->dA1, b * H * 4));
  TPB_CUDA(cudaMalloc(&p->av, b * 4));
  TPB_CUDA(cudaMalloc(&p->bv, b * 4));
  TPB_CUDA(cudaMalloc(&p->wv, b * 4));
  TPB_CUDA(cudaMalloc(&p->gy, b * 4));
  TPB_CUDA(cudaMalloc(&p->lossv, b * 4));
  TPB_CUDA(cudaMalloc(&p->yv, b * 4));
  p->cap_batch = nB;
  return SBD_TPB_OK;
}

size_t gemm_smem(int Np) { return 2 * ((size_t)128 * kChunk * 2 + (size_t)Np * kChunk * 2) + 64; }

// D (+ split partials reduced into out when splits > 1) = A[M x Kp] . B[Np x Kp]^T
int gemm(sbd_tpb_precond *p, const bf16 *A, const bf16 *B, int M, int Kp, int Np, int want_splits, float *out) {
  if (M % 128 || Kp % kChunk || Np % 16 || Np > 256)
    return fail(SBD_TPB_ERR_INVALID, "mlp gemm: unsupported shape");
  const int nch = Kp / kChunk;
  int splits = std::max(1, std::min(want_splits, nch));
  const int kper = (nch + splits - 1) / splits;
  splits = (nch + kper - 1) / kper;
  float *D = out;
  if (splits > 1) {
    const size_t need = (size_t)splits * M * Np;
    if (p->dp_cap < need) {
      free_dev(p->Dp);
      p->dp_cap = 0;
      TPB_CUDA(cudaMalloc(&p->Dp, need * sizeof(float)));
      p->dp_cap = need;
    }
    D = p->Dp;
  }
  const size_t smem = gemm_smem(Np);
  TPB_CUDA(cudaFuncSetAttribute(tc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  tc_gemm_kernel<<<dim3(M / 128, splits), 128, smem, p->stream>>>(A, B, D, Kp, Np, kper, M, p->err);
  TPB_CUDA(cudaGetLastError());
  if (splits > 1) {
    const size_t mn = (size_t)M * Np;
    reduce_split_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, p->stream>>>(p->Dp, splits, mn, out);
    TPB_CUDA(cudaGetLastError());
  }
  return SBD_TPB_OK;
}

int pack_weights(sbd_tpb_precond *p) {
  pack_weights_kernel<<<(H * H + 255) / 256, 256, 0, p->stream>>>(p->P, p->W1p, p->W2p, p->W2Tp);
  TPB_CUDA(cudaGetLastError());
  return SBD_TPB_OK;
}

// batch rows packed; forward (and backward into p->G when grads) of nB rows, inv_n the loss scale
int fwd_bwd(sbd_tpb_precond *p, int nB, float inv_n, bool grads) {
  TPB_CHECK(gemm(p, p->Xa, p->W1p, nB, F, H, 1, p->Z1));
  act1_kernel<<<(unsigned)(((size_t)nB * H + 255) / 256), 256, 0, p->stream>>>(p->Z1, p->P, nB, p->A1a, p->A1bT);
  TPB_CUDA(cudaGetLastError());
  TPB_CHECK(gemm(p, p->A1a, p->W2p, nB, H, H, 1, p->Z2));
  head_kernel<<<(nB + 7) / 8, 256, 0, p->stream>>>(p->Z2, p->P, p->av, p->bv, p->wv, nB, inv_n, p->G2, p->A2,
                                                   p->gy, p->lossv, p->yv, p->G2a, p->G2Ta);
  TPB_CUDA(cudaGetLastError());
  head_sums_kernel<<<1, H, 0, p->stream>>>(p->G2, p->A2, p->gy, p->lossv, nB, p->G, p->dloss);
  TPB_CUDA(cudaGetLastError());
  if (!grads) return SBD_TPB_OK;
  const int splits = std::max(1, nB / 512);
  TPB_CHECK(gemm(p, p->G2Ta, p->A1bT, H, nB, H, splits, p->G + oW2));
  TPB_CHECK(gemm(p, p->G2a, p->W2Tp, nB, H, H, 1, p->dA1));
  act1_bwd_kernel<<<(unsigned)(((size_t)nB * H + 255) / 256), 256, 0, p->stream>>>(p->dA1, p->Z1, nB, p->G1Ta);
  TPB_CUDA(cudaGetLastError());
  colsum_kernel<<<1, H, 0, p->stream>>>(p->dA1, nB, p->G + ob1);
  TPB_CUDA(cudaGetLastError());
  TPB_CHECK(gemm(p, p->G1Ta, p->XbT, H, nB, F, splits, p->G + oW1));
  return SBD_TPB_OK;
}

SampleView view_of(const sbd_tpb_precond::Set &s) {
  return SampleView{s.fe, s.fr, s.a, s.b, s.w, s.oa, s.ob};
}

int grow_set(sbd_tpb_precond::Set &s, size_t need, cudaStream_t st) {
  if (s.cap >= need) return SBD_TPB_OK;
  const size_t cap = std::max(need, s.cap * 2);
  sbd_tpb_precond::Set t;
  TPB_CUDA(cudaMalloc(&t.fe, cap * 4));
  TPB_CUDA(cudaMalloc(&t.fr, cap * 4));
  TPB_CUDA(cudaMalloc(&t.a, cap * 4));
  TPB_CUDA(cudaMalloc(&t.b, cap * 4));
  TPB_CUDA(cudaMalloc(&t.w, cap * 4));
  TPB_CUDA(cudaMalloc(&t.oa, cap * 4));
  TPB_CUDA(cudaMalloc(&t.ob, cap * 4));
  if (s.n) {
    TPB_CUDA(cudaMemcpyAsync(t.fe, s.fe, s.n * 4, cudaMemcpyDeviceToDevice, st));
    TPB_CUDA(cudaMemcpyAsync(t.fr, s.fr, s.n * 4, cudaMemcpyDeviceToDevice, st));
    TPB_CUDA(cudaMemcpyAsync(t.a, s.a, s.n * 4, cudaMemcpyDeviceToDevice, st));
    TPB_CUDA(cudaMemcpyAsync(t.b, s.b, s.n * 4, cudaMemcpyDeviceToDevice, st));
    TPB_CUDA(cudaMemcpyAsync(t.w, s.w, s.n * 4, cudaMemcpyDeviceToDevice, st));
    TPB_CUDA(cudaMemcpyAsync(t.oa, s.oa, s.n * 4, cudaMemcpyDeviceToDevice, st));
    TPB_CUDA(cudaMemcpyAsync(t.ob, s.ob, s.n * 4, cudaMemcpyDeviceToDevice, st));
    TPB_CUDA(cudaStreamSynchronize(st));
  }
  t.n = s.n;
  t.cap = cap;
  free_set(s);
  s = t;
  t = sbd_tpb_precond::Set();
  return SBD_TPB_OK;
}

// pair index of the 8-fold packed integral store: (ij) = max(i,j)(max(i,j)+1)/2 + min(i,j)
inline size_t pair_of(size_t i, size_t j) { return i > j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

// Per string: the occupation window around the Fermi level and the sum of the exchange integrals
// (pq|qp) over its occupied pairs (what separates H_ii from the spin-free diagonal).
int ensure_occ_windows(sbd_tpb_handle *h) {
  if (h->d_occw_a) return SBD_TPB_OK;
  const int L = h->L;
  auto win = [](const std::vector<uint64_t> &v) {
    std::vector<uint32_t> o(v.size());
    const int nel = v.empty() ? 0 : __builtin_popcountll(v[0]);
    for (size_t i = 0; i < v.size(); i++) o[i] = occ_window(v[i], nel);
    return o;
  };
  auto exch = [&](const std::vector<uint64_t> &v) {
    std::vector<double> o(v.size(), 0.0);
    for (size_t i = 0; i < v.size(); i++)
      for (int p = 0; p < L; p++)
        if ((v[i] >> p) & 1)
          for (int q = p + 1; q < L; q++)
            if ((v[i] >> q) & 1) {
              const size_t pq = pair_of(p, q);
              o[i] += h->eri_packed[pair_of(pq, pq)];
            }
    return o;
  };
  const std::vector<uint32_t> a = win(h->astr), b = win(h->bstr);
  const std::vector<double> ka = exch(h->astr), kb = exch(h->bstr);
  TPB_CUDA(cudaMalloc(&h->d_occw_a, sizeof(uint32_t) * std::max<size_t>(1, a.size())));
  TPB_CUDA(cudaMalloc(&h->d_occw_b, sizeof(uint32_t) * std::max<size_t>(1, b.size())));
  TPB_CUDA(cudaMalloc(&h->d_kx_a, sizeof(double) * std::max<size_t>(1, ka.size())));
  TPB_CUDA(cudaMalloc(&h->d_kx_b, sizeof(double) * std::max<size_t>(1, kb.size())));
  TPB_CUDA(cudaMemcpy(h->d_occw_a, a.data(), sizeof(uint32_t) * a.size(), cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(h->d_occw_b, b.data(), sizeof(uint32_t) * b.size(), cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(h->d_kx_a, ka.data(), sizeof(double) * ka.size(), cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(h->d_kx_b, kb.data(), sizeof(double) * kb.size(), cudaMemcpyHostToDevice));
  return SBD_TPB_OK;
}

// Training pairs of recorded step k appended to set s.  gpsi[j] = vec_j . Psi for every basis vector.
int add_step_pairs(sbd_tpb_precond *p, sbd_tpb_handle *h, const DavRecord &rec, size_t k, const double *Psi,
                   const std::vector<double> &gpsi, size_t samples, sbd_tpb_precond::Set &s) {
  const size_t n = h->ndet();
  const int nblk = h->num_sms * 4;
  const std::vector<int> &bas = rec.basis[k];
  if (bas.empty() || (int)bas.size() > kMaxBasis) return SBD_TPB_OK;
  PairArgs a{};
  a.d = rec.d[k];
  a.Psi = Psi;
  a.m = (int)bas.size();
  double g2 = 0.0;  // sum_j (C_j . Psi)^2
  for (int j = 0; j < a.m; j++) {
    const double sc = rec.scale[bas[j]], cj = sc * gpsi[bas[j]];
    a.C[j] = rec.vec[bas[j]];
    a.g[j] = cj * sc;
    g2 += cj * cj;
  }
  a.e0 = rec.e0[k];
  a.seed = p->seed * 0x9E3779B97F4A7C15ull + (uint64_t)(p->steps_seen++) * 0xD1B54A32D192ED03ull + 0x1234567ull;
  double *part = nullptr;
  uint8_t *flags = nullptr;
  uint32_t *counts = nullptr;
  uint64_t *offs = nullptr;
  TPB_CUDA(cudaMalloc(&part, sizeof(double) * ((kMaxBasis + 4) * (size_t)nblk + kMaxBasis + 4)));
  double *res = part + (kMaxBasis + 4) * (size_t)nblk;
  int rc = SBD_TPB_OK;
  do {
    // C_j . d for the projection of d
    double cd[kMaxBasis];
    basis_dots_kernel<<<nblk, 256, 0, h->stream>>>(a, Psi, a.d, n, a.m, part);
    sum_partials_kernel<<<1, 32, 0, h->stream>>>(part, nblk, a.m, res);
    if (cudaMemcpyAsync(cd, res, sizeof(double) * a.m, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
      rc = fail(SBD_TPB_ERR_CUDA, "precond collect: basis dots");
      break;
    }
    for (int j = 0; j < a.m; j++) {
      const double sc = rec.scale[bas[j]];
      a.hd[j] = sc * sc * cd[j];
    }
    double sums[4];
    pair_sums_kernel<<<nblk, 256, 0, h->stream>>>(a, n, 0, part);
    sum_partials_kernel<<<1, 32, 0, h->stream>>>(part, nblk, 4, res);
    if (cudaMemcpyAsync(sums, res, sizeof(sums), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
      rc = fail(SBD_TPB_ERR_CUDA, "precond collect: sums");
      break;
    }
    const double dd = sums[0], pdpd = sums[1], pdPsi = sums[2], pp = 1.0 - g2;
    if (!(dd > 0.0) || !(pdpd > 1e-30 * dd) || !(pp > 1e-14)) break;  // nothing to learn from this step
    a.inv_dn = 1.0 / std::sqrt(dd);
    a.alpha = pdPsi / pp;
    pair_sums_kernel<<<nblk, 256, 0, h->stream>>>(a, n, 1, part);
    sum_partials_kernel<<<1, 32, 0, h->stream>>>(part, nblk, 4, res);
    if (cudaMemcpyAsync(sums, res, sizeof(sums), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
      rc = fail(SBD_TPB_ERR_CUDA, "precond collect: sums");
      break;
    }
    if (!(sums[3] > 0.0)) break;
    a.c = (double)samples / sums[3];
    const size_t chunk = (n + nblk - 1) / nblk;
    if (cudaMalloc(&flags, n) != cudaSuccess || cudaMalloc(&counts, sizeof(uint32_t) * nblk) != cudaSuccess ||
        cudaMalloc(&offs, sizeof(uint64_t) * nblk) != cudaSuccess) {
      rc = fail(SBD_TPB_ERR_OOM, "precond collect: flags");
      break;
    }
    pair_flag_kernel<<<nblk, 256, 0, h->stream>>>(a, n, chunk, flags, counts);
    std::vector<uint32_t> cnt(nblk);
    if (cudaMemcpyAsync(cnt.data(), counts, sizeof(uint32_t) * nblk, cudaMemcpyDeviceToHost, h->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
      rc = fail(SBD_TPB_ERR_CUDA, "precond collect: counts");
      break;
    }
    std::vector<uint64_t> off(nblk);
    uint64_t tot = 0;
    for (int b = 0; b < nblk; b++) {
      off[b] = s.n + tot;
      tot += cnt[b];
    }
    if ((rc = grow_set(s, s.n + tot, h->stream)) != SBD_TPB_OK) break;
    if (cudaMemcpyAsync(offs, off.data(), sizeof(uint64_t) * nblk, cudaMemcpyHostToDevice, h->stream) !=
        cudaSuccess) {
      rc = fail(SBD_TPB_ERR_CUDA, "precond collect: offsets");
      break;
    }
    SampleOut o{s.fe, s.fr, s.a, s.b, s.w, s.oa, s.ob};
    pair_write_kernel<<<nblk, 256, 0, h->stream>>>(a, h->d_hii, h->d_kx_a, h->d_kx_b, h->d_occw_a, h->d_occw_b,
                                                   (uint32_t)h->bstr.size(), n, chunk, flags, offs, o);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
      rc = fail(SBD_TPB_ERR_CUDA, "precond collect: write");
      break;
    }
    s.n += tot;
  } while (0);
  cudaFree(part);
  if (flags) cudaFree(flags);
  if (counts) cudaFree(counts);
  if (offs) cudaFree(offs);
  return rc;
}

// vec_j . Psi for every recorded basis vector
int basis_psi_dots(sbd_tpb_handle *h, const DavRecord &rec, const double *Psi, std::vector<double> &out) {
  const size_t n = h->ndet();
  const int nblk = h->num_sms * 4;
  out.assign(rec.vec.size(), 0.0);
  double *part = nullptr;
  TPB_CUDA(cudaMalloc(&part, sizeof(double) * (kMaxBasis * (size_t)nblk + kMaxBasis)));
  double *res = part + kMaxBasis * (size_t)nblk;
  int rc = SBD_TPB_OK;
  for (size_t j0 = 0; j0 < rec.vec.size() && rc == SBD_TPB_OK; j0 += kMaxBasis) {
    const int nv = (int)std::min<size_t>(kMaxBasis, rec.vec.size() - j0);
    PairArgs a{};
    for (int j = 0; j < nv; j++) a.C[j] = rec.vec[j0 + j];
    basis_dots_kernel<<<nblk, 256, 0, h->stream>>>(a, Psi, nullptr, n, nv, part);
    sum_partials_kernel<<<1, 32, 0, h->stream>>>(part, nblk, nv, res);
    if (cudaMemcpyAsync(out.data() + j0, res, sizeof(double) * nv, cudaMemcpyDeviceToHost, h->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
      rc = fail(SBD_TPB_ERR_CUDA, "precond collect: basis dots");
  }
  cudaFree(part);
  return rc;
}

}  // namespace

template <typename T>
int precond_apply(sbd_tpb_handle *h, sbd_tpb_precond *p, T *t, double e0, double rnorm, double tt) {
  TPB_CHECK(ensure_occ_windows(h));
  InferArgs a{};
  a.hii = h->d_hii;
  a.kxa = h->d_kx_a;
  a.kxb = h->d_kx_b;
  a.e0 = e0;
  (void)rnorm;  // the residual-entry input is held at zero (spin symmetry)
  a.occ_a = h->d_occw_a;
  a.occ_b = h->d_occw_b;
  a.nb = (uint32_t)h->bstr.size();
  const size_t n = h->ndet();
  a.idx = nullptr;
  a.count = n;
  if (n > kMlpBudget && tt > 0.0 && n < ((size_t)1 << 32)) {
    // correct only the entries that carry the correction: |d_i| >= |d| / sqrt(budget)
    if (!h->d_mlp_idx) {
      TPB_CUDA(cudaMalloc(&h->d_mlp_idx, sizeof(uint32_t) * kMlpBudget + sizeof(unsigned long long)));
    }
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(h->d_mlp_idx + kMlpBudget);
    TPB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), h->stream));
    select_kernel<T><<<h->num_sms * 8, 256, 0, h->stream>>>(t, n, std::sqrt(tt / (double)kMlpBudget),
                                                            h->d_mlp_idx, (uint32_t)kMlpBudget, cnt);
    TPB_LAUNCHED(h);
    unsigned long long c = 0;
    TPB_CUDA(cudaMemcpyAsync(&c, cnt, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
    TPB_CUDA(cudaStreamSynchronize(h->stream));
    a.idx = h->d_mlp_idx;
    a.count = (size_t)std::min<unsigned long long>(c, kMlpBudget);
    if (a.count == 0) return SBD_TPB_OK;
  }
  a.W1p = p->W1p;
  a.W2p = p->W2p;
  a.P = p->P;
  a.err = p->err;
  if (kSmInfer > h->smem_optin) return fail(SBD_TPB_ERR_INVALID, "learned preconditioner: shared memory");
  TPB_CUDA(cudaFuncSetAttribute(mlp_infer_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmInfer));
  const size_t ntiles = (a.count + 127) / 128;
  const unsigned grid = (unsigned)std::min<size_t>(ntiles, (size_t)h->num_sms);
  // the weights may have been written on the preconditioner's stream
  TPB_CUDA(cudaStreamSynchronize(p->stream));
  mlp_infer_kernel<T><<<grid, kInfThreads, kSmInfer, h->stream>>>(a, t);
  TPB_LAUNCHED(h);
  int e = 0;
  TPB_CUDA(cudaMemcpyAsync(&e, p->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  if (e) {
    cudaMemset(p->err, 0, sizeof(int));
    return fail(SBD_TPB_ERR_CUDA, "learned preconditioner: tensor-core wait expired (code " + std::to_string(e) + ")");
  }
  return SBD_TPB_OK;
}

template int precond_apply<double>(sbd_tpb_handle *, sbd_tpb_precond *, double *, double, double, double);
template int precond_apply<float>(sbd_tpb_handle *, sbd_tpb_precond *, float *, double, double, double);

int precond_collect(sbd_tpb_precond *p, sbd_tpb_handle *h, const sbd_tpb_params *prm, size_t samples, int role,
                    double *energy) {
  TPB_CHECK(ensure_occ_windows(h));
  DavRecord rec;
  double *Psi = nullptr;
  TPB_CUDA(cudaMalloc(&Psi, sizeof(double) * h->ndet()));
  double E = 0.0;
  // a run with the learned correction collects pairs along the learned solver's own trajectory
  int rc = davidson_record(h, prm, &rec, Psi, &E, prm->preconditioner == SBD_TPB_PRECOND_LEARNED ? p : nullptr);
  std::vector<double> gpsi;
  if (rc == SBD_TPB_OK) rc = basis_psi_dots(h, rec, Psi, gpsi);
  for (size_t k = 0; rc == SBD_TPB_OK && k < rec.d.size(); k++)
    rc = add_step_pairs(p, h, rec, k, Psi, gpsi, samples, p->set[role]);
  cudaFree(Psi);
  if (energy) *energy = E;
  return rc;
}

}  // namespace sbdtpb

sbd_tpb_precond::~sbd_tpb_precond() {
  using namespace sbdtpb;
  if (device >= 0) cudaSetDevice(device);
  free_set(set[0]);
  free_set(set[1]);
  free_batch(this);
  free_dev(P);
  free_dev(G);
  free_dev(m);
  free_dev(v);
  free_dev(W1p);
  free_dev(W2p);
  free_dev(W2Tp);
  free_dev(err);
  free_dev(Dp);
  free_dev(dloss);
  free_dev(xraw);
  if (stream) cudaStreamDestroy(stream);
}

// ==================================================================== C ABI
using namespace sbdtpb;

extern "C" int sbd_tpb_precond_create(int device, uint64_t seed, sbd_tpb_precond **out) {
  if (!out) return fail(SBD_TPB_ERR_INVALID, "null output");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return fail(SBD_TPB_ERR_NO_DEVICE, "precond: no such CUDA device");
  cudaDeviceProp prop;
  TPB_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) return fail(SBD_TPB_ERR_NO_DEVICE, "precond: needs an sm_100 device");
  TPB_CUDA(cudaSetDevice(device));
  sbd_tpb_precond *p = new sbd_tpb_precond();
  p->device = device;
  p->seed = seed;
  p->num_sms = prop.multiProcessorCount;
  int rc = SBD_TPB_OK;
  auto al = [&](auto **ptr, size_t bytes) {
    if (rc == SBD_TPB_OK && cudaMalloc(ptr, bytes) != cudaSuccess) rc = fail(SBD_TPB_ERR_OOM, "precond: cudaMalloc");
  };
  if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess)
    rc = fail(SBD_TPB_ERR_CUDA, "precond: stream");
  al(&p->P, kParams * 4);
  al(&p->G, kParams * 4);
  al(&p->m, kParams * 4);
  al(&p->v, kParams * 4);
  al(&p->W1p, (size_t)H * F * 2);
  al(&p->W2p, (size_t)H * H * 2);
  al(&p->W2Tp, (size_t)H * H * 2);
  al(&p->err, sizeof(int));
  al(&p->dloss, sizeof(double));
  if (rc != SBD_TPB_OK) {
    delete p;
    return rc;
  }
  // He-style initialisation of W1 (real inputs only) and W2; w3 = b3 = 0 (the diagonal)
  std::vector<float> P(kParams, 0.f);
  std::mt19937_64 g(seed);
  std::normal_distribution<float> n1(0.f, std::sqrt(2.f / 50.f)), n2(0.f, std::sqrt(2.f / H));
  for (int o = 0; o < H; o++)
    for (int k = 0; k < 2 + 2 * kMlpWin; k++) P[oW1 + (size_t)o * F + k] = n1(g);
  for (size_t i = 0; i < (size_t)H * H; i++) P[oW2 + i] = n2(g);
  cudaMemcpy(p->P, P.data(), kParams * 4, cudaMemcpyHostToDevice);
  cudaMemset(p->m, 0, kParams * 4);
  cudaMemset(p->v, 0, kParams * 4);
  cudaMemset(p->G, 0, kParams * 4);
  cudaMemset(p->err, 0, sizeof(int));
  if (pack_weights(p) != SBD_TPB_OK || cudaStreamSynchronize(p->stream) != cudaSuccess) {
    delete p;
    return fail(SBD_TPB_ERR_CUDA, "precond: init");
  }
  *out = p;
  return SBD_TPB_OK;
}

extern "C" int sbd_tpb_precond_destroy(sbd_tpb_precond *p) {
  delete p;
  return SBD_TPB_OK;
}

extern "C" int sbd_tpb_precond_collect(sbd_tpb_precond *p, sbd_tpb_handle *h, const sbd_tpb_params *params,
                                       size_t samples_per_step, int role, double *energy) {
  if (!p || !h || !params) return fail(SBD_TPB_ERR_INVALID, "null argument");
  if (role != 0 && role != 1) return fail(SBD_TPB_ERR_INVALID, "role must be 0 or 1");
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  if (h->device != p->device) return fail(SBD_TPB_ERR_INVALID, "handle and preconditioner on different devices");
  TPB_CUDA(cudaSetDevice(h->device));
  return precond_collect(p, h, params, samples_per_step, role, energy);
}

extern "C" int sbd_tpb_precond_num_samples(sbd_tpb_precond *p, int role, size_t *n) {
  if (!p || !n || (role != 0 && role != 1)) return fail(SBD_TPB_ERR_INVALID, "bad argument");
  *n = p->set[role].n;
  return SBD_TPB_OK;
}

extern "C" int sbd_tpb_precond_train(sbd_tpb_precond *p, int epochs, int batch, double lr, double *last_loss) {
  if (!p || epochs < 0 || batch < 128 || batch % 128) return fail(SBD_TPB_ERR_INVALID, "bad argument");
  TPB_CUDA(cudaSetDevice(p->device));
  const sbd_tpb_precond::Set &s = p->set[0];
  if (s.n == 0) return fail(SBD_TPB_ERR_STATE, "precond: no training pairs collected");
  TPB_CHECK(ensure_batch(p, batch));
  uint32_t *idx = nullptr;
  TPB_CUDA(cudaMalloc(&idx, sizeof(uint32_t) * s.n));
  std::vector<uint32_t> perm(s.n);
  std::iota(perm.begin(), perm.end(), 0u);
  std::mt19937_64 g(p->seed ^ 0xA5A5A5A5ull);
  double loss = 0.0;
  int rc = SBD_TPB_OK;
  for (int ep = 0; ep < epochs && rc == SBD_TPB_OK; ep++) {
    std::shuffle(perm.begin(), perm.end(), g);
    if (cudaMemcpyAsync(idx, perm.data(), sizeof(uint32_t) * s.n, cudaMemcpyHostToDevice, p->stream) !=
        cudaSuccess) {
      rc = fail(SBD_TPB_ERR_CUDA, "precond train: upload");
      break;
    }
    for (size_t base = 0; base < s.n && rc == SBD_TPB_OK; base += batch) {
      const size_t real = std::min<size_t>(batch, s.n - base);
      pack_batch_kernel<<<(batch + 127) / 128, 128, 0, p->stream>>>(view_of(s), nullptr, idx, base, s.n, batch,
                                                                     p->Xa, p->XbT, p->av, p->bv, p->wv);
      if ((rc = fwd_bwd(p, batch, 1.f / (float)real, true)) != SBD_TPB_OK) break;
      p->adam_t++;
      const float c1 = 1.f - std::pow(0.9f, (float)p->adam_t), c2 = 1.f - std::pow(0.999f, (float)p->adam_t);
      adam_kernel<<<(unsigned)((kParams + 255) / 256), 256, 0, p->stream>>>(p->P, p->G, p->m, p->v, kParams,
                                                                            (float)lr, c1, c2);
      if ((rc = pack_weights(p)) != SBD_TPB_OK) break;
    }
    if (rc == SBD_TPB_OK) {
      if (cudaMemcpyAsync(&loss, p->dloss, sizeof(double), cudaMemcpyDeviceToHost, p->stream) != cudaSuccess)
        rc = fail(SBD_TPB_ERR_CUDA, "precond train: loss");
      else
        rc = check_err(p, "precond train");
    }
  }
  cudaFree(idx);
  TPB_CHECK(rc);
  TPB_CUDA(cudaStreamSynchronize(p->stream));
  if (last_loss) *last_loss = loss;
  return SBD_TPB_OK;
}

extern "C" int sbd_tpb_precond_evaluate(sbd_tpb_precond *p, int role, double *loss_learned, double *loss_diagonal) {
  if (!p || (role != 0 && role != 1)) return fail(SBD_TPB_ERR_INVALID, "bad argument");
  TPB_CUDA(cudaSetDevice(p->device));
  const sbd_tpb_precond::Set &s = p->set[role];
  const int batch = 8192;
  TPB_CHECK(ensure_batch(p, batch));
  double ll = 0.0, ld = 0.0;
  std::vector<float> y(batch), av(batch), bv(batch), wv(batch);
  for (size_t base = 0; base < s.n; base += batch) {
    const int real = (int)std::min<size_t>(batch, s.n - base);
    pack_batch_kernel<<<(batch + 127) / 128, 128, 0, p->stream>>>(view_of(s), nullptr, nullptr, base, s.n, batch,
                                                                   p->Xa, p->XbT, p->av, p->bv, p->wv);
    TPB_CHECK(fwd_bwd(p, batch, 1.f, false));
    TPB_CUDA(cudaMemcpyAsync(y.data(), p->yv, 4 * real, cudaMemcpyDeviceToHost, p->stream));
    TPB_CUDA(cudaMemcpyAsync(av.data(), p->av, 4 * real, cudaMemcpyDeviceToHost, p->stream));
    TPB_CUDA(cudaMemcpyAsync(bv.data(), p->bv, 4 * real, cudaMemcpyDeviceToHost, p->stream));
    TPB_CUDA(cudaMemcpyAsync(wv.data(), p->wv, 4 * real, cudaMemcpyDeviceToHost, p->stream));
    TPB_CUDA(cudaStreamSynchronize(p->stream));
    for (int r = 0; r < real; r++) {
      const double el = av[r] * (1.0 + y[r]) - bv[r], ed = (double)av[r] - bv[r];
      ll += wv[r] * el * el;
      ld += wv[r] * ed * ed;
    }
  }
  TPB_CHECK(check_err(p, "precond evaluate"));
  if (loss_learned) *loss_learned = ll;
  if (loss_diagonal) *loss_diagonal = ld;
  return SBD_TPB_OK;
}

extern "C" int sbd_tpb_precond_get_params(sbd_tpb_precond *p, float *params, size_t n) {
  if (!p || !params || n != kParams) return fail(SBD_TPB_ERR_INVALID, "bad argument");
  TPB_CUDA(cudaSetDevice(p->device));
  TPB_CUDA(cudaMemcpyAsync(params, p->P, kParams * 4, cudaMemcpyDeviceToHost, p->stream));
  TPB_CUDA(cudaStreamSynchronize(p->stream));
  return SBD_TPB_OK;
}

extern "C" int sbd_tpb_precond_set_params(sbd_tpb_precond *p, const float *params, size_t n) {
  if (!p || !params || n != kParams) return fail(SBD_TPB_ERR_INVALID, "bad argument");
  TPB_CUDA(cudaSetDevice(p->device));
  TPB_CUDA(cudaMemcpyAsync(p->P, params, kParams * 4, cudaMemcpyHostToDevice, p->stream));
  TPB_CHECK(pack_weights(p));
  TPB_CUDA(cudaStreamSynchronize(p->stream));
  return SBD_TPB_OK;
}

extern "C" int sbd_tpb_precond_gradients(sbd_tpb_precond *p, size_t n, const float *x, const float *a,
                                         const float *b, const float *w, float *grad, double *loss, float *y) {
  if (!p || !x || !a || !b || !w || n == 0 || n > (1u << 20)) return fail(SBD_TPB_ERR_INVALID, "bad argument");
  TPB_CUDA(cudaSetDevice(p->device));
  const int nB = (int)((n + 127) / 128 * 128);
  TPB_CHECK(ensure_batch(p, nB));
  const size_t need = n * F + 3 * n;
  if (p->xraw_cap < need) {
    free_dev(p->xraw);
    p->xraw_cap = 0;
    TPB_CUDA(cudaMalloc(&p->xraw, need * 4));
    p->xraw_cap = need;
  }
  float *xa = p->xraw, *aa = xa + n * F, *ba = aa + n, *wa = ba + n;
  TPB_CUDA(cudaMemcpyAsync(xa, x, n * F * 4, cudaMemcpyHostToDevice, p->stream));
  TPB_CUDA(cudaMemcpyAsync(aa, a, n * 4, cudaMemcpyHostToDevice, p->stream));
  TPB_CUDA(cudaMemcpyAsync(ba, b, n * 4, cudaMemcpyHostToDevice, p->stream));
  TPB_CUDA(cudaMemcpyAsync(wa, w, n * 4, cudaMemcpyHostToDevice, p->stream));
  SampleView v{nullptr, nullptr, aa, ba, wa, nullptr, nullptr};
  pack_batch_kernel<<<(nB + 127) / 128, 128, 0, p->stream>>>(v, xa, nullptr, 0, n, nB, p->Xa, p->XbT, p->av, p->bv,
                                                             p->wv);
  TPB_CUDA(cudaGetLastError());
  TPB_CHECK(fwd_bwd(p, nB, 1.f / (float)n, true));
  if (grad) TPB_CUDA(cudaMemcpyAsync(grad, p->G, kParams * 4, cudaMemcpyDeviceToHost, p->stream));
  if (y) TPB_CUDA(cudaMemcpyAsync(y, p->yv, n * 4, cudaMemcpyDeviceToHost, p->stream));
  double l = 0.0;
  TPB_CUDA(cudaMemcpyAsync(&l, p->dloss, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  TPB_CHECK(check_err(p, "precond gradients"));
  if (loss) *loss = l;
  return SBD_TPB_OK;
}

extern "C" int sbd_tpb_precond_apply(sbd_tpb_handle *h, sbd_tpb_precond *p, const double *d, double e0,
                                     double rnorm, double *t) {
  if (!h || !p || !d || !t) return fail(SBD_TPB_ERR_INVALID, "null argument");
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  if (h->device != p->device) return fail(SBD_TPB_ERR_INVALID, "handle and preconditioner on different devices");
  TPB_CUDA(cudaSetDevice(h->device));
  const size_t n = h->ndet();
  double *dv = nullptr;
  TPB_CUDA(cudaMalloc(&dv, n * sizeof(double)));
  int rc = SBD_TPB_OK;
  if (cudaMemcpyAsync(dv, d, n * sizeof(double), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
    rc = fail(SBD_TPB_ERR_CUDA, "precond apply: upload");
  double tt = 0.0;  // |d|^2: beyond the budget only the large entries are corrected
  for (size_t i = 0; i < n; i++) tt += d[i] * d[i];
  if (rc == SBD_TPB_OK) rc = precond_apply<double>(h, p, dv, e0, rnorm, tt);
  if (rc == SBD_TPB_OK && (cudaMemcpyAsync(t, dv, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
                           cudaStreamSynchronize(h->stream) != cudaSuccess))
    rc = fail(SBD_TPB_ERR_CUDA, "precond apply: download");
  cudaFree(dv);
  return rc;
}

extern "C" int sbd_tpb_set_preconditioner(sbd_tpb_handle *h, sbd_tpb_precond *p) {
  if (!h) return fail(SBD_TPB_ERR_INVALID, "null handle");
  if (p && p->device != h->device) return fail(SBD_TPB_ERR_INVALID, "handle and preconditioner on different devices");
  h->precond = p;
  return SBD_TPB_OK;
}
