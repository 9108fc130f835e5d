// Davidson vector kernels.
//
// The reference runs each Davidson vector operation as its own pass (2k+1 AXPYs, k dots, a
// normalize; tpb/davidson.h:758-880, basic/davidson_thrust.h:176-330) with one device->host sync
// per dot product (framework/cuda_reduce.h:17-174).  Here the passes are fused: one kernel reads
// all k subspace vectors once and produces W, the residual, the preconditioned correction and
// the first Gram-Schmidt overlaps together.  Dot products accumulate in FP64 whatever the
// storage type, per block in a fixed order, and the block partials are summed in a fixed order
// by a second kernel, so every reduction is run-to-run deterministic.
#include <algorithm>
#include <type_traits>

#include "tpb_common.cuh"
#include "vecops.cuh"

namespace sbdtpb {
namespace {

template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], int nv, double *partials,
                                                   int nblocks) {
  __shared__ double red[32][NV];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; j++) {
    double x = v[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[wid][j] = x;
  }
  __syncthreads();
  if (threadIdx.x < nv) {
    double s = 0.0;
    for (int w = 0; w < nw; w++) s += red[w][threadIdx.x];
    partials[(size_t)threadIdx.x * nblocks + blockIdx.x] = s;
  }
}

// W consecutive elements: one 16-byte access when W = 16 / sizeof(T), scalars when W = 1 (tail)
template <typename T, int W>
__device__ __forceinline__ void ldv(const T *__restrict__ p, T (&v)[W]) {
  if constexpr (W == 4 && sizeof(T) == 4) {
    const float4 f = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = f.x, v[1] = f.y, v[2] = f.z, v[3] = f.w;
  } else if constexpr (W == 2 && sizeof(T) == 8) {
    const double2 f = __ldg(reinterpret_cast<const double2 *>(p));
    v[0] = f.x, v[1] = f.y;
  } else {
#pragma unroll
    for (int l = 0; l < W; l++) v[l] = __ldg(p + l);
  }
}
template <typename T, int W>
__device__ __forceinline__ void stv(T *__restrict__ p, const T (&v)[W]) {
  if constexpr (W == 4 && sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else if constexpr (W == 2 && sizeof(T) == 8) {
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
  } else {
#pragma unroll
    for (int l = 0; l < W; l++) p[l] = v[l];
  }
}

// Every vector pass walks the vectors in 16-byte groups (grid-stride), and block 0 finishes the
// n % VW tail element by element; `body<W>(i)` handles elements i .. i+W-1.
template <typename T, typename Body>
__device__ __forceinline__ void for_each_group(size_t n, Body &&body) {
  constexpr int VW = 16 / sizeof(T);
  const size_t ng = n / VW;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < ng; g += (size_t)gridDim.x * blockDim.x)
    body.template run<VW>(g * VW);
  if (blockIdx.x == 0 && threadIdx.x < n - ng * VW) body.template run<1>(ng * VW + threadIdx.x);
}

// out[j] = X_j . y, j < K
template <typename T, int K>
struct DotBody {
  const VecPtrs<T> &X;
  const T *y;
  double (&acc)[K];
  template <int W>
  __device__ __forceinline__ void run(size_t i) {
    T yv[W];
    ldv<T, W>(y + i, yv);
#pragma unroll
    for (int j = 0; j < K; j++) {
      T xv[W];
      ldv<T, W>(X.p[j] + i, xv);
#pragma unroll
      for (int l = 0; l < W; l++) acc[j] += (double)xv[l] * (double)yv[l];
    }
  }
};

template <typename T, int K>
__global__ void __launch_bounds__(kVecThreads)
    multi_dot_kernel(VecPtrs<T> X, const T *__restrict__ y, size_t n, double *partials) {
  double acc[K];
#pragma unroll
  for (int j = 0; j < K; j++) acc[j] = 0.0;
  DotBody<T, K> b{X, y, acc};
  for_each_group<T>(n, b);
  block_reduce_store<K>(acc, K, partials, gridDim.x);
}

__global__ void reduce_partials_kernel(const double *__restrict__ partials, int nblocks,
                                       double *__restrict__ out) {
  __shared__ double s[256];
  const double *p = partials + (size_t)blockIdx.x * nblocks;
  double x = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) x += p[i];
  s[threadIdx.x] = x;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

// W = sum_k u_k S_k ; r = E' W - sum_k u_k sigma(S_k) ; t = r / (E0 - H_ii) (regularised as
// tpb/davidson.h:861-868) ; partials: [0] = W.W, [1] = r.r, [2+k] = S_k . t, [2+M] = t.t
template <typename T, int M>
struct ResidualBody {
  const ResidualArgs<T> &a;
  double (&acc)[M + 3];
  template <int W>
  __device__ __forceinline__ void run(size_t i) {
    T c[M][W];
    double w[W], hc[W];
#pragma unroll
    for (int l = 0; l < W; l++) w[l] = hc[l] = 0.0;
#pragma unroll
    for (int k = 0; k < M; k++) {
      T hv[W];
      ldv<T, W>(a.C.p[k] + i, c[k]);
      ldv<T, W>(a.HC.p[k] + i, hv);
#pragma unroll
      for (int l = 0; l < W; l++) {
        w[l] += a.u[k] * (double)c[k][l];
        hc[l] += a.u[k] * (double)hv[l];
      }
    }
    T wt[W], tt[W];
#pragma unroll
    for (int l = 0; l < W; l++) {
      const double r = a.e_shifted * w[l] - hc[l];
      wt[l] = (T)w[l];
      acc[0] += w[l] * w[l];
      acc[1] += r * r;
      if (a.t) {
        // E0 - H_ii, or with the FP32 diagonal (E0 - H_00) - (H_ii - H_00)
        const double d = a.hii32 ? a.e_shifted - (double)__ldg(&a.hii32[i + l]) : a.e0 - __ldg(&a.hii[i + l]);
        tt[l] = (T)((fabs(d) > 1.0e-12) ? r / d : r / (d - 1.0e-12));
      }
    }
    if (a.W) stv<T, W>(a.W + i, wt);
    if (a.t) {
      stv<T, W>(a.t + i, tt);
#pragma unroll
      for (int l = 0; l < W; l++) {
#pragma unroll
        for (int k = 0; k < M; k++) acc[2 + k] += (double)c[k][l] * (double)tt[l];
        acc[2 + M] += (double)tt[l] * (double)tt[l];
      }
    }
  }
};

template <typename T, int M>
__global__ void __launch_bounds__(kVecThreads) residual_kernel(ResidualArgs<T> a, size_t n, double *partials) {
  if (a.u_dev) {
    // Ritz coefficients and value of the device Rayleigh-Ritz solve
#pragma unroll
    for (int k = 0; k < M; k++) a.u[k] = __ldg(&a.u_dev[k]);
    a.e_shifted = __ldg(&a.e_dev[0]);
    a.e0 = a.e_shifted + a.shift;
  }
  double acc[M + 3];
#pragma unroll
  for (int j = 0; j < M + 3; j++) acc[j] = 0.0;
  ResidualBody<T, M> b{a, acc};
  for_each_group<T>(n, b);
  block_reduce_store<M + 3>(acc, M + 3, partials, gridDim.x);
}

// t -= sum_k o_k C_k ; partials: [0] = t.t, [1+k] = C_k . t (for a second Gram-Schmidt round)
template <typename T, int M, bool kDots>
struct CgsBody {
  const VecPtrs<T> &C;
  const double (&o)[M];
  T *t;
  double (&acc)[M + 1];
  template <int W>
  __device__ __forceinline__ void run(size_t i) {
    T tv[W], c[M][W];
    ldv<T, W>(t + i, tv);
    double x[W];
#pragma unroll
    for (int l = 0; l < W; l++) x[l] = (double)tv[l];
#pragma unroll
    for (int k = 0; k < M; k++) {
      ldv<T, W>(C.p[k] + i, c[k]);
#pragma unroll
      for (int l = 0; l < W; l++) x[l] -= o[k] * (double)c[k][l];
    }
    T xt[W];
#pragma unroll
    for (int l = 0; l < W; l++) {
      xt[l] = (T)x[l];
      acc[0] += (double)xt[l] * (double)xt[l];
      if (kDots) {
#pragma unroll
        for (int k = 0; k < M; k++) acc[1 + k] += (double)c[k][l] * (double)xt[l];
      }
    }
    stv<T, W>(t + i, xt);
  }
};

// o_k = co.v[k] * (ov ? ov[k] : 1): the overlaps may come straight from a device reduction
// pred (may be null): run only when pred[1] < 0.5 * pred[0] (the second Gram-Schmidt round, decided
// on the device from the first round's |t|^2 before and after); a skipped launch writes zero
// partials (its reduction is then 0 and nothing else changes)
template <typename T, int M, bool kDots>
__global__ void __launch_bounds__(kVecThreads)
    cgs_update_kernel(VecPtrs<T> C, CoefArray co, const double *__restrict__ ov, T *__restrict__ t, size_t n,
                      double *partials, const double *__restrict__ pred0 = nullptr,
                      const double *__restrict__ pred1 = nullptr) {
  double acc[M + 1];
#pragma unroll
  for (int j = 0; j < M + 1; j++) acc[j] = 0.0;
  if (pred0 && !(__ldg(pred1) < 0.5 * __ldg(pred0))) {
    if (threadIdx.x <= (kDots ? M : 0)) partials[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = 0.0;
    return;
  }
  double o[M];
#pragma unroll
  for (int k = 0; k < M; k++) o[k] = co.v[k] * (ov ? __ldg(&ov[k]) : 1.0);
  CgsBody<T, M, kDots> b{C, o, t, acc};
  for_each_group<T>(n, b);
  block_reduce_store<M + 1>(acc, kDots ? M + 1 : 1, partials, gridDim.x);
}

template <typename T>
__global__ void scale_kernel(T *__restrict__ x, double a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    x[i] = (T)((double)x[i] * a);
}

template <typename S, typename D>
__global__ void convert_kernel(const S *__restrict__ x, D *__restrict__ y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = (D)x[i];
}

// y = a*x + b*y
template <typename T>
__global__ void axpby_kernel(const T *__restrict__ x, T *__restrict__ y, double a, double b,
                             size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = (T)(a * (double)x[i] + b * (double)y[i]);
}

// t <- (t + t^T) / 2 for a square nb x nb vector (alpha and beta strings identical), in place,
// t <- (t + t^T) / 2 in place, one 32 x 32 tile pair (bi <= bj) at a time through shared memory;
// each thread moves VW consecutive elements of a tile row (one 16-byte access when VW = 16 /
// sizeof(T), which needs nb a multiple of VW; scalars when VW = 1).  partials[block] = sum of the
// new t^2 over the block's tile pairs (fixed assignment, so the sum is deterministic).  Measured
// at nb = 20,000: FP32 0.65 ms, FP64 1.10 ms (a plain copy of the same bytes: 0.55 / 1.09 ms);
// 64 x 64 tiles with scalar accesses, as before, took 1.30 / 1.62 ms.
constexpr int kSymTile = 32;
constexpr int kSymBlocksPerSm = 16;

// kAvg false: t <- t + t^T (the symmetric sigma's B + B^T), no norm.
template <typename T, int VW, bool kAvg = true>
__global__ void __launch_bounds__(256) symmetrize_kernel(T *__restrict__ t, uint32_t nb, double *partials) {
  constexpr int TS = kSymTile, TPR = TS / VW, RS = 256 / TPR;  // threads per tile row, row step
  __shared__ T A[TS][TS + 1], B[TS][TS + 1];
  const uint32_t nt = (nb + TS - 1) / TS;
  const size_t npairs = (size_t)nt * (nt + 1) / 2;
  const int cx = (threadIdx.x % TPR) * VW, ty = threadIdx.x / TPR;
  auto load = [&](const T *p, bool in, T (&v)[VW]) {
    if (!in) {
#pragma unroll
      for (int l = 0; l < VW; l++) v[l] = T(0);
    } else {
      ldv<T, VW>(p, v);
    }
  };
  double acc = 0.0;
  for (size_t p = blockIdx.x; p < npairs; p += gridDim.x) {
    // p -> (bi, bj), bi <= bj, row-major over the upper triangle
    uint32_t bi = (uint32_t)((2.0 * nt + 1.0 - sqrt((2.0 * nt + 1.0) * (2.0 * nt + 1.0) - 8.0 * (double)p)) / 2.0);
    while (bi > 0 && (size_t)bi * nt - (size_t)bi * (bi - 1) / 2 > p) bi--;
    while ((size_t)(bi + 1) * nt - (size_t)(bi + 1) * bi / 2 <= p) bi++;
    const uint32_t bj = bi + (uint32_t)(p - ((size_t)bi * nt - (size_t)bi * (bi - 1) / 2));
    __syncthreads();
#pragma unroll
    for (int r = ty; r < TS; r += RS) {
      // a group of VW columns is wholly in range or wholly out (nb is a multiple of VW)
      const uint32_t i = bi * TS + r, j = bj * TS + cx, i2 = bj * TS + r, j2 = bi * TS + cx;
      T va[VW], vb[VW];
      load(t + (size_t)i * nb + j, i < nb && j < nb, va);
      load(t + (size_t)i2 * nb + j2, i2 < nb && j2 < nb, vb);
#pragma unroll
      for (int l = 0; l < VW; l++) {
        A[r][cx + l] = va[l];
        B[r][cx + l] = vb[l];
      }
    }
    __syncthreads();
    const double mult = bi == bj ? 1.0 : 2.0;
#pragma unroll
    for (int r = ty; r < TS; r += RS) {
      // new A[r][c] = (A[r][c] + B[c][r]) / 2, written to both (i, j) and (j, i)
      const uint32_t i = bi * TS + r, j = bj * TS + cx;
      T v[VW];
#pragma unroll
      for (int l = 0; l < VW; l++)
        v[l] = kAvg ? (T)(((double)A[r][cx + l] + (double)B[cx + l][r]) * 0.5)
                    : (T)((double)A[r][cx + l] + (double)B[cx + l][r]);
      if (i < nb && j < nb) {
        stv<T, VW>(t + (size_t)i * nb + j, v);
        if (kAvg) {
#pragma unroll
          for (int l = 0; l < VW; l++) acc += mult * (double)v[l] * (double)v[l];
        }
      }
    }
    if (bi != bj) {
#pragma unroll
      for (int r = ty; r < TS; r += RS) {
        const uint32_t i2 = bj * TS + r, j2 = bi * TS + cx;
        T v[VW];
#pragma unroll
        for (int l = 0; l < VW; l++)
          v[l] = kAvg ? (T)(((double)A[cx + l][r] + (double)B[r][cx + l]) * 0.5)
                      : (T)((double)A[cx + l][r] + (double)B[r][cx + l]);
        if (i2 < nb && j2 < nb) stv<T, VW>(t + (size_t)i2 * nb + j2, v);
      }
    }
  }
  if (kAvg) {
    double v[1] = {acc};
    block_reduce_store<1>(v, 1, partials, gridDim.x);
  }
}

// t <- t + t^T in place (the symmetric sigma's B + B^T, tile pairs as symmetrize_kernel) and the
// block partials of S_k . t_new for k < m: S_k and the new t are exactly symmetric, so the (bj, bi)
// tile of a pair repeats the (bi, bj) tile's products and each off-diagonal pair is counted twice
// from its (bi, bj) tile (half the S_k bytes of a separate dot pass, and no second read of t).
// kAvg: t <- (t + t^T) / 2 (the exchange projection) and partial m is t_new . t_new.
template <typename T, int VW, bool kAvg = false>
__global__ void __launch_bounds__(256)
    sym_add_dots_kernel(T *__restrict__ t, uint32_t nb, VecPtrs<T> S, int m, double *partials) {
  constexpr int TS = kSymTile, TPR = TS / VW, RS = 256 / TPR;
  constexpr double kW = kAvg ? 0.5 : 1.0;
  __shared__ T A[TS][TS + 1], B[TS][TS + 1];
  const uint32_t nt = (nb + TS - 1) / TS;
  const size_t npairs = (size_t)nt * (nt + 1) / 2;
  const int cx = (threadIdx.x % TPR) * VW, ty = threadIdx.x / TPR;
  double acc[kMaxSub + 1];
#pragma unroll
  for (int k = 0; k <= kMaxSub; k++) acc[k] = 0.0;
  for (size_t p = blockIdx.x; p < npairs; p += gridDim.x) {
    uint32_t bi = (uint32_t)((2.0 * nt + 1.0 - sqrt((2.0 * nt + 1.0) * (2.0 * nt + 1.0) - 8.0 * (double)p)) / 2.0);
    while (bi > 0 && (size_t)bi * nt - (size_t)bi * (bi - 1) / 2 > p) bi--;
    while ((size_t)(bi + 1) * nt - (size_t)(bi + 1) * bi / 2 <= p) bi++;
    const uint32_t bj = bi + (uint32_t)(p - ((size_t)bi * nt - (size_t)bi * (bi - 1) / 2));
    __syncthreads();
#pragma unroll
    for (int r = ty; r < TS; r += RS) {
      const uint32_t i = bi * TS + r, j = bj * TS + cx, i2 = bj * TS + r, j2 = bi * TS + cx;
      T va[VW], vb[VW];
      if (i < nb && j < nb) ldv<T, VW>(t + (size_t)i * nb + j, va);
      else {
#pragma unroll
        for (int l = 0; l < VW; l++) va[l] = T(0);
      }
      if (i2 < nb && j2 < nb) ldv<T, VW>(t + (size_t)i2 * nb + j2, vb);
      else {
#pragma unroll
        for (int l = 0; l < VW; l++) vb[l] = T(0);
      }
#pragma unroll
      for (int l = 0; l < VW; l++) {
        A[r][cx + l] = va[l];
        B[r][cx + l] = vb[l];
      }
    }
    __syncthreads();
    const double mult = bi == bj ? 1.0 : 2.0;
#pragma unroll
    for (int r = ty; r < TS; r += RS) {
      const uint32_t i = bi * TS + r, j = bj * TS + cx;
      T v[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) v[l] = (T)(((double)A[r][cx + l] + (double)B[cx + l][r]) * kW);
      if (i < nb && j < nb) {
        stv<T, VW>(t + (size_t)i * nb + j, v);
        if (kAvg) {
          double d = 0.0;
#pragma unroll
          for (int l = 0; l < VW; l++) d += (double)v[l] * (double)v[l];
          acc[kMaxSub] += mult * d;
        }
#pragma unroll
        for (int k = 0; k < kMaxSub; k++) {
          if (k < m) {
            T sv[VW];
            ldv<T, VW>(S.p[k] + (size_t)i * nb + j, sv);
            double d = 0.0;
#pragma unroll
            for (int l = 0; l < VW; l++) d += (double)v[l] * (double)sv[l];
            acc[k] += mult * d;
          }
        }
      }
    }
    if (bi != bj) {
#pragma unroll
      for (int r = ty; r < TS; r += RS) {
        const uint32_t i2 = bj * TS + r, j2 = bi * TS + cx;
        T v[VW];
#pragma unroll
        for (int l = 0; l < VW; l++) v[l] = (T)(((double)A[cx + l][r] + (double)B[r][cx + l]) * kW);
        if (i2 < nb && j2 < nb) stv<T, VW>(t + (size_t)i2 * nb + j2, v);
      }
    }
  }
  if (kAvg) {
#pragma unroll
    for (int k = 0; k < kMaxSub; k++)
      if (k == m) acc[k] = acc[kMaxSub];  // (acc[m] is unused: dots run over k < m)
  }
  block_reduce_store<kMaxSub + 1>(acc, kAvg ? m + 1 : m, partials, gridDim.x);
}

// Tile-pair forms of the Davidson step's vector passes for exchange-symmetric subspaces (every S_k
// and sigma(S_k) exactly symmetric: the symmetric sigma and the projection make them so).  Each
// block walks 32 x 32 tile pairs (bi <= bj) as symmetrize_kernel does, reads the operands of the
// (bi, bj) tile only, and writes the result to both tiles through shared memory; the reductions
// count an off-diagonal pair's products twice.

// tile-pair index p -> (bi, bj), bi <= bj, row-major over the upper triangle of nt x nt tiles
__device__ __forceinline__ void tile_pair(size_t p, uint32_t nt, uint32_t &bi, uint32_t &bj) {
  bi = (uint32_t)((2.0 * nt + 1.0 - sqrt((2.0 * nt + 1.0) * (2.0 * nt + 1.0) - 8.0 * (double)p)) / 2.0);
  while (bi > 0 && (size_t)bi * nt - (size_t)bi * (bi - 1) / 2 > p) bi--;
  while ((size_t)(bi + 1) * nt - (size_t)(bi + 1) * bi / 2 <= p) bi++;
  bj = bi + (uint32_t)(p - ((size_t)bi * nt - (size_t)bi * (bi - 1) / 2));
}

// The residual pass with the exchange projection folded in: r = E' W - sum_k u_k sigma(S_k) on the
// (bi, bj) tile (r is symmetric), t = r / (E0 - H_ii) at both (i, j) and (j, i) (H_ii differs
// between the two in its last bits), t_sym = (t(i,j) + t(j,i)) / 2 written to both tiles -- what
// residual_kernel followed by symmetrize_kernel produce, with half the subspace bytes read.
// partials: [0] W.W, [1] r.r, [2+k] S_k.t_sym, [2+M] t_sym.t_sym.
template <typename T, int VW, int M>
__global__ void __launch_bounds__(256)
    residual_sym_kernel(ResidualArgs<T> a, uint32_t nb, double *partials) {
  constexpr int TS = kSymTile, TPR = TS / VW, RS = 256 / TPR;
  // the diagonal of the (bj, bi) tile as stored: H_ii - H_00 in FP32 for FP32 vectors, H_ii in FP64
  __shared__ T Hd[TS][TS + 1];
  __shared__ T Tt[TS][TS + 1];  // t_sym of the (bi, bj) tile, read transposed for (bj, bi)
  if (a.u_dev) {
#pragma unroll
    for (int k = 0; k < M; k++) a.u[k] = __ldg(&a.u_dev[k]);
    a.e_shifted = __ldg(&a.e_dev[0]);
    a.e0 = a.e_shifted + a.shift;
  }
  const uint32_t nt = (nb + TS - 1) / TS;
  const size_t npairs = (size_t)nt * (nt + 1) / 2;
  const int cx = (threadIdx.x % TPR) * VW, ty = threadIdx.x / TPR;
  double acc[M + 3];
#pragma unroll
  for (int j = 0; j < M + 3; j++) acc[j] = 0.0;
  // E0 - H_ii from the stored diagonal value (as residual_kernel forms it)
  auto hdiff = [&](T hv) -> double { return sizeof(T) == 4 ? a.e_shifted - (double)hv : a.e0 - (double)hv; };
  const T *hsrc = sizeof(T) == 4 ? reinterpret_cast<const T *>(a.hii32) : reinterpret_cast<const T *>(a.hii);
  for (size_t p = blockIdx.x; p < npairs; p += gridDim.x) {
    uint32_t bi, bj;
    tile_pair(p, nt, bi, bj);
    __syncthreads();
    // the diagonal of the (bj, bi) tile
    for (int e = threadIdx.x; e < TS * TS; e += blockDim.x) {
      const int rr = e / TS, cc = e % TS;
      const uint32_t i2 = bj * TS + rr, j2 = bi * TS + cc;
      Hd[rr][cc] = (i2 < nb && j2 < nb) ? __ldg(&hsrc[(size_t)i2 * nb + j2]) : T(0);
    }
    __syncthreads();
    const double mult = bi == bj ? 1.0 : 2.0;
#pragma unroll
    for (int r = ty; r < TS; r += RS) {
      const uint32_t i = bi * TS + r, j = bj * TS + cx;
      if (i >= nb || j >= nb) continue;
      const size_t base = (size_t)i * nb + j;
      T c[M][VW];
      double w[VW], hc[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) w[l] = hc[l] = 0.0;
#pragma unroll
      for (int k = 0; k < M; k++) {
        T hv[VW];
        ldv<T, VW>(a.C.p[k] + base, c[k]);
        ldv<T, VW>(a.HC.p[k] + base, hv);
#pragma unroll
        for (int l = 0; l < VW; l++) {
          w[l] += a.u[k] * (double)c[k][l];
          hc[l] += a.u[k] * (double)hv[l];
        }
      }
      T v[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) {
        const double rv = a.e_shifted * w[l] - hc[l];
        acc[0] += mult * w[l] * w[l];
        acc[1] += mult * rv * rv;
        const double d1 = hdiff(__ldg(&hsrc[base + l])), d2 = hdiff(Hd[cx + l][r]);
        const T t1 = (T)((fabs(d1) > 1.0e-12) ? rv / d1 : rv / (d1 - 1.0e-12));
        const T t2 = (T)((fabs(d2) > 1.0e-12) ? rv / d2 : rv / (d2 - 1.0e-12));
        v[l] = (T)(((double)t1 + (double)t2) * 0.5);
        Tt[r][cx + l] = v[l];
#pragma unroll
        for (int k = 0; k < M; k++) acc[2 + k] += mult * (double)c[k][l] * (double)v[l];
        acc[2 + M] += mult * (double)v[l] * (double)v[l];
      }
      stv<T, VW>(a.t + base, v);
    }
    __syncthreads();
    if (bi != bj) {
#pragma unroll
      for (int r = ty; r < TS; r += RS) {
        const uint32_t i2 = bj * TS + r, j2 = bi * TS + cx;
        if (i2 >= nb || j2 >= nb) continue;
        T v[VW];
#pragma unroll
        for (int l = 0; l < VW; l++) v[l] = Tt[cx + l][r];
        stv<T, VW>(a.t + (size_t)i2 * nb + j2, v);
      }
    }
  }
  block_reduce_store<M + 3>(acc, M + 3, partials, gridDim.x);
}

// Gram-Schmidt round t -= sum_k o_k S_k on the (bi, bj) tile, written to both tiles; partials
// [0] t.t, [1+k] S_k.t (kDots).  pred as in cgs_update_kernel.
template <typename T, int VW, int M, bool kDots>
__global__ void __launch_bounds__(256)
    cgs_sym_kernel(VecPtrs<T> C, CoefArray co, const double *__restrict__ ov, T *__restrict__ t, uint32_t nb,
                   double *partials, const double *__restrict__ pred0, const double *__restrict__ pred1) {
  constexpr int TS = kSymTile, TPR = TS / VW, RS = 256 / TPR;
  __shared__ T Tt[TS][TS + 1];
  double acc[M + 1];
#pragma unroll
  for (int j = 0; j < M + 1; j++) acc[j] = 0.0;
  if (pred0 && !(__ldg(pred1) < 0.5 * __ldg(pred0))) {
    if (threadIdx.x <= (kDots ? M : 0)) partials[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = 0.0;
    return;
  }
  double o[M];
#pragma unroll
  for (int k = 0; k < M; k++) o[k] = co.v[k] * (ov ? __ldg(&ov[k]) : 1.0);
  const uint32_t nt = (nb + TS - 1) / TS;
  const size_t npairs = (size_t)nt * (nt + 1) / 2;
  const int cx = (threadIdx.x % TPR) * VW, ty = threadIdx.x / TPR;
  for (size_t p = blockIdx.x; p < npairs; p += gridDim.x) {
    uint32_t bi, bj;
    tile_pair(p, nt, bi, bj);
    const double mult = bi == bj ? 1.0 : 2.0;
    __syncthreads();
#pragma unroll
    for (int r = ty; r < TS; r += RS) {
      const uint32_t i = bi * TS + r, j = bj * TS + cx;
      if (i >= nb || j >= nb) continue;
      const size_t base = (size_t)i * nb + j;
      T tv[VW], c[M][VW];
      ldv<T, VW>(t + base, tv);
      double x[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) x[l] = (double)tv[l];
#pragma unroll
      for (int k = 0; k < M; k++) {
        ldv<T, VW>(C.p[k] + base, c[k]);
#pragma unroll
        for (int l = 0; l < VW; l++) x[l] -= o[k] * (double)c[k][l];
      }
      T xt[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) {
        xt[l] = (T)x[l];
        Tt[r][cx + l] = xt[l];
        acc[0] += mult * (double)xt[l] * (double)xt[l];
        if (kDots) {
#pragma unroll
          for (int k = 0; k < M; k++) acc[1 + k] += mult * (double)c[k][l] * (double)xt[l];
        }
      }
      stv<T, VW>(t + base, xt);
    }
    __syncthreads();
    if (bi != bj) {
#pragma unroll
      for (int r = ty; r < TS; r += RS) {
        const uint32_t i2 = bj * TS + r, j2 = bi * TS + cx;
        if (i2 >= nb || j2 >= nb) continue;
        T v[VW];
#pragma unroll
        for (int l = 0; l < VW; l++) v[l] = Tt[cx + l][r];
        stv<T, VW>(t + (size_t)i2 * nb + j2, v);
      }
    }
  }
  block_reduce_store<M + 1>(acc, kDots ? M + 1 : 1, partials, gridDim.x);
}

// FP32 forms of the two tile-pair passes above for 16-byte rows (32 x 32 tiles, one tile row per
// thread): every global load of a tile pair -- the thread's rows of both tiles, of the S_k / sigma(S_k)
// it multiplies, and of the diagonal -- is issued before the first barrier, so a tile pair waits on one
// round of memory latency instead of two or three (the general forms loaded the subspace tiles only
// after the barrier and ran FP32 at ~3 TB/s).  Same arithmetic, same order per element.
template <int M, bool kAvg = false>
__global__ void __launch_bounds__(256)
    sym_add_dots_f32_kernel(float *__restrict__ t, uint32_t nb, VecPtrs<float> S, double *partials) {
  constexpr int TS = kSymTile, VW = 4, TPR = TS / VW;
  static_assert(256 / TPR == TS, "one tile row per thread");
  constexpr double kW = kAvg ? 0.5 : 1.0;
  __shared__ float A[TS][TS + 1], B[TS][TS + 1];
  const uint32_t nt = (nb + TS - 1) / TS;
  const size_t npairs = (size_t)nt * (nt + 1) / 2;
  const int cx = (threadIdx.x % TPR) * VW, r = threadIdx.x / TPR;
  double acc[M + 1];
#pragma unroll
  for (int k = 0; k <= M; k++) acc[k] = 0.0;
  for (size_t p = blockIdx.x; p < npairs; p += gridDim.x) {
    uint32_t bi, bj;
    tile_pair(p, nt, bi, bj);
    const uint32_t i = bi * TS + r, j = bj * TS + cx, i2 = bj * TS + r, j2 = bi * TS + cx;
    const bool in1 = i < nb && j < nb, in2 = i2 < nb && j2 < nb;
    float va[VW] = {0.f, 0.f, 0.f, 0.f}, vb[VW] = {0.f, 0.f, 0.f, 0.f}, sv[M][VW];
    if (in1) ldv<float, VW>(t + (size_t)i * nb + j, va);
    if (in2) ldv<float, VW>(t + (size_t)i2 * nb + j2, vb);
#pragma unroll
    for (int k = 0; k < M; k++) {
      if (in1) ldv<float, VW>(S.p[k] + (size_t)i * nb + j, sv[k]);
      else {
#pragma unroll
        for (int l = 0; l < VW; l++) sv[k][l] = 0.f;
      }
    }
    __syncthreads();
#pragma unroll
    for (int l = 0; l < VW; l++) {
      A[r][cx + l] = va[l];
      B[r][cx + l] = vb[l];
    }
    __syncthreads();
    const double mult = bi == bj ? 1.0 : 2.0;
    if (in1) {
      float v[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) v[l] = (float)(((double)A[r][cx + l] + (double)B[cx + l][r]) * kW);
      stv<float, VW>(t + (size_t)i * nb + j, v);
#pragma unroll
      for (int k = 0; k < M; k++) {
        double d = 0.0;
#pragma unroll
        for (int l = 0; l < VW; l++) d += (double)v[l] * (double)sv[k][l];
        acc[k] += mult * d;
      }
      if (kAvg) {
        double d = 0.0;
#pragma unroll
        for (int l = 0; l < VW; l++) d += (double)v[l] * (double)v[l];
        acc[M] += mult * d;
      }
    }
    if (bi != bj && in2) {
      float v[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) v[l] = (float)(((double)A[cx + l][r] + (double)B[r][cx + l]) * kW);
      stv<float, VW>(t + (size_t)i2 * nb + j2, v);
    }
  }
  block_reduce_store<M + 1>(acc, kAvg ? M + 1 : M, partials, gridDim.x);
}

template <int M>
__global__ void __launch_bounds__(256)
    residual_sym_f32_kernel(ResidualArgs<float> a, uint32_t nb, double *partials) {
  constexpr int TS = kSymTile, VW = 4, TPR = TS / VW;
  static_assert(256 / TPR == TS, "one tile row per thread");
  __shared__ float Hd[TS][TS + 1];  // H_ii - H_00 of the (bj, bi) tile
  __shared__ float Tt[TS][TS + 1];  // t_sym of the (bi, bj) tile, read transposed for (bj, bi)
  if (a.u_dev) {
#pragma unroll
    for (int k = 0; k < M; k++) a.u[k] = __ldg(&a.u_dev[k]);
    a.e_shifted = __ldg(&a.e_dev[0]);
    a.e0 = a.e_shifted + a.shift;
  }
  const uint32_t nt = (nb + TS - 1) / TS;
  const size_t npairs = (size_t)nt * (nt + 1) / 2;
  const int cx = (threadIdx.x % TPR) * VW, r = threadIdx.x / TPR;
  double acc[M + 3];
#pragma unroll
  for (int k = 0; k < M + 3; k++) acc[k] = 0.0;
  for (size_t p = blockIdx.x; p < npairs; p += gridDim.x) {
    uint32_t bi, bj;
    tile_pair(p, nt, bi, bj);
    const uint32_t i = bi * TS + r, j = bj * TS + cx, i2 = bj * TS + r, j2 = bi * TS + cx;
    const bool in1 = i < nb && j < nb, in2 = i2 < nb && j2 < nb;
    const size_t base = (size_t)i * nb + j;
    float c[M][VW], hv[M][VW], hij[VW] = {0.f, 0.f, 0.f, 0.f}, hji[VW] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < M; k++) {
      if (in1) {
        ldv<float, VW>(a.C.p[k] + base, c[k]);
        ldv<float, VW>(a.HC.p[k] + base, hv[k]);
      } else {
#pragma unroll
        for (int l = 0; l < VW; l++) c[k][l] = hv[k][l] = 0.f;
      }
    }
    if (in1) ldv<float, VW>(a.hii32 + base, hij);
    if (in2) ldv<float, VW>(a.hii32 + (size_t)i2 * nb + j2, hji);
    __syncthreads();
#pragma unroll
    for (int l = 0; l < VW; l++) Hd[r][cx + l] = hji[l];
    __syncthreads();
    const double mult = bi == bj ? 1.0 : 2.0;
    if (in1) {
      double w[VW], hc[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) w[l] = hc[l] = 0.0;
#pragma unroll
      for (int k = 0; k < M; k++) {
#pragma unroll
        for (int l = 0; l < VW; l++) {
          w[l] += a.u[k] * (double)c[k][l];
          hc[l] += a.u[k] * (double)hv[k][l];
        }
      }
      float v[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) {
        const double rv = a.e_shifted * w[l] - hc[l];
        acc[0] += mult * w[l] * w[l];
        acc[1] += mult * rv * rv;
        const double d1 = a.e_shifted - (double)hij[l], d2 = a.e_shifted - (double)Hd[cx + l][r];
        const float t1 = (float)((fabs(d1) > 1.0e-12) ? rv / d1 : rv / (d1 - 1.0e-12));
        const float t2 = (float)((fabs(d2) > 1.0e-12) ? rv / d2 : rv / (d2 - 1.0e-12));
        v[l] = (float)(((double)t1 + (double)t2) * 0.5);
        Tt[r][cx + l] = v[l];
#pragma unroll
        for (int k = 0; k < M; k++) acc[2 + k] += mult * (double)c[k][l] * (double)v[l];
        acc[2 + M] += mult * (double)v[l] * (double)v[l];
      }
      stv<float, VW>(a.t + base, v);
    }
    __syncthreads();
    if (bi != bj && in2) {
      float v[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) v[l] = Tt[cx + l][r];
      stv<float, VW>(a.t + (size_t)i2 * nb + j2, v);
    }
  }
  block_reduce_store<M + 3>(acc, M + 3, partials, gridDim.x);
}

// 16-byte asynchronous global -> shared copy (zero fill when !valid; gmem must still be a valid
// address), its commit and wait
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// The tile-pair residual pass as a two-stage pipeline: while a block computes one tile pair from
// shared memory, the copies of its next pair (the (bi, bj) tiles of every C_k and sigma(S_k) and of
// the stored diagonal, and the (bj, bi) tile of the diagonal) are in flight, so the bytes in flight
// do not live in registers (the register forms hold one pair: the FP32 one ran one block per SM and
// ~2.7 TB/s at M = 6..8).  Each thread copies and later reads back only its own 16-byte chunks,
// except for the transposed diagonal tile, which every thread reads across the tile after a
// barrier; its chunks are XOR-swizzled by row so those reads spread over the banks.  The block
// walks its tile pairs incrementally (one square root per block, not per pair and thread).
//
// Arithmetic, chosen for instruction count (the register forms issued ~280 instructions per
// element, most of them FP32<->FP64 conversions, which run at a quarter of the FP64 rate, and two
// FP64 divisions): W = sum u_k C_k, sum u_k sigma_k, r = E' W - sum u_k sigma_k, W.W and r.r in
// FP64 (r cancels), then t_sym = r (1/(E0 - H_ij) + 1/(E0 - H_ji)) / 2 as r (d1 + d2) / (2 d1 d2),
// one division, in the vector type (FP32 vectors: FP32, from r rounded to FP32 and
// E0 - H = (E'_hi - H') + E'_lo; each d with the reference's 1e-12 regularisation), and the
// overlaps S_k . t_sym and t_sym . t_sym from per-thread partial sums of four FP32 products that are
// added in FP64.  t differs from the register forms' in its last bits only.  Used while both stages
// fit in shared memory (FP32 up to M = 8, FP64 up to 5).
template <typename T, int M>
constexpr size_t residual_pipe_smem() {
  return (2 * (size_t)(2 * M + 2) * kSymTile * kSymTile + (size_t)kSymTile * (kSymTile + 1)) * sizeof(T);
}
template <typename T>
constexpr int residual_pipe_max() {
  return sizeof(T) == 4 ? 8 : 5;
}
static_assert(residual_pipe_smem<float, residual_pipe_max<float>()>() <= 227 * 1024, "FP32 stages");
static_assert(residual_pipe_smem<double, residual_pipe_max<double>()>() <= 227 * 1024, "FP64 stages");
// (bi, bj) of the tile pair `step` positions further in the row-major upper triangle
__device__ __forceinline__ void tile_pair_advance(uint32_t nt, uint32_t step, uint32_t &bi, uint32_t &bj) {
  uint32_t off = bj - bi + step;
  while (bi < nt && off >= nt - bi) {
    off -= nt - bi;
    bi++;
  }
  bj = bi + off;
}
template <typename T, int M>
__global__ void __launch_bounds__(256)
    residual_sym_pipe_kernel(ResidualArgs<T> a, uint32_t nb, double *partials) {
  constexpr int TS = kSymTile, VW = 16 / sizeof(T), CPR = TS / VW;  // chunks per tile row
  constexpr int NCH = TS * CPR / 256;                                 // chunks of a tile per thread
  constexpr int RS = 256 / CPR;                                       // rows between a thread's chunks
  constexpr int kTile = TS * TS, kStage = (2 * M + 2) * kTile;
  constexpr bool kF32 = sizeof(T) == 4;
  static_assert(CPR >= 8 && NCH * 256 == TS * CPR, "tile of whole 16-byte chunks");
  extern __shared__ __align__(16) unsigned char psm_raw[];
  T *psm = reinterpret_cast<T *>(psm_raw);
  T(*Tt)[TS + 1] = reinterpret_cast<T(*)[TS + 1]>(psm + 2 * kStage);
  if (a.u_dev) {
#pragma unroll
    for (int k = 0; k < M; k++) a.u[k] = __ldg(&a.u_dev[k]);
    a.e_shifted = __ldg(&a.e_dev[0]);
    a.e0 = a.e_shifted + a.shift;
  }
  // E0 - H_ii: from H_ii - H_00 (FP32, against E0 - H_00 split in two floats) or from H_ii (FP64)
  const float e_hi = (float)a.e_shifted, e_lo = (float)(a.e_shifted - (double)e_hi);
  const T *hsrc = kF32 ? reinterpret_cast<const T *>(a.hii32) : reinterpret_cast<const T *>(a.hii);
  const uint32_t nt = (nb + TS - 1) / TS;
  const size_t npairs = (size_t)nt * (nt + 1) / 2;
  const int q = threadIdx.x % CPR, cx = q * VW, ty = threadIdx.x / CPR;
  auto issue = [&](uint32_t bi, uint32_t bj, T *st) {
#pragma unroll
    for (int hh = 0; hh < NCH; hh++) {
      const int r = ty + hh * RS;
      const uint32_t i = bi * TS + r, j = bj * TS + cx, i2 = bj * TS + r, j2 = bi * TS + cx;
      const bool in1 = i < nb && j < nb, in2 = i2 < nb && j2 < nb;
      const size_t base = in1 ? (size_t)i * nb + j : 0, base2 = in2 ? (size_t)i2 * nb + j2 : 0;
      const int own = r * TS + cx, own_sw = r * TS + ((q ^ ((r / VW) & 7)) * VW);
#pragma unroll
      for (int k = 0; k < M; k++) {
        cp_async16(st + k * kTile + own, a.C.p[k] + base, in1);
        cp_async16(st + (M + k) * kTile + own, a.HC.p[k] + base, in1);
      }
      cp_async16(st + 2 * M * kTile + own, hsrc + base, in1);
      cp_async16(st + (2 * M + 1) * kTile + own_sw, hsrc + base2, in2);
    }
  };
  double acc[M + 3];
#pragma unroll
  for (int k = 0; k < M + 3; k++) acc[k] = 0.0;
  int s = 0;
  uint32_t bi = 0, bj = 0;
  if (blockIdx.x < npairs) {
    tile_pair(blockIdx.x, nt, bi, bj);
    issue(bi, bj, psm);
  }
  cp_async_commit();
  for (size_t p = blockIdx.x; p < npairs; p += gridDim.x, s ^= 1) {
    uint32_t nbi = bi, nbj = bj;
    tile_pair_advance(nt, gridDim.x, nbi, nbj);
    if (p + gridDim.x < npairs) issue(nbi, nbj, psm + (s ^ 1) * kStage);
    cp_async_commit();
    cp_async_wait<1>();  // this pair's copies (this thread's) have landed
    __syncthreads();     // ... and every thread's, for the transposed diagonal tile
    const T *st = psm + s * kStage;
    const double mult = bi == bj ? 1.0 : 2.0;
#pragma unroll
    for (int hh = 0; hh < NCH; hh++) {
      const int r = ty + hh * RS, own = r * TS + cx;
      const uint32_t i = bi * TS + r, j = bj * TS + cx;
      if (i >= nb || j >= nb) continue;
      double w[VW], hc[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) w[l] = hc[l] = 0.0;
#pragma unroll
      for (int k = 0; k < M; k++) {
#pragma unroll
        for (int l = 0; l < VW; l++) {
          w[l] += a.u[k] * (double)st[k * kTile + own + l];
          hc[l] += a.u[k] * (double)st[(M + k) * kTile + own + l];
        }
      }
      // the transposed entry (j + l, i): row cx + l, column r of the swizzled tile
      const T *ht = st + (2 * M + 1) * kTile + (((r / VW) ^ (q & 7)) * VW) + (r % VW);
      T v[VW];
      double ww = 0.0, rr = 0.0;
#pragma unroll
      for (int l = 0; l < VW; l++) {
        const double rv = a.e_shifted * w[l] - hc[l];
        ww += w[l] * w[l];
        rr += rv * rv;
        const T h1 = st[2 * M * kTile + own + l], h2 = ht[(cx + l) * TS];
        if constexpr (kF32) {
          float d1 = (e_hi - (float)h1) + e_lo, d2 = (e_hi - (float)h2) + e_lo;
          d1 = fabsf(d1) > 1.0e-12f ? d1 : d1 - 1.0e-12f;
          d2 = fabsf(d2) > 1.0e-12f ? d2 : d2 - 1.0e-12f;
          v[l] = (T)(0.5f * (float)rv * (d1 + d2) / (d1 * d2));
        } else {
          double d1 = a.e0 - (double)h1, d2 = a.e0 - (double)h2;
          d1 = fabs(d1) > 1.0e-12 ? d1 : d1 - 1.0e-12;
          d2 = fabs(d2) > 1.0e-12 ? d2 : d2 - 1.0e-12;
          v[l] = (T)(0.5 * rv * (d1 + d2) / (d1 * d2));
        }
        Tt[r][cx + l] = v[l];
      }
      acc[0] += mult * ww;
      acc[1] += mult * rr;
      if constexpr (kF32) {
#pragma unroll
        for (int k = 0; k < M; k++) {
          float pk = 0.f;
#pragma unroll
          for (int l = 0; l < VW; l++) pk = fmaf((float)st[k * kTile + own + l], (float)v[l], pk);
          acc[2 + k] += mult * (double)pk;
        }
        float vv = 0.f;
#pragma unroll
        for (int l = 0; l < VW; l++) vv = fmaf((float)v[l], (float)v[l], vv);
        acc[2 + M] += mult * (double)vv;
      } else {
#pragma unroll
        for (int k = 0; k < M; k++) {
          double pk = 0.0;
#pragma unroll
          for (int l = 0; l < VW; l++) pk += (double)st[k * kTile + own + l] * (double)v[l];
          acc[2 + k] += mult * pk;
        }
        double vv = 0.0;
#pragma unroll
        for (int l = 0; l < VW; l++) vv += (double)v[l] * (double)v[l];
        acc[2 + M] += mult * vv;
      }
      stv<T, VW>(a.t + (size_t)i * nb + j, v);
    }
    __syncthreads();
    if (bi != bj) {
#pragma unroll
      for (int hh = 0; hh < NCH; hh++) {
        const int r = ty + hh * RS;
        const uint32_t i2 = bj * TS + r, j2 = bi * TS + cx;
        if (i2 >= nb || j2 >= nb) continue;
        T v[VW];
#pragma unroll
        for (int l = 0; l < VW; l++) v[l] = Tt[cx + l][r];
        stv<T, VW>(a.t + (size_t)i2 * nb + j2, v);
      }
    }
    bi = nbi;
    bj = nbj;
  }
  cp_async_wait<0>();
  block_reduce_store<M + 3>(acc, M + 3, partials, gridDim.x);
}

// The last step of a Davidson cycle on an exchange-symmetric subspace: W = sum u_k S_k and
// r = E' W - sum u_k sigma(S_k) from the (bi, bj) tile of each tile pair only (W and r are
// symmetric), W written to both tiles, W.W and r.r counted twice off the diagonal; no correction.
// The same W, bit for bit, as residual_kernel (same per-element sums in the same order), from half
// the subspace bytes.  Each thread streams its chunks of C_k and sigma(S_k) straight into the two
// sums, so nothing but the sums stays live and the pass runs at full occupancy without staging.
// partials: [0] W.W, [1] r.r, [2, M + 3) zero (the layout of residual_kernel's).
template <typename T, int M>
__global__ void __launch_bounds__(256)
    residual_w_sym_kernel(ResidualArgs<T> a, uint32_t nb, double *partials) {
  constexpr int TS = kSymTile, VW = 16 / sizeof(T), TPR = TS / VW, RS = 256 / TPR;
  __shared__ T Wt[TS][TS + 1];  // W of the (bi, bj) tile, read transposed for (bj, bi)
  if (a.u_dev) {
#pragma unroll
    for (int k = 0; k < M; k++) a.u[k] = __ldg(&a.u_dev[k]);
    a.e_shifted = __ldg(&a.e_dev[0]);
  }
  const uint32_t nt = (nb + TS - 1) / TS;
  const size_t npairs = (size_t)nt * (nt + 1) / 2;
  const int cx = (threadIdx.x % TPR) * VW, ty = threadIdx.x / TPR;
  double acc[M + 3];
#pragma unroll
  for (int k = 0; k < M + 3; k++) acc[k] = 0.0;
  uint32_t bi = 0, bj = 0;
  if (blockIdx.x < npairs) tile_pair(blockIdx.x, nt, bi, bj);
  for (size_t p = blockIdx.x; p < npairs; p += gridDim.x) {
    const double mult = bi == bj ? 1.0 : 2.0;
#pragma unroll
    for (int r = ty; r < TS; r += RS) {
      const uint32_t i = bi * TS + r, j = bj * TS + cx;
      if (i >= nb || j >= nb) continue;
      const size_t base = (size_t)i * nb + j;
      double w[VW], hc[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) w[l] = hc[l] = 0.0;
#pragma unroll
      for (int k = 0; k < M; k++) {
        T c[VW], hv[VW];
        ldv<T, VW>(a.C.p[k] + base, c);
        ldv<T, VW>(a.HC.p[k] + base, hv);
#pragma unroll
        for (int l = 0; l < VW; l++) {
          w[l] += a.u[k] * (double)c[l];
          hc[l] += a.u[k] * (double)hv[l];
        }
      }
      T wv[VW];
#pragma unroll
      for (int l = 0; l < VW; l++) {
        const double rv = a.e_shifted * w[l] - hc[l];
        acc[0] += mult * w[l] * w[l];
        acc[1] += mult * rv * rv;
        wv[l] = (T)w[l];
        Wt[r][cx + l] = wv[l];
      }
      stv<T, VW>(a.W + base, wv);
    }
    __syncthreads();
    if (bi != bj) {
#pragma unroll
      for (int r = ty; r < TS; r += RS) {
        const uint32_t i2 = bj * TS + r, j2 = bi * TS + cx;
        if (i2 >= nb || j2 >= nb) continue;
        T v[VW];
#pragma unroll
        for (int l = 0; l < VW; l++) v[l] = Wt[cx + l][r];
        stv<T, VW>(a.W + (size_t)i2 * nb + j2, v);
      }
    }
    __syncthreads();
    tile_pair_advance(nt, gridDim.x, bi, bj);
  }
  block_reduce_store<M + 3>(acc, M + 3, partials, gridDim.x);
}

// The reference's seeded random start (Randomize, framework/dm_vector.h:101-178): element i is
// a uniform value in [-1, 1) from a splitmix64-style mix of (seed, i) -- the same integer steps as
// sbd_elem_hash / sbd_hash_to_uniform (dm_vector.h:100-112), so the same values for any launch
// shape -- in the reference's determinant order and sign convention; the caller normalises.
__device__ __forceinline__ double seeded_uniform(unsigned long long seed, unsigned long long i) {
  unsigned long long x = seed * 6364136223846793005ULL + i * 2862933555777941757ULL;
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebULL;
  x ^= x >> 31;
  return (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

__global__ void random_start_kernel(double *__restrict__ x, size_t n, unsigned long long seed) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = seeded_uniform(seed, i);
}

// Rayleigh-Ritz of the Davidson subspace on one warp.  Hs (ld kMaxSub, column-major, persistent
// across the steps of a cycle) gets column and row ib = f_k f_ib ov_k; the leading n = ib + 1
// block is diagonalised by cyclic Jacobi rotations in shared memory (each rotation's row and
// column updates split over the lanes), the eigenvalues sorted ascending as dsyev returns them.
// Outputs: u[k] = V[k][lowest] * f_k, e[0..n) ascending, eig4[0..3] = the lowest four (0 past n).
__global__ void __launch_bounds__(32) rr_kernel(double *__restrict__ Hs, const double *__restrict__ ov,
                                                ScaleArray f, int ib, double *__restrict__ u,
                                                double *__restrict__ e, double *__restrict__ eig4) {
  constexpr int S = kMaxSub;
  __shared__ double M[S][S + 1], V[S][S + 1];
  __shared__ int ord[S];
  const int lane = threadIdx.x, n = ib + 1;
  if (lane <= ib) {
    const double v = f.v[lane] * f.v[ib] * ov[lane];
    Hs[lane + S * ib] = v;
    Hs[ib + S * lane] = v;
  }
  __syncwarp();
  for (int idx = lane; idx < n * n; idx += 32) {
    const int i = idx % n, j = idx / n;
    M[i][j] = Hs[i + S * j];
    V[i][j] = i == j ? 1.0 : 0.0;
  }
  __syncwarp();
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, diag = 0.0;
    for (int idx = lane; idx < n * n; idx += 32) {
      const int i = idx % n, j = idx / n;
      if (i == j) diag += M[i][j] * M[i][j];
      else if (i < j) off += M[i][j] * M[i][j];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      diag += __shfl_xor_sync(0xffffffffu, diag, o);
    }
    if (off <= 1e-32 * (diag + 1e-300)) break;
    for (int p = 0; p < n; p++) {
      for (int q = p + 1; q < n; q++) {
        const double apq = M[p][q];
        if (fabs(apq) < 1e-300) continue;
        const double app = M[p][p], aqq = M[q][q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        __syncwarp();
        if (lane < n) {  // columns p, q
          const double mkp = M[lane][p], mkq = M[lane][q];
          M[lane][p] = c * mkp - s * mkq;
          M[lane][q] = s * mkp + c * mkq;
        }
        __syncwarp();
        if (lane < n) {  // rows p, q
          const double mpk = M[p][lane], mqk = M[q][lane];
          M[p][lane] = c * mpk - s * mqk;
          M[q][lane] = s * mpk + c * mqk;
        } else if (lane >= 16 && lane - 16 < n) {  // eigenvectors
          const int k = lane - 16;
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
        __syncwarp();
      }
    }
  }
  __syncwarp();
  if (lane == 0) {
    for (int i = 0; i < n; i++) ord[i] = i;
    for (int i = 0; i < n; i++)
      for (int j = i + 1; j < n; j++)
        if (M[ord[j]][ord[j]] < M[ord[i]][ord[i]]) {
          const int x = ord[i];
          ord[i] = ord[j];
          ord[j] = x;
        }
  }
  __syncwarp();
  if (lane < n) {
    e[lane] = M[ord[lane]][ord[lane]];
    u[lane] = V[lane][ord[0]] * f.v[lane];
  }
  if (lane < 4) eig4[lane] = lane < n ? M[ord[lane]][ord[lane]] : 0.0;
}

}  // namespace

int ensure_partials(sbd_tpb_handle *h, size_t n) {
  if (h->partials_cap >= n) return SBD_TPB_OK;
  if (h->d_partials) cudaFree(h->d_partials);
  h->d_partials = nullptr;
  h->partials_cap = 0;
  TPB_CUDA(cudaMalloc(&h->d_partials, n * sizeof(double)));
  h->partials_cap = n;
  return SBD_TPB_OK;
}

int vec_blocks(sbd_tpb_handle *h) { return h->num_sms * 4; }

// device slots for reductions whose results are read back together (pinned host mirror)
// (with them the Rayleigh-Ritz state: the projected matrix, u and the eigenvalues)
constexpr int kRrDoubles = kMaxSub * kMaxSub + 2 * kMaxSub;
static int ensure_scalars(sbd_tpb_handle *h) {
  if (h->d_scal) return SBD_TPB_OK;
  TPB_CUDA(cudaMalloc(&h->d_scal, sizeof(double) * (kScalarSlots + kRrDoubles)));
  TPB_CUDA(cudaMemset(h->d_scal, 0, sizeof(double) * (kScalarSlots + kRrDoubles)));
  TPB_CUDA(cudaMallocHost(&h->h_scal, sizeof(double) * kScalarSlots));
  return SBD_TPB_OK;
}

static double *rr_base(sbd_tpb_handle *h) { return h->d_scal + kScalarSlots; }
const double *rr_u(sbd_tpb_handle *h) { return rr_base(h) + kMaxSub * kMaxSub; }
const double *rr_e(sbd_tpb_handle *h) { return rr_base(h) + kMaxSub * kMaxSub + kMaxSub; }

int rr_solve(sbd_tpb_handle *h, int ib, const ScaleArray &f, int ov_slot, int eig_slot) {
  if (ib < 0 || ib >= kMaxSub) return fail(SBD_TPB_ERR_INVALID, "subspace larger than supported");
  TPB_CHECK(ensure_scalars(h));
  double *base = rr_base(h);
  rr_kernel<<<1, 32, 0, h->stream>>>(base, h->d_scal + ov_slot, f, ib, base + kMaxSub * kMaxSub,
                                     base + kMaxSub * kMaxSub + kMaxSub, h->d_scal + eig_slot);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

// sums nvals rows of block partials (nblocks per row; the vector kernels' grid by default)
static int reduce_into(sbd_tpb_handle *h, int nvals, double *d_dst, int nblocks = 0) {
  const int nb = nblocks > 0 ? nblocks : vec_blocks(h);
  reduce_partials_kernel<<<nvals, 256, 0, h->stream>>>(h->d_partials, nb, d_dst);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

static int finish_reduce(sbd_tpb_handle *h, int nvals, double *host_out, int nblocks = 0) {
  const int nb = nblocks > 0 ? nblocks : vec_blocks(h);
  double *d_out = h->d_partials + std::max((size_t)(kMaxVec + 3) * vec_blocks(h), (size_t)nb * nvals);
  reduce_partials_kernel<<<nvals, 256, 0, h->stream>>>(h->d_partials, nb, d_out);
  TPB_LAUNCHED(h);
  TPB_CUDA(cudaMemcpyAsync(host_out, d_out, sizeof(double) * nvals, cudaMemcpyDeviceToHost,
                           h->stream));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  return SBD_TPB_OK;
}

// compile-time subspace size from a runtime one (1 .. kMaxVec)
template <int N, typename F>
int dispatch_n(int n, F &&f) {
  if constexpr (N > kMaxVec) {
    return fail(SBD_TPB_ERR_INVALID, "subspace larger than supported");
  } else {
    if (n == N) return f(std::integral_constant<int, N>());
    return dispatch_n<N + 1>(n, f);
  }
}

template <typename T>
int multi_dot(sbd_tpb_handle *h, const T *const *X, int k, const T *y, size_t n, double *out) {
  const int nb = vec_blocks(h);
  TPB_CHECK(ensure_partials(h, (size_t)(kMaxVec + 3) * nb + kMaxVec + 3));
  for (int j0 = 0; j0 < k; j0 += kMaxVec) {
    const int kk = std::min(kMaxVec, k - j0);
    VecPtrs<T> P;
    for (int j = 0; j < kMaxVec; j++) P.p[j] = (j < kk) ? X[j0 + j] : nullptr;
    TPB_CHECK(dispatch_n<1>(kk, [&](auto K) {
      multi_dot_kernel<T, decltype(K)::value><<<nb, kVecThreads, 0, h->stream>>>(P, y, n, h->d_partials);
      TPB_LAUNCHED(h);
      return SBD_TPB_OK;
    }));
    TPB_CHECK(finish_reduce(h, kk, out + j0));
  }
  return SBD_TPB_OK;
}

template <typename T>
int residual_step(sbd_tpb_handle *h, const ResidualArgs<T> &a, size_t n, double *out) {
  if (a.m < 1 || a.m > kMaxSub) return fail(SBD_TPB_ERR_INVALID, "subspace larger than supported");
  const int nb = vec_blocks(h);
  TPB_CHECK(ensure_partials(h, (size_t)(kMaxVec + 3) * nb + kMaxVec + 3));
  TPB_CHECK(dispatch_n<1>(a.m, [&](auto K) {
    constexpr int M = decltype(K)::value;
    if constexpr (M <= kMaxSub) {
      residual_kernel<T, M><<<nb, kVecThreads, 0, h->stream>>>(a, n, h->d_partials);
      TPB_LAUNCHED(h);
    }
    return SBD_TPB_OK;
  }));
  return finish_reduce(h, a.m + 3, out);  // [0] ww, [1] rr, [2..2+m) S_k.t, [2+m] t.t
}

template <typename T>
static int launch_cgs(sbd_tpb_handle *h, const T *const *C, int m, const double *coef, const double *ov_dev, T *t,
                      size_t n, int want_dots) {
  if (m < 1 || m > kMaxSub) return fail(SBD_TPB_ERR_INVALID, "subspace larger than supported");
  const int nb = vec_blocks(h);
  TPB_CHECK(ensure_partials(h, (size_t)(kMaxVec + 3) * nb + kMaxVec + 3));
  VecPtrs<T> P;
  CoefArray co;
  for (int j = 0; j < kMaxVec; j++) P.p[j] = j < m ? C[j] : nullptr;
  for (int j = 0; j < kMaxSub; j++) co.v[j] = j < m ? coef[j] : 0.0;
  return dispatch_n<1>(m, [&](auto K) {
    constexpr int M = decltype(K)::value;
    if constexpr (M <= kMaxSub) {
      if (want_dots)
        cgs_update_kernel<T, M, true><<<nb, kVecThreads, 0, h->stream>>>(P, co, ov_dev, t, n, h->d_partials);
      else
        cgs_update_kernel<T, M, false><<<nb, kVecThreads, 0, h->stream>>>(P, co, ov_dev, t, n, h->d_partials);
      TPB_LAUNCHED(h);
    }
    return SBD_TPB_OK;
  });
}

template <typename T>
int cgs_update(sbd_tpb_handle *h, const T *const *C, int m, const double *o, T *t, size_t n,
               int want_dots, double *out) {
  TPB_CHECK(launch_cgs<T>(h, C, m, o, nullptr, t, n, want_dots));
  return finish_reduce(h, want_dots ? 1 + m : 1, out);
}

template <typename T>
int residual_step_async(sbd_tpb_handle *h, const ResidualArgs<T> &a, size_t n, int slot) {
  if (a.m < 1 || a.m > kMaxSub) return fail(SBD_TPB_ERR_INVALID, "subspace larger than supported");
  TPB_CHECK(ensure_scalars(h));
  const int nb = vec_blocks(h);
  TPB_CHECK(ensure_partials(h, (size_t)(kMaxVec + 3) * nb + kMaxVec + 3));
  TPB_CHECK(dispatch_n<1>(a.m, [&](auto K) {
    constexpr int M = decltype(K)::value;
    if constexpr (M <= kMaxSub) {
      residual_kernel<T, M><<<nb, kVecThreads, 0, h->stream>>>(a, n, h->d_partials);
      TPB_LAUNCHED(h);
    }
    return SBD_TPB_OK;
  }));
  return reduce_into(h, a.m + 3, h->d_scal + slot);
}

template <typename T>
int cgs_update_async(sbd_tpb_handle *h, const T *const *C, int m, const double *coef, int ov_slot, T *t,
                     size_t n, int want_dots, int slot) {
  TPB_CHECK(ensure_scalars(h));
  TPB_CHECK(launch_cgs<T>(h, C, m, coef, h->d_scal + ov_slot, t, n, want_dots));
  return reduce_into(h, want_dots ? 1 + m : 1, h->d_scal + slot);
}

template <typename T>
int multi_dot_async(sbd_tpb_handle *h, const T *const *X, int k, const T *y, size_t n, int slot) {
  if (k < 1 || k > kMaxVec) return fail(SBD_TPB_ERR_INVALID, "subspace larger than supported");
  TPB_CHECK(ensure_scalars(h));
  const int nb = vec_blocks(h);
  TPB_CHECK(ensure_partials(h, (size_t)(kMaxVec + 3) * nb + kMaxVec + 3));
  VecPtrs<T> P;
  for (int j = 0; j < kMaxVec; j++) P.p[j] = (j < k) ? X[j] : nullptr;
  TPB_CHECK(dispatch_n<1>(k, [&](auto K) {
    multi_dot_kernel<T, decltype(K)::value><<<nb, kVecThreads, 0, h->stream>>>(P, y, n, h->d_partials);
    TPB_LAUNCHED(h);
    return SBD_TPB_OK;
  }));
  return reduce_into(h, k, h->d_scal + slot);
}

template <typename T>
int cgs_second_round_async(sbd_tpb_handle *h, const T *const *C, int m, const double *coef, int ov_slot, T *t,
                           size_t n, int t0_slot, int tt_slot, int slot) {
  if (m < 1 || m > kMaxSub) return fail(SBD_TPB_ERR_INVALID, "subspace larger than supported");
  TPB_CHECK(ensure_scalars(h));
  const int nb = vec_blocks(h);
  TPB_CHECK(ensure_partials(h, (size_t)(kMaxVec + 3) * nb + kMaxVec + 3));
  VecPtrs<T> P;
  CoefArray co;
  for (int j = 0; j < kMaxVec; j++) P.p[j] = j < m ? C[j] : nullptr;
  for (int j = 0; j < kMaxSub; j++) co.v[j] = j < m ? coef[j] : 0.0;
  TPB_CHECK(dispatch_n<1>(m, [&](auto K) {
    constexpr int M = decltype(K)::value;
    if constexpr (M <= kMaxSub) {
      cgs_update_kernel<T, M, false><<<nb, kVecThreads, 0, h->stream>>>(
          P, co, h->d_scal + ov_slot, t, n, h->d_partials, h->d_scal + t0_slot, h->d_scal + tt_slot);
      TPB_LAUNCHED(h);
    }
    return SBD_TPB_OK;
  }));
  return reduce_into(h, 1, h->d_scal + slot);
}

const double *fetch_scalars(sbd_tpb_handle *h, int count) {
  if (ensure_scalars(h) != SBD_TPB_OK) return nullptr;
  if (cudaMemcpyAsync(h->h_scal, h->d_scal, sizeof(double) * count, cudaMemcpyDeviceToHost, h->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess) {
    fail(SBD_TPB_ERR_CUDA, "fetching reduction results failed");
    return nullptr;
  }
  return h->h_scal;
}

template <typename T>
static int launch_symmetrize(sbd_tpb_handle *h, T *t, int *nblk_out) {
  const uint32_t nb = (uint32_t)h->bstr.size();
  const int nblk = h->num_sms * kSymBlocksPerSm;
  TPB_CHECK(ensure_partials(h, std::max<size_t>((size_t)(kMaxVec + 3) * vec_blocks(h) + kMaxVec + 3,
                                                (size_t)nblk + 1)));
  constexpr int VW = 16 / sizeof(T);
  if (nb % VW == 0 && reinterpret_cast<uintptr_t>(t) % 16 == 0)
    symmetrize_kernel<T, VW><<<nblk, 256, 0, h->stream>>>(t, nb, h->d_partials);
  else
    symmetrize_kernel<T, 1><<<nblk, 256, 0, h->stream>>>(t, nb, h->d_partials);
  TPB_LAUNCHED(h);
  *nblk_out = nblk;
  return SBD_TPB_OK;
}

template <typename T>
int symmetrize_async(sbd_tpb_handle *h, T *t, int slot) {
  TPB_CHECK(ensure_scalars(h));
  int nblk = 0;
  TPB_CHECK(launch_symmetrize<T>(h, t, &nblk));
  return reduce_into(h, 1, h->d_scal + slot, nblk);
}

template <typename T>
int symmetrize(sbd_tpb_handle *h, T *t, double *tt) {
  int nblk = 0;
  TPB_CHECK(launch_symmetrize<T>(h, t, &nblk));
  return finish_reduce(h, 1, tt, nblk);
}

template <typename T>
int sym_add(sbd_tpb_handle *h, T *x) {
  const uint32_t nb = (uint32_t)h->bstr.size();
  const int nblk = h->num_sms * kSymBlocksPerSm;
  constexpr int VW = 16 / sizeof(T);
  if (nb % VW == 0 && reinterpret_cast<uintptr_t>(x) % 16 == 0)
    symmetrize_kernel<T, VW, false><<<nblk, 256, 0, h->stream>>>(x, nb, nullptr);
  else
    symmetrize_kernel<T, 1, false><<<nblk, 256, 0, h->stream>>>(x, nb, nullptr);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

// kAvg: x <- (x + x^T) / 2 and x.x after S_k.x (m + 1 slots from `slot`)
template <typename T, bool kAvg>
static int sym_dots_impl(sbd_tpb_handle *h, T *x, const T *const *S, int m, int slot) {
  if (m < 1 || m > kMaxSub) return fail(SBD_TPB_ERR_INVALID, "subspace larger than supported");
  TPB_CHECK(ensure_scalars(h));
  const uint32_t nb = (uint32_t)h->bstr.size();
  const int nblk = h->num_sms * kSymBlocksPerSm;
  TPB_CHECK(ensure_partials(h, std::max<size_t>((size_t)(kMaxVec + 3) * vec_blocks(h) + kMaxVec + 3,
                                                (size_t)kMaxSub * nblk + 1)));
  VecPtrs<T> P;
  for (int j = 0; j < kMaxVec; j++) P.p[j] = j < m ? S[j] : nullptr;
  constexpr int VW = 16 / sizeof(T);
  bool vec = nb % VW == 0 && reinterpret_cast<uintptr_t>(x) % 16 == 0;
  for (int j = 0; j < m; j++) vec = vec && reinterpret_cast<uintptr_t>(S[j]) % 16 == 0;
  if (vec && sizeof(T) == 4) {
    TPB_CHECK(dispatch_n<1>(m, [&](auto K) {
      constexpr int M = decltype(K)::value;
      if constexpr (M <= kMaxSub) {
        sym_add_dots_f32_kernel<M, kAvg><<<nblk, 256, 0, h->stream>>>(
            reinterpret_cast<float *>(x), nb, *reinterpret_cast<VecPtrs<float> *>(&P), h->d_partials);
        TPB_LAUNCHED(h);
      }
      return SBD_TPB_OK;
    }));
  } else {
    if (vec) sym_add_dots_kernel<T, VW, kAvg><<<nblk, 256, 0, h->stream>>>(x, nb, P, m, h->d_partials);
    else sym_add_dots_kernel<T, 1, kAvg><<<nblk, 256, 0, h->stream>>>(x, nb, P, m, h->d_partials);
    TPB_LAUNCHED(h);
  }
  return reduce_into(h, kAvg ? m + 1 : m, h->d_scal + slot, nblk);
}

template <typename T>
int sym_add_dots(sbd_tpb_handle *h, T *x, const T *const *S, int m, int slot) {
  return sym_dots_impl<T, false>(h, x, S, m, slot);
}

template <typename T>
int symmetrize_dots(sbd_tpb_handle *h, T *x, const T *const *S, int m, int slot) {
  return sym_dots_impl<T, true>(h, x, S, m, slot);
}

template <typename T>
static bool pair_vec_ok(uint32_t nb, const void *const *ptrs, int count) {
  constexpr int VW = 16 / sizeof(T);
  if (nb % VW) return false;
  for (int j = 0; j < count; j++)
    if (ptrs[j] && reinterpret_cast<uintptr_t>(ptrs[j]) % 16) return false;
  return true;
}

template <typename T>
int residual_sym_async(sbd_tpb_handle *h, const ResidualArgs<T> &a, int slot) {
  if (a.m < 1 || a.m > kMaxSub || !a.t || a.W || (sizeof(T) == 4) != (a.hii32 != nullptr))
    return fail(SBD_TPB_ERR_INVALID, "residual_sym: bad arguments");
  TPB_CHECK(ensure_scalars(h));
  const uint32_t nb = (uint32_t)h->bstr.size();
  const int nblk = h->num_sms * kSymBlocksPerSm;
  TPB_CHECK(ensure_partials(h, std::max<size_t>((size_t)(kMaxVec + 3) * vec_blocks(h) + kMaxVec + 3,
                                                (size_t)(kMaxSub + 3) * nblk + 1)));
  const void *ptrs[2 * kMaxSub + 1];
  int np = 0;
  for (int k = 0; k < a.m; k++) {
    ptrs[np++] = a.C.p[k];
    ptrs[np++] = a.HC.p[k];
  }
  ptrs[np++] = a.t;
  const bool vec = pair_vec_ok<T>(nb, ptrs, np);
  int grid = nblk;
  TPB_CHECK(dispatch_n<1>(a.m, [&](auto K) {
    constexpr int M = decltype(K)::value;
    if constexpr (M <= kMaxSub) {
      constexpr bool kPipe = M <= residual_pipe_max<T>();
      constexpr int MP = kPipe ? M : 1;
      constexpr size_t smem = residual_pipe_smem<T, MP>();
      if (vec && kPipe && smem <= h->smem_optin) {
        const auto kern = residual_sym_pipe_kernel<T, MP>;
        TPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        TPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
        grid = h->num_sms * std::max(1, std::min(per_sm, kSymBlocksPerSm));
        kern<<<grid, 256, smem, h->stream>>>(a, nb, h->d_partials);
      } else if (!vec) {
        residual_sym_kernel<T, 1, M><<<nblk, 256, 0, h->stream>>>(a, nb, h->d_partials);
      } else if constexpr (sizeof(T) == 4) {
        residual_sym_f32_kernel<M><<<nblk, 256, 0, h->stream>>>(a, nb, h->d_partials);
      } else {
        residual_sym_kernel<T, 16 / sizeof(T), M><<<nblk, 256, 0, h->stream>>>(a, nb, h->d_partials);
      }
      TPB_LAUNCHED(h);
    }
    return SBD_TPB_OK;
  }));
  return reduce_into(h, a.m + 3, h->d_scal + slot, grid);
}

int random_start_vector(sbd_tpb_handle *h, double *x, size_t n, unsigned long long seed) {
  random_start_kernel<<<h->num_sms * 8, 256, 0, h->stream>>>(x, n, seed);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

template <typename T>
int residual_w_sym_async(sbd_tpb_handle *h, const ResidualArgs<T> &a, int slot) {
  if (a.m < 1 || a.m > kMaxSub || !a.W || a.t) return fail(SBD_TPB_ERR_INVALID, "residual_w_sym: bad arguments");
  TPB_CHECK(ensure_scalars(h));
  const uint32_t nb = (uint32_t)h->bstr.size();
  const int nblk = h->num_sms * kSymBlocksPerSm;
  TPB_CHECK(ensure_partials(h, std::max<size_t>((size_t)(kMaxVec + 3) * vec_blocks(h) + kMaxVec + 3,
                                                (size_t)(kMaxSub + 3) * nblk + 1)));
  const void *ptrs[2 * kMaxSub + 1];
  int np = 0;
  for (int k = 0; k < a.m; k++) {
    ptrs[np++] = a.C.p[k];
    ptrs[np++] = a.HC.p[k];
  }
  ptrs[np++] = a.W;
  if (!pair_vec_ok<T>(nb, ptrs, np)) return residual_step_async<T>(h, a, h->ndet(), slot);
  TPB_CHECK(dispatch_n<1>(a.m, [&](auto K) {
    constexpr int M = decltype(K)::value;
    if constexpr (M <= kMaxSub) {
      residual_w_sym_kernel<T, M><<<nblk, 256, 0, h->stream>>>(a, nb, h->d_partials);
      TPB_LAUNCHED(h);
    }
    return SBD_TPB_OK;
  }));
  return reduce_into(h, a.m + 3, h->d_scal + slot, nblk);
}

template <typename T>
int cgs_sym_async(sbd_tpb_handle *h, const T *const *C, int m, const double *coef, int ov_slot, T *t,
                  int want_dots, int slot, int t0_slot, int tt_slot) {
  if (m < 1 || m > kMaxSub) return fail(SBD_TPB_ERR_INVALID, "subspace larger than supported");
  TPB_CHECK(ensure_scalars(h));
  const uint32_t nb = (uint32_t)h->bstr.size();
  const int nblk = h->num_sms * kSymBlocksPerSm;
  TPB_CHECK(ensure_partials(h, std::max<size_t>((size_t)(kMaxVec + 3) * vec_blocks(h) + kMaxVec + 3,
                                                (size_t)(kMaxSub + 1) * nblk + 1)));
  VecPtrs<T> P;
  CoefArray co;
  const void *ptrs[kMaxSub + 1];
  for (int j = 0; j < kMaxVec; j++) P.p[j] = j < m ? C[j] : nullptr;
  for (int j = 0; j < kMaxSub; j++) co.v[j] = j < m ? coef[j] : 0.0;
  for (int j = 0; j < m; j++) ptrs[j] = C[j];
  ptrs[m] = t;
  const bool vec = pair_vec_ok<T>(nb, ptrs, m + 1);
  const double *p0 = t0_slot >= 0 ? h->d_scal + t0_slot : nullptr;
  const double *p1 = t0_slot >= 0 ? h->d_scal + tt_slot : nullptr;
  TPB_CHECK(dispatch_n<1>(m, [&](auto K) {
    constexpr int M = decltype(K)::value;
    if constexpr (M <= kMaxSub) {
      constexpr int VW = 16 / sizeof(T);
      if (want_dots) {
        if (vec) cgs_sym_kernel<T, VW, M, true><<<nblk, 256, 0, h->stream>>>(P, co, h->d_scal + ov_slot, t, nb, h->d_partials, p0, p1);
        else cgs_sym_kernel<T, 1, M, true><<<nblk, 256, 0, h->stream>>>(P, co, h->d_scal + ov_slot, t, nb, h->d_partials, p0, p1);
      } else {
        if (vec) cgs_sym_kernel<T, VW, M, false><<<nblk, 256, 0, h->stream>>>(P, co, h->d_scal + ov_slot, t, nb, h->d_partials, p0, p1);
        else cgs_sym_kernel<T, 1, M, false><<<nblk, 256, 0, h->stream>>>(P, co, h->d_scal + ov_slot, t, nb, h->d_partials, p0, p1);
      }
      TPB_LAUNCHED(h);
    }
    return SBD_TPB_OK;
  }));
  return reduce_into(h, want_dots ? 1 + m : 1, h->d_scal + slot, nblk);
}

template <typename T>
int scale_vec(sbd_tpb_handle *h, T *x, double a, size_t n) {
  scale_kernel<T><<<vec_blocks(h), kVecThreads, 0, h->stream>>>(x, a, n);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

template <typename S, typename D>
int convert_vec(sbd_tpb_handle *h, const S *x, D *y, size_t n) {
  convert_kernel<S, D><<<vec_blocks(h), kVecThreads, 0, h->stream>>>(x, y, n);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

template <typename T>
int axpby(sbd_tpb_handle *h, const T *x, T *y, double a, double b, size_t n) {
  axpby_kernel<T><<<vec_blocks(h), kVecThreads, 0, h->stream>>>(x, y, a, b, n);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

template int multi_dot_async<double>(sbd_tpb_handle *, const double *const *, int, const double *, size_t, int);
template int multi_dot_async<float>(sbd_tpb_handle *, const float *const *, int, const float *, size_t, int);
template int cgs_second_round_async<double>(sbd_tpb_handle *, const double *const *, int, const double *, int,
                                            double *, size_t, int, int, int);
template int cgs_second_round_async<float>(sbd_tpb_handle *, const float *const *, int, const double *, int,
                                           float *, size_t, int, int, int);
template int sym_add_dots<double>(sbd_tpb_handle *, double *, const double *const *, int, int);
template int sym_add_dots<float>(sbd_tpb_handle *, float *, const float *const *, int, int);
template int symmetrize_dots<double>(sbd_tpb_handle *, double *, const double *const *, int, int);
template int symmetrize_dots<float>(sbd_tpb_handle *, float *, const float *const *, int, int);
template int residual_sym_async<double>(sbd_tpb_handle *, const ResidualArgs<double> &, int);
template int residual_sym_async<float>(sbd_tpb_handle *, const ResidualArgs<float> &, int);
template int residual_w_sym_async<double>(sbd_tpb_handle *, const ResidualArgs<double> &, int);
template int residual_w_sym_async<float>(sbd_tpb_handle *, const ResidualArgs<float> &, int);
template int cgs_sym_async<double>(sbd_tpb_handle *, const double *const *, int, const double *, int, double *, int,
                                   int, int, int);
template int cgs_sym_async<float>(sbd_tpb_handle *, const float *const *, int, const double *, int, float *, int,
                                  int, int, int);
template int sym_add<double>(sbd_tpb_handle *, double *);
template int sym_add<float>(sbd_tpb_handle *, float *);
template int multi_dot<double>(sbd_tpb_handle *, const double *const *, int, const double *,
                               size_t, double *);
template int multi_dot<float>(sbd_tpb_handle *, const float *const *, int, const float *, size_t,
                              double *);
template int residual_step<double>(sbd_tpb_handle *, const ResidualArgs<double> &, size_t,
                                   double *);
template int residual_step<float>(sbd_tpb_handle *, const ResidualArgs<float> &, size_t, double *);
template int cgs_update<double>(sbd_tpb_handle *, const double *const *, int, const double *,
                                double *, size_t, int, double *);
template int cgs_update<float>(sbd_tpb_handle *, const float *const *, int, const double *,
                               float *, size_t, int, double *);
template int residual_step_async<double>(sbd_tpb_handle *, const ResidualArgs<double> &, size_t, int);
template int residual_step_async<float>(sbd_tpb_handle *, const ResidualArgs<float> &, size_t, int);
template int cgs_update_async<double>(sbd_tpb_handle *, const double *const *, int, const double *, int, double *,
                                      size_t, int, int);
template int cgs_update_async<float>(sbd_tpb_handle *, const float *const *, int, const double *, int, float *,
                                     size_t, int, int);
template int symmetrize_async<double>(sbd_tpb_handle *, double *, int);
template int symmetrize_async<float>(sbd_tpb_handle *, float *, int);
template int symmetrize<double>(sbd_tpb_handle *, double *, double *);
template int symmetrize<float>(sbd_tpb_handle *, float *, double *);
template int scale_vec<double>(sbd_tpb_handle *, double *, double, size_t);
template int scale_vec<float>(sbd_tpb_handle *, float *, double, size_t);
template int convert_vec<double, float>(sbd_tpb_handle *, const double *, float *, size_t);
template int convert_vec<float, double>(sbd_tpb_handle *, const float *, double *, size_t);
template int convert_vec<float, float>(sbd_tpb_handle *, const float *, float *, size_t);
template int axpby<double>(sbd_tpb_handle *, const double *, double *, double, double, size_t);
template int axpby<float>(sbd_tpb_handle *, const float *, float *, double, double, size_t);

}  // namespace sbdtpb
