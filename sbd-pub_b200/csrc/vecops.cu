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

template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    multi_dot_kernel(VecPtrs<T> X, int k, const T *__restrict__ y, size_t n, double *partials) {
  double acc[kMaxVec];
#pragma unroll
  for (int j = 0; j < kMaxVec; j++) acc[j] = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double yi = (double)y[i];
#pragma unroll
    for (int j = 0; j < kMaxVec; j++)
      if (j < k) acc[j] += (double)X.p[j][i] * yi;
  }
  block_reduce_store<kMaxVec>(acc, k, partials, gridDim.x);
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
// tpb/davidson.h:861-868) ; partials: [0] = W.W, [1] = r.r, [2+k] = S_k . t, [2+m] = t.t
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    residual_kernel(ResidualArgs<T> a, size_t n, double *partials) {
  double acc[kMaxVec];
#pragma unroll
  for (int j = 0; j < kMaxVec; j++) acc[j] = 0.0;
  const int m = a.m;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    double c[kMaxSub];
    double w = 0.0, hc = 0.0;
#pragma unroll
    for (int k = 0; k < kMaxSub; k++) {
      if (k < m) {
        c[k] = (double)a.C.p[k][i];
        w += a.u[k] * c[k];
        hc += a.u[k] * (double)a.HC.p[k][i];
      }
    }
    const double r = a.e_shifted * w - hc;
    if (a.W) a.W[i] = (T)w;
    acc[0] += w * w;
    acc[1] += r * r;
    if (a.t) {
      const double hd = a.hii32 ? (double)a.hii32[i] : a.hii[i];
      const double d = a.e0 - hd;
      const double t = (fabs(d) > 1.0e-12) ? r / d : r / (d - 1.0e-12);
      const T tt = (T)t;
      a.t[i] = tt;
#pragma unroll
      for (int k = 0; k < kMaxSub; k++)
        if (k < m) acc[2 + k] += c[k] * (double)tt;
      acc[kMaxVec - 1] += (double)tt * (double)tt;
    }
  }
  block_reduce_store<kMaxVec>(acc, kMaxVec, partials, gridDim.x);
}

// t -= sum_k o_k C_k ; partials: [0] = t.t, [1+k] = C_k . t (for a second Gram-Schmidt round)
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    cgs_update_kernel(VecPtrs<T> C, int m, CoefArray o, T *__restrict__ t, size_t n,
                      double *partials, int want_dots) {
  double acc[kMaxVec];
#pragma unroll
  for (int j = 0; j < kMaxVec; j++) acc[j] = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    double c[kMaxSub];
    double x = (double)t[i];
#pragma unroll
    for (int k = 0; k < kMaxSub; k++) {
      if (k < m) {
        c[k] = (double)C.p[k][i];
        x -= o.v[k] * c[k];
      }
    }
    const T xt = (T)x;
    t[i] = xt;
    acc[0] += (double)xt * (double)xt;
    if (want_dots) {
#pragma unroll
      for (int k = 0; k < kMaxSub; k++)
        if (k < m) acc[1 + k] += c[k] * (double)xt;
    }
  }
  block_reduce_store<kMaxVec>(acc, want_dots ? 1 + m : 1, partials, gridDim.x);
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

static int finish_reduce(sbd_tpb_handle *h, int nvals, double *host_out) {
  const int nb = vec_blocks(h);
  double *d_out = h->d_partials + (size_t)kMaxVec * nb;
  reduce_partials_kernel<<<nvals, 256, 0, h->stream>>>(h->d_partials, nb, d_out);
  TPB_LAUNCHED(h);
  TPB_CUDA(cudaMemcpyAsync(host_out, d_out, sizeof(double) * nvals, cudaMemcpyDeviceToHost,
                           h->stream));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  return SBD_TPB_OK;
}

template <typename T>
int multi_dot(sbd_tpb_handle *h, const T *const *X, int k, const T *y, size_t n, double *out) {
  const int nb = vec_blocks(h);
  TPB_CHECK(ensure_partials(h, (size_t)(kMaxVec + 1) * nb + kMaxVec));
  for (int j0 = 0; j0 < k; j0 += kMaxVec) {
    const int kk = std::min(kMaxVec, k - j0);
    VecPtrs<T> P;
    for (int j = 0; j < kMaxVec; j++) P.p[j] = (j < kk) ? X[j0 + j] : nullptr;
    multi_dot_kernel<T><<<nb, kVecThreads, 0, h->stream>>>(P, kk, y, n, h->d_partials);
    TPB_LAUNCHED(h);
    TPB_CHECK(finish_reduce(h, kk, out + j0));
  }
  return SBD_TPB_OK;
}

template <typename T>
int residual_step(sbd_tpb_handle *h, const ResidualArgs<T> &a, size_t n, double *out) {
  if (a.m > kMaxSub) return fail(SBD_TPB_ERR_INVALID, "subspace larger than supported");
  const int nb = vec_blocks(h);
  TPB_CHECK(ensure_partials(h, (size_t)(kMaxVec + 1) * nb + kMaxVec));
  residual_kernel<T><<<nb, kVecThreads, 0, h->stream>>>(a, n, h->d_partials);
  TPB_LAUNCHED(h);
  TPB_CHECK(finish_reduce(h, kMaxVec, out));
  out[2 + a.m] = out[kMaxVec - 1];  // t.t right after the m overlaps
  return SBD_TPB_OK;
}

template <typename T>
int cgs_update(sbd_tpb_handle *h, const T *const *C, int m, const double *o, T *t, size_t n,
               int want_dots, double *out) {
  if (m > kMaxSub) return fail(SBD_TPB_ERR_INVALID, "subspace larger than supported");
  const int nb = vec_blocks(h);
  TPB_CHECK(ensure_partials(h, (size_t)(kMaxVec + 1) * nb + kMaxVec));
  VecPtrs<T> P;
  CoefArray co;
  for (int j = 0; j < kMaxVec; j++) P.p[j] = j < m ? C[j] : nullptr;
  for (int j = 0; j < kMaxSub; j++) co.v[j] = j < m ? o[j] : 0.0;
  cgs_update_kernel<T><<<nb, kVecThreads, 0, h->stream>>>(P, m, co, t, n, h->d_partials, want_dots);
  TPB_LAUNCHED(h);
  return finish_reduce(h, want_dots ? 1 + m : 1, out);
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
template int scale_vec<double>(sbd_tpb_handle *, double *, double, size_t);
template int scale_vec<float>(sbd_tpb_handle *, float *, double, size_t);
template int convert_vec<double, float>(sbd_tpb_handle *, const double *, float *, size_t);
template int convert_vec<float, double>(sbd_tpb_handle *, const float *, double *, size_t);
template int axpby<double>(sbd_tpb_handle *, const double *, double *, double, double, size_t);
template int axpby<float>(sbd_tpb_handle *, const float *, float *, double, double, size_t);

}  // namespace sbdtpb
