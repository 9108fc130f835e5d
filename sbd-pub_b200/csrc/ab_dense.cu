// Alpha-beta term of sigma as gather -> dense (pq|rs) contraction -> scatter.
//
// The reference evaluates every alpha-single x beta-single pair on its own
// (MultAlphaBeta, tpb/mult_thrust.h:382-520; TwoExcite per pair, tpb/mult.h:820-846): for FCI-like
// string sets that is ~S_a*S_b/N ~ 10^3 element evaluations and random gathers per determinant.
// In the separated convention the pair element factorises, H = s_a(Ia->Ja) s_b(Ib->Jb) (pq|rs),
// so the same sum is
//   D[rs][Ja, Ib] = sum_{Jb: Ib->Jb has label rs} s_b C[Ja, Jb]          (gather)
//   E[pq][Ja, Ib] = sum_rs (pq|rs) D[rs][Ja, Ib]                          (dense contraction)
//   sigma[Ia, Ib] += sum_{Ja: Ia->Ja has label pq} s_a E[pq][Ja, Ib]      (scatter)
// with the contraction a GEMM of M = na*nb rows and K, N = the number of distinct beta / alpha
// single labels.  D and E are stored label-major ([label][det]) so the gather writes and the
// scatter reads are coalesced along Ib.  The path is chosen when the pair count per determinant is
// high and D, E fit the memory budget (FCI-like problems); sparse string sets keep the direct loop
// of the row kernel.  The FP64 contraction runs on FP64 units; the FP32 path splits D and (pq|rs)
// into BF16 hi + lo parts on the tensor cores (ab_tc.cu) with FP32 accumulation.
#include <algorithm>
#include <map>
#include <vector>

#include "ab_tc.cuh"
#include "tpb_common.cuh"

namespace sbdtpb {
namespace {

template <typename T>
__global__ void ab_gather_kernel(const T *__restrict__ C, uint32_t na, uint32_t nb,
                                 const uint32_t *__restrict__ b_off, const uint32_t *__restrict__ b_ket,
                                 const int32_t *__restrict__ b_label, size_t M, T *__restrict__ D) {
  const size_t total = (size_t)na * nb;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < total;
       j += (size_t)gridDim.x * blockDim.x) {
    const uint32_t ja = (uint32_t)(j / nb), ib = (uint32_t)(j - (size_t)ja * nb);
    const T *crow = C + (size_t)ja * nb;
    for (uint32_t e = b_off[ib]; e < b_off[ib + 1]; e++) {
      const int32_t lab = b_label[e];
      const T c = crow[b_ket[e]];
      D[(size_t)((lab > 0 ? lab : -lab) - 1) * M + j] = lab > 0 ? c : -c;
    }
  }
}

template <typename T>
__global__ void ab_scatter_kernel(const T *__restrict__ E, uint32_t na, uint32_t nb,
                                  const uint32_t *__restrict__ a_off, const uint32_t *__restrict__ a_ket,
                                  const int32_t *__restrict__ a_label, size_t M, T *__restrict__ sigma,
                                  T scale) {
  const size_t total = (size_t)na * nb;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t ia = (uint32_t)(i / nb), ib = (uint32_t)(i - (size_t)ia * nb);
    T acc = T(0);
    for (uint32_t e = a_off[ia]; e < a_off[ia + 1]; e++) {
      const int32_t lab = a_label[e];
      const T x = E[(size_t)((lab > 0 ? lab : -lab) - 1) * M + (size_t)a_ket[e] * nb + ib];
      acc += lab > 0 ? x : -x;
    }
    sigma[i] += acc * scale;
  }
}

// E[n][j] = sum_k V[n][k] D[k][j]  (row-major, V: N x K, D: K x M, E: N x M) on CUDA cores.
// CTA tile 64 (n) x 128 (j), K chunks of 16, each thread 4 x 8 outputs.
template <typename T>
__global__ void __launch_bounds__(256)
    ab_gemm_kernel(const T *__restrict__ V, const T *__restrict__ D, T *__restrict__ E, int N, int K,
                   size_t M) {
  __shared__ T sV[16][64 + 1];
  __shared__ T sD[16][128];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // 16 x 16 threads
  const int n0 = blockIdx.y * 64;
  const size_t j0 = (size_t)blockIdx.x * 128;
  T acc[4][8];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 8; b++) acc[a][b] = T(0);
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int t = threadIdx.x; t < 16 * 64; t += 256) {
      const int kk = t % 16, nn = t / 16;
      sV[kk][nn] = (n0 + nn < N && k0 + kk < K) ? V[(size_t)(n0 + nn) * K + k0 + kk] : T(0);
    }
    for (int t = threadIdx.x; t < 16 * 128; t += 256) {
      const int kk = t / 128, jj = t % 128;
      sD[kk][jj] = (k0 + kk < K && j0 + jj < M) ? D[(size_t)(k0 + kk) * M + j0 + jj] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      T v[4], d[8];
#pragma unroll
      for (int a = 0; a < 4; a++) v[a] = sV[kk][ty * 4 + a];
#pragma unroll
      for (int b = 0; b < 8; b++) d[b] = sD[kk][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] += v[a] * d[b];
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; a++) {
    const int n = n0 + ty * 4 + a;
    if (n >= N) continue;
#pragma unroll
    for (int b = 0; b < 8; b++) {
      const size_t j = j0 + tx + 16 * b;
      if (j < M) E[(size_t)n * M + j] = acc[a][b];
    }
  }
}

template <typename T>
void free_dev(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

}  // namespace

int ab_dense_setup(sbd_tpb_handle *h, int enable) {
  ABDense &ab = h->ab;
  free_dev(ab.pq_of_label);
  free_dev(ab.rs_of_label);
  free_dev(ab.a_label);
  free_dev(ab.b_label);
  free_dev(ab.V);
  free_dev(ab.Vf);
  free_dev(ab.Vhi);
  free_dev(ab.Vlo);
  free_dev(ab.err);
  ab = ABDense();
  if (h->d_ab_work) cudaFree(h->d_ab_work);
  h->d_ab_work = nullptr;
  h->ab_work_bytes = 0;
  if (!enable || h->ta_s.nnz == 0 || h->tb_s.nnz == 0) return SBD_TPB_OK;
  const int L = h->L;
  const size_t na = h->astr.size(), nb = h->bstr.size(), n = na * nb;
  // labels of the singles tables
  auto labels = [&](const ExTable &t, const std::vector<uint64_t> &str, std::vector<int32_t> &lab,
                    std::vector<int> &pairs) -> int {
    std::vector<uint32_t> off(str.size() + 1), lb(t.nnz);
    TPB_CUDA(cudaMemcpy(off.data(), t.off, sizeof(uint32_t) * off.size(), cudaMemcpyDeviceToHost));
    TPB_CUDA(cudaMemcpy(lb.data(), t.lab, sizeof(uint32_t) * t.nnz, cudaMemcpyDeviceToHost));
    std::map<int, int> id;
    lab.resize(t.nnz);
    for (size_t i = 0; i < str.size(); i++) {
      for (uint32_t e = off[i]; e < off[i + 1]; e++) {
        const int cr = lb[e] & 0xff, an = (lb[e] >> 8) & 0xff;
        const int pair = an * L + cr;
        auto it = id.find(pair);
        int k;
        if (it == id.end()) {
          k = (int)pairs.size();
          id[pair] = k;
          pairs.push_back(pair);
        } else {
          k = it->second;
        }
        const int lo = std::min(cr, an), hi = std::max(cr, an);
        const bool neg = __builtin_popcountll(str[i] & open_mask(lo, hi)) & 1;
        lab[e] = neg ? -(k + 1) : (k + 1);
      }
    }
    return SBD_TPB_OK;
  };
  std::vector<int32_t> alab, blab;
  std::vector<int> apairs, bpairs;
  TPB_CHECK(labels(h->ta_s, h->astr, alab, apairs));
  TPB_CHECK(labels(h->tb_s, h->bstr, blab, bpairs));
  ab.npq = (int)apairs.size();
  ab.nrs = (int)bpairs.size();
  // V[pq][rs] = (pq|rs), pair index an*L + cr on both sides
  std::vector<double> V((size_t)ab.npq * ab.nrs);
  std::vector<double> eri((size_t)L * L * L * L);
  TPB_CUDA(cudaMemcpy(eri.data(), h->d_eri, sizeof(double) * eri.size(), cudaMemcpyDeviceToHost));
  for (int p = 0; p < ab.npq; p++)
    for (int r = 0; r < ab.nrs; r++)
      V[(size_t)p * ab.nrs + r] = eri[(size_t)apairs[p] * L * L + bpairs[r]];
  std::vector<float> Vf(V.begin(), V.end());
  TPB_CUDA(cudaMalloc(&ab.a_label, sizeof(int32_t) * alab.size()));
  TPB_CUDA(cudaMalloc(&ab.b_label, sizeof(int32_t) * blab.size()));
  TPB_CUDA(cudaMalloc(&ab.V, sizeof(double) * V.size()));
  TPB_CUDA(cudaMalloc(&ab.Vf, sizeof(float) * Vf.size()));
  TPB_CUDA(cudaMemcpy(ab.a_label, alab.data(), sizeof(int32_t) * alab.size(), cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(ab.b_label, blab.data(), sizeof(int32_t) * blab.size(), cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(ab.V, V.data(), sizeof(double) * V.size(), cudaMemcpyHostToDevice));
  TPB_CUDA(cudaMemcpy(ab.Vf, Vf.data(), sizeof(float) * Vf.size(), cudaMemcpyHostToDevice));
  TPB_CHECK(ab_tc_setup(h));
  ab.enabled = true;
  (void)n;
  return SBD_TPB_OK;
}

bool ab_dense_worthwhile(sbd_tpb_handle *h) {
  // direct cost ~ pairs per determinant; dense memory = n * (nrs + npq) values
  const double n = (double)h->ndet();
  if (h->ta_s.nnz == 0 || h->tb_s.nnz == 0 || n == 0) return false;
  const double pairs_per_det = (double)h->ta_s.nnz * (double)h->tb_s.nnz / n;
  if (pairs_per_det < 64.0) return false;
  // distinct labels are at most L(L-1); bound the two work arrays by 4 GB at FP64
  const double labels = (double)h->L * (h->L - 1);
  return n * 2.0 * labels * 8.0 <= 4.0e9;
}

template <typename T>
int ab_dense_apply(sbd_tpb_handle *h, const T *C, T *sigma, double scale) {
  ABDense &ab = h->ab;
  const uint32_t na = (uint32_t)h->astr.size(), nb = (uint32_t)h->bstr.size();
  const size_t M = (size_t)na * nb;
  const bool tc = sizeof(T) == 4 && ab.tc_ready;
  const bool fused = tc && ab.tc_fused_stages > 0;
  const size_t need = fused ? ab_tc_fused_work_bytes(h)
                            : tc ? ab_tc_work_bytes(h) : sizeof(T) * M * (size_t)(ab.npq + ab.nrs);
  if (h->ab_work_bytes < need) {
    if (h->d_ab_work) cudaFree(h->d_ab_work);
    h->d_ab_work = nullptr;
    h->ab_work_bytes = 0;
    TPB_CUDA(cudaMalloc(&h->d_ab_work, need));
    h->ab_work_bytes = need;
  }
  const int grid = h->num_sms * 8;
  T *E = nullptr;
  if (fused) {
    E = reinterpret_cast<T *>(h->d_ab_work);
    TPB_CHECK(ab_tc_fused(h, reinterpret_cast<const float *>(C), reinterpret_cast<float *>(E), M));
  } else if (tc) {
    const size_t Mp = (M + 127) / 128 * 128;
    E = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(h->d_ab_work) +
                              Mp * ab.Kp * 2 * sizeof(uint16_t));
    TPB_CHECK(ab_tc_gather(h, reinterpret_cast<const float *>(C), M));
    TPB_CHECK(ab_tc_gemm(h, nullptr, reinterpret_cast<float *>(E), M));
  } else {
    T *D = reinterpret_cast<T *>(h->d_ab_work);
    E = D + M * ab.nrs;
    TPB_CUDA(cudaMemsetAsync(D, 0, sizeof(T) * M * ab.nrs, h->stream));
    ab_gather_kernel<T><<<grid, 256, 0, h->stream>>>(C, na, nb, h->tb_s.off, h->tb_s.ket, ab.b_label, M, D);
    TPB_LAUNCHED(h);
    dim3 g((unsigned)((M + 127) / 128), (unsigned)((ab.npq + 63) / 64));
    const T *V = sizeof(T) == 8 ? reinterpret_cast<const T *>(ab.V) : reinterpret_cast<const T *>(ab.Vf);
    ab_gemm_kernel<T><<<g, 256, 0, h->stream>>>(V, D, E, ab.npq, ab.nrs, M);
    TPB_LAUNCHED(h);
  }
  ab_scatter_kernel<T><<<grid, 256, 0, h->stream>>>(E, na, nb, h->ta_s.off, h->ta_s.ket, ab.a_label, M, sigma,
                                                    (T)scale);
  TPB_LAUNCHED(h);
  if (tc) TPB_CHECK(ab_tc_check(h));
  return SBD_TPB_OK;
}

template int ab_dense_apply<double>(sbd_tpb_handle *, const double *, double *, double);
template int ab_dense_apply<float>(sbd_tpb_handle *, const float *, float *, double);

}  // namespace sbdtpb
