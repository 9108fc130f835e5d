// Internal declarations shared by the CUDA translation units of libsbdtpb.
//
// Sign convention inside the library.  The reference evaluates every matrix element on the
// interleaved determinant (alpha orbital p -> spin-orbital 2p, beta p -> 2p+1;
// basic/determinants.h:97-142), so same-spin signs depend on the other spin's string.  The
// library works in the separated ordering (all alpha creators, then all beta), where
// H_sep = D H_ref D with D = diag((-1)^phi(Ia,Ib)) and phi = #{(p in Ia, q in Ib) : q < p}.
// In that ordering the alpha part of H acts on the alpha index only (up to the diagonal-in-beta
// Coulomb term of alpha singles), which is what lets sigma run as row/column SpMM and as a
// gather -> dense (pq|rs) contraction -> scatter.  Energies, RDMs and iteration counts are
// invariant; vectors crossing the C ABI are multiplied by D on the way in and out.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <chrono>

#include <string>
#include <vector>

#include "../../include/sbd_tpb.h"

namespace sbdtpb {

// ---- error plumbing: every CUDA call goes through this and turns into a status ------------
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);

#define TPB_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      int code_ = (e_ == cudaErrorMemoryAllocation) ? SBD_TPB_ERR_OOM : SBD_TPB_ERR_CUDA;   \
      return ::sbdtpb::fail(code_, std::string(#call) + ": " + cudaGetErrorString(e_));    \
    }                                                                                       \
  } while (0)

#define TPB_LAUNCHED(h)                                                                     \
  do {                                                                                      \
    (h)->launches++;                                                                        \
    cudaError_t e_ = cudaGetLastError();                                                    \
    if (e_ != cudaSuccess)                                                                  \
      return ::sbdtpb::fail(SBD_TPB_ERR_CUDA, std::string("kernel launch: ") +              \
                                                  cudaGetErrorString(e_));                  \
  } while (0)

#define TPB_CHECK(expr)            \
  do {                             \
    int rc_ = (expr);              \
    if (rc_ != SBD_TPB_OK) return rc_; \
  } while (0)

// ---- device bit helpers ---------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t open_mask(int lo, int hi) {
  // bits strictly between lo and hi (0 <= lo < hi <= 63)
  return ((1ull << hi) - 1ull) & ~((2ull << lo) - 1ull);
}

__device__ __forceinline__ int lowest_bit(uint64_t x) { return __ffsll((long long)x) - 1; }
__device__ __forceinline__ int highest_bit(uint64_t x) { return 63 - __clzll((long long)x); }

// Sign bit (0 or 1) of the interleaved -> separated reordering of determinant (a, b):
// parity of #{(p in a, q in b): q < p} = popcount(b & P(a)), P(a)_q = parity of a's bits > q.
__host__ __device__ __forceinline__ uint64_t above_parity_mask(uint64_t a) {
  uint64_t s = a;
  s ^= s >> 1;
  s ^= s >> 2;
  s ^= s >> 4;
  s ^= s >> 8;
  s ^= s >> 16;
  s ^= s >> 32;  // bit q = xor of a's bits at positions >= q
  return s >> 1;  // bit q = xor of a's bits at positions > q
}

// ---- device-resident tables -----------------------------------------------------------------
// One spin's excitation table in CSR form.  lab packs the spatial orbitals of an entry:
// singles (cr | an << 8), doubles (cr0 | cr1 << 8 | an0 << 16 | an1 << 24), cr < 64.
struct ExTable {
  uint32_t *off = nullptr;  // [n+1]
  uint32_t *ket = nullptr;  // [nnz]
  uint32_t *lab = nullptr;  // [nnz]
  size_t nnz = 0;
  uint32_t max_row = 0;     // longest bra row
};

// One spin's sigma program: the separated-convention matrix element of every excitation-table
// entry, aligned with the table (same offsets and ket indices).  Singles carry, in s_pair,
// +-(an*L + cr + 1): the sign of the element and the orbital pair of the other-spin Coulomb term
// sgn * sum_{k in other string} (an cr|kk) that the sigma kernels add.
struct SigmaProg {
  const ExTable *s = nullptr, *d = nullptr;  // singles / doubles tables (offsets, kets)
  double *s_val = nullptr;
  float *s_valf = nullptr;
  int32_t *s_pair = nullptr;
  double *d_val = nullptr;
  float *d_valf = nullptr;
  // other-spin Coulomb sums of the singles: jtab[pidx(pq)][c] = sum_{k in string c of the column
  // spin} (pq|kk), one row per pair pq that some single of this program carries (pmap[pq] = its
  // row, -1 for the others); built by build_coulomb_table
  double *jtab = nullptr;
  int32_t *pmap = nullptr;
  uint32_t npair = 0;
  bool jtab_tried = false;  // built, or found too large, once per program
};

// Dense-path data for the alpha-beta term as gather -> (pq|rs) contraction -> scatter.
struct ABDense {
  bool enabled = false;
  int npq = 0, nrs = 0;           // distinct alpha / beta single labels
  int *pq_of_label = nullptr;     // unused placeholders kept for layout stability
  int *rs_of_label = nullptr;
  int32_t *a_label = nullptr;     // [alpha singles] +-(label+1), sign = s_a
  int32_t *b_label = nullptr;     // [beta singles]  +-(label+1), sign = s_b
  double *V = nullptr;            // [npq][nrs] (pq|rs), FP64
  float *Vf = nullptr;            // same in FP32
  // tensor-core path (FP32 sigma): V as BF16 hi/lo in the tcgen05 canonical layout
  bool tc_ready = false;
  int Kp = 0, Np = 0;
  int tc_fused_stages = 0;        // A stages of the fused gather + contraction kernel (0: unfused)
  uint16_t *Vhi = nullptr, *Vlo = nullptr;
  int *err = nullptr;             // bounded-wait status of the tensor-core kernel
};

}  // namespace sbdtpb

struct sbd_tpb_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_k[4] = {nullptr, nullptr, nullptr, nullptr};  // between sigma kernels
  uint64_t launches = 0;
  float last_sigma_ms = 0.f;
  int sigma_kernels = 0;  // kernels timed in the last sigma (ev0, ev_k[0..], ev1)
  cudaEvent_t ev_co[2] = {nullptr, nullptr};  // around the weight pass of the last carry-over
  float last_carryover_ms[2] = {0.f, 0.f};    // weight pass, whole call
  float last_parse_ms = 0.f;                   // last string-file parse (copy, parse, sort)
  void *h_stage = nullptr;                     // pinned staging of string files (grow-only)
  size_t stage_cap = 0;
  int num_sms = 148;
  size_t smem_optin = 0;

  // problem (host copies)
  int L = 0, nelec = 0;
  double I0 = 0.0;
  std::vector<double> h1;          // L*L
  std::vector<double> eri_packed;  // packed store
  std::vector<uint64_t> astr, bstr;
  int n_alpha = 0, n_beta = 0;
  bool have_ham = false, have_strings = false, have_tables = false;

  // device data
  double *d_eri = nullptr;   // [L*L][L*L] full (pq|rs)
  double *d_vd = nullptr;    // [L*L][L] (pq|kk)
  double *d_J = nullptr;     // [L][L] (pp|qq)
  uint64_t *d_astr = nullptr, *d_bstr = nullptr;
  uint64_t *d_apar = nullptr;  // [na] above_parity_mask(astr)
  double *d_Ea = nullptr, *d_Eb = nullptr;  // same-spin string energies
  double *d_uJ = nullptr;    // [na][L]: sum_{p in Ia} (pp|qq)
  double *d_hii = nullptr;   // [na*nb] FP64 diagonal
  float *d_hii32 = nullptr;  // [na*nb] H_ii - H_00 in FP32 (FP32 sigma)
  double h00 = 0.0;          // H_00
  sbdtpb::ExTable ta_s, ta_d, tb_s, tb_d;
  sbdtpb::SigmaProg pa, pb;
  sbdtpb::ABDense ab;

  // scratch
  double *d_partials = nullptr;  // reduction partial sums
  size_t partials_cap = 0;
  double *d_scal = nullptr, *h_scal = nullptr;  // reduction results read back together (pinned)
  // N-vectors of finished Davidson runs kept for the next run (allocating tens of GB per solve
  // costs a noticeable and variable fraction of a solve); freed with the problem
  std::vector<std::pair<void *, size_t>> vec_pool;
  double *d_tmp64 = nullptr;     // one N-vector FP64 (sign conversion staging)
  double *d_tmp64b = nullptr;
  float *d_tmp32 = nullptr, *d_tmp32b = nullptr;
  uint32_t blk_max[4] = {0, 0, 0, 0};  // per-block table entries (alpha d/s, beta d/s)
  const void *blk_for = nullptr;        // tables blk_max was computed for
  void *d_ct = nullptr;          // C^T staging of the beta pass of sigma
  size_t ct_bytes = 0;
  void *d_ab_work = nullptr;     // dense alpha-beta intermediates
  size_t ab_work_bytes = 0;
  // sparse alpha-beta term: alpha rows and beta columns that have at least one single
  uint32_t *d_ab_rows = nullptr;
  uint2 *d_ab_colp = nullptr;  // per ket range, per beta column with singles (most singles first): (column, first entry); then (0, end of the range's entries)
  uint2 *d_ab_bsp = nullptr;   // beta singles entries packed as (ket position in d_ab_kets, signed pair label)
  uint32_t *d_ab_kets = nullptr;  // distinct kets of the beta singles, ascending
  uint32_t ab_nkets = 0;
  uint32_t ab_nrows = 0, ab_ncols = 0, ab_max_k = 0;  // ab_max_k: most singles of one alpha row
  uint32_t ab_nchunks = 1, ab_chunk = 0;              // ket ranges of the beta program, kets per range
  bool ab_dense = false;                              // beta program of more than 4 entries per ket
  // learned preconditioner attached by sbd_tpb_set_preconditioner (not owned) and the
  // occupation windows of the strings it reads
  struct sbd_tpb_precond *precond = nullptr;
  uint32_t *d_occw_a = nullptr, *d_occw_b = nullptr;
  double *d_kx_a = nullptr, *d_kx_b = nullptr;  // same-spin exchange sum of each string
  uint32_t *d_mlp_idx = nullptr;  // determinants selected for the learned correction (+ counter)
  size_t ndet() const { return astr.size() * bstr.size(); }
};

namespace sbdtpb {
// strings.cu: parse/sort/unique a string file held in host memory; ms (may be null) receives the
// device time from the copy to the last kernel
int parse_strings_device(sbd_tpb_handle *h, const void *host_bytes, size_t nbytes, int format, int norb,
                         uint64_t *out, size_t cap, size_t *count, float *ms);
// carryover.cu: carry-over strings of a device vector (either sign convention)
int carryover_device(sbd_tpb_handle *h, const double *dW, sbd_tpb_carryover *co);
// tables.cu
int build_excitation_tables(sbd_tpb_handle *h);
int copy_table_reference_layout(sbd_tpb_handle *h, int kind, uint64_t *off, uint64_t *ket,
                                int32_t *cran);
// hamiltonian.cu
int upload_hamiltonian(sbd_tpb_handle *h);
int build_string_data(sbd_tpb_handle *h);
int build_sigma_programs(sbd_tpb_handle *h);
// jtab/pmap of a sigma program whose columns are the strings col_str[0..ncols)
int build_coulomb_table(sbd_tpb_handle *h, SigmaProg &p, const uint64_t *col_str, size_t ncols);
int compute_diagonal(sbd_tpb_handle *h);
void free_device_problem(sbd_tpb_handle *h);
// sigma.cu
template <typename T>
int sigma_sep(sbd_tpb_handle *h, const T *C, T *sigma, int accumulate);
// sigma (+)= (H - shift) C
template <typename T>
int sigma_sep_shift(sbd_tpb_handle *h, const T *C, T *sigma, int accumulate, double shift);
// sigma (+)= H C with a caller-provided C^T buffer of ndet elements; no device allocation
template <typename T>
int sigma_sep_given_ct(sbd_tpb_handle *h, const T *C, T *sigma, int accumulate, T *CT);
// sigma = (H - shift) C for C = C^T over identical alpha and beta strings: one gathering pass and
// an in-place B + B^T (see sigma.cu)
template <typename T>
int sigma_sep_sym(sbd_tpb_handle *h, const T *C, T *sigma, double shift, const T *const *S = nullptr, int m = 0,
                  int slot = 0);
// per-block table sizes of the sigma launches, read back once per table build (blk_max, blk_for)
int prepare_block_sizes(sbd_tpb_handle *h);
int reorder_sign_apply_f64(sbd_tpb_handle *h, const double *x, double *y);
int reorder_sign_apply_f32(sbd_tpb_handle *h, const float *x, float *y);
// ab_dense.cu: alpha-beta term as gather -> dense (pq|rs) contraction -> scatter
int ab_dense_setup(sbd_tpb_handle *h, int enable);
bool ab_dense_worthwhile(sbd_tpb_handle *h);
template <typename T>
int ab_dense_apply(sbd_tpb_handle *h, const T *C, T *sigma, double scale = 1.0);
// vecops.cu
int ensure_partials(sbd_tpb_handle *h, size_t n);
template <typename T>
int multi_dot(sbd_tpb_handle *h, const T *const *X, int k, const T *y, size_t n, double *out);
// rdm.cu
// W: device FP64 vector in the separated convention; outputs are host arrays (any may be null):
// one [2L^2], two [4L^4] in the reference layouts, density [2L].
// vector pool (davidson.cu): a block of at least `bytes` (reused if one of at most twice the size
// is free, else cudaMalloc, emptying the pool and retrying once if memory is short), its return,
// and the release of every kept block
int pool_get(sbd_tpb_handle *h, size_t bytes, void **out);
void pool_put(sbd_tpb_handle *h, void *p, size_t bytes);
void pool_clear(sbd_tpb_handle *h);
// an N-vector from the pool, returned to it on scope exit (or by release())
template <typename T>
struct DevVec {
  sbd_tpb_handle *h = nullptr;
  T *p = nullptr;
  size_t bytes = 0;
  int get(sbd_tpb_handle *hh, size_t count) {
    h = hh;
    bytes = count * sizeof(T);
    void *q = nullptr;
    const int rc = pool_get(h, bytes, &q);
    p = static_cast<T *>(q);
    return rc;
  }
  DevVec() = default;
  DevVec(const DevVec &) = delete;
  DevVec &operator=(const DevVec &) = delete;
  DevVec(DevVec &&o) noexcept : h(o.h), p(o.p), bytes(o.bytes) { o.p = nullptr; }
  void release() {
    if (p) pool_put(h, p, bytes);
    p = nullptr;
  }
  ~DevVec() { release(); }
};
int rdm_sep(sbd_tpb_handle *h, const double *W, double *one, double *two, double *density);
// davidson.cu
int davidson_run(sbd_tpb_handle *h, const sbd_tpb_params *p, const double *W0,
                 sbd_tpb_result *res);
// after a solve: final FP64 sigma of the device vector dW (separated convention) for the energy
// <W|H|W> and |HW - E W| (reported unless resid >= 0 is given), then the caller's CI vector,
// occupations/RDMs and carry-over strings; fills res and returns the solve's status
int solve_finish(sbd_tpb_handle *h, double *dW, sbd_tpb_result *res,
                 std::chrono::steady_clock::time_point t0, int nsig, int conv, double resid,
                 bool sym_w = false);
// lanczos.cu
int lanczos_run(sbd_tpb_handle *h, const sbd_tpb_params *p, const double *W0, sbd_tpb_result *res);
}  // namespace sbdtpb
