// String files on the GPU: parsing, sorting and de-duplication of alpha/beta occupation strings
// as LoadAlphaDets leaves them (basic/makedeterminants.h:160-186).
//
//   text (.txt): one string per line, orbital 0 the LAST of the first norb characters
//     (from_string, framework/bit_manipulation.h:215-230).  As the library's host reader does:
//     trailing '\r' and spaces are dropped, empty lines skipped, characters after the first norb
//     ignored; a line shorter than norb, or a character other than 0/1 among the first norb, is an
//     error (the reference reads past short lines and takes any character but '1' as 0).
//   binary (.bin): records of ceil(norb/8) bytes, an unsigned big-endian integer whose low norb
//     bits are orbitals 0..norb-1 (DecodeAlphaDets, basic/makedeterminants.h:63-108: the leading
//     8*bytes - norb bits are skipped, the rest read from the most significant bit and reversed);
//     a trailing partial record is ignored, as the reference's read loop does.
//   Then ascending sort and duplicates removed (sort_bitarray, bit_manipulation.h:381-392).
//
// The bytes are copied to HBM once; newline positions come from a flagged selection over all
// bytes, every text line is parsed by one warp (two characters a lane, ballots give the bit
// mask, one bit reversal puts orbital 0 at bit 0), and the strings are sorted by a radix sort
// over the low norb bits and made unique (CUB).
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "tpb_common.cuh"

namespace sbdtpb {
namespace {

constexpr int kStrThreads = 256;

// error record: (failing line, 1-based) << 2 | kind, kind 1 = short line, 2 = a character other
// than 0/1; the smallest line wins (ULLONG_MAX: none)

struct IsNewline {
  const char *b;
  __device__ __forceinline__ bool operator()(const uint32_t &i) const { return b[i] == '\n'; }
};
struct NewlineCount {
  const char *b;
  __device__ __forceinline__ uint32_t operator()(const uint32_t &i) const { return b[i] == '\n' ? 1u : 0u; }
};

__device__ __forceinline__ void record_error(unsigned long long *e, unsigned long long line, int kind) {
  atomicMin(e, (line << 2) | (unsigned long long)kind);
}

// warp per line: line k spans [start, end) with start = nl[k-1] + 1 (0 for k = 0) and end = nl[k]
// (the byte count for the last line when the file does not end in a newline)
__global__ void __launch_bounds__(kStrThreads) parse_lines_kernel(const char *__restrict__ bytes, size_t nbytes,
                                                                  const uint32_t *__restrict__ nl, size_t nnl,
                                                                  size_t nlines, int norb,
                                                                  uint64_t *__restrict__ out,
                                                                  uint8_t *__restrict__ keep,
                                                                  unsigned long long *__restrict__ err) {
  const size_t k = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (k >= nlines) return;
  const size_t start = k ? nl[k - 1] + 1 : 0;
  size_t end = k < nnl ? nl[k] : nbytes;
  // trailing '\r' and spaces
  while (end > start && (bytes[end - 1] == '\r' || bytes[end - 1] == ' ')) end--;
  const size_t len = end - start;
  if (len == 0) {
    if (lane == 0) {
      keep[k] = 0;
      out[k] = 0;
    }
    return;
  }
  if (len < (size_t)norb) {
    if (lane == 0) {
      keep[k] = 0;
      out[k] = 0;
      record_error(err, k + 1, 1);
    }
    return;
  }
  // character j of the line is orbital norb-1-j
  const int j0 = lane, j1 = lane + 32;
  const char c0 = j0 < norb ? bytes[start + j0] : '0';
  const char c1 = j1 < norb ? bytes[start + j1] : '0';
  const unsigned ones0 = __ballot_sync(0xffffffffu, c0 == '1');
  const unsigned ones1 = __ballot_sync(0xffffffffu, c1 == '1');
  const unsigned bad = __ballot_sync(0xffffffffu, (c0 != '0' && c0 != '1') || (c1 != '0' && c1 != '1'));
  if (lane == 0) {
    const uint64_t m = (uint64_t)ones0 | ((uint64_t)ones1 << 32);  // bit j = character j
    out[k] = __brevll(m) >> (64 - norb);
    keep[k] = bad ? 0 : 1;
    if (bad) record_error(err, k + 1, 2);
  }
}

// record i: bytes [i*rb, (i+1)*rb) as a big-endian integer, low norb bits
__global__ void parse_records_kernel(const unsigned char *__restrict__ bytes, size_t nrec, int rb, int norb,
                                     uint64_t *__restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrec) return;
  const unsigned char *p = bytes + i * (size_t)rb;
  uint64_t v = 0;
  for (int b = 0; b < rb; b++) v = (v << 8) | p[b];
  out[i] = norb == 64 ? v : (v & ((1ull << norb) - 1ull));
}

inline unsigned grid_for(size_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

struct Bufs {
  sbd_tpb_handle *h;
  std::vector<std::pair<void *, size_t>> got;
  explicit Bufs(sbd_tpb_handle *hh) : h(hh) {}
  ~Bufs() {
    for (auto &g : got) pool_put(h, g.first, g.second);
  }
  template <typename T>
  int get(T **out, size_t count) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    void *p = nullptr;
    TPB_CHECK(pool_get(h, bytes, &p));
    got.emplace_back(p, bytes);
    *out = (T *)p;
    return SBD_TPB_OK;
  }
};

}  // namespace

int parse_strings_device(sbd_tpb_handle *h, const void *host_bytes, size_t nbytes, int format, int norb,
                         uint64_t *out, size_t cap, size_t *count, float *ms) {
  if (norb < 1 || norb > 64) return fail(SBD_TPB_ERR_INVALID, "strings: norb must be in [1, 64]");
  if (format != SBD_TPB_STRINGS_TEXT && format != SBD_TPB_STRINGS_BINARY)
    return fail(SBD_TPB_ERR_INVALID, "strings: unknown format");
  if (!host_bytes && nbytes) return fail(SBD_TPB_ERR_INVALID, "strings: null buffer");
  *count = 0;
  Bufs B(h);
  char *d_bytes = nullptr;
  TPB_CHECK(B.get(&d_bytes, nbytes + 8));
  TPB_CUDA(cudaEventRecord(h->ev_co[0], h->stream));
  if (nbytes) TPB_CUDA(cudaMemcpyAsync(d_bytes, host_bytes, nbytes, cudaMemcpyHostToDevice, h->stream));
  size_t nstr = 0;
  uint64_t *d_vals = nullptr, *d_keys = nullptr;
  if (format == SBD_TPB_STRINGS_BINARY) {
    const int rb = (norb + 7) / 8;
    nstr = nbytes / rb;
    if (nstr > (size_t)INT32_MAX) return fail(SBD_TPB_ERR_INVALID, "strings: more than 2^31 records");
    TPB_CHECK(B.get(&d_vals, nstr));
    if (nstr) {
      parse_records_kernel<<<grid_for(nstr, 256), 256, 0, h->stream>>>((const unsigned char *)d_bytes, nstr, rb,
                                                                        norb, d_vals);
      TPB_LAUNCHED(h);
    }
  } else {
    if (nbytes > (size_t)INT32_MAX)
      return fail(SBD_TPB_ERR_INVALID, "strings: text files above 2 GiB are not supported");
    // newline count, then their positions (32-bit: text files below 2 GiB)
    thrust::counting_iterator<uint32_t> idx(0);
    uint32_t *d_cnt = nullptr;
    int *d_nnl = nullptr;
    TPB_CHECK(B.get(&d_cnt, 1));
    TPB_CHECK(B.get(&d_nnl, 1));
    thrust::transform_iterator<NewlineCount, thrust::counting_iterator<uint32_t>> flags(idx, NewlineCount{d_bytes});
    size_t tc = 0;
    TPB_CUDA(cub::DeviceReduce::Sum(nullptr, tc, flags, d_cnt, (int)nbytes, h->stream));
    void *tmpc = nullptr;
    TPB_CHECK(B.get((uint8_t **)&tmpc, tc));
    TPB_CUDA(cub::DeviceReduce::Sum(tmpc, tc, flags, d_cnt, (int)nbytes, h->stream));
    uint32_t cnt = 0;
    char last = '\n';
    TPB_CUDA(cudaMemcpyAsync(&cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream));
    if (nbytes) TPB_CUDA(cudaMemcpyAsync(&last, d_bytes + nbytes - 1, 1, cudaMemcpyDeviceToHost, h->stream));
    TPB_CUDA(cudaStreamSynchronize(h->stream));
    uint32_t *d_nl = nullptr;
    TPB_CHECK(B.get(&d_nl, cnt));
    size_t tb = 0;
    TPB_CUDA(cub::DeviceSelect::If(nullptr, tb, idx, d_nl, d_nnl, (int)nbytes, IsNewline{d_bytes}, h->stream));
    void *tmp = nullptr;
    TPB_CHECK(B.get((uint8_t **)&tmp, tb));
    TPB_CUDA(cub::DeviceSelect::If(tmp, tb, idx, d_nl, d_nnl, (int)nbytes, IsNewline{d_bytes}, h->stream));
    const int nnl = (int)cnt;
    const size_t nlines = (size_t)nnl + ((nbytes && last != '\n') ? 1 : 0);
    uint64_t *d_line = nullptr;
    uint8_t *d_keep = nullptr;
    unsigned long long *d_err = nullptr;
    int *d_nval = nullptr;
    TPB_CHECK(B.get(&d_line, nlines));
    TPB_CHECK(B.get(&d_keep, nlines));
    TPB_CHECK(B.get(&d_err, 1));
    TPB_CHECK(B.get(&d_nval, 1));
    TPB_CHECK(B.get(&d_vals, nlines));
    TPB_CUDA(cudaMemsetAsync(d_err, 0xff, sizeof(unsigned long long), h->stream));
    if (nlines) {
      parse_lines_kernel<<<grid_for(nlines * 32, kStrThreads), kStrThreads, 0, h->stream>>>(
          d_bytes, nbytes, d_nl, (size_t)nnl, nlines, norb, d_line, d_keep, d_err);
      TPB_LAUNCHED(h);
    }
    unsigned long long he = 0;
    TPB_CUDA(cudaMemcpyAsync(&he, d_err, sizeof(he), cudaMemcpyDeviceToHost, h->stream));
    size_t tf = 0;
    TPB_CUDA(cub::DeviceSelect::Flagged(nullptr, tf, d_line, d_keep, d_vals, d_nval, (int)nlines, h->stream));
    void *tmp2 = nullptr;
    TPB_CHECK(B.get((uint8_t **)&tmp2, tf));
    TPB_CUDA(cub::DeviceSelect::Flagged(tmp2, tf, d_line, d_keep, d_vals, d_nval, (int)nlines, h->stream));
    int nval = 0;
    TPB_CUDA(cudaMemcpyAsync(&nval, d_nval, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    TPB_CUDA(cudaStreamSynchronize(h->stream));
    if (he != ~0ull)
      return fail(SBD_TPB_ERR_IO, std::string("strings: line ") + std::to_string(he >> 2) +
                                      ((he & 3) == 1 ? " is shorter than norb" : " has characters other than 0/1"));
    nstr = (size_t)nval;
  }
  // ascending and unique (sort_bitarray)
  int *d_nu = nullptr;
  TPB_CHECK(B.get(&d_keys, nstr));
  uint64_t *d_uniq = nullptr;
  TPB_CHECK(B.get(&d_uniq, nstr));
  TPB_CHECK(B.get(&d_nu, 1));
  size_t t1 = 0, t2 = 0;
  TPB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, t1, d_vals, d_keys, (int)nstr, 0, norb, h->stream));
  TPB_CUDA(cub::DeviceSelect::Unique(nullptr, t2, d_keys, d_uniq, d_nu, (int)nstr, h->stream));
  void *tmp3 = nullptr;
  TPB_CHECK(B.get((uint8_t **)&tmp3, std::max(t1, t2)));
  int nu = 0;
  if (nstr) {
    TPB_CUDA(cub::DeviceRadixSort::SortKeys(tmp3, t1, d_vals, d_keys, (int)nstr, 0, norb, h->stream));
    TPB_CUDA(cub::DeviceSelect::Unique(tmp3, t2, d_keys, d_uniq, d_nu, (int)nstr, h->stream));
    TPB_CUDA(cudaMemcpyAsync(&nu, d_nu, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  }
  TPB_CUDA(cudaEventRecord(h->ev_co[1], h->stream));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  if (ms) TPB_CUDA(cudaEventElapsedTime(ms, h->ev_co[0], h->ev_co[1]));
  *count = (size_t)nu;
  if (!out || cap < (size_t)nu)
    return fail(SBD_TPB_ERR_CAPACITY, "strings: output buffer missing or too small (count returned)");
  if (nu) TPB_CUDA(cudaMemcpy(out, d_uniq, sizeof(uint64_t) * nu, cudaMemcpyDeviceToHost));
  return SBD_TPB_OK;
}

}  // namespace sbdtpb
