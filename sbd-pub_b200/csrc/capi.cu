// C ABI of libsbdtpb (declared in include/sbd_tpb.h).
//
// Every entry point validates its arguments, runs on the handle's stream, converts CUDA errors
// into status codes and records a message for sbd_tpb_last_error(); nothing throws across the
// ABI and nothing exits the process (the reference throws, exit()s or MPI_Abort()s instead:
// tpb/helper.h:342-345, framework/fcidump.h:34-35, framework/cuda_utility.h:21-28).
#include <algorithm>
#include <cstdio>
#include <chrono>
#include <cstring>
#include <new>
#include <string>

#include "tpb_common.cuh"
#include "vecops.cuh"

namespace sbdtpb {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

}  // namespace sbdtpb

using namespace sbdtpb;

namespace {

int use_device(sbd_tpb_handle *h) {
  TPB_CUDA(cudaSetDevice(h->device));
  return SBD_TPB_OK;
}

#define TPB_HANDLE(h)                                                     \
  do {                                                                    \
    if (!(h)) return fail(SBD_TPB_ERR_INVALID, "null handle");            \
    TPB_CHECK(use_device(h));                                             \
  } while (0)

int ensure_tmp64(sbd_tpb_handle *h) {
  const size_t n = h->ndet();
  if (!h->d_tmp64) TPB_CUDA(cudaMalloc(&h->d_tmp64, sizeof(double) * n));
  if (!h->d_tmp64b) TPB_CUDA(cudaMalloc(&h->d_tmp64b, sizeof(double) * n));
  return SBD_TPB_OK;
}

int ensure_tmp32(sbd_tpb_handle *h) {
  const size_t n = h->ndet();
  if (!h->d_tmp32) TPB_CUDA(cudaMalloc(&h->d_tmp32, sizeof(float) * n));
  if (!h->d_tmp32b) TPB_CUDA(cudaMalloc(&h->d_tmp32b, sizeof(float) * n));
  return SBD_TPB_OK;
}

void free_tmps(sbd_tpb_handle *h) {
  for (double **p : {&h->d_tmp64, &h->d_tmp64b})
    if (*p) {
      cudaFree(*p);
      *p = nullptr;
    }
  for (float **p : {&h->d_tmp32, &h->d_tmp32b})
    if (*p) {
      cudaFree(*p);
      *p = nullptr;
    }
}

}  // namespace

extern "C" {

void sbd_tpb_default_params(sbd_tpb_params *p) {
  if (!p) return;
  p->max_it = 1;
  p->max_nb = 10;
  p->eps = 1.0e-4;
  p->max_time = 86400.0;
  p->init = 0;
  p->do_rdm = 0;
  p->precision = SBD_TPB_FP64;
  p->preconditioner = SBD_TPB_PRECOND_DIAGONAL;
  p->verbose = 0;
  p->device = 0;
  p->symmetry = 1;
  p->method = SBD_TPB_METHOD_DAVIDSON;
  p->seed = 1729;
}

const char *sbd_tpb_last_error(void) { return g_last_error.c_str(); }

int sbd_tpb_create(int device, sbd_tpb_handle **out) {
  if (!out) return fail(SBD_TPB_ERR_INVALID, "null output pointer");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(SBD_TPB_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(SBD_TPB_ERR_INVALID, "device ordinal out of range");
  cudaDeviceProp prop;
  TPB_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(SBD_TPB_ERR_NO_DEVICE, std::string("device is not sm_100 class: ") + prop.name);
  TPB_CUDA(cudaSetDevice(device));
  sbd_tpb_handle *h = new (std::nothrow) sbd_tpb_handle();
  if (!h) return fail(SBD_TPB_ERR_OOM, "host allocation failed");
  h->device = device;
  h->num_sms = prop.multiProcessorCount;
  h->smem_optin = prop.sharedMemPerBlockOptin;
  bool ev_ok = cudaEventCreate(&h->ev0) == cudaSuccess && cudaEventCreate(&h->ev1) == cudaSuccess;
  for (cudaEvent_t &e : h->ev_k) ev_ok = ev_ok && cudaEventCreate(&e) == cudaSuccess;
  for (cudaEvent_t &e : h->ev_co) ev_ok = ev_ok && cudaEventCreate(&e) == cudaSuccess;
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess || !ev_ok) {
    delete h;
    return fail(SBD_TPB_ERR_CUDA, "stream/event creation failed");
  }
  *out = h;
  return SBD_TPB_OK;
}

int sbd_tpb_destroy(sbd_tpb_handle *h) {
  if (!h) return SBD_TPB_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_device_problem(h);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  for (cudaEvent_t e : h->ev_k)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : h->ev_co)
    if (e) cudaEventDestroy(e);
  if (h->h_stage) cudaFreeHost(h->h_stage);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return SBD_TPB_OK;
}

int sbd_tpb_set_hamiltonian(sbd_tpb_handle *h, const sbd_tpb_hamiltonian *ham) {
  TPB_HANDLE(h);
  if (!ham || !ham->h1 || !ham->eri_packed) return fail(SBD_TPB_ERR_INVALID, "null Hamiltonian");
  const int L = ham->norb;
  if (L < 1 || L > 64) return fail(SBD_TPB_ERR_INVALID, "norb must be in [1, 64]");
  const size_t B = (size_t)L * (L + 1) / 2;
  if (ham->n_eri_packed != B * (B + 1) / 2)
    return fail(SBD_TPB_ERR_INVALID, "eri_packed length must be B(B+1)/2 with B = L(L+1)/2");
  if (h->have_strings && h->L != L) {
    free_device_problem(h);
    h->have_strings = false;
  }
  h->L = L;
  h->nelec = ham->nelec;
  h->I0 = ham->core_energy;
  h->h1.assign(ham->h1, ham->h1 + (size_t)L * L);
  // symmetrise exactly as SetupIntegrals writes both orders of each one-electron entry
  for (int i = 0; i < L; i++)
    for (int j = 0; j < i; j++) h->h1[(size_t)j * L + i] = h->h1[(size_t)i * L + j];
  h->eri_packed.assign(ham->eri_packed, ham->eri_packed + ham->n_eri_packed);
  TPB_CHECK(upload_hamiltonian(h));
  h->have_ham = true;
  h->have_tables = false;
  return SBD_TPB_OK;
}

int sbd_tpb_set_strings(sbd_tpb_handle *h, const uint64_t *astr, size_t na, const uint64_t *bstr,
                        size_t nb) {
  TPB_HANDLE(h);
  if (!h->have_ham) return fail(SBD_TPB_ERR_STATE, "set the Hamiltonian before the strings");
  if (!astr || !bstr || na == 0 || nb == 0) return fail(SBD_TPB_ERR_INVALID, "empty string set");
  if (na > 0xffffffffull || nb > 0xffffffffull || (double)na * (double)nb > 4.0e12)
    return fail(SBD_TPB_ERR_INVALID, "string sets too large");
  const uint64_t mask = h->L >= 64 ? ~0ull : ((1ull << h->L) - 1ull);
  auto check = [&](const uint64_t *s, size_t n, const char *what, int *nel) -> int {
    for (size_t i = 0; i < n; i++) {
      if (s[i] & ~mask) return fail(SBD_TPB_ERR_INVALID, std::string(what) + " string wider than norb");
      const int c = __builtin_popcountll(s[i]);
      if (i == 0) *nel = c;
      else if (c != *nel)
        return fail(SBD_TPB_ERR_INVALID, std::string(what) + " strings differ in electron count");
    }
    return SBD_TPB_OK;
  };
  int nea = 0, neb = 0;
  TPB_CHECK(check(astr, na, "alpha", &nea));
  TPB_CHECK(check(bstr, nb, "beta", &neb));
  // the order is the caller's (sorted, or shuffled as --shuffle does); entries must be unique
  for (int spin = 0; spin < 2; spin++) {
    std::vector<uint64_t> v(spin ? bstr : astr, spin ? bstr + nb : astr + na);
    std::sort(v.begin(), v.end());
    if (std::adjacent_find(v.begin(), v.end()) != v.end())
      return fail(SBD_TPB_ERR_INVALID, spin ? "duplicate beta strings" : "duplicate alpha strings");
  }
  // drop everything that depends on the previous strings
  {
    std::vector<double> h1 = h->h1, eri = h->eri_packed;
    free_device_problem(h);
    free_tmps(h);
    h->h1 = h1;
    h->eri_packed = eri;
    TPB_CHECK(upload_hamiltonian(h));
  }
  h->astr.assign(astr, astr + na);
  h->bstr.assign(bstr, bstr + nb);
  h->n_alpha = nea;
  h->n_beta = neb;
  TPB_CHECK(build_string_data(h));
  h->have_strings = true;
  h->have_tables = false;
  return SBD_TPB_OK;
}

int sbd_tpb_build_tables(sbd_tpb_handle *h) {
  TPB_HANDLE(h);
  if (!h->have_strings) return fail(SBD_TPB_ERR_STATE, "set strings before building tables");
  TPB_CHECK(build_excitation_tables(h));
  TPB_CHECK(prepare_block_sizes(h));
  TPB_CHECK(build_sigma_programs(h));
  TPB_CHECK(compute_diagonal(h));
  TPB_CHECK(ab_dense_setup(h, ab_dense_worthwhile(h) ? 1 : 0));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  h->have_tables = true;
  return SBD_TPB_OK;
}

int sbd_tpb_table_size(sbd_tpb_handle *h, int kind, size_t *nrows, size_t *nnz) {
  TPB_HANDLE(h);
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  const ExTable *t = nullptr;
  size_t n = 0;
  switch (kind) {
    case SBD_TPB_SINGLES_ALPHA: t = &h->ta_s; n = h->astr.size(); break;
    case SBD_TPB_DOUBLES_ALPHA: t = &h->ta_d; n = h->astr.size(); break;
    case SBD_TPB_SINGLES_BETA: t = &h->tb_s; n = h->bstr.size(); break;
    case SBD_TPB_DOUBLES_BETA: t = &h->tb_d; n = h->bstr.size(); break;
    default: return fail(SBD_TPB_ERR_INVALID, "unknown table kind");
  }
  if (nrows) *nrows = n;
  if (nnz) *nnz = t->nnz;
  return SBD_TPB_OK;
}

int sbd_tpb_get_table(sbd_tpb_handle *h, int kind, uint64_t *off, uint64_t *ket, int32_t *cran) {
  TPB_HANDLE(h);
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  return copy_table_reference_layout(h, kind, off, ket, cran);
}

int sbd_tpb_diagonal(sbd_tpb_handle *h, double *hii, int mem) {
  TPB_HANDLE(h);
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  if (!hii) return fail(SBD_TPB_ERR_INVALID, "null output");
  TPB_CUDA(cudaMemcpyAsync(hii, h->d_hii, sizeof(double) * h->ndet(),
                           mem == SBD_TPB_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           h->stream));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  return SBD_TPB_OK;
}

int sbd_tpb_sigma(sbd_tpb_handle *h, const double *C, double *sigma, int accumulate, int mem) {
  TPB_HANDLE(h);
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  if (!C || !sigma) return fail(SBD_TPB_ERR_INVALID, "null vector");
  const size_t n = h->ndet();
  TPB_CHECK(ensure_tmp64(h));
  // reference convention in, separated convention inside: x = D C
  if (mem == SBD_TPB_DEVICE) {
    TPB_CHECK(reorder_sign_apply_f64(h, C, h->d_tmp64));
  } else {
    TPB_CUDA(cudaMemcpyAsync(h->d_tmp64b, C, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    TPB_CHECK(reorder_sign_apply_f64(h, h->d_tmp64b, h->d_tmp64));
  }
  TPB_CHECK(sigma_sep<double>(h, h->d_tmp64, h->d_tmp64b, 0));
  TPB_CUDA(cudaEventSynchronize(h->ev1));
  TPB_CUDA(cudaEventElapsedTime(&h->last_sigma_ms, h->ev0, h->ev1));
  TPB_CHECK(reorder_sign_apply_f64(h, h->d_tmp64b, h->d_tmp64));
  if (mem == SBD_TPB_DEVICE) {
    if (accumulate) TPB_CHECK(axpby<double>(h, h->d_tmp64, sigma, 1.0, 1.0, n));
    else TPB_CUDA(cudaMemcpyAsync(sigma, h->d_tmp64, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
  } else {
    if (accumulate) {
      TPB_CUDA(cudaMemcpyAsync(h->d_tmp64b, sigma, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
      TPB_CHECK(axpby<double>(h, h->d_tmp64, h->d_tmp64b, 1.0, 1.0, n));
      TPB_CUDA(cudaMemcpyAsync(sigma, h->d_tmp64b, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    } else {
      TPB_CUDA(cudaMemcpyAsync(sigma, h->d_tmp64, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    }
  }
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  return SBD_TPB_OK;
}

int sbd_tpb_sigma_f32(sbd_tpb_handle *h, const float *C, float *sigma, int accumulate, int mem) {
  TPB_HANDLE(h);
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  if (!C || !sigma) return fail(SBD_TPB_ERR_INVALID, "null vector");
  const size_t n = h->ndet();
  TPB_CHECK(ensure_tmp32(h));
  if (mem == SBD_TPB_DEVICE) {
    TPB_CHECK(reorder_sign_apply_f32(h, C, h->d_tmp32));
  } else {
    TPB_CUDA(cudaMemcpyAsync(h->d_tmp32b, C, sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
    TPB_CHECK(reorder_sign_apply_f32(h, h->d_tmp32b, h->d_tmp32));
  }
  TPB_CHECK(sigma_sep<float>(h, h->d_tmp32, h->d_tmp32b, 0));
  TPB_CUDA(cudaEventSynchronize(h->ev1));
  TPB_CUDA(cudaEventElapsedTime(&h->last_sigma_ms, h->ev0, h->ev1));
  TPB_CHECK(reorder_sign_apply_f32(h, h->d_tmp32b, h->d_tmp32));
  if (mem == SBD_TPB_DEVICE) {
    if (accumulate) TPB_CHECK(axpby<float>(h, h->d_tmp32, sigma, 1.0, 1.0, n));
    else TPB_CUDA(cudaMemcpyAsync(sigma, h->d_tmp32, sizeof(float) * n, cudaMemcpyDeviceToDevice, h->stream));
  } else {
    if (accumulate) {
      TPB_CUDA(cudaMemcpyAsync(h->d_tmp32b, sigma, sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
      TPB_CHECK(axpby<float>(h, h->d_tmp32, h->d_tmp32b, 1.0, 1.0, n));
      TPB_CUDA(cudaMemcpyAsync(sigma, h->d_tmp32b, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
    } else {
      TPB_CUDA(cudaMemcpyAsync(sigma, h->d_tmp32, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
    }
  }
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  return SBD_TPB_OK;
}

int sbd_tpb_sigma_device(sbd_tpb_handle *h, const void *C, void *sigma, int dtype, int accumulate,
                         int convention) {
  TPB_HANDLE(h);
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  if (!C || !sigma) return fail(SBD_TPB_ERR_INVALID, "null vector");
  if (dtype != 0 && dtype != 1) return fail(SBD_TPB_ERR_INVALID, "dtype must be 0 (double) or 1 (float)");
  if (convention == 0) {
    return dtype == 0 ? sbd_tpb_sigma(h, (const double *)C, (double *)sigma, accumulate, SBD_TPB_DEVICE)
                      : sbd_tpb_sigma_f32(h, (const float *)C, (float *)sigma, accumulate, SBD_TPB_DEVICE);
  }
  if (convention != 1 && convention != 2) return fail(SBD_TPB_ERR_INVALID, "convention must be 0, 1 or 2");
  // the passes read C while they write sigma
  if (C == sigma) return fail(SBD_TPB_ERR_INVALID, "sigma_device: C and sigma must be distinct buffers");
  if (convention == 2) {
    if (accumulate) return fail(SBD_TPB_ERR_INVALID, "sigma_device: convention 2 does not accumulate");
    if (dtype == 0) TPB_CHECK(sigma_sep_sym<double>(h, (const double *)C, (double *)sigma, 0.0));
    else TPB_CHECK(sigma_sep_sym<float>(h, (const float *)C, (float *)sigma, 0.0));
  } else if (dtype == 0) {
    TPB_CHECK(sigma_sep<double>(h, (const double *)C, (double *)sigma, accumulate));
  } else {
    TPB_CHECK(sigma_sep<float>(h, (const float *)C, (float *)sigma, accumulate));
  }
  TPB_CUDA(cudaEventSynchronize(h->ev1));
  TPB_CUDA(cudaEventElapsedTime(&h->last_sigma_ms, h->ev0, h->ev1));
  return SBD_TPB_OK;
}

int sbd_tpb_davidson(sbd_tpb_handle *h, const sbd_tpb_params *params, const double *W0,
                     sbd_tpb_result *result) {
  TPB_HANDLE(h);
  if (!params || !result) return fail(SBD_TPB_ERR_INVALID, "null params/result");
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  if (params->init != 0 && params->init != 1) return fail(SBD_TPB_ERR_INVALID, "init must be 0 or 1");
  return davidson_run(h, params, W0, result);
}

int sbd_tpb_lanczos(sbd_tpb_handle *h, const sbd_tpb_params *params, const double *W0,
                    sbd_tpb_result *result) {
  TPB_HANDLE(h);
  if (!params || !result) return fail(SBD_TPB_ERR_INVALID, "null params/result");
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  if (params->init != 0 && params->init != 1) return fail(SBD_TPB_ERR_INVALID, "init must be 0 or 1");
  return lanczos_run(h, params, W0, result);
}

int sbd_tpb_rdm(sbd_tpb_handle *h, const double *W, double *one, double *two, int mem) {
  TPB_HANDLE(h);
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  if (!W || !one) return fail(SBD_TPB_ERR_INVALID, "null vector/output");
  const size_t n = h->ndet();
  TPB_CHECK(ensure_tmp64(h));
  if (mem == SBD_TPB_DEVICE) {
    TPB_CHECK(reorder_sign_apply_f64(h, W, h->d_tmp64));
  } else {
    TPB_CUDA(cudaMemcpyAsync(h->d_tmp64b, W, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    TPB_CHECK(reorder_sign_apply_f64(h, h->d_tmp64b, h->d_tmp64));
  }
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  return rdm_sep(h, h->d_tmp64, one, two, nullptr);
}

int sbd_tpb_parse_strings(sbd_tpb_handle *h, const void *bytes, size_t nbytes, int format, int norb, uint64_t *out,
                          size_t cap, size_t *count) {
  TPB_HANDLE(h);
  if (!count) return fail(SBD_TPB_ERR_INVALID, "null count");
  return parse_strings_device(h, bytes, nbytes, format, norb, out, cap, count, &h->last_parse_ms);
}

int sbd_tpb_read_strings(sbd_tpb_handle *h, const char *path, int norb, uint64_t *out, size_t cap, size_t *count) {
  TPB_HANDLE(h);
  if (!path || !count) return fail(SBD_TPB_ERR_INVALID, "null path/count");
  std::FILE *f = std::fopen(path, "rb");
  if (!f) return fail(SBD_TPB_ERR_IO, std::string("cannot open ") + path);
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz < 0) {
    std::fclose(f);
    return fail(SBD_TPB_ERR_IO, std::string("cannot size ") + path);
  }
  // pinned staging (kept on the handle) so the copy to HBM runs at link speed
  if (h->stage_cap < (size_t)sz + 1) {
    if (h->h_stage) cudaFreeHost(h->h_stage);
    h->h_stage = nullptr;
    h->stage_cap = 0;
    if (cudaMallocHost(&h->h_stage, (size_t)sz + 1) != cudaSuccess) {
      cudaGetLastError();
      h->h_stage = nullptr;
      std::fclose(f);
      return fail(SBD_TPB_ERR_OOM, "pinned staging for the string file");
    }
    h->stage_cap = (size_t)sz + 1;
  }
  void *buf = h->h_stage;
  const size_t got = sz ? std::fread(buf, 1, (size_t)sz, f) : 0;
  std::fclose(f);
  if (got != (size_t)sz) return fail(SBD_TPB_ERR_IO, std::string("short read of ") + path);
  const std::string p(path);
  const int format = (p.size() >= 4 && p.compare(p.size() - 4, 4, ".bin") == 0) ? SBD_TPB_STRINGS_BINARY
                                                                                   : SBD_TPB_STRINGS_TEXT;
  return parse_strings_device(h, buf, got, format, norb, out, cap, count, &h->last_parse_ms);
}

double sbd_tpb_last_parse_ms(sbd_tpb_handle *h) { return h ? (double)h->last_parse_ms : 0.0; }

int sbd_tpb_carryover_strings(sbd_tpb_handle *h, const double *W, int mem, sbd_tpb_carryover *co) {
  TPB_HANDLE(h);
  if (!h->have_strings) return fail(SBD_TPB_ERR_STATE, "strings not set");
  if (!W || !co) return fail(SBD_TPB_ERR_INVALID, "null vector/carry-over record");
  if (mem == SBD_TPB_DEVICE) return carryover_device(h, W, co);
  TPB_CHECK(ensure_tmp64(h));
  TPB_CUDA(cudaMemcpyAsync(h->d_tmp64, W, sizeof(double) * h->ndet(), cudaMemcpyHostToDevice, h->stream));
  return carryover_device(h, h->d_tmp64, co);
}

int sbd_tpb_last_carryover_ms(sbd_tpb_handle *h, double *ms) {
  if (!h || !ms) return fail(SBD_TPB_ERR_INVALID, "null handle/output");
  ms[0] = h->last_carryover_ms[0];
  ms[1] = h->last_carryover_ms[1];
  return SBD_TPB_OK;
}

size_t sbd_tpb_carryover_capacity(sbd_tpb_handle *h, int type, int spin) {
  if (!h || !h->have_strings) return 0;
  const size_t n = spin ? h->bstr.size() : h->astr.size();
  if (type == SBD_TPB_CARRYOVER_DOMINANT) return n;
  if (type != SBD_TPB_CARRYOVER_DOMINANT_SINGLES && type != SBD_TPB_CARRYOVER_CUTOFF_SINGLES) return 0;
  // every string and its e(L - e) singles, at most C(L, e) distinct strings
  const int L = h->L, e = spin ? h->n_beta : h->n_alpha;
  double binom = 1.0;
  for (int k = 1; k <= e; k++) binom = binom * (L - e + k) / k;
  const double bound = std::min((double)n * (1.0 + (double)e * (L - e)), std::floor(binom + 0.5));
  return (size_t)bound;
}

int sbd_tpb_diag(const sbd_tpb_params *params, const sbd_tpb_hamiltonian *ham,
                 const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                 sbd_tpb_result *result) {
  return sbd_tpb_diag_from(params, ham, astr, na, bstr, nb, nullptr, result);
}

int sbd_tpb_diag_from(const sbd_tpb_params *params, const sbd_tpb_hamiltonian *ham,
                      const uint64_t *astr, size_t na, const uint64_t *bstr, size_t nb,
                      const double *W0, sbd_tpb_result *result) {
  if (!params || !result) return fail(SBD_TPB_ERR_INVALID, "null params/result");
  const auto t0 = std::chrono::steady_clock::now();
  sbd_tpb_handle *h = nullptr;
  TPB_CHECK(sbd_tpb_create(params->device, &h));
  int rc = sbd_tpb_set_hamiltonian(h, ham);
  if (rc == SBD_TPB_OK) rc = sbd_tpb_set_strings(h, astr, na, bstr, nb);
  const auto t1 = std::chrono::steady_clock::now();
  if (rc == SBD_TPB_OK) rc = sbd_tpb_build_tables(h);
  const auto t2 = std::chrono::steady_clock::now();
  result->seconds_tables = std::chrono::duration<double>(t2 - t1).count();
  if (rc == SBD_TPB_OK) {
    // --rdm 0: occupations only (tpb/sbdiag.h:609-640); --rdm 1: full 1/2-RDMs (:643-667)
    double *one = result->one_rdm, *two = result->two_rdm;
    if (!params->do_rdm) {
      result->one_rdm = nullptr;
      result->two_rdm = nullptr;
    }
    if (params->method == SBD_TPB_METHOD_LANCZOS) rc = sbd_tpb_lanczos(h, params, W0, result);
    else if (params->method == SBD_TPB_METHOD_DAVIDSON) rc = sbd_tpb_davidson(h, params, W0, result);
    else rc = fail(SBD_TPB_ERR_INVALID, "method must be 0 (Davidson) or 2 (Lanczos)");
    result->one_rdm = one;
    result->two_rdm = two;
  }
  std::string msg = rc == SBD_TPB_OK ? std::string() : std::string(sbd_tpb_last_error());
  sbd_tpb_destroy(h);
  if (rc != SBD_TPB_OK) set_error(msg);
  result->seconds_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return rc;
}

void *sbd_tpb_stream(sbd_tpb_handle *h) { return h ? (void *)h->stream : nullptr; }

double sbd_tpb_last_sigma_ms(sbd_tpb_handle *h) { return h ? (double)h->last_sigma_ms : 0.0; }

int sbd_tpb_last_sigma_kernels(sbd_tpb_handle *h, double *ms, int max_n) {
  if (!h || !ms) return fail(SBD_TPB_ERR_INVALID, "null handle/output");
  TPB_CHECK(use_device(h));
  const int n = std::min(h->sigma_kernels, max_n);
  cudaEvent_t prev = h->ev0;
  for (int k = 0; k < n; k++) {
    float t = 0.f;
    TPB_CUDA(cudaEventSynchronize(h->ev_k[k]));
    TPB_CUDA(cudaEventElapsedTime(&t, prev, h->ev_k[k]));
    ms[k] = t;
    prev = h->ev_k[k];
  }
  return n;
}

uint64_t sbd_tpb_kernel_launches(sbd_tpb_handle *h) { return h ? h->launches : 0; }

int sbd_tpb_release_work(sbd_tpb_handle *h) {
  TPB_HANDLE(h);
  TPB_CUDA(cudaSetDevice(h->device));
  TPB_CUDA(cudaStreamSynchronize(h->stream));
  pool_clear(h);
  free_tmps(h);
  if (h->d_ct) cudaFree(h->d_ct);
  h->d_ct = nullptr;
  h->ct_bytes = 0;
  return SBD_TPB_OK;
}

}  // extern "C"
