// sbd_tpb_sigma_noalloc: sigma on device vectors without any device allocation.
//
// Some callers cannot let a library call cudaMalloc while they run: a code that has reserved
// nearly all of HBM up front through its own pool (a framework caching allocator, a solver that
// sized its Krylov space to the card), where one more cudaMalloc fails or forces the pool to
// flush, and a host code whose memory policy forbids allocations after its set-up phase.  The
// regular sigma entry points allocate their C^T staging buffer (and the dense alpha-beta work
// arrays) lazily on first use; this variant uses instead a fixed scratch array that lives in the
// library's own device image, and evaluates the alpha-single x beta-single terms with the direct
// loop, which needs no work arrays.  Everything else it reads (tables, sigma programs, the
// diagonal, the per-block table sizes) is built by sbd_tpb_build_tables.
//
// Limits and sharing rules:
//   * the scratch holds C^T: ndet * sizeof(element) must not exceed
//     SBD_TPB_NOALLOC_SCRATCH_BYTES (16 MiB: 2,097,152 FP64 or 4,194,304 FP32 determinants);
//     larger problems are rejected with SBD_TPB_ERR_INVALID;
//   * every GPU that loads the library holds the 16 MiB until the process exits;
//   * all calls on a device share the one array, which keeps the last call's contents.  Nothing
//     in it has to start at zero (the alpha pass writes every element of C^T before the beta pass
//     reads it), but two calls whose kernels overlap on the GPU race on it: serialise them (one
//     stream, or events between streams);
//   * the first call on each device looks up the array's device address with
//     cudaGetSymbolAddress (which may load the library's device code) and keeps it for the rest
//     of the process, so make that first call before any stream capture; a cudaDeviceReset
//     invalidates the kept address, so do not call this entry point on a device after resetting it.
#include <mutex>
#include <string>

#include "tpb_common.cuh"

namespace {

constexpr size_t kScratchBytes = SBD_TPB_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_sigma_scratch[kScratchBytes];

std::mutex g_scratch_mutex;
void *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array on `device` (current), looked up once per device.
int scratch_for_device(int device, void **out) {
  if (device < 0 || device >= kMaxDevices)
    return sbdtpb::fail(SBD_TPB_ERR_INVALID, "sbd_tpb_sigma_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sigma_scratch);
    if (e != cudaSuccess || !p)
      return sbdtpb::fail(SBD_TPB_ERR_CUDA, std::string("sbd_tpb_sigma_noalloc: cudaGetSymbolAddress: ") +
                                                cudaGetErrorString(e));
    g_scratch_ptr[device] = p;
  }
  *out = g_scratch_ptr[device];
  return SBD_TPB_OK;
}

}  // namespace

extern "C" int sbd_tpb_sigma_noalloc(sbd_tpb_handle *h, const void *C, void *sigma, int dtype,
                                     int accumulate) {
  using namespace sbdtpb;
  if (!h) return fail(SBD_TPB_ERR_INVALID, "null handle");
  if (!h->have_tables) return fail(SBD_TPB_ERR_STATE, "tables not built");
  if (!C || !sigma) return fail(SBD_TPB_ERR_INVALID, "null vector");
  if (C == sigma)
    return fail(SBD_TPB_ERR_INVALID, "sbd_tpb_sigma_noalloc: C and sigma must be distinct buffers");
  if (dtype != 0 && dtype != 1) return fail(SBD_TPB_ERR_INVALID, "dtype must be 0 (double) or 1 (float)");
  // the per-block table sizes are read back at table build; without them the launch would need a
  // synchronous copy here
  if (h->blk_for != (const void *)h->ta_d.ket)
    return fail(SBD_TPB_ERR_STATE, "sbd_tpb_sigma_noalloc: table block sizes missing; rebuild the tables");
  const size_t esz = dtype == 0 ? sizeof(double) : sizeof(float);
  const size_t need = h->ndet() * esz;
  if (need > kScratchBytes)
    return fail(SBD_TPB_ERR_INVALID,
                "sbd_tpb_sigma_noalloc: " + std::to_string(h->ndet()) + " determinants x " +
                    std::to_string(esz) + " bytes exceed its fixed " +
                    std::to_string(kScratchBytes >> 20) +
                    " MiB scratch; use sbd_tpb_sigma_device for larger problems");
  TPB_CUDA(cudaSetDevice(h->device));
  void *scratch = nullptr;
  TPB_CHECK(scratch_for_device(h->device, &scratch));
  if (dtype == 0)
    TPB_CHECK(sigma_sep_given_ct<double>(h, (const double *)C, (double *)sigma, accumulate,
                                         (double *)scratch));
  else
    TPB_CHECK(sigma_sep_given_ct<float>(h, (const float *)C, (float *)sigma, accumulate,
                                        (float *)scratch));
  return SBD_TPB_OK;
}
