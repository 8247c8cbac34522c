// cb2_static_scratch.cu -- cb2_energies_static: the volume energy diagnostics
// with no device memory allocation.
//
// Who needs it: a host that must not touch the CUDA allocator once its run is
// set up -- for example a Fortran driver whose device memory is budgeted and
// owned by another component of the same process, or a monitoring loop that
// reads energies every few steps and must not add allocation latency or
// fragmentation to a long run.  cb2_energies keeps its partial sums in a
// buffer owned by the context; this entry point keeps them in the file-scope
// array below instead, so calling it never allocates.
//
// Limits and sharing:
//   * the array holds kScratchDoubles doubles (3.5 MiB): 7 * jmax + 7 must
//     fit, i.e. jmax = (L+1)^2 <= 65536, truncation L <= 255.  Larger
//     contexts get CB2_ERR_ARG and a message; nothing is launched.
//   * there is one array per device, shared by every context and every call
//     on that device.  It keeps whatever the last call left in it; nothing in
//     it needs to start at zero, because each call writes every element it
//     later reads.  Two calls whose work overlaps on the same device (two
//     host threads, or two contexts on different streams) race on the array
//     and may return each other's sums: serialise them.
//   * cb2_create looks up the array's device address on its device with
//     cudaGetSymbolAddress (with that device current) and caches it, so the
//     module that holds the array is loaded -- and its memory reserved --
//     while the context is set up (with lazy module loading, the CUDA
//     default, that would otherwise happen at the first call).  No call of
//     cb2_energies_static itself allocates.
#include <mutex>

#include "cb2_internal.cuh"

namespace cb2 {
namespace {

constexpr size_t kScratchDoubles = 7 * 65536 + 7;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_energy_scratch[kScratchDoubles];

std::mutex g_mu;
double *g_ptr[kMaxDevices] = {nullptr};

// device address of g_energy_scratch on `device` (looked up once per device)
int scratch_on(int device, double **out) {
  if (device < 0 || device >= kMaxDevices) {
    set_error("cb2_energies_static: device ordinal out of range");
    return CB2_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_ptr[device]) {
    int prev = -1;
    CB2_CUDA(cudaGetDevice(&prev));
    if (prev != device) CB2_CUDA(cudaSetDevice(device));
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_energy_scratch);
    if (prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_energy_scratch)");
    g_ptr[device] = static_cast<double *>(p);
  }
  *out = g_ptr[device];
  return 0;
}

}  // namespace

int static_scratch_setup(int device) {
  double *p = nullptr;
  return scratch_on(device, &p);
}

}  // namespace cb2

using namespace cb2;

extern "C" int cb2_energies_static(cb2_ctx *c, double out[7]) {
  if (!c || !out) {
    set_error("cb2_energies_static: null argument");
    return CB2_ERR_ARG;
  }
  if (7 * (size_t)c->jmax + 7 > kScratchDoubles) {
    set_error("cb2_energies_static: jmax = " + std::to_string(c->jmax) +
              " needs more than the static scratch holds (7 * 65536 + 7 doubles, L <= 255); "
              "use cb2_energies");
    return CB2_ERR_ARG;
  }
  double *scratch = nullptr;
  int rc = scratch_on(c->device, &scratch);
  if (rc) return rc;
  int prev = -1;
  CB2_CUDA(cudaGetDevice(&prev));
  if (prev != c->device) CB2_CUDA(cudaSetDevice(c->device));
  rc = check_status(*c);
  if (!rc) rc = rj_energies_scratch(*c, scratch, out);
  if (prev != c->device) cudaSetDevice(prev);
  return rc;
}
