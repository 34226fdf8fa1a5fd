// C ABI: pseudopotential adjoint that allocates nothing.
//
// dh_hamiltonian_pseudopotential_adjoint needs a [blocks][factors] FP64 scratch array for the
// per-block bins of its kernel and allocates it (and staging buffers for host vectors) on first
// use.  Some callers cannot allocate device memory at all: an application whose framework owns
// every byte of device memory through its own allocator or a fixed arena, where a library's
// cudaMalloc would fail or break that framework's accounting.  This entry point runs the same
// kernels with their scratch in a file-scope static device array instead, and stages nothing: u
// and v must already be on the device.  The array is sized for lz_max <= 33 (2S <= 33, at most
// DH_STATIC_ADJOINT_MAX_FACTORS interaction factors) and DH_STATIC_ADJOINT_BLOCKS blocks; it costs
// about 7.6 MB on every GPU that loads the library, held until the process exits.
//
// The call is synchronous: it waits on the handle's stream for the summed bins, copies them into a
// static host array and contracts them with dfactor/dV_m on the host.  A process-wide mutex
// serialises the calls (on every GPU), so two calls never use the array at the same time.
#include <cuda_runtime.h>
#include <mutex>

#include "dh_internal.h"
#include "dh_objects.h"

using namespace dh;

namespace {

constexpr int kMaxDevices = 64;

// per-block bins ([DH_STATIC_ADJOINT_BLOCKS][factors], row stride = factors) followed by the summed bins
static __device__ __align__(256) double g_adjoint_scratch[DH_STATIC_ADJOINT_BLOCKS * DH_STATIC_ADJOINT_MAX_FACTORS +
                                                          DH_STATIC_ADJOINT_MAX_FACTORS];

// In host code g_adjoint_scratch names a host-side stand-in, not device memory: the device address
// is looked up once per device (with that device current) and cached here.
double* g_scratch_address[kMaxDevices] = {};
std::mutex g_scratch_mutex;
// host copy of the summed bins (a static array, so the call allocates nothing on the host either)
double g_host_bins[DH_STATIC_ADJOINT_MAX_FACTORS];

int scratch_address(double** out) {
  int dev = 0;
  DH_CUDA(cudaGetDevice(&dev));
  DH_CHECK(dev >= 0 && dev < kMaxDevices, DH_ERR_UNSUPPORTED, "device %d beyond the %d devices supported", dev,
           kMaxDevices);
  if (!g_scratch_address[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_adjoint_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_adjoint_scratch)", __FILE__, __LINE__);
    g_scratch_address[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_address[dev];
  return DH_OK;
}

}  // namespace

extern "C" int dh_hamiltonian_pseudopotential_adjoint_static(dh_hamiltonian_t h, const double* u, const double* v,
                                                             double* out) {
  DH_CHECK(h && u && v && out, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK(h->kind == SPACE_FERMION && !h->l2_only, DH_ERR_UNSUPPORTED,
           "the pseudopotential adjoint needs an FQHE interaction Hamiltonian");
  DH_CHECK(is_device_pointer(u) && is_device_pointer(v), DH_ERR_ARGUMENT,
           "u and v must be device pointers: this entry point stages nothing");
  const int nf = h->tabs.nbr_factors;
  DH_CHECK(nf <= DH_STATIC_ADJOINT_MAX_FACTORS, DH_ERR_UNSUPPORTED,
           "%d interaction factors exceed the static scratch of %d (lz_max <= 33)", nf, DH_STATIC_ADJOINT_MAX_FACTORS);
  dh_space_s* sp = h->space;
  int current = -1;
  DH_CUDA(cudaGetDevice(&current));
  DH_CHECK(current == sp->device, DH_ERR_STATE,
           "device %d is current but the Hamiltonian's space lives on device %d: make that device current", current,
           sp->device);
  // the lookup mode's table is built when the mode is selected, so nothing is allocated here
  DH_CHECK(sp->index_mode != DH_INDEX_LOOKUP || sp->lookup.ptr, DH_ERR_STATE, "lookup table missing");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  double* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != DH_OK) return rc;
  double* partial = scratch;
  double* bins = scratch + (size_t)DH_STATIC_ADJOINT_BLOCKS * DH_STATIC_ADJOINT_MAX_FACTORS;
  // every block overwrites its whole partial row and the sum kernel overwrites the bins, so the
  // previous call's contents need no clearing
  rc = launch_fqhe_bins(fqhe_device(sp, h, DH_PRECISION_FP64), u, v, partial, DH_STATIC_ADJOINT_BLOCKS, bins, h->stream);
  if (rc != DH_OK) return rc;
  DH_CUDA(cudaMemcpyAsync(g_host_bins, bins, nf * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DH_CUDA(cudaStreamSynchronize(h->stream));
  const int nlz = h->tabs.lz_max + 1;
  double grad[64];
  for (int m = 0; m < nlz; ++m) {
    double acc = 0.0;
    for (int f = 0; f < nf; ++f) acc += g_host_bins[f] * h->tabs.dfactor[(size_t)f * nlz + m];
    grad[m] = acc;
  }
  if (is_device_pointer(out)) {
    DH_CUDA(cudaMemcpyAsync(out, grad, nlz * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    DH_CUDA(cudaStreamSynchronize(h->stream));
  } else {
    for (int m = 0; m < nlz; ++m) out[m] = grad[m];
  }
  return DH_OK;
}
