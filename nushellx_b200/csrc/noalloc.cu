// nsx_matvec_noalloc: the FP64 H.v with its scratch in a fixed device array.
//
// Why: nsx_matvec allocates its Y intermediates with cudaMalloc on the first
// product of a handle.  Some callers cannot allow that during the call:
// cudaMalloc synchronises the whole device (it would stall the caller's other
// streams), and hosts that hand all device memory to their own pool allocator
// leave nothing to allocate from.  This entry point allocates nothing; its Y
// scratch is the file-scope array below, of a fixed maximum size.
//
// Rules for callers:
// * The array holds NOALLOC_Y_MAX FP64 elements (64 MiB); a problem whose
//   intermediates (Y and the stacked Zbar) need more is rejected with NSX_E_ARG
//   and a message.
// * Every call looks up the array's device address on the handle's device
//   (the first call on a device loads the library's module there if it is not
//   loaded yet); make that first call before any stream capture.  Every GPU that loads the
//   library holds the array until the process exits.
// * All calls share the one array and it keeps the last call's contents; the
//   product writes every scratch element it later reads, so the previous
//   call's contents do not matter and nothing is cleared.  Calls that overlap
//   on the GPU (different streams, or different handles on the same device,
//   without ordering) race on the array.
#include "nsx_internal.h"

namespace nsx {

constexpr int64_t NOALLOC_Y_MAX = int64_t(8) << 20;  // FP64 elements (64 MiB)

static __device__ __align__(256) double g_noalloc_y[NOALLOC_Y_MAX];

// Device address of g_noalloc_y on the current device.  Looked up on every call (cheap once
// the module is loaded on the device), so a cached address can never outlive a context reset.
static double *noalloc_scratch() {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_y);
  if (e != cudaSuccess) fail(NSX_E_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_y): ") + cudaGetErrorString(e));
  return static_cast<double *>(p);
}

int noalloc_guarded(nsx_handle *h, const double *x, double *y, void *stream);

}  // namespace nsx

int nsx::noalloc_guarded(nsx_handle *h, const double *x, double *y, void *stream) {
  if (!h || !x || !y) fail(NSX_E_ARG, "null argument");
  if (x == y) fail(NSX_E_ARG, "x and y must not alias");
  const int64_t need = zbar_scratch_offset(h) + h->z_elems;
  if (need > NOALLOC_Y_MAX)
    fail(NSX_E_ARG, "problem needs " + std::to_string(need) + " FP64 scratch elements; the fixed array of "
                        "nsx_matvec_noalloc holds " + std::to_string(NOALLOC_Y_MAX) + " (use nsx_matvec)");
  if (h->device < 0) fail(NSX_E_CUDA, "the handle was created without a device (plan only)");
  DeviceGuard dg(h->device);
  double *Y = noalloc_scratch();
  // k_a copies Zbar rows with 16-byte asynchronous copies: Zbar must start 16-byte aligned
  if ((reinterpret_cast<uintptr_t>(Y + zbar_scratch_offset(h)) & 15) != 0)
    fail(NSX_E_CUDA, "the Zbar part of the fixed scratch array is not 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  // the array holds Y then Zbar; the Y stage writes every element of Y (zeros where no density
  // block reaches) and the mixing stage every element of Zbar, so nothing is cleared beforehand
  matvec_fp64_with_scratch(h, x, y, Y, s);
  return NSX_OK;
}
