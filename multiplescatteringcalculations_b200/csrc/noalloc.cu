// msc_matvec_noalloc: the slab operator y = (I - G0 T0) x with no device
// allocation on the call path.
//
// Some callers cannot allocate device memory when they apply the operator: a host
// framework whose allocator owns all device memory and forbids allocations outside
// it, or a real-time loop that must not risk the latency or the failure of
// cudaMalloc in the middle of a run. msc_matvec allocates its two field copies
// lazily on first use; this entry point instead takes its scratch from one static
// device array of this library, of at most NOALLOC_SCRATCH_BYTES. That array is
// created when the library's device code is loaded and stays resident on every GPU
// that loads it until the process exits. The plan (spectrum, T0, twiddles) must
// exist already; building it allocates, this call does not.
//
// Every call, from every plan and thread, shares the one array and leaves its last
// contents there: calls whose GPU work overlaps (different streams, or concurrent
// host threads) race on it and must be serialised by the caller. Each call writes
// every scratch element it later reads, so nothing has to be cleared beforehand.
#include <mutex>

#include "mv_common.cuh"

namespace msc {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(64) << 20;  // 64 MiB

// Device-side array. In host code this name is only a stand-in: its device address
// comes from cudaGetSymbolAddress on each device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of the array per device, looked up on the first call on that
// device (with that device current) and kept for the life of the process. A
// cudaDeviceReset destroys the array's allocation together with every plan of that
// device, so the library does not support being used across a device reset.
static int scratch_address(int dev, void** out) {
  static std::mutex mu;
  static void* addr[128] = {nullptr};
  if (dev < 0 || dev >= 128) {
    set_error("device ordinal %d out of range", dev);
    return MSC_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error("cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
      return MSC_ERR_CUDA;
    }
    addr[dev] = p;
  }
  *out = addr[dev];
  return MSC_OK;
}

static inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

template <typename T>
static int matvec_static(msc_plan* pl, const cx<T>* x_ref, cx<T>* y_ref, unsigned char* scratch) {
  const Geo& g = pl->g;
  const size_t nf = field_elems(g);
  cx<T>* W = reinterpret_cast<cx<T>*>(scratch);
  cx<T>* xs = reinterpret_cast<cx<T>*>(scratch + align256(sizeof(cx<T>) * ws_elems(g)));
  cx<T>* ys = reinterpret_cast<cx<T>*>(reinterpret_cast<unsigned char*>(xs) + align256(sizeof(cx<T>) * nf));
  MSC_TRY((launch_ref_to_soa<T, T>(pl, x_ref, xs)));
  MSC_TRY(launch_matvec_ws<T>(pl, xs, nullptr, ys, W, nullptr));
  MSC_TRY((launch_soa_to_ref<T, T>(pl, ys, y_ref)));
  return MSC_OK;
}

template <typename T> static size_t static_need(const Geo& g) {
  return align256(sizeof(cx<T>) * ws_elems(g)) + 2 * align256(sizeof(cx<T>) * field_elems(g));
}

}  // namespace msc

using namespace msc;

extern "C" int msc_matvec_noalloc(msc_plan* pl, const void* x, void* y, int precision) {
  StreamFence fence(pl);
  if (!pl || !x || !y) {
    set_error("null argument");
    return MSC_ERR_INVALID;
  }
  if (x == y) {
    set_error("x and y may not alias");
    return MSC_ERR_INVALID;
  }
  if (precision != MSC_COMPLEX64 && precision != MSC_COMPLEX128) {
    set_error("precision must be 0 (complex64) or 1 (complex128)");
    return MSC_ERR_INVALID;
  }
  if (!pl->has_t0 || !pl->has_g0) {
    set_error("matvec needs build_t0 and build_g0 first");
    return MSC_ERR_STATE;
  }
  const size_t need = precision == MSC_COMPLEX128 ? static_need<double>(pl->g) : static_need<float>(pl->g);
  if (need > NOALLOC_SCRATCH_BYTES) {
    set_error("msc_matvec_noalloc: this plan needs %zu bytes of scratch, above the static limit of %zu bytes "
              "(use msc_matvec, or complex64, or a smaller lattice)",
              need, (size_t)NOALLOC_SCRATCH_BYTES);
    return MSC_ERR_INVALID;
  }
  int dev = 0;
  MSC_CUDA(cudaGetDevice(&dev));
  if (dev != pl->device) {
    // the array's address is per device: another device's copy would be read by
    // kernels launched on this plan's stream
    set_error("msc_matvec_noalloc: the current device is %d but the plan lives on device %d; make the plan's "
              "device current first", dev, pl->device);
    return MSC_ERR_INVALID;
  }
  void* base = nullptr;
  MSC_TRY(scratch_address(dev, &base));
  unsigned char* s = static_cast<unsigned char*>(base);
  if (precision == MSC_COMPLEX128) return matvec_static<double>(pl, (const double2*)x, (double2*)y, s);
  return matvec_static<float>(pl, (const float2*)x, (float2*)y, s);
}
