// C-ABI entry points of libmsc_b200.so (declared in include/msc.h).
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>

#include "mv_common.cuh"
#include "pc.cuh"

namespace msc {

static thread_local char g_err[512] = "";
static std::atomic<long long> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

// Plan buffers come from the stream-ordered allocator on the plan's stream: an
// allocation or a release never synchronises the device, so plans on different
// streams (the batch workers) build and solve concurrently. A reallocation bumps
// the plan's generation, which invalidates its captured solver graphs.
//
// The allocations draw on one memory pool of the library per device whose release
// threshold is 1/8 of the device memory, at most 16 GiB: memory freed by a plan stays
// reserved up to that amount and the next plan (a batch over slabs of many shapes
// creates and destroys plans all the time) reuses it without mapping it again, which
// the default pool (threshold 0) does at every synchronisation. Above the threshold the
// pool returns memory to the driver at synchronisation.
namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};
}  // namespace

cudaMemPool_t device_pool(int device) {
  if (device < 0 || device >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pools[device]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    size_t fr = 0, total = 0;
    if (cudaMemGetInfo(&fr, &total) != cudaSuccess) {
      cudaGetLastError();
      total = 0;
    }
    uint64_t thr = std::min<uint64_t>(16ull << 30, total / 8);
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    g_pools[device] = pool;
  }
  return g_pools[device];
}

cudaError_t pool_alloc(void** p, size_t bytes, int device, cudaStream_t st) {
  cudaMemPool_t pool = device_pool(device);
  if (!pool) return cudaMallocAsync(p, bytes, st);
  return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

int dalloc(msc_plan* pl, DBuf& b, size_t bytes) {
  if (b.p && b.bytes >= bytes) return MSC_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(pl->stream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
    set_error("internal: device allocation while a solver cycle is being captured");
    return MSC_ERR_STATE;
  }
  if (b.p) dfree(pl, b);
  if (bytes == 0) bytes = 16;
  void* p = nullptr;
  cudaError_t e = pool_alloc(&p, bytes, pl->device, pl->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return MSC_ERR_NOMEM;
  }
  b.p = p;
  b.bytes = bytes;
  pl->bytes += (int64_t)bytes;
  ++pl->gen;
  return MSC_OK;
}

void dfree(msc_plan* pl, DBuf& b) {
  if (b.p) {
    cudaFreeAsync(b.p, pl->stream);
    pl->bytes -= (int64_t)b.bytes;
    ++pl->gen;
  }
  b.p = nullptr;
  b.bytes = 0;
}

// Multiply an SoA field by exp(sign * i k_par . x) at the cube centres.
__global__ void k_bloch(double2* v, int M, int nsite, double a, double kx, double ky, int sign) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 9LL * nsite) return;
  const int s = (int)(e % nsite);
  const int j = s % M, i = (s / M) % M;
  const double d = 2.0 * a;
  const double x = (i - (M - 1) / 2.0) * d, y = (j - (M - 1) / 2.0) * d;
  double sn, cs;
  sincos(sign * (kx * x + ky * y), &sn, &cs);
  v[e] = v[e] * make_double2(cs, sn);
}

__global__ void k_narrow(const double2* __restrict__ a, float2* __restrict__ b, size_t n) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) b[e] = make_float2((float)a[e].x, (float)a[e].y);
}

int launch_narrow(msc_plan* pl, const double2* a, float2* b, size_t n) {
  k_narrow<<<ceil_div((long long)n, 256), 256, 0, pl->stream>>>(a, b, n); ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}

int bloch_modulate(msc_plan* pl, double2* v, int sign) {
  const Geo& g = pl->g;
  k_bloch<<<ceil_div(9LL * g.nsite, 256), 256, 0, pl->stream>>>(v, g.M, g.nsite, pl->desc.a, pl->kpar[0], pl->kpar[1],
                                                                sign); ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}

// Smallest power of two >= n.
static int pow2_at_least(int n) {
  int L = 1;
  while (L < n) L *= 2;
  return L;
}

// Smallest FFT length >= n whose factors are 2, 3, 5, 7 -- or the next power of two
// when that is at most 1/16 longer: the power-of-two lengths run the compile-time and
// register FFT kernels and, at 64 and 128, the fused plane passes, several times faster
// than the mixed-radix ones (2 M - 1 = 63 for M = 32: 64 instead of 63).
static int nice_length(int n) {
  for (int L = std::max(n, 1);; ++L) {
    int r = L;
    for (int p : {2, 3, 5, 7})
      while (r % p == 0) r /= p;
    if (r == 1) {
      const int p2 = pow2_at_least(n);
      return 16 * p2 <= 17 * L ? p2 : L;
    }
  }
}

int read_small(msc_plan* pl, const void* dev, void* out, size_t bytes) {
  if (bytes > 64) {
    set_error("internal: a small read of %zu bytes", bytes);
    return MSC_ERR_STATE;
  }
  if (!pl->hpin) MSC_CUDA(cudaMallocHost(&pl->hpin, 64));
  MSC_CUDA(cudaMemcpyAsync(pl->hpin, dev, bytes, cudaMemcpyDeviceToHost, pl->stream));
  MSC_CUDA(cudaStreamSynchronize(pl->stream));
  memcpy(out, pl->hpin, bytes);
  return MSC_OK;
}

int read_status(msc_plan* pl, int* word) {
  *word = 0;
  if (!pl->status.p) return MSC_OK;
  MSC_TRY(read_small(pl, pl->status.p, word, sizeof(int)));
  if (*word) MSC_CUDA(cudaMemsetAsync(pl->status.p, 0, sizeof(int), pl->stream));
  return MSC_OK;
}

}  // namespace msc

using namespace msc;

extern "C" int msc_plan_create(const msc_slab_desc* d, void* stream, msc_plan** out);

namespace msc {
namespace {

// Microseconds per complex64 operator application of the descriptor's lattice padded to
// L laterally: a throwaway plan with a zero spectrum and zero T0 (the kernels' timing does
// not depend on the values), 2 untimed and 5 timed applications on the plan's stream.
// Negative when the plan cannot be built.
double time_lateral(const msc_slab_desc* d, int L, void* stream) {
  msc_slab_desc dd = *d;
  dd.Lxy = L;
  msc_plan* t = nullptr;
  if (msc_plan_create(&dd, stream, &t) != MSC_OK) return -1.0;
  double us = -1.0;
  const Geo& g = t->g;
  DBuf x, y;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  t->E = 45;
  bool ok = dalloc(t, t->khat32, sizeof(float2) * khat_elems_t<float>(g, 45)) == MSC_OK &&
            dalloc(t, t->t4_32, sizeof(float2) * 4 * (size_t)g.nsite) == MSC_OK &&
            dalloc(t, x, sizeof(float2) * field_elems(g)) == MSC_OK &&
            dalloc(t, y, sizeof(float2) * field_elems(g)) == MSC_OK &&
            cudaMemsetAsync(t->khat32.p, 0, t->khat32.bytes, t->stream) == cudaSuccess &&
            cudaMemsetAsync(t->t4_32.p, 0, t->t4_32.bytes, t->stream) == cudaSuccess &&
            cudaMemsetAsync(x.p, 0, x.bytes, t->stream) == cudaSuccess &&
            cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
  if (ok) {
    t->has_t0 = t->has_g0 = true;
    for (int i = 0; i < 7 && ok; ++i) {
      if (i == 2) ok = cudaEventRecord(e0, t->stream) == cudaSuccess;
      if (ok) ok = launch_matvec<float>(t, (const float2*)x.p, nullptr, (float2*)y.p, nullptr) == MSC_OK;
    }
    float ms = 0.f;
    if (ok && cudaEventRecord(e1, t->stream) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
      us = 1e3 * ms / 5.0;
  }
  cudaGetLastError();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  dfree(t, x);
  dfree(t, y);
  msc_plan_destroy(t);
  return us;
}

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_tune;  // (device, M, N_z, Lz) -> lateral length

}  // namespace

// The autotuned lateral FFT length of an aperiodic plan (descriptor Lxy = -1): the
// smallest 2,3,5,7-smooth length >= 2M - 1 or the next power of two, whichever runs the
// complex64 operator faster on this device (the power of two takes the compile-time,
// register and fused plane kernels; the smooth length moves less data). Timed once per
// device and lattice shape in the process and remembered.
int tuned_lateral(const msc_slab_desc* d, int Lz, void* stream) {
  const int n = 2 * d->M - 1;
  const int p2 = pow2_at_least(n);
  int smooth = n;
  for (;; ++smooth) {
    int r = smooth;
    for (int p : {2, 3, 5, 7})
      while (r % p == 0) r /= p;
    if (r == 1) break;
  }
  if (smooth == p2) return p2;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, d->M, d->N_z, Lz);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
  }
  const double ts = time_lateral(d, smooth, stream), tp = time_lateral(d, p2, stream);
  const int pick = (tp > 0 && (ts <= 0 || tp < ts)) ? p2 : smooth;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = pick;
  return pick;
}

}  // namespace msc

extern "C" {

const char* msc_status_string(int s) {
  switch (s) {
    case MSC_OK: return "MSC_OK";
    case MSC_NOT_CONVERGED: return "MSC_NOT_CONVERGED";
    case MSC_BREAKDOWN: return "MSC_BREAKDOWN";
    case MSC_ERR_INVALID: return "MSC_ERR_INVALID";
    case MSC_ERR_UNSUPPORTED: return "MSC_ERR_UNSUPPORTED";
    case MSC_ERR_CUDA: return "MSC_ERR_CUDA";
    case MSC_ERR_NOMEM: return "MSC_ERR_NOMEM";
    case MSC_ERR_STATE: return "MSC_ERR_STATE";
    case MSC_ERR_NONFINITE: return "MSC_ERR_NONFINITE";
    case MSC_ERR_TIMEOUT: return "MSC_ERR_TIMEOUT";
    default: return "MSC_UNKNOWN";
  }
}

const char* msc_last_error(void) { return g_err; }
int64_t msc_launch_count(void) { return g_launches.load(); }
const char* msc_version(void) { return "msc_b200 0.1.0 (sm_100a)"; }

int msc_plan_create(const msc_slab_desc* d, void* stream, msc_plan** out) {
  if (!d || !out) {
    set_error("null argument");
    return MSC_ERR_INVALID;
  }
  *out = nullptr;
  if (d->M < 1) { set_error("M must be >= 1, got %d", d->M); return MSC_ERR_INVALID; }
  if (d->N_z < 1) { set_error("N_z must be >= 1, got %d", d->N_z); return MSC_ERR_INVALID; }
  if (!(d->a > 0)) { set_error("a must be > 0, got %g", d->a); return MSC_ERR_INVALID; }
  if (!(d->alpha > 0) || !(d->beta > 0) || !(d->rho > 0)) {
    set_error("alpha, beta, rho must be positive");
    return MSC_ERR_INVALID;
  }
  if (!(d->alpha > d->beta)) {
    set_error("alpha must exceed beta (Poisson ratio below 1/2)");
    return MSC_ERR_INVALID;
  }
  const long long nsite = (long long)d->N_z * d->M * d->M;
  if (9LL * nsite >= (1LL << 31)) {
    set_error("lattice too large: 9*N_z*M*M must be < 2^31");
    return MSC_ERR_INVALID;
  }
  msc_plan* pl = new msc_plan();
  pl->desc = *d;
  pl->user = (cudaStream_t)stream;
  cudaGetDevice(&pl->device);
  Geo& g = pl->g;
  g.M = d->M;
  g.Nz = d->N_z;
  g.nsite = (int)nsite;
  // z padding: a power of two (the z spectrum exists only in shared memory; power-of-two
  // lengths use the compile-time FFT kernels and their pruned first and last stages)
  int Lz = d->Lz > 0 ? d->Lz : pow2_at_least(2 * d->N_z - 1);
  if (Lz < 2 * d->N_z - 1) {
    delete pl;
    set_error("Lz=%d is below 2*N_z-1=%d", Lz, 2 * d->N_z - 1);
    return MSC_ERR_INVALID;
  }
  int Lxy;
  if (d->periodic) Lxy = d->M;
  else {
    if (d->Lxy < -1) {
      delete pl;
      set_error("Lxy must be >= -1 (-1: autotuned, 0: automatic), got %d", d->Lxy);
      return MSC_ERR_INVALID;
    }
    Lxy = d->Lxy > 0 ? d->Lxy : d->Lxy == -1 ? tuned_lateral(d, Lz, stream) : nice_length(2 * d->M - 1);
    if (Lxy < 2 * d->M - 1) {
      delete pl;
      set_error("Lxy=%d is below 2*M-1=%d", Lxy, 2 * d->M - 1);
      return MSC_ERR_INVALID;
    }
  }
  g.Lz = Lz;
  g.Lx = g.Ly = Lxy;
  set_spectrum_box(g, true);
  if (!make_fft_plan(Lz, &pl->fz) || !make_fft_plan(Lxy, &pl->fxy)) {
    delete pl;
    set_error("FFT lengths (Lz=%d, Lxy=%d) need prime factors <= 11 and length <= 4096", Lz, Lxy);
    return MSC_ERR_UNSUPPORTED;
  }
  // the fused z-pass kernel holds at least 36 lines of Lz complex128 twice
  if (zbz_min_smem64(Lz) > (size_t)ZBZ_SMEM_LIMIT) {
    delete pl;
    set_error("Lz=%d exceeds the shared memory of the fused z pass (Lz <= 192, N_z <= 96)", Lz);
    return MSC_ERR_UNSUPPORTED;
  }
  if (cudaStreamCreateWithFlags(&pl->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&pl->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&pl->ev_out, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    if (pl->stream) cudaStreamDestroy(pl->stream);
    if (pl->ev_in) cudaEventDestroy(pl->ev_in);
    delete pl;
    set_error("could not create the plan's stream");
    return MSC_ERR_CUDA;
  }
  StreamFence fence(pl);
  int s = build_twiddles(pl);
  if (s == MSC_OK) s = dalloc(pl, pl->status, 64);
  if (s == MSC_OK && cudaMemsetAsync(pl->status.p, 0, 64, pl->stream) != cudaSuccess) s = MSC_ERR_CUDA;
  if (s == MSC_OK) s = dalloc(pl, pl->W64, sizeof(double2) * ws_elems(g));
  if (s == MSC_OK) s = dalloc(pl, pl->W32, sizeof(float2) * ws_elems(g));
  if (s != MSC_OK) {
    fence.pl = nullptr;
    msc_plan_destroy(pl);
    return s;
  }
  *out = pl;
  return MSC_OK;
}

int msc_plan_destroy(msc_plan* pl) {
  if (!pl) return MSC_OK;
  if (pl->stream) cudaStreamSynchronize(pl->stream);
  else cudaDeviceSynchronize();
  gmres_free(pl);
  if (pl->nf) {
    dfree(pl, pl->nf->g64_dev);
    dfree(pl, pl->nf->g32_dev);
    dfree(pl, pl->nf->g16_dev);
    dfree(pl, pl->nf->tmp32);
    dfree(pl, pl->nf->tmp64);
    delete pl->nf;
    pl->nf = nullptr;
  }
  DBuf* bufs[] = {&pl->tw64_z, &pl->tw64_xy, &pl->tw32_z, &pl->tw32_xy, &pl->t4_64, &pl->t4_32, &pl->khat64,
                  &pl->khat32, &pl->va_blocks, &pl->g0_scratch, &pl->g0_near, &pl->W64, &pl->W32, &pl->Wm64, &pl->Wm32, &pl->f64a, &pl->f64b, &pl->f32a, &pl->f32b,
                  &pl->red, &pl->status};
  for (DBuf* b : bufs) dfree(pl, *b);
  cudaStreamSynchronize(pl->stream);
  if (pl->ev_in) cudaEventDestroy(pl->ev_in);
  if (pl->ev_out) cudaEventDestroy(pl->ev_out);
  if (pl->stream) cudaStreamDestroy(pl->stream);
  if (pl->hpin) cudaFreeHost(pl->hpin);
  delete pl;
  return MSC_OK;
}

int msc_plan_set_stream(msc_plan* pl, void* stream) {
  if (!pl) { set_error("null plan"); return MSC_ERR_INVALID; }
  // the plan's own stream stays; later calls are ordered after `stream`
  pl->user = (cudaStream_t)stream;
  return MSC_OK;
}

int msc_plan_fft_sizes(const msc_plan* pl, int32_t* o) {
  if (!pl || !o) { set_error("null argument"); return MSC_ERR_INVALID; }
  o[0] = pl->g.Lz;
  o[1] = pl->g.Lx;
  o[2] = pl->g.Ly;
  return MSC_OK;
}

int64_t msc_plan_device_bytes(const msc_plan* pl) { return pl ? pl->bytes : 0; }

int msc_plan_set_wait_limit(msc_plan* pl, int64_t polls, int inject) {
  if (!pl) { set_error("null plan"); return MSC_ERR_INVALID; }
  if (polls < 0) { set_error("the wait limit must be >= 0 (0 = default), got %lld", (long long)polls); return MSC_ERR_INVALID; }
  if (inject != 0 && inject != 1) { set_error("inject must be 0 or 1, got %d", inject); return MSC_ERR_INVALID; }
  pl->wait_limit = polls;
  pl->inject_wait = inject;
  ++pl->gen;  // captured solver graphs bind both as kernel parameters
  return MSC_OK;
}

int msc_plan_status(msc_plan* pl, int32_t* word) {
  StreamFence fence(pl);
  if (!pl || !word) { set_error("null argument"); return MSC_ERR_INVALID; }
  int w = 0;
  MSC_TRY(read_status(pl, &w));
  *word = w;
  return MSC_OK;
}

int msc_build_t0(msc_plan* pl, const double* dlam, const double* dmu, const double* drho, double omega) {
  StreamFence fence(pl);
  if (!pl || !dlam || !dmu || !drho) { set_error("null argument"); return MSC_ERR_INVALID; }
  if (!(omega > 0)) { set_error("omega must be > 0, got %g", omega); return MSC_ERR_INVALID; }
  MSC_TRY(launch_t0(pl, dlam, dmu, drho, omega));
  pl->has_t0 = true;
  pl->omega_t0 = omega;
  return MSC_OK;
}

int msc_t0_scalars(const msc_plan* pl, void* out) {
  StreamFence fence(const_cast<msc_plan*>(pl));
  if (!pl || !out) { set_error("null argument"); return MSC_ERR_INVALID; }
  if (!pl->has_t0) { set_error("build_t0 first"); return MSC_ERR_STATE; }
  MSC_CUDA(cudaMemcpyAsync(out, pl->t4_64.p, sizeof(double2) * 4 * pl->g.nsite, cudaMemcpyDeviceToDevice, pl->stream));
  return MSC_OK;
}

int msc_set_t0_scalars(msc_plan* pl, const void* t4, double omega) {
  StreamFence fence(pl);
  if (!pl || !t4) { set_error("null argument"); return MSC_ERR_INVALID; }
  const size_t n = (size_t)4 * pl->g.nsite;
  MSC_TRY(dalloc(pl, pl->t4_64, sizeof(double2) * n));
  MSC_TRY(dalloc(pl, pl->t4_32, sizeof(float2) * n));
  MSC_CUDA(cudaMemcpyAsync(pl->t4_64.p, t4, sizeof(double2) * n, cudaMemcpyDeviceToDevice, pl->stream));
  MSC_TRY(launch_narrow(pl, (const double2*)pl->t4_64.p, (float2*)pl->t4_32.p, n));
  pl->has_t0 = true;
  pl->omega_t0 = omega;
  return MSC_OK;
}

int msc_build_g0(msc_plan* pl, double omega, const double* kpar, int volume_averaged, int n_orders) {
  StreamFence fence(pl);
  if (!pl) { set_error("null plan"); return MSC_ERR_INVALID; }
  if (!(omega > 0)) { set_error("omega must be > 0, got %g", omega); return MSC_ERR_INVALID; }
  if (n_orders < 0) { set_error("n_orders must be >= 0"); return MSC_ERR_INVALID; }
  if (kpar && !pl->desc.periodic) {
    set_error("a Bloch wavevector needs a periodic plan");
    return MSC_ERR_INVALID;
  }
  pl->bloch = kpar != nullptr;
  pl->kpar[0] = kpar ? kpar[0] : 0.0;
  pl->kpar[1] = kpar ? kpar[1] : 0.0;
  MSC_TRY(launch_g0(pl, omega, kpar, volume_averaged ? 1 : 0, n_orders));
  pl->has_g0 = true;
  pl->omega_g0 = omega;
  pl->va = volume_averaged ? 1 : 0;
  pl->n_orders = n_orders;
  return MSC_OK;
}

int msc_incident(msc_plan* pl, double omega, const double* k_hat, int wave_type, void* psi0) {
  StreamFence fence(pl);
  if (!pl || !k_hat || !psi0) { set_error("null argument"); return MSC_ERR_INVALID; }
  return launch_incident(pl, omega, k_hat, wave_type, (double2*)psi0, nullptr, false);
}

int msc_matvec(msc_plan* pl, const void* x, void* y, int precision) {
  StreamFence fence(pl);
  if (!pl || !x || !y) { set_error("null argument"); return MSC_ERR_INVALID; }
  if (x == y) { set_error("x and y may not alias"); return MSC_ERR_INVALID; }
  const size_t n = field_elems(pl->g);
  if (precision == MSC_COMPLEX128) {
    MSC_TRY(dalloc(pl, pl->f64a, sizeof(double2) * n));
    MSC_TRY(dalloc(pl, pl->f64b, sizeof(double2) * n));
    MSC_TRY((launch_ref_to_soa<double, double>(pl, (const double2*)x, (double2*)pl->f64a.p)));
    MSC_TRY(launch_matvec<double>(pl, (const double2*)pl->f64a.p, nullptr, (double2*)pl->f64b.p, nullptr));
    MSC_TRY((launch_soa_to_ref<double, double>(pl, (const double2*)pl->f64b.p, (double2*)y)));
  } else if (precision == MSC_COMPLEX64) {
    MSC_TRY(dalloc(pl, pl->f32a, sizeof(float2) * n));
    MSC_TRY(dalloc(pl, pl->f32b, sizeof(float2) * n));
    MSC_TRY((launch_ref_to_soa<float, float>(pl, (const float2*)x, (float2*)pl->f32a.p)));
    MSC_TRY(launch_matvec<float>(pl, (const float2*)pl->f32a.p, nullptr, (float2*)pl->f32b.p, nullptr));
    MSC_TRY((launch_soa_to_ref<float, float>(pl, (const float2*)pl->f32b.p, (float2*)y)));
  } else {
    set_error("precision must be 0 (complex64) or 1 (complex128)");
    return MSC_ERR_INVALID;
  }
  return MSC_OK;
}

int msc_matvec_soa(msc_plan* pl, const void* x, void* y, int precision) {
  StreamFence fence(pl);
  if (!pl || !x || !y) { set_error("null argument"); return MSC_ERR_INVALID; }
  if (x == y) { set_error("x and y may not alias"); return MSC_ERR_INVALID; }
  if (precision == MSC_COMPLEX128) return launch_matvec<double>(pl, (const double2*)x, nullptr, (double2*)y, nullptr);
  if (precision == MSC_COMPLEX64) return launch_matvec<float>(pl, (const float2*)x, nullptr, (float2*)y, nullptr);
  set_error("precision must be 0 (complex64) or 1 (complex128)");
  return MSC_ERR_INVALID;
}

int msc_set_nearfield(msc_plan* pl, int degree, const double* coef, const double* dblocks) {
  if (!pl) { set_error("null plan"); return MSC_ERR_INVALID; }
  if (degree < 1 || degree > NF_MAXL) { set_error("degree must be in [1, %d], got %d", NF_MAXL, degree); return MSC_ERR_INVALID; }
  if (!pl->nf) pl->nf = new NearField();
  NearField* nf = pl->nf;
  nf->L = degree;
  for (int l = 0; l <= NF_MAXL; ++l)
    nf->coef[l] = (coef && l <= degree) ? make_double2(coef[2 * l], coef[2 * l + 1]) : make_double2(1.0, 0.0);
  if (dblocks) {
    nf->dg.assign((size_t)degree * NF_OFFS * 81, make_double2(0, 0));
    for (size_t i = 0; i < nf->dg.size(); ++i) nf->dg[i] = make_double2(dblocks[2 * i], dblocks[2 * i + 1]);
  } else {
    nf->dg.clear();
  }
  nf->dirty = true;
  ++pl->gen;
  return MSC_OK;
}

int msc_set_nearfield_weights(msc_plan* pl, int format) {
  if (!pl) { set_error("null plan"); return MSC_ERR_INVALID; }
  if (format != MSC_NF_WEIGHTS_FP32 && format != MSC_NF_WEIGHTS_BF16 && format != MSC_NF_WEIGHTS_BF16_TC) {
    set_error("weight format must be 0 (FP32), 1 (BF16) or 2 (BF16 on the tensor cores), got %d", format);
    return MSC_ERR_INVALID;
  }
  if (!pl->nf) pl->nf = new NearField();
  pl->nf->wbf16 = format;
  ++pl->gen;  // the captured solver graphs bind the block pointer
  return MSC_OK;
}

int msc_nearfield_blocks(const msc_plan* pl, double* out) {
  if (!pl || !out) { set_error("null argument"); return MSC_ERR_INVALID; }
  if (!pl->nf || !pl->nf->ready) { set_error("the near-field blocks need build_g0 first"); return MSC_ERR_STATE; }
  MSC_TRY(nf_host_sync(pl));
  for (int i = 0; i < NF_OFFS * 81; ++i) {
    out[2 * i] = pl->nf->g64[i].x;
    out[2 * i + 1] = pl->nf->g64[i].y;
  }
  return MSC_OK;
}

int msc_precondition(msc_plan* pl, const void* x, void* z, int precision) {
  StreamFence fence(pl);
  if (!pl || !x || !z) { set_error("null argument"); return MSC_ERR_INVALID; }
  if (x == z) { set_error("x and z may not alias"); return MSC_ERR_INVALID; }
  if (!pl->has_t0) { set_error("the preconditioner needs build_t0 first"); return MSC_ERR_STATE; }
  const size_t n = field_elems(pl->g);
  if (precision == MSC_COMPLEX128) {
    MSC_TRY(dalloc(pl, pl->f64a, sizeof(double2) * n));
    MSC_TRY(dalloc(pl, pl->f64b, sizeof(double2) * n));
    MSC_TRY((launch_ref_to_soa<double, double>(pl, (const double2*)x, (double2*)pl->f64a.p)));
    MSC_TRY(nearfield_apply<double>(pl, (const double2*)pl->f64a.p, nullptr, (double2*)pl->f64b.p, nullptr));
    MSC_TRY((launch_soa_to_ref<double, double>(pl, (const double2*)pl->f64b.p, (double2*)z)));
  } else if (precision == MSC_COMPLEX64) {
    MSC_TRY(dalloc(pl, pl->f32a, sizeof(float2) * n));
    MSC_TRY(dalloc(pl, pl->f32b, sizeof(float2) * n));
    MSC_TRY((launch_ref_to_soa<float, float>(pl, (const float2*)x, (float2*)pl->f32a.p)));
    MSC_TRY(nearfield_apply<float>(pl, (const float2*)pl->f32a.p, nullptr, (float2*)pl->f32b.p, nullptr));
    MSC_TRY((launch_soa_to_ref<float, float>(pl, (const float2*)pl->f32b.p, (float2*)z)));
  } else {
    set_error("precision must be 0 (complex64) or 1 (complex128)");
    return MSC_ERR_INVALID;
  }
  return MSC_OK;
}

int msc_solve(msc_plan* pl, const void* b, void* x, const msc_solve_opts* o, msc_solve_stats* st) {
  StreamFence fence(pl);
  if (!pl || !b || !x || !o) { set_error("null argument"); return MSC_ERR_INVALID; }
  if (o->precision != MSC_SOLVE_MIXED && o->precision != MSC_SOLVE_FP64) {
    set_error("precision must be mixed (0) or fp64 (1)");
    return MSC_ERR_INVALID;
  }
  if (o->initial_guess != 0 && o->initial_guess != 1) {
    set_error("initial_guess must be 0 (born) or 1 (zero)");
    return MSC_ERR_INVALID;
  }
  return solve(pl, (const double2*)b, (double2*)x, o, st);
}

int msc_solve_multi(msc_plan* pl, int nrhs, const void* b, void* x, const msc_solve_opts* o, msc_solve_stats* st) {
  StreamFence fence(pl);
  if (!pl || !b || !x || !o) { set_error("null argument"); return MSC_ERR_INVALID; }
  if (nrhs < 1 || nrhs > MSC_MAX_RHS) { set_error("nrhs must be in [1, %d], got %d", MSC_MAX_RHS, nrhs); return MSC_ERR_INVALID; }
  if (b == x) { set_error("b and x may not alias"); return MSC_ERR_INVALID; }
  if (o->precision != MSC_SOLVE_MIXED && o->precision != MSC_SOLVE_FP64) {
    set_error("precision must be mixed (0) or fp64 (1)");
    return MSC_ERR_INVALID;
  }
  if (o->initial_guess != 0 && o->initial_guess != 1) {
    set_error("initial_guess must be 0 (born) or 1 (zero)");
    return MSC_ERR_INVALID;
  }
  return solve_multi(pl, nrhs, (const double2*)b, (double2*)x, o, st);
}

int msc_matvec_multi(msc_plan* pl, int nrhs, const void* x, void* y, int precision) {
  StreamFence fence(pl);
  if (!pl || !x || !y) { set_error("null argument"); return MSC_ERR_INVALID; }
  if (nrhs < 1 || nrhs > MSC_MAX_RHS) { set_error("nrhs must be in [1, %d], got %d", MSC_MAX_RHS, nrhs); return MSC_ERR_INVALID; }
  if (x == y) { set_error("x and y may not alias"); return MSC_ERR_INVALID; }
  if (!pl->has_t0 || !pl->has_g0) { set_error("matvec needs build_t0 and build_g0 first"); return MSC_ERR_STATE; }
  const Geo& g = pl->g;
  if (precision == MSC_COMPLEX128) {
    MSC_TRY(dalloc(pl, pl->Wm64, sizeof(double2) * ws_elems(g) * nrhs));
    return launch_matvec_ws<double>(pl, (const double2*)x, nullptr, (double2*)y, (double2*)pl->Wm64.p, nullptr, nrhs);
  }
  if (precision == MSC_COMPLEX64) {
    MSC_TRY(dalloc(pl, pl->Wm32, sizeof(float2) * ws_elems(g) * nrhs));
    return launch_matvec_ws<float>(pl, (const float2*)x, nullptr, (float2*)y, (float2*)pl->Wm32.p, nullptr, nrhs);
  }
  set_error("precision must be 0 (complex64) or 1 (complex128)");
  return MSC_ERR_INVALID;
}

int msc_rpp_periodic(msc_plan* pl, const void* psi, double omega, double p, int flags, double* out) {
  StreamFence fence(pl);
  if (!pl || !psi || !out) { set_error("null argument"); return MSC_ERR_INVALID; }
  if (flags & ~(MSC_RPP_BLOCH | MSC_RPP_PLANE_WAVE_MOMENT)) { set_error("unknown R_PP flags %d", flags); return MSC_ERR_INVALID; }
  return rpp_periodic(pl, (const double2*)psi, omega, p, flags, out);
}

int msc_reflected_field(msc_plan* pl, const void* psi, double omega, const double* k_hat, double* out) {
  StreamFence fence(pl);
  if (!pl || !psi || !k_hat || !out) { set_error("null argument"); return MSC_ERR_INVALID; }
  return reflected_field(pl, (const double2*)psi, omega, k_hat, out);
}

}  // extern "C"
