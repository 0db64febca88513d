// Internal plan state shared by the translation units of libmsc_b200.so.
#pragma once
#include <algorithm>
#include <string>
#include <vector>

#include "fft_smem.cuh"
#include "msc_common.cuh"

namespace msc {

// Lattice and padded FFT grid. Internal field vectors are component-major
// ("SoA"): v[c][n][i][j], c = 0..8, site = (n*M + i)*M + j.
struct Geo {
  int M, Nz;
  int Lz, Lx, Ly;  // padded FFT lengths (Lx = Ly)
  // Stored spectrum box kz < Hz, ky < Hy, kx < Hx. Octant (oct = 1): H = L/2 + 1 on
  // each axis; the kernel is mirror symmetric, K(R_a k) = S_a K(k) S_a for the
  // reflection of each axis a, and every wavevector reads its mirror image in the
  // box. Full (oct = 0, Bloch-phased kernels, which lose the symmetry): H = L.
  int Hz, Hy, Hx;
  int oct;
  int nsite;       // Nz*M*M
};

void set_error(const char* fmt, ...);
// counts kernel launches of this library (msc_launch_count)
void note_launch();

#define MSC_CUDA(...)                                                                           \
  do {                                                                                          \
    cudaError_t e_ = (__VA_ARGS__);                                                             \
    if (e_ != cudaSuccess) {                                                                    \
      ::msc::set_error("%s:%d %s: %s", __FILE__, __LINE__, #__VA_ARGS__, cudaGetErrorString(e_)); \
      return MSC_ERR_CUDA;                                                                      \
    }                                                                                           \
  } while (0)

#define MSC_TRY(...)           \
  do {                         \
    int s_ = (__VA_ARGS__);    \
    if (s_ < 0) return s_;     \
  } while (0)

// Device buffer owned by a plan.
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct GmresWork;
struct NearField;

}  // namespace msc

struct msc_plan {
  msc_slab_desc desc;
  msc::Geo g;
  // All work of a plan runs on its own non-blocking stream (capturable into graphs);
  // every entry point orders it after the caller's stream `user` and the caller's
  // stream after it (StreamFence).
  cudaStream_t stream = nullptr;
  cudaStream_t user = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  void* hpin = nullptr;  // 64 page-locked bytes for small device-to-host reads
  int device = 0;
  msc::FftPlan1D fz, fxy;
  // twiddles exp(-2 pi i t / L) for Lz and Lxy
  msc::DBuf tw64_z, tw64_xy, tw32_z, tw32_xy;
  // T0
  bool has_t0 = false;
  double omega_t0 = 0;
  msc::DBuf t4_64, t4_32;  // [4][nsite]
  // G0 spectrum: octant, blocked per the fused z pass layout; full: [E][Hz][Hy][Hx]
  bool has_g0 = false;
  int E = 0;               // 45 (symmetric form) or 81 (full, volume averaged)
  int va = 0, n_orders = 2;
  double omega_g0 = 0;
  bool bloch = false;
  double kpar[2] = {0, 0};
  msc::DBuf khat64, khat32;
  msc::DBuf va_blocks;     // [26][81] double
  msc::DBuf g0_scratch;    // [E][Lz][Ly][Lx] complex128, the spectrum build's work array
  msc::DBuf g0_near;       // [E][27] spatial kernel within one cell of the origin (fused G0 build)
  // matvec workspace [9][Nz][Ly][Lx] (y and x transformed, z in space)
  msc::DBuf W64, W32;
  // boundary scratch: SoA copies of in/out fields
  msc::DBuf f64a, f64b, f32a, f32b;
  // reduction scratch (partials, results)
  msc::DBuf red;
  // device status words: [0] = a bounded wait of a kernel timed out
  msc::DBuf status;
  // polls of an mbarrier before a kernel's bounded wait gives up (0 = the kernel's default)
  long long wait_limit = 0;
  // 1: the tensor-core stencil also waits on an mbarrier that never completes, so its
  // bounded wait runs out (msc_plan_set_wait_limit's failure-path test)
  int inject_wait = 0;
  // right-hand sides of the solve in progress (msc_solve_multi: > 1); the matvec then
  // runs on [nrhs][9][nsite] fields with the workspace Wm
  int nrhs = 1;
  msc::DBuf Wm64, Wm32;
  // GMRES workspace (lazily grown)
  msc::GmresWork* gw = nullptr;
  // near-field preconditioner (blocks from the last G0 build, coefficients)
  msc::NearField* nf = nullptr;
  int64_t bytes = 0;
  // bumped by every (re)allocation, spectrum build and preconditioner change: the
  // captured solver graphs of an older generation are stale
  uint64_t gen = 1;
  // capture GMRES cycles into graphs (off for the batch's short-lived plans)
  bool graphs = true;
};

namespace msc {

// Orders the plan's stream after the caller's on entry and the caller's after the
// plan's on exit.
struct StreamFence {
  msc_plan* pl;
  explicit StreamFence(msc_plan* p) : pl(p) {
    if (pl && pl->ev_in) {
      cudaEventRecord(pl->ev_in, pl->user);
      cudaStreamWaitEvent(pl->stream, pl->ev_in, 0);
    }
  }
  ~StreamFence() {
    if (pl && pl->ev_out) {
      cudaEventRecord(pl->ev_out, pl->stream);
      cudaStreamWaitEvent(pl->user, pl->ev_out, 0);
    }
  }
};

int dalloc(msc_plan* pl, DBuf& b, size_t bytes);
// Reads `bytes` (<= 64) from the device on the plan's stream into `out` through the plan's
// page-locked scratch (a pageable destination makes the copy wait for the host's staging
// path with the device idle); synchronises the stream.
int read_small(msc_plan* pl, const void* dev, void* out, size_t bytes);
void dfree(msc_plan* pl, DBuf& b);
// stream-ordered allocation from the library's memory pool of `device`
cudaError_t pool_alloc(void** p, size_t bytes, int device, cudaStream_t st);

// ---- launches (all enqueue on pl->stream) ------------------------------------
int build_twiddles(msc_plan* pl);
int launch_t0(msc_plan* pl, const double* dlam, const double* dmu, const double* drho, double omega);
int launch_g0(msc_plan* pl, double omega, const double* kpar, int va, int n_orders);
int launch_incident(msc_plan* pl, double omega, const double* k_hat, int wave, double2* ref_out, double2* soa_out,
                    bool demod);
// layout conversion between the reference layout (site-major, 9 DOF inner) and SoA
template <typename Tin, typename Tout>
int launch_ref_to_soa(msc_plan* pl, const cx<Tin>* in, cx<Tout>* out);
template <typename Tin, typename Tout>
int launch_soa_to_ref(msc_plan* pl, const cx<Tin>* in, cx<Tout>* out);
// y = x - G0 T0 (scale * x), SoA; scale may be null (1). done may be null. With
// pl->nrhs = R > 1, x and y hold R fields one after the other ([R][9][nsite]) and the
// operator is applied to each (the plan's multi-RHS workspace).
template <typename T>
int launch_matvec(msc_plan* pl, const cx<T>* x, const double* scale, cx<T>* y, const int* done);
// complex64 plane passes with the y and x transforms fused (mv_plane_fused.cu)
bool plane_fused_ok(const msc_plan* pl);
int launch_plane_fwd(msc_plan* pl, const float2* x, const double* scale, float2* W, const int* done, int nrhs);
int launch_plane_inv(msc_plan* pl, const float2* W, const float2* x, const double* scale, float2* y,
                     const int* done, int nrhs);
// complex64 inverse y pass on the register four-step engine, Ly in {64, 128, 256}
// (mv_plane_reg.cu)
bool y_reg_ok(const msc_plan* pl);
int launch_fft_y_out_reg(msc_plan* pl, const float2* W, const float2* x, const double* scale, float2* y,
                         const int* done, int nrhs);
// the same on a caller-provided workspace of nrhs * ws_elems(g) elements, for nrhs
// fields [nrhs][9][nsite]
template <typename T>
int launch_matvec_ws(msc_plan* pl, const cx<T>* x, const double* scale, cx<T>* y, cx<T>* W, const int* done,
                     int nrhs = 1);

int rpp_periodic(msc_plan* pl, const double2* psi_ref, double omega, double p, int flags, double* out);
int reflected_field(msc_plan* pl, const double2* psi_ref, double omega, const double* k_hat, double* out);
int solve(msc_plan* pl, const double2* b_ref, double2* x_ref, const msc_solve_opts* o, msc_solve_stats* st);
// R right-hand sides b_ref[R][N_z][M][M][9] as one stacked system (msc_solve_multi)
int solve_multi(msc_plan* pl, int R, const double2* b_ref, double2* x_ref, const msc_solve_opts* o,
                msc_solve_stats* stats);
// read the plan's device status word (synchronising the plan's stream) and clear it;
// *word = 1 when a kernel's bounded wait ran out since the last read
int read_status(msc_plan* pl, int* word);
void gmres_free(msc_plan* pl);
// v *= exp(sign i k_par . x) at the cube centres (SoA complex128 field)
int bloch_modulate(msc_plan* pl, double2* v, int sign);

inline size_t field_elems(const Geo& g) { return (size_t)9 * g.nsite; }
inline size_t ws_elems(const Geo& g) { return (size_t)9 * g.Nz * g.Ly * g.Lx; }
// Set the stored spectrum box: octant (mirror-symmetric kernel) or full.
inline void set_spectrum_box(Geo& g, bool octant) {
  g.oct = octant ? 1 : 0;
  g.Hz = octant ? g.Lz / 2 + 1 : g.Lz;
  g.Hy = octant ? g.Ly / 2 + 1 : g.Ly;
  g.Hx = octant ? g.Lx / 2 + 1 : g.Lx;
}

}  // namespace msc
