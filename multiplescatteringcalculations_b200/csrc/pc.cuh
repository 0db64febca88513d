// Near-field preconditioner of the slab operator A = I - G0 T0.
//
// S x = G_nn (T0 x), G_nn the 27-point nearest-neighbour part of the spatial
// kernel (offsets |dz|, |dx|, |dy| <= 1, self term zero), zero outside the slab.
// The preconditioner is the polynomial P x = sum_l c_l S^l x, l = 0..L; the
// truncated Neumann series of A^{-1} = sum (G0 T0)^l restricted to the near field
// is c = (1, 1, ..., 1). A learned preconditioner sets the coefficients and adds
// corrections to the stencil blocks of each layer (pc.cu).
#pragma once
#include <cuda_bf16.h>

#include "plan.cuh"

namespace msc {

constexpr int NF_OFFS = 27;   // stencil offsets, o = ((dz + 1) * 3 + dx + 1) * 3 + dy + 1
constexpr int NF_MAXL = 6;    // polynomial degree limit
// One layer's blocks packed as the tensor-core operand (pc_tc.cu): 33 tiles of 32 rows x
// 16 BF16 (27 offsets for DOFs 0-7, 6 for DOF 8).
constexpr int NF_TC_LAYER_BYTES = (NF_OFFS + 6) * 1024;

// Per-plan state of the preconditioner.
struct NearField {
  NearField() {
    for (auto& c : coef) c = make_double2(1.0, 0.0);
  }
  bool ready = false;          // blocks extracted from the current G0
  int L = 2;                   // degree
  double2 coef[NF_MAXL + 1];   // c_0..c_L
  std::vector<double2> g64;    // [27][9][9] physical near-field blocks (host copy)
  std::vector<double2> dg;     // [L][27][9][9] learned block corrections (empty = none)
  // Per-layer blocks g64 + dg[l] on the device, [L][27][81], y_a(v) += g[o][a][b] tau_b(v - o).
  // The kernels read them through these pointers, so a captured solver graph stays valid
  // when the blocks change (a new frequency): only the buffers' contents are refreshed.
  DBuf g64_dev, g32_dev, g16_dev, gtc_dev;
  int wbf16 = 0;               // complex64 path: msc_nf_weights (1, 2: BF16 blocks g16_dev; 2: tensor cores)
  std::vector<double2> h64;    // host staging of the refresh
  std::vector<float2> h32;
  std::vector<__nv_bfloat162> h16;
  std::vector<uint16_t> htc;
  DBuf tmp32, tmp64;           // two field-size work vectors per precision
  bool dirty = true;           // layer blocks to rebuild from g64, dg
  // g64 arrives by an asynchronous copy into `pin` (page-locked), complete at `ev`: the
  // G0 build does not wait for it; nf_host_sync finishes it before g64 is read.
  double2* pin = nullptr;
  cudaEvent_t ev = nullptr;
  bool host_pending = false;
  ~NearField() {
    if (pin) cudaFreeHost(pin);
    if (ev) cudaEventDestroy(ev);
  }
};

// Completes the host copy g64 of the near-field blocks (waits for the copy's event).
int nf_host_sync(const msc_plan* pl);

// Extract the near-field blocks from the spatial kernel of the G0 build (values
// times `scale`), laid out on the padded box of the plan's geometry or on `box`.
int nearfield_extract(msc_plan* pl, const double2* Ks_spatial, double scale, const Geo* box = nullptr);
// Upload the per-layer blocks after a change (synchronises the plan's stream; must not
// run while a graph is being captured).
int nearfield_refresh(msc_plan* pl);
// Pack one layer's BF16 blocks [27][9][9] into the tensor-core operand layout
// (NF_TC_LAYER_BYTES bytes at out).
void nf_tc_pack_layer(const __nv_bfloat162* G16, uint16_t* out);
// One complex64 stencil layer on the tensor cores (pc_tc.cu): the arguments as the
// CUDA-core layer kernel of pc.cu, with the layer's packed blocks on the device.
int launch_nf_tc(msc_plan* pl, const float2* x, const double* scale, const float2* t4, float2* h, float2* acc,
                 float2 ch, float2 c0, int init, const void* Bpacked, const int* done);
// z = P(s v), s = *scale (1 when null); `done` as in the matvec.
template <typename T>
int nearfield_apply(msc_plan* pl, const cx<T>* v, const double* scale, cx<T>* z, const int* done);

}  // namespace msc
