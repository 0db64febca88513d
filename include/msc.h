/* C-ABI of the B200 slab Foldy-Lax solver (libmsc_b200.so).
 *
 * Solves (I - G0 T0) psi = psi0 for an M x M x N_z lattice of cubes, the
 * operator of tmnestor/MultipleScatteringCalculations
 * cubic_scattering/slab_scattering.py and slab_scattering_gpu.py.
 *
 * Conventions (the reference's): axis order (z, x, y), z down; 9 DOF per voxel
 * [u_z, u_x, u_y, e_zz, e_xx, e_yy, 2e_xy, 2e_zy, 2e_zx]; fields are complex
 * arrays laid out psi[N_z][M][M][9] (C order); `a` is the cube half-width.
 *
 * All pointers to arrays are DEVICE pointers on the plan's device unless stated.
 * Complex numbers are (re, im) pairs: complex128 = 2 doubles, complex64 = 2 floats.
 * Work is enqueued on the plan's stream; functions that return results to host
 * memory (statistics, R_PP) synchronise that stream. Plans are not thread safe.
 * Every function returns MSC_OK (0), a positive warning status, or a negative
 * error status; msc_status_string() names it and msc_last_error() explains it.
 */
#ifndef MSC_H
#define MSC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum msc_status {
  MSC_OK = 0,
  MSC_NOT_CONVERGED = 1,     /* iteration limit reached above tolerance (reference: warnings.warn) */
  MSC_BREAKDOWN = 2,         /* Krylov breakdown before convergence */
  MSC_ERR_INVALID = -1,      /* invalid argument (reference: ValueError) */
  MSC_ERR_UNSUPPORTED = -2,  /* size whose FFT length has a prime factor > 11 */
  MSC_ERR_CUDA = -3,         /* CUDA runtime error */
  MSC_ERR_NOMEM = -4,        /* device allocation failed */
  MSC_ERR_STATE = -5,        /* call out of order (e.g. matvec before build_t0/build_g0) */
  MSC_ERR_NONFINITE = -6,    /* NaN/Inf met in the solve */
  MSC_ERR_TIMEOUT = -7       /* a kernel's bounded wait ran out (msc_plan_set_wait_limit); the result is invalid */
};

enum msc_precision { MSC_COMPLEX64 = 0, MSC_COMPLEX128 = 1 };
enum msc_solver_precision { MSC_SOLVE_MIXED = 0, MSC_SOLVE_FP64 = 1 };
enum msc_wave { MSC_WAVE_P = 0, MSC_WAVE_S = 1 };
/* MSC_PC_NEARFIELD: flexible GMRES with the near-field preconditioner on the right, in
 * the cycles where it earns its cost: after a few preconditioned cycles one plain cycle
 * is measured, each cycle's residual reduction per unit of device time is compared, and
 * the faster form runs (the slower one is measured again now and then).
 * MSC_PC_NEARFIELD_ALWAYS: every cycle preconditioned. Under both, a preconditioned
 * cycle without any progress turns the preconditioner off for the solve. */
enum msc_preconditioner { MSC_PC_NONE = 0, MSC_PC_NEARFIELD = 1, MSC_PC_NEARFIELD_ALWAYS = 2 };

typedef struct msc_slab_desc {
  int32_t M;         /* lateral cubes per side (SlabGeometry.M) */
  int32_t N_z;       /* layers (SlabGeometry.N_z) */
  double a;          /* cube half-width (SlabGeometry.a) */
  double alpha;      /* background P speed (ReferenceMedium.alpha) */
  double beta;       /* background S speed (ReferenceMedium.beta) */
  double rho;        /* background density (ReferenceMedium.rho) */
  int32_t periodic;  /* 1 = circular convolution over M x M (reference periodic=True) */
  int32_t Lz;        /* padded z FFT length, 0 = automatic (>= 2 N_z - 1) */
  int32_t Lxy;       /* padded lateral FFT length (>= 2M - 1; ignored if periodic): 0 = automatic (the
                        smallest 2,3,5,7-smooth length, or the next power of two when that is at
                        most 1/16 longer); -1 = autotuned: of the smallest smooth length and the
                        next power of two, the one whose complex64 operator runs faster on the
                        current device, timed once per device and lattice shape in the process */
} msc_slab_desc;

typedef struct msc_solve_opts {
  double tol;             /* relative residual target ||b - A x|| / ||b|| (gmres_tol) */
  int32_t max_iter;       /* matvec budget (max_iter) */
  int32_t restart;        /* GMRES restart length m (reference CPU path: scipy default 20) */
  int32_t precision;      /* msc_solver_precision */
  int32_t initial_guess;  /* 0 = Born (x0 = psi0), 1 = zero */
  double inner_tol;       /* mixed precision: relative tolerance of each complex64 inner solve (0 = default) */
  int32_t ortho;          /* Arnoldi: 0 = default (mixed: CGS1, fp64: CGS2), 1 = CGS1, 2 = CGS2 */
  int32_t preconditioner; /* msc_preconditioner: right preconditioner of flexible GMRES */
} msc_solve_opts;

typedef struct msc_solve_stats {
  int32_t n_matvec;      /* operator applications of all precisions (reference: n_gmres_iter) */
  int32_t n_matvec64;    /* of which complex128 */
  int32_t n_outer;       /* refinement sweeps (mixed) or restart cycles (fp64) */
  int32_t status;        /* msc_status of the solve */
  double residual;       /* true relative residual in FP64 (reference: gmres_residual) */
  int32_t n_precond;     /* preconditioner applications */
  int32_t pc_fallback;   /* 1: a preconditioned cycle failed to reduce the residual; plain GMRES finished */
  int32_t pc_cycles;     /* GMRES cycles run with the preconditioner (flexible GMRES) */
  int32_t plain_cycles;  /* cycles run without it: the policy's measurement cycles, the ones where the plain
                            form reduced the residual faster per unit time, and the fallback */
} msc_solve_stats;

typedef struct msc_plan msc_plan;

/* Create a plan for one slab geometry on the current CUDA device. `stream` is a
 * cudaStream_t (NULL = legacy default stream). Replaces the setup of
 * compute_slab_scattering_gpu (slab_scattering_gpu.py:158-226). */
int msc_plan_create(const msc_slab_desc* desc, void* stream, msc_plan** plan);
int msc_plan_destroy(msc_plan* plan);
int msc_plan_set_stream(msc_plan* plan, void* stream);
/* Padded FFT sizes chosen by the plan: out[0..2] = (Lz, Lx, Ly). */
int msc_plan_fft_sizes(const msc_plan* plan, int32_t* out3);
/* Device bytes currently held by the plan. */
int64_t msc_plan_device_bytes(const msc_plan* plan);
/* Polls of an mbarrier before a bounded wait inside the tensor-core stencil gives up
 * (0 = the default, 2^22 polls, far beyond any wait of a correct launch; a poll may
 * itself suspend the thread for a short hardware-defined time). When a wait runs out
 * the kernel stops issuing work, drains its copies and MMAs already in flight, frees
 * its tensor memory, records the timeout in the plan's status word and returns;
 * msc_solve then returns MSC_ERR_TIMEOUT. inject = 1 makes the stencil also wait on an
 * mbarrier that nothing completes, so that this path runs (with a small limit, quickly)
 * and can be tested without a fault; inject = 0 for normal work. No counterpart in the
 * reference (failure handling of this library). */
int msc_plan_set_wait_limit(msc_plan* plan, int64_t polls, int inject);
/* The plan's status word (synchronises the plan's stream) and clear it: *word = 1 when
 * a bounded wait ran out since the last read. No counterpart in the reference. */
int msc_plan_status(msc_plan* plan, int32_t* word);

/* Per-voxel T0 from the contrasts dlam, dmu, drho (device, float64, N_z*M*M each,
 * (N_z, M, M) C order) at angular frequency omega. Replaces compute_slab_tmatrices
 * (slab_scattering.py:169-205) with compute_cube_tmatrix (effective_contrasts.py:454-532)
 * and _sub_cell_tmatrix_9x9 (resonance_tmatrix.py:461-487). */
int msc_build_t0(msc_plan* plan, const double* dlam, const double* dmu, const double* drho, double omega);
/* T0 as 4 complex scalars per voxel, out (4, N_z, M, M) complex128 (device):
 * T0 = diag(t_u I3, [t_l + t_d delta_ij] on the normal strains, t_s I3 on the shears). */
int msc_t0_scalars(const msc_plan* plan, void* out);

/* Set T0 directly from 4 complex scalars per voxel (the layout of msc_t0_scalars),
 * e.g. extracted from user-supplied 9x9 T-matrices (reference T_local arrays). */
int msc_set_t0_scalars(msc_plan* plan, const void* t4, double omega);

/* G0 spectrum at omega. kpar = NULL: the reference's fold (periodic) or the plain
 * linear convolution (aperiodic); kpar = 2 doubles (k_x, k_y): Bloch-phased periodic
 * fold (the field is solved in the demodulated frame psi exp(-i k_par.x)).
 * volume_averaged/n_orders as the reference. Replaces _build_slab_kernels
 * (slab_scattering.py:267-351) and _build_slab_kernels_gpu (slab_scattering_gpu.py:34-92). */
int msc_build_g0(msc_plan* plan, double omega, const double* kpar, int volume_averaged, int n_orders);

/* Incident plane wave psi0 (complex128, (N_z, M, M, 9), device). Replaces
 * _build_slab_incident_field (slab_scattering.py:426-478). */
int msc_incident(msc_plan* plan, double omega, const double* k_hat, int wave_type, void* psi0);

/* y = (I - G0 T0) x for x, y (N_z, M, M, 9) complex of the given precision
 * (msc_precision). Replaces _slab_matvec_gpu (slab_scattering_gpu.py:95-155) and
 * _slab_matvec (slab_scattering.py:359-418). x and y may not alias. */
int msc_matvec(msc_plan* plan, const void* x, void* y, int precision);

/* The same operator on the component-major layout the solver keeps its Krylov
 * vectors in: x, y (9, N_z, M, M) complex, x[c][n][i][j]. No layout conversion and no
 * allocation (the plan's workspace exists from msc_plan_create); this is the operator
 * alone, as GMRES applies it. x and y may not alias. The reference has one layout
 * only; this is the kernel part of _slab_matvec_gpu (slab_scattering_gpu.py:95-155). */
int msc_matvec_soa(msc_plan* plan, const void* x, void* y, int precision);

/* The same operator as msc_matvec, for callers that cannot allocate device memory
 * when they apply it: a host framework whose allocator owns the device memory and
 * forbids other allocations, or a real-time loop that must not risk an allocation's
 * latency or failure mid-run. msc_matvec allocates two field copies on first use;
 * this call allocates nothing. Its scratch is one static device array of this
 * library, at most 64 MiB, resident on every GPU that loads the library until the
 * process exits. A plan needing more (a workspace of 9*N_z*Ly*Lx complex elements
 * plus two fields of 9*N_z*M*M, each part aligned up to 256 bytes; (Lz, Lx, Ly) from
 * msc_plan_fft_sizes) is rejected with MSC_ERR_INVALID, and so is a call made while
 * another device than the plan's is current. The first call on a device looks the
 * array up with cudaGetSymbolAddress (make it before any stream capture); the address
 * is kept until exit, so the library is not usable across a cudaDeviceReset. All
 * calls share the array: calls whose GPU work overlaps race on it. No counterpart
 * in the reference. */
int msc_matvec_noalloc(msc_plan* plan, const void* x, void* y, int precision);

/* Near-field polynomial preconditioner (an addition of this library; the reference
 * solves unpreconditioned). S_l x = (G_nn + dG_l)(T0 x) with G_nn the 27 nearest-
 * neighbour 9x9 blocks of the slab kernel (self term zero, zero outside the slab)
 * and P = sum_{l=0..L} c_l S_l ... S_1. The default, degree 2 with c = 1, is the
 * truncated Neumann series of (I - G_nn T0)^{-1}. msc_set_nearfield sets the degree
 * L in [1, 6], the coefficients (2(L+1) doubles re/im, NULL = all ones) and
 * per-layer block corrections (L x 27 x 81 complex128 re/im, NULL = none); the
 * settings hold until changed and survive build_g0. Entries that the mirror symmetry
 * of the lattice sets to zero (where the offset has a zero component along an axis,
 * those odd under that axis' reflection) are not applied, corrections included. */
int msc_set_nearfield(msc_plan* plan, int degree, const double* coef, const double* dblocks);
/* The 27 x 9 x 9 blocks G_nn (complex128 re/im into out[2 x 27 x 81]) of the last
 * build_g0; offset o = ((dz+1) 3 + dx+1) 3 + dy+1, out block a,b: y_a += G_ab tau_b(v - o). */
int msc_nearfield_blocks(const msc_plan* plan, double* out);
/* z = P x, fields (N_z, M, M, 9) on the device in the precision given. */
int msc_precondition(msc_plan* plan, const void* x, void* z, int precision);
/* Storage of the layer blocks G_nn + dG_l for the complex64 preconditioner:
 * MSC_NF_WEIGHTS_FP32 (default), MSC_NF_WEIGHTS_BF16 (rounded to bfloat16, FP32
 * accumulation; the form the learned network is trained in) or MSC_NF_WEIGHTS_BF16_TC
 * (BF16 blocks and BF16 activations on the tensor cores, FP32 accumulation in tensor
 * memory). The complex128 path always uses FP64 blocks. */
enum msc_nf_weights { MSC_NF_WEIGHTS_FP32 = 0, MSC_NF_WEIGHTS_BF16 = 1, MSC_NF_WEIGHTS_BF16_TC = 2 };
int msc_set_nearfield_weights(msc_plan* plan, int format);

/* Learned near-field preconditioner: training on the GPU. The network is the
 * polynomial above with learned coefficients c_l and block corrections
 * dG_l = s w_l, s = msc_nearfield_scale(plan) = max |G_nn| (0 before build_g0); the
 * weights w are dimensionless (L x 27 x 81 complex, re/im doubles) and carry over
 * between frequencies. Objective per residual r, the residual of one GMRES step on
 * the preconditioned operator: loss = min_alpha || alpha A P r^ - r^ ||^2
 * = 1 - |<A P r^, r^>|^2 / ||A P r^||^2, r^ = r / ||r||, A = I - G0 T0. Needs the
 * point-propagator kernel without a Bloch phase (MSC_ERR_UNSUPPORTED otherwise).
 * No counterpart in the reference, which solves without a preconditioner. */
double msc_nearfield_scale(const msc_plan* plan);
/* Loss and gradients with respect to conj(c) (gcoef: 2(L+1) doubles) and conj(w)
 * (gw: L x 27 x 81 complex) for one residual r (N_z, M, M, 9) on the device in the
 * precision given; complex64 evaluates with BF16 layer weights. */
int msc_nf_loss_grad(msc_plan* plan, const void* r, int precision, int degree, const double* coef,
                     const double* w, double* loss, double* gcoef, double* gw);
/* `steps` Adam steps (beta 0.9/0.999, eps 1e-8, FP32 master weights, BF16 layer
 * weights) over n_res complex64 residuals r[n_res][N_z][M][M][9] on the device, one
 * residual per step in turn. coef, w are updated in place; adam (2 n_par + 1 doubles,
 * n_par = 2(L+1) + 2 L 27 81: first moments, second moments, step count; zeros to
 * start) carries the optimiser state between calls; losses (steps doubles) may be NULL. */
int msc_nf_train(msc_plan* plan, const void* r, int n_res, int degree, int steps, double lr, double* coef, double* w,
                 double* adam, double* losses);

/* Largest number of right-hand sides of msc_solve_multi and msc_matvec_multi. */
#define MSC_MAX_RHS 64

/* y_r = (I - G0 T0) x_r for nrhs fields at once: x, y (nrhs, 9, N_z, M, M) complex of
 * the given precision in the component-major layout of msc_matvec_soa, one field after
 * the other. Each block of the fused z pass stages its slice of the G0 spectrum once
 * and applies it to the same columns of all nrhs fields, so the spectrum is read once
 * per application instead of once per field. The plan keeps a workspace of nrhs
 * fields (allocated on first use). The reference applies its operator one column at a
 * time (sphere_scattering_fft_gpu.py:199-216); this is the batched form. */
int msc_matvec_multi(msc_plan* plan, int nrhs, const void* x, void* y, int precision);

/* Solve (I - G0 T0) x_r = b_r for nrhs right-hand sides at once; b, x complex128
 * (nrhs, N_z, M, M, 9). Each b_r is scaled to unit norm and the stacked system is
 * solved by one restarted GMRES (mixed precision or FP64 as opts->precision; the near-
 * field preconditioner as opts->preconditioner) whose operator applications are
 * msc_matvec_multi, to a stacked relative residual of tol / sqrt(nrhs), which bounds
 * every right-hand side's relative residual by tol. stats (nrhs entries, may be NULL)
 * gets the shared counters (n_matvec counts multi-RHS applications) with each right-
 * hand side's FP64 residual and status; the return is the worst status. Replaces the
 * loop of one GMRES solve per incident pattern of compute_sphere_foldy_lax_fft_gpu
 * (sphere_scattering_fft_gpu.py:199-216). */
int msc_solve_multi(msc_plan* plan, int nrhs, const void* b, void* x, const msc_solve_opts* opts,
                    msc_solve_stats* stats);

/* Solve (I - G0 T0) x = b; b, x complex128 (N_z, M, M, 9). Restarted GMRES with
 * CGS2 Arnoldi and FP64 Givens/least squares; precision MIXED runs complex64
 * inner solves inside FP64 iterative refinement. Replaces torch_gmres
 * (torch_gmres.py:83-205) and the scipy gmres call (slab_scattering.py:539-552).
 * Non-convergence returns MSC_NOT_CONVERGED with x the best iterate. */
int msc_solve(msc_plan* plan, const void* b, void* x, const msc_solve_opts* opts, msc_solve_stats* stats);

/* One slab of a batch (msc_batch_solve). Inputs are host memory read during the
 * call; outputs are written in place. */
typedef struct msc_batch_item {
  msc_slab_desc desc;      /* geometry, background medium, periodicity, padding */
  const double* dlam;      /* (N_z, M, M) contrasts, host float64 */
  const double* dmu;
  const double* drho;
  double omega;            /* angular frequency */
  double k_hat[3];         /* incidence direction (z, x, y) */
  int32_t wave_type;       /* msc_wave */
  int32_t bloch;           /* periodic only: Bloch-phased fold at the incidence's k_par */
  int32_t volume_averaged; /* 1: volume-averaged nearest-neighbour blocks (reference volume_averaged) */
  int32_t n_orders;        /* orders of the volume-averaged blocks, 0 = 2 (the reference's default) */
  double rpp_p;            /* horizontal slowness at which R_PP is evaluated (the reference's p); < 0: the
                              incidence's slowness for Bloch items, 0 (normal incidence) for the others */
  void* psi;               /* out (may be NULL): (N_z, M, M, 9) complex128, host */
  double rpp[2];           /* out: specular R_PP (re, im) by the Weyl sum of the solution */
  msc_solve_stats stats;   /* out */
  int32_t status;          /* out: msc_status of this item */
  char error[160];         /* out: message of a failed item */
} msc_batch_item;

/* Solve n independent slabs (uneven sizes, frequencies and incidences) on the
 * current device: T0 and G0 builds, incident field, solve with opts, R_PP and the
 * field, per item. `workers` host threads with a stream and a plan cache each run
 * items concurrently (0 = choose by timing the first items at 1, 2 and 4 workers, and
 * autotune the lateral FFT length of aperiodic items whose Lxy is 0, as Lxy = -1 does;
 * the count used is written to *workers_used when not NULL). Returns MSC_OK when
 * every item converged, MSC_NOT_CONVERGED when any item failed or did not converge
 * (its own status and message say which), negative only for errors of the call
 * itself (arguments, streams). Replaces a loop of compute_slab_scattering_gpu calls
 * (slab_scattering_gpu.py:158-256), e.g. the frequency loop of
 * compute_ocean_bottom_reflection (ocean_bottom.py:290-307). */
int msc_batch_solve(msc_batch_item* items, int n, const msc_solve_opts* opts, int workers, int* workers_used);

/* Flags of msc_rpp_periodic. */
#define MSC_RPP_BLOCH 1             /* demodulate the sources by exp(-i k_par.x), k_par the plan's Bloch wavevector */
#define MSC_RPP_PLANE_WAVE_MOMENT 2 /* moment term with |k| = omega/alpha instead of the reference's kz
                                       (the two agree at p = 0; see the reference formula below) */

/* Specular periodic R_PP (host out[2] = re, im) of psi (complex128, device) at
 * horizontal slowness p. flags = 0 is the reference formula.
 * Replaces slab_rpp_periodic (slab_scattering.py:672-735). */
int msc_rpp_periodic(msc_plan* plan, const void* psi, double omega, double p, int flags, double* out);

/* Reflected far-field amplitudes (host out[6] = R_PP, R_PS, R_SP as re, im).
 * Replaces slab_reflected_field (slab_scattering.py:589-669). */
int msc_reflected_field(msc_plan* plan, const void* psi, double omega, const double* k_hat, double* out);

const char* msc_status_string(int status);
/* Message of the last error on this thread. */
const char* msc_last_error(void);
/* Kernel launches issued by this library since it was loaded (all plans, all threads). */
int64_t msc_launch_count(void);
/* Library version string. */
const char* msc_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MSC_H */
