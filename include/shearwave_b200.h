/*
 * shearwave_b200 — C ABI of the B200 (sm_100a) implementation of the
 * pinton-lab/shearwave hot path: the shear_fdtd time loop, the Helmholtz-Hodge
 * force projection with its conjugate-gradient Poisson solve, and the strain
 * post-pass.
 *
 * Conventions shared by every entry point
 * ---------------------------------------
 *  - Every pointer is a DEVICE pointer unless the comment says "host".  The
 *    caller owns all memory (the Python layer allocates it through torch);
 *    the library borrows pointers for the duration of a call and allocates
 *    nothing itself.
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).  Work is
 *    enqueued on it; calls that must read a device-side flag (the CG loop)
 *    synchronise that stream and return when the work is complete.
 *  - `dtype` is SW_F32 or SW_F64.
 *  - Dense arrays are C-ordered (nx, ny, nz[, k]) like the reference's numpy
 *    arrays.  Padded fields use a z pitch pz = sw_pitch(nz) (a multiple of 8)
 *    and hold vector components as separate planes of ncell = nx*ny*pz
 *    elements.  The one-voxel shell of every padded field is zero.
 *  - Every entry point returns SW_OK (0) or an error code; sw_last_error()
 *    gives a message for the last failure on the calling thread.
 *
 * Reference interfaces (paths within pinton-lab/shearwave):
 *  src/shearwave/solver.py:27-243     shear_fdtd             -> sw_fdtd_*
 *  src/shearwave/solver.py:246-566    shear_fdtd_jax extras  -> snaps / traces in sw_fdtd_desc
 *  src/shearwave/solver.py:644-683    project_vector_field   -> sw_project
 *  src/shearwave/solver.py:1010-1050  poisson_cg             -> sw_project (CG stage)
 *  src/shearwave/solver.py:686-729    laplacian/divergence/gradient_center -> sw_laplacian, ...
 *  src/shearwave/solver.py:569-625    elastic_solve_static   -> sw_static_solve
 *  src/shearwave/strain.py:16-135     compute_strain_tensor / _invariants -> sw_strain*
 */
#ifndef SHEARWAVE_B200_H
#define SHEARWAVE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SW_ABI_VERSION 1

enum sw_dtype { SW_F32 = 0, SW_F64 = 1 };

enum sw_status {
  SW_OK = 0,
  SW_EINVAL = 1,      /* bad argument (null pointer, shape, size) */
  SW_ECUDA = 2,       /* a CUDA runtime call or launch failed */
  SW_ENONFINITE = 3,  /* non-finite values detected in the state */
  SW_ERANGE = 4,      /* size above a compiled-in maximum */
  SW_EWORKSPACE = 5,  /* workspace smaller than the *_workspace_bytes query */
  SW_ETIMEOUT = 6     /* a bounded device-side wait ran out, or a step launch refused to
                       * run: the solve's state is incomplete (sw_fdtd_status) */
};

/* Why a CG solve stopped (solver.py:1033-1048 plus the early exit of 672-676). */
enum sw_cg_reason {
  SW_CG_RUNNING = 0,
  SW_CG_CONVERGED = 1,  /* sqrt(r.r / rs0) < tol */
  SW_CG_BREAKDOWN = 2,  /* p.Ap non-finite or <= 0 (x untouched that iteration) */
  SW_CG_NONFINITE = 3,  /* r.r non-finite after the update */
  SW_CG_MAXITERS = 4,   /* max_iters updates done */
  SW_CG_EARLY_EXIT = 5  /* max|div f| < 1e-12: no solve, f returned masked */
};

enum sw_precision {
  SW_PLAIN_F64 = 0, /* FP64 fields, reference arithmetic (the plain drop-in) */
  SW_MIXED_F32 = 1  /* FP32 fields in increment form (u compensated when desc.kahan) */
};

/* ---- library --------------------------------------------------------- */
int sw_abi_version(void);
const char* sw_last_error(void);
/* Make `device` current for this thread's subsequent calls. */
int sw_set_device(int device);
/* Padded z pitch used for padded fields (nz rounded up to a multiple of 8). */
int sw_pitch(int nz);
/* sizeof(sw_fdtd_desc), so a binding can check its mirror of the struct. */
size_t sw_fdtd_desc_size(void);
/* Number of kernels this library has launched in the process so far. */
uint64_t sw_launch_count(void);
/* Number of host-side enqueue calls behind those kernels (a CUDA-graph
 * replay of a segment of the time loop launches many kernels with one). */
uint64_t sw_host_enqueue_count(void);

/* Launch-shape knobs of the step kernels (no counterpart in the reference:
 * the autotuner in shearwave_b200/tune.py sweeps them per workload).  They
 * change how the grid is cut into tiles, never the results.  Process-wide;
 * set them between solves, not while one is running.                      */
enum sw_tune_knob {
  SW_TUNE_STEP_CTAS_PER_SM = 0,    /* step CTAs per SM a launch is sized for: 1 or 2 (2) */
  SW_TUNE_BATCH_TILES_PER_CTA = 1, /* batched launches: tiles per CTA, 1..64 (8)   */
  SW_TUNE_XCHUNK = 2,              /* planes per x chunk, 0 = automatic (0)          */
  SW_TUNE_TILE_SHAPE = 3,          /* mixed step tiles: 0 auto, 1 64-wide, 2 32-wide */
  SW_TUNE_STEPS_PER_PASS = 4,      /* mixed solves whose steps_per_pass is 0: 0 auto (two
                                    * per pass), 1 or 2 steps per pass (0) */
  SW_TUNE_WAIT_BUDGET = 5,         /* step kernels: how long a CTA waits on its pipeline
                                    * (after the first failed test) before it abandons its
                                    * tiles and flags their solves, in units of 1024 cycles,
                                    * 1..4000000 (3906250, about 4e9 cycles) */
  SW_TUNE_COUNT = 6
};
/* SW_EINVAL for an unknown knob or a value out of range. */
int sw_tune_set(int knob, int value);
/* Current value, or -1 for an unknown knob. */
int sw_tune_get(int knob);

/* ---- collocated FD operators on dense arrays (solver.py:686-729) ------- */
/* laplacian_center: interior 7-point Laplacian, zero shell. */
int sw_laplacian(int dtype, const void* f, void* out, int nx, int ny, int nz, double dX,
                 double dY, double dZ, void* stream);
/* divergence_center: interior 2h central divergence, zero shell. */
int sw_divergence(int dtype, const void* fx, const void* fy, const void* fz, void* out, int nx,
                  int ny, int nz, double dX, double dY, double dZ, void* stream);
/* gradient_center: interior 2h central gradient, zero shell. */
int sw_gradient(int dtype, const void* phi, void* gx, void* gy, void* gz, int nx, int ny, int nz,
                double dX, double dY, double dZ, void* stream);

/* ---- Helmholtz-Hodge projection (solver.py:644-683, 1010-1050) --------- */
typedef struct sw_cg_stats {
  int32_t iters;   /* completed CG updates */
  int32_t reason;  /* enum sw_cg_reason */
  double rel;      /* sqrt(r.r / rs0) at exit (NaN when no update ran) */
  double max_div;  /* max |div_c f| of the masked input */
} sw_cg_stats;

/* Bytes of device workspace sw_project needs for an (nx, ny, nz) grid. */
size_t sw_project_workspace_bytes(int nx, int ny, int nz);

/* Project (fx, fy, fz) onto discretely divergence-free fields in FP64.
 * Input: dtype `in_dtype`, element (x, y, z) at x*in_sx + y*in_sy + z*in_sz
 * (elements; dense arrays: ny*nz, nz, 1).  A NULL component is zero.
 * Output: `out` holds 3 padded FP64 components (pitch sw_pitch(nz)).
 * The CG runs in FP64 with the reference's stopping rule; the call returns
 * once the solve has finished (it synchronises `stream`).  `stats` is host. */
int sw_project(int in_dtype, const void* fx, const void* fy, const void* fz, int64_t in_sx,
               int64_t in_sy, int64_t in_sz, int nx, int ny, int nz, double dX, double dY,
               double dZ, double tol, int max_iters, double* out, void* workspace,
               size_t workspace_bytes, sw_cg_stats* stats, void* stream);

/* Bytes of device workspace sw_project_spectral needs for an (nx, ny, nz) grid. */
size_t sw_project_spectral_workspace_bytes(int nx, int ny, int nz);

/* The same projection with the Poisson problem solved directly instead of by
 * CG: A = -div_c(grad_c) is separable into per-axis operators whose
 * eigenvectors are discrete sine / cosine bases, so phi is three forward
 * per-axis transforms, a division by the eigenvalue sums and three inverse
 * transforms, in FP64.  Gives the exact (minimum-norm) solution the
 * reference's CG approaches as tol -> 0; keeps the max|div| < 1e-12 early
 * exit.  stats->iters is 0. */
int sw_project_spectral(int in_dtype, const void* fx, const void* fy, const void* fz,
                        int64_t in_sx, int64_t in_sy, int64_t in_sz, int nx, int ny, int nz,
                        double dX, double dY, double dZ, double* out, void* workspace,
                        size_t workspace_bytes, sw_cg_stats* stats, void* stream);

/* Host helper: the orthonormal basis Q (m x m row-major, m = n - 2) and the
 * eigenvalues lam (m) of one axis' 1-D operator for n grid points of
 * spacing h (host buffers). */
int sw_spectral_basis(int n, double h, double* Q, double* lam);

/* One solve of a batched projection (fields as for sw_project). */
typedef struct sw_project_job {
  int32_t in_dtype;
  const void* fx;
  const void* fy;
  const void* fz;
  int64_t sx, sy, sz;
  int32_t nx, ny, nz;
  double dX, dY, dZ, tol;
  int32_t max_iters;
  double* out;            /* 3 padded FP64 components */
  void* workspace;        /* sw_project_workspace_bytes(nx, ny, nz) bytes */
  size_t workspace_bytes;
} sw_project_job;

/* Device bytes of the instance table sw_project_batch needs for n jobs. */
size_t sw_project_batch_table_bytes(int n);

/* Project n independent fields together: every CG launch advances all
 * unfinished solves (same dtype for all jobs); each solve keeps its own
 * stopping rule and iteration count.  `stats` (host) receives n entries. */
int sw_project_batch(const sw_project_job* jobs, int n, void* table, size_t table_bytes,
                     sw_cg_stats* stats, void* stream);

/* sw_project for callers that cannot allocate device memory.  No counterpart
 * in the reference: it exists for hosts that give the library nothing but
 * their own input and output buffers (applications whose device memory is
 * reserved up front by their own pool or budget and may not grow, bindings
 * with no way to allocate a device workspace).  Same arguments, solve and
 * results as sw_project, without the workspace: the CG scratch is a fixed
 * array of sw_project_noalloc_scratch_bytes() (32 MiB) compiled into the
 * library, resident on every GPU that loads it until the process exits.
 * Grids whose scratch would not fit (more than about 0.7 million padded
 * cells) are rejected with SW_ERANGE.  The array's device address is looked
 * up on the first call made on each device, so make that first call before
 * any stream capture.  Every call shares the array: calls whose work
 * overlaps on the GPU (e.g. on two streams) race and corrupt each other.
 * Nothing is allocated: no cudaMalloc, no cudaFree, no heap. */
size_t sw_project_noalloc_scratch_bytes(void);
int sw_project_noalloc(int in_dtype, const void* fx, const void* fy, const void* fz,
                       int64_t in_sx, int64_t in_sy, int64_t in_sz, int nx, int ny, int nz,
                       double dX, double dY, double dZ, double tol, int max_iters, double* out,
                       sw_cg_stats* stats, void* stream);

/* dst = src * scale / rho (rho NULL: dst = src * scale) for `ncomp` padded FP64
 * components into `dst` (dtype out_dtype, element (x,y,z) of component c at
 * c*dst_cs + x*dst_sx + y*dst_sy + z*dst_sz).  rho is dense or strided like
 * the input of sw_project (rho_sx, rho_sy, rho_sz). */
int sw_convert(int ncomp, const double* src, int nx, int ny, int nz, int out_dtype, void* dst,
               int64_t dst_cs, int64_t dst_sx, int64_t dst_sy, int64_t dst_sz, double scale,
               int rho_dtype, const void* rho, int64_t rho_sx, int64_t rho_sy, int64_t rho_sz,
               void* stream);

/* ---- static elastic solve (solver.py:569-625) ---------------------------- */
/* CG on (-mu L7) u = b with zero shell, in FP64, with the reference's loop
 * (break on p.Ap <= 0, stop at sqrt(r.r / rs0) < tol).  b and mu (NULL: the
 * scalar mu_s) are `dtype` arrays with element strides (sx, sy, sz); u is
 * written to `out` as one padded FP64 field.  Workspace: as sw_project. */
int sw_static_solve(int dtype, const void* b, const void* mu, double mu_s, int64_t sx,
                    int64_t sy, int64_t sz, int nx, int ny, int nz, double dX, double dY,
                    double dZ, double tol, int max_iters, double* out, void* workspace,
                    size_t workspace_bytes, sw_cg_stats* stats, void* stream);

/* ---- time loop (solver.py:27-243) --------------------------------------- */
typedef struct sw_fdtd_desc {
  int32_t precision;       /* enum sw_precision */
  int32_t nx, ny, nz, pz;  /* pz must equal sw_pitch(nz) */
  int32_t n_steps;         /* total steps of the solve (term table length) */
  double dX, dY, dZ, dT, vel_damp;
  /* SW_PLAIN_F64: state[0..2] are three rotating FP64 buffers of 3 padded
   *   components (u_prev, u_curr, u_next).
   * SW_MIXED_F32: state[0..2] are three FP32 buffers of 9 padded
   *   components (u, d = u - u_prev, Kahan compensation c); the state after
   *   t steps is in buffer t mod 3 (a kernel fusing two steps reads one
   *   buffer and writes another). */
  void* state[3];
  /* Material coefficients, padded, written by sw_fdtd_materials:
   *   F64: coef_m = mu/rho, coef_e = eta/rho (NULL: no viscosity), inv_rho = 1/rho.
   *   F32: coef_m = dT^2 mu/rho, coef_e = dT eta/rho (NULL: none), inv_rho unused.
   * The TMA kernels (kernel == 0) need coef_e == coef_m + ncell elements. */
  void* coef_m;
  void* coef_e;
  void* inv_rho;
  /* Projected force patterns, n_patterns x 3 padded components:
   *   F64: f_S;  F32: dT^2 f_S / rho. */
  const void* patterns;
  int32_t n_patterns;
  /* Force terms of step it: j in [term_off[it], term_off[it+1]) adds
   * term_scale[j] * patterns[term_pat[j]] (term_off has n_steps+1 entries). */
  const int32_t* term_off;
  const int32_t* term_pat;
  const double* term_scale;
  int32_t kahan;          /* F32: 1 = compensated u update */
  int32_t snap_stride;    /* > 0: write u after every snap_stride steps */
  void* snaps;            /* dense (n_steps/snap_stride, nx, ny, nz, 3) of the field dtype */
  int32_t n_traces;       /* > 0: record u_z at trace cells every step */
  const int32_t* trace_cells; /* n_traces x (ix, iy, iz) */
  void* traces;           /* dense (n_traces, n_steps) of the field dtype */
  int32_t* flags;         /* device int: bit 0 a non-finite u (set by sw_fdtd_finish), bit 1 a
                           * step kernel's bounded wait ran out, bit 2 a step launch refused
                           * to run; a solve with bit 1 or 2 set is skipped by later step
                           * launches (may be NULL) */
  int32_t xchunk;         /* planes per tile along x (0 = automatic) */
  int32_t steps_per_pass; /* F32: 2 = two steps per pass over HBM where two remain and the
                           * compensated sum is off; 1 = one step per pass; 0 (automatic) =
                           * two */
  int32_t kernel;         /* 0: TMA-staged step kernels (default), 1: direct-load kernels */
  /* Device int the step loop may use as its step counter: with it, long runs
   * of sw_fdtd_steps replay one instantiated CUDA graph of 32 steps instead
   * of launching every step (NULL: direct launches only). */
  int32_t* clock;
  /* Two device int32s, zero at the first call (the kernels leave them zero):
   * the launch-wide tile queue of this solve's own step launches, which
   * balances tiles over the SMs (NULL: tiles in a fixed stride). */
  int32_t* queue;
  /* Testing switch (0 in normal use): non-zero makes the TMA step kernels
   * leave the first ring stage of each of this solve's tiles unarmed, so
   * that the consumers' bounded waits run out (nothing faults or hangs: the
   * CTA drains its copies, flags the solve and returns).  Lets a test drive
   * the timeout path of sw_fdtd_status. */
  int32_t stall_test;
} sw_fdtd_desc;

/* Material coefficients from rho, mu, eta.  Each of rho/mu/eta is a dense
 * (nx,ny,nz) array of `in_dtype`, or NULL to use the scalar.  eta_mode: 0 no
 * viscosity, 1 use eta/eta_s. */
int sw_fdtd_materials(const sw_fdtd_desc* d, int in_dtype, const void* rho, double rho_s,
                      const void* mu, double mu_s, int eta_mode, const void* eta, double eta_s,
                      void* stream);

/* Initial state from initial_u / initial_v (dense (nx,ny,nz,3) of the field
 * dtype, or NULL for zero), solver.py:157-171.  Zeroes all state buffers. */
int sw_fdtd_init(const sw_fdtd_desc* d, const void* init_u, const void* init_v, void* stream);

/* Advance steps it0 .. it0+nsteps-1 (0-based step indices). */
int sw_fdtd_steps(const sw_fdtd_desc* d, int32_t it0, int32_t nsteps, void* stream);

/* Write u and v = (u_curr - u_prev)/dT after `steps_done` steps as dense
 * (nx,ny,nz,3) arrays of the field dtype (either may be NULL). */
int sw_fdtd_finish(const sw_fdtd_desc* d, int32_t steps_done, void* u_out, void* v_out,
                   void* stream);

/* Status of a solve after its steps: synchronises `stream`, copies the
 * solve's device flag word into *host_flags (may be NULL) and returns
 * SW_ETIMEOUT when a step kernel abandoned any of the solve's tiles (a
 * bounded wait ran out, or a launch refused a misaligned TMA destination),
 * SW_ENONFINITE when sw_fdtd_finish found a non-finite u, else SW_OK.
 * Flag bits: 1 non-finite, 2 wait timeout, 4 refused launch.  The
 * reference's time loop has no such check (solver.py:194-239). */
int sw_fdtd_status(const sw_fdtd_desc* d, int32_t* host_flags, void* stream);

/* Device bytes of the instance table sw_fdtd_batch_steps needs for n solves. */
size_t sw_fdtd_batch_table_bytes(int n);

/* Advance a batch of independent solves (same precision, TMA kernels, no
 * traces).  Solve i runs its local step it - begins[i] at global step it
 * when 0 <= it - begins[i] < n_steps (begins NULL: all start at 0).  One
 * launch per global step covers the tiles of every running solve, so small
 * and large grids share the GPU.  `table`: 64-byte aligned device memory of
 * sw_fdtd_batch_table_bytes(n) bytes. */
int sw_fdtd_batch_steps(const sw_fdtd_desc* descs, const int32_t* begins, int n, int32_t it0,
                        int32_t nsteps, void* table, size_t table_bytes, void* stream);

/* Project the state in place after `steps_done` steps (reproject_every,
 * solver.py:236-239): u_curr and u_prev each go through sw_project. */
int sw_fdtd_reproject(const sw_fdtd_desc* d, int32_t steps_done, double tol, int max_iters,
                      double* tmp, void* workspace, size_t workspace_bytes, sw_cg_stats* stats,
                      void* stream);

/* ---- strain post-pass (strain.py:16-135) -------------------------------- */
/* From displacement components (element (x,y,z) at x*sx + y*sy + z*sz) write
 * any of: eps (dense (nx,ny,nz,6) Voigt, engineering shear), volumetric,
 * deviatoric, max_shear (dense, dtype) and von_mises (dense, always FP64). */
int sw_strain(int dtype, const void* ux, const void* uy, const void* uz, int64_t sx, int64_t sy,
              int64_t sz, int nx, int ny, int nz, double dX, double dY, double dZ, void* eps,
              void* vol, void* dev, void* max_shear, double* von_mises, void* stream);

/* Invariants of n Voigt 6-vectors (dense (n, 6) of dtype). */
int sw_strain_invariants(int dtype, const void* eps, int64_t n, void* vol, void* dev,
                         void* max_shear, double* von_mises, void* stream);

/* ---- acoustic radiation force (radiation_force.py:27-157) ------------- */
/* Inputs are the reference's (nx, ny, nz, nt) records, time fastest: cell k's
 * series is p[k*nt .. k*nt+nt-1]; ncell = nx*ny*nz.                        */
/* Workspace of sw_arf_envelope (FP64 per-block partial sums). */
size_t sw_arf_workspace_bytes(int64_t ncell, int32_t nt);
/* Auto-gate envelope (radiation_force.py:63-68): env[t] = mean over cells of
 * p[., t]^2, accumulated in FP64 in a fixed order; env is nt doubles on the
 * device.  The caller thresholds it (>= 0.1 max) to pick the gate.         */
int sw_arf_envelope(int dtype, const void* p, int64_t ncell, int32_t nt, double* env,
                    void* workspace, size_t workspace_bytes, void* stream);
/* Radiation force over the gated time indices gate[0..n_gate) (each in
 * [0, nt); indices outside are skipped).  n_fields 1:
 * compute_radiation_force (radiation_force.py:71-85),
 *   out0 = 2 alpha_Np (mean p^2 / (rho c)) / c;
 * n_fields 3: compute_radiation_force_velocity (radiation_force.py:141-157),
 *   out_i = (2 alpha_Np / c) mean(p v_i) with v = (vx, vy, vz);
 * alpha_Np = alpha * (f0 / 1e6) / 8.685889638 * 100.  Maps are FP64 per cell
 * (map_stride 1) or one value for every cell (map_stride 0); outputs are
 * ncell values of out_dtype.  Sums run in FP64.                             */
int sw_arf_force(int dtype, int n_fields, const void* p, const void* vx, const void* vy,
                 const void* vz, int64_t ncell, int32_t nt, const int32_t* gate, int32_t n_gate,
                 const double* c_map, const double* rho_map, const double* alpha_map,
                 int64_t map_stride, double f0, int out_dtype, void* out0, void* out1,
                 void* out2, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SHEARWAVE_B200_H */
