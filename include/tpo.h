/*
 * tpo.h -- C ABI of libtpo, the sm_100a kernels behind the SIMP
 * compliance-minimisation loop of tomohiron907/toptimization.
 *
 * Plain C types only (pointers, sizes, PODs); no torch types. Every function
 * returns a tpo_status code, is asynchronous on the given stream unless noted,
 * never allocates or frees caller buffers, and takes device pointers that the
 * caller owns (PyTorch tensors in the Python host). Scratch comes from a
 * caller-provided workspace whose size the matching *_workspace_bytes query
 * returns; workspaces must be 256-byte aligned and not shared between calls
 * that may run concurrently.
 *
 * Layouts (2D structured Q4 grid, nelx x nely unit elements):
 *   node (ix, iy)          -> ix*(nely+1) + iy            (iy fastest)
 *   nodal vector  v        -> v[2*node + {0:x, 1:y}]     (2*(nelx+1)*(nely+1))
 *   element (ex, ey)       -> ex*nely + ey                (nelx*nely)
 *   fixed mask             -> uint8 per node, bit0 = x fixed, bit1 = y fixed
 * These are the reference's numbering (src/toptimization/mesh.py:1-24,
 * src/toptimization/problem.py:167-173); the fixed mask replaces its int32
 * per-DOF `is_fixed` field (src/toptimization/fem/fields.py:146-148).
 */
#ifndef TPO_H
#define TPO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void *tpo_stream; /* a cudaStream_t; NULL = legacy default stream */

typedef enum tpo_status {
  TPO_OK = 0,
  TPO_ERR_ARGS = 1,          /* bad sizes, null or misaligned pointers */
  TPO_ERR_CUDA = 2,          /* a CUDA call failed; see tpo_last_error_string */
  TPO_ERR_NOT_CONVERGED = 3, /* not returned by solves: see tpo_solve_result */
  TPO_ERR_BREAKDOWN = 4,
  TPO_ERR_NONFINITE = 5,
  TPO_ERR_TIMEOUT = 6,
  TPO_ERR_NO_STIFFNESS = 7,  /* tpo_set_stiffness not called on this device */
  TPO_ERR_WORKSPACE = 8      /* workspace smaller than the query returned */
} tpo_status;

/* Solve outcome codes (tpo_solve_result.status). */
enum {
  TPO_SOLVE_RUNNING = 0,
  TPO_SOLVE_CONVERGED = 1,
  TPO_SOLVE_MAX_ITER = 2,
  TPO_SOLVE_BREAKDOWN = 3,   /* |p.Ap| < 1e-30 (reference solver.py:114-115) */
  TPO_SOLVE_NONFINITE = 4,
  TPO_SOLVE_ZERO_RHS = 5,    /* ||f|| < 1e-30: u = 0 (reference solver.py:61-63) */
  TPO_SOLVE_TIMEOUT = 7,     /* tpo_pcg_solve_async: a bounded pipeline wait ran out */
  TPO_SOLVE_LOOP_LIMIT = 8   /* tpo_pcg_solve_async: the device loop reached its body
                                limit with the solve still running */
};

/* Preconditioners. */
enum {
  TPO_PRECOND_NONE = 0,
  TPO_PRECOND_JACOBI = 1,       /* reference "jacobi" (kernels.py:65-101) */
  TPO_PRECOND_BLOCK_JACOBI = 2, /* reference "block_jacobi": element-block form
                                   (fem/preconditioner.py:47-108) */
  TPO_PRECOND_NODAL_BLOCK = 3   /* 2x2 nodal block-Jacobi; no reference counterpart */
};

/* Solve precisions. */
enum {
  TPO_PRECISION_FP64 = 0,  /* plain FP64 PCG */
  TPO_PRECISION_MIXED = 1  /* FP32 inner PCG inside FP64 iterative refinement */
};

/* PCG recurrence. AUTO: one launch per iteration (Chronopoulos-Gear form,
 * one global reduction) for the plain FP64 solve with a point preconditioner
 * (none, Jacobi, nodal block); two launches otherwise (element-block
 * preconditioner, mixed form). STANDARD: the reference's own recurrence
 * (fem/solver.py:27-159), two launches per iteration. SINGLE: the one-launch
 * form; TPO_ERR_ARGS for the element-block preconditioner or the mixed form
 * (its s = K p recurrence is not kept accurately in FP32 storage). Both forms
 * give the same iterates in exact arithmetic and use the reference's stop,
 * breakdown and beta rules. */
enum {
  TPO_RECURRENCE_AUTO = 0,
  TPO_RECURRENCE_STANDARD = 1,
  TPO_RECURRENCE_SINGLE = 2
};

typedef struct tpo_grid {
  int32_t nelx, nely;
  double e_min;    /* SIMP floor: scale = e_min + rho^penalty (1 - e_min) */
  double penalty;  /* (reference fem/kernels.py:92,160) */
} tpo_grid;

typedef struct tpo_solve_cfg {
  int32_t precond;      /* TPO_PRECOND_* */
  int32_t precision;    /* TPO_PRECISION_* */
  int32_t max_iter;     /* FP64: PCG iterations; mixed: inner iterations per solve */
  int32_t warm_start;   /* nonzero: start from u as passed (fixed DOFs zeroed) */
  double tol;           /* stop when ||r||^2 < (tol*||f||)^2 */
  double f_norm_sq;     /* ||f||^2, computed once by the caller */
  double inner_tol;     /* mixed: relative tolerance of each inner solve */
  int32_t max_outer;    /* mixed: refinement steps */
  int32_t poll_every;   /* iterations between host checks of the device status
                           (0 = library default); no effect on results */
  int32_t recurrence;   /* TPO_RECURRENCE_*: how an iteration is organised */
} tpo_solve_cfg;

typedef struct tpo_solve_result {
  int32_t status;       /* TPO_SOLVE_* */
  int32_t iters;        /* the reference's count: it+1 on convergence, max_iter
                           otherwise (also after a breakdown), 0 for zero rhs;
                           mixed: total inner iterations */
  int32_t outer_iters;  /* mixed: refinement steps taken (FP64: 1) */
  int32_t updates;      /* PCG updates actually performed */
  double rr;            /* last ||r||^2 seen (mixed: true FP64 residual) */
  int32_t launches;     /* kernels the solve ran (tpo_pcg_solve_async: each loop
                           body's kernels counted every time the body ran) */
  int32_t bodies;       /* tpo_pcg_solve_async: device loop bodies run (else 0) */
} tpo_solve_result;

int tpo_version(void);
const char *tpo_last_error_string(void);

/* Failure tests only; no counterpart in the reference. The next stencil
 * launch of this process withholds the bulk copies of its column group
 * `group` (in every CTA), so that the bounded waits for it run out (about
 * 1.3 s each): the kernel sets its error flag, lets its other copies land
 * and returns, and the solve reports TPO_ERR_TIMEOUT (tpo_pcg_solve) or
 * TPO_SOLVE_TIMEOUT (tpo_pcg_solve_async). The device stays usable. */
int tpo_test_withhold_stage(int32_t group);

/* Element stiffness (8x8 Q4, row-major), its regularised inverse and the
 * regulariser (reference fem/fields.py:133-143), copied to constant memory of
 * the CURRENT device. Must be called once per device before any kernel. */
int tpo_set_stiffness(const double ke[64], const double ke_inv[64], double alpha_reg);

/* ---- matrix-free K(rho) p --------------------------------------------------
 * ap = K(rho) p with identity rows at fixed DOFs; *pap_out (device, nullable)
 * = p.ap. Replaces compute_matvec_2d / matvec_and_dot_2d
 * (reference fem/kernels.py:143-176, fem/fused_kernels.py:21-56). */
size_t tpo_matvec_workspace_bytes(const tpo_grid *g);
int tpo_matvec_f64(const tpo_grid *g, const double *rho, const uint8_t *fixed,
                   const double *p, double *ap, double *pap_out,
                   void *ws, size_t ws_bytes, tpo_stream s);
int tpo_matvec_f32(const tpo_grid *g, const float *rho, const uint8_t *fixed,
                   const float *p, float *ap, double *pap_out,
                   void *ws, size_t ws_bytes, tpo_stream s);

/* Same operator with the SIMP scales already computed (scale[e] =
 * e_min + rho_e^p (1 - e_min)): the matvec the PCG applies every iteration. */
int tpo_apply_stiffness_f64(const tpo_grid *g, const double *scale, const uint8_t *fixed,
                            const double *p, double *ap, double *pap_out,
                            void *ws, size_t ws_bytes, tpo_stream s);
int tpo_apply_stiffness_f32(const tpo_grid *g, const float *scale, const uint8_t *fixed,
                            const float *p, float *ap, double *pap_out,
                            void *ws, size_t ws_bytes, tpo_stream s);

/* ---- PCG solve K(rho) u = f ------------------------------------------------
 * Replaces fem/solver.py:27-159 (host loop + fused kernels) with a
 * device-resident PCG: alpha/beta/convergence are decided on the GPU; the host
 * only polls a status word every cfg->poll_every iterations. BLOCKING: returns
 * when the solve has finished on the device. u holds the warm start on entry
 * and the solution on exit (the reference's u_prev/u pair). */
size_t tpo_pcg_workspace_bytes(const tpo_grid *g, const tpo_solve_cfg *c);
int tpo_pcg_solve(const tpo_grid *g, const tpo_solve_cfg *c,
                  const double *rho_phys, const double *f, const uint8_t *fixed,
                  double *u, void *ws, size_t ws_bytes,
                  tpo_solve_result *out, tpo_stream s);

/* The same solve, asynchronous on the stream (replaces the host loop of the
 * reference's fem/solver.py:107-156): no host synchronisation; the PCG loop
 * runs on the device as a CUDA graph conditional WHILE node (bodies of 16
 * iterations, the stop, breakdown and refinement rules decided by the
 * kernels, a bound on the number of bodies), and the result is written to
 * `out_dev`, DEVICE memory (8-byte aligned), when the solve has finished.
 * Same kernels in the same order as tpo_pcg_solve, so the same results.
 * If `s` is capturing, the solve's nodes are added to that capture (so a
 * whole OC iteration can be one graph); otherwise the call captures them
 * itself and launches the graph once. Make one call (or tpo_pcg_solve) on a
 * device before capturing: launch plans are set up on first use. ws, u and
 * out_dev must stay valid until the stream reaches the end of the solve.
 * Errors found while enqueueing are returned; a pipeline wait that runs out
 * shows as TPO_SOLVE_TIMEOUT in out_dev->status. */
int tpo_pcg_solve_async(const tpo_grid *g, const tpo_solve_cfg *c,
                        const double *rho_phys, const double *f, const uint8_t *fixed,
                        double *u, void *ws, size_t ws_bytes,
                        tpo_solve_result *out_dev, tpo_stream s);

/* ---- compliance and sensitivity --------------------------------------------
 * dc[e] = -p rho^(p-1) (1-e_min) u_e^T Ke u_e; *compliance_out (device) =
 * sum_e scale_e u_e^T Ke u_e. Replaces compute_sensitivity_2d
 * (reference fem/kernels.py:234-272). */
size_t tpo_sensitivity_workspace_bytes(const tpo_grid *g);
int tpo_sensitivity(const tpo_grid *g, const double *rho_phys, const double *u,
                    double *dc, double *compliance_out,
                    void *ws, size_t ws_bytes, tpo_stream s);

/* Same computation with no workspace argument and no allocation anywhere:
 * for callers that cannot allocate device memory themselves -- for example a
 * host whose framework reserves the whole device memory budget up front in
 * its own pool (a separate cudaMalloc there can fail or fragment the pool),
 * or a foreign-language binding that only receives finished device buffers
 * and has no allocator to create a workspace with. No counterpart in the
 * reference.
 * Scratch lives in one file-scope device array of TPO_SENS_NOALLOC_SCRATCH
 * bytes inside libtpo, present on every device that loads the library until
 * the process exits. Limit: ceil(nely/128) * ceil(nelx/16) <= 32736 (about
 * 67 million elements); larger grids return TPO_ERR_ARGS. The first call on
 * a device looks up the array's device address (once per device, with that
 * device current); make that first call before any stream capture. Every
 * call reuses the same array, so calls that may overlap on the GPU (other
 * streams, other threads) race with each other: serialise them. */
#define TPO_SENS_NOALLOC_SCRATCH (256 * 1024)
int tpo_sensitivity_noalloc(const tpo_grid *g, const double *rho_phys, const double *u,
                            double *dc, double *compliance_out, tpo_stream s);

/* ---- hat-weight filters ----------------------------------------------------
 * out[e] = sum_j w_ej x_j / (sum_j w_ej + 1e-20), w = max(0, rmin - dist)
 * over the in-domain box |dx|,|dy| <= ceil(rmin). Used for both the density
 * filter and the dc projection (reference optimizer/filter.py:22-149).
 * scale_out / scale32_out (nullable): SIMP scale of out, FP64 / FP32.
 * Supports ceil(rmin) <= 16. */
int tpo_density_filter(const tpo_grid *g, double rmin, const double *x, double *out,
                       double *scale_out, float *scale32_out, tpo_stream s);
/* out[e] = sum_j w rho_j dc_j / (rho_e sum_j w + 1e-20)
 * (reference optimizer/filter.py:152-171). */
int tpo_sensitivity_filter(const tpo_grid *g, double rmin, const double *rho,
                           const double *dc, double *out, tpo_stream s);

/* ---- OC update -------------------------------------------------------------
 * Bisection on lambda in [0, 1e9] (<= 50 steps, stop when
 * (hi-lo)/(hi+lo+1e-30) < 1e-4), all steps on the device; rho_out = the
 * update at the last midpoint evaluated (may alias rho_in). result_out
 * (device, 4 doubles) = {max change, mean(rho_out), last lambda, steps}.
 * dv may be NULL (all ones). Replaces optimizer/oc.py:21-93 and
 * fem/kernels.py:330-336. */
size_t tpo_oc_workspace_bytes(const tpo_grid *g);
int tpo_oc_update(const tpo_grid *g, double volfrac, double move,
                  const double *rho_in, const double *dc, const double *dv,
                  double *rho_out, double *result_out,
                  void *ws, size_t ws_bytes, tpo_stream s);

/* ---- kernel timing (diagnostics) ------------------------------------------
 * When enabled, tpo_pcg_solve brackets every PCG kernel launch with CUDA
 * events and accumulates the device time of the launches that did work
 * (replaces the host timers of the reference's checker/profile_bottleneck.py).
 * Adds two event records per launch; off by default. */
typedef struct tpo_profile {
  int64_t dir_launches;     /* direction + matvec kernel */
  double dir_ms;
  int64_t update_launches;  /* update + preconditioner kernel */
  double update_ms;
  int64_t dir_bytes;        /* algorithmic bytes moved by those launches */
  int64_t update_bytes;
  int64_t launches;         /* every libtpo kernel launch since the last reset
                               (counted whether or not timing is enabled) */
  int64_t apply_launches;   /* stiffness kernel of tpo_matvec_* / tpo_apply_stiffness_* */
  double apply_ms;
  int64_t apply_bytes;
  int64_t step_launches;    /* one-launch PCG iteration kernel (TPO_RECURRENCE_SINGLE) */
  double step_ms;
  int64_t step_bytes;
} tpo_profile;
int tpo_profile_enable(int on);
int tpo_profile_reset(void);
int tpo_profile_read(tpo_profile *out);

/* ---- batched designs -------------------------------------------------------
 * Many independent designs (uneven sizes) advance together: every kernel step
 * of an OC iteration (filter, scales, PCG, sensitivity, OC bisection) is ONE
 * launch over all active designs, each design's CTAs found through a job
 * table. No reference counterpart: the reference runs one problem per process
 * (optimizer/simp.py:19-312, module-global Taichi fields in fem/fields.py).
 * The per-design work is that of one OC iteration of the reference loop with
 * the mixed-precision PCG and the density filter; a design's launch geometry
 * depends only on its own size and the batch's strip lengths, so its results
 * do not depend on which other designs share the batch.
 * Memory: the library allocates no device memory. The caller gives a batch
 * workspace (tpo_batch_workspace_bytes) and, per design, a design workspace
 * (tpo_batch_design_workspace_bytes) that holds that design's resident state
 * until it is removed. Host bookkeeping lives in the opaque tpo_batch. */
typedef struct tpo_batch tpo_batch;

typedef struct tpo_batch_cfg {
  int32_t precond;       /* TPO_PRECOND_NONE / JACOBI / NODAL_BLOCK */
  int32_t precision;     /* TPO_PRECISION_MIXED */
  int32_t use_graph;     /* nonzero: each OC iteration is one CUDA graph launch (a while
                            node runs the PCG loop on the device); 0: host-polled loop */
  int32_t stencil_cols;  /* columns per CTA of the stencil kernels (0: default 16) */
  int32_t update_cols;   /* nodes per thread of the update kernel (0: default 8) */
  int32_t round_steps;   /* PCG steps per round of tpo_batch_round (0: default 32) */
} tpo_batch_cfg;

typedef struct tpo_batch_design {
  int32_t nelx, nely;
  double e_min, penalty;
  double volfrac, move;  /* OC (reference optimizer/oc.py:21-93) */
  double rmin;           /* density filter radius, <= 16 */
  double tol;            /* stop when it > 5 and change < tol (0: run max_oc_iter) */
  double cg_tol;         /* FP64 residual stop ||f - K u|| < cg_tol ||f|| */
  double inner_tol;      /* residual replacement when the FP32 residual drops by this */
  double f_norm_sq;      /* ||f||^2 */
  double rho0;           /* initial uniform density */
  int32_t max_oc_iter;   /* OC iterations to run */
  int32_t max_cg_iter;   /* PCG iterations per solve */
  int32_t max_outer;     /* FP64 residual evaluations per solve */
  int32_t pad;
} tpo_batch_design;

/* byte offsets, inside a design workspace, of the caller-visible fields:
 * rho (design density, nelx*nely, element ex*nely+ey), rho_phys (filtered),
 * u (displacement, 2*(nelx+1)*(nely+1), reference DOF numbering) and hist
 * (max_oc_iter rows of 6 doubles: compliance, volume, change, PCG iterations,
 * FP64 residual evaluations, PCG status). All FP64. */
typedef struct tpo_batch_layout {
  size_t rho, rho_phys, u, hist;
} tpo_batch_layout;

size_t tpo_batch_workspace_bytes(int32_t max_designs);
size_t tpo_batch_design_workspace_bytes(const tpo_batch_design *d, tpo_batch_layout *layout);
int tpo_batch_create(int32_t max_designs, const tpo_batch_cfg *cfg, void *ws, size_t ws_bytes,
                     tpo_batch **out);
int tpo_batch_destroy(tpo_batch *b);
/* Admits a design (f: its load vector, fixed: its per-node fixed mask, both
 * device arrays in reference numbering, read during the call only). Blocks
 * on the stream. */
int tpo_batch_add(tpo_batch *b, const tpo_batch_design *d, const double *f, const uint8_t *fixed,
                  void *design_ws, size_t design_ws_bytes, tpo_stream s, int32_t *slot_out);
/* Releases a slot (its workspace may be reused once this returns). */
int tpo_batch_remove(tpo_batch *b, int32_t slot);
/* The design in `slot` takes only the PCG steps i of each loop body with
 * i % period == 0 (default 1: every step). The design computes the same
 * iterates, only spread over more loop bodies; a server gives large designs
 * a longer period so that a loop body of small ones does not wait on them.
 * Synchronous; takes effect from the next launch. No reference counterpart. */
int tpo_batch_set_step_period(tpo_batch *b, int32_t slot, int32_t period);
int tpo_batch_set_tiles(tpo_batch *b, int32_t stencil_cols, int32_t update_cols);
/* One OC iteration of every active design; blocks until it is done. With
 * use_graph the iteration is one CUDA graph launch. */
int tpo_batch_oc_iteration(tpo_batch *b, tpo_stream s);
/* `rounds` rounds of continuous batching, then one status read. In a round,
 * designs about to start an OC iteration start it, every design inside its
 * PCG solve advances by one loop body (one FP64 residual check and
 * round_steps PCG steps), and designs whose solve stopped finish their OC
 * iteration. Designs at different OC iterations share every launch; none
 * waits for another's solve. Blocks until done. */
int tpo_batch_round(tpo_batch *b, int32_t rounds, tpo_stream s);
/* Per slot 0..n-1: OC iterations done (-1: empty slot) and whether more remain. */
int tpo_batch_states(tpo_batch *b, int32_t n, int32_t *it_out, int32_t *active_out);
/* Device time of `steps` PCG steps with the current tiles (for the autotuner;
 * advances the designs' PCG state, so use a scratch batch). */
int tpo_batch_time_steps(tpo_batch *b, int32_t steps, tpo_stream s, float *ms_out);

/* ---- 3D: trilinear hexahedra (H8) ------------------------------------------
 * Structured nelx x nely x nelz grid of unit cubes in the reference's
 * numbering (src/toptimization/mesh.py:68-112), used as it is (no padding):
 *   node (ix, iy, iz)    -> (ix*(nely+1) + iy)*(nelz+1) + iz   (iz fastest)
 *   nodal vector v       -> v[3*node + {0:x, 1:y, 2:z}]       (3*(nelx+1)(nely+1)(nelz+1))
 *   element (ex, ey, ez) -> (ex*nely + ey)*nelz + ez
 *   fixed mask           -> uint8 per node, bit0/1/2 = x/y/z fixed
 * FP64 throughout; nodal vectors need 8-byte alignment. The reference runs
 * these through the same entry points as 2D with dim == 3 (fem/kernels.py
 * compute_*_3d, fem/fused_kernels.py:59-94, fem/preconditioner.py:112-156,
 * optimizer/filter.py:75-97); here they are separate functions. */
typedef struct tpo_grid3 {
  int32_t nelx, nely, nelz, pad;
  double e_min;    /* scale = e_min + rho^penalty (1 - e_min) */
  double penalty;
} tpo_grid3;

/* 24x24 H8 stiffness (row-major, DOFs [x,y,z] per corner in mesh.py:87-96
 * order), its regularised inverse (Ke + alpha I)^-1 and alpha (reference
 * material.py:89-171, fem/fields.py:133-143), into constant memory of the
 * CURRENT device. Must be called once per device before any tpo3_* kernel.
 * When ke is the isotropic unit-cube H8 stiffness (lam K_lam + mu K_mu, every
 * entry within 1e-12 of the largest), the stiffness applications use a
 * structured element operator with the fitted lam, mu; any other ke is applied
 * as the dense 24x24 matrix. Both give the same operator to rounding. */
int tpo_set_stiffness3(const double ke[576], const double ke_inv[576], double alpha_reg);

/* ap = K(rho) p, identity rows at fixed DOFs; *pap_out (device, nullable) =
 * p.ap. Replaces compute_matvec_3d / matvec_and_dot_3d (fem/kernels.py:179-212,
 * fem/fused_kernels.py:59-94). */
size_t tpo3_matvec_workspace_bytes(const tpo_grid3 *g);
int tpo3_matvec_f64(const tpo_grid3 *g, const double *rho, const uint8_t *fixed,
                    const double *p, double *ap, double *pap_out,
                    void *ws, size_t ws_bytes, tpo_stream s);

/* PCG solve K(rho) u = f with the reference's rules (fem/solver.py:27-159):
 * precond TPO_PRECOND_NONE / JACOBI / BLOCK_JACOBI, precision FP64,
 * recurrence AUTO or STANDARD (two launches per iteration; three with the
 * element-block preconditioner). BLOCKING, like tpo_pcg_solve. */
size_t tpo3_pcg_workspace_bytes(const tpo_grid3 *g, const tpo_solve_cfg *c);
int tpo3_pcg_solve(const tpo_grid3 *g, const tpo_solve_cfg *c,
                   const double *rho_phys, const double *f, const uint8_t *fixed,
                   double *u, void *ws, size_t ws_bytes,
                   tpo_solve_result *out, tpo_stream s);

/* dc and compliance as tpo_sensitivity (fem/kernels.py:275-308). */
size_t tpo3_sensitivity_workspace_bytes(const tpo_grid3 *g);
int tpo3_sensitivity(const tpo_grid3 *g, const double *rho_phys, const double *u,
                     double *dc, double *compliance_out,
                     void *ws, size_t ws_bytes, tpo_stream s);

/* Hat-weight filters over the box |dx|,|dy|,|dz| <= ceil(rmin) <= 8
 * (optimizer/filter.py:75-97,106-171); same formulas as the 2D ones. */
int tpo3_density_filter(const tpo_grid3 *g, double rmin, const double *x, double *out,
                        tpo_stream s);
int tpo3_sensitivity_filter(const tpo_grid3 *g, double rmin, const double *rho,
                            const double *dc, double *out, tpo_stream s);

/* OC update over the nelx*nely*nelz elements, as tpo_oc_update
 * (optimizer/oc.py:21-93). */
size_t tpo3_oc_workspace_bytes(const tpo_grid3 *g);
int tpo3_oc_update(const tpo_grid3 *g, double volfrac, double move,
                   const double *rho_in, const double *dc, const double *dv,
                   double *rho_out, double *result_out,
                   void *ws, size_t ws_bytes, tpo_stream s);

#ifdef __cplusplus
}
#endif

#endif /* TPO_H */
