/*
 * slc_b200.h -- C ABI of the B200 (sm_100a) SL-BDF2 channel step.
 *
 * This is the drop-in boundary for slChannel's semi-Lagrangian BDF2 path
 * (gmcavallazzi/SLchannel v1.0.1; reference paths below are relative to that
 * project).  A host binding (the Python package slchannel_b200 uses ctypes)
 * passes plain device pointers, sizes and a cudaStream_t; no torch types cross
 * this boundary.
 *
 * Conventions
 *  - Fields are float64, row-major (x, y, z) with z contiguous, in the
 *    reference's ghost-shaped layouts (one ghost layer per side):
 *      u (nx+1, ny+2, nz+2)   v (nx+2, ny+1, nz+2)   w (nx+2, ny+2, nz+1)
 *      p (nx+2, ny+2, nz+2)
 *    The caller owns field memory; the library owns its tables, FFT plans and
 *    workspaces (allocated in slc_grid_create).
 *  - Every function returns 0 on success or a nonzero SLC_E* code; it never
 *    traps.  slc_last_error() gives the message of the last failure on that
 *    handle.  Work is enqueued on `stream` (NULL = legacy default stream) and
 *    is asynchronous unless stated otherwise.
 *  - A handle is not thread-safe: use one handle per host thread / stream.
 */
#ifndef SLC_B200_H
#define SLC_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define SLC_API __attribute__((visibility("default")))
#else
#define SLC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SLC_OK 0
#define SLC_E_INVALID 1 /* bad argument (maps to the reference's ValueError) */
#define SLC_E_CUDA 2    /* a CUDA runtime / driver call failed (RuntimeError) */
#define SLC_E_CUFFT 3   /* a cuFFT call failed (RuntimeError) */
#define SLC_E_NOMEM 4   /* device allocation failed (RuntimeError) */

#define SLC_PREC_FP64 0  /* plain float64 path (parity form) */
#define SLC_PREC_MIXED 1 /* FP32 fluctuation about an FP64 plane mean in trace+gather */

typedef struct slc_grid slc_grid; /* opaque */

/* Grid description.  Mirrors the arguments of
 * SLAdvector.__init__ (slchannel/semilag.py:133-153) plus the transport
 * and boundary parameters the step needs (slchannel/solver.py:168-282). */
typedef struct {
    int32_t nx, ny, nz;        /* interior cells; x, y periodic, z walls */
    double Lx, Ly, Lz;         /* domain extents */
    double gamma;              /* tanh stretching parameter */
    int32_t stretching;        /* 0 = 'symmetric', 1 = 'bottom' */
    int32_t order;             /* 4 (tricubic) or 6 (triquintic) */
    int32_t traj_order;        /* 2 (trilinear) or 4 (tricubic Lagrange) */
    int32_t n_traj_iters;      /* midpoint fixed-point iterations (>= 1) */
    int32_t top_wall_neumann;  /* 0 = 'dirichlet' (no-slip), 1 = 'neumann' */
    int32_t precision;         /* SLC_PREC_FP64 or SLC_PREC_MIXED */
    double nu;                 /* kinematic viscosity 1/Re */
    const double *z_f;         /* HOST pointer, nz+1 face coordinates */
    const double *z_c;         /* HOST pointer, nz+2 centres incl. ghosts */
    int32_t device;            /* CUDA device ordinal the handle lives on */
    int32_t xy_rhs_lagged;     /* 0 = 'extrap' (2R^n - R^{n-1}), 1 = 'lagged' (R^n) */
} slc_grid_desc;

/* Library version string, e.g. "slc_b200 0.1". */
SLC_API const char *slc_version(void);

/* Build a handle: z tables, Lagrange inverse-denominator tables, cuFFT plans
 * and workspaces.  Replaces SLAdvector.__init__ (semilag.py:133-381) and
 * initialize_fft_solver (slchannel/projection.py:24-131).  Synchronous. */
SLC_API int slc_grid_create(const slc_grid_desc *desc, slc_grid **out);

/* Release a handle and everything it allocated.  Synchronous. */
SLC_API int slc_grid_destroy(slc_grid *g);

/* Message of the last failure on `g` (or of the last failed create when
 * g == NULL).  Valid until the next call on the handle. */
SLC_API const char *slc_last_error(const slc_grid *g);

/* Ghost-cell boundary conditions on u, v, w in place: periodic x, y; no-slip
 * (or free-slip top) u, v; w = 0 on both walls.
 * Replaces apply_bc_all (slchannel/solver.py:70-107). */
SLC_API int slc_apply_bc(slc_grid *g, double *u, double *v, double *w, void *stream);

/* Continuous face index of n wall-normal coordinates (device arrays).
 * Replaces SLAdvector._face_coord (semilag.py:400-411). */
SLC_API int slc_face_coord(slc_grid *g, const double *z, int64_t n, double *kf, void *stream);

/* Interpolate one component's node buffer (NX, NY, NZ) contiguous, at n
 * arbitrary points with Lagrange order 2, 4 or 6.  With count_clamp, z is
 * clamped to [z_lo, z_hi] and the clamps are ADDED to *nclamp (device int64).
 * Replaces SLAdvector._build_iw + _apply_iw (semilag.py:460-510). */
SLC_API int slc_interp_points(slc_grid *g, int comp, int order, const double *nodebuf, const double *x,
                      const double *y, const double *z, int64_t n, int count_clamp, double *out,
                      int64_t *nclamp, void *stream);

/* Departure points (x_d, y_d, z_d) of every arrival point of `comp`
 * (arrival-shaped, z fastest), traced through the trajectory velocity given
 * as three node buffers (NX, NY, NZ) contiguous.
 * Replaces SLAdvector.departure_coords (semilag.py:534-552). */
SLC_API int slc_departure(slc_grid *g, int comp, const double *mid_u, const double *mid_v,
                  const double *mid_w, double dt, double *xd, double *yd, double *zd,
                  void *stream);

/* One semi-Lagrangian foot for all three components: trace each arrival
 * point through (mid_u, mid_v, mid_w) over dt and interpolate (fu, fv, fw)
 * there.  All inputs and outputs are ghost-shaped; only the interiors of
 * ou, ov, ow are written (w wall faces and ghosts untouched).  The number of
 * clamped feet is WRITTEN to *nclamp (device int64).
 * Replaces SLAdvector.advect (semilag.py:584-671). */
SLC_API int slc_advect(slc_grid *g, const double *fu, const double *fv, const double *fw,
               const double *mid_u, const double *mid_v, const double *mid_w, double dt,
               double *ou, double *ov, double *ow, int64_t *nclamp, void *stream);

/* slc_advect with extra field triples interpolated at the same feet:
 * every arrival point is traced once, and (fu, fv, fw) plus each of the
 * n_extra triples extra_in[3 t + c] (c = 0 u, 1 v, 2 w; ghost-shaped) are
 * interpolated there.  (ou, ov, ow) receive the advected triple as in
 * slc_advect (ghost-shaped interiors); extra_out[3 t + c] receive triple t
 * ARRIVAL-shaped and contiguous, (nx, ny, nz) for u and v and (nx, ny, nz-1)
 * for w, z fastest.  *nclamp (device int64) receives the clamp count of the
 * feet, counted once.  In the FP64 form up to 7 extra triples share one
 * trace with the advected triple (more are traced again per group of 8); the
 * mixed form packs and gathers each triple in turn at the same FP32 feet.
 * n_extra <= SLC_MAX_EXTRA.
 * Replaces SLAdvector.advect(..., extra_rhs) (semilag.py:584-671). */
#define SLC_MAX_EXTRA 64
SLC_API int slc_advect_extra(slc_grid *g, const double *fu, const double *fv, const double *fw,
                             const double *mid_u, const double *mid_v, const double *mid_w,
                             double dt, double *ou, double *ov, double *ow, int n_extra,
                             const double *const *extra_in, double *const *extra_out,
                             int64_t *nclamp, void *stream);

/* Fused BDF2 predictor: both feet of every arrival point traced with
 * U* = 2 V^n - V^{n-1} (depths dt and 2 dt), V^n and V^{n-1} interpolated
 * there, and u_hat = 4/3 ubar - 1/3 ubarbar + (2/3) dt (2 R^n - R^{n-1})
 * written to the interiors of (ou, ov, ow), R the explicit x,y diffusion.
 * cur/prev/out are ghost-shaped; cur and prev must be BC-consistent.
 * *nclamp (device int64) receives the clamp count over both feet.  This
 * entry point gathers through L1 in both precisions (slc_step_bdf2 on a
 * mixed handle gathers from TMA-staged boxes, the results being equal).
 * Replaces solver.py:846-903 (the two SLAdvector.advect calls and the
 * BDF2 combination). */
SLC_API int slc_trace_gather_bdf2(slc_grid *g, const double *un, const double *vn, const double *wn,
                          const double *unm1, const double *vnm1, const double *wnm1, double dt,
                          double *ou, double *ov, double *ow, int64_t *nclamp, void *stream);

/* One SL-BDF2 step with its bulk shift (slc_step_bdf2 + slc_bulk_shift) for
 * a caller whose state lives in HOST memory (page-locked for overlap):
 * uploads cur = V^n and prev = V^{n-1}, and downloads next = V^{n+1}, p and
 * bulk_out2 = (u_bulk, forcing).  All are host pointers; the device state is
 * the library's (double-buffered).  Uploads, compute and downloads overlap:
 * the copies run on two copy streams in pieces, and an upload whose host
 * source an earlier call is still downloading into waits for the overlapping
 * pieces only, so feeding each call's next back as the following call's cur
 * pipelines the round trip.  FP64 handles with nx >= 96 also stream the step
 * itself by x slab: cur and next move slab by slab, and each slab's
 * trace+gather starts once its neighbour slabs of cur are on the device
 * (when its feet provably stay within them; otherwise after the last
 * slab).  The results equal slc_step_bdf2's followed by slc_bulk_shift.  Returns after enqueueing; the outputs are on the
 * host, and the host buffers may be touched again, once `stream` completes.
 * The step computes on an internal stream of the handle: ordered after the
 * handle's previous host-state call (and, at the first call, after work
 * already enqueued on `stream`), not after later work of the caller's, so
 * one call's compute overlaps the previous call's downloads.  So any work
 * of another entry point on the same handle (on `stream` or any other
 * stream) must have COMPLETED before the next host-state call is made
 * (synchronise its stream first): the internal stream does not wait for
 * it, and both would use the handle's workspaces.  Likewise, synchronise
 * `stream` after a host-state call before other entry points use the handle.
 * No counterpart in the reference (its state is device- or CPU-resident). */
SLC_API int slc_step_bdf2_host(slc_grid *g, const double *const cur[3], const double *const prev[3],
                               double *const next[3], double *p, double *bulk_out2, double U_bulk,
                               double dt, void *stream);

/* How the handle's host-state calls ran: out4[0] calls streamed by x slab,
 * out4[1] calls run whole (mixed handles, nx < 96), out4[2] slabs of the last
 * call (0 when it ran whole), out4[3] slabs of the last call whose feet left
 * the slabs on the device when it was released, and that were recomputed
 * after all of V^n had arrived.  Synchronises the handle's compute.  No
 * counterpart in the reference. */
SLC_API int slc_host_step_stats(slc_grid *g, int64_t *out4);

/* slc_trace_gather_bdf2 with each block's two gather source boxes staged
 * in shared memory by the Tensor Memory Accelerator (3-D cp.async.bulk.tensor
 * loads of halo-padded node copies; otherwise identical to
 * slc_trace_gather_bdf2).  Results are bit-identical to
 * slc_trace_gather_bdf2's.  FP64 handles (nz >= 47): the padded copies are
 * written with U*; not the FP64 step's default, since at the 256^3
 * benchmark that extra pass takes back the kernel's gain, while where the
 * feet spread (trajectory CFL 3) this call is the faster of the two.  Mixed
 * handles (nz >= 62): FP32 fluctuation boxes, the padded copies written by
 * the mixed pack itself; slc_step_bdf2 on a mixed handle gathers this way.
 * slc_gather_stats reports how many boxes were staged.  Synchronous: it
 * waits for `stream` and returns SLC_E_CUDA if any bulk copy of this call
 * did not complete within the kernel's bounded waits (the affected blocks
 * gathered through L1, but a copy that lands after its block exited may have
 * written another block's shared memory, so the results are not trusted).
 * No counterpart in the reference. */
SLC_API int slc_trace_gather_bdf2_staged(slc_grid *g, const double *un, const double *vn,
                                         const double *wn, const double *unm1, const double *vnm1,
                                         const double *wnm1, double dt, double *ou, double *ov,
                                         double *ow, int64_t *nclamp, void *stream);

/* theta = 1 implicit wall-normal diffusion, in place on the interiors:
 * (I - dt nu Dzz) f_new = f.
 * Replaces solve_implicit_diffusion_{u,v,w} (slchannel/operators.py:382-630). */
SLC_API int slc_zsolve(slc_grid *g, double *u, double *v, double *w, double dt, void *stream);

/* The implicit wall-normal diffusion of slc_zsolve, for callers that must
 * not allocate device memory: no handle, no cudaMalloc/cudaFree, no
 * allocating library call.  This has no counterpart in the reference.
 * It is meant for host codes whose own memory manager owns the device (a
 * pooled or budgeted allocator that a library cudaMalloc would bypass or
 * fail against) and for tight time loops where cudaMalloc's implicit device
 * synchronisation is not acceptable.  The caller passes the fields (solved in
 * place on their interiors, ghost-shaped as everywhere in this header) and the
 * grid spacings dz_c (nz+1) and dz_f (nz) as device arrays; nu is the
 * kinematic viscosity, top_wall_neumann selects the free-slip top closure.
 * The Thomas tables live in one fixed device array of 6 * 1024 doubles
 * (48 KiB) that every GPU loading the library keeps until process exit, so
 * nz > 1024 is rejected with SLC_E_INVALID.  Each call looks up that array's
 * address on the current device (cudaGetSymbolAddress, no allocation); the
 * first call on a device also loads the library's device code there, so make
 * that first call before any stream capture.  All calls on a device share the array and each call
 * rewrites it before reading it: calls that overlap on the GPU (different
 * streams, no ordering between them) race on it.  Errors are reported
 * through slc_last_error(NULL). */
SLC_API int slc_zsolve_noalloc(int nx, int ny, int nz, double nu, int top_wall_neumann,
                               const double *dz_c, const double *dz_f, double dt, double *u,
                               double *v, double *w, void *stream);

/* Divergence of the staggered field, interior-shaped (nx, ny, nz) output.
 * Replaces compute_divergence (slchannel/utils.py:166-180). */
SLC_API int slc_divergence(slc_grid *g, const double *u, const double *v, const double *w, double *div,
                   void *stream);

/* Handle-free divergence for callers that hold only the grid spacings:
 * dz_f is a device array of nz face spacings.  Same result as slc_divergence.
 * Replaces compute_divergence (slchannel/utils.py:166-180) as called with
 * explicit (nx, ny, nz, dx, dy, dz_f). */
SLC_API int slc_divergence_raw(int nx, int ny, int nz, double dx, double dy, const double *dz_f,
                               const double *u, const double *v, const double *w, double *div,
                               void *stream);

/* Pressure projection: phi solves Lap phi = div(u)/dt_div (FFT in x, y,
 * Thomas in z, (0,0) mode pinned); u -= dt_proj grad phi on the interiors;
 * p (ghost-shaped) receives phi with its ghost cells; then BCs on u, v, w.
 * Replaces compute_divergence + solve_poisson_fft + project_velocity
 * (slchannel/projection.py:133-272, solver.py:983-998). */
SLC_API int slc_project(slc_grid *g, double *u, double *v, double *w, double *p, double dt_div,
                double dt_proj, void *stream);

/* Bulk velocity sum(u dx dy dz_f) / (Lx Ly Lz) into *out (device double).
 * Replaces compute_bulk_velocity (slchannel/utils.py:147-163). */
SLC_API int slc_bulk_velocity(slc_grid *g, const double *u, double *out, void *stream);

/* Number of doubles of device scratch slc_bulk_velocity_raw needs. */
SLC_API int slc_bulk_scratch_doubles(void);

/* Handle-free bulk velocity: out = inv_volume * sum_{i,j,k} u_int(i,j,k) *
 * vol_k[k], with vol_k the per-level cell volume dx*dy*dz_f (device, nz) and
 * scratch at least slc_bulk_scratch_doubles() device doubles.  Summed in a
 * fixed order (bit-reproducible).
 * Replaces compute_bulk_velocity (slchannel/utils.py:147-163) for the
 * cell-volume tensor the solver builds (solver.py:303-306). */
SLC_API int slc_bulk_velocity_raw(int nx, int ny, int nz, const double *u, const double *vol_k,
                                  double inv_volume, double *scratch, double *out, void *stream);

/* Exact mass-flux constraint: c = U_bulk - bulk(u); u_int += c; BCs;
 * out2[0] = bulk(u) after the shift, out2[1] = c / dt (device doubles).
 * Replaces SLChannelFlow._apply_bulk_forcing (slchannel/solver.py:694-723). */
SLC_API int slc_bulk_shift(slc_grid *g, double *u, double *v, double *w, double U_bulk, double dt,
                   double *out2, void *stream);

/* One BDF1 bootstrap step up to (not including) the bulk shift:
 * next <- advect(cur; U* = cur, dt) + dt R(cur); z-solve at dt; projection
 * at dt; p <- phi.  cur gets its BCs applied first.  The caller afterwards
 * treats cur as V^{n-1} and next as V^n.  next's w wall faces must hold 0 on
 * entry (the divergence reads them before the ghost refresh).
 * Replaces SLChannelFlow._step_sl_bdf1_bootstrap (solver.py:729-811)
 * without its final _bdf2_forcing_update call. */
SLC_API int slc_step_bdf1(slc_grid *g, double *const cur[3], double *const next[3], double *p, double dt,
                  int64_t *nclamp, void *stream);

/* One BDF2 step up to (not including) the bulk shift: slc_trace_gather_bdf2
 * into next, z-solve at 2dt/3, projection at 2dt/3, p <- phi.  The caller
 * afterwards rotates (prev, cur, next) <- (cur, next, prev).  As in
 * slc_step_bdf1, next's w wall faces must hold 0 on entry (a zeroed buffer
 * or one from an earlier step): the divergence reads them before the ghost
 * refresh.
 * Replaces SLChannelFlow.step_sl_bdf2 (solver.py:813-1018, noninc pressure)
 * without its final _bdf2_forcing_update call. */
SLC_API int slc_step_bdf2(slc_grid *g, double *const cur[3], double *const prev[3], double *const next[3],
                  double *p, double dt, int64_t *nclamp, void *stream);

/* ---- Profiling -------------------------------------------------------------
 * Phases timed with CUDA events on the launching stream when timing is on. */
#define SLC_PHASE_BC 0      /* start-of-step boundary conditions */
#define SLC_PHASE_MID 1     /* U* = 2 V^n - V^{n-1} */
#define SLC_PHASE_SL 2      /* fused trace + gather (+ BDF epilogue) kernels */
#define SLC_PHASE_ZSOLVE 3  /* implicit wall-normal diffusion */
#define SLC_PHASE_PROJECT 4 /* divergence, FFTs, Thomas, projection, BCs */
#define SLC_PHASE_BULK 5    /* bulk-flux shift */
#define SLC_NPHASE 6

/* ---- The Eulerian IMEX scheme (the SL step's comparison baseline) ---------
 * Explicit x,y diffusion minus flux-form advection of u, v, w on the
 * interiors (compute_momentum_rhs_fused_imex, operators.py:638-832), one
 * fused pass; ghosts of ru, rv, rw are not written. */
SLC_API int slc_imex_rhs(slc_grid *g, const double *u, const double *v, const double *w, double *ru,
                         double *rv, double *rw, void *stream);

/* One IMEX step up to (not including) the bulk shift (step_imex,
 * solver.py:1055-1135): rhs_cur <- the explicit right-hand side of vel;
 * vel += dt (1.5 rhs_cur - 0.5 rhs_prev) (forward Euler without a history);
 * theta-method z-diffusion (theta 0.5: Crank-Nicolson, its explicit half with
 * the reference's wall closures); projection at dt; p <- phi.  rhs_prev is
 * used as workspace afterwards: the caller then swaps the two, as the
 * reference does (solver.py:1081-1083). */
SLC_API int slc_step_imex(slc_grid *g, double *const vel[3], double *p, double *const rhs_cur[3],
                          double *const rhs_prev[3], int have_prev, double dt, double theta,
                          void *stream);

/* Turn per-phase event timing on (1) or off (0) for a handle; resets the
 * accumulated record.  Adds two cudaEventRecord calls per phase per call. */
SLC_API int slc_timing(slc_grid *g, int enable);

/* One BDF2 step with the incremental pressure (sl.bdf2_pressure: inc,
 * solver.py:905-941, 1001-1012), up to the bulk shift.  p_cur holds the full
 * pressure p^n and p_prev p^{n-1} (have_prev = 0 on the first BDF2 step after
 * a BDF1 bootstrap, whose p is its phi).  The predictor gets
 * -(2dt/3) grad(p_ext), p_ext = 2 p^n - p^{n-1} (p^n without a history),
 * before the z-solve.  On return p_cur = p_ext + phi and p_prev = the old
 * p_cur.  Ghost-shaped pressures; next's w wall faces must hold 0. */
SLC_API int slc_step_bdf2_inc(slc_grid *g, double *const cur[3], double *const prev[3],
                              double *const next[3], double *p_cur, double *p_prev, int have_prev,
                              double dt, int64_t *nclamp, void *stream);

/* Synchronise on the recorded events and return, per phase, the summed
 * elapsed milliseconds and the number of timed intervals; resets the record.
 * ms and count each hold SLC_NPHASE entries. */
SLC_API int slc_timing_read(slc_grid *g, double *ms, int64_t *count);

/* Counters of slc_trace_gather_bdf2_staged, accumulated
 * since creation or the last reset: out4[0] staged boxes that did not arrive
 * within the poll limit (the block then gathered through L1; results are
 * unaffected), out4[1] blocks, out4[2] near-foot boxes staged, out4[3]
 * far-foot boxes staged (the rest gathered through L1).  Synchronous. */
SLC_API int slc_gather_stats(slc_grid *g, int64_t *out4, int reset);

/* ---- Diagnostics and statistics (on the device, no host synchronisation) ----
 * out4 (device, 4 doubles) <- [max |div| over the interior (utils.py:166-180),
 * u_tau (utils.py:116-144: wall-adjacent plane means of u, ghosts included,
 * bottom only for a free-slip top), the CFL inverse max(1/dt) of
 * compute_cfl_fused (operators.py:839-940), the bulk velocity
 * (utils.py:147-163)].  Fixed-order reductions: reruns agree bit for bit.
 * The raw form needs no handle; scratch holds
 * slc_diagnostics_scratch_doubles() device doubles and z_c nz+2 centres. */
SLC_API int slc_diagnostics(slc_grid *g, const double *u, const double *v, const double *w, double *out4,
                            void *stream);
SLC_API int slc_diagnostics_scratch_doubles(void);
SLC_API int slc_diagnostics_raw(int nx, int ny, int nz, double dx, double dy, const double *dz_f,
                                const double *dz_c, const double *z_c, double nu, int top_neumann,
                                double Lx, double Ly, double Lz, const double *u, const double *v,
                                const double *w, double *out4, double *scratch, void *stream);

/* One snapshot of TurbulenceStats.accumulate_statistics (turbstats.py:156-360)
 * added to device accumulators:
 *  - prof (11 nz doubles, or NULL): U, u'u', v'v', w'w', u'w', V, W, U^2, V^2,
 *    W^2 and U W, each an nz-level profile about the instantaneous plane
 *    means, as the reference forms them;
 *  - spec (4 (nx/2) (ny/2) doubles, or NULL): the folded 2-D spectra
 *    E_uu, E_vv, E_ww, E_uw, averaged over the interior levels k_bot and
 *    k_top (1-based, as the reference's k_bot / k_top; w negated at the top).
 * Fixed-order reductions. */
SLC_API int slc_stats_accumulate(slc_grid *g, const double *u, const double *v, const double *w,
                                 double *prof, double *spec, int k_bot, int k_top, void *stream);

/* Number of kernels this library has launched in the process so far (its
 * own kernels; cuFFT's are not counted). */
SLC_API int64_t slc_kernel_launches(void);

/* FMA-pipe throughput of the current device in GFLOP/s (FMA = 2 flops),
 * FP64 (fp64 = 1) or FP32 (fp64 = 0): a register-resident chain kernel over
 * every SM at full occupancy, best of three timed launches on `stream`
 * (synchronises it).  Measurement support, no counterpart in the reference:
 * the denominator for the trace+gather kernels' arithmetic rate. */
SLC_API int slc_fma_peak(int fp64, double *gflops, void *stream);

/* A measurement of the gather formulation, not on the step path: the
 * order-6 Lagrange gather of a synthetic FP32 field at n^3 smoothly displaced
 * feet (n = 64, 128, 192 or 256), done by one thread per point with 216
 * scalar loads (the mixed form's gather) and by tensor cores (mma.sync
 * m16n8k16, FP16 hi/lo split of field and weights, three products, FP32
 * accumulation, over the union of 16 points' stencil rows), each launched
 * `reps` times.  out4 = (ms per scalar launch, ms per tensor-core launch,
 * max |difference| / max |value|, tensor-core groups that fell back to the
 * scalar gather per launch).  Allocates its own buffers; synchronous.
 * No counterpart in the reference. */
SLC_API int slc_gather_probe(int n, int reps, double *out4, void *stream);

/* ---- Adjoint (reverse mode) of the step ----------------------------------------
 * No counterpart in the reference, which relies on torch autograd through its
 * eager path.  Gradients of a loss on the velocity with respect to earlier
 * velocities, FP64 handles only.  Adjoint fields lam_* are ghost-shaped like
 * the velocity; their ghost entries may hold contributions that belong to
 * interior values until slc_adjoint_bc folds them in. */

/* Transpose of the ghost refresh (apply_bc_all, solver.py:70-107): add each
 * ghost's adjoint, with the copy's sign, to its interior source, and zero
 * every ghost (and w wall) entry. */
SLC_API int slc_adjoint_bc(slc_grid *g, double *lam_u, double *lam_v, double *lam_w, void *stream);

/* Reverse of one step.
 *  - mode 2: slc_step_bdf2 + slc_bulk_shift, from cur = V^n and prev = V^{n-1};
 *  - mode 1: the BDF1 bootstrap slc_step_bdf1 + slc_bulk_shift, from cur = V^0
 *    (prev and lam_prev unused).
 * cur and prev are the forward's states with their ghosts refreshed.
 * lam_next = dJ/dV^{n+1} is consumed (overwritten as workspace).  The step's
 * contributions are ADDED to lam_cur (dJ/dV^n) and lam_prev (dJ/dV^{n-1}).
 * The transposed gathers are deterministic (no floating-point atomics).
 * Allocates its workspace on first use. */
SLC_API int slc_adjoint_step(slc_grid *g, int mode, double *const cur[3], double *const prev[3],
                             double *const lam_next[3], double *const lam_cur[3],
                             double *const lam_prev[3], double dt, void *stream);

/* ---- Ensembles of independent channels --------------------------------------
 * No counterpart in the reference, which advances one channel per process.
 * An ensemble advances n channels of uneven grids, viscosities and time steps
 * together.  Every substep of the BDF2 step is one launch over all of them:
 *  - the trace+gather is a persistent kernel over an (instance, component,
 *    tile) work queue;
 *  - the Poisson FFTs are one cuFFT call per group of instances sharing
 *    (nx, ny);
 *  - the step can be captured once per phase into a CUDA graph.
 * Per instance the arithmetic is that of slc_step_bdf2 followed by
 * slc_bulk_shift, so an instance matches the same channel stepped alone, in
 * the FP64 or (all instances alike) the mixed form. */
typedef struct slc_ensemble slc_ensemble; /* opaque */

/* n instances; descs[i] as for slc_grid_create (one order, one device, one
 * precision, nz >= 2).  Synchronous. */
SLC_API int slc_ensemble_create(const slc_grid_desc *descs, int n, slc_ensemble **out);
SLC_API int slc_ensemble_destroy(slc_ensemble *e);
SLC_API int slc_ensemble_size(const slc_ensemble *e);
/* The instance's own handle (BDF1 bootstrap, diagnostics); owned by e. */
SLC_API slc_grid *slc_ensemble_grid(slc_ensemble *e, int i);
SLC_API const char *slc_ensemble_last_error(const slc_ensemble *e);

/* Bind the caller's device fields and per-instance parameters:
 *  - lev[(i * 3 + level) * 3 + comp]: three time levels of (u, v, w) per
 *    instance, ghost-shaped;
 *  - p[i]: the pressure;
 *  - dt[i], U_bulk[i]: HOST arrays;
 *  - nclamp: n device int64 clamp counters, or NULL;
 *  - bulk_out: 2 n device doubles, [u_bulk, forcing] per instance.
 * The step of phase ph reads V^{n-1} from level ph % 3 and V^n from level
 * (ph + 1) % 3, and writes V^{n+1} into level (ph + 2) % 3.  Allocates the
 * group FFT pools, plans and z-solve tables.  Drops captured graphs.
 * Synchronous. */
SLC_API int slc_ensemble_bind(slc_ensemble *e, double *const *lev, double *const *p,
                              const double *dt, const double *U_bulk, int64_t *nclamp,
                              double *bulk_out);

/* Per-instance SL tile shape: 2^tkl[i] z points x 2^(8 - tkl[i]) y rows,
 * tkl in [3, 8].  Results do not depend on it. */
SLC_API int slc_ensemble_set_tiles(slc_ensemble *e, const int *tkl);
SLC_API int slc_ensemble_get_tiles(const slc_ensemble *e, int *tkl);

/* Tile-shape autotuner.  For each distinct grid shape it times the
 * trace+gather of that shape's instances with z tiles of 32, 64 and 128
 * points (`reps` launches each, after one warm-up) and keeps the fastest.
 * Runs the phase's U* and trace+gather, so it overwrites the V^{n+1} level
 * and the clamp counters.  tkl_out (n) and timings_ms (3 n) may be NULL.
 * Synchronous. */
SLC_API int slc_ensemble_autotune(slc_ensemble *e, int phase, int reps, int *tkl_out,
                                  double *timings_ms, void *stream);

/* One SL-BDF2 step of every instance, bulk shift included, in phase
 * `phase` (0, 1, 2).  With use_graph, the first call per phase captures the
 * step into a CUDA graph on a private stream; every call then launches it
 * on `stream`.  The first call per phase must therefore not itself be under
 * stream capture. */
SLC_API int slc_ensemble_step_bdf2(slc_ensemble *e, int phase, int use_graph, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SLC_B200_H */
