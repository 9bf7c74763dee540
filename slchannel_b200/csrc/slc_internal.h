// slc_internal.h -- launch wrappers shared between the .cu files of the
// library (not part of the public ABI; see include/slc_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "slc_common.cuh"

// Number of this library's kernel launches (slc_kernel_launches()).
extern std::atomic<long long> g_slc_launches;
inline void count_launches(int n) { g_slc_launches.fetch_add(n, std::memory_order_relaxed); }

// Raw pointers of a velocity triple (ghost-shaped arrays or node buffers).
struct Tri {
    const double *u, *v, *w;
};
struct TriMut {
    double *u, *v, *w;
};

// ---- sl_trace_gather.cu ----------------------------------------------------
// mode: 0 = one foot (advect), 1 = BDF1 predictor, 2 = BDF2 predictor.
// `mid_node` selects the layout of `mid`: true = node buffers (NX, NY, NZ),
// false = ghost-shaped arrays.
cudaError_t launch_sl(const SlcParams &P, int mode, Tri fn, Tri fnm1, Tri mid, bool mid_node,
                      double dt, TriMut out, unsigned long long *nclamp, cudaStream_t s);
// One foot per arrival point shared by nf <= kMaxMultiFields fields of one
// component each (SLAdvector.advect with extra_rhs): field f = in[3 f + c]
// of component c, its result at out[3 f + c][maps[3 f + c]]; the clamps of
// the foot are added to *nclamp (none when nclamp is null).
constexpr int kMaxMultiFields = 8;
cudaError_t launch_advect_multi(const SlcParams &P, int nf, const double *const *in,
                                double *const *out, const OutMap *maps, Tri mid, double dt,
                                unsigned long long *nclamp, cudaStream_t s);
cudaError_t launch_departure(const SlcParams &P, int comp, Tri mid_node, double dt, double *xd,
                             double *yd, double *zd, cudaStream_t s);
cudaError_t launch_interp(const SlcParams &P, int comp, int order, const double *buf,
                          const double *x, const double *y, const double *z, int64_t n,
                          int count_clamp, double *out, unsigned long long *nclamp,
                          cudaStream_t s);
cudaError_t launch_face_coord(const SlcParams &P, const double *z, int64_t n, double *kf,
                              cudaStream_t s);
cudaError_t launch_lincomb(const double *a, const double *b, double ca, double cb, double *out,
                           int64_t n, cudaStream_t s);

// ---- zsolve.cu ---------------------------------------------------------------
// Thomas factorisation tables of (I - dt nu Dzz) with the wall closures:
// tab_uv = [alpha | invden | cprime] for u and v, tab_w likewise for w (nz-1 rows).
// Column chunk per lane of the z-solve (ceil(nz/32) rounded up to an
// instantiated size) and the table layout: each of the six tables (alpha,
// invden, c' for u/v, then for w) holds 32 * chunk entries, entry k at
// (k % chunk) * 32 + k / chunk so that a warp's lanes read consecutive words.
__host__ __device__ inline int zsolve_chunk(int nz)
{
    const int need = (nz + 31) / 32;
    return need <= 1 ? 1 : need <= 2 ? 2 : need <= 4 ? 4 : need <= 8 ? 8 : need <= 12 ? 12
         : need <= 16 ? 16 : 32;
}
inline size_t zsolve_table_doubles(int nz) { return (size_t)6 * 32 * zsolve_chunk(nz); }
cudaError_t launch_zsolve_tables(const SlcParams &P, const double *dz_c, const double *dz_f,
                                 double dt, double *tab_uv, double *tab_w, cudaStream_t s);
cudaError_t launch_zsolve(const SlcParams &P, TriMut f, const double *tab_uv, const double *tab_w,
                          cudaStream_t s);

// ---- poisson.cu --------------------------------------------------------------
cudaError_t launch_apply_bc(const SlcParams &P, double *u, double *v, double *w, double *p,
                            cudaStream_t s);
cudaError_t launch_div_pack(const SlcParams &P, Tri f, const double *dz_f, double dt_div,
                            double *rhs_zmajor, cudaStream_t s);
cudaError_t launch_divergence(const SlcParams &P, Tri f, const double *dz_f, double *div,
                              cudaStream_t s);
cudaError_t launch_thomas_poisson(const SlcParams &P, double *hat, double *cp, const double *kx2,
                                  const double *ky2, const double *cl, const double *cr,
                                  cudaStream_t s);
cudaError_t launch_project(const SlcParams &P, const double *phi_zmajor, TriMut f, double *p,
                           const double *dz_c, double dt, cudaStream_t s);
// bulk: partial sums of u*dz_f over the interior (shift c added first when
// c_dev != NULL), then a fixed-order finish.  out[0] = bulk; with
// shift_out != NULL: shift_out[0] = U_bulk - bulk, shift_out[1] = that / dt.
cudaError_t launch_bulk_partials(const SlcParams &P, double *u, const double *dz_f,
                                 const double *c_dev, double *partials, cudaStream_t s);
cudaError_t launch_bulk_finish(const SlcParams &P, const double *partials, double Lx, double Ly,
                               double U_bulk, double dt, double *bulk_out, double *shift_out,
                               cudaStream_t s);

// u, v, w interiors -= c grad(p) for a ghost-shaped p (the inc branch).
cudaError_t launch_grad_sub(const SlcParams &P, const double *p, TriMut f, const double *dz_c, double c,
                            cudaStream_t s);

constexpr int kBulkBlocks = 1184;  // 8 x 148 SMs; fixed, so the sum order is too

// Message of a failed handle-free call, for slc_last_error(NULL); returns code.
int slc_report_error(int code, const char *msg);

// ---- sl_mixed.cu -------------------------------------------------------------
// Workspace of the mixed form.  Slot q = comp + 3 * which, which = 0 the near
// field (V^n), 1 the far field (V^{n-1}), 2 the trajectory velocity U*.
struct MixedWS {
    float *f32[9];    // FP32 fluctuation node buffers (nx, ny, nzp[comp])
    double *mean[9];  // FP64 plane-mean profiles (nz+2 levels for u, v; nz+1 for w)
    float *mean32[9]; // the same profiles rounded to FP32 (trajectory samples)
    double *partials; // mixed_partials_doubles() scratch for the plane means
    int nzp[3];       // padded node-buffer row length per component
};
int mixed_nzp(int NZ);
size_t mixed_partials_doubles(const SlcParams &P);
// Plane means + FP32 packs of A, B and U* (= M when M.u != NULL, else 2A - B).
// With pad: the V^n and V^{n-1} fluctuations go to pad's halo-padded copies
// instead of ws.f32[0..5] (struct TmaMixed below).
struct TmaMixed;
cudaError_t launch_mixed_prepare(const SlcParams &P, Tri A, Tri B, Tri M, const MixedWS &ws,
                                 cudaStream_t s, const TmaMixed *pad = nullptr);
// mode 0 one foot of A, 1 BDF1 predictor, 2 BDF2 predictor; fn/fnm1 FP64 fields for R.
cudaError_t launch_sl_mixed(const SlcParams &P, int mode, Tri fn, Tri fnm1, const MixedWS &ws,
                            double dt, TriMut out, unsigned long long *nclamp, cudaStream_t s,
                            const OutMap *om = nullptr);

// ---- ensemble kernels (many independent channels, one launch per substep) ----
// One channel as the multi-instance kernels see it.  The three time levels of
// (u, v, w) are cycled by the step phase ph: V^{n-1} = lev[ph % 3],
// V^n = lev[(ph + 1) % 3], V^{n+1} = lev[(ph + 2) % 3].
struct EnsInst {
    SlcParams P;
    double *lev[3][3];
    double *p;
    double *mid[3];                 // U* = 2 V^n - V^{n-1}, ghost-shaped
    const double *dzf, *dzc, *kx2, *ky2, *cl, *cr;
    double *rhs, *hat, *cpw;        // Poisson workspaces (rhs, hat inside a group's FFT pools)
    const double *zs_uv, *zs_w;     // z-solve tables at dt_eff = 2 dt / 3
    double *partials, *scal;        // kBulkBlocks partial sums; [shift, forcing]
    unsigned long long *ncl;        // departure-clamp counter
    double *bulk_out;               // [u_bulk after the shift, forcing]
    double dt, Lx, Ly, U_bulk;
    int tkl;                        // SL tile: 2^tkl z points x 2^(8 - tkl) y rows
    int mixed;                      // mixed form: mws holds the FP32 workspace
    MixedWS mws;
};
// A block's work: instance and three kernel-specific coordinates.
struct EnsItem {
    int inst, a, b, c;
};
__host__ __device__ inline int ens_prev(int ph) { return ph % 3; }
__host__ __device__ inline int ens_cur(int ph) { return (ph + 1) % 3; }
__host__ __device__ inline int ens_next(int ph) { return (ph + 2) % 3; }

// sl_trace_gather.cu: persistent BDF2 trace+gather over the queue `items`
// (inst, comp, i, tile index); `queue` is a zeroed counter.
cudaError_t launch_sl_ens(const EnsInst *ins, const EnsItem *items, int nitems, int ph, int order,
                          unsigned *queue, int grid, cudaStream_t s);
int sl_ens_blocks_per_sm();
int sl_mixed_ens_blocks_per_sm();  // resident blocks of the mixed persistent kernel
// U* for every instance: items (inst, comp, chunk of 1024 elements).
cudaError_t launch_lincomb_ens(const EnsInst *ins, const EnsItem *items, int nitems, int ph,
                               cudaStream_t s);
// zsolve.cu: items (inst, block of kZWarps columns) of instances whose
// zsolve_chunk(nz) is ch.
constexpr int kZsChunks = 7;
constexpr int kZsChunkValues[kZsChunks] = {1, 2, 4, 8, 12, 16, 32};
cudaError_t launch_zsolve_ens(const EnsInst *ins, const EnsItem *items, int nitems, int lvl,
                              int ch, cudaStream_t s);
int zsolve_ens_warps();
// poisson.cu
cudaError_t launch_bc_ens(const EnsInst *ins, const EnsItem *items, int nitems, int lvl,
                          int with_p, cudaStream_t s);
cudaError_t launch_div_pack_ens(const EnsInst *ins, const EnsItem *items, int nitems, int lvl,
                                cudaStream_t s);
cudaError_t launch_thomas_ens(const EnsInst *ins, const EnsItem *items, int nitems,
                              cudaStream_t s);
cudaError_t launch_project_ens(const EnsInst *ins, const EnsItem *items, int nitems, int lvl,
                               cudaStream_t s);
cudaError_t launch_bulk_partials_ens(const EnsInst *ins, const EnsItem *items, int nitems,
                                     int lvl, int with_shift, cudaStream_t s);
// mode 0: scal = [U_bulk - bulk, (U_bulk - bulk) / dt]; mode 1: bulk_out = [bulk, scal[1]].
cudaError_t launch_bulk_finish_ens(const EnsInst *ins, int ninst, int mode, cudaStream_t s);

// ---- sl_tma.cu: BDF2 trace+gather with TMA-staged source boxes ---------------
// Halo-padded node copies of V^n (slots 0-2) and V^{n-1} (3-5) and their
// tensor maps (CUtensorMap, 128 bytes each, stored opaquely here).
struct TmaSL {
    double *pad[6];
    alignas(64) unsigned char maps[6 * 128];
};
int tma_padded_nz(int NZ);
size_t tma_padded_elems(const SlcParams &P, int comp);
bool tma_supported(const SlcParams &P);
cudaError_t tma_encode(const SlcParams &P, TmaSL &T);
// U* (node entries of the ghost-shaped mid arrays) and the padded copies.
cudaError_t launch_mid_pack(const SlcParams &P, Tri cur, Tri prev, TriMut mid, const TmaSL &T,
                            cudaStream_t s);
// stats (device, accumulated): [0] staged boxes that did not arrive within
// the poll limit (that block then gathers through L1; results stay exact),
// [1] blocks, [2] near-foot boxes staged, [3] far-foot boxes staged.
cudaError_t launch_sl_tma(const SlcParams &P, Tri fn, Tri fnm1, Tri mid, double dt, TriMut out,
                          unsigned long long *nclamp, unsigned long long *stats, const TmaSL &T,
                          cudaStream_t s);

// One 3-D tiled tensor map (128 bytes at map128; z innermost, zero fill):
// FP32 or FP64 elements, dims (z, y, x), y and x strides in bytes, box
// (z, y, x) in elements.
cudaError_t tma_encode_3d(void *map128, bool fp32, const void *base, const unsigned long long dims[3],
                          const unsigned long long strides[2], const unsigned box[3]);

// ---- sl_mixed.cu: the mixed BDF2 trace+gather with TMA-staged FP32 boxes -------
// Halo-padded FP32 fluctuation copies of V^n (slots 0-2) and V^{n-1} (3-5):
// (nx + PX_HALO, ny + PY_HALO, nzp[comp]) with node (i, j) also at
// (i + nx, j), (i, j + ny) and (i + nx, j + ny) where those fall inside,
// written by launch_mixed_prepare when it is given this workspace, and their
// tensor maps.
struct TmaMixed {
    float *pad[6];
    int PX, PY;
    alignas(64) unsigned char maps[6 * 128];
};
bool mixed_tma_supported(const SlcParams &P);
size_t mixed_tma_elems(const SlcParams &P, const MixedWS &ws, int comp);
cudaError_t mixed_tma_encode(const SlcParams &P, const MixedWS &ws, TmaMixed &T);
// stats as launch_sl_tma's
cudaError_t launch_sl_mixed_tma(const SlcParams &P, Tri fn, Tri fnm1, const MixedWS &ws, const TmaMixed &T,
                                double dt, TriMut out, unsigned long long *nclamp,
                                unsigned long long *stats, cudaStream_t s);

// sl_mixed.cu, ensemble forms of the mixed predictor: plane means of V^n and
// V^{n-1} (items (inst, column group, field 0..5)), their finish, the FP32
// packs (items (inst, bx, by, bz) of k_pack_mixed's grid), and the
// persistent trace+gather.
int mixed_mean_blocks();
int mixed_pack_cols();              // y columns one k_pack_mixed block covers
int mixed_pack_threads(int nzp);     // its block size for nzp padded levels
cudaError_t launch_mixed_prepare_ens(const EnsInst *ins, int ninst, const EnsItem *pp_items, int n_pp,
                                     const EnsItem *pack_items, int n_pack, int pack_threads, int ph,
                                     cudaStream_t s);
// traj: the instances' common trajectory order (2 or 4), 0 when they differ
cudaError_t launch_sl_mixed_ens(const EnsInst *ins, const EnsItem *items, int nitems, int ph, int order,
                                int traj,
                                unsigned *queue, int grid, cudaStream_t s);

// ---- host_step.cu: the host-state step streamed by x slab ----------------------
// The x nodes [0, nx) are cut into S slabs at b[0] = 0 < b[1] < ... < b[S] = nx.
// While V^n arrives slab by slab, a slab's BDF2 trace+gather is released once
// its neighbour slabs are on the device; the launch reads snap[slab] (max |U*_u|
// over the slabs prepared so far) and runs only when the feet of every point
// of the slab provably stay within the prepared slabs.  Otherwise it sets
// deferred[slab] and the slab is recomputed by launch_sl_fix after the last
// slab has arrived, so the results never depend on the arrival order.
constexpr int kMaxSlabs = 16;
struct SlabGate {
    unsigned long long umax;             // bits of max |U*_u| (NaN compares above inf)
    unsigned long long snap[kMaxSlabs];  // umax when slab s was released
    int deferred[kMaxSlabs];
};
struct SlabBounds {
    int S;
    int b[kMaxSlabs + 1];
};
// BDF2 trace+gather of component comp for arrival x indices [i0, i1) (slab
// `slab`): runs when 2 dt max|U*_u| / dx (times the trajectory interpolant's
// bound) <= limit nodes, else marks the slab deferred.
cudaError_t launch_sl_slab(const SlcParams &P, int comp, const double *fn, const double *fnm1, Tri mid,
                           double dt, double *out, unsigned long long *nclamp, SlabGate *gate, int slab,
                           int i0, int i1, double limit, cudaStream_t s);
// The deferred slabs of component comp, all x indices of each.
cudaError_t launch_sl_fix(const SlcParams &P, int comp, const double *fn, const double *fnm1, Tri mid,
                          double dt, double *out, unsigned long long *nclamp, const SlabGate *gate,
                          const SlabBounds &sb, cudaStream_t s);
