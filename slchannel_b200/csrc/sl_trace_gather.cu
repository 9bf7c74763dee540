// sl_trace_gather.cu -- the fused semi-Lagrangian trace + Lagrange gather
// (+ BDF2 epilogue) for sm_100a.
//
// One thread per arrival point.  The midpoint fixed-point iteration
// (semilag.py:534-552) samples the frozen trajectory velocity trilinearly;
// its first iteration is evaluated at the arrival point itself and is shared
// by the near (dt) and the far (2 dt) foot, which are otherwise integrated
// independently from the arrival point (solver.py:813-826).  Both feet stay in
// registers; the order-O tensor-product Lagrange interpolation
// (semilag.py:44-59, 426-500) reads V^n / V^{n-1} directly from the caller's
// ghost-shaped arrays (periodic wrap by index arithmetic instead of the
// reference's node-buffer copy, semilag.py:387-394), and the epilogue forms
// 4/3 ubar - 1/3 ubarbar + dt_eff (2 R^n - R^{n-1}) with the explicit x,y
// diffusion R evaluated at the arrival point (operators.py:293-367,
// solver.py:846-903).
#include "slc_internal.h"

namespace {

constexpr int kThreads = 256;
// resident blocks per SM the trace+gather kernel is compiled for (register cap)
#ifndef SLC_SL_MIN_BLOCKS
#define SLC_SL_MIN_BLOCKS 2
#endif
// The tricubic (order-4) gather holds 4x4x4 weights instead of 6x6x6: at four
// blocks per SM (64 registers, <= 16 bytes of spill) its step at 256^3 is 12 %
// faster than at two (6.78 against 7.60 ms; three blocks: 6.85 ms).
#ifndef SLC_SL_O4_MIN_BLOCKS
#define SLC_SL_O4_MIN_BLOCKS 4
#endif
#ifndef SLC_SL_ENS_MIN_BLOCKS  // the persistent ensemble form
#define SLC_SL_ENS_MIN_BLOCKS 2
#endif

#include "sl_device.cuh"

// MODE 0: one foot of depth dt on field fn (SLAdvector.advect).
// MODE 1: BDF1 predictor ubar + dt R(fn)            (solver.py:760-771).
// MODE 2: BDF2 predictor 4/3 ubar - 1/3 ubarbar + (2/3)dt Rh (solver.py:846-903).
// Launch geometry of k_sl: a block is kTileK consecutive z arrival points
// (one warp each 32) x kTileJ y-rows at one x index; grid (z tiles, y tiles, nx).
#ifndef SLC_SL_TILE_K
#define SLC_SL_TILE_K 64
#endif
constexpr int kTileK = SLC_SL_TILE_K, kTileJ = kThreads / kTileK;



// One arrival point (i, j, k) of component C; out-of-range points only
// contribute nothing.  Shared by the single-grid kernel below and the
// persistent ensemble kernel, so both do the same arithmetic per point.
// RH_FIRST: evaluate the explicit x,y diffusion (its ten loads) before the
// trace instead of after the gathers.  Measured at 256^3: 1 % faster for the
// tricubic kernel and for the ensemble kernel, 1 % slower for the triquintic
// single-grid kernel, so only those two use it.
template <int C, int O, int MODE, int TO = 0, bool RH_FIRST = false>
__device__ __forceinline__ void sl_point(const SlcParams &P, const Vel3 &M,
                                         const double *__restrict__ fn,
                                         const double *__restrict__ fnm1, double dt,
                                         double *__restrict__ out, int i, int j, int k,
                                         unsigned &ncl)
{
    const int nzi = (C == 2) ? P.nz - 1 : P.nz;
    if (k < nzi && j < P.ny) {
        double xa, ya, za;
        arrival_point<C>(P, i, j, k, xa, ya, za);
        double Rh_early = 0.0;
        if (MODE == 2 && RH_FIRST) {
            const double Rn = xy_diffusion<C>(P, fn, i, j, k);
            Rh_early = P.xy_lagged ? Rn : 2.0 * Rn - xy_diffusion<C>(P, fnm1, i, j, k);
        }
        double us0, vs0, ws0;
        first_sample<C, TO>(P, M, i, j, k, xa, ya, za, us0, vs0, ws0);

        const NodeView<double> Fn = ghost_view<double>(C, fn, P.nx, P.ny, P.nz);
        double xd, yd, zd;
        trace_foot<TO>(P, M, xa, ya, za, 0.5 * dt, us0, vs0, ws0, xd, yd, zd);
        // the far foot is traced before the near foot's gather (its samples do
        // not depend on it), so the two traces' loads overlap: 1-2 % off the
        // step at 256^3, both orders
        double xf = 0.0, yf = 0.0, zf = 0.0;
        if (MODE == 2) trace_foot<TO>(P, M, xa, ya, za, dt, us0, vs0, ws0, xf, yf, zf);  // half of 2 dt
        const double ubar = gather_foot<C, O>(P, Fn, xd, yd, zd, ncl);
        double res;
        if (MODE == 0) {
            res = ubar;
        } else if (MODE == 1) {
            res = ubar + dt * xy_diffusion<C>(P, fn, i, j, k);
        } else {
            const NodeView<double> Fm = ghost_view<double>(C, fnm1, P.nx, P.ny, P.nz);
            const double ubb = gather_foot<C, O>(P, Fm, xf, yf, zf, ncl);
            double Rh = Rh_early;
            if (!RH_FIRST) {
                const double Rn = xy_diffusion<C>(P, fn, i, j, k);
                Rh = P.xy_lagged ? Rn : 2.0 * Rn - xy_diffusion<C>(P, fnm1, i, j, k);
            }
            res = ubar * (4.0 / 3.0) + ubb * (-1.0 / 3.0);
            res = res + ((2.0 / 3.0) * dt) * Rh;
        }
        const GhostShape g = ghost_shape(C, P.nx, P.ny, P.nz);
        out[(size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z + (k + 1)] = res;
    }
}

template <int C, int O, int MODE, int TO>
__global__ void __launch_bounds__(kThreads, O == 4 ? SLC_SL_O4_MIN_BLOCKS : SLC_SL_MIN_BLOCKS) k_sl(const __grid_constant__ SlcParams P, const __grid_constant__ Vel3 M, const double *__restrict__ fn,
                                                    const double *__restrict__ fnm1, double dt,
                                                    double *__restrict__ out,
                                                    unsigned long long *nclamp)
{
    const int k = blockIdx.x * kTileK + (threadIdx.x % kTileK);
    const int j = blockIdx.y * kTileJ + (threadIdx.x / kTileK);
    const int i = blockIdx.z;
    unsigned ncl = 0;
    sl_point<C, O, MODE, TO, O == 4>(P, M, fn, fnm1, dt, out, i, j, k, ncl);
    add_clamps(nclamp, ncl);
}

// The slab-streamed forms of k_sl's BDF2 mode (host_step.cu): the same
// per-point arithmetic (sl_point), on the x indices of one slab.  The gated
// launch checks once per block that the feet stay within the slabs already on
// the device (block-uniform: every block reads the same snapshot); the fix
// launch runs the slabs whose gated launch stood down, one block per (z, y)
// tile walking the slab's x indices.
__device__ __forceinline__ bool slab_window_ok(const SlcParams &P, const SlabGate *gate, int slab,
                                               double dt, double interp_bound, double limit)
{
    const double um = __longlong_as_double((long long)__ldcg(&gate->snap[slab]));
    return 2.0 * dt * um * P.inv_dx * interp_bound <= limit;  // false for NaN
}

template <int C, int O, int TO>
__global__ void __launch_bounds__(kThreads, O == 4 ? SLC_SL_O4_MIN_BLOCKS : SLC_SL_MIN_BLOCKS)
    k_sl_slab(const __grid_constant__ SlcParams P, const __grid_constant__ Vel3 M,
              const double *__restrict__ fn, const double *__restrict__ fnm1, double dt,
              double *__restrict__ out, unsigned long long *nclamp, SlabGate *gate, int slab, int i0,
              double limit)
{
    // a tricubic trajectory sample can exceed the node maximum (Lebesgue
    // constant of the 4-point Lagrange basis, below 2 in 3-D); 4 bounds it
    if (!slab_window_ok(P, gate, slab, dt, TO == 4 ? 4.0 : 1.0, limit)) {
        if (threadIdx.x == 0) gate->deferred[slab] = 1;
        return;
    }
    const int k = blockIdx.x * kTileK + (threadIdx.x % kTileK);
    const int j = blockIdx.y * kTileJ + (threadIdx.x / kTileK);
    unsigned ncl = 0;
    sl_point<C, O, 2, TO, O == 4>(P, M, fn, fnm1, dt, out, i0 + (int)blockIdx.z, j, k, ncl);
    add_clamps(nclamp, ncl);
}

template <int C, int O, int TO>
__global__ void __launch_bounds__(kThreads, O == 4 ? SLC_SL_O4_MIN_BLOCKS : SLC_SL_MIN_BLOCKS)
    k_sl_fix(const __grid_constant__ SlcParams P, const __grid_constant__ Vel3 M,
             const double *__restrict__ fn, const double *__restrict__ fnm1, double dt,
             double *__restrict__ out, unsigned long long *nclamp, const SlabGate *gate,
             const __grid_constant__ SlabBounds sb)
{
    const int slab = blockIdx.z;
    if (!__ldcg(&gate->deferred[slab])) return;
    const int k = blockIdx.x * kTileK + (threadIdx.x % kTileK);
    const int j = blockIdx.y * kTileJ + (threadIdx.x / kTileK);
    unsigned ncl = 0;
    for (int i = sb.b[slab]; i < sb.b[slab + 1]; ++i)
        sl_point<C, O, 2, TO, O == 4>(P, M, fn, fnm1, dt, out, i, j, k, ncl);
    add_clamps(nclamp, ncl);
}

// One foot per arrival point of component C, shared by the F.nf fields of
// that component: traced once through M over dt, clamped and counted once,
// one stencil built for the foot, and every field interpolated with it
// (SLAdvector.advect with extra_rhs interpolates each extra triple at the
// same departure points, semilag.py:584-671).  The per-field arithmetic is
// sl_point's MODE 0, so field 0 matches slc_advect.
struct MultiIO {
    const double *in[kMaxMultiFields];
    double *out[kMaxMultiFields];
    OutMap map[kMaxMultiFields];  // sx == 0: the ghost-shaped interior
    int nf;
};

template <int C, int O, int TO>
__global__ void __launch_bounds__(kThreads) k_advect_multi(const __grid_constant__ SlcParams P,
                                                           const __grid_constant__ Vel3 M,
                                                           const __grid_constant__ MultiIO F,
                                                           double dt, unsigned long long *nclamp)
{
    const int k = blockIdx.x * kTileK + (threadIdx.x % kTileK);
    const int j = blockIdx.y * kTileJ + (threadIdx.x / kTileK);
    const int i = blockIdx.z;
    const int nzi = (C == 2) ? P.nz - 1 : P.nz;
    unsigned ncl = 0;
    if (k < nzi && j < P.ny) {
        double xa, ya, za;
        arrival_point<C>(P, i, j, k, xa, ya, za);
        double us0, vs0, ws0;
        first_sample<C, TO>(P, M, i, j, k, xa, ya, za, us0, vs0, ws0);
        double xd, yd, zd;
        trace_foot<TO>(P, M, xa, ya, za, 0.5 * dt, us0, vs0, ws0, xd, yd, zd);
        if (zd < P.z_lo || zd > P.z_hi) ncl += 1;
        const double z = clampz(P, zd);
        const int c = face_cell(P, z);
        const NodeView<double> V0 = ghost_view<double>(C, F.in[0], P.nx, P.ny, P.nz);
        Stencil<O, double> st;
        build_stencil<C, O, double>(P, V0.sx, V0.sy, xd, yd, z, c, st);
        const GhostShape g = ghost_shape(C, P.nx, P.ny, P.nz);
        for (int f = 0; f < F.nf; ++f) {
            const NodeView<double> V = ghost_view<double>(C, F.in[f], P.nx, P.ny, P.nz);
            const double val = gather_sum<O, double, double>(V.p, st);
            const OutMap om = F.map[f];
            if (om.sx != 0)
                F.out[f][om.off + (long long)i * om.sx + (long long)j * om.sy + k] = val;
            else
                F.out[f][(size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z + (k + 1)] = val;
        }
    }
    if (nclamp) add_clamps(nclamp, ncl);
}

template <int C>
__global__ void __launch_bounds__(kThreads) k_departure(const __grid_constant__ SlcParams P, const __grid_constant__ Vel3 M, double dt,
                                                        double *xd, double *yd, double *zd)
{
    const int nzi = (C == 2) ? P.nz - 1 : P.nz;
    const long long n = (long long)P.nx * P.ny * nzi;
    const long long p = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (p >= n) return;
    const int k = (int)(p % nzi);
    const long long q = p / nzi;
    const int j = (int)(q % P.ny);
    const int i = (int)(q / P.ny);
    double xa, ya, za;
    arrival_point<C>(P, i, j, k, xa, ya, za);
    double us0, vs0, ws0;
    first_sample<C>(P, M, i, j, k, xa, ya, za, us0, vs0, ws0);
    trace_foot(P, M, xa, ya, za, 0.5 * dt, us0, vs0, ws0, xd[p], yd[p], zd[p]);
}

template <int C, int O>
__global__ void __launch_bounds__(kThreads) k_interp(SlcParams P, NodeView<double> F,
                                                     const double *x, const double *y,
                                                     const double *z, long long n, int count_clamp,
                                                     double *out, unsigned long long *nclamp)
{
    const long long p = (long long)blockIdx.x * kThreads + threadIdx.x;
    unsigned ncl = 0;
    if (p < n) {
        double zz = z[p];
        if (count_clamp) {
            if (zz < P.z_lo || zz > P.z_hi) ncl = 1;
            zz = clampz(P, zz);
        }
        int c = face_cell(P, zz);
        Stencil<O, double> st;
        build_stencil<C, O, double>(P, F.sx, F.sy, x[p], y[p], zz, c, st);
        out[p] = gather_sum<O, double, double>(F.p, st);
    }
    if (count_clamp) add_clamps(nclamp, ncl);
}

__global__ void k_face_coord(SlcParams P, const double *z, long long n, double *kf)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) kf[p] = face_coord(P, z[p]);
}

__global__ void k_lincomb(const double *__restrict__ a, const double *__restrict__ b, double ca,
                          double cb, double *__restrict__ out, long long n)
{
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x)
        out[p] = ca * a[p] + cb * b[p];
}

inline unsigned blocks_for(long long n, int t = kThreads) { return (unsigned)((n + t - 1) / t); }

Vel3 make_vel(const SlcParams &P, Tri mid, bool node)
{
    Vel3 M;
    if (node) {
        M.u = node_view<double>(mid.u, P.ny, P.nz + 2);
        M.v = node_view<double>(mid.v, P.ny, P.nz + 2);
        M.w = node_view<double>(mid.w, P.ny, P.nz + 1);
    } else {
        M.u = ghost_view<double>(0, mid.u, P.nx, P.ny, P.nz);
        M.v = ghost_view<double>(1, mid.v, P.nx, P.ny, P.nz);
        M.w = ghost_view<double>(2, mid.w, P.nx, P.ny, P.nz);
    }
    return M;
}

// Persistent BDF2 trace+gather over an ensemble's queue of (instance,
// component, x index, tile) items.  The grid is sized to the resident limit;
// each block takes the next item from an atomic counter, prefetched while it
// works on the current one.  The instance's SlcParams are copied to shared
// memory when the block moves to another instance.  Per point the arithmetic
// is sl_point's, so an instance's result does not depend on the tile shape
// or on the other instances.
template <int O>
__global__ void __launch_bounds__(kThreads, SLC_SL_ENS_MIN_BLOCKS) k_sl_ens(const EnsInst *__restrict__ ins,
                                                        const EnsItem *__restrict__ items,
                                                        int nitems, int ph, unsigned *queue)
{
    __shared__ SlcParams sP;
    __shared__ int s_item;
    if (threadIdx.x == 0) s_item = (int)atomicAdd(queue, 1u);
    int have = -1;
    for (;;) {
        __syncthreads();  // the previous item is done everywhere; s_item is published
        const int it = s_item;
        if (it >= nitems) break;
        const EnsItem w = items[it];
        if (w.inst != have) {
            const unsigned long long *src = (const unsigned long long *)&ins[w.inst].P;
            unsigned long long *dst = (unsigned long long *)&sP;
            for (int q = threadIdx.x; q < (int)(sizeof(SlcParams) / 8); q += kThreads) dst[q] = src[q];
            have = w.inst;
        }
        __syncthreads();  // sP ready; every thread has read s_item
        if (threadIdx.x == 0) s_item = (int)atomicAdd(queue, 1u);
        const EnsInst &I = ins[w.inst];
        const int tkl = I.tkl;
        const int k = ((w.c & 0xffff) << tkl) + (threadIdx.x & ((1 << tkl) - 1));
        const int j = ((w.c >> 16) << (8 - tkl)) + (threadIdx.x >> tkl);
        const int i = w.b;
        Vel3 M;
        M.u = ghost_view<double>(0, I.mid[0], sP.nx, sP.ny, sP.nz);
        M.v = ghost_view<double>(1, I.mid[1], sP.nx, sP.ny, sP.nz);
        M.w = ghost_view<double>(2, I.mid[2], sP.nx, sP.ny, sP.nz);
        const double *fn = I.lev[ens_cur(ph)][w.a];
        const double *fnm1 = I.lev[ens_prev(ph)][w.a];
        double *out = I.lev[ens_next(ph)][w.a];
        unsigned ncl = 0;
        if (w.a == 0) sl_point<0, O, 2, 0, true>(sP, M, fn, fnm1, I.dt, out, i, j, k, ncl);
        else if (w.a == 1) sl_point<1, O, 2, 0, true>(sP, M, fn, fnm1, I.dt, out, i, j, k, ncl);
        else sl_point<2, O, 2, 0, true>(sP, M, fn, fnm1, I.dt, out, i, j, k, ncl);
        add_clamps(I.ncl, ncl);
    }
}

__global__ void k_lincomb_ens(const EnsInst *__restrict__ ins, const EnsItem *__restrict__ items,
                              int ph, double ca, double cb)
{
    const EnsItem w = items[blockIdx.x];
    const EnsInst &I = ins[w.inst];
    const GhostShape g = ghost_shape(w.a, I.P.nx, I.P.ny, I.P.nz);
    const long long n = (long long)g.X * g.Y * g.Z;
    const double *a = I.lev[ens_cur(ph)][w.a], *b = I.lev[ens_prev(ph)][w.a];
    double *o = I.mid[w.a];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const long long p = (long long)w.b * 1024 + q * 256 + threadIdx.x;
        if (p < n) o[p] = ca * a[p] + cb * b[p];
    }
}

template <int O, int MODE, int TO>
void launch_sl_tt(const SlcParams &P, const Vel3 &M, Tri fn, Tri fnm1, double dt, TriMut out,
                  unsigned long long *ncl, cudaStream_t s)
{
    const dim3 gc((P.nz + kTileK - 1) / kTileK, (P.ny + kTileJ - 1) / kTileJ, P.nx);
    const dim3 gw((P.nz - 1 + kTileK - 1) / kTileK, (P.ny + kTileJ - 1) / kTileJ, P.nx);
    k_sl<0, O, MODE, TO><<<gc, kThreads, 0, s>>>(P, M, fn.u, fnm1.u, dt, out.u, ncl);
    k_sl<1, O, MODE, TO><<<gc, kThreads, 0, s>>>(P, M, fn.v, fnm1.v, dt, out.v, ncl);
    if (P.nz > 1) k_sl<2, O, MODE, TO><<<gw, kThreads, 0, s>>>(P, M, fn.w, fnm1.w, dt, out.w, ncl);
    count_launches(P.nz > 1 ? 3 : 2);
}

template <int O, int MODE>
void launch_sl_t(const SlcParams &P, const Vel3 &M, Tri fn, Tri fnm1, double dt, TriMut out,
                 unsigned long long *ncl, cudaStream_t s)
{
    if (P.traj_order == 4) launch_sl_tt<O, MODE, 4>(P, M, fn, fnm1, dt, out, ncl, s);
    else launch_sl_tt<O, MODE, 2>(P, M, fn, fnm1, dt, out, ncl, s);
}

}  // namespace

cudaError_t launch_sl(const SlcParams &P, int mode, Tri fn, Tri fnm1, Tri mid, bool mid_node,
                      double dt, TriMut out, unsigned long long *nclamp, cudaStream_t s)
{
    const Vel3 M = make_vel(P, mid, mid_node);
    if (P.order == 4) {
        if (mode == 0) launch_sl_t<4, 0>(P, M, fn, fnm1, dt, out, nclamp, s);
        else if (mode == 1) launch_sl_t<4, 1>(P, M, fn, fnm1, dt, out, nclamp, s);
        else launch_sl_t<4, 2>(P, M, fn, fnm1, dt, out, nclamp, s);
    } else {
        if (mode == 0) launch_sl_t<6, 0>(P, M, fn, fnm1, dt, out, nclamp, s);
        else if (mode == 1) launch_sl_t<6, 1>(P, M, fn, fnm1, dt, out, nclamp, s);
        else launch_sl_t<6, 2>(P, M, fn, fnm1, dt, out, nclamp, s);
    }
    return cudaGetLastError();
}

namespace {
template <int O, int TO>
void launch_slab_t(const SlcParams &P, int comp, const Vel3 &M, const double *fn, const double *fnm1,
                   double dt, double *out, unsigned long long *ncl, SlabGate *gate, int slab, int i0,
                   int i1, double limit, const SlabBounds *sb, cudaStream_t s)
{
    const int rows_k = comp == 2 ? P.nz - 1 : P.nz;
    const unsigned zt = (unsigned)((rows_k + kTileK - 1) / kTileK), yt = (unsigned)((P.ny + kTileJ - 1) / kTileJ);
    if (sb) {  // the fix launch: one block per (z, y) tile and slab
        const dim3 g(zt, yt, (unsigned)sb->S);
        if (comp == 0) k_sl_fix<0, O, TO><<<g, kThreads, 0, s>>>(P, M, fn, fnm1, dt, out, ncl, gate, *sb);
        else if (comp == 1) k_sl_fix<1, O, TO><<<g, kThreads, 0, s>>>(P, M, fn, fnm1, dt, out, ncl, gate, *sb);
        else k_sl_fix<2, O, TO><<<g, kThreads, 0, s>>>(P, M, fn, fnm1, dt, out, ncl, gate, *sb);
    } else {
        const dim3 g(zt, yt, (unsigned)(i1 - i0));
        if (comp == 0) k_sl_slab<0, O, TO><<<g, kThreads, 0, s>>>(P, M, fn, fnm1, dt, out, ncl, gate, slab, i0, limit);
        else if (comp == 1) k_sl_slab<1, O, TO><<<g, kThreads, 0, s>>>(P, M, fn, fnm1, dt, out, ncl, gate, slab, i0, limit);
        else k_sl_slab<2, O, TO><<<g, kThreads, 0, s>>>(P, M, fn, fnm1, dt, out, ncl, gate, slab, i0, limit);
    }
    count_launches(1);
}

cudaError_t launch_slab_any(const SlcParams &P, int comp, const double *fn, const double *fnm1, Tri mid,
                            double dt, double *out, unsigned long long *ncl, SlabGate *gate, int slab,
                            int i0, int i1, double limit, const SlabBounds *sb, cudaStream_t s)
{
    if (comp < 0 || comp > 2 || (comp == 2 && P.nz <= 1)) return cudaErrorInvalidValue;
    if (!sb && i1 <= i0) return cudaSuccess;
    const Vel3 M = make_vel(P, mid, false);
    const bool t4 = P.traj_order == 4;
    if (P.order == 4) {
        if (t4) launch_slab_t<4, 4>(P, comp, M, fn, fnm1, dt, out, ncl, gate, slab, i0, i1, limit, sb, s);
        else launch_slab_t<4, 2>(P, comp, M, fn, fnm1, dt, out, ncl, gate, slab, i0, i1, limit, sb, s);
    } else {
        if (t4) launch_slab_t<6, 4>(P, comp, M, fn, fnm1, dt, out, ncl, gate, slab, i0, i1, limit, sb, s);
        else launch_slab_t<6, 2>(P, comp, M, fn, fnm1, dt, out, ncl, gate, slab, i0, i1, limit, sb, s);
    }
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_sl_slab(const SlcParams &P, int comp, const double *fn, const double *fnm1, Tri mid,
                           double dt, double *out, unsigned long long *nclamp, SlabGate *gate, int slab,
                           int i0, int i1, double limit, cudaStream_t s)
{
    return launch_slab_any(P, comp, fn, fnm1, mid, dt, out, nclamp, gate, slab, i0, i1, limit, nullptr, s);
}

cudaError_t launch_sl_fix(const SlcParams &P, int comp, const double *fn, const double *fnm1, Tri mid,
                          double dt, double *out, unsigned long long *nclamp, const SlabGate *gate,
                          const SlabBounds &sb, cudaStream_t s)
{
    return launch_slab_any(P, comp, fn, fnm1, mid, dt, out, nclamp, const_cast<SlabGate *>(gate), 0, 0, 0,
                           0.0, &sb, s);
}

namespace {
template <int O, int TO>
void launch_multi_t(const SlcParams &P, const MultiIO *io, const Vel3 &M, double dt,
                    unsigned long long *ncl, cudaStream_t s)
{
    const dim3 gc((P.nz + kTileK - 1) / kTileK, (P.ny + kTileJ - 1) / kTileJ, P.nx);
    const dim3 gw((P.nz - 1 + kTileK - 1) / kTileK, (P.ny + kTileJ - 1) / kTileJ, P.nx);
    k_advect_multi<0, O, TO><<<gc, kThreads, 0, s>>>(P, M, io[0], dt, ncl);
    k_advect_multi<1, O, TO><<<gc, kThreads, 0, s>>>(P, M, io[1], dt, ncl);
    if (P.nz > 1) k_advect_multi<2, O, TO><<<gw, kThreads, 0, s>>>(P, M, io[2], dt, ncl);
    count_launches(P.nz > 1 ? 3 : 2);
}
}  // namespace

cudaError_t launch_advect_multi(const SlcParams &P, int nf, const double *const *in,
                                double *const *out, const OutMap *maps, Tri mid, double dt,
                                unsigned long long *nclamp, cudaStream_t s)
{
    if (nf < 1 || nf > kMaxMultiFields) return cudaErrorInvalidValue;
    MultiIO io[3];
    for (int c = 0; c < 3; ++c) {
        io[c].nf = nf;
        for (int f = 0; f < nf; ++f) {
            io[c].in[f] = in[3 * f + c];
            io[c].out[f] = out[3 * f + c];
            io[c].map[f] = maps[3 * f + c];
        }
    }
    const Vel3 M = make_vel(P, mid, false);
    const bool t4 = P.traj_order == 4;
    if (P.order == 4) {
        if (t4) launch_multi_t<4, 4>(P, io, M, dt, nclamp, s);
        else launch_multi_t<4, 2>(P, io, M, dt, nclamp, s);
    } else {
        if (t4) launch_multi_t<6, 4>(P, io, M, dt, nclamp, s);
        else launch_multi_t<6, 2>(P, io, M, dt, nclamp, s);
    }
    return cudaGetLastError();
}

cudaError_t launch_departure(const SlcParams &P, int comp, Tri mid_node, double dt, double *xd,
                             double *yd, double *zd, cudaStream_t s)
{
    const Vel3 M = make_vel(P, mid_node, true);
    const long long n = (long long)P.nx * P.ny * (comp == 2 ? P.nz - 1 : P.nz);
    if (n <= 0) return cudaSuccess;
    if (comp == 0) k_departure<0><<<blocks_for(n), kThreads, 0, s>>>(P, M, dt, xd, yd, zd);
    else if (comp == 1) k_departure<1><<<blocks_for(n), kThreads, 0, s>>>(P, M, dt, xd, yd, zd);
    else k_departure<2><<<blocks_for(n), kThreads, 0, s>>>(P, M, dt, xd, yd, zd);
    count_launches(1);
    return cudaGetLastError();
}

namespace {
template <int C>
void launch_interp_c(const SlcParams &P, int order, NodeView<double> F, const double *x,
                     const double *y, const double *z, long long n, int cc, double *out,
                     unsigned long long *ncl, cudaStream_t s)
{
    if (order == 2) k_interp<C, 2><<<blocks_for(n), kThreads, 0, s>>>(P, F, x, y, z, n, cc, out, ncl);
    else if (order == 4) k_interp<C, 4><<<blocks_for(n), kThreads, 0, s>>>(P, F, x, y, z, n, cc, out, ncl);
    else k_interp<C, 6><<<blocks_for(n), kThreads, 0, s>>>(P, F, x, y, z, n, cc, out, ncl);
}
}  // namespace

cudaError_t launch_interp(const SlcParams &P, int comp, int order, const double *buf,
                          const double *x, const double *y, const double *z, int64_t n,
                          int count_clamp, double *out, unsigned long long *nclamp,
                          cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    const int NZ = comp == 2 ? P.nz + 1 : P.nz + 2;
    const NodeView<double> F = node_view<double>(buf, P.ny, NZ);
    if (comp == 0) launch_interp_c<0>(P, order, F, x, y, z, n, count_clamp, out, nclamp, s);
    else if (comp == 1) launch_interp_c<1>(P, order, F, x, y, z, n, count_clamp, out, nclamp, s);
    else launch_interp_c<2>(P, order, F, x, y, z, n, count_clamp, out, nclamp, s);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_face_coord(const SlcParams &P, const double *z, int64_t n, double *kf,
                              cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_face_coord<<<blocks_for(n), kThreads, 0, s>>>(P, z, n, kf);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_lincomb(const double *a, const double *b, double ca, double cb, double *out,
                           int64_t n, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    unsigned blocks = blocks_for(n);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_lincomb<<<blocks, kThreads, 0, s>>>(a, b, ca, cb, out, n);
    count_launches(1);
    return cudaGetLastError();
}

int sl_ens_blocks_per_sm()
{
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_sl_ens<6>, kThreads, 0) != cudaSuccess)
        return 1;
    int nb4 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb4, k_sl_ens<4>, kThreads, 0) != cudaSuccess)
        return 1;
    const int m = nb < nb4 ? nb : nb4;
    return m > 0 ? m : 1;
}

cudaError_t launch_sl_ens(const EnsInst *ins, const EnsItem *items, int nitems, int ph, int order,
                          unsigned *queue, int grid, cudaStream_t s)
{
    if (nitems <= 0) return cudaSuccess;
    if (order == 4) k_sl_ens<4><<<grid, kThreads, 0, s>>>(ins, items, nitems, ph, queue);
    else k_sl_ens<6><<<grid, kThreads, 0, s>>>(ins, items, nitems, ph, queue);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_lincomb_ens(const EnsInst *ins, const EnsItem *items, int nitems, int ph,
                               cudaStream_t s)
{
    if (nitems <= 0) return cudaSuccess;
    k_lincomb_ens<<<nitems, 256, 0, s>>>(ins, items, ph, 2.0, -1.0);
    count_launches(1);
    return cudaGetLastError();
}
