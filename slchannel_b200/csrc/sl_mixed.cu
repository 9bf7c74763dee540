// sl_mixed.cu -- the mixed-precision form of the SL trace + gather (sm_100a).
//
// Each advected and trajectory field is split into its FP64 plane-mean profile
// m(k) (the x,y average at every z level) and an FP32 fluctuation f = V - m
// stored as a padded node buffer (nx, ny, NZp).  The characteristic trace and
// the order^3 gather read the FP32 fluctuations with FP32 weights and FP32
// accumulation, and add the mean profile interpolated in z in FP64; positions,
// stencil location, the BDF epilogue (with the FP64 explicit x,y diffusion)
// and everything after the predictor stay FP64.  The reference's counterpart
// is its 'fp32_accum64' path (semilag.py:249-256, semilag_triton.py), which
// runs the whole interpolation in FP32 instead.
#include <algorithm>
#include <climits>

#include "slc_internal.h"
#include "slc_tma.cuh"

namespace {

constexpr int kThreads = 256;
#ifndef SLC_SLM_TILE_K
#define SLC_SLM_TILE_K 32
#endif
constexpr int kTileK = SLC_SLM_TILE_K, kTileJ = kThreads / kTileK;


// resident blocks per SM the mixed trace+gather kernel is compiled for
#ifndef SLC_SLM_MIN_BLOCKS
#define SLC_SLM_MIN_BLOCKS 4
#endif
#ifndef SLC_SLM_ENS_MIN_BLOCKS  // the persistent ensemble form (more live state)
#define SLC_SLM_ENS_MIN_BLOCKS 3
#endif
constexpr int kMeanBlocks = 148;  // column groups of the plane-mean partial sums

struct Vel3M {
    MixedView u, v, w;
};

__device__ __forceinline__ void add_clamps(unsigned long long *counter, unsigned cnt)
{
    unsigned tot = __reduce_add_sync(0xffffffffu, cnt);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(counter, (unsigned long long)tot);
}

// ---- FP32 characteristic trace -------------------------------------------
// A trajectory point is its arrival point plus an FP32 displacement.  In
// index space (s = x/dx + shift) the arrival point is an integer or a
// half-integer for both shifts 0 and -1/2, kept as an exact int part and a
// float fraction in {0, 1/2}; adding the (small) displacement to the
// fraction keeps positions accurate to FP32 round-off of a few cells, not of
// the domain.  z is an absolute FP32 coordinate (z in [0, Lz]).
struct Arr32 {
    int xa, xb, ya, yb;      // integer parts for shift 0 (a) and -1/2 (b)
    float fxa, fxb, fya, fyb;
    double za;               // arrival height (exact); z = za + dz, dz FP32
    float dzlo, dzhi;        // clamp bounds z_lo - za, z_hi - za
};

template <int C>
__device__ __forceinline__ Arr32 arrival32(const SlcParams &P, int i, int j, int k)
{
    Arr32 a;
    if (C == 0) {  // u: x = (i+1) dx, y = (j+1/2) dy, z = z_c[k+1]
        a.xa = i + 1; a.fxa = 0.f; a.xb = i; a.fxb = 0.5f;
        a.ya = j; a.fya = 0.5f; a.yb = j; a.fyb = 0.f;
        a.za = __ldg(P.zc + k + 1);
    } else if (C == 1) {  // v: x = (i+1/2) dx, y = (j+1) dy, z = z_c[k+1]
        a.xa = i; a.fxa = 0.5f; a.xb = i; a.fxb = 0.f;
        a.ya = j + 1; a.fya = 0.f; a.yb = j; a.fyb = 0.5f;
        a.za = __ldg(P.zc + k + 1);
    } else {  // w: x = (i+1/2) dx, y = (j+1/2) dy, z = z_f[k+1]
        a.xa = i; a.fxa = 0.5f; a.xb = i; a.fxb = 0.f;
        a.ya = j; a.fya = 0.5f; a.yb = j; a.fyb = 0.f;
        a.za = __ldg(P.zf + k + 1);
    }
    a.dzlo = (float)(P.z_lo - a.za);
    a.dzhi = (float)(P.z_hi - a.za);
    return a;
}

__device__ __forceinline__ int wrap_int(int v, int n)
{
    if (v >= 0 && v < n) return v;
    int r = v % n;
    return r < 0 ? r + n : r;
}

// Cell base and fraction of index-space coordinate (ip + fr), any float fr
// (NaN or huge displacements end inside the period).
__device__ __forceinline__ void split32(int ip, float fr, int n, int &base, float &t)
{
    fr = fminf(fmaxf(fr, -1.0e6f), 1.0e6f);
    const float fl = floorf(fr);
    t = fr - fl;
    base = wrap_int(ip + (int)fl, n);
}

// Height displacement clamped so that za + dz stays in [z_lo, z_hi].
__device__ __forceinline__ float clampdz(const Arr32 &A, float dz)
{
    return dz < A.dzlo ? A.dzlo : (dz > A.dzhi ? A.dzhi : dz);
}

// FP32 face cell (analytic inverse tanh map, semilag.py:400-416).
__device__ __forceinline__ int face_cell32(const SlcParams &P, float z)
{
    const float lim = 0.99999994f;
    float kf;
    if (P.symmetric) {
        float arg = (z * (float)P.two_over_Lz - 1.0f) * (float)P.tanh_g;
        arg = fminf(fmaxf(arg, -lim), lim);
        kf = (atanhf(arg) * (float)P.inv_gamma + 1.0f) * (float)P.half_nz;
    } else {
        float arg = (1.0f - z * (float)P.inv_Lz) * (float)P.tanh_g;
        arg = fminf(fmaxf(arg, -lim), lim);
        kf = (1.0f - atanhf(arg) * (float)P.inv_gamma) * (float)P.nzd;
    }
    kf = fminf(fmaxf(floorf(kf), 0.0f), (float)(P.nz - 1));
    return (int)kf;
}

__device__ __forceinline__ float tri32(MixedView V, int i0, int i1, float tx, int j0, int j1,
                                       float ty, int k0, float wz0, float wz1)
{
    const NodeView<float> F = V.f;
    const float *p00 = F.p + i0 * F.sx + j0 * F.sy + k0;
    const float *p01 = F.p + i0 * F.sx + j1 * F.sy + k0;
    const float *p10 = F.p + i1 * F.sx + j0 * F.sy + k0;
    const float *p11 = F.p + i1 * F.sx + j1 * F.sy + k0;
    const float a00 = wz0 * __ldg(p00) + wz1 * __ldg(p00 + 1);
    const float a01 = wz0 * __ldg(p01) + wz1 * __ldg(p01 + 1);
    const float a10 = wz0 * __ldg(p10) + wz1 * __ldg(p10 + 1);
    const float a11 = wz0 * __ldg(p11) + wz1 * __ldg(p11 + 1);
    const float fl = (1.f - tx) * ((1.f - ty) * a00 + ty * a01) + tx * ((1.f - ty) * a10 + ty * a11);
    return fl + (wz0 * __ldg(V.mean32 + k0) + wz1 * __ldg(V.mean32 + k0 + 1));
}

// Trajectory velocity at arrival + (ddx, ddy) (index units) and height
// za + dz.  Heights enter the weights as differences formed in FP64 (an FP32
// absolute height near z = Lz would carry ~1e-7 absolute error, a sizeable
// fraction of the near-wall spacing).
__device__ __forceinline__ void sample3_32(const SlcParams &P, const Vel3M &M, const Arr32 &A,
                                           float ddx, float ddy, float dz, float &us, float &vs,
                                           float &ws)
{
    int ia0, ib0, ja0, jb0;
    float txa, txb, tya, tyb;
    split32(A.xa, A.fxa + ddx, P.nx, ia0, txa);
    split32(A.xb, A.fxb + ddx, P.nx, ib0, txb);
    split32(A.ya, A.fya + ddy, P.ny, ja0, tya);
    split32(A.yb, A.fyb + ddy, P.ny, jb0, tyb);
    const int ia1 = (ia0 + 1 == P.nx) ? 0 : ia0 + 1, ib1 = (ib0 + 1 == P.nx) ? 0 : ib0 + 1;
    const int ja1 = (ja0 + 1 == P.ny) ? 0 : ja0 + 1, jb1 = (jb0 + 1 == P.ny) ? 0 : jb0 + 1;
    const double z = A.za + (double)dz;
    const int c = face_cell32(P, (float)z);
    const int kc = min(max(c + (z >= __ldg(P.zc + c + 1) ? 1 : 0), 0), P.nz);
    const int kf = min(max(c, 0), P.nz - 1);
    const float *dc = P.dinv_c32[2] + kc;  // order-2 tables: nz+1 / nz rows
    const float *df = P.dinv_f32[2] + kf;
    const float wc0 = (float)(z - __ldg(P.zc + kc + 1)) * __ldg(dc);
    const float wc1 = (float)(z - __ldg(P.zc + kc)) * __ldg(dc + P.nz + 1);
    const float wf0 = (float)(z - __ldg(P.zf + kf + 1)) * __ldg(df);
    const float wf1 = (float)(z - __ldg(P.zf + kf)) * __ldg(df + P.nz);
    us = tri32(M.u, ia0, ia1, txa, jb0, jb1, tyb, kc, wc0, wc1);
    vs = tri32(M.v, ib0, ib1, txb, ja0, ja1, tya, kc, wc0, wc1);
    ws = tri32(M.w, ib0, ib1, txb, jb0, jb1, tyb, kf, wf0, wf1);
}

// Tricubic trajectory velocity (traj_interp_order 4), defined below.
__device__ __noinline__ void sample3_32_o4(const SlcParams &P, const Vel3M &M, const Arr32 &A,
                                           float ddx, float ddy, float dz, float &us, float &vs,
                                           float &ws);

// Iterated midpoint rule (semilag.py:542-552) in FP32 displacements; returns
// the foot as displacements from the arrival point (x, y in index units).
// TO: trajectory sampling order 2 or 4, or 0 to read P.traj_order.
template <int TO>
__device__ __forceinline__ void trace_foot32(const SlcParams &P, const Vel3M &M, const Arr32 &A,
                                             float hdt, float us0, float vs0, float ws0,
                                             float &ddx, float &ddy, float &ddz)
{
    const float idx = (float)P.inv_dx, idy = (float)P.inv_dy;
    float mx = -hdt * us0 * idx;
    float my = -hdt * vs0 * idy;
    float mz = clampdz(A, -hdt * ws0);
    for (int it = 1; it < P.n_iters; ++it) {
        float us, vs, ws;
        if (TO == 4 || (TO == 0 && P.traj_order == 4)) sample3_32_o4(P, M, A, mx, my, mz, us, vs, ws);
        else sample3_32(P, M, A, mx, my, mz, us, vs, ws);
        mx = -hdt * us * idx;
        my = -hdt * vs * idy;
        mz = clampdz(A, -hdt * ws);
    }
    ddx = 2.f * mx;
    ddy = 2.f * my;
    ddz = 2.f * mz;
}

// Clamp-and-count the foot and interpolate the mixed field F there: FP32
// weights and accumulation for the fluctuation, the FP64 mean profile through
// the (FP32) z weights.  MEAN32: the mean profile rounded to FP32 and summed
// in FP32 instead, as the trajectory samples do.
template <int C, int O, bool MEAN32 = false>
__device__ __forceinline__ double gather_foot32(const SlcParams &P, MixedView F, const Arr32 &A,
                                                float ddx, float ddy, float ddz, unsigned &ncl)
{
    constexpr int h = O / 2 - 1;
    const int NZ = Comp<C>::centers ? P.nz + 2 : P.nz + 1;
    if (ddz < A.dzlo || ddz > A.dzhi) ncl += 1;
    const double z = A.za + (double)clampdz(A, ddz);
    const int xi = (C == 0) ? A.xa : A.xb;
    const float xf = (C == 0) ? A.fxa : A.fxb;
    const int yi = (C == 1) ? A.ya : A.yb;
    const float yf = (C == 1) ? A.fya : A.fyb;
    int bx, by;
    float tx, ty;
    split32(xi, xf + ddx, P.nx, bx, tx);
    split32(yi, yf + ddy, P.ny, by, ty);
    StencilM<O> st;
#pragma unroll
    for (int m = 0; m < O; ++m) st.xoff[m] = wrap_index(bx + m - h, P.nx) * F.f.sx;
#pragma unroll
    for (int m = 0; m < O; ++m) st.yoff[m] = wrap_index(by + m - h, P.ny) * F.f.sy;
    uniform_weights<O, float>(P, tx, st.wx);
    uniform_weights<O, float>(P, ty, st.wy);
    const int c = face_cell32(P, (float)z);
    const int m0 = Comp<C>::centers ? c + (z >= __ldg(P.zc + c + 1) ? 1 : 0) : c;
    const int k0 = min(max(m0 - h, 0), NZ - O);
    st.k0 = k0;
    // z - z_node from the FP64 node table: FP32-rounded nodes would break
    // sum(weights) = 1 at the level of (round-off / spacing), biasing the
    // interpolant in proportion to the field itself
    {
        const double *zn = Comp<C>::centers ? P.zc : P.zf;
        const float *di = (Comp<C>::centers ? P.dinv_c32[O] : P.dinv_f32[O]) + k0;
        float d[O], pre[O];
#pragma unroll
        for (int l = 0; l < O; ++l) d[l] = (float)(z - __ldg(zn + k0 + l));
        pre[0] = 1.f;
#pragma unroll
        for (int l = 1; l < O; ++l) pre[l] = pre[l - 1] * d[l - 1];
        float suf = 1.f;
#pragma unroll
        for (int m = O - 1; m >= 0; --m) {
            st.wz[m] = pre[m] * suf * __ldg(di + m * (NZ - O + 1));
            suf = suf * d[m];
        }
    }
    float acc = 0.f;
#pragma unroll
    for (int i = 0; i < O; ++i) {
        float accy = 0.f;
#pragma unroll
        for (int j = 0; j < O; ++j) {
            const float *row = F.f.p + st.xoff[i] + st.yoff[j] + k0;
            float accz = 0.f;
#pragma unroll
            for (int k = 0; k < O; ++k) accz = fmaf(st.wz[k], __ldg(row + k), accz);
            accy = fmaf(st.wy[j], accz, accy);
        }
        acc = fmaf(st.wx[i], accy, acc);
    }
    if constexpr (MEAN32) {
        float m = 0.f;
#pragma unroll
        for (int k = 0; k < O; ++k) m = fmaf(st.wz[k], __ldg(F.mean32 + k0 + k), m);
        return (double)(acc + m);
    }
    double mean = 0.0;
#pragma unroll
    for (int k = 0; k < O; ++k) mean = fma((double)st.wz[k], __ldg(F.mean + k0 + k), mean);
    return (double)acc + mean;
}

// The trajectory velocity with tricubic Lagrange sampling (traj_interp_order
// 4, semilag.py:206-209, 512-528): the order-4 mixed gather of each U*
// component at arrival + displacement, on that component's own node grid
// (gather_foot32 picks the grid's shifts from the arrival record), all in
// FP32 like the trilinear samples (FP32 mean profile).  The midpoint is
// already inside [z_lo, z_hi]; no clamp is counted.
__device__ __noinline__ void sample3_32_o4(const SlcParams &P, const Vel3M &M, const Arr32 &A,
                                           float ddx, float ddy, float dz, float &us, float &vs,
                                           float &ws)
{
    unsigned none = 0;
    us = (float)gather_foot32<0, 4, true>(P, M.u, A, ddx, ddy, dz, none);
    vs = (float)gather_foot32<1, 4, true>(P, M.v, A, ddx, ddy, dz, none);
    ws = (float)gather_foot32<2, 4, true>(P, M.w, A, ddx, ddy, dz, none);
}

struct NodeValMixed32 {
    __device__ __forceinline__ double operator()(MixedView V, int I, int J, int K) const
    {
        return (double)(__ldg(V.f.p + I * V.f.sx + J * V.f.sy + K) + __ldg(V.mean32 + K));
    }
};

template <int C>
__device__ __forceinline__ double xy_diffusion64(const SlcParams &P, const double *__restrict__ f,
                                                 int i, int j, int k)
{
    const GhostShape g = ghost_shape(C, P.nx, P.ny, P.nz);
    const size_t sx = (size_t)g.Y * g.Z, sy = g.Z;
    const int I = i + 1, J = j + 1, K = k + 1;
    int Ip = I + 1, Jp = J + 1;
    if (C == 0 && Ip == P.nx + 1) Ip = 1;
    if (C == 1 && Jp == P.ny + 1) Jp = 1;
    const double fc = __ldg(f + I * sx + J * sy + K);
    const double d2x =
        (__ldg(f + Ip * sx + J * sy + K) - 2.0 * fc + __ldg(f + (I - 1) * sx + J * sy + K)) * P.inv_dx2;
    const double d2y =
        (__ldg(f + I * sx + Jp * sy + K) - 2.0 * fc + __ldg(f + I * sx + (J - 1) * sy + K)) * P.inv_dy2;
    return P.nu * (d2x + d2y);
}

// MODE 0: one foot of A (advect); 1: BDF1 predictor; 2: BDF2 predictor.
// FA/FB: the mixed views of the near (V^n) and far (V^{n-1}) fields of
// component C; fn/fnm1: the same fields in FP64 (ghost-shaped) for R.
// FAR_FIRST: trace the far foot before the near foot's gather, so the two
// traces' loads overlap.  That pays in the persistent ensemble kernel (2 %
// at 48 channels, where it also spills less) but not in the single-grid one
// at its 64-register cap (52 bytes of spill, 0.8 % slower at 256^3; at three
// blocks per SM and 80 registers it is 7 % slower).
template <int C, int O, int MODE, int TO = 0, bool FAR_FIRST = false>
__device__ __forceinline__ void sl_point_mixed(const SlcParams &P, const Vel3M &M, const MixedView &FA,
                                               const MixedView &FB, const double *__restrict__ fn,
                                               const double *__restrict__ fnm1, double dt,
                                               double *__restrict__ out, int i, int j, int k,
                                               unsigned &ncl, OutMap om = OutMap{0, 0, 0})
{
    const int nzi = (C == 2) ? P.nz - 1 : P.nz;
    if (k < nzi && j < P.ny) {
        const Arr32 A = arrival32<C>(P, i, j, k);
        // first fixed-point sample at the arrival point: exact node values
        // for trilinear sampling, the tricubic stencils otherwise
        float us0, vs0, ws0;
        if (TO == 4 || (TO == 0 && P.traj_order == 4)) {
            sample3_32_o4(P, M, A, 0.f, 0.f, 0.f, us0, vs0, ws0);
        } else {
            double u0, v0, w0;
            arrival_sample<C>(P, M, i, j, k, NodeValMixed32(), u0, v0, w0);
            us0 = (float)u0;
            vs0 = (float)v0;
            ws0 = (float)w0;
        }
        float ddx, ddy, ddz;
        trace_foot32<TO>(P, M, A, (float)(0.5 * dt), us0, vs0, ws0, ddx, ddy, ddz);
        float fdx = 0.f, fdy = 0.f, fdz = 0.f;
        if (MODE == 2 && FAR_FIRST) trace_foot32<TO>(P, M, A, (float)dt, us0, vs0, ws0, fdx, fdy, fdz);
        const double ubar = gather_foot32<C, O>(P, FA, A, ddx, ddy, ddz, ncl);
        double res;
        if (MODE == 0) {
            res = ubar;
        } else if (MODE == 1) {
            res = ubar + dt * xy_diffusion64<C>(P, fn, i, j, k);
        } else {
            if (FAR_FIRST) {
                ddx = fdx;
                ddy = fdy;
                ddz = fdz;
            } else {
                trace_foot32<TO>(P, M, A, (float)dt, us0, vs0, ws0, ddx, ddy, ddz);
            }
            const double ubb = gather_foot32<C, O>(P, FB, A, ddx, ddy, ddz, ncl);
            const double Rn = xy_diffusion64<C>(P, fn, i, j, k);
            const double Rh = P.xy_lagged ? Rn : 2.0 * Rn - xy_diffusion64<C>(P, fnm1, i, j, k);
            res = ubar * (4.0 / 3.0) + ubb * (-1.0 / 3.0);
            res = res + ((2.0 / 3.0) * dt) * Rh;
        }
        if (MODE == 0 && om.sx != 0) {
            out[om.off + (long long)i * om.sx + (long long)j * om.sy + k] = res;
        } else {
            const GhostShape g = ghost_shape(C, P.nx, P.ny, P.nz);
            out[(size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z + (k + 1)] = res;
        }
    }
}

// om: where MODE 0 stores its results (ghost-shaped when om.sx == 0).
template <int C, int O, int MODE, int TO>
__global__ void __launch_bounds__(kThreads, SLC_SLM_MIN_BLOCKS)
    k_sl_mixed(const __grid_constant__ SlcParams P, const __grid_constant__ Vel3M M,
               const __grid_constant__ MixedView FA, const __grid_constant__ MixedView FB,
               const double *__restrict__ fn,
               const double *__restrict__ fnm1, double dt, double *__restrict__ out,
               unsigned long long *nclamp, const OutMap om)
{
    const int k = blockIdx.x * kTileK + (threadIdx.x % kTileK);
    const int j = blockIdx.y * kTileJ + (threadIdx.x / kTileK);
    const int i = blockIdx.z;
    unsigned ncl = 0;
    sl_point_mixed<C, O, MODE, TO>(P, M, FA, FB, fn, fnm1, dt, out, i, j, k, ncl, om);
    add_clamps(nclamp, ncl);
}

// ---- the BDF2 trace+gather with TMA-staged FP32 boxes ------------------------
// A block is 2 (x) x 4 (y) x 32 (z) arrival points, one warp per 32 z, with
// one box buffer.  Its threads trace the near foot (the FP32 trace above);
// the block takes the min and max of the feet's stencil bases, and where the
// bounding box fits kMBX x kMBY x kMBZ nodes one thread loads it by TMA (no
// multicast) from the halo-padded FP32 copy of V^n onto an mbarrier and the
// threads gather from it; then the far foot goes through the same buffer
// from the copy of V^{n-1}.  A box row is 64 floats = 256 bytes, two whole
// bank cycles, so a lane whose stencil base moved one row in x or y (the
// floor of its foot coordinate flipped) keeps its bank.  Blocks whose feet
// spread wider gather through L1 from the same padded copies.  Weights, the
// contraction order and the FP64 mean term are gather_foot32's, so the
// results equal k_sl_mixed's.
constexpr int kMTI = 2, kMTJ = 4, kMTK = 32;   // arrival tile (x, y, z)
// staged box (x, y, z) in nodes: 30.7 KB, five blocks per SM (48 registers).
// Measured at 256^3 (mixed trace+gather per step): both feet's boxes at
// once, 10 x 10 at four blocks per SM 6.04 ms (10 x 12 at three 6.56, two
// blocks 7.98); one buffer, 10 x 10 at four 6.12, at five 5.94, at six 6.11,
// 10 x 12 at five 5.99 ms, kept for the room it leaves feet that spread.
#ifndef SLC_SLMT_BOX_Y
#define SLC_SLMT_BOX_Y 12
#endif
constexpr int kMBX = 10, kMBY = SLC_SLMT_BOX_Y, kMBZ = 64;
constexpr int kMBoxElems = kMBX * kMBY * kMBZ;
constexpr size_t kMBoxBytes = (size_t)kMBoxElems * sizeof(float);
#ifndef SLC_SLMT_MIN_BLOCKS
#define SLC_SLMT_MIN_BLOCKS 5
#endif
static_assert(kMTI * kMTJ * kMTK == kThreads, "one thread per arrival point");
static_assert((kMBZ * sizeof(float)) % 128 == 0, "box rows of whole bank cycles");

#ifndef SLC_SLMT_F32X2  // packed FP32x2 FMAs in the box gather: 5.99 -> 5.81 ms per step at 256^3
#define SLC_SLMT_F32X2 1
#endif
__device__ __forceinline__ unsigned long long pack_f32x2(float lo, float hi)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void unpack_f32x2(unsigned long long v, float &lo, float &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long fma_f32x2(unsigned long long a, unsigned long long b,
                                                       unsigned long long c)
{
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// A foot located for the staged gather: x and y stencil bases (unwrapped,
// relative to the tile origin), their fractions, the clamped height and the
// z base; split32's and gather_foot32's arithmetic without the wrap.
struct FootM32 {
    double z;
    float tx, ty;
    int rx, ry, k0;
};

template <int C, int O>
__device__ __forceinline__ FootM32 locate_foot_m32(const SlcParams &P, const Arr32 &A, float ddx, float ddy,
                                                   float ddz, int i0, int j0, unsigned &ncl)
{
    constexpr int h = O / 2 - 1;
    const int NZ = Comp<C>::centers ? P.nz + 2 : P.nz + 1;
    if (ddz < A.dzlo || ddz > A.dzhi) ncl += 1;
    FootM32 F;
    F.z = A.za + (double)clampdz(A, ddz);
    const int xi = (C == 0) ? A.xa : A.xb;
    const float xf = (C == 0) ? A.fxa : A.fxb;
    const int yi = (C == 1) ? A.ya : A.yb;
    const float yf = (C == 1) ? A.fya : A.fyb;
    float fr = fminf(fmaxf(xf + ddx, -1.0e6f), 1.0e6f);
    float fl = floorf(fr);
    F.tx = fr - fl;
    F.rx = xi + (int)fl - h - i0;
    fr = fminf(fmaxf(yf + ddy, -1.0e6f), 1.0e6f);
    fl = floorf(fr);
    F.ty = fr - fl;
    F.ry = yi + (int)fl - h - j0;
    const int c = face_cell32(P, (float)F.z);
    const int m0 = Comp<C>::centers ? c + (F.z >= __ldg(P.zc + c + 1) ? 1 : 0) : c;
    F.k0 = min(max(m0 - h, 0), NZ - O);
    return F;
}

// gather_foot32's weights and contraction over a staged box (ox, oy, oz:
// the stencil's first node inside the box) plus its FP64 mean term.
template <int C, int O>
__device__ __forceinline__ double gather_box_m32(const SlcParams &P, const MixedView &F, const float *box,
                                                 const FootM32 &f, int ox, int oy, int oz)
{
    const int NZ = Comp<C>::centers ? P.nz + 2 : P.nz + 1;
    float wx[O], wy[O], wz[O];
    uniform_weights<O, float>(P, f.tx, wx);
    uniform_weights<O, float>(P, f.ty, wy);
    {
        const double *zn = Comp<C>::centers ? P.zc : P.zf;
        const float *di = (Comp<C>::centers ? P.dinv_c32[O] : P.dinv_f32[O]) + f.k0;
        float d[O], pre[O];
#pragma unroll
        for (int l = 0; l < O; ++l) d[l] = (float)(f.z - __ldg(zn + f.k0 + l));
        pre[0] = 1.f;
#pragma unroll
        for (int l = 1; l < O; ++l) pre[l] = pre[l - 1] * d[l - 1];
        float suf = 1.f;
#pragma unroll
        for (int m = O - 1; m >= 0; --m) {
            wz[m] = pre[m] * suf * __ldg(di + m * (NZ - O + 1));
            suf = suf * d[m];
        }
    }
    const float *b = box + (ox * kMBY + oy) * kMBZ + oz;
    float acc = 0.f;
#if SLC_SLMT_F32X2
    // two rows' z contractions per packed FP32x2 FMA (each lane an IEEE fma,
    // so the sums equal the scalar ones)
    unsigned long long w2[O];
#pragma unroll
    for (int k = 0; k < O; ++k) w2[k] = pack_f32x2(wz[k], wz[k]);
#pragma unroll
    for (int i = 0; i < O; ++i) {
        float accy = 0.f;
#pragma unroll
        for (int j = 0; j < O; j += 2) {
            const float *r0 = b + (i * kMBY + j) * kMBZ, *r1 = r0 + kMBZ;
            unsigned long long a2 = 0ull;  // (+0, +0)
#pragma unroll
            for (int k = 0; k < O; ++k) a2 = fma_f32x2(w2[k], pack_f32x2(r0[k], r1[k]), a2);
            float z0, z1;
            unpack_f32x2(a2, z0, z1);
            accy = fmaf(wy[j], z0, accy);
            accy = fmaf(wy[j + 1], z1, accy);
        }
        acc = fmaf(wx[i], accy, acc);
    }
#else
#pragma unroll
    for (int i = 0; i < O; ++i) {
        float accy = 0.f;
#pragma unroll
        for (int j = 0; j < O; ++j) {
            const float *row = b + (i * kMBY + j) * kMBZ;
            float accz = 0.f;
#pragma unroll
            for (int k = 0; k < O; ++k) accz = fmaf(wz[k], row[k], accz);
            accy = fmaf(wy[j], accz, accy);
        }
        acc = fmaf(wx[i], accy, acc);
    }
#endif
    double mean = 0.0;
#pragma unroll
    for (int k = 0; k < O; ++k) mean = fma((double)wz[k], __ldg(F.mean + f.k0 + k), mean);
    return (double)acc + mean;
}


__device__ __forceinline__ void block_minmax3_m(int *red, bool act, int a, int b, int c)
{
    const int v[3] = {a, b, c};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int lo = __reduce_min_sync(0xffffffffu, act ? v[q] : INT_MAX);
        const int hi = __reduce_max_sync(0xffffffffu, act ? v[q] : INT_MIN);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&red[2 * q], lo);
            atomicMax(&red[2 * q + 1], hi);
        }
    }
}

template <int O>
__device__ __forceinline__ bool mbox_fits(const int *r, int i0, int j0, const SlcParams &P, int &X0, int &Y0,
                                          int &Z0)
{
    const bool fit = r[0] <= r[1] && r[1] - r[0] + O <= kMBX && r[3] - r[2] + O <= kMBY &&
                     r[5] + O - (r[4] & ~3) <= kMBZ;
    X0 = Y0 = Z0 = 0;
    if (fit) {
        X0 = (i0 + r[0]) % P.nx;
        if (X0 < 0) X0 += P.nx;
        Y0 = (j0 + r[2]) % P.ny;
        if (Y0 < 0) Y0 += P.ny;
        Z0 = r[4] & ~3;
    }
    return fit;
}

template <int C, int O, int TO>
__global__ void __launch_bounds__(kThreads, SLC_SLMT_MIN_BLOCKS)
    k_sl_mixed_tma(const __grid_constant__ SlcParams P, const __grid_constant__ Vel3M M,
                       const __grid_constant__ MixedView FA, const __grid_constant__ MixedView FB,
                       const double *__restrict__ fn, const double *__restrict__ fnm1, double dt,
                       double *__restrict__ out, unsigned long long *nclamp, unsigned long long *stats,
                       const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB)
{
    extern __shared__ unsigned char smraw[];
    __shared__ __align__(8) unsigned long long mbar[2];
    __shared__ int red[12];
    __shared__ int near_lost;
    float *box = (float *)(((uintptr_t)smraw + 127) & ~(uintptr_t)127);
    const int tid = threadIdx.x, lane = tid & 31;
    const int i0 = blockIdx.z * kMTI, j0 = blockIdx.y * kMTJ;
    const int k = blockIdx.x * kMTK + lane;
    const int j = j0 + ((tid >> 5) & (kMTJ - 1));
    const int i = i0 + (tid >> 7);
    const int nzi = (C == 2) ? P.nz - 1 : P.nz;
    const bool act = k < nzi && j < P.ny && i < P.nx;
    const unsigned barA = smem_u32(&mbar[0]), barB = smem_u32(&mbar[1]);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            red[2 * q] = INT_MAX;
            red[2 * q + 1] = INT_MIN;
        }
        near_lost = 0;
        mbar_init(barA, 1);
        mbar_init(barB, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    unsigned ncl = 0;
    Arr32 A{};
    float us0 = 0.f, vs0 = 0.f, ws0 = 0.f, dx = 0.f, dy = 0.f, dz = 0.f;
    FootM32 F{};
    if (act) {
        A = arrival32<C>(P, i, j, k);
        if (TO == 4) {
            sample3_32_o4(P, M, A, 0.f, 0.f, 0.f, us0, vs0, ws0);
        } else {
            double u0, v0, w0;
            arrival_sample<C>(P, M, i, j, k, NodeValMixed32(), u0, v0, w0);
            us0 = (float)u0;
            vs0 = (float)v0;
            ws0 = (float)w0;
        }
        trace_foot32<TO>(P, M, A, (float)(0.5 * dt), us0, vs0, ws0, dx, dy, dz);
        F = locate_foot_m32<C, O>(P, A, dx, dy, dz, i0, j0, ncl);
    }
    block_minmax3_m(red, act, F.rx, F.ry, F.k0);
    __syncthreads();
    int X0, Y0, Z0;
    const bool fitA = mbox_fits<O>(red, i0, j0, P, X0, Y0, Z0);
    if (tid == 0) {
        // stats: [0] time-outs, [1] blocks, [2] near boxes staged, [3] far boxes staged
        atomicAdd(stats + 1, 1ull);
        if (fitA) {
            atomicAdd(stats + 2, 1ull);
            mbar_expect_tx(barA, (unsigned)kMBoxBytes);
            tma_load_3d(smem_u32(box), &tmA, Z0, Y0, X0, barA);
        }
    }
    double ubar = 0.0;
    unsigned none = 0;  // the clamps were counted when the feet were located
    if (act) {
        const bool staged = fitA && mbar_wait(barA);
        if (fitA && !staged) atomicAdd(stats, 1ull);
        if (staged)
            ubar = gather_box_m32<C, O>(P, FA, box, F, F.rx - red[0], F.ry - red[2], F.k0 - Z0);
        else
            ubar = gather_foot32<C, O>(P, FA, A, dx, dy, dz, none);
    }
    __syncthreads();  // every thread is done with the near box
    if (tid == 0 && fitA && !mbar_wait(barA)) {
        atomicAdd(stats, 1ull);
        near_lost = 1;
    }
    if (act) {
        trace_foot32<TO>(P, M, A, (float)dt, us0, vs0, ws0, dx, dy, dz);
        F = locate_foot_m32<C, O>(P, A, dx, dy, dz, i0, j0, ncl);
    }
    block_minmax3_m(red + 6, act, F.rx, F.ry, F.k0);
    __syncthreads();
    const bool fitB = !near_lost && mbox_fits<O>(red + 6, i0, j0, P, X0, Y0, Z0);
    if (tid == 0 && fitB) {
        atomicAdd(stats + 3, 1ull);
        mbar_expect_tx(barB, (unsigned)kMBoxBytes);
        tma_load_3d(smem_u32(box), &tmB, Z0, Y0, X0, barB);
    }
    if (act) {
        double ubb;
        const bool staged = fitB && mbar_wait(barB);
        if (fitB && !staged) atomicAdd(stats, 1ull);
        if (staged)
            ubb = gather_box_m32<C, O>(P, FB, box, F, F.rx - red[6], F.ry - red[8], F.k0 - Z0);
        else
            ubb = gather_foot32<C, O>(P, FB, A, dx, dy, dz, none);
        const double Rn = xy_diffusion64<C>(P, fn, i, j, k);
        const double Rh = P.xy_lagged ? Rn : 2.0 * Rn - xy_diffusion64<C>(P, fnm1, i, j, k);
        double res = ubar * (4.0 / 3.0) + ubb * (-1.0 / 3.0);
        res = res + ((2.0 / 3.0) * dt) * Rh;
        const GhostShape g = ghost_shape(C, P.nx, P.ny, P.nz);
        out[(size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z + (k + 1)] = res;
    }
    add_clamps(nclamp, ncl);
    if (tid == 0 && fitB && !mbar_wait(barB)) atomicAdd(stats, 1ull);
}

// ---- plane means -----------------------------------------------------------
// Field f of `srcs` (component comp[f], ghost-shaped FP64): block (b, f) sums
// the b-th of G contiguous ranges of node columns level by level (threads
// over k, coalesced) into partials[(f * G + b) * ldp + k].  Fixed order:
// bit-reproducible.
struct MeanSrcs {
    const double *p[9];
    int comp[9];
};

__device__ __forceinline__ void plane_partial(const SlcParams &P, const double *src, int C,
                                              double *partials, int ldp, int f, int b, int G)
{
    const int NZ = C == 2 ? P.nz + 1 : P.nz + 2;
    const NodeView<double> V = ghost_view<double>(C, src, P.nx, P.ny, P.nz);
    constexpr int kMaxPer = 5;  // levels per thread: NZ <= 5 blockDim.x
    double acc[kMaxPer];
#pragma unroll
    for (int q = 0; q < kMaxPer; ++q) acc[q] = 0.0;
    // block b sums the contiguous column range [c0, c1), eight adjacent
    // columns' loads in flight, added in column order
    const int ncol = P.nx * P.ny;
    const int c0 = (int)(((long long)ncol * b) / G), c1 = (int)(((long long)ncol * (b + 1)) / G);
    constexpr int kCols = 8;
    for (int col0 = c0; col0 < c1; col0 += kCols) {
        const int i0 = col0 / P.ny, j0 = col0 - i0 * P.ny;
#pragma unroll
        for (int q = 0; q < kMaxPer; ++q) {
            const int k = threadIdx.x + q * blockDim.x;
            if (k < NZ) {
                double val[kCols];
                int i = i0, j = j0;
#pragma unroll
                for (int r = 0; r < kCols; ++r) {
                    val[r] = (col0 + r < c1) ? __ldg(V.p + (size_t)i * V.sx + (size_t)j * V.sy + k) : 0.0;
                    if (++j == P.ny) {
                        j = 0;
                        ++i;
                    }
                }
#pragma unroll
                for (int r = 0; r < kCols; ++r)
                    if (col0 + r < c1) acc[q] += val[r];
            }
        }
    }
    double *out = partials + ((size_t)f * G + b) * ldp;
#pragma unroll
    for (int q = 0; q < kMaxPer; ++q) {
        const int k = threadIdx.x + q * blockDim.x;
        if (k < NZ) out[k] = acc[q];
    }
}

__global__ void __launch_bounds__(1024) k_plane_partials(SlcParams P, const __grid_constant__ MeanSrcs S, double *partials,
                                                        int ldp)
{
    const int f = blockIdx.y;
    plane_partial(P, S.p[f], S.comp[f], partials, ldp, f, blockIdx.x, gridDim.x);
}

// means[f][k] = sum_b partials / (nx ny); with derived_star, fields 6..8 (U*)
// are 2 mean(A) - mean(B) instead of summed.
struct MeanPtrs {
    double *m[9];
    float *m32[9];
};

__device__ __forceinline__ void plane_finish(const SlcParams &P, int nf, const double *partials,
                                             int ldp, int G, double *mean, float *mean32,
                                             int derived_star, int f)
{
    const int NZ = (f % 3) == 2 ? P.nz + 1 : P.nz + 2;
    const double inv = 1.0 / ((double)P.nx * (double)P.ny);
    // sums over the G column groups in group order, eight groups' loads in flight
    auto group_sum = [&](int fs, int k) {
        constexpr int kU = 8;
        const double *p = partials + (size_t)fs * G * ldp + k;
        double s = 0.0;
        for (int b0 = 0; b0 < G; b0 += kU) {
            double v[kU];
#pragma unroll
            for (int r = 0; r < kU; ++r) v[r] = (b0 + r < G) ? p[(size_t)(b0 + r) * ldp] : 0.0;
#pragma unroll
            for (int r = 0; r < kU; ++r)
                if (b0 + r < G) s += v[r];
        }
        return s;
    };
    for (int k = threadIdx.x; k < NZ; k += blockDim.x) {
        double m;
        if (f >= 6 && derived_star) {
            const double sa = group_sum(f - 6, k), sb = group_sum(f - 3, k);
            m = 2.0 * (sa * inv) - sb * inv;
        } else {
            if (f >= nf) return;
            m = group_sum(f, k) * inv;
        }
        mean[k] = m;
        mean32[k] = (float)m;
    }
}

__global__ void k_plane_finish(SlcParams P, int nf, const double *partials, int ldp, int G,
                               const __grid_constant__ MeanPtrs out, int derived_star)
{
    plane_finish(P, nf, partials, ldp, G, out.m[blockIdx.x], out.m32[blockIdx.x], derived_star,
                 blockIdx.x);
}

// FP32 fluctuation node buffers: field slot q = comp (0..2) + 3 * which
// (0 A, 1 B, 2 U*), U* = M or 2A - B.
struct PackArgs {
    const double *A[3], *B[3], *M[3];
    float *f32[9];
    const double *mean[9];
    int nzp[3];
    float *pad[6];  // non-null: V^n, V^{n-1} go to these halo-padded copies instead
    int PX, PY;
};

// One thread per level (blockDim.x >= NZp, or a loop over levels) over kPackJ
// adjacent columns (i, jb kPackJ + q) of component comp; the columns' loads
// are issued before any store.
constexpr int kPackJ = 4;

// One component's sources and destinations, resolved by the caller.
struct PackOne {
    const double *A, *B, *M;           // ghost-shaped; M null: U* = 2A - B
    float *fa, *fb, *fm;               // node buffers, NZp levels per column
    const double *ma, *mb, *mm;        // plane means
    int NZp;
    float *pa = nullptr, *pb = nullptr;  // halo-padded (PX, PY, NZp) copies in place of fa, fb
    int PX = 0, PY = 0;
};

__device__ __forceinline__ void pack_mixed(const SlcParams &P, const PackOne &a, int comp, int i,
                                           int jb)
{
    const int NZ = comp == 2 ? P.nz + 1 : P.nz + 2;
    const int NZp = a.NZp;
    const NodeView<double> VA = ghost_view<double>(comp, a.A, P.nx, P.ny, P.nz);
    const NodeView<double> VB = ghost_view<double>(comp, a.B, P.nx, P.ny, P.nz);
    const double *pm = a.M ? ghost_view<double>(comp, a.M, P.nx, P.ny, P.nz).p : nullptr;
    for (int k = threadIdx.x; k < NZp; k += blockDim.x) {
        const bool in = k < NZ;
        const double ma = in ? a.ma[k] : 0.0, mb = in ? a.mb[k] : 0.0, mm = in ? a.mm[k] : 0.0;
        double va[kPackJ], vb[kPackJ], vm[kPackJ];
#pragma unroll
        for (int q = 0; q < kPackJ; ++q) {
            const int j = jb * kPackJ + q;
            const bool ok = in && j < P.ny;
            const size_t n = (size_t)i * VA.sx + (size_t)j * VA.sy + k;
            va[q] = ok ? VA.p[n] : 0.0;
            vb[q] = ok ? VB.p[n] : 0.0;
            vm[q] = (ok && pm) ? pm[n] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < kPackJ; ++q) {
            const int j = jb * kPackJ + q;
            if (j >= P.ny) continue;
            const size_t o = ((size_t)i * P.ny + j) * NZp + k;
            float fa = 0.f, fb = 0.f, fm = 0.f;  // padding levels stay zero
            if (in) {
                const double m = pm ? vm[q] : 2.0 * va[q] - vb[q];
                fa = (float)(va[q] - ma);
                fb = (float)(vb[q] - mb);
                fm = (float)(m - mm);
            }
            a.fm[o] = fm;
            if (a.pa) {  // node (i, j) and its periodic images inside the halo
                for (int x = i; x < a.PX; x += P.nx)
                    for (int y = j; y < a.PY; y += P.ny) {
                        const size_t po = ((size_t)x * a.PY + y) * NZp + k;
                        a.pa[po] = fa;
                        a.pb[po] = fb;
                    }
            } else {
                a.fa[o] = fa;
                a.fb[o] = fb;
            }
        }
    }
}

__global__ void __launch_bounds__(1024) k_pack_mixed(SlcParams P, const __grid_constant__ PackArgs a)
{
    const int comp = blockIdx.y / P.nx, i = blockIdx.y - comp * P.nx;
    PackOne o;
    o.A = a.A[comp];
    o.B = a.B[comp];
    o.M = a.M[comp];
    o.fa = a.f32[comp];
    o.fb = a.f32[comp + 3];
    o.fm = a.f32[comp + 6];
    o.ma = a.mean[comp];
    o.mb = a.mean[comp + 3];
    o.mm = a.mean[comp + 6];
    o.NZp = a.nzp[comp];
    if (a.pad[comp]) {
        o.pa = a.pad[comp];
        o.pb = a.pad[comp + 3];
        o.PX = a.PX;
        o.PY = a.PY;
    }
    pack_mixed(P, o, comp, i, blockIdx.x);
}

// ---- ensemble forms (one launch per substep over all instances) ----
__device__ __forceinline__ MixedView mview_dev(const MixedWS &ws, int slot, const SlcParams &P)
{
    MixedView v;
    const int comp = slot % 3;
    v.f = node_view<float>(ws.f32[slot], P.ny, ws.nzp[comp]);
    v.mean = ws.mean[slot];
    v.mean32 = ws.mean32[slot];
    return v;
}

// items (inst, column group b, field f): f < 3 the near field V^n, else V^{n-1}
__global__ void __launch_bounds__(256) k_plane_partials_ens(const EnsInst *__restrict__ ins,
                                                            const EnsItem *__restrict__ items, int ph)
{
    const EnsItem it = items[blockIdx.x];
    const EnsInst &I = ins[it.inst];
    const int f = it.b;
    const double *src = f < 3 ? I.lev[ens_cur(ph)][f] : I.lev[ens_prev(ph)][f - 3];
    plane_partial(I.P, src, f % 3, I.mws.partials, I.P.nz + 2, f, it.a, kMeanBlocks);
}

// block (inst * 9 + f)
__global__ void k_plane_finish_ens(const EnsInst *__restrict__ ins)
{
    const EnsInst &I = ins[blockIdx.x / 9];
    const int f = blockIdx.x % 9;
    plane_finish(I.P, 6, I.mws.partials, I.P.nz + 2, kMeanBlocks, I.mws.mean[f], I.mws.mean32[f], 1,
                 f);
}

// items (inst, bx, by, bz) as k_pack_mixed's grid
__global__ void __launch_bounds__(1024) k_pack_mixed_ens(const EnsInst *__restrict__ ins,
                                                        const EnsItem *__restrict__ items, int ph)
{
    const EnsItem it = items[blockIdx.x];
    const EnsInst &I = ins[it.inst];
    const int comp = it.b / I.P.nx, i = it.b - comp * I.P.nx;
    PackOne o;
    o.A = I.lev[ens_cur(ph)][comp];
    o.B = I.lev[ens_prev(ph)][comp];
    o.M = nullptr;
    o.fa = I.mws.f32[comp];
    o.fb = I.mws.f32[comp + 3];
    o.fm = I.mws.f32[comp + 6];
    o.ma = I.mws.mean[comp];
    o.mb = I.mws.mean[comp + 3];
    o.mm = I.mws.mean[comp + 6];
    o.NZp = I.mws.nzp[comp];
    pack_mixed(I.P, o, comp, i, it.a);
}

// Persistent mixed-form BDF2 trace+gather over the (instance, component, x
// index, tile) queue; the structure of the FP64 ensemble kernel.
// TO: the instances' common trajectory order (2 or 4), or 0 for a mixture
// (read per instance).
template <int O, int TO>
__global__ void __launch_bounds__(kThreads, SLC_SLM_ENS_MIN_BLOCKS) k_sl_mixed_ens(const EnsInst *__restrict__ ins,
                                                              const EnsItem *__restrict__ items,
                                                              int nitems, int ph, unsigned *queue)
{
    __shared__ SlcParams sP;
    __shared__ int s_item;
    if (threadIdx.x == 0) s_item = (int)atomicAdd(queue, 1u);
    int have = -1;
    for (;;) {
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const EnsItem w = items[it];
        if (w.inst != have) {
            const unsigned long long *src = (const unsigned long long *)&ins[w.inst].P;
            unsigned long long *dst = (unsigned long long *)&sP;
            for (int q = threadIdx.x; q < (int)(sizeof(SlcParams) / 8); q += kThreads) dst[q] = src[q];
            have = w.inst;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_item = (int)atomicAdd(queue, 1u);
        const EnsInst &I = ins[w.inst];
        const int tkl = I.tkl;
        const int k = ((w.c & 0xffff) << tkl) + (threadIdx.x & ((1 << tkl) - 1));
        const int j = ((w.c >> 16) << (8 - tkl)) + (threadIdx.x >> tkl);
        const int i = w.b;
        const Vel3M M{mview_dev(I.mws, 6, sP), mview_dev(I.mws, 7, sP), mview_dev(I.mws, 8, sP)};
        const MixedView FA = mview_dev(I.mws, w.a, sP), FB = mview_dev(I.mws, w.a + 3, sP);
        const double *fn = I.lev[ens_cur(ph)][w.a];
        const double *fnm1 = I.lev[ens_prev(ph)][w.a];
        double *out = I.lev[ens_next(ph)][w.a];
        unsigned ncl = 0;
        const OutMap ghost{0, 0, 0};
        if (w.a == 0) sl_point_mixed<0, O, 2, TO, true>(sP, M, FA, FB, fn, fnm1, I.dt, out, i, j, k, ncl, ghost);
        else if (w.a == 1) sl_point_mixed<1, O, 2, TO, true>(sP, M, FA, FB, fn, fnm1, I.dt, out, i, j, k, ncl, ghost);
        else sl_point_mixed<2, O, 2, TO, true>(sP, M, FA, FB, fn, fnm1, I.dt, out, i, j, k, ncl, ghost);
        add_clamps(I.ncl, ncl);
    }
}

MixedView mview(const MixedWS &ws, int slot, const SlcParams &P)
{
    MixedView v;
    const int comp = slot % 3;
    v.f = node_view<float>(ws.f32[slot], P.ny, ws.nzp[comp]);
    v.mean = ws.mean[slot];
    v.mean32 = ws.mean32[slot];
    return v;
}

template <int O, int MODE, int TO>
void launch_tt(const SlcParams &P, Tri fn, Tri fnm1, const MixedWS &ws, double dt, TriMut out,
               unsigned long long *ncl, const OutMap *om, cudaStream_t s)
{
    Vel3M M{mview(ws, 6, P), mview(ws, 7, P), mview(ws, 8, P)};
    const dim3 gc((P.nz + kTileK - 1) / kTileK, (P.ny + kTileJ - 1) / kTileJ, P.nx);
    const dim3 gw((P.nz - 1 + kTileK - 1) / kTileK, (P.ny + kTileJ - 1) / kTileJ, P.nx);
    const OutMap ghost{0, 0, 0};
    k_sl_mixed<0, O, MODE, TO><<<gc, kThreads, 0, s>>>(P, M, mview(ws, 0, P), mview(ws, 3, P), fn.u,
                                                    fnm1.u, dt, out.u, ncl, om ? om[0] : ghost);
    k_sl_mixed<1, O, MODE, TO><<<gc, kThreads, 0, s>>>(P, M, mview(ws, 1, P), mview(ws, 4, P), fn.v,
                                                    fnm1.v, dt, out.v, ncl, om ? om[1] : ghost);
    if (P.nz > 1)
        k_sl_mixed<2, O, MODE, TO><<<gw, kThreads, 0, s>>>(P, M, mview(ws, 2, P), mview(ws, 5, P),
                                                        fn.w, fnm1.w, dt, out.w, ncl,
                                                        om ? om[2] : ghost);
    count_launches(P.nz > 1 ? 3 : 2);
}

template <int O, int MODE>
void launch_t(const SlcParams &P, Tri fn, Tri fnm1, const MixedWS &ws, double dt, TriMut out,
              unsigned long long *ncl, const OutMap *om, cudaStream_t s)
{
    if (P.traj_order == 4) launch_tt<O, MODE, 4>(P, fn, fnm1, ws, dt, out, ncl, om, s);
    else launch_tt<O, MODE, 2>(P, fn, fnm1, ws, dt, out, ncl, om, s);
}

}  // namespace

int mixed_nzp(int NZ) { return (NZ + 3) & ~3; }
size_t mixed_partials_doubles(const SlcParams &P) { return (size_t)9 * kMeanBlocks * (P.nz + 2); }

cudaError_t launch_mixed_prepare(const SlcParams &P, Tri A, Tri B, Tri M, const MixedWS &ws,
                                 cudaStream_t s, const TmaMixed *pad)
{
    MeanSrcs S{};
    const bool explicit_m = M.u != nullptr;
    const int nf = explicit_m ? 9 : 6;
    const double *src[9] = {A.u, A.v, A.w, B.u, B.v, B.w, M.u, M.v, M.w};
    for (int f = 0; f < 9; ++f) {
        S.p[f] = src[f];
        S.comp[f] = f % 3;
    }
    const int ldp = P.nz + 2;
    // one thread per level (a warp covering the last few levels alone would
    // make a second dependent round of loads the block's critical path)
    const int pt = std::min(1024, (P.nz + 2 + 31) / 32 * 32);
    k_plane_partials<<<dim3(kMeanBlocks, nf), pt, 0, s>>>(P, S, ws.partials, ldp);
    MeanPtrs mp;
    for (int f = 0; f < 9; ++f) {
        mp.m[f] = ws.mean[f];
        mp.m32[f] = ws.mean32[f];
    }
    k_plane_finish<<<9, 256, 0, s>>>(P, nf, ws.partials, ldp, kMeanBlocks, mp, explicit_m ? 0 : 1);
    PackArgs a{};
    for (int c = 0; c < 3; ++c) {
        a.A[c] = src[c];
        a.B[c] = src[3 + c];
        a.M[c] = explicit_m ? src[6 + c] : nullptr;
        a.nzp[c] = ws.nzp[c];
    }
    for (int q = 0; q < 9; ++q) {
        a.f32[q] = ws.f32[q];
        a.mean[q] = ws.mean[q];
    }
    if (pad) {
        for (int q = 0; q < 6; ++q) a.pad[q] = pad->pad[q];
        a.PX = pad->PX;
        a.PY = pad->PY;
    }
    const int nzp_max = ws.nzp[0] > ws.nzp[2] ? ws.nzp[0] : ws.nzp[2];
    k_pack_mixed<<<dim3((P.ny + kPackJ - 1) / kPackJ, 3 * P.nx), mixed_pack_threads(nzp_max), 0, s>>>(P, a);
    count_launches(3);
    return cudaGetLastError();
}

cudaError_t launch_sl_mixed(const SlcParams &P, int mode, Tri fn, Tri fnm1, const MixedWS &ws,
                            double dt, TriMut out, unsigned long long *nclamp, cudaStream_t s,
                            const OutMap *om)
{
    if (mode != 0) om = nullptr;  // the predictors always write ghost-shaped interiors
    if (P.order == 4) {
        if (mode == 0) launch_t<4, 0>(P, fn, fnm1, ws, dt, out, nclamp, om, s);
        else if (mode == 1) launch_t<4, 1>(P, fn, fnm1, ws, dt, out, nclamp, om, s);
        else launch_t<4, 2>(P, fn, fnm1, ws, dt, out, nclamp, om, s);
    } else {
        if (mode == 0) launch_t<6, 0>(P, fn, fnm1, ws, dt, out, nclamp, om, s);
        else if (mode == 1) launch_t<6, 1>(P, fn, fnm1, ws, dt, out, nclamp, om, s);
        else launch_t<6, 2>(P, fn, fnm1, ws, dt, out, nclamp, om, s);
    }
    return cudaGetLastError();
}

namespace {
template <int O, int TO>
cudaError_t launch_mtma_t(const SlcParams &P, const Vel3M &M, const MixedView *FA, const MixedView *FB, Tri fn,
                          Tri fnm1, double dt, TriMut out, unsigned long long *ncl, unsigned long long *stats,
                          const CUtensorMap *tm, cudaStream_t s)
{
    const dim3 gc((P.nz + kMTK - 1) / kMTK, (P.ny + kMTJ - 1) / kMTJ, (P.nx + kMTI - 1) / kMTI);
    const dim3 gw((P.nz - 1 + kMTK - 1) / kMTK, (P.ny + kMTJ - 1) / kMTJ, (P.nx + kMTI - 1) / kMTI);

    // the attributes are per device context, so set on every launch (a
    // host-side attribute write)
    const size_t sm = kMBoxBytes + 128;
    cudaError_t e = cudaFuncSetAttribute(k_sl_mixed_tma<0, O, TO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sm);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sl_mixed_tma<1, O, TO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sl_mixed_tma<2, O, TO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_sl_mixed_tma<0, O, TO><<<gc, kThreads, sm, s>>>(P, M, FA[0], FB[0], fn.u, fnm1.u, dt, out.u, ncl, stats,
                                                      tm[0], tm[3]);
    k_sl_mixed_tma<1, O, TO><<<gc, kThreads, sm, s>>>(P, M, FA[1], FB[1], fn.v, fnm1.v, dt, out.v, ncl, stats,
                                                      tm[1], tm[4]);
    if (P.nz > 1)
        k_sl_mixed_tma<2, O, TO><<<gw, kThreads, sm, s>>>(P, M, FA[2], FB[2], fn.w, fnm1.w, dt, out.w, ncl,
                                                          stats, tm[2], tm[5]);
    count_launches(P.nz > 1 ? 3 : 2);
    return cudaGetLastError();
}
}  // namespace

bool mixed_tma_supported(const SlcParams &P)
{
    // every padded row holds a whole box depth (the shallower w rows too)
    return mixed_nzp(P.nz + 1) >= kMBZ;
}

size_t mixed_tma_elems(const SlcParams &P, const MixedWS &ws, int comp)
{
    return (size_t)(P.nx + kMBX) * (P.ny + kMBY) * ws.nzp[comp];
}

cudaError_t mixed_tma_encode(const SlcParams &P, const MixedWS &ws, TmaMixed &T)
{
    static_assert(sizeof(CUtensorMap) == 128, "tensor-map storage");
    T.PX = P.nx + kMBX;
    T.PY = P.ny + kMBY;
    for (int q = 0; q < 6; ++q) {
        const unsigned long long nzp = (unsigned long long)ws.nzp[q % 3];
        const unsigned long long dims[3] = {nzp, (unsigned long long)T.PY, (unsigned long long)T.PX};
        const unsigned long long strides[2] = {nzp * 4, nzp * 4 * (unsigned long long)T.PY};
        const unsigned box[3] = {(unsigned)kMBZ, (unsigned)kMBY, (unsigned)kMBX};
        cudaError_t e = tma_encode_3d(T.maps + 128 * q, true, T.pad[q], dims, strides, box);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_sl_mixed_tma(const SlcParams &P, Tri fn, Tri fnm1, const MixedWS &ws, const TmaMixed &T,
                                double dt, TriMut out, unsigned long long *nclamp,
                                unsigned long long *stats, cudaStream_t s)
{
    const Vel3M M{mview(ws, 6, P), mview(ws, 7, P), mview(ws, 8, P)};
    MixedView FA[3], FB[3];
    for (int c = 0; c < 3; ++c) {
        for (int w = 0; w < 2; ++w) {
            MixedView &v = w == 0 ? FA[c] : FB[c];
            v.f.p = T.pad[c + 3 * w];
            v.f.sy = ws.nzp[c];
            v.f.sx = T.PY * ws.nzp[c];
            v.mean = ws.mean[c + 3 * w];
            v.mean32 = ws.mean32[c + 3 * w];
        }
    }
    const CUtensorMap *tm = (const CUtensorMap *)T.maps;
    const bool t4 = P.traj_order == 4;
    if (P.order == 4)
        return t4 ? launch_mtma_t<4, 4>(P, M, FA, FB, fn, fnm1, dt, out, nclamp, stats, tm, s)
                  : launch_mtma_t<4, 2>(P, M, FA, FB, fn, fnm1, dt, out, nclamp, stats, tm, s);
    return t4 ? launch_mtma_t<6, 4>(P, M, FA, FB, fn, fnm1, dt, out, nclamp, stats, tm, s)
              : launch_mtma_t<6, 2>(P, M, FA, FB, fn, fnm1, dt, out, nclamp, stats, tm, s);
}

int mixed_mean_blocks() { return kMeanBlocks; }

int sl_mixed_ens_blocks_per_sm()
{
    // the smallest residency over the instantiations the ensemble may launch
    const void *k[6] = {(const void *)k_sl_mixed_ens<6, 2>, (const void *)k_sl_mixed_ens<4, 2>,
                        (const void *)k_sl_mixed_ens<6, 4>, (const void *)k_sl_mixed_ens<4, 4>,
                        (const void *)k_sl_mixed_ens<6, 0>, (const void *)k_sl_mixed_ens<4, 0>};
    int m = 1 << 30;
    for (int q = 0; q < 6; ++q) {
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k[q], kThreads, 0) != cudaSuccess) return 1;
        m = nb < m ? nb : m;
    }
    return m > 0 ? m : 1;
}
int mixed_pack_cols() { return kPackJ; }
int mixed_pack_threads(int nzp) { return std::min(1024, (nzp + 31) / 32 * 32); }

cudaError_t launch_mixed_prepare_ens(const EnsInst *ins, int ninst, const EnsItem *pp_items, int n_pp,
                                     const EnsItem *pack_items, int n_pack, int pack_threads, int ph,
                                     cudaStream_t s)
{
    // no items: every instance packs its own buffers (the staged gather)
    if (ninst <= 0 || n_pp <= 0 || n_pack <= 0) return cudaSuccess;
    k_plane_partials_ens<<<n_pp, 256, 0, s>>>(ins, pp_items, ph);
    k_plane_finish_ens<<<9 * ninst, 256, 0, s>>>(ins);
    k_pack_mixed_ens<<<n_pack, pack_threads, 0, s>>>(ins, pack_items, ph);
    count_launches(3);
    return cudaGetLastError();
}

cudaError_t launch_sl_mixed_ens(const EnsInst *ins, const EnsItem *items, int nitems, int ph, int order,
                                int traj,
                                unsigned *queue, int grid, cudaStream_t s)
{
    if (nitems <= 0) return cudaSuccess;
#define SLM_ENS(OV, TV) k_sl_mixed_ens<OV, TV><<<grid, kThreads, 0, s>>>(ins, items, nitems, ph, queue)
    if (order == 4) {
        if (traj == 2) SLM_ENS(4, 2);
        else if (traj == 4) SLM_ENS(4, 4);
        else SLM_ENS(4, 0);
    } else {
        if (traj == 2) SLM_ENS(6, 2);
        else if (traj == 4) SLM_ENS(6, 4);
        else SLM_ENS(6, 0);
    }
#undef SLM_ENS
    count_launches(1);
    return cudaGetLastError();
}
