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
#include "slc_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr int kTileK = 64, kTileJ = kThreads / kTileK;
constexpr int kMeanBlocks = 148;  // column groups of the plane-mean partial sums

struct Vel3M {
    MixedView u, v, w;
};

__device__ __forceinline__ void add_clamps(unsigned long long *counter, unsigned cnt)
{
    unsigned tot = __reduce_add_sync(0xffffffffu, cnt);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(counter, (unsigned long long)tot);
}

__device__ __forceinline__ void sample3_m(const SlcParams &P, const Vel3M &M, double x, double y,
                                          double z, double &us, double &vs, double &ws)
{
    const double zc = clampz(P, z);
    TriShared t;
    tri_shared(P, x, y, zc, face_cell(P, zc), t);
    us = tri_sample_mixed(M.u, t.ia0, t.ia1, t.txa, t.jb0, t.jb1, t.tyb, t.kc, t.wc0, t.wc1);
    vs = tri_sample_mixed(M.v, t.ib0, t.ib1, t.txb, t.ja0, t.ja1, t.tya, t.kc, t.wc0, t.wc1);
    ws = tri_sample_mixed(M.w, t.ib0, t.ib1, t.txb, t.jb0, t.jb1, t.tyb, t.kf, t.wf0, t.wf1);
}

__device__ __forceinline__ void trace_foot_m(const SlcParams &P, const Vel3M &M, double xa,
                                             double ya, double za, double half_dt, double us0,
                                             double vs0, double ws0, double &xd, double &yd,
                                             double &zd)
{
    double xm = xa - half_dt * us0;
    double ym = ya - half_dt * vs0;
    double zm = clampz(P, za - half_dt * ws0);
    for (int it = 1; it < P.n_iters; ++it) {
        double us, vs, ws;
        sample3_m(P, M, xm, ym, zm, us, vs, ws);
        xm = xa - half_dt * us;
        ym = ya - half_dt * vs;
        zm = clampz(P, za - half_dt * ws);
    }
    xd = 2.0 * xm - xa;
    yd = 2.0 * ym - ya;
    zd = 2.0 * zm - za;
}

template <int C, int O>
__device__ __forceinline__ double gather_foot_m(const SlcParams &P, MixedView F, double xd,
                                                double yd, double zd, unsigned &ncl)
{
    if (zd < P.z_lo || zd > P.z_hi) ncl += 1;
    const double z = clampz(P, zd);
    const int c = face_cell(P, z);
    StencilM<O> st;
    build_stencil_mixed<C, O>(P, F.f.sx, F.f.sy, xd, yd, z, c, st);
    return gather_mixed<O>(F, st);
}

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
template <int C, int O, int MODE>
__global__ void __launch_bounds__(kThreads, 2)
    k_sl_mixed(SlcParams P, Vel3M M, MixedView FA, MixedView FB, const double *__restrict__ fn,
               const double *__restrict__ fnm1, double dt, double *__restrict__ out,
               unsigned long long *nclamp)
{
    const int nzi = (C == 2) ? P.nz - 1 : P.nz;
    const int k = blockIdx.x * kTileK + (threadIdx.x % kTileK);
    const int j = blockIdx.y * kTileJ + (threadIdx.x / kTileK);
    const int i = blockIdx.z;
    unsigned ncl = 0;
    if (k < nzi && j < P.ny) {
        double xa, ya, za;
        arrival_point<C>(P, i, j, k, xa, ya, za);
        double us0, vs0, ws0;
        arrival_sample<C>(P, M, i, j, k, NodeValMixed(), us0, vs0, ws0);
        double xd, yd, zd;
        trace_foot_m(P, M, xa, ya, za, 0.5 * dt, us0, vs0, ws0, xd, yd, zd);
        const double ubar = gather_foot_m<C, O>(P, FA, xd, yd, zd, ncl);
        double res;
        if (MODE == 0) {
            res = ubar;
        } else if (MODE == 1) {
            res = ubar + dt * xy_diffusion64<C>(P, fn, i, j, k);
        } else {
            trace_foot_m(P, M, xa, ya, za, dt, us0, vs0, ws0, xd, yd, zd);
            const double ubb = gather_foot_m<C, O>(P, FB, xd, yd, zd, ncl);
            const double Rn = xy_diffusion64<C>(P, fn, i, j, k);
            const double Rh = P.xy_lagged ? Rn : 2.0 * Rn - xy_diffusion64<C>(P, fnm1, i, j, k);
            res = ubar * (4.0 / 3.0) + ubb * (-1.0 / 3.0);
            res = res + ((2.0 / 3.0) * dt) * Rh;
        }
        const GhostShape g = ghost_shape(C, P.nx, P.ny, P.nz);
        out[(size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z + (k + 1)] = res;
    }
    add_clamps(nclamp, ncl);
}

// ---- plane means -----------------------------------------------------------
// Field f of `srcs` (component comp[f], ghost-shaped FP64): block (b, f) sums
// the node columns b, b + G, ... level by level (threads over k, coalesced)
// into partials[(f * G + b) * ldp + k].  Fixed order: bit-reproducible.
struct MeanSrcs {
    const double *p[9];
    int comp[9];
};

__global__ void __launch_bounds__(256) k_plane_partials(SlcParams P, MeanSrcs S, double *partials,
                                                        int ldp)
{
    const int f = blockIdx.y, b = blockIdx.x, G = gridDim.x;
    const int C = S.comp[f];
    const int NZ = C == 2 ? P.nz + 1 : P.nz + 2;
    const NodeView<double> V = ghost_view<double>(C, S.p[f], P.nx, P.ny, P.nz);
    constexpr int kMaxPer = 5;  // NZ <= 1026 levels over 256 threads
    double acc[kMaxPer];
#pragma unroll
    for (int q = 0; q < kMaxPer; ++q) acc[q] = 0.0;
    const int ncol = P.nx * P.ny;
    for (int col = b; col < ncol; col += G) {
        const int i = col / P.ny, j = col - (col / P.ny) * P.ny;
        const double *c = V.p + (size_t)i * V.sx + (size_t)j * V.sy;
#pragma unroll
        for (int q = 0; q < kMaxPer; ++q) {
            const int k = threadIdx.x + q * 256;
            if (k < NZ) acc[q] += __ldg(c + k);
        }
    }
    double *out = partials + ((size_t)f * G + b) * ldp;
#pragma unroll
    for (int q = 0; q < kMaxPer; ++q) {
        const int k = threadIdx.x + q * 256;
        if (k < NZ) out[k] = acc[q];
    }
}

// means[f][k] = sum_b partials / (nx ny); with derived_star, fields 6..8 (U*)
// are 2 mean(A) - mean(B) instead of summed.
struct MeanPtrs {
    double *m[9];
};

__global__ void k_plane_finish(SlcParams P, int nf, const double *partials, int ldp, int G,
                               MeanPtrs out, int derived_star)
{
    const int f = blockIdx.x;
    const int NZ = (f % 3) == 2 ? P.nz + 1 : P.nz + 2;
    const double inv = 1.0 / ((double)P.nx * (double)P.ny);
    for (int k = threadIdx.x; k < NZ; k += blockDim.x) {
        double m;
        if (f >= 6 && derived_star) {
            double sa = 0.0, sb = 0.0;
            for (int b = 0; b < G; ++b) {
                sa += partials[((size_t)(f - 6) * G + b) * ldp + k];
                sb += partials[((size_t)(f - 3) * G + b) * ldp + k];
            }
            m = 2.0 * (sa * inv) - sb * inv;
        } else {
            if (f >= nf) return;
            double s = 0.0;
            for (int b = 0; b < G; ++b) s += partials[((size_t)f * G + b) * ldp + k];
            m = s * inv;
        }
        out.m[f][k] = m;
    }
}

// FP32 fluctuation node buffers: field slot q = comp (0..2) + 3 * which
// (0 A, 1 B, 2 U*), U* = M or 2A - B.
struct PackArgs {
    const double *A[3], *B[3], *M[3];
    float *f32[9];
    const double *mean[9];
    int nzp[3];
};

__global__ void __launch_bounds__(128) k_pack_mixed(SlcParams P, PackArgs a)
{
    const int comp = blockIdx.z / P.nx, i = blockIdx.z - comp * P.nx;
    const int j = blockIdx.y;
    const int k = blockIdx.x * 128 + threadIdx.x;
    const int NZ = comp == 2 ? P.nz + 1 : P.nz + 2;
    const int NZp = a.nzp[comp];
    if (k >= NZp) return;
    const size_t o = ((size_t)i * P.ny + j) * NZp + k;
    if (k >= NZ) {
        a.f32[comp][o] = 0.f;
        a.f32[comp + 3][o] = 0.f;
        a.f32[comp + 6][o] = 0.f;
        return;
    }
    const NodeView<double> VA = ghost_view<double>(comp, a.A[comp], P.nx, P.ny, P.nz);
    const NodeView<double> VB = ghost_view<double>(comp, a.B[comp], P.nx, P.ny, P.nz);
    const size_t n = (size_t)i * VA.sx + (size_t)j * VA.sy + k;
    const double va = VA.p[n], vb = VB.p[n];
    double vm;
    if (a.M[comp]) {
        const NodeView<double> VM = ghost_view<double>(comp, a.M[comp], P.nx, P.ny, P.nz);
        vm = VM.p[n];
    } else {
        vm = 2.0 * va - vb;
    }
    a.f32[comp][o] = (float)(va - a.mean[comp][k]);
    a.f32[comp + 3][o] = (float)(vb - a.mean[comp + 3][k]);
    a.f32[comp + 6][o] = (float)(vm - a.mean[comp + 6][k]);
}

MixedView mview(const MixedWS &ws, int slot, const SlcParams &P)
{
    MixedView v;
    const int comp = slot % 3;
    v.f = node_view<float>(ws.f32[slot], P.ny, ws.nzp[comp]);
    v.mean = ws.mean[slot];
    return v;
}

template <int O, int MODE>
void launch_t(const SlcParams &P, Tri fn, Tri fnm1, const MixedWS &ws, double dt, TriMut out,
              unsigned long long *ncl, cudaStream_t s)
{
    Vel3M M{mview(ws, 6, P), mview(ws, 7, P), mview(ws, 8, P)};
    const dim3 gc((P.nz + kTileK - 1) / kTileK, (P.ny + kTileJ - 1) / kTileJ, P.nx);
    const dim3 gw((P.nz - 1 + kTileK - 1) / kTileK, (P.ny + kTileJ - 1) / kTileJ, P.nx);
    k_sl_mixed<0, O, MODE><<<gc, kThreads, 0, s>>>(P, M, mview(ws, 0, P), mview(ws, 3, P), fn.u,
                                                    fnm1.u, dt, out.u, ncl);
    k_sl_mixed<1, O, MODE><<<gc, kThreads, 0, s>>>(P, M, mview(ws, 1, P), mview(ws, 4, P), fn.v,
                                                    fnm1.v, dt, out.v, ncl);
    if (P.nz > 1)
        k_sl_mixed<2, O, MODE><<<gw, kThreads, 0, s>>>(P, M, mview(ws, 2, P), mview(ws, 5, P),
                                                        fn.w, fnm1.w, dt, out.w, ncl);
    count_launches(P.nz > 1 ? 3 : 2);
}

}  // namespace

int mixed_nzp(int NZ) { return (NZ + 3) & ~3; }
size_t mixed_partials_doubles(const SlcParams &P) { return (size_t)9 * kMeanBlocks * (P.nz + 2); }

cudaError_t launch_mixed_prepare(const SlcParams &P, Tri A, Tri B, Tri M, const MixedWS &ws,
                                 cudaStream_t s)
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
    k_plane_partials<<<dim3(kMeanBlocks, nf), 256, 0, s>>>(P, S, ws.partials, ldp);
    MeanPtrs mp;
    for (int f = 0; f < 9; ++f) mp.m[f] = ws.mean[f];
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
    const int nzp_max = ws.nzp[0] > ws.nzp[2] ? ws.nzp[0] : ws.nzp[2];
    k_pack_mixed<<<dim3((nzp_max + 127) / 128, P.ny, 3 * P.nx), 128, 0, s>>>(P, a);
    count_launches(3);
    return cudaGetLastError();
}

cudaError_t launch_sl_mixed(const SlcParams &P, int mode, Tri fn, Tri fnm1, const MixedWS &ws,
                            double dt, TriMut out, unsigned long long *nclamp, cudaStream_t s)
{
    if (P.order == 4) {
        if (mode == 0) launch_t<4, 0>(P, fn, fnm1, ws, dt, out, nclamp, s);
        else if (mode == 1) launch_t<4, 1>(P, fn, fnm1, ws, dt, out, nclamp, s);
        else launch_t<4, 2>(P, fn, fnm1, ws, dt, out, nclamp, s);
    } else {
        if (mode == 0) launch_t<6, 0>(P, fn, fnm1, ws, dt, out, nclamp, s);
        else if (mode == 1) launch_t<6, 1>(P, fn, fnm1, ws, dt, out, nclamp, s);
        else launch_t<6, 2>(P, fn, fnm1, ws, dt, out, nclamp, s);
    }
    return cudaGetLastError();
}
