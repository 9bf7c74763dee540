// slc_common.cuh -- grid parameters and device helpers shared by the SL-BDF2
// kernels (sm_100a).  Reference paths are relative to gmcavallazzi/SLchannel
// v1.0.1.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define SLC_MAX_ORDER 6

// Everything a kernel needs to know about the grid, passed by value.
struct SlcParams {
    int nx, ny, nz;
    int symmetric;     // tanh map: 1 symmetric, 0 bottom
    int order;         // field interpolation order (4 or 6)
    int n_iters;       // midpoint fixed-point iterations
    int traj_order;    // trajectory sampling: 2 trilinear, 4 tricubic Lagrange
    int top_neumann;   // free-slip top wall for u, v
    int xy_lagged;     // BDF2 explicit xy-rhs: 0 extrap (2R^n - R^{n-1}), 1 lagged (R^n)
    double dx, dy, inv_dx, inv_dy, inv_dx2, inv_dy2;
    double Lz, two_over_Lz, inv_Lz;
    double gamma, inv_gamma, tanh_g, half_nz, nzd;
    double z_lo, z_hi;  // departure z kept in [z_lo, z_hi] (semilag.py:244-247)
    double nu;
    const double *zc;   // nz+2 centres incl. ghosts (u, v node z)
    const double *zf;   // nz+1 faces (w node z)
    // inverse Lagrange denominators per order, (NZ - o + 1, o) row-major,
    // for centre nodes (NZ = nz+2) and face nodes (NZ = nz+1); semilag.py:102-114
    const double *dinv_c[SLC_MAX_ORDER + 1];
    const double *dinv_f[SLC_MAX_ORDER + 1];
    const float *dinv_c32[SLC_MAX_ORDER + 1];  // FP32 copies for the mixed form
    const float *dinv_f32[SLC_MAX_ORDER + 1];
    const float *zc32, *zf32;
    double udenom[SLC_MAX_ORDER + 1][SLC_MAX_ORDER];  // semilag.py:117-127
};

// Read-only view of one component's node grid (i in [0,NX), j in [0,NY),
// k in [0,NZ)), stored in some 3-D array: element = p[i*sx + j*sy + k].
// The offset of node (0,0,0) inside a ghost-shaped array is folded into p.
template <typename T>
struct NodeView {
    const T *p;
    int sx, sy;
};

// Component node grids (semilag.py:258-286): u and v on cell centres incl.
// the two ghost centres (NZ = nz+2), w on faces incl. walls (NZ = nz+1).
// Node coordinate s_x = x/dx + shift_x.
template <int C>
struct Comp {
    static constexpr double shift_x = (C == 0) ? 0.0 : -0.5;
    static constexpr double shift_y = (C == 1) ? 0.0 : -0.5;
    static constexpr bool centers = (C != 2);
};

// Ghost-shaped array geometry of component C (0 u, 1 v, 2 w, 3 p).
struct GhostShape {
    int X, Y, Z;   // array extents
    int ox, oy;    // index of node (0,0) inside the array
};

__host__ __device__ inline GhostShape ghost_shape(int C, int nx, int ny, int nz)
{
    switch (C) {
    case 0: return {nx + 1, ny + 2, nz + 2, 0, 1};
    case 1: return {nx + 2, ny + 1, nz + 2, 1, 0};
    case 2: return {nx + 2, ny + 2, nz + 1, 1, 1};
    default: return {nx + 2, ny + 2, nz + 2, 1, 1};
    }
}

template <typename T>
__host__ __device__ inline NodeView<T> ghost_view(int C, const T *base, int nx, int ny, int nz)
{
    GhostShape s = ghost_shape(C, nx, ny, nz);
    NodeView<T> v;
    v.sy = s.Z;
    v.sx = s.Y * s.Z;
    v.p = base + (size_t)s.ox * v.sx + (size_t)s.oy * v.sy;
    return v;
}

// Where a one-foot result of arrival point (i, j, k) is stored:
// out[off + i*sx + j*sy + k].  sx == 0 selects the ghost-shaped array of the
// component (interior entry (i+1, j+1, k+1)).
struct OutMap {
    long long off, sx, sy;
};

template <typename T>
__host__ __device__ inline NodeView<T> node_view(const T *base, int NY, int NZ)
{
    NodeView<T> v;
    v.p = base;
    v.sy = NZ;
    v.sx = NY * NZ;
    return v;
}

__device__ __forceinline__ int wrap_index(int i, int n)
{
    // an already wrapped base in [0, n) plus an offset in [-3, 3]: one
    // branch-free correction each way when n >= 4 (n is uniform, so the
    // fallback loop for tiny periods costs no divergence)
    if (n >= 4) {
        i += (i < 0) ? n : 0;
        i -= (i >= n) ? n : 0;
        return i;
    }
    while (i < 0) i += n;
    while (i >= n) i -= n;
    return i;
}

__device__ __forceinline__ int wrap_base(double f, int n)
{
    // f = floor(s), an integer-valued double.  Fast path: already in [0, n)
    // (every foot within a period); otherwise reduce with floor division.
    // NaN or huge values end in [0, n) too, so indices never leave the array.
    const double dn = (double)n;
    if (f >= 0.0 && f < dn) return (int)f;
    double r = f - dn * floor(f / dn);
    if (!(r >= 0.0)) r = 0.0;
    if (r >= dn) r = dn - 1.0;
    return (int)r;
}

// Continuous face index kf in [0, nz] of a physical z: analytic inverse of
// the tanh map (semilag.py:400-411).
__device__ __forceinline__ double face_coord(const SlcParams &P, double z)
{
    const double lo = -1.0 + 1e-15, hi = 1.0 - 1e-15;
    if (P.symmetric) {
        double arg = (z * P.two_over_Lz - 1.0) * P.tanh_g;
        arg = fmin(fmax(arg, lo), hi);
        return (atanh(arg) * P.inv_gamma + 1.0) * P.half_nz;
    } else {
        double arg = (1.0 - z * P.inv_Lz) * P.tanh_g;
        arg = fmin(fmax(arg, lo), hi);
        return (1.0 - atanh(arg) * P.inv_gamma) * P.nzd;
    }
}

// Face cell c = clamp(floor(kf), 0, nz-1) (semilag.py:413-416).
__device__ __forceinline__ int face_cell(const SlcParams &P, double z)
{
    double kf = floor(face_coord(P, z));
    kf = fmin(fmax(kf, 0.0), (double)(P.nz - 1));  // NaN -> 0
    return (int)kf;
}

// Interval index m0 with znodes[m0] <= z < znodes[m0+1] (semilag.py:417-420).
__device__ __forceinline__ int locate_m0(const SlcParams &P, bool centers, int c, double z)
{
    if (!centers) return c;
    return c + (z >= __ldg(P.zc + c + 1) ? 1 : 0);
}

// Lagrange weights on the integer offsets m - (O/2 - 1), t in [0, 1)
// (semilag.py:426-439), via prefix/suffix products.
template <int O, typename T>
__device__ __forceinline__ void uniform_weights(const SlcParams &P, T t, T (&w)[O])
{
    constexpr int h = O / 2 - 1;
    T d[O];
#pragma unroll
    for (int l = 0; l < O; ++l) d[l] = t - (T)(l - h);
    T pre[O];
    pre[0] = (T)1;
#pragma unroll
    for (int l = 1; l < O; ++l) pre[l] = pre[l - 1] * d[l - 1];
    T suf = (T)1;
#pragma unroll
    for (int m = O - 1; m >= 0; --m) {
        w[m] = pre[m] * suf * (T)P.udenom[O][m];
        suf = suf * d[m];
    }
}

// Lagrange inverse-denominator tables (semilag.py:102-114) are stored
// node-major: the factor of stencil node m for the stencil starting at z node
// b is dinv[m * rows + b], rows = NZ - O + 1 stencil starts, so lanes at
// consecutive b read consecutive words.
__host__ __device__ inline int denom_rows(bool centers, int nz, int O)
{
    return (centers ? nz + 2 : nz + 1) - O + 1;
}

// Nonuniform Lagrange weights against the actual z nodes (semilag.py:441-454).
template <int O, typename T>
__device__ __forceinline__ void z_weights(const T *__restrict__ zn, const T *__restrict__ dinv,
                                          int rows, int k0, T z, T (&w)[O])
{
    T d[O];
#pragma unroll
    for (int l = 0; l < O; ++l) d[l] = z - __ldg(zn + k0 + l);
    T pre[O];
    pre[0] = (T)1;
#pragma unroll
    for (int l = 1; l < O; ++l) pre[l] = pre[l - 1] * d[l - 1];
    T suf = (T)1;
    const T *di = dinv + k0;
#pragma unroll
    for (int m = O - 1; m >= 0; --m) {
        w[m] = pre[m] * suf * __ldg(di + m * rows);
        suf = suf * d[m];
    }
}

// Full Lagrange stencil of order O for component C at (x, y, z), z already
// inside [z_lo, z_hi] (semilag.py:471-500).
template <int O, typename T>
struct Stencil {
    int xoff[O];  // i * sx for the O x-nodes (wrapped)
    int yoff[O];  // j * sy for the O y-nodes (wrapped)
    int k0;
    T wx[O], wy[O], wz[O];
};

template <int C, int O, typename T>
__device__ __forceinline__ void build_stencil(const SlcParams &P, int sx, int sy, double x, double y,
                                              double z, int c_face, Stencil<O, T> &st)
{
    constexpr int h = O / 2 - 1;
    const int NZ = Comp<C>::centers ? P.nz + 2 : P.nz + 1;
    double s = x * P.inv_dx + Comp<C>::shift_x;
    double f = floor(s);
    T t = (T)(s - f);
    int b = wrap_base(f, P.nx);
#pragma unroll
    for (int m = 0; m < O; ++m) st.xoff[m] = wrap_index(b + m - h, P.nx) * sx;
    uniform_weights<O, T>(P, t, st.wx);

    s = y * P.inv_dy + Comp<C>::shift_y;
    f = floor(s);
    t = (T)(s - f);
    b = wrap_base(f, P.ny);
#pragma unroll
    for (int m = 0; m < O; ++m) st.yoff[m] = wrap_index(b + m - h, P.ny) * sy;
    uniform_weights<O, T>(P, t, st.wy);

    int m0 = locate_m0(P, Comp<C>::centers, c_face, z);
    int k0 = min(max(m0 - h, 0), NZ - O);
    st.k0 = k0;
    const double *zn = Comp<C>::centers ? P.zc : P.zf;
    const double *dinv = Comp<C>::centers ? P.dinv_c[O] : P.dinv_f[O];
    if constexpr (sizeof(T) == 8) {
        z_weights<O, double>(zn, dinv, NZ - O + 1, k0, z, st.wz);
    } else {
        const float *zn32 = Comp<C>::centers ? P.zc32 : P.zf32;
        const float *dinv32 = Comp<C>::centers ? P.dinv_c32[O] : P.dinv_f32[O];
        z_weights<O, float>(zn32, dinv32, NZ - O + 1, k0, (float)z, st.wz);
    }
}

// Separable tensor-product contraction: z first (O^3 FMAs), then y, then x
// (the reference sums the O^3 products in one sequence, semilag.py:44-59;
// the grouping here differs only by rounding).
template <int O, typename T, typename A>
__device__ __forceinline__ A gather_sum(const T *__restrict__ F, const Stencil<O, T> &st)
{
    A acc = (A)0;
#pragma unroll
    for (int i = 0; i < O; ++i) {
        A accy = (A)0;
#pragma unroll
        for (int j = 0; j < O; ++j) {
            const T *row = F + st.xoff[i] + st.yoff[j] + st.k0;
            A accz = (A)0;
#pragma unroll
            for (int k = 0; k < O; ++k) accz = fma((A)st.wz[k], (A)__ldg(row + k), accz);
            accy = fma((A)st.wy[j], accz, accy);
        }
        acc = fma((A)st.wx[i], accy, acc);
    }
    return acc;
}

// One trilinear sample of node view V from precomputed corner indices and
// weights (x: i0, i1, tx; y: j0, j1, ty; z: k0, wz0, wz1).
template <typename T>
__device__ __forceinline__ double tri_sample(NodeView<T> V, int i0, int i1, double tx, int j0, int j1,
                                             double ty, int k0, double wz0, double wz1)
{
    const T *p00 = V.p + i0 * V.sx + j0 * V.sy + k0;
    const T *p01 = V.p + i0 * V.sx + j1 * V.sy + k0;
    const T *p10 = V.p + i1 * V.sx + j0 * V.sy + k0;
    const T *p11 = V.p + i1 * V.sx + j1 * V.sy + k0;
    const double a00 = wz0 * (double)__ldg(p00) + wz1 * (double)__ldg(p00 + 1);
    const double a01 = wz0 * (double)__ldg(p01) + wz1 * (double)__ldg(p01 + 1);
    const double a10 = wz0 * (double)__ldg(p10) + wz1 * (double)__ldg(p10 + 1);
    const double a11 = wz0 * (double)__ldg(p11) + wz1 * (double)__ldg(p11 + 1);
    const double wx0 = 1.0 - tx, wy0 = 1.0 - ty;
    return wx0 * (wy0 * a00 + ty * a01) + tx * (wy0 * a10 + ty * a11);
}

// The pieces of the three trilinear stencils at one point that the staggered
// components share (semilag.py:512-528 with traj_order = 2): x offsets with
// shift 0 (u) and -1/2 (v, w), y offsets with shift 0 (v) and -1/2 (u, w),
// z intervals on the centres (u, v) and on the faces (w).
struct TriShared {
    int ia0, ia1, ib0, ib1;  // x: shift 0 / -1/2
    int ja0, ja1, jb0, jb1;  // y: shift 0 / -1/2
    double txa, txb, tya, tyb;
    int kc, kf;              // z interval bases: centres / faces
    double wc0, wc1, wf0, wf1;
};

__device__ __forceinline__ void tri_shared(const SlcParams &P, double x, double y, double z,
                                           int c_face, TriShared &t)
{
    double sa = x * P.inv_dx;
    double f = floor(sa);
    t.txa = sa - f;
    t.ia0 = wrap_base(f, P.nx);
    t.ia1 = (t.ia0 + 1 == P.nx) ? 0 : t.ia0 + 1;
    double sb = sa - 0.5;
    f = floor(sb);
    t.txb = sb - f;
    t.ib0 = wrap_base(f, P.nx);
    t.ib1 = (t.ib0 + 1 == P.nx) ? 0 : t.ib0 + 1;
    sa = y * P.inv_dy;
    f = floor(sa);
    t.tya = sa - f;
    t.ja0 = wrap_base(f, P.ny);
    t.ja1 = (t.ja0 + 1 == P.ny) ? 0 : t.ja0 + 1;
    sb = sa - 0.5;
    f = floor(sb);
    t.tyb = sb - f;
    t.jb0 = wrap_base(f, P.ny);
    t.jb1 = (t.jb0 + 1 == P.ny) ? 0 : t.jb0 + 1;
    // centres: interval m0 = c + (z >= zc[c+1]), clamped to [0, nz]; faces: c in [0, nz-1]
    int kc = c_face + (z >= __ldg(P.zc + c_face + 1) ? 1 : 0);
    kc = min(max(kc, 0), P.nz);
    const int kf = min(max(c_face, 0), P.nz - 1);
    t.kc = kc;
    t.kf = kf;
    const double *dc = P.dinv_c[2] + kc;  // order-2 tables: nz+1 / nz rows
    const double *df = P.dinv_f[2] + kf;
    t.wc0 = (z - __ldg(P.zc + kc + 1)) * __ldg(dc);
    t.wc1 = (z - __ldg(P.zc + kc)) * __ldg(dc + P.nz + 1);
    t.wf0 = (z - __ldg(P.zf + kf + 1)) * __ldg(df);
    t.wf1 = (z - __ldg(P.zf + kf)) * __ldg(df + P.nz);
}

// Node value accessor for the arrival-point sample below (FP64 node views).
struct NodeValF64 {
    __device__ __forceinline__ double operator()(NodeView<double> V, int I, int J, int K) const
    {
        return __ldg(V.p + I * V.sx + J * V.sy + K);
    }
};

// The trajectory velocity at the arrival point of component C (the first
// fixed-point iteration of semilag.py:542-549, which samples at x_m = x_a).
// The arrival point is a node of its own component and a cell centre/face of
// the others, so the trilinear weights are exact halves and node values
// (z between faces or centres uses the actual node tables):
//   u at (i+1, j+1/2, c_{k+1}), v at (i+1/2, j+1, c_{k+1}), w at (i+1/2, j+1/2, f_{k+1})
// in units of (dx, dy) and node tables c = z_c, f = z_f.  The reference's
// generic weights agree with these to round-off.
template <int C, class V3, class Val>
__device__ __forceinline__ void arrival_sample(const SlcParams &P, const V3 &M, int i, int j, int k,
                                               Val val, double &us, double &vs, double &ws)
{
    const int ip = (i + 1 == P.nx) ? 0 : i + 1;
    const int jp = (j + 1 == P.ny) ? 0 : j + 1;
    if (C == 0) {
        us = val(M.u, ip, j, k + 1);
        vs = 0.25 * ((val(M.v, i, j, k + 1) + val(M.v, ip, j, k + 1)) +
                     (val(M.v, i, jp, k + 1) + val(M.v, ip, jp, k + 1)));
        const double z = __ldg(P.zc + k + 1);
        const double *df = P.dinv_f[2] + k;  // face interval k
        const double w0 = (z - __ldg(P.zf + k + 1)) * __ldg(df);
        const double w1 = (z - __ldg(P.zf + k)) * __ldg(df + P.nz);
        ws = 0.5 * ((w0 * val(M.w, i, j, k) + w1 * val(M.w, i, j, k + 1)) +
                    (w0 * val(M.w, ip, j, k) + w1 * val(M.w, ip, j, k + 1)));
    } else if (C == 1) {
        us = 0.25 * ((val(M.u, i, j, k + 1) + val(M.u, ip, j, k + 1)) +
                     (val(M.u, i, jp, k + 1) + val(M.u, ip, jp, k + 1)));
        vs = val(M.v, i, jp, k + 1);
        const double z = __ldg(P.zc + k + 1);
        const double *df = P.dinv_f[2] + k;
        const double w0 = (z - __ldg(P.zf + k + 1)) * __ldg(df);
        const double w1 = (z - __ldg(P.zf + k)) * __ldg(df + P.nz);
        ws = 0.5 * ((w0 * val(M.w, i, j, k) + w1 * val(M.w, i, j, k + 1)) +
                    (w0 * val(M.w, i, jp, k) + w1 * val(M.w, i, jp, k + 1)));
    } else {
        const double z = __ldg(P.zf + k + 1);
        const double *dc = P.dinv_c[2] + (k + 1);  // centre interval k+1
        const double c0 = (z - __ldg(P.zc + k + 2)) * __ldg(dc);
        const double c1 = (z - __ldg(P.zc + k + 1)) * __ldg(dc + P.nz + 1);
        us = 0.5 * ((c0 * val(M.u, i, j, k + 1) + c1 * val(M.u, i, j, k + 2)) +
                    (c0 * val(M.u, ip, j, k + 1) + c1 * val(M.u, ip, j, k + 2)));
        vs = 0.5 * ((c0 * val(M.v, i, j, k + 1) + c1 * val(M.v, i, j, k + 2)) +
                    (c0 * val(M.v, i, jp, k + 1) + c1 * val(M.v, i, jp, k + 2)));
        ws = val(M.w, i, j, k + 1);
    }
}

// Arrival point of flat interior index (i, j, k) of component C
// (semilag.py:292-307).
template <int C>
__device__ __forceinline__ void arrival_point(const SlcParams &P, int i, int j, int k, double &xa,
                                              double &ya, double &za)
{
    double ar = (double)(i + 1), aj = (double)(j + 1);
    if (C == 0) {
        xa = ar * P.dx;
        ya = (aj - 0.5) * P.dy;
        za = __ldg(P.zc + k + 1);
    } else if (C == 1) {
        xa = (ar - 0.5) * P.dx;
        ya = aj * P.dy;
        za = __ldg(P.zc + k + 1);
    } else {
        xa = (ar - 0.5) * P.dx;
        ya = (aj - 0.5) * P.dy;
        za = __ldg(P.zf + k + 1);
    }
}

// torch.clamp semantics: NaN stays NaN (the stencil locate below guards its
// indices, so a NaN coordinate yields a NaN value, never a stray access).
__device__ __forceinline__ double clampz(const SlcParams &P, double z)
{
    return z < P.z_lo ? P.z_lo : (z > P.z_hi ? P.z_hi : z);
}

// ---------------------------------------------------------------------------
// Mixed form: a component stored as an FP32 node buffer of fluctuations about
// an FP64 per-level (plane-mean) profile, value(i,j,k) = mean[k] + f[i,j,k]
// (mean32: the profile rounded to FP32, for trajectory samples).
// ---------------------------------------------------------------------------
struct MixedView {
    NodeView<float> f;
    const double *mean;
    const float *mean32;
};

template <int O>
struct StencilM {
    int xoff[O], yoff[O], k0;
    float wx[O], wy[O], wz[O];
};
