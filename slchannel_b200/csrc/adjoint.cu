// adjoint.cu -- reverse mode of the SL-BDF2 step and of its BDF1 bootstrap
// (solver.py:729-1018) for a loss on the velocity, FP64.
//
// The step is V^{n+1} = B(P(Z(SL(V^{n-1}, V^n)))) with ghost refreshes in
// between: SL the fused trace + Lagrange gather + BDF2 combination, Z the
// theta = 1 z-solve, P the FFT-Poisson projection and B the exact bulk shift.
// Given lambda^{n+1} = dJ/dV^{n+1}, slc_adjoint_step adds the step's
// contributions to lambda^n and lambda^{n-1}:
//  * ghost refresh (apply_bc_all, solver.py:70-107): every ghost is a signed
//    copy of one interior value, so its transpose folds ghost adjoints into
//    their sources (a pull over each interior value's ghost preimages);
//  * bulk shift u += U_b - sum(w u): lambda_u -= w * sum(lambda_u);
//  * projection u - G L^-1 D u: lambda - D^T L^-T G^T lambda, where L^-T is
//    the same rfft2 / per-(kx, ky) tridiagonal / irfft2 pipeline with every
//    column's system transposed (the Fourier basis diagonalises the x, y
//    part and the coefficients are real);
//  * z-solve A^-1: A^-T per column (sequential Thomas on the transpose);
//  * SL: the gather's transpose is a deterministic segmented scatter-add.
//    Each foot becomes a record (stencil base, fractional position,
//    coefficient); records are counting-sorted by base (ties by record id),
//    and every target node pulls the records of the O^3 bases whose stencil
//    covers it, in a fixed order.  No floating-point atomics, so reruns agree
//    bit for bit.  The gradient through the foot positions uses the
//    derivative of the Lagrange interpolant at the foot and is propagated
//    back through the midpoint iterations (trilinear samples of U* and their
//    gradients; clamped z components carry no derivative), giving trilinear
//    records on U* = 2V^n - V^{n-1} (U* = V^n in the bootstrap).  The
//    explicit x, y diffusion is the periodic 5-point Laplacian, self-adjoint.
#include <cufft.h>

#include <string>

#include "slc_grid.h"

namespace {

constexpr int kT = 256;
constexpr int kMaxIters = 4;

inline unsigned nblk(long long n, int t = kT) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ int wrapn(int i, int n)
{
    i %= n;
    return i < 0 ? i + n : i;
}

// Periodic wrap of i in (-6, n + 6) (a stencil base plus an offset below 6):
// branch-free for n >= 6 (n is uniform, so no divergence), modulo otherwise.
__device__ __forceinline__ int wrap6(int i, int n)
{
    if (n >= 6) {
        i += (i < 0) ? n : 0;
        i -= (i >= n) ? n : 0;
        return i;
    }
    return wrapn(i, n);
}

struct V3 {
    NodeView<double> u, v, w;
};

// ---- Lagrange basis values and derivatives ----------------------------------
template <int O>
__device__ __forceinline__ void ubasis_all(const SlcParams &P, double t, double (&w)[O],
                                           double (&dw)[O])
{
    constexpr int h = O / 2 - 1;
    double d[O];
#pragma unroll
    for (int l = 0; l < O; ++l) d[l] = t - (double)(l - h);
#pragma unroll
    for (int m = 0; m < O; ++m) {
        double pr = 1.0, s = 0.0;
#pragma unroll
        for (int l = 0; l < O; ++l)
            if (l != m) pr *= d[l];
#pragma unroll
        for (int q = 0; q < O; ++q) {
            if (q == m) continue;
            double pq = 1.0;
#pragma unroll
            for (int l = 0; l < O; ++l)
                if (l != m && l != q) pq *= d[l];
            s += pq;
        }
        w[m] = pr * P.udenom[O][m];
        dw[m] = s * P.udenom[O][m];
    }
}

template <int O>
__device__ __forceinline__ void zbasis_all(const double *zn, const double *dinv, int rows, int k0, double z,
                                           double (&w)[O], double (&dw)[O])
{
    double d[O];
#pragma unroll
    for (int l = 0; l < O; ++l) d[l] = z - __ldg(zn + k0 + l);
#pragma unroll
    for (int m = 0; m < O; ++m) {
        double pr = 1.0, s = 0.0;
#pragma unroll
        for (int l = 0; l < O; ++l)
            if (l != m) pr *= d[l];
#pragma unroll
        for (int q = 0; q < O; ++q) {
            if (q == m) continue;
            double pq = 1.0;
#pragma unroll
            for (int l = 0; l < O; ++l)
                if (l != m && l != q) pq *= d[l];
            s += pq;
        }
        const double di = __ldg(dinv + m * rows + k0);
        w[m] = pr * di;
        dw[m] = s * di;
    }
}

// Stencil base of the order-O gather of component C at (x, y, z), z inside
// [z_lo, z_hi] (the forward's build_stencil): nodes (bx0 + m) mod nx,
// (by0 + m) mod ny, k0 + m.
template <int C, int O>
struct GBase {
    int bx0, by0, k0;
    double tx, ty;
};

template <int C, int O>
__device__ __forceinline__ GBase<C, O> gather_base(const SlcParams &P, double x, double y, double z)
{
    constexpr int h = O / 2 - 1;
    GBase<C, O> g;
    double s = x * P.inv_dx + Comp<C>::shift_x;
    double f = floor(s);
    g.tx = s - f;
    g.bx0 = wrapn(wrap_base(f, P.nx) - h, P.nx);
    s = y * P.inv_dy + Comp<C>::shift_y;
    f = floor(s);
    g.ty = s - f;
    g.by0 = wrapn(wrap_base(f, P.ny) - h, P.ny);
    const int NZ = Comp<C>::centers ? P.nz + 2 : P.nz + 1;
    const int m0 = locate_m0(P, Comp<C>::centers, face_cell(P, z), z);
    g.k0 = min(max(m0 - h, 0), NZ - O);
    return g;
}

// Gradient of the order-O interpolant of node view F at (x, y, z).
template <int C, int O>
__device__ void grad_interp(const SlcParams &P, NodeView<double> F, double x, double y, double z,
                            double &gx, double &gy, double &gz)
{
    const GBase<C, O> b = gather_base<C, O>(P, x, y, z);
    double wx[O], dwx[O], wy[O], dwy[O], wz[O], dwz[O];
    ubasis_all<O>(P, b.tx, wx, dwx);
    ubasis_all<O>(P, b.ty, wy, dwy);
    const double *zn = Comp<C>::centers ? P.zc : P.zf;
    const double *dinv = Comp<C>::centers ? P.dinv_c[O] : P.dinv_f[O];
    zbasis_all<O>(zn, dinv, denom_rows(Comp<C>::centers, P.nz, O), b.k0, z, wz, dwz);
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int i = 0; i < O; ++i) {
        const int xo = wrap6(b.bx0 + i, P.nx) * F.sx;
        double sy_w = 0.0, sy_dw = 0.0, sy_wz = 0.0;
        for (int j = 0; j < O; ++j) {
            const double *row = F.p + xo + wrap6(b.by0 + j, P.ny) * F.sy + b.k0;
            double s = 0.0, sd = 0.0;
#pragma unroll
            for (int k = 0; k < O; ++k) {
                const double v = __ldg(row + k);
                s = fma(wz[k], v, s);
                sd = fma(dwz[k], v, sd);
            }
            sy_w = fma(wy[j], s, sy_w);
            sy_dw = fma(dwy[j], s, sy_dw);
            sy_wz = fma(wy[j], sd, sy_wz);
        }
        ax = fma(dwx[i], sy_w, ax);
        ay = fma(wx[i], sy_dw, ay);
        az = fma(wx[i], sy_wz, az);
    }
    gx = ax * P.inv_dx;
    gy = ay * P.inv_dy;
    gz = az;
}

// Trilinear pieces of field c (0 u, 1 v, 2 w) of the trajectory velocity at
// (x, y, z): base node (i0, j0, k0), fractions and z weights with their
// z-derivatives.
struct TriPiece {
    int i0, i1, j0, j1, k0;
    double tx, ty, wz0, wz1, dwz0, dwz1;
};

__device__ __forceinline__ TriPiece tri_piece(const SlcParams &P, int c, const TriShared &t)
{
    TriPiece r;
    if (c == 0) {
        r.i0 = t.ia0; r.i1 = t.ia1; r.tx = t.txa;
    } else {
        r.i0 = t.ib0; r.i1 = t.ib1; r.tx = t.txb;
    }
    if (c == 1) {
        r.j0 = t.ja0; r.j1 = t.ja1; r.ty = t.tya;
    } else {
        r.j0 = t.jb0; r.j1 = t.jb1; r.ty = t.tyb;
    }
    if (c < 2) {
        r.k0 = t.kc; r.wz0 = t.wc0; r.wz1 = t.wc1;
        r.dwz0 = __ldg(P.dinv_c[2] + t.kc);
        r.dwz1 = __ldg(P.dinv_c[2] + (P.nz + 1) + t.kc);
    } else {
        r.k0 = t.kf; r.wz0 = t.wf0; r.wz1 = t.wf1;
        r.dwz0 = __ldg(P.dinv_f[2] + t.kf);
        r.dwz1 = __ldg(P.dinv_f[2] + P.nz + t.kf);
    }
    return r;
}

// Value and gradient of a trilinear sample.
__device__ __forceinline__ double tri_value_grad(const SlcParams &P, NodeView<double> V, const TriPiece &q,
                                                 double &gx, double &gy, double &gz)
{
    auto at = [&](int i, int j, int k) { return __ldg(V.p + i * V.sx + j * V.sy + k); };
    const double v000 = at(q.i0, q.j0, q.k0), v001 = at(q.i0, q.j0, q.k0 + 1);
    const double v010 = at(q.i0, q.j1, q.k0), v011 = at(q.i0, q.j1, q.k0 + 1);
    const double v100 = at(q.i1, q.j0, q.k0), v101 = at(q.i1, q.j0, q.k0 + 1);
    const double v110 = at(q.i1, q.j1, q.k0), v111 = at(q.i1, q.j1, q.k0 + 1);
    const double a00 = q.wz0 * v000 + q.wz1 * v001, d00 = q.dwz0 * v000 + q.dwz1 * v001;
    const double a01 = q.wz0 * v010 + q.wz1 * v011, d01 = q.dwz0 * v010 + q.dwz1 * v011;
    const double a10 = q.wz0 * v100 + q.wz1 * v101, d10 = q.dwz0 * v100 + q.dwz1 * v101;
    const double a11 = q.wz0 * v110 + q.wz1 * v111, d11 = q.dwz0 * v110 + q.dwz1 * v111;
    const double wx0 = 1.0 - q.tx, wy0 = 1.0 - q.ty;
    const double r0 = wy0 * a00 + q.ty * a01, r1 = wy0 * a10 + q.ty * a11;
    gx = (r1 - r0) * P.inv_dx;
    gy = (wx0 * (a01 - a00) + q.tx * (a11 - a10)) * P.inv_dy;
    gz = wx0 * (wy0 * d00 + q.ty * d01) + q.tx * (wy0 * d10 + q.ty * d11);
    return wx0 * r0 + q.tx * r1;
}

// Trajectory velocity samples (values and gradients) at one point.
__device__ __forceinline__ void sample3_grad(const SlcParams &P, const V3 &M, double x, double y,
                                             double z, double (&s)[3], double (&g)[3][3])
{
    const double zc = clampz(P, z);
    TriShared t;
    tri_shared(P, x, y, zc, face_cell(P, zc), t);
    const NodeView<double> F[3] = {M.u, M.v, M.w};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const TriPiece q = tri_piece(P, c, t);
        s[c] = tri_value_grad(P, F[c], q, g[c][0], g[c][1], g[c][2]);
    }
}

// One foot traced again from the arrival point, and its adjoint: given
// gbar = dJ/d(foot), writes the trilinear sample records (positions m_1 ..
// m_{n-1} with coefficients) and adds -h * dJ/d(m_1) to s0bar.
struct FootTrace {
    double m[kMaxIters][3];   // m[it] = iterate it+1 (z clamped)
    bool zcl[kMaxIters];      // clamp active on iterate it+1's z
    double d[3];              // foot (unclamped z)
};

__device__ __forceinline__ void trace_forward(const SlcParams &P, const V3 &M, const double a[3],
                                              double h, const double s0[3], FootTrace &T)
{
    double zr = a[2] - h * s0[2];
    T.m[0][0] = a[0] - h * s0[0];
    T.m[0][1] = a[1] - h * s0[1];
    T.m[0][2] = clampz(P, zr);
    T.zcl[0] = zr < P.z_lo || zr > P.z_hi;
    for (int it = 1; it < P.n_iters; ++it) {
        double s[3], g[3][3];
        sample3_grad(P, M, T.m[it - 1][0], T.m[it - 1][1], T.m[it - 1][2], s, g);
        zr = a[2] - h * s[2];
        T.m[it][0] = a[0] - h * s[0];
        T.m[it][1] = a[1] - h * s[1];
        T.m[it][2] = clampz(P, zr);
        T.zcl[it] = zr < P.z_lo || zr > P.z_hi;
    }
    const int n = P.n_iters - 1;
#pragma unroll
    for (int c = 0; c < 3; ++c) T.d[c] = 2.0 * T.m[n][c] - a[c];
}

// Records of one trilinear sample: position (z clamped) and three coefficients.
struct TriRec {
    double x, y, z, cu, cv, cw;
};

__device__ __forceinline__ void trace_backward(const SlcParams &P, const V3 &M, const FootTrace &T,
                                               double h, const double gbar[3], double s0bar[3],
                                               TriRec *out, long long slot_stride)
{
    const int n = P.n_iters - 1;
    double mb[3] = {2.0 * gbar[0], 2.0 * gbar[1], 2.0 * gbar[2]};
    if (T.zcl[n]) mb[2] = 0.0;
    for (int it = n; it >= 1; --it) {
        // m[it] = a - h S(m[it-1]):  sbar = -h mbar
        const double sb[3] = {-h * mb[0], -h * mb[1], -h * mb[2]};
        double s[3], g[3][3];
        sample3_grad(P, M, T.m[it - 1][0], T.m[it - 1][1], T.m[it - 1][2], s, g);
        TriRec r;
        r.x = T.m[it - 1][0];
        r.y = T.m[it - 1][1];
        r.z = T.m[it - 1][2];
        r.cu = sb[0];
        r.cv = sb[1];
        r.cw = sb[2];
        out[(long long)(it - 1) * slot_stride] = r;
        double nb[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) nb[q] = sb[0] * g[0][q] + sb[1] * g[1][q] + sb[2] * g[2][q];
        if (T.zcl[it - 1]) nb[2] = 0.0;
        mb[0] = nb[0];
        mb[1] = nb[1];
        mb[2] = nb[2];
    }
    // m[0] = a - h s0
    s0bar[0] += -h * mb[0];
    s0bar[1] += -h * mb[1];
    s0bar[2] += -h * mb[2];
}

// Per arrival point of component C: the adjoint of the SL predictor.
// Record slots (n = n_iters): slot 0 the arrival sample; slots 1 .. n-1 the
// near foot's iterates; slots n .. 2n-2 the far foot's (MODE 2).
template <int C, int O, int MODE>
__global__ void __launch_bounds__(kT) k_sl_adj_points(SlcParams P, V3 M, const double *__restrict__ fn,
                                                      const double *__restrict__ fnm1,
                                                      const double *__restrict__ lam_hat, double dt,
                                                      double4 *__restrict__ rec_near,
                                                      double4 *__restrict__ rec_far,
                                                      TriRec *__restrict__ tri, long long pbase,
                                                      long long ntot)
{
    const int nzi = (C == 2) ? P.nz - 1 : P.nz;
    const long long np = (long long)P.nx * P.ny * nzi;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const int k = (int)(q % nzi);
    const int j = (int)((q / nzi) % P.ny);
    const int i = (int)(q / ((long long)nzi * P.ny));
    const GhostShape gs = ghost_shape(C, P.nx, P.ny, P.nz);
    const double lam = lam_hat[(size_t)(i + 1) * gs.Y * gs.Z + (size_t)(j + 1) * gs.Z + (k + 1)];
    double a[3];
    arrival_point<C>(P, i, j, k, a[0], a[1], a[2]);
    double s0[3];
    arrival_sample<C>(P, M, i, j, k, NodeValF64(), s0[0], s0[1], s0[2]);
    double s0bar[3] = {0.0, 0.0, 0.0};
    const long long gp = pbase + q;

    // near foot: depth dt (half-step dt / 2)
    {
        FootTrace T;
        trace_forward(P, M, a, 0.5 * dt, s0, T);
        const double zd = T.d[2];
        const double zdc = clampz(P, zd);
        const double coef = (MODE == 2 ? 4.0 / 3.0 : 1.0) * lam;
        double gx, gy, gz;
        grad_interp<C, O>(P, ghost_view<double>(C, fn, P.nx, P.ny, P.nz), T.d[0], T.d[1], zdc, gx, gy, gz);
        if (zd < P.z_lo || zd > P.z_hi) gz = 0.0;
        const double gbar[3] = {coef * gx, coef * gy, coef * gz};
        trace_backward(P, M, T, 0.5 * dt, gbar, s0bar, tri + gp + ntot, ntot);
        rec_near[q] = make_double4(T.d[0], T.d[1], zdc, coef);
    }
    if (MODE == 2) {
        FootTrace T;
        trace_forward(P, M, a, dt, s0, T);
        const double zd = T.d[2];
        const double zdc = clampz(P, zd);
        const double coef = (-1.0 / 3.0) * lam;
        double gx, gy, gz;
        grad_interp<C, O>(P, ghost_view<double>(C, fnm1, P.nx, P.ny, P.nz), T.d[0], T.d[1], zdc, gx, gy,
                          gz);
        if (zd < P.z_lo || zd > P.z_hi) gz = 0.0;
        const double gbar[3] = {coef * gx, coef * gy, coef * gz};
        trace_backward(P, M, T, dt, gbar, s0bar, tri + gp + (long long)P.n_iters * ntot, ntot);
        rec_far[q] = make_double4(T.d[0], T.d[1], zdc, coef);
    }
    TriRec r;
    r.x = a[0];
    r.y = a[1];
    r.z = a[2];
    r.cu = s0bar[0];
    r.cv = s0bar[1];
    r.cw = s0bar[2];
    tri[gp] = r;
}

// ---- records -> (key, payload) -----------------------------------------------
// Gather records (x, y, z, coef) of component C: key = (bx0 * ny + by0) * NZ + k0.
template <int C, int O>
__global__ void k_gather_keys(SlcParams P, const double4 *__restrict__ rec, long long n,
                              int *__restrict__ keys)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const double4 R = rec[r];
    const GBase<C, O> b = gather_base<C, O>(P, R.x, R.y, R.z);
    const int NZ = Comp<C>::centers ? P.nz + 2 : P.nz + 1;
    keys[r] = (b.bx0 * P.ny + b.by0) * NZ + b.k0;
}

// The sorted gather records' separable weights, node-major (SoA) in key order:
// record p adds coef wx[mx] * wy[my] * wz[mz] to node base + (mx, my, mz), with
// W[mx * n + p] = coef wx[mx], W[(O + my) * n + p] = wy[my],
// W[(2 O + mz) * n + p] = wz[mz] (the forward gather's own weight functions)
// and kz[p] its stencil's first z node.
template <int C, int O>
__global__ void __launch_bounds__(kT) k_sorted_weights(SlcParams P, const double4 *__restrict__ rec,
                                                       const int *__restrict__ order, long long n,
                                                       double *__restrict__ W, int *__restrict__ kz)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double4 R = rec[__ldg(order + p)];
    const GBase<C, O> b = gather_base<C, O>(P, R.x, R.y, R.z);
    const int NZ = Comp<C>::centers ? P.nz + 2 : P.nz + 1;
    const double *zn = Comp<C>::centers ? P.zc : P.zf;
    const double *dinv = Comp<C>::centers ? P.dinv_c[O] : P.dinv_f[O];
    double wx[O], wy[O], wz[O];
    uniform_weights<O, double>(P, b.tx, wx);
    uniform_weights<O, double>(P, b.ty, wy);
    z_weights<O, double>(zn, dinv, NZ - O + 1, b.k0, R.z, wz);
#pragma unroll
    for (int m = 0; m < O; ++m) {
        W[(size_t)m * n + p] = R.w * wx[m];
        W[(size_t)(O + m) * n + p] = wy[m];
        W[(size_t)(2 * O + m) * n + p] = wz[m];
    }
    kz[p] = b.k0;
}

// Trilinear records for field c of U*: payload (tx, ty, wz1, coef_c).
__global__ void k_tri_keys(SlcParams P, int c, const TriRec *__restrict__ tri, long long n,
                           int *__restrict__ keys, double4 *__restrict__ pay)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const TriRec R = tri[r];
    const double zc = clampz(P, R.z);
    TriShared t;
    tri_shared(P, R.x, R.y, zc, face_cell(P, zc), t);
    const TriPiece q = tri_piece(P, c, t);
    const int NZ = c < 2 ? P.nz + 2 : P.nz + 1;
    keys[r] = (q.i0 * P.ny + q.j0) * NZ + q.k0;
    const double coef = c == 0 ? R.cu : (c == 1 ? R.cv : R.cw);
    pay[r] = make_double4(q.tx, q.ty, q.wz1, coef);
}

// ---- counting sort by key (integer atomics only; deterministic order) -------
__global__ void k_izero(int *a, long long n)
{
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x)
        a[p] = 0;
}

__global__ void k_count(const int *__restrict__ keys, long long n, int *counts)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) atomicAdd(counts + keys[r], 1);
}

constexpr int kScanT = 1024;

// Exclusive scan of one 1024-element chunk per block; chunk totals to sums.
__global__ void __launch_bounds__(kScanT) k_scan_blocks(const int *__restrict__ in, int *__restrict__ out,
                                                        int *__restrict__ sums, long long n)
{
    __shared__ int warp_tot[32];
    const long long p = (long long)blockIdx.x * kScanT + threadIdx.x;
    const int v = p < n ? in[p] : 0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = warp_tot[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        warp_tot[lane] = t;  // inclusive
    }
    __syncthreads();
    const int before = (w > 0 ? warp_tot[w - 1] : 0) + x - v;
    if (p < n) out[p] = before;
    if (threadIdx.x == kScanT - 1) sums[blockIdx.x] = warp_tot[31];
}

// In-place exclusive scan of the chunk totals (one block, sequential chunks).
__global__ void __launch_bounds__(kScanT) k_scan_sums(int *sums, int nb, int *total)
{
    __shared__ int warp_tot[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < nb; base += kScanT) {
        const int p = base + threadIdx.x;
        const int v = p < nb ? sums[p] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[w] = x;
        __syncthreads();
        if (w == 0) {
            int t = warp_tot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t;
        }
        __syncthreads();
        const int before = carry + (w > 0 ? warp_tot[w - 1] : 0) + x - v;
        const int chunk_total = warp_tot[31];
        __syncthreads();
        if (p < nb) sums[p] = before;
        if (threadIdx.x == 0) carry += chunk_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanT) k_scan_add(int *out, const int *__restrict__ sums, long long n)
{
    const long long p = (long long)blockIdx.x * kScanT + threadIdx.x;
    if (p < n) out[p] += sums[blockIdx.x];
}

__global__ void k_place(const int *__restrict__ keys, long long n, const int *__restrict__ starts,
                        int *fill, int *__restrict__ order)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int key = keys[r];
    const int pos = starts[key] + atomicAdd(fill + key, 1);
    order[pos] = (int)r;
}

// Each segment's record ids ascending (insertion sort; segments are short).
__global__ void k_sort_segments(const int *__restrict__ starts, long long nkeys, int *order)
{
    const long long key = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (key >= nkeys) return;
    const int a = starts[key], b = starts[key + 1];
    for (int p = a + 1; p < b; ++p) {
        const int v = order[p];
        int q = p - 1;
        while (q >= a && order[q] > v) {
            order[q + 1] = order[q];
            --q;
        }
        order[q + 1] = v;
    }
}

// ---- pulls: every target node sums the records whose stencil covers it -----
// For each (mx, my), the stencil starts covering node iz along z are the
// consecutive keys k0 = iz - O + 1 .. iz, so their records are one contiguous
// range of the sorted order: two starts loads per (mx, my), then four
// coalesced loads per record (lanes are consecutive iz, their ranges shifted
// by one key).  Records are summed in key order, then record id: a fixed
// order, so the result is reproducible bit for bit.
#ifndef SLC_PULL_UNROLL
#define SLC_PULL_UNROLL 2
#endif
constexpr int kPullUnroll = SLC_PULL_UNROLL;  // records per trip of the pull's inner loop
template <int C, int O>
__global__ void __launch_bounds__(kT) k_pull_gather(SlcParams P, const double *__restrict__ W,
                                                    const int *__restrict__ kz, long long nrec,
                                                    const int *__restrict__ starts, double *lam)
{
    const int NZ = Comp<C>::centers ? P.nz + 2 : P.nz + 1;
    const long long nn = (long long)P.nx * P.ny * NZ;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nn) return;
    const int iz = (int)(t % NZ);
    const int iy = (int)((t / NZ) % P.ny);
    const int ix = (int)(t / ((long long)NZ * P.ny));
    const int klo = max(iz - (O - 1), 0), khi = min(iz, NZ - O);
    double acc = 0.0;
    if (klo <= khi) {
        for (int mx = 0; mx < O; ++mx) {
            const int bx = wrap6(ix - mx, P.nx);
            const double *cwx = W + (size_t)mx * nrec;
            for (int my = 0; my < O; ++my) {
                const int by = wrap6(iy - my, P.ny);
                const double *wyv = W + (size_t)(O + my) * nrec;
                const int kb = (bx * P.ny + by) * NZ;
                const int a = __ldg(starts + kb + klo), b = __ldg(starts + kb + khi + 1);
#pragma unroll kPullUnroll
                for (int p = a; p < b; ++p) {
                    const int mz = iz - __ldg(kz + p);
                    const double wz = __ldg(W + (size_t)(2 * O + mz) * nrec + p);
                    acc = fma(__ldg(cwx + p) * __ldg(wyv + p), wz, acc);
                }
            }
        }
    }
    const NodeView<double> V = ghost_view<double>(C, lam, P.nx, P.ny, P.nz);
    double *dst = const_cast<double *>(V.p) + (size_t)ix * V.sx + (size_t)iy * V.sy + iz;
    *dst += acc;
}

// Trilinear transposes in two passes.  About 9 records share each base key
// (every arrival point's trajectory samples land in each field's grid), so
// (1) one thread per key sums its records into the 8 corner partials of that
// base, records in sorted order, stored corner-major S[corner * nkeys + key];
// (2) each node adds the partials of the 8 bases covering it, corners in a
// fixed order.  Both orders are fixed, so the result is reproducible.
__global__ void __launch_bounds__(kT) k_tri_segsum(const double4 *__restrict__ pay,
                                                   const int *__restrict__ order,
                                                   const int *__restrict__ starts, long long nkeys,
                                                   double *__restrict__ S)
{
    const long long key = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (key >= nkeys) return;
    double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const int a = __ldg(starts + key), b = __ldg(starts + key + 1);
    for (int p = a; p < b; ++p) {
        const double4 R = pay[__ldg(order + p)];
        const double wx[2] = {1.0 - R.x, R.x}, wy[2] = {1.0 - R.y, R.y}, wz[2] = {1.0 - R.z, R.z};
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] = fma(R.w, wx[q >> 2] * wy[(q >> 1) & 1] * wz[q & 1], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) S[(size_t)q * nkeys + key] = acc[q];
}

__global__ void __launch_bounds__(kT) k_pull_tri(SlcParams P, int c, const double *__restrict__ S,
                                                 double *lam)
{
    const int NZ = c < 2 ? P.nz + 2 : P.nz + 1;
    const int kmax = c < 2 ? P.nz : P.nz - 1;  // largest base interval
    const long long nn = (long long)P.nx * P.ny * NZ;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nn) return;
    const int iz = (int)(t % NZ);
    const int iy = (int)((t / NZ) % P.ny);
    const int ix = (int)(t / ((long long)NZ * P.ny));
    double acc = 0.0;
#pragma unroll
    for (int mx = 0; mx < 2; ++mx) {
        const int bx = wrap6(ix - mx, P.nx);
#pragma unroll
        for (int my = 0; my < 2; ++my) {
            const int by = wrap6(iy - my, P.ny);
#pragma unroll
            for (int mz = 0; mz < 2; ++mz) {
                const int k0 = iz - mz;
                if (k0 < 0 || k0 > kmax) continue;
                const long long key = ((long long)bx * P.ny + by) * NZ + k0;
                acc += __ldg(S + (size_t)(mx * 4 + my * 2 + mz) * nn + key);
            }
        }
    }
    const NodeView<double> V = ghost_view<double>(c, lam, P.nx, P.ny, P.nz);
    double *dst = const_cast<double *>(V.p) + (size_t)ix * V.sx + (size_t)iy * V.sy + iz;
    *dst += acc;
}

// ---- explicit x, y diffusion: periodic Laplacian of lam_hat, added twice ----
template <int C>
__global__ void k_diff_adj(SlcParams P, const double *__restrict__ lh, double *lc, double cc,
                           double *lp, double cp)
{
    const int nzi = (C == 2) ? P.nz - 1 : P.nz;
    const long long np = (long long)P.nx * P.ny * nzi;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const int k = (int)(q % nzi);
    const int j = (int)((q / nzi) % P.ny);
    const int i = (int)(q / ((long long)nzi * P.ny));
    const GhostShape g = ghost_shape(C, P.nx, P.ny, P.nz);
    const size_t sx = (size_t)g.Y * g.Z, sy = g.Z;
    auto at = [&](int ii, int jj) {
        return lh[(size_t)(wrap6(ii, P.nx) + 1) * sx + (size_t)(wrap6(jj, P.ny) + 1) * sy + (k + 1)];
    };
    const double c0 = at(i, j);
    const double lap = (at(i + 1, j) - 2.0 * c0 + at(i - 1, j)) * P.inv_dx2 +
                       (at(i, j + 1) - 2.0 * c0 + at(i, j - 1)) * P.inv_dy2;
    const size_t idx = (size_t)(i + 1) * sx + (size_t)(j + 1) * sy + (k + 1);
    lc[idx] += cc * P.nu * lap;
    if (lp) lp[idx] += cp * P.nu * lap;
}

// ---- ghost refresh transpose ---------------------------------------------------
template <int C>
__global__ void k_bc_adj(SlcParams P, double *lam)
{
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int nzi = (C == 2) ? nz - 1 : nz;
    const long long np = (long long)nx * ny * nzi;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const int K = (int)(q % nzi) + 1;
    const int J = (int)((q / nzi) % ny) + 1;
    const int I = (int)(q / ((long long)nzi * ny)) + 1;
    const GhostShape g = ghost_shape(C, nx, ny, nz);
    int px[3], py[3], pz[3], nxp = 0, nyp = 0, nzp = 0;
    double sz[3];
    px[nxp++] = I;
    if (I == nx) px[nxp++] = 0;
    if (C != 0 && I == 1) px[nxp++] = nx + 1;
    py[nyp++] = J;
    if (J == ny) py[nyp++] = 0;
    if (C != 1 && J == 1) py[nyp++] = ny + 1;
    pz[nzp] = K;
    sz[nzp++] = 1.0;
    if (C != 2) {
        if (K == 1) {
            pz[nzp] = 0;
            sz[nzp++] = -1.0;
        }
        if (K == nz) {
            pz[nzp] = nz + 1;
            sz[nzp++] = P.top_neumann ? 1.0 : -1.0;
        }
    }
    double acc = 0.0;
    for (int a = 0; a < nxp; ++a)
        for (int b = 0; b < nyp; ++b)
            for (int c = 0; c < nzp; ++c)
                acc += sz[c] * lam[(size_t)px[a] * g.Y * g.Z + (size_t)py[b] * g.Z + pz[c]];
    lam[(size_t)I * g.Y * g.Z + (size_t)J * g.Z + K] = acc;
}

// zero every element outside the interior box (ghosts and w walls)
template <int C>
__global__ void k_zero_ghosts(SlcParams P, double *lam)
{
    const GhostShape g = ghost_shape(C, P.nx, P.ny, P.nz);
    const long long n = (long long)g.X * g.Y * g.Z;
    const int kmax = (C == 2) ? P.nz - 1 : P.nz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int K = (int)(t % g.Z);
        const int J = (int)((t / g.Z) % g.Y);
        const int I = (int)(t / ((long long)g.Z * g.Y));
        const bool interior = I >= 1 && I <= P.nx && J >= 1 && J <= P.ny && K >= 1 && K <= kmax;
        if (!interior) lam[t] = 0.0;
    }
}

// ---- bulk shift transpose: lam_u -= w_k * sum(lam_u) ------------------------
constexpr int kSumBlocks = 592;

__global__ void __launch_bounds__(kT) k_sum_partials(SlcParams P, const double *__restrict__ u,
                                                     double *partials)
{
    __shared__ double red[kT];
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    double acc = 0.0;
    for (long long col = blockIdx.x; col < (long long)nx * ny; col += gridDim.x) {
        const int i = (int)(col / ny), j = (int)(col % ny);
        for (int k = threadIdx.x; k < nz; k += blockDim.x)
            acc += u[(size_t)(i + 1) * usx + (size_t)(j + 1) * usy + 1 + k];
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(kT) k_sum_finish(const double *__restrict__ partials, int n,
                                                   double *out)
{
    __shared__ double red[kT];
    double acc = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) acc += partials[b];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

__global__ void k_bulk_adj_apply(SlcParams P, double *u, const double *__restrict__ dz_f,
                                 const double *__restrict__ S, double w_scale)
{
    const long long n = (long long)P.nx * P.ny * P.nz;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int k = (int)(q % P.nz);
    const int j = (int)((q / P.nz) % P.ny);
    const int i = (int)(q / ((long long)P.nz * P.ny));
    const size_t usx = (size_t)(P.ny + 2) * (P.nz + 2), usy = P.nz + 2;
    u[(size_t)(i + 1) * usx + (size_t)(j + 1) * usy + 1 + k] -= w_scale * dz_f[k] * (*S);
}

// ---- projection transpose -------------------------------------------------------
// psi[k][i][j] = (G^T lam)(i, j, k), G the forward's gradient (projection.py:250-272).
__global__ void k_gradT_pack(SlcParams P, const double *__restrict__ lu, const double *__restrict__ lv,
                             const double *__restrict__ lw, const double *__restrict__ dz_c,
                             double *__restrict__ psi)
{
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const long long n = (long long)nx * ny * nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int j = (int)(t % ny);
    const int i = (int)((t / ny) % nx);
    const int k = (int)(t / ((long long)ny * nx));
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    const size_t vsx = (size_t)(ny + 1) * (nz + 2), vsy = nz + 2;
    const size_t wsx = (size_t)(ny + 2) * (nz + 1), wsy = nz + 1;
    const int im = i == 0 ? nx - 1 : i - 1, jm = j == 0 ? ny - 1 : j - 1;
    auto U = [&](int ii, int jj) { return lu[(size_t)(ii + 1) * usx + (size_t)(jj + 1) * usy + k + 1]; };
    auto Vv = [&](int ii, int jj) { return lv[(size_t)(ii + 1) * vsx + (size_t)(jj + 1) * vsy + k + 1]; };
    double s = (U(im, j) - U(i, j)) * P.inv_dx + (Vv(i, jm) - Vv(i, j)) * P.inv_dy;
    const size_t wc = (size_t)(i + 1) * wsx + (size_t)(j + 1) * wsy;
    if (k >= 1) s += lw[wc + k] / dz_c[k];             // w face k (interior k-1)
    if (k <= nz - 2) s -= lw[wc + k + 1] / dz_c[k + 1];  // w face k+1 (interior k)
    psi[t] = s;
}

// Transposed Thomas sweep per (kx, ky) column (the forward's rows, with the
// sub- and super-diagonals exchanged), 1/(nx ny) folded in.
__global__ void __launch_bounds__(kT) k_thomas_T(SlcParams P, double *__restrict__ hat,
                                                 double *__restrict__ cpw, const double *__restrict__ kx2,
                                                 const double *__restrict__ ky2,
                                                 const double *__restrict__ cl,
                                                 const double *__restrict__ cr, double norm)
{
    const int nky = P.ny / 2 + 1;
    const int ncol = P.nx * nky;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int col = t >> 1, part = t & 1;
    const bool active = col < ncol;
    const int nz = P.nz;
    const size_t st = 2 * (size_t)ncol;
    double *h = hat + 2 * (size_t)(active ? col : 0) + part;
    double *cpc = cpw + (active ? col : 0);
    double k2 = 0.0;
    if (active) {
        const int kx = col / nky, ky = col - (col / nky) * nky;
        k2 = kx2[kx] + ky2[ky];
    }
    auto rows = [&](int k, double &a, double &b, double &c) {
        a = k > 0 ? cl[k] : 0.0;
        b = -(cl[k] + cr[k] + k2);
        if (k == 0) b += cl[0];
        if (k == nz - 1) b += cr[nz - 1];
        c = k < nz - 1 ? cr[k] : 0.0;
        if (col == 0 && k == 0) {
            b = 1.0;
            c = 0.0;
        }
    };
    if (active) {
        double cprev = 0.0, dprev = 0.0;
        for (int k = 0; k < nz; ++k) {
            double a, b, c, an, bn, cn, ap, bp, cpv;
            rows(k, a, b, c);
            // transpose: sub_k = c_{k-1}, super_k = a_{k+1}
            double sub = 0.0, sup = 0.0;
            if (k > 0) {
                rows(k - 1, ap, bp, cpv);
                sub = cpv;
            }
            if (k < nz - 1) {
                rows(k + 1, an, bn, cn);
                sup = an;
            }
            const double id = 1.0 / (b - sub * cprev);
            cprev = sup * id;
            dprev = (h[k * st] - sub * dprev) * id;
            h[k * st] = dprev;
            if (part == 0) cpc[k * (size_t)ncol] = cprev;
        }
    }
    __syncwarp();
    if (active) {
        double x = 0.0;
        for (int k = nz - 1; k >= 0; --k) {
            const double dk = h[k * st];
            x = (k == nz - 1) ? dk : dk - cpc[k * (size_t)ncol] * x;
            h[k * st] = x * norm;
        }
    }
}

// lam -= c * D^T phi (phi z-major), D the forward's divergence (utils.py:166-180).
__global__ void k_divT(SlcParams P, const double *__restrict__ phi, const double *__restrict__ dz_f,
                       double c, double *lu, double *lv, double *lw)
{
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const long long n = (long long)nx * ny * nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int k = (int)(t % nz);
    const int j = (int)((t / nz) % ny);
    const int i = (int)(t / ((long long)nz * ny));
    auto F = [&](int ii, int jj, int kk) { return phi[((size_t)kk * nx + ii) * ny + jj]; };
    const int ip = i + 1 == nx ? 0 : i + 1, jp = j + 1 == ny ? 0 : j + 1;
    const double f0 = F(i, j, k);
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    const size_t vsx = (size_t)(ny + 1) * (nz + 2), vsy = nz + 2;
    const size_t wsx = (size_t)(ny + 2) * (nz + 1), wsy = nz + 1;
    lu[(size_t)(i + 1) * usx + (size_t)(j + 1) * usy + k + 1] -= c * (f0 - F(ip, j, k)) * P.inv_dx;
    lv[(size_t)(i + 1) * vsx + (size_t)(j + 1) * vsy + k + 1] -= c * (f0 - F(i, jp, k)) * P.inv_dy;
    if (k < nz - 1)  // interior w face k+1: div(k) has +w/dz_f[k], div(k+1) has -w/dz_f[k+1]
        lw[(size_t)(i + 1) * wsx + (size_t)(j + 1) * wsy + k + 1] -=
            c * (f0 / dz_f[k] - F(i, j, k + 1) / dz_f[k + 1]);
}

// ---- z-solve transpose: A^T x = d per column -----------------------------------
__global__ void k_zsolve_T(SlcParams P, const double *__restrict__ dz_c, const double *__restrict__ dz_f,
                           double dt, double *lu, double *lv, double *lw, double *scratch)
{
    const long long ncol = (long long)P.nx * P.ny;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * ncol) return;
    const int comp = (int)(t / ncol);
    const int col = (int)(t % ncol);
    const int i = col / P.ny, j = col % P.ny;
    const GhostShape g = ghost_shape(comp, P.nx, P.ny, P.nz);
    double *base = comp == 0 ? lu : (comp == 1 ? lv : lw);
    double *x = base + (size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z + 1;
    const int which = comp == 2 ? 1 : 0;
    const int n = which == 0 ? P.nz : P.nz - 1;
    const double alpha = 1.0 * dt * P.nu;
    auto rows = [&](int k, double &a, double &b, double &c) {
        double dl, dr, dc;
        if (which == 0) {
            dl = dz_c[k];
            dr = dz_c[k + 1];
            dc = dz_f[k];
        } else {
            dl = dz_f[k];
            dr = dz_f[k + 1];
            dc = dz_c[k + 1];
        }
        const double lower = -alpha / (dl * dc);
        const double center = 1.0 + alpha * (1.0 / dl + 1.0 / dr) / dc;
        const double upper = -alpha / (dr * dc);
        a = lower;
        b = center;
        c = upper;
        if (k == 0) {
            a = 0.0;
            if (which == 0) b = center - lower;
        }
        if (k == n - 1) {
            c = 0.0;
            if (which == 0) b = P.top_neumann ? center + upper : center - upper;
        }
    };
    double cprev = 0.0, dprev = 0.0;
    for (int k = 0; k < n; ++k) {
        double a, b, c, a2, b2, c2;
        rows(k, a, b, c);
        double sub = 0.0, sup = 0.0;
        if (k > 0) {
            rows(k - 1, a2, b2, c2);
            sub = c2;
        }
        if (k < n - 1) {
            rows(k + 1, a2, b2, c2);
            sup = a2;
        }
        const double id = 1.0 / (b - sub * cprev);
        cprev = sup * id;
        dprev = (x[k] - sub * dprev) * id;
        x[k] = dprev;
        scratch[(size_t)k * 3 * ncol + t] = cprev;
    }
    double y = 0.0;
    for (int k = n - 1; k >= 0; --k) {
        y = (k == n - 1) ? x[k] : x[k] - scratch[(size_t)k * 3 * ncol + t] * y;
        x[k] = y;
    }
}

__global__ void k_axpy(double *y, const double *__restrict__ x, double a, long long n)
{
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x)
        y[p] += a * x[p];
}

}  // namespace

// ---- host side -------------------------------------------------------------------

struct AdjWS {
    long long n_c[3] = {0, 0, 0}, ntot = 0, nkeys_max = 0, nrec_max = 0;
    double4 *rec_near = nullptr, *rec_far = nullptr, *pay = nullptr;
    TriRec *tri = nullptr;
    int *keys = nullptr, *order = nullptr, *counts = nullptr, *starts = nullptr, *fill = nullptr;
    int *sums = nullptr, *total = nullptr;
    double *lam_mid[3] = {nullptr, nullptr, nullptr};
    double *scratch = nullptr, *partials = nullptr, *S = nullptr;
    double *W = nullptr;  // sorted gather weights, 3 O arrays of n_c[0]
    int *kz = nullptr;    // sorted gather records' first z node
    double *Stri = nullptr;  // trilinear corner partials, 8 arrays of nkeys_max
};

namespace {

#define ADJ_CK(call, what)                                                                     \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            g->err = std::string(what) + ": " + cudaGetErrorString(e_);                        \
            return SLC_E_CUDA;                                                                 \
        }                                                                                      \
    } while (0)

template <typename T>
int adj_alloc(slc_grid *g, T **p, size_t n, const char *what)
{
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T) > 0 ? n * sizeof(T) : 16);
    if (e != cudaSuccess) {
        g->err = std::string("cudaMalloc ") + what + ": " + cudaGetErrorString(e);
        return SLC_E_NOMEM;
    }
    g->allocs.push_back(q);
    *p = (T *)q;
    return SLC_OK;
}

int ensure_adj(slc_grid *g)
{
    if (g->adj) return SLC_OK;
    const SlcParams &P = g->P;
    AdjWS *w = new AdjWS();
    const long long plane = (long long)P.nx * P.ny;
    w->n_c[0] = w->n_c[1] = plane * P.nz;
    w->n_c[2] = plane * (P.nz - 1);
    w->ntot = w->n_c[0] + w->n_c[1] + w->n_c[2];
    const long long slots = 2LL * P.n_iters - 1;
    w->nkeys_max = plane * (P.nz + 2);
    w->nrec_max = slots * w->ntot;
    const long long nb = (w->nkeys_max + 1 + kScanT - 1) / kScanT;
    int rc = adj_alloc(g, &w->rec_near, (size_t)w->n_c[0], "adjoint near records");
    if (!rc) rc = adj_alloc(g, &w->rec_far, (size_t)w->n_c[0], "adjoint far records");
    if (!rc) rc = adj_alloc(g, &w->tri, (size_t)w->nrec_max, "adjoint trajectory records");
    if (!rc) rc = adj_alloc(g, &w->pay, (size_t)w->nrec_max, "adjoint payload");
    if (!rc) rc = adj_alloc(g, &w->keys, (size_t)w->nrec_max, "adjoint keys");
    if (!rc) rc = adj_alloc(g, &w->order, (size_t)w->nrec_max, "adjoint order");
    if (!rc) rc = adj_alloc(g, &w->counts, (size_t)w->nkeys_max + 1, "adjoint counts");
    if (!rc) rc = adj_alloc(g, &w->starts, (size_t)w->nkeys_max + 1, "adjoint starts");
    if (!rc) rc = adj_alloc(g, &w->fill, (size_t)w->nkeys_max + 1, "adjoint fill");
    if (!rc) rc = adj_alloc(g, &w->sums, (size_t)nb, "adjoint scan sums");
    if (!rc) rc = adj_alloc(g, &w->total, (size_t)1, "adjoint scan total");
    for (int c = 0; c < 3 && !rc; ++c) rc = adj_alloc(g, &w->lam_mid[c], g->ghost_elems[c], "adjoint U*");
    if (!rc) rc = adj_alloc(g, &w->scratch, (size_t)3 * plane * P.nz, "adjoint z-solve scratch");
    if (!rc) rc = adj_alloc(g, &w->partials, (size_t)kSumBlocks, "adjoint partials");
    if (!rc) rc = adj_alloc(g, &w->S, (size_t)1, "adjoint sum");
    if (!rc) rc = adj_alloc(g, &w->W, (size_t)3 * SLC_MAX_ORDER * w->n_c[0], "adjoint gather weights");
    if (!rc) rc = adj_alloc(g, &w->kz, (size_t)w->n_c[0], "adjoint gather z bases");
    if (!rc) rc = adj_alloc(g, &w->Stri, (size_t)8 * w->nkeys_max, "adjoint trilinear partials");
    if (rc) {
        delete w;
        return rc;
    }
    g->adj = w;
    return SLC_OK;
}

// Counting sort of w->keys[0, n) over nkeys keys into w->order / w->starts.
int sort_records(slc_grid *g, AdjWS *w, long long n, long long nkeys, cudaStream_t s)
{
    k_izero<<<nblk(nkeys + 1), kT, 0, s>>>(w->counts, nkeys + 1);
    k_izero<<<nblk(nkeys + 1), kT, 0, s>>>(w->fill, nkeys + 1);
    if (n > 0) k_count<<<nblk(n), kT, 0, s>>>(w->keys, n, w->counts);
    const long long m = nkeys + 1;
    const int nb = (int)((m + kScanT - 1) / kScanT);
    k_scan_blocks<<<nb, kScanT, 0, s>>>(w->counts, w->starts, w->sums, m);
    k_scan_sums<<<1, kScanT, 0, s>>>(w->sums, nb, w->total);
    k_scan_add<<<nb, kScanT, 0, s>>>(w->starts, w->sums, m);
    if (n > 0) k_place<<<nblk(n), kT, 0, s>>>(w->keys, n, w->starts, w->fill, w->order);
    k_sort_segments<<<nblk(nkeys), kT, 0, s>>>(w->starts, nkeys, w->order);
    count_launches(n > 0 ? 9 : 7);
    ADJ_CK(cudaGetLastError(), "adjoint record sort");
    return SLC_OK;
}

template <int O, int MODE>
int sl_adjoint_t(slc_grid *g, AdjWS *w, const V3 &M, const double *const cur[3],
                 const double *const prev[3], double *const lam_hat[3], double *const lam_cur[3],
                 double *const lam_prev[3], double dt, cudaStream_t s)
{
    const SlcParams &P = g->P;
    long long pbase[3] = {0, w->n_c[0], w->n_c[0] + w->n_c[1]};
    const double *fnm1[3] = {prev ? prev[0] : nullptr, prev ? prev[1] : nullptr, prev ? prev[2] : nullptr};
    for (int C = 0; C < 3; ++C) {
        const long long n = w->n_c[C];
        if (n <= 0) continue;
        // points -> records
        if (C == 0)
            k_sl_adj_points<0, O, MODE><<<nblk(n), kT, 0, s>>>(P, M, cur[0], fnm1[0], lam_hat[0], dt,
                                                               w->rec_near, w->rec_far, w->tri, pbase[0], w->ntot);
        else if (C == 1)
            k_sl_adj_points<1, O, MODE><<<nblk(n), kT, 0, s>>>(P, M, cur[1], fnm1[1], lam_hat[1], dt,
                                                               w->rec_near, w->rec_far, w->tri, pbase[1], w->ntot);
        else
            k_sl_adj_points<2, O, MODE><<<nblk(n), kT, 0, s>>>(P, M, cur[2], fnm1[2], lam_hat[2], dt,
                                                               w->rec_near, w->rec_far, w->tri, pbase[2], w->ntot);
        count_launches(1);
        const int NZ = C < 2 ? P.nz + 2 : P.nz + 1;
        const long long nkeys = (long long)P.nx * P.ny * NZ;
        // near foot -> lam_cur[C]; far foot -> lam_prev[C]
        for (int foot = 0; foot < (MODE == 2 ? 2 : 1); ++foot) {
            const double4 *rec = foot == 0 ? w->rec_near : w->rec_far;
            double *dst = foot == 0 ? lam_cur[C] : lam_prev[C];
            if (C == 0) k_gather_keys<0, O><<<nblk(n), kT, 0, s>>>(P, rec, n, w->keys);
            else if (C == 1) k_gather_keys<1, O><<<nblk(n), kT, 0, s>>>(P, rec, n, w->keys);
            else k_gather_keys<2, O><<<nblk(n), kT, 0, s>>>(P, rec, n, w->keys);
            count_launches(1);
            int rc = sort_records(g, w, n, nkeys, s);
            if (rc) return rc;
            if (C == 0) {
                k_sorted_weights<0, O><<<nblk(n), kT, 0, s>>>(P, rec, w->order, n, w->W, w->kz);
                k_pull_gather<0, O><<<nblk(nkeys), kT, 0, s>>>(P, w->W, w->kz, n, w->starts, dst);
            } else if (C == 1) {
                k_sorted_weights<1, O><<<nblk(n), kT, 0, s>>>(P, rec, w->order, n, w->W, w->kz);
                k_pull_gather<1, O><<<nblk(nkeys), kT, 0, s>>>(P, w->W, w->kz, n, w->starts, dst);
            } else {
                k_sorted_weights<2, O><<<nblk(n), kT, 0, s>>>(P, rec, w->order, n, w->W, w->kz);
                k_pull_gather<2, O><<<nblk(nkeys), kT, 0, s>>>(P, w->W, w->kz, n, w->starts, dst);
            }
            count_launches(2);
        }
        // explicit x, y diffusion
        const double cc = MODE == 2 ? (P.xy_lagged ? (2.0 / 3.0) * dt : (4.0 / 3.0) * dt) : dt;
        const double cpv = MODE == 2 && !P.xy_lagged ? -(2.0 / 3.0) * dt : 0.0;
        double *lp = (MODE == 2 && !P.xy_lagged) ? lam_prev[C] : nullptr;
        if (C == 0) k_diff_adj<0><<<nblk(n), kT, 0, s>>>(P, lam_hat[0], lam_cur[0], cc, lp, cpv);
        else if (C == 1) k_diff_adj<1><<<nblk(n), kT, 0, s>>>(P, lam_hat[1], lam_cur[1], cc, lp, cpv);
        else k_diff_adj<2><<<nblk(n), kT, 0, s>>>(P, lam_hat[2], lam_cur[2], cc, lp, cpv);
        count_launches(1);
    }
    // trajectory records -> lam_U* per field
    const long long nrec = (long long)(MODE == 2 ? 2 * P.n_iters - 1 : P.n_iters) * w->ntot;
    for (int c = 0; c < 3; ++c) {
        ADJ_CK(cudaMemsetAsync(w->lam_mid[c], 0, g->ghost_elems[c] * sizeof(double), s), "memset");
        k_tri_keys<<<nblk(nrec), kT, 0, s>>>(P, c, w->tri, nrec, w->keys, w->pay);
        count_launches(1);
        const int NZ = c < 2 ? P.nz + 2 : P.nz + 1;
        const long long nkeys = (long long)P.nx * P.ny * NZ;
        int rc = sort_records(g, w, nrec, nkeys, s);
        if (rc) return rc;
        k_tri_segsum<<<nblk(nkeys), kT, 0, s>>>(w->pay, w->order, w->starts, nkeys, w->Stri);
        k_pull_tri<<<nblk(nkeys), kT, 0, s>>>(P, c, w->Stri, w->lam_mid[c]);
        count_launches(2);
        // U* = 2 V^n - V^{n-1} (BDF2) or V^n (BDF1)
        const long long ne = (long long)g->ghost_elems[c];
        k_axpy<<<148 * 8, kT, 0, s>>>(lam_cur[c], w->lam_mid[c], MODE == 2 ? 2.0 : 1.0, ne);
        if (MODE == 2) k_axpy<<<148 * 8, kT, 0, s>>>(lam_prev[c], w->lam_mid[c], -1.0, ne);
        count_launches(MODE == 2 ? 2 : 1);
    }
    ADJ_CK(cudaGetLastError(), "SL adjoint");
    return SLC_OK;
}

int bc_adjoint(slc_grid *g, double *const lam[3], cudaStream_t s)
{
    const SlcParams &P = g->P;
    const long long plane = (long long)P.nx * P.ny;
    k_bc_adj<0><<<nblk(plane * P.nz), kT, 0, s>>>(P, lam[0]);
    k_bc_adj<1><<<nblk(plane * P.nz), kT, 0, s>>>(P, lam[1]);
    if (P.nz > 1) k_bc_adj<2><<<nblk(plane * (P.nz - 1)), kT, 0, s>>>(P, lam[2]);
    k_zero_ghosts<0><<<148 * 4, kT, 0, s>>>(P, lam[0]);
    k_zero_ghosts<1><<<148 * 4, kT, 0, s>>>(P, lam[1]);
    k_zero_ghosts<2><<<148 * 4, kT, 0, s>>>(P, lam[2]);
    count_launches(6);
    ADJ_CK(cudaGetLastError(), "ghost refresh adjoint");
    return SLC_OK;
}

}  // namespace

void adj_free(AdjWS *w) { delete w; }

extern "C" {

int slc_adjoint_bc(slc_grid *g, double *lam_u, double *lam_v, double *lam_w, void *stream)
{
    if (!g) return SLC_E_INVALID;
    if (!lam_u || !lam_v || !lam_w) {
        g->err = "null pointer";
        return SLC_E_INVALID;
    }
    cudaSetDevice(g->device);
    double *lam[3] = {lam_u, lam_v, lam_w};
    return bc_adjoint(g, lam, (cudaStream_t)stream);
}

int slc_adjoint_step(slc_grid *g, int mode, double *const cur[3], double *const prev[3],
                     double *const lam_next[3], double *const lam_cur[3], double *const lam_prev[3],
                     double dt, void *stream)
{
    if (!g) return SLC_E_INVALID;
    if (mode != 1 && mode != 2) {
        g->err = "mode must be 1 (BDF1 bootstrap) or 2 (BDF2)";
        return SLC_E_INVALID;
    }
    if (g->mixed) {
        g->err = "the adjoint is implemented for the FP64 form";
        return SLC_E_INVALID;
    }
    if (!cur || !lam_next || !lam_cur || (mode == 2 && (!prev || !lam_prev))) {
        g->err = "null pointer";
        return SLC_E_INVALID;
    }
    for (int c = 0; c < 3; ++c)
        if (!cur[c] || !lam_next[c] || !lam_cur[c] || (mode == 2 && (!prev[c] || !lam_prev[c]))) {
            g->err = "null field pointer";
            return SLC_E_INVALID;
        }
    if (!(dt > 0.0)) {
        g->err = "dt must be positive";
        return SLC_E_INVALID;
    }
    if (g->P.traj_order != 2) {
        g->err = "the adjoint supports the trilinear trajectory (traj_interp_order 2)";
        return SLC_E_INVALID;
    }
    if (g->P.n_iters < 1 || g->P.n_iters > kMaxIters) {
        g->err = "the adjoint supports 1 to 4 trajectory iterations";
        return SLC_E_INVALID;
    }
    if (g->P.nz < 2) {
        g->err = "the adjoint needs nz >= 2";
        return SLC_E_INVALID;
    }
    cudaSetDevice(g->device);
    cudaStream_t s = (cudaStream_t)stream;
    int rc = ensure_adj(g);
    if (rc) return rc;
    AdjWS *w = g->adj;
    const SlcParams &P = g->P;
    const double dt_eff = mode == 2 ? (2.0 / 3.0) * dt : dt;
    const long long plane = (long long)P.nx * P.ny;
    const long long n = plane * P.nz;

    // 1. ghost refresh after the bulk shift, then the shift itself (u only)
    rc = bc_adjoint(g, lam_next, s);
    if (rc) return rc;
    k_sum_partials<<<kSumBlocks, kT, 0, s>>>(P, lam_next[0], w->partials);
    k_sum_finish<<<1, kT, 0, s>>>(w->partials, kSumBlocks, w->S);
    k_bulk_adj_apply<<<nblk(n), kT, 0, s>>>(P, lam_next[0], g->dzf, w->S,
                                            (P.dx * P.dy) / (g->Lx * g->Ly * P.Lz));
    count_launches(3);
    // 2. projection: lam -= D^T L^-T G^T lam  (dt_div = dt_proj)
    k_gradT_pack<<<nblk(n), kT, 0, s>>>(P, lam_next[0], lam_next[1], lam_next[2], g->dzc, g->rhs);
    count_launches(1);
    if (cufftSetStream(g->fwd, s) != CUFFT_SUCCESS ||
        cufftExecD2Z(g->fwd, g->rhs, (cufftDoubleComplex *)g->hat) != CUFFT_SUCCESS) {
        g->err = "cufftExecD2Z (adjoint)";
        return SLC_E_CUFFT;
    }
    {
        const long long nthr = 2LL * P.nx * (P.ny / 2 + 1);
        const double norm = 1.0 / ((double)P.nx * (double)P.ny);
        k_thomas_T<<<nblk(nthr), kT, 0, s>>>(P, g->hat, g->cpw, g->kx2, g->ky2, g->cl, g->cr, norm);
        count_launches(1);
    }
    if (cufftSetStream(g->inv, s) != CUFFT_SUCCESS ||
        cufftExecZ2D(g->inv, (cufftDoubleComplex *)g->hat, g->rhs) != CUFFT_SUCCESS) {
        g->err = "cufftExecZ2D (adjoint)";
        return SLC_E_CUFFT;
    }
    k_divT<<<nblk(n), kT, 0, s>>>(P, g->rhs, g->dzf, 1.0, lam_next[0], lam_next[1], lam_next[2]);
    count_launches(1);
    // 3. z-solve
    k_zsolve_T<<<nblk(3 * plane), kT, 0, s>>>(P, g->dzc, g->dzf, dt_eff, lam_next[0], lam_next[1],
                                               lam_next[2], w->scratch);
    count_launches(1);
    ADJ_CK(cudaGetLastError(), "projection / z-solve adjoint");
    // 4. SL predictor: U* recomputed
    V3 M;
    if (mode == 2) {
        for (int c = 0; c < 3; ++c)
            if (!g->mid[c]) {
                void *q = nullptr;
                ADJ_CK(cudaMalloc(&q, g->ghost_elems[c] * sizeof(double)), "U* workspace");
                g->allocs.push_back(q);
                g->mid[c] = (double *)q;
            }
        for (int c = 0; c < 3; ++c)
            ADJ_CK(launch_lincomb(cur[c], prev[c], 2.0, -1.0, g->mid[c], (int64_t)g->ghost_elems[c], s),
                   "U*");
        M.u = ghost_view<double>(0, g->mid[0], P.nx, P.ny, P.nz);
        M.v = ghost_view<double>(1, g->mid[1], P.nx, P.ny, P.nz);
        M.w = ghost_view<double>(2, g->mid[2], P.nx, P.ny, P.nz);
    } else {
        M.u = ghost_view<double>(0, cur[0], P.nx, P.ny, P.nz);
        M.v = ghost_view<double>(1, cur[1], P.nx, P.ny, P.nz);
        M.w = ghost_view<double>(2, cur[2], P.nx, P.ny, P.nz);
    }
    const double *cc[3] = {cur[0], cur[1], cur[2]};
    const double *pp[3] = {prev ? prev[0] : nullptr, prev ? prev[1] : nullptr, prev ? prev[2] : nullptr};
    if (P.order == 4)
        rc = mode == 2 ? sl_adjoint_t<4, 2>(g, w, M, cc, pp, lam_next, lam_cur, lam_prev, dt, s)
                       : sl_adjoint_t<4, 1>(g, w, M, cc, pp, lam_next, lam_cur, lam_prev, dt, s);
    else
        rc = mode == 2 ? sl_adjoint_t<6, 2>(g, w, M, cc, pp, lam_next, lam_cur, lam_prev, dt, s)
                       : sl_adjoint_t<6, 1>(g, w, M, cc, pp, lam_next, lam_cur, lam_prev, dt, s);
    return rc;
}

}  // extern "C"
