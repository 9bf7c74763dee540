// sl_device.cuh -- device pieces of the FP64 trace+gather shared by the
// single-grid, ensemble and shared-memory-staged kernels.  Included inside
// each translation unit's anonymous namespace.
#pragma once

struct Vel3 {
    NodeView<double> u, v, w;
};

__device__ __forceinline__ void add_clamps(unsigned long long *counter, unsigned cnt)
{
    unsigned tot = __reduce_add_sync(0xffffffffu, cnt);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(counter, (unsigned long long)tot);
}

// Trajectory velocity at one point (semilag.py:512-528, traj_order = 2):
// z clamped to [z_lo, z_hi], one face-locate shared by the three samples.
__device__ __forceinline__ void sample3(const SlcParams &P, const Vel3 &M, double x, double y,
                                        double z, double &us, double &vs, double &ws)
{
    const double zc = clampz(P, z);
    TriShared t;
    tri_shared(P, x, y, zc, face_cell(P, zc), t);
    us = tri_sample(M.u, t.ia0, t.ia1, t.txa, t.jb0, t.jb1, t.tyb, t.kc, t.wc0, t.wc1);
    vs = tri_sample(M.v, t.ib0, t.ib1, t.txb, t.ja0, t.ja1, t.tya, t.kc, t.wc0, t.wc1);
    ws = tri_sample(M.w, t.ib0, t.ib1, t.txb, t.jb0, t.jb1, t.tyb, t.kf, t.wf0, t.wf1);
}

// The same with tricubic Lagrange sampling (traj_interp_order 4,
// semilag.py:206-209, 512-528): the order-4 tensor-product stencils of the
// field gather on the three trajectory components.  Kept out of line so the
// trilinear path's register allocation does not carry it.
__device__ __noinline__ void sample3_o4(const SlcParams &P, const Vel3 &M, double x, double y,
                                        double z, double &us, double &vs, double &ws)
{
    const double zc = clampz(P, z);
    const int c = face_cell(P, zc);
    Stencil<4, double> st;
    build_stencil<0, 4, double>(P, M.u.sx, M.u.sy, x, y, zc, c, st);
    us = gather_sum<4, double, double>(M.u.p, st);
    build_stencil<1, 4, double>(P, M.v.sx, M.v.sy, x, y, zc, c, st);
    vs = gather_sum<4, double, double>(M.v.p, st);
    build_stencil<2, 4, double>(P, M.w.sx, M.w.sy, x, y, zc, c, st);
    ws = gather_sum<4, double, double>(M.w.p, st);
}

// Trajectory sampling order as a template argument: 2 or 4 fixed at compile
// time, 0 read from P.traj_order at run time.
template <int TO>
__device__ __forceinline__ bool traj4(const SlcParams &P)
{
    return TO == 4 || (TO == 0 && P.traj_order == 4);
}

// First fixed-point sample at the arrival point (i, j, k) of component C:
// exact node values for trilinear sampling, the stencils for tricubic.
template <int C, int TO = 0>
__device__ __forceinline__ void first_sample(const SlcParams &P, const Vel3 &M, int i, int j, int k,
                                             double xa, double ya, double za, double &us0,
                                             double &vs0, double &ws0)
{
    if (traj4<TO>(P)) sample3_o4(P, M, xa, ya, za, us0, vs0, ws0);
    else arrival_sample<C>(P, M, i, j, k, NodeValF64(), us0, vs0, ws0);
}

// Iterated midpoint rule continued from the first-iteration sample
// (us0, vs0, ws0) taken at the arrival point; returns the unclamped foot.
template <int TO = 0>
__device__ __forceinline__ void trace_foot(const SlcParams &P, const Vel3 &M, double xa, double ya,
                                           double za, double half_dt, double us0, double vs0,
                                           double ws0, double &xd, double &yd, double &zd)
{
    double xm = xa - half_dt * us0;
    double ym = ya - half_dt * vs0;
    double zm = clampz(P, za - half_dt * ws0);
    for (int it = 1; it < P.n_iters; ++it) {
        double us, vs, ws;
        if (traj4<TO>(P)) sample3_o4(P, M, xm, ym, zm, us, vs, ws);
        else sample3(P, M, xm, ym, zm, us, vs, ws);
        xm = xa - half_dt * us;
        ym = ya - half_dt * vs;
        zm = clampz(P, za - half_dt * ws);
    }
    xd = 2.0 * xm - xa;
    yd = 2.0 * ym - ya;
    zd = 2.0 * zm - za;
}

// Clamp-and-count the foot (semilag.py:472-474) and interpolate F there.
template <int C, int O>
__device__ __forceinline__ double gather_foot(const SlcParams &P, NodeView<double> F, double xd,
                                              double yd, double zd, unsigned &ncl)
{
    if (zd < P.z_lo || zd > P.z_hi) ncl += 1;
    double z = clampz(P, zd);
    int c = face_cell(P, z);
    Stencil<O, double> st;
    build_stencil<C, O, double>(P, F.sx, F.sy, xd, yd, z, c, st);
    return gather_sum<O, double, double>(F.p, st);
}

// nu (d2/dx2 + d2/dy2) f at interior point (i, j, k) of component C, with the
// reference's periodic extensions u[nx+1] = u[1] and v[:, ny+1] = v[:, 1]
// (operators.py:301-306, 329-333).
template <int C>
__device__ __forceinline__ double xy_diffusion(const SlcParams &P, const double *__restrict__ f,
                                               int i, int j, int k)
{
    GhostShape g = ghost_shape(C, P.nx, P.ny, P.nz);
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

