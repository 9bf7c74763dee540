// poisson.cu -- ghost-cell boundary conditions, divergence, the FFT-Poisson
// tridiagonal sweep, the projection and the bulk-flux reductions (sm_100a).
//
// Layout of the Poisson workspaces: the right-hand side and phi are z-major
// planes rhs[k][i][j] (j fastest), so cuFFT transforms nz contiguous (nx, ny)
// planes and every (kx, ky) column of the half spectrum hat[k][kx][ky] is
// walked by one thread with coalesced accesses across the warp.  The
// divergence and projection kernels transpose between that layout and the
// z-contiguous velocity arrays through a 32 x 32 shared-memory tile.
#include "slc_bc.cuh"
#include "slc_internal.h"

namespace {

// --------------------------------------------------------------------------
// Boundary conditions (solver.py:70-107; projection.py:180-195 for p).
// Every ghost element is a copy (or a negated copy) of one interior element,
// so each is gathered independently from its source.
// --------------------------------------------------------------------------

struct BcCounts {
    long long a, b, c;  // x-ghost planes, y-ghost planes (x interior), z-ghost planes
};

__host__ __device__ inline BcCounts bc_counts(int C, int nx, int ny, int nz)
{
    GhostShape g = ghost_shape(C, nx, ny, nz);
    BcCounts r;
    r.a = (long long)n_xghost(C) * g.Y * g.Z;
    r.b = (long long)nx * n_yghost(C) * g.Z;
    r.c = (long long)nx * ny * 2;
    return r;
}

__device__ inline void bc_one(const SlcParams &P, int C, double *f, long long t)
{
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const GhostShape g = ghost_shape(C, nx, ny, nz);
    const BcCounts cnt = bc_counts(C, nx, ny, nz);
    int I, J, K;
    if (t < cnt.a) {
        K = (int)(t % g.Z);
        long long q = t / g.Z;
        J = (int)(q % g.Y);
        const int which = (int)(q / g.Y);
        I = which == 0 ? 0 : nx + 1;
    } else if (t < cnt.a + cnt.b) {
        t -= cnt.a;
        K = (int)(t % g.Z);
        long long q = t / g.Z;
        const int which = (int)(q % n_yghost(C));
        I = (int)(q / n_yghost(C)) + 1;
        J = which == 0 ? 0 : ny + 1;
    } else {
        t -= cnt.a + cnt.b;
        const int which = (int)(t & 1);
        long long q = t >> 1;
        J = (int)(q % ny) + 1;
        I = (int)(q / ny) + 1;
        K = which == 0 ? 0 : g.Z - 1;
    }
    const BcSrc r = bc_src(C, nx, ny, nz, P.top_neumann, I, J, K);
    const double val = r.zero ? 0.0 : r.sign * f[(size_t)r.Is * g.Y * g.Z + (size_t)r.Js * g.Z + r.Ks];
    f[(size_t)I * g.Y * g.Z + (size_t)J * g.Z + K] = val;
}

__global__ void k_apply_bc(SlcParams P, double *u, double *v, double *w, double *p, long long n0,
                           long long n1, long long n2, long long n3)
{
    const long long total = n0 + n1 + n2 + n3;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        if (t < n0) bc_one(P, 0, u, t);
        else if (t < n0 + n1) bc_one(P, 1, v, t - n0);
        else if (t < n0 + n1 + n2) bc_one(P, 2, w, t - n0 - n1);
        else bc_one(P, 3, p, t - n0 - n1 - n2);
    }
}

// --------------------------------------------------------------------------
// Divergence (utils.py:166-180).  The x-1 / y-1 neighbours use the periodic
// image directly, so the field's ghosts need not be current.
// --------------------------------------------------------------------------

__device__ __forceinline__ double div_at(const SlcParams &P, const double *__restrict__ u,
                                         const double *__restrict__ v,
                                         const double *__restrict__ w,
                                         const double *__restrict__ dz_f, int i, int j, int k)
{
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    const size_t vsx = (size_t)(ny + 1) * (nz + 2), vsy = nz + 2;
    const size_t wsx = (size_t)(ny + 2) * (nz + 1), wsy = nz + 1;
    const int im = i == 0 ? nx : i;  // u row i (0-based interior i-1) ; ghost row 0 == row nx
    const int jm = j == 0 ? ny : j;
    const double du = (u[(i + 1) * usx + (j + 1) * usy + k + 1] - u[im * usx + (j + 1) * usy + k + 1]) * P.inv_dx;
    const double dv = (v[(i + 1) * vsx + (j + 1) * vsy + k + 1] - v[(i + 1) * vsx + jm * vsy + k + 1]) * P.inv_dy;
    const double dw = (w[(i + 1) * wsx + (j + 1) * wsy + k + 1] - w[(i + 1) * wsx + (j + 1) * wsy + k]) / dz_f[k];
    return du + dv + dw;
}

// rhs[k][i][j] = div(i, j, k) / dt_div, through a shared-memory transpose.
__device__ __forceinline__ void div_pack_tile(const SlcParams &P, const double *__restrict__ u,
                                              const double *__restrict__ v,
                                              const double *__restrict__ w,
                                              const double *__restrict__ dz_f, double dt_div,
                                              double *__restrict__ rhs, int bx, int by, int bz)
{
    __shared__ double tile[32][33];
    const int i = bz, j0 = by * 32, k0 = bx * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // block (32, 8): rows ty + 8q
    double val[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {  // all four rows' loads in flight together
        const int j = j0 + ty + 8 * q, k = k0 + tx;
        val[q] = (j < P.ny && k < P.nz) ? div_at(P, u, v, w, dz_f, i, j, k) / dt_div : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) tile[ty + 8 * q][tx] = val[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int r = ty + 8 * q;
        const int k = k0 + r, j = j0 + tx;
        if (k < P.nz && j < P.ny) rhs[((size_t)k * P.nx + i) * P.ny + j] = tile[tx][r];
    }
}

__global__ void __launch_bounds__(256) k_div_pack(SlcParams P, const double *__restrict__ u,
                                                  const double *__restrict__ v,
                                                  const double *__restrict__ w,
                                                  const double *__restrict__ dz_f, double dt_div,
                                                  double *__restrict__ rhs)
{
    div_pack_tile(P, u, v, w, dz_f, dt_div, rhs, blockIdx.x, blockIdx.y, blockIdx.z);
}

__global__ void k_divergence(SlcParams P, const double *__restrict__ u,
                             const double *__restrict__ v, const double *__restrict__ w,
                             const double *__restrict__ dz_f, double *__restrict__ div)
{
    const long long n = (long long)P.nx * P.ny * P.nz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % P.nz);
        const long long q = t / P.nz;
        const int j = (int)(q % P.ny), i = (int)(q / P.ny);
        div[t] = div_at(P, u, v, w, dz_f, i, j, k);
    }
}

// --------------------------------------------------------------------------
// Thomas sweep per (kx, ky) column of the half spectrum (projection.py:199-247)
// with the modified-wavenumber diagonals (projection.py:47-114) built on the
// fly; the (0, 0) mode's first row is the identity (projection.py:113-114).
// The inverse-FFT normalisation 1/(nx ny) is folded into the back
// substitution.
// --------------------------------------------------------------------------

constexpr int kPre = 8;  // loads kept in flight per thread in the sweeps

// Row k of the (kx, ky) column's system: sub-diagonal a, diagonal b,
// super-diagonal c (projection.py:47-114), Neumann rows folded into b; the
// (0, 0) mode's first row is the identity (projection.py:113-114).
struct Row3 {
    double a, b, c;
};

__device__ __forceinline__ Row3 poisson_row(const double *__restrict__ cl,
                                            const double *__restrict__ cr, double k2, int nz, int k,
                                            bool pinned)
{
    Row3 r;
    r.a = k > 0 ? cl[k] : 0.0;
    r.b = -(cl[k] + cr[k] + k2);
    if (k == 0) r.b += cl[0];
    if (k == nz - 1) r.b += cr[nz - 1];
    r.c = k < nz - 1 ? cr[k] : 0.0;
    if (pinned && k == 0) {
        r.b = 1.0;
        r.c = 0.0;
    }
    return r;
}

// Twisted (two-ended) Thomas elimination: four threads per column, part (re /
// im) x half.  Half 0 eliminates rows 0 .. m-1 downwards as the reference's
// Thomas sweep does; half 1 eliminates rows nz-1 .. m+1 upwards (sub- and
// super-diagonal exchanged); the two meet at row m = nz/2, which the adjacent
// lanes solve from each other's last pivot row (one shuffle), then each back-
// substitutes its half.  Twice the threads of a one-ended sweep in flight for
// the same arithmetic; the meeting row changes results by rounding only.  The
// coefficients are real, so the real and imaginary parts are independent
// systems; the part-0 thread of each half stores the pivot ratios g (same
// values for both parts), read back by both after a warp barrier.
__device__ __forceinline__ void thomas_column(const SlcParams &P, double *__restrict__ hat,
                                              double *__restrict__ cpw,
                                              const double *__restrict__ kx2,
                                              const double *__restrict__ ky2,
                                              const double *__restrict__ cl,
                                              const double *__restrict__ cr, double norm, int t)
{
    const int nky = P.ny / 2 + 1;
    const int ncol = P.nx * nky;
    const int col = t >> 2, part = (t >> 1) & 1, half = t & 1;
    const bool active = col < ncol;
    const int nz = P.nz, m = nz / 2;
    const size_t st = 2 * (size_t)ncol;  // doubles per k-plane of the spectrum
    double *h = hat + 2 * (size_t)(active ? col : 0) + part;
    double *cpc = cpw + (active ? col : 0);
    double k2 = 0.0;
    if (active) {
        const int kx = col / nky, ky = col - (col / nky) * nky;
        k2 = kx2[kx] + ky2[ky];
    }
    const bool pinned = active && col == 0;
    const int cnt = active ? (half ? nz - 1 - m : m) : 0;  // rows this thread eliminates
    // row of elimination step q: downwards from 0, or upwards from nz-1
#define TH_ROW(q) (half ? nz - 1 - (q) : (q))
    double buf[kPre];
#pragma unroll
    for (int q = 0; q < kPre; ++q) buf[q] = q < cnt ? h[TH_ROW(q) * st] : 0.0;
    double gprev = 0.0, dprev = 0.0;
    for (int q0 = 0; q0 < cnt; q0 += kPre) {
#pragma unroll
        for (int u = 0; u < kPre; ++u) {
            const int q = q0 + u;
            if (q < cnt) {
                const int k = TH_ROW(q);
                const double d = buf[u];
                if (q + kPre < cnt) buf[u] = h[TH_ROW(q + kPre) * st];
                const Row3 R = poisson_row(cl, cr, k2, nz, k, pinned);
                const double e = half ? R.c : R.a, f = half ? R.a : R.c;
                const double id = 1.0 / (R.b - e * gprev);
                gprev = f * id;
                dprev = (d - e * dprev) * id;
                h[k * st] = dprev;
                if (part == 0) cpc[k * (size_t)ncol] = gprev;
            }
        }
    }
#undef TH_ROW
    // the meeting row m from both halves' last pivot rows
    const double og = __shfl_xor_sync(0xffffffffu, gprev, 1);
    const double od = __shfl_xor_sync(0xffffffffu, dprev, 1);
    __syncwarp();  // the pivot ratios stored above are visible to the whole warp
    const double gt = half ? og : gprev, dtp = half ? od : dprev;  // row m-1 (top)
    const double gb = half ? gprev : og, dbt = half ? dprev : od;  // row m+1 (bottom)
    const Row3 R = poisson_row(cl, cr, k2, nz, m, pinned);
    const double dm = active ? h[m * st] : 0.0;
    const double xm = (dm - R.a * dtp - R.c * dbt) / (R.b - R.a * gt - R.c * gb);
    // back substitution outwards from m, prefetching d and g
    double cb[kPre];
#pragma unroll
    for (int q = 0; q < kPre; ++q) {
        const int k = half ? m + 1 + q : m - 1 - q;
        buf[q] = q < cnt ? h[k * st] : 0.0;
        cb[q] = q < cnt ? cpc[k * (size_t)ncol] : 0.0;
    }
    __syncwarp();  // every lane has read row m before the top half writes it
    if (active && half == 0) h[m * st] = xm * norm;
    double x = xm;
    for (int q0 = 0; q0 < cnt; q0 += kPre) {
#pragma unroll
        for (int u = 0; u < kPre; ++u) {
            const int q = q0 + u;
            if (q < cnt) {
                const int k = half ? m + 1 + q : m - 1 - q;
                const double dk = buf[u], gk = cb[u];
                if (q + kPre < cnt) {
                    const int kn = half ? k + kPre : k - kPre;
                    buf[u] = h[kn * st];
                    cb[u] = cpc[kn * (size_t)ncol];
                }
                x = dk - gk * x;
                h[k * st] = x * norm;
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_thomas(SlcParams P, double *__restrict__ hat,
                                                double *__restrict__ cpw,
                                                const double *__restrict__ kx2,
                                                const double *__restrict__ ky2,
                                                const double *__restrict__ cl,
                                                const double *__restrict__ cr, double norm)
{
    thomas_column(P, hat, cpw, kx2, ky2, cl, cr, norm, blockIdx.x * blockDim.x + threadIdx.x);
}

// --------------------------------------------------------------------------
// Projection (projection.py:250-272): u -= dt dphi/dx, v -= dt dphi/dy,
// w -= dt dphi/dz on the interiors, p interior <- phi.  phi is z-major; a tile
// (i fixed, 33 j x 33 k, plus the x+1 plane) goes through shared memory.
// --------------------------------------------------------------------------

__device__ __forceinline__ void project_tile(const SlcParams &P, const double *__restrict__ phi,
                                             double *__restrict__ u, double *__restrict__ v,
                                             double *__restrict__ w, double *__restrict__ p,
                                             const double *__restrict__ dz_c, double dt, int bx,
                                             int by, int bz)
{
    __shared__ double t0[33][33];  // [k][j], plane i
    __shared__ double t1[32][33];  // [k][j], plane i+1 (periodic)
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int i = bz, j0 = by * 32, k0 = bx * 32;
    const int i1 = (i + 1 == nx) ? 0 : i + 1;
    const int tx = threadIdx.x, ty = threadIdx.y;  // block (32, 8): rows ty + 8q
    // phi rows k0 .. k0+32 (33 with the k+1 halo) of columns j0 .. j0+32
    // (the last one periodic), all loads issued before the tile is written
    {
        double a0[5], a1[5], a2[5];
        const int jc = j0 + tx;                  // column tx
        const int jw = (jc == ny) ? 0 : jc;
        const int jh = (j0 + 32 == ny) ? 0 : j0 + 32;  // column 32 (thread tx 0)
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const int r = ty + 8 * q, k = k0 + r;
            const bool row = r < 33 && k < nz;
            const size_t b0 = ((size_t)k * nx + i) * ny, b1 = ((size_t)k * nx + i1) * ny;
            a0[q] = (row && jc <= ny) ? phi[b0 + jw] : 0.0;
            a1[q] = (row && r < 32 && jc <= ny) ? phi[b1 + jw] : 0.0;
            a2[q] = (row && tx == 0 && j0 + 32 <= ny) ? phi[b0 + jh] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const int r = ty + 8 * q;
            if (r < 33) {
                t0[r][tx] = a0[q];
                if (r < 32) t1[r][tx] = a1[q];
                if (tx == 0) t0[r][32] = a2[q];
            }
        }
    }
    __syncthreads();
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    const size_t vsx = (size_t)(ny + 1) * (nz + 2), vsy = nz + 2;
    const size_t wsx = (size_t)(ny + 2) * (nz + 1), wsy = nz + 1;
    const size_t psx = (size_t)(ny + 2) * (nz + 2), psy = nz + 2;
    // the four rows' velocity loads are issued before any update is stored
    const int k = k0 + tx;
    const size_t I = i + 1, K = k + 1;
    double uo[4], vo[4], wo[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = j0 + ty + 8 * q;
        const bool in = j < ny && k < nz;
        const size_t J = j + 1;
        uo[q] = in ? u[I * usx + J * usy + K] : 0.0;
        vo[q] = in ? v[I * vsx + J * vsy + K] : 0.0;
        wo[q] = (in && k < nz - 1) ? w[I * wsx + J * wsy + K] : 0.0;
    }
    const double rdz = (k < nz - 1) ? dz_c[k + 1] : 1.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int r = ty + 8 * q, j = j0 + r;
        if (j >= ny || k >= nz) continue;
        const double f0 = t0[tx][r];
        const double fx = t1[tx][r];
        const double fy = t0[tx][r + 1];
        const size_t J = j + 1;
        u[I * usx + J * usy + K] = uo[q] - dt * ((fx - f0) * P.inv_dx);
        v[I * vsx + J * vsy + K] = vo[q] - dt * ((fy - f0) * P.inv_dy);
        if (k < nz - 1) {
            const double fz = t0[tx + 1][r];
            w[I * wsx + J * wsy + K] = wo[q] - dt * ((fz - f0) / rdz);
        }
        p[I * psx + J * psy + K] = f0;
    }
}

__global__ void __launch_bounds__(256) k_project(SlcParams P, const double *__restrict__ phi,
                                                 double *__restrict__ u, double *__restrict__ v,
                                                 double *__restrict__ w, double *__restrict__ p,
                                                 const double *__restrict__ dz_c, double dt)
{
    project_tile(P, phi, u, v, w, p, dz_c, dt, blockIdx.x, blockIdx.y, blockIdx.z);
}

// --------------------------------------------------------------------------
// Bulk velocity (utils.py:147-163): sum u dx dy dz_f / (Lx Ly Lz), summed in a
// fixed order (fixed grid, fixed block tree, fixed finish) so reruns agree
// bit for bit.  With c_dev, the shift u += c (solver.py:714-717) is applied
// first and the sum taken over the shifted field.
// --------------------------------------------------------------------------

__device__ __forceinline__ void bulk_partial(const SlcParams &P, double *__restrict__ u,
                                             const double *__restrict__ dz_f,
                                             const double *__restrict__ c_dev,
                                             double *__restrict__ partials, int bx, int G)
{
    __shared__ double red[256];
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int ncol = nx * ny;
    const double c = c_dev ? *c_dev : 0.0;
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    double acc = 0.0;
    // block b owns columns b, b + G, b + 2G, ...; its threads stride over k.
    // Four columns are loaded before they are accumulated (memory-level
    // parallelism); the summation order is fixed, so the result is too.
    for (int col0 = bx; col0 < ncol; col0 += 4 * G) {
        for (int k = threadIdx.x; k < nz; k += blockDim.x) {
            double val[4];
            double *ptr[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int col = col0 + q * G;
                ptr[q] = nullptr;
                val[q] = 0.0;
                if (col < ncol) {
                    const int i = col / ny, j = col - (col / ny) * ny;
                    ptr[q] = u + (size_t)(i + 1) * usx + (size_t)(j + 1) * usy + 1 + k;
                    val[q] = *ptr[q];
                }
            }
            const double dz = __ldg(dz_f + k);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (ptr[q]) {
                    double v = val[q];
                    if (c_dev) {
                        v = v + c;
                        *ptr[q] = v;
                    }
                    acc = fma(v, dz, acc);
                }
            }
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[bx] = red[0];
}

__global__ void __launch_bounds__(256) k_bulk_partials(SlcParams P, double *__restrict__ u,
                                                       const double *__restrict__ dz_f,
                                                       const double *__restrict__ c_dev,
                                                       double *__restrict__ partials)
{
    bulk_partial(P, u, dz_f, c_dev, partials, blockIdx.x, gridDim.x);
}

__device__ __forceinline__ void bulk_finish(const double *__restrict__ partials, int nparts,
                                            double dxdy_over_V, double U_bulk, double dt,
                                            double *bulk_out, double *shift_out)
{
    __shared__ double red[256];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) acc += partials[b];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double bulk = red[0] * dxdy_over_V;
        if (bulk_out) *bulk_out = bulk;
        if (shift_out) {
            const double corr = U_bulk - bulk;
            shift_out[0] = corr;
            shift_out[1] = corr / dt;
        }
    }
}

__global__ void k_bulk_finish(const double *__restrict__ partials, int nparts, double dxdy_over_V,
                              double U_bulk, double dt, double *bulk_out, double *shift_out)
{
    bulk_finish(partials, nparts, dxdy_over_V, U_bulk, dt, bulk_out, shift_out);
}

// ---- ensemble forms: one block per item, the instance's own arithmetic ----

__global__ void k_bc_ens(const EnsInst *__restrict__ ins, const EnsItem *__restrict__ items,
                         int lvl, int with_p)
{
    const EnsItem it = items[blockIdx.x];
    const EnsInst &I = ins[it.inst];
    const SlcParams &P = I.P;
    long long n[4];
    for (int c = 0; c < 4; ++c) {
        const BcCounts b = bc_counts(c, P.nx, P.ny, P.nz);
        n[c] = (c < 3 || with_p) ? b.a + b.b + b.c : 0;
    }
    const long long t0 = (long long)it.a * blockDim.x + threadIdx.x;
    for (long long t = t0; t < n[0] + n[1] + n[2] + n[3]; t += (long long)it.b * blockDim.x) {
        if (t < n[0]) bc_one(P, 0, I.lev[lvl][0], t);
        else if (t < n[0] + n[1]) bc_one(P, 1, I.lev[lvl][1], t - n[0]);
        else if (t < n[0] + n[1] + n[2]) bc_one(P, 2, I.lev[lvl][2], t - n[0] - n[1]);
        else bc_one(P, 3, I.p, t - n[0] - n[1] - n[2]);
    }
}

__global__ void __launch_bounds__(256) k_div_pack_ens(const EnsInst *__restrict__ ins,
                                                      const EnsItem *__restrict__ items, int lvl)
{
    const EnsItem it = items[blockIdx.x];
    const EnsInst &I = ins[it.inst];
    div_pack_tile(I.P, I.lev[lvl][0], I.lev[lvl][1], I.lev[lvl][2], I.dzf, (2.0 / 3.0) * I.dt,
                  I.rhs, it.a, it.b, it.c);
}

__global__ void __launch_bounds__(256) k_thomas_ens(const EnsInst *__restrict__ ins,
                                                    const EnsItem *__restrict__ items)
{
    const EnsItem it = items[blockIdx.x];
    const EnsInst &I = ins[it.inst];
    const double norm = 1.0 / ((double)I.P.nx * (double)I.P.ny);
    thomas_column(I.P, I.hat, I.cpw, I.kx2, I.ky2, I.cl, I.cr, norm,
                  it.a * blockDim.x + threadIdx.x);
}

__global__ void __launch_bounds__(256) k_project_ens(const EnsInst *__restrict__ ins,
                                                     const EnsItem *__restrict__ items, int lvl)
{
    const EnsItem it = items[blockIdx.x];
    const EnsInst &I = ins[it.inst];
    project_tile(I.P, I.rhs, I.lev[lvl][0], I.lev[lvl][1], I.lev[lvl][2], I.p, I.dzc,
                 (2.0 / 3.0) * I.dt, it.a, it.b, it.c);
}

__global__ void __launch_bounds__(256) k_bulk_partials_ens(const EnsInst *__restrict__ ins,
                                                           const EnsItem *__restrict__ items,
                                                           int lvl, int with_shift)
{
    const EnsItem it = items[blockIdx.x];
    const EnsInst &I = ins[it.inst];
    bulk_partial(I.P, I.lev[lvl][0], I.dzf, with_shift ? I.scal : nullptr, I.partials, it.a,
                 kBulkBlocks);
}

__global__ void k_bulk_finish_ens(const EnsInst *__restrict__ ins, int mode)
{
    const EnsInst &I = ins[blockIdx.x];
    const double dxdy_over_V = (I.P.dx * I.P.dy) / (I.Lx * I.Ly * I.P.Lz);
    if (mode == 0) {
        bulk_finish(I.partials, kBulkBlocks, dxdy_over_V, I.U_bulk, I.dt, nullptr, I.scal);
    } else {
        bulk_finish(I.partials, kBulkBlocks, dxdy_over_V, 0.0, 1.0, I.bulk_out, nullptr);
        if (threadIdx.x == 0) I.bulk_out[1] = I.scal[1];
    }
}

// u, v, w interiors -= c grad(p), p ghost-shaped (projection.py:250-272 on a
// ghost-filled pressure); the incremental branch's predictor term
// -dt_eff grad(2 p^n - p^{n-1}) (solver.py:905-941).
__global__ void k_grad_sub(SlcParams P, const double *__restrict__ p, double *u, double *v, double *w,
                           const double *__restrict__ dz_c, double c)
{
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const long long n = (long long)nx * ny * nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int k = (int)(t % nz);
    const int j = (int)((t / nz) % ny);
    const int i = (int)(t / ((long long)nz * ny));
    const size_t I = i + 1, J = j + 1, K = k + 1;
    const size_t psx = (size_t)(ny + 2) * (nz + 2), psy = nz + 2;
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    const size_t vsx = (size_t)(ny + 1) * (nz + 2), vsy = nz + 2;
    const size_t wsx = (size_t)(ny + 2) * (nz + 1), wsy = nz + 1;
    const double p0 = p[I * psx + J * psy + K];
    u[I * usx + J * usy + K] -= c * ((p[(I + 1) * psx + J * psy + K] - p0) / P.dx);
    v[I * vsx + J * vsy + K] -= c * ((p[I * psx + (J + 1) * psy + K] - p0) / P.dy);
    if (k < nz - 1) w[I * wsx + J * wsy + K] -= c * ((p[I * psx + J * psy + K + 1] - p0) / dz_c[K]);
}

}  // namespace

cudaError_t launch_apply_bc(const SlcParams &P, double *u, double *v, double *w, double *p,
                            cudaStream_t s)
{
    auto tot = [&](int C) {
        BcCounts c = bc_counts(C, P.nx, P.ny, P.nz);
        return c.a + c.b + c.c;
    };
    const long long n0 = u ? tot(0) : 0, n1 = v ? tot(1) : 0, n2 = w ? tot(2) : 0,
                    n3 = p ? tot(3) : 0;
    const long long total = n0 + n1 + n2 + n3;
    if (total == 0) return cudaSuccess;
    long long blocks = (total + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_apply_bc<<<(unsigned)blocks, 256, 0, s>>>(P, u, v, w, p, n0, n1, n2, n3);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_div_pack(const SlcParams &P, Tri f, const double *dz_f, double dt_div,
                            double *rhs_zmajor, cudaStream_t s)
{
    dim3 grid((P.nz + 31) / 32, (P.ny + 31) / 32, P.nx), block(32, 8);
    k_div_pack<<<grid, block, 0, s>>>(P, f.u, f.v, f.w, dz_f, dt_div, rhs_zmajor);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_divergence(const SlcParams &P, Tri f, const double *dz_f, double *div,
                              cudaStream_t s)
{
    long long n = (long long)P.nx * P.ny * P.nz;
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_divergence<<<(unsigned)blocks, 256, 0, s>>>(P, f.u, f.v, f.w, dz_f, div);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_thomas_poisson(const SlcParams &P, double *hat, double *cp, const double *kx2,
                                  const double *ky2, const double *cl, const double *cr,
                                  cudaStream_t s)
{
    const long long nthr = 4LL * P.nx * (P.ny / 2 + 1);  // thomas_column: 4 per column
    const double norm = 1.0 / ((double)P.nx * (double)P.ny);
    k_thomas<<<(unsigned)((nthr + 255) / 256), 256, 0, s>>>(P, hat, cp, kx2, ky2, cl, cr, norm);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_project(const SlcParams &P, const double *phi_zmajor, TriMut f, double *p,
                           const double *dz_c, double dt, cudaStream_t s)
{
    dim3 grid((P.nz + 31) / 32, (P.ny + 31) / 32, P.nx), block(32, 8);
    k_project<<<grid, block, 0, s>>>(P, phi_zmajor, f.u, f.v, f.w, p, dz_c, dt);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_bulk_partials(const SlcParams &P, double *u, const double *dz_f,
                                 const double *c_dev, double *partials, cudaStream_t s)
{
    k_bulk_partials<<<kBulkBlocks, 256, 0, s>>>(P, u, dz_f, c_dev, partials);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_bulk_finish(const SlcParams &P, const double *partials, double Lx, double Ly,
                               double U_bulk, double dt, double *bulk_out, double *shift_out,
                               cudaStream_t s)
{
    const double dxdy_over_V = (P.dx * P.dy) / (Lx * Ly * P.Lz);
    k_bulk_finish<<<1, 256, 0, s>>>(partials, kBulkBlocks, dxdy_over_V, U_bulk, dt, bulk_out,
                                    shift_out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_bc_ens(const EnsInst *ins, const EnsItem *items, int nitems, int lvl,
                          int with_p, cudaStream_t s)
{
    if (nitems <= 0) return cudaSuccess;
    k_bc_ens<<<nitems, 256, 0, s>>>(ins, items, lvl, with_p);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_div_pack_ens(const EnsInst *ins, const EnsItem *items, int nitems, int lvl,
                                cudaStream_t s)
{
    if (nitems <= 0) return cudaSuccess;
    k_div_pack_ens<<<nitems, dim3(32, 8), 0, s>>>(ins, items, lvl);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_thomas_ens(const EnsInst *ins, const EnsItem *items, int nitems, cudaStream_t s)
{
    if (nitems <= 0) return cudaSuccess;
    k_thomas_ens<<<nitems, 256, 0, s>>>(ins, items);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_project_ens(const EnsInst *ins, const EnsItem *items, int nitems, int lvl,
                               cudaStream_t s)
{
    if (nitems <= 0) return cudaSuccess;
    k_project_ens<<<nitems, dim3(32, 8), 0, s>>>(ins, items, lvl);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_bulk_partials_ens(const EnsInst *ins, const EnsItem *items, int nitems,
                                     int lvl, int with_shift, cudaStream_t s)
{
    if (nitems <= 0) return cudaSuccess;
    k_bulk_partials_ens<<<nitems, 256, 0, s>>>(ins, items, lvl, with_shift);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_bulk_finish_ens(const EnsInst *ins, int ninst, int mode, cudaStream_t s)
{
    if (ninst <= 0) return cudaSuccess;
    k_bulk_finish_ens<<<ninst, 256, 0, s>>>(ins, mode);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_grad_sub(const SlcParams &P, const double *p, TriMut f, const double *dz_c, double c,
                            cudaStream_t s)
{
    const long long n = (long long)P.nx * P.ny * P.nz;
    k_grad_sub<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, p, f.u, f.v, f.w, dz_c, c);
    count_launches(1);
    return cudaGetLastError();
}
