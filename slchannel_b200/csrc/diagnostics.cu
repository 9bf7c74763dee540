// diagnostics.cu -- on-device diagnostics and statistics of the channel
// state: the quantities the reference's run loop computes every n_out /
// n_stats steps with host synchronisations (solver.py:1355-1392):
//  * slc_diagnostics(_raw): max|div| (utils.py:166-180), u_tau
//    (utils.py:116-144), the CFL inverse of compute_cfl_fused
//    (operators.py:839-940) and the bulk velocity (utils.py:147-163), from
//    one pass of fixed-grid partial reductions and a fixed-order finish;
//  * slc_stats_accumulate: one snapshot of TurbulenceStats.accumulate_statistics
//    (turbstats.py:156-360) -- plane means, second moments about them, the
//    plane-mean moments, and the 2-D spectra at a pair of wall-parallel
//    planes (batched cuFFT, folded), added to device accumulators.
// Everything stays on the device; results are read when the caller wants.
#include <cufft.h>

#include <string>

#include "slc_grid.h"

namespace {

constexpr int kDiagBlocks = 296;
constexpr int kDiagParts = 7;  // max div, max dti x/y/z, sum u dz_f, sum u(k=1), sum u(k=nz)
constexpr int kT = 256;

struct DiagArgs {
    int nx, ny, nz, top_neumann;
    double dx, dy, nu, Lx, Ly, Lz;
    const double *dz_f, *dz_c, *z_c;
    const double *u, *v, *w;
};

__global__ void __launch_bounds__(kT) k_diag_partials(DiagArgs a, double *partials)
{
    __shared__ double red[kDiagParts][kT];
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    const size_t vsx = (size_t)(ny + 1) * (nz + 2), vsy = nz + 2;
    const size_t wsx = (size_t)(ny + 2) * (nz + 1), wsy = nz + 1;
    const double dxi = 1.0 / a.dx, dyi = 1.0 / a.dy;
    auto U = [&](int I, int J, int K) { return a.u[(size_t)I * usx + (size_t)J * usy + K]; };
    auto V = [&](int I, int J, int K) { return a.v[(size_t)I * vsx + (size_t)J * vsy + K]; };
    auto W = [&](int I, int J, int K) { return a.w[(size_t)I * wsx + (size_t)J * wsy + K]; };
    double mdiv = 0.0, mx = 0.0, my = 0.0, mz = 0.0, sb = 0.0, s1 = 0.0, sn = 0.0;
    for (long long col = blockIdx.x; col < (long long)nx * ny; col += gridDim.x) {
        const int i = (int)(col / ny), j = (int)(col % ny);
        const int I = i + 1, J = j + 1;
        for (int k = threadIdx.x; k < nz; k += blockDim.x) {
            const int K = k + 1;
            // divergence (utils.py:166-180): periodic x-1 / y-1 through the ghosts
            const double dv = (U(I, J, K) - U(I - 1, J, K)) / a.dx + (V(I, J, K) - V(I, J - 1, K)) / a.dy +
                              (W(I, J, K) - W(I, J, K - 1)) / a.dz_f[k];
            mdiv = fmax(mdiv, fabs(dv));
            // CFL inverse (operators.py:859-928)
            const double dzfi = 1.0 / a.dz_f[k];
            const double ux = fabs(U(I, J, K));
            const double vx = 0.25 * fabs(V(I, J, K) + V(I, J - 1, K) + V(I + 1, J, K) + V(I + 1, J - 1, K));
            const double wx = 0.25 * fabs(W(I, J, K) + W(I, J, K - 1) + W(I + 1, J, K) + W(I + 1, J, K - 1));
            mx = fmax(mx, ux * dxi + vx * dyi + wx * dzfi);
            const double uy = 0.25 * fabs(U(I, J, K) + U(I, J + 1, K) + U(I - 1, J + 1, K) + U(I - 1, J, K));
            const double vy = fabs(V(I, J, K));
            const double wy = 0.25 * fabs(W(I, J, K) + W(I, J + 1, K) + W(I, J + 1, K - 1) + W(I, J, K - 1));
            my = fmax(my, uy * dxi + vy * dyi + wy * dzfi);
            if (k < nz - 1) {
                const double dzci = 1.0 / a.dz_c[K];
                const double uz = 0.25 * fabs(U(I, J, K) + U(I - 1, J, K) + U(I - 1, J, K + 1) + U(I, J, K + 1));
                const double vz = 0.25 * fabs(V(I, J, K) + V(I, J - 1, K) + V(I, J - 1, K + 1) + V(I, J, K + 1));
                const double wz = fabs(W(I, J, K));
                mz = fmax(mz, uz * dxi + vz * dyi + wz * dzci);
            }
            sb += U(I, J, K) * a.dz_f[k];  // bulk (utils.py:147-163)
        }
    }
    // wall-adjacent planes of u for u_tau, ghosts included (utils.py:127, 141)
    const long long npl = (long long)(nx + 1) * (ny + 2);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < npl;
         e += (long long)gridDim.x * blockDim.x) {
        s1 += a.u[(size_t)e * usy + 1];
        sn += a.u[(size_t)e * usy + nz];
    }
    const double vals[kDiagParts] = {mdiv, mx, my, mz, sb, s1, sn};
#pragma unroll
    for (int q = 0; q < kDiagParts; ++q) red[q][threadIdx.x] = vals[q];
    __syncthreads();
    for (int s = kT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
#pragma unroll
            for (int q = 0; q < 4; ++q) red[q][threadIdx.x] = fmax(red[q][threadIdx.x], red[q][threadIdx.x + s]);
#pragma unroll
            for (int q = 4; q < kDiagParts; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x < kDiagParts) partials[threadIdx.x * gridDim.x + blockIdx.x] = red[threadIdx.x][0];
}

__global__ void k_diag_finish(DiagArgs a, const double *partials, int G, double *out4)
{
    if (threadIdx.x != 0) return;
    double m[4] = {0.0, 0.0, 0.0, 0.0}, s[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < G; ++b) {
        for (int q = 0; q < 4; ++q) m[q] = fmax(m[q], partials[q * G + b]);
        for (int q = 0; q < 3; ++q) s[q] += partials[(4 + q) * G + b];
    }
    const double npl = (double)(a.nx + 1) * (double)(a.ny + 2);
    const double dist = a.z_c[1];
    const double ub = sqrt(fabs(a.nu * (s[1] / npl) / dist));
    const double ut = sqrt(fabs(a.nu * (s[2] / npl) / dist));
    out4[0] = m[0];
    out4[1] = a.top_neumann ? ub : 0.5 * (ub + ut);
    out4[2] = fmax(fmax(m[1], m[2]), m[3]);
    out4[3] = s[0] * a.dx * a.dy / (a.Lx * a.Ly * a.Lz);
}

// ---- statistics (turbstats.py:156-360) --------------------------------------
// means[q][k]: 0 U (u at cell centres), 1 V, 2 W, 3 u at its nodes, 4 v at its
// nodes (levels 0..nz-1), 5 w at its faces (levels 0..nz); one block per level.
struct StatArgs {
    int nx, ny, nz;
    const double *u, *v, *w;
    double *means;   // 6 x (nz + 1)
    double *moms;    // 4 x (nz + 1): uu, vv, ww at faces, uw
};

__device__ __forceinline__ double block_sum(double x, double *red)
{
    red[threadIdx.x] = x;
    __syncthreads();
    for (int s = kT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kT) k_stat_means(StatArgs a)
{
    __shared__ double red[kT];
    const int nx = a.nx, ny = a.ny, nz = a.nz, k = blockIdx.x;  // 0..nz
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    const size_t vsx = (size_t)(ny + 1) * (nz + 2), vsy = nz + 2;
    const size_t wsx = (size_t)(ny + 2) * (nz + 1), wsy = nz + 1;
    const long long n = (long long)nx * ny;
    double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (long long e = threadIdx.x; e < n; e += blockDim.x) {
        const int i = (int)(e / ny), j = (int)(e % ny);
        if (k < nz) {
            const int K = k + 1;
            s[0] += 0.5 * (a.u[(size_t)i * usx + (j + 1) * usy + K] + a.u[(size_t)(i + 1) * usx + (j + 1) * usy + K]);
            s[1] += 0.5 * (a.v[(size_t)(i + 1) * vsx + j * vsy + K] + a.v[(size_t)(i + 1) * vsx + (j + 1) * vsy + K]);
            s[2] += 0.5 * (a.w[(size_t)(i + 1) * wsx + (j + 1) * wsy + k] + a.w[(size_t)(i + 1) * wsx + (j + 1) * wsy + k + 1]);
            s[3] += a.u[(size_t)(i + 1) * usx + (j + 1) * usy + K];
            s[4] += a.v[(size_t)(i + 1) * vsx + (j + 1) * vsy + K];
        }
        s[5] += a.w[(size_t)(i + 1) * wsx + (j + 1) * wsy + k];
    }
    const double inv = 1.0 / (double)n;
    for (int q = 0; q < 6; ++q) {
        const double t = block_sum(s[q], red);
        if (threadIdx.x == 0 && (q == 5 || k < nz)) a.means[q * (nz + 1) + k] = t * inv;
    }
}

__global__ void __launch_bounds__(kT) k_stat_moments(StatArgs a)
{
    __shared__ double red[kT];
    const int nx = a.nx, ny = a.ny, nz = a.nz, k = blockIdx.x;
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    const size_t vsx = (size_t)(ny + 1) * (nz + 2), vsy = nz + 2;
    const size_t wsx = (size_t)(ny + 2) * (nz + 1), wsy = nz + 1;
    const long long n = (long long)nx * ny;
    const int L = nz + 1;
    const double Um = k < nz ? a.means[0 * L + k] : 0.0, Wm = k < nz ? a.means[2 * L + k] : 0.0;
    const double Un = k < nz ? a.means[3 * L + k] : 0.0, Vn = k < nz ? a.means[4 * L + k] : 0.0;
    const double Wf = a.means[5 * L + k];
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long e = threadIdx.x; e < n; e += blockDim.x) {
        const int i = (int)(e / ny), j = (int)(e % ny);
        if (k < nz) {
            const int K = k + 1;
            const double un = a.u[(size_t)(i + 1) * usx + (j + 1) * usy + K] - Un;
            const double vn = a.v[(size_t)(i + 1) * vsx + (j + 1) * vsy + K] - Vn;
            s[0] += un * un;
            s[1] += vn * vn;
            const double uc = 0.5 * (a.u[(size_t)i * usx + (j + 1) * usy + K] +
                                     a.u[(size_t)(i + 1) * usx + (j + 1) * usy + K]) - Um;
            const double wc = 0.5 * (a.w[(size_t)(i + 1) * wsx + (j + 1) * wsy + k] +
                                     a.w[(size_t)(i + 1) * wsx + (j + 1) * wsy + k + 1]) - Wm;
            s[3] += uc * wc;
        }
        const double wf = a.w[(size_t)(i + 1) * wsx + (j + 1) * wsy + k] - Wf;
        s[2] += wf * wf;
    }
    const double inv = 1.0 / (double)n;
    for (int q = 0; q < 4; ++q) {
        const double t = block_sum(s[q], red);
        if (threadIdx.x == 0 && (q == 2 || k < nz)) a.moms[q * L + k] = t * inv;
    }
}

// prof (11 x nz): U, uu, vv, ww, uw, Vm, Wm, Um2, Vm2, Wm2, UmWm sums
__global__ void k_stat_accum(StatArgs a, double *prof)
{
    const int nz = a.nz, L = nz + 1;
    for (int k = threadIdx.x + blockIdx.x * blockDim.x; k < nz; k += blockDim.x * gridDim.x) {
        const double U = a.means[0 * L + k], V = a.means[1 * L + k], W = a.means[2 * L + k];
        prof[0 * nz + k] += U;
        prof[1 * nz + k] += a.moms[0 * L + k];
        prof[2 * nz + k] += a.moms[1 * L + k];
        prof[3 * nz + k] += 0.5 * (a.moms[2 * L + k] + a.moms[2 * L + k + 1]);
        prof[4 * nz + k] += a.moms[3 * L + k];
        prof[5 * nz + k] += V;
        prof[6 * nz + k] += W;
        prof[7 * nz + k] += U * U;
        prof[8 * nz + k] += V * V;
        prof[9 * nz + k] += W * W;
        prof[10 * nz + k] += U * W;
    }
}

// Six (nx, ny) planes: u, v node fluctuations and the cell-centred w
// fluctuation at level kb-1, the same at kt-1 with w negated (turbstats.py:264-279).
__global__ void k_stat_planes(StatArgs a, int kb, int kt, double *planes)
{
    const int nx = a.nx, ny = a.ny, nz = a.nz, L = nz + 1;
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    const size_t vsx = (size_t)(ny + 1) * (nz + 2), vsy = nz + 2;
    const size_t wsx = (size_t)(ny + 2) * (nz + 1), wsy = nz + 1;
    const long long n = (long long)nx * ny;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < 6 * n;
         e += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(e / n);
        const long long r = e - q * n;
        const int i = (int)(r / ny), j = (int)(r % ny);
        const int k = (q < 3 ? kb : kt) - 1;  // interior level
        double val;
        if (q % 3 == 0) {
            val = a.u[(size_t)(i + 1) * usx + (j + 1) * usy + k + 1] - a.means[3 * L + k];
        } else if (q % 3 == 1) {
            val = a.v[(size_t)(i + 1) * vsx + (j + 1) * vsy + k + 1] - a.means[4 * L + k];
        } else {
            val = 0.5 * (a.w[(size_t)(i + 1) * wsx + (j + 1) * wsy + k] +
                         a.w[(size_t)(i + 1) * wsx + (j + 1) * wsy + k + 1]) - a.means[2 * L + k];
            if (q == 5) val = -val;
        }
        planes[e] = val;
    }
}

// spec (4 x nkx x nky) += folded 0.5 (bottom + top) auto/cross spectra.
__global__ void k_stat_spectra(int nx, int ny, const double2 *hat, double *spec)
{
    const int nkx = nx / 2, nky = ny / 2, nyh = ny / 2 + 1;
    const long long per = (long long)nx * nyh;
    const double norm = ((double)nx * ny) * ((double)nx * ny);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nkx * nky; t += gridDim.x * blockDim.x) {
        const int i = t / nky, j = t % nky;
        double e[4] = {0.0, 0.0, 0.0, 0.0};
        const int rows[2] = {i + 1, nx - 1 - i};  // E(kx) and the flipped E(-kx)
        for (int h = 0; h < 2; ++h) {
            const long long o = (long long)rows[h] * nyh + (j + 1);
            double part[4];
            for (int wall = 0; wall < 2; ++wall) {
                const double2 U = hat[(3 * wall + 0) * per + o];
                const double2 Vv = hat[(3 * wall + 1) * per + o];
                const double2 Ww = hat[(3 * wall + 2) * per + o];
                const double uu = (U.x * U.x + U.y * U.y) / norm;
                const double vv = (Vv.x * Vv.x + Vv.y * Vv.y) / norm;
                const double ww = (Ww.x * Ww.x + Ww.y * Ww.y) / norm;
                const double uw = (U.x * Ww.x + U.y * Ww.y) / norm;
                if (wall == 0) {
                    part[0] = uu; part[1] = vv; part[2] = ww; part[3] = uw;
                } else {
                    part[0] = 0.5 * (part[0] + uu);
                    part[1] = 0.5 * (part[1] + vv);
                    part[2] = 0.5 * (part[2] + ww);
                    part[3] = 0.5 * (part[3] + uw);
                }
            }
            for (int q = 0; q < 4; ++q) e[q] += part[q];
        }
        for (int q = 0; q < 4; ++q) spec[(size_t)q * nkx * nky + t] += e[q];
    }
}

}  // namespace

struct StatsWS {
    double *means = nullptr, *moms = nullptr, *planes = nullptr, *hat = nullptr, *diag = nullptr;
    cufftHandle plan = 0;
    bool planned = false;
};

void stats_free(StatsWS *s)
{
    if (!s) return;
    if (s->planned) cufftDestroy(s->plan);
    delete s;
}

namespace {

int sfail(slc_grid *g, int code, const std::string &m)
{
    g->err = m;
    return code;
}

int ensure_stats(slc_grid *g)
{
    if (g->stats) return SLC_OK;
    const SlcParams &P = g->P;
    StatsWS *s = new StatsWS();
    g->stats = s;
    auto al = [&](double **p, size_t n) -> bool {
        void *q = nullptr;
        if (cudaMalloc(&q, n * sizeof(double)) != cudaSuccess) return false;
        g->allocs.push_back(q);
        *p = (double *)q;
        return true;
    };
    const size_t plane = (size_t)P.nx * P.ny, half = (size_t)P.nx * (P.ny / 2 + 1);
    if (!al(&s->means, 6 * (size_t)(P.nz + 1)) || !al(&s->moms, 4 * (size_t)(P.nz + 1)) ||
        !al(&s->planes, 6 * plane) || !al(&s->hat, 12 * half) ||
        !al(&s->diag, (size_t)kDiagParts * kDiagBlocks))
        return sfail(g, SLC_E_NOMEM, "statistics workspace");
    int dims[2] = {P.nx, P.ny};
    if (cufftPlanMany(&s->plan, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, 6) != CUFFT_SUCCESS)
        return sfail(g, SLC_E_CUFFT, "cufftPlanMany (statistics spectra)");
    s->planned = true;
    return SLC_OK;
}

DiagArgs diag_args(int nx, int ny, int nz, double dx, double dy, const double *dz_f, const double *dz_c,
                   const double *z_c, double nu, int top_neumann, double Lx, double Ly, double Lz,
                   const double *u, const double *v, const double *w)
{
    DiagArgs a;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.top_neumann = top_neumann;
    a.dx = dx;
    a.dy = dy;
    a.nu = nu;
    a.Lx = Lx;
    a.Ly = Ly;
    a.Lz = Lz;
    a.dz_f = dz_f;
    a.dz_c = dz_c;
    a.z_c = z_c;
    a.u = u;
    a.v = v;
    a.w = w;
    return a;
}

cudaError_t launch_diag(const DiagArgs &a, double *scratch, double *out4, cudaStream_t s)
{
    k_diag_partials<<<kDiagBlocks, kT, 0, s>>>(a, scratch);
    k_diag_finish<<<1, 32, 0, s>>>(a, scratch, kDiagBlocks, out4);
    count_launches(2);
    return cudaGetLastError();
}

}  // namespace

extern "C" {

int slc_diagnostics_scratch_doubles(void) { return kDiagParts * kDiagBlocks; }

int slc_diagnostics_raw(int nx, int ny, int nz, double dx, double dy, const double *dz_f,
                        const double *dz_c, const double *z_c, double nu, int top_neumann, double Lx,
                        double Ly, double Lz, const double *u, const double *v, const double *w,
                        double *out4, double *scratch, void *stream)
{
    if (nx < 1 || ny < 1 || nz < 2 || !dz_f || !dz_c || !z_c || !u || !v || !w || !out4 || !scratch)
        return slc_report_error(SLC_E_INVALID, "bad diagnostics arguments");
    cudaError_t e = launch_diag(diag_args(nx, ny, nz, dx, dy, dz_f, dz_c, z_c, nu, top_neumann, Lx, Ly, Lz,
                                          u, v, w),
                                scratch, out4, (cudaStream_t)stream);
    if (e != cudaSuccess)
        return slc_report_error(SLC_E_CUDA, (std::string("diagnostics: ") + cudaGetErrorString(e)).c_str());
    return SLC_OK;
}

int slc_diagnostics(slc_grid *g, const double *u, const double *v, const double *w, double *out4,
                    void *stream)
{
    if (!g) return SLC_E_INVALID;
    if (!u || !v || !w || !out4) return sfail(g, SLC_E_INVALID, "null pointer");
    cudaSetDevice(g->device);
    int rc = ensure_stats(g);
    if (rc) return rc;
    const SlcParams &P = g->P;
    cudaError_t e = launch_diag(diag_args(P.nx, P.ny, P.nz, P.dx, P.dy, g->dzf, g->dzc, g->zc, P.nu,
                                          P.top_neumann, g->Lx, g->Ly, P.Lz, u, v, w),
                                g->stats->diag, out4, (cudaStream_t)stream);
    if (e != cudaSuccess) return sfail(g, SLC_E_CUDA, std::string("diagnostics: ") + cudaGetErrorString(e));
    return SLC_OK;
}

int slc_stats_accumulate(slc_grid *g, const double *u, const double *v, const double *w, double *prof,
                         double *spec, int k_bot, int k_top, void *stream)
{
    if (!g) return SLC_E_INVALID;
    if (!u || !v || !w) return sfail(g, SLC_E_INVALID, "null pointer");
    const SlcParams &P = g->P;
    if (spec && (k_bot < 1 || k_bot > P.nz || k_top < 1 || k_top > P.nz))
        return sfail(g, SLC_E_INVALID, "spectra planes must be interior levels 1..nz");
    cudaSetDevice(g->device);
    int rc = ensure_stats(g);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    StatsWS *w_ = g->stats;
    StatArgs a{P.nx, P.ny, P.nz, u, v, w, w_->means, w_->moms};
    k_stat_means<<<P.nz + 1, kT, 0, s>>>(a);
    count_launches(1);
    if (prof) {
        k_stat_moments<<<P.nz + 1, kT, 0, s>>>(a);
        k_stat_accum<<<(P.nz + 255) / 256, 256, 0, s>>>(a, prof);
        count_launches(2);
    }
    if (spec) {
        k_stat_planes<<<148 * 4, kT, 0, s>>>(a, k_bot, k_top, w_->planes);
        count_launches(1);
        if (cufftSetStream(w_->plan, s) != CUFFT_SUCCESS ||
            cufftExecD2Z(w_->plan, w_->planes, (cufftDoubleComplex *)w_->hat) != CUFFT_SUCCESS)
            return sfail(g, SLC_E_CUFFT, "cufftExecD2Z (statistics spectra)");
        k_stat_spectra<<<148, kT, 0, s>>>(P.nx, P.ny, (const double2 *)w_->hat, spec);
        count_launches(1);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return sfail(g, SLC_E_CUDA, std::string("statistics: ") + cudaGetErrorString(e));
    return SLC_OK;
}

}  // extern "C"
