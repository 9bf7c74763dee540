// eulerian.cu -- the reference's Eulerian IMEX step (SLChannelFlow.step_imex,
// solver.py:1055-1135): AB2 explicit advection + x,y diffusion, Crank-Nicolson
// implicit z-diffusion, projection and the exact bulk shift.  It is the
// comparison baseline of the semi-Lagrangian step (benchmarks/bench_step.py:
// wall-clock per simulated time unit at each scheme's operating dt).
//
// k_rhs_imex fuses the flux-form advection and the explicit x,y diffusion of
// all three components (compute_momentum_rhs_fused_imex, operators.py:638-832)
// into one pass, one thread per interior point: each output reads its 3x3x3
// neighbourhood of u, v, w once.  k_cn_explicit forms the Crank-Nicolson
// right-hand side increment (1 - theta) dt nu d2/dz2 with the reference's wall
// closures (operators.py:443-461, 610-622); the implicit part reuses the
// warp z-solve with tables at theta dt.
#include <string>

#include "slc_grid.h"

namespace {

constexpr int kT = 256;

struct ImexArgs {
    int nx, ny, nz;
    double dx_inv, dy_inv, nu_dx2, nu_dy2;
    const double *dz_f, *dz_c;
    const double *u, *v, *w;
};

// rhs = diffusion_xy - advection on the interiors; ghosts untouched.
__global__ void __launch_bounds__(kT) k_rhs_imex(ImexArgs a, double *ru, double *rv, double *rw)
{
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long long n = (long long)nx * ny * nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int k = (int)(t % nz);
    const int j = (int)((t / nz) % ny);
    const int i = (int)(t / ((long long)nz * ny));
    const int I = i + 1, J = j + 1, K = k + 1;
    const size_t usx = (size_t)(ny + 2) * (nz + 2), usy = nz + 2;
    const size_t vsx = (size_t)(ny + 1) * (nz + 2), vsy = nz + 2;
    const size_t wsx = (size_t)(ny + 2) * (nz + 1), wsy = nz + 1;
    // u extended periodically in x past nx (index nx + 1 -> 1); v in y past ny
    auto U = [&](int ii, int jj, int kk) {
        return a.u[(size_t)(ii == nx + 1 ? 1 : ii) * usx + (size_t)jj * usy + kk];
    };
    auto Uy = [&](int ii, int jj, int kk) { return a.u[(size_t)ii * usx + (size_t)jj * usy + kk]; };
    auto V = [&](int ii, int jj, int kk) {
        return a.v[(size_t)ii * vsx + (size_t)(jj == ny + 1 ? 1 : jj) * vsy + kk];
    };
    auto W = [&](int ii, int jj, int kk) { return a.w[(size_t)ii * wsx + (size_t)jj * wsy + kk]; };
    const double dzfi = 1.0 / a.dz_f[k];

    // ---- u at (I, J, K) ----
    {
        double ui = 0.5 * (U(I, J, K) + U(I + 1, J, K));
        const double uu_r = ui * ui;
        ui = 0.5 * (U(I - 1, J, K) + U(I, J, K));
        const double duudx = (uu_r - ui * ui) * a.dx_inv;
        double vi = 0.5 * (a.v[(size_t)I * vsx + (size_t)J * vsy + K] + a.v[(size_t)(I + 1) * vsx + (size_t)J * vsy + K]);
        double uiy = 0.5 * (U(I, J, K) + U(I, J + 1, K));
        const double vu_t = vi * uiy;
        vi = 0.5 * (a.v[(size_t)I * vsx + (size_t)(J - 1) * vsy + K] + a.v[(size_t)(I + 1) * vsx + (size_t)(J - 1) * vsy + K]);
        uiy = 0.5 * (U(I, J - 1, K) + U(I, J, K));
        const double dvudy = (vu_t - vi * uiy) * a.dy_inv;
        double wi = 0.5 * (W(I, J, K) + W(I + 1, J, K));
        double uiz = 0.5 * (U(I, J, K) + U(I, J, K + 1));
        const double wu_t = wi * uiz;
        wi = 0.5 * (W(I, J, K - 1) + W(I + 1, J, K - 1));
        uiz = 0.5 * (U(I, J, K - 1) + U(I, J, K));
        const double dwudz = (wu_t - wi * uiz) * dzfi;
        const double adv = duudx + dvudy + dwudz;
        const double d2x = (U(I + 1, J, K) - 2.0 * U(I, J, K) + U(I - 1, J, K)) * a.nu_dx2;
        const double d2y = (Uy(I, J + 1, K) - 2.0 * Uy(I, J, K) + Uy(I, J - 1, K)) * a.nu_dy2;
        ru[(size_t)I * usx + (size_t)J * usy + K] = (d2x + d2y) - adv;
    }
    // ---- v at (I, J, K) ----
    {
        double ui = 0.5 * (Uy(I, J, K) + Uy(I, J + 1, K));
        double vix = 0.5 * (V(I, J, K) + V(I + 1, J, K));
        const double uv_r = ui * vix;
        ui = 0.5 * (Uy(I - 1, J, K) + Uy(I - 1, J + 1, K));
        vix = 0.5 * (V(I - 1, J, K) + V(I, J, K));
        const double duvdx = (uv_r - ui * vix) * a.dx_inv;
        double vi = 0.5 * (V(I, J, K) + V(I, J + 1, K));
        const double vv_t = vi * vi;
        vi = 0.5 * (V(I, J - 1, K) + V(I, J, K));
        const double dvvdy = (vv_t - vi * vi) * a.dy_inv;
        double wi = 0.5 * (W(I, J, K) + W(I, J + 1, K));
        double viz = 0.5 * (V(I, J, K) + V(I, J, K + 1));
        const double wv_t = wi * viz;
        wi = 0.5 * (W(I, J, K - 1) + W(I, J + 1, K - 1));
        viz = 0.5 * (V(I, J, K - 1) + V(I, J, K));
        const double dwvdz = (wv_t - wi * viz) * dzfi;
        const double adv = duvdx + dvvdy + dwvdz;
        const double vc = a.v[(size_t)I * vsx + (size_t)J * vsy + K];
        const double d2x = (a.v[(size_t)(I + 1) * vsx + (size_t)J * vsy + K] - 2.0 * vc +
                            a.v[(size_t)(I - 1) * vsx + (size_t)J * vsy + K]) * a.nu_dx2;
        const double d2y = (V(I, J + 1, K) - 2.0 * V(I, J, K) + V(I, J - 1, K)) * a.nu_dy2;
        rv[(size_t)I * vsx + (size_t)J * vsy + K] = (d2x + d2y) - adv;
    }
    // ---- w at interior face (I, J, K), K = 1 .. nz-1 ----
    if (k < nz - 1) {
        double ui = 0.5 * (Uy(I, J, K) + Uy(I, J, K + 1));
        double wix = 0.5 * (W(I, J, K) + W(I + 1, J, K));
        const double uw_r = ui * wix;
        ui = 0.5 * (Uy(I - 1, J, K) + Uy(I - 1, J, K + 1));
        wix = 0.5 * (W(I - 1, J, K) + W(I, J, K));
        const double duwdx = (uw_r - ui * wix) * a.dx_inv;
        double vi = 0.5 * (a.v[(size_t)I * vsx + (size_t)J * vsy + K] + a.v[(size_t)I * vsx + (size_t)J * vsy + K + 1]);
        double wiy = 0.5 * (W(I, J, K) + W(I, J + 1, K));
        const double vw_t = vi * wiy;
        vi = 0.5 * (a.v[(size_t)I * vsx + (size_t)(J - 1) * vsy + K] + a.v[(size_t)I * vsx + (size_t)(J - 1) * vsy + K + 1]);
        wiy = 0.5 * (W(I, J - 1, K) + W(I, J, K));
        const double dvwdy = (vw_t - vi * wiy) * a.dy_inv;
        double wi = 0.5 * (W(I, J, K) + W(I, J, K + 1));
        const double ww_t = wi * wi;
        wi = 0.5 * (W(I, J, K - 1) + W(I, J, K));
        const double dwwdz = (ww_t - wi * wi) / a.dz_c[K];
        const double adv = duwdx + dvwdy + dwwdz;
        const double d2x = (W(I + 1, J, K) - 2.0 * W(I, J, K) + W(I - 1, J, K)) * a.nu_dx2;
        const double d2y = (W(I, J + 1, K) - 2.0 * W(I, J, K) + W(I, J - 1, K)) * a.nu_dy2;
        rw[(size_t)I * wsx + (size_t)J * wsy + K] = (d2x + d2y) - adv;
    }
}

// f += dt (ca rc + cb rp) on the interiors (AB2, or forward Euler with cb = 0)
__global__ void k_ab2(int nx, int ny, int nz, int comp, double *f, const double *rc, const double *rp,
                      double dt, double ca, double cb)
{
    const GhostShape g = ghost_shape(comp, nx, ny, nz);
    const int nzi = comp == 2 ? nz - 1 : nz;
    const long long n = (long long)nx * ny * nzi;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % nzi);
        const int j = (int)((t / nzi) % ny);
        const int i = (int)(t / ((long long)nzi * ny));
        const size_t o = (size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z + (k + 1);
        f[o] += rp ? dt * (ca * rc[o] - (-cb) * rp[o]) : dt * rc[o];
    }
}

// inc = beta d2/dz2 f on the interiors with the reference's closures; the
// w stencil keeps its index convention (faces m-1, m, m+1 for unknown m).
__global__ void k_cn_explicit(int nx, int ny, int nz, int comp, int top_neumann, const double *f,
                              const double *dz_c, const double *dz_f, double beta, double *inc)
{
    const GhostShape g = ghost_shape(comp, nx, ny, nz);
    const int nzi = comp == 2 ? nz - 1 : nz;
    const long long n = (long long)nx * ny * nzi;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % nzi);
        const int j = (int)((t / nzi) % ny);
        const int i = (int)(t / ((long long)nzi * ny));
        const double *col = f + (size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z;
        double d2;
        if (comp < 2) {  // F = col[0 .. nz+1]; unknown k is level k + 1
            const double dl = dz_c[k], dr = dz_c[k + 1], dc = dz_f[k];
            if (k == 0)
                d2 = ((col[2] - col[1]) / dr - 2.0 * col[1] / dl) / dc;
            else if (k == nz - 1)
                d2 = top_neumann ? (-(col[nz] - col[nz - 1]) / dl) / dc
                                 : (-2.0 * col[nz] / dr - (col[nz] - col[nz - 1]) / dl) / dc;
            else
                d2 = ((col[k + 2] - col[k + 1]) / dr - (col[k + 1] - col[k]) / dl) / dc;
        } else {  // W = col[0 .. nz]; ni = nz - 1 unknowns
            const int ni = nz - 1;
            const double dl = dz_f[k], dr = dz_f[k + 1], dcv = dz_c[k + 1];
            if (k == 0)
                d2 = ((col[1] - col[0]) / dr - col[0] / dl) / dcv;
            else if (k == ni - 1)
                d2 = (-col[ni - 1] / dr - (col[ni - 1] - col[ni - 2]) / dl) / dcv;
            else
                d2 = ((col[k + 1] - col[k]) / dr - (col[k] - col[k - 1]) / dl) / dcv;
        }
        inc[(size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z + (k + 1)] = beta * d2;
    }
}

}  // namespace

// slc_api.cu internals used by the step
int slc_internal_zsolve_theta(slc_grid *g, double *u, double *v, double *w, double dt_implicit, cudaStream_t s);
int slc_internal_project(slc_grid *g, double *u, double *v, double *w, double *p, double dt_div,
                         double dt_proj, cudaStream_t s);
int slc_internal_apply_bc(slc_grid *g, double *u, double *v, double *w, cudaStream_t s);

extern "C" int slc_imex_rhs(slc_grid *g, const double *u, const double *v, const double *w, double *ru,
                            double *rv, double *rw, void *stream)
{
    if (!g) return SLC_E_INVALID;
    if (!u || !v || !w || !ru || !rv || !rw) {
        g->err = "null pointer";
        return SLC_E_INVALID;
    }
    cudaSetDevice(g->device);
    const SlcParams &P = g->P;
    ImexArgs a{P.nx, P.ny, P.nz, 1.0 / P.dx, 1.0 / P.dy, P.nu * (1.0 / (P.dx * P.dx)),
               P.nu * (1.0 / (P.dy * P.dy)), g->dzf, g->dzc, u, v, w};
    const long long n = (long long)P.nx * P.ny * P.nz;
    k_rhs_imex<<<(unsigned)((n + kT - 1) / kT), kT, 0, (cudaStream_t)stream>>>(a, ru, rv, rw);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g->err = std::string("IMEX right-hand side: ") + cudaGetErrorString(e);
        return SLC_E_CUDA;
    }
    return SLC_OK;
}

extern "C" int slc_step_imex(slc_grid *g, double *const vel[3], double *p, double *const rhs_cur[3],
                             double *const rhs_prev[3], int have_prev, double dt, double theta,
                             void *stream)
{
    if (!g) return SLC_E_INVALID;
    if (!vel || !p || !rhs_cur || !rhs_prev) {
        g->err = "null pointer";
        return SLC_E_INVALID;
    }
    for (int c = 0; c < 3; ++c)
        if (!vel[c] || !rhs_cur[c] || !rhs_prev[c]) {
            g->err = "null field pointer";
            return SLC_E_INVALID;
        }
    if (!(dt > 0.0) || !(theta > 0.0 && theta <= 1.0)) {
        g->err = "dt must be positive and theta in (0, 1]";
        return SLC_E_INVALID;
    }
    cudaSetDevice(g->device);
    cudaStream_t s = (cudaStream_t)stream;
    const SlcParams &P = g->P;
    int rc = slc_internal_apply_bc(g, vel[0], vel[1], vel[2], s);
    if (rc) return rc;
    rc = slc_imex_rhs(g, vel[0], vel[1], vel[2], rhs_cur[0], rhs_cur[1], rhs_cur[2], stream);
    if (rc) return rc;
    const int blocks = 148 * 8;
    for (int c = 0; c < 3; ++c)
        k_ab2<<<blocks, kT, 0, s>>>(P.nx, P.ny, P.nz, c, vel[c], rhs_cur[c], have_prev ? rhs_prev[c] : nullptr,
                                    dt, 1.5, -0.5);
    count_launches(3);
    rc = slc_internal_apply_bc(g, vel[0], vel[1], vel[2], s);
    if (rc) return rc;
    // Crank-Nicolson: f += (1 - theta) dt nu d2f/dz2 (into the spent rhs_prev), then the implicit solve
    if (theta < 1.0) {
        const double beta = (1.0 - theta) * dt * P.nu;
        for (int c = 0; c < 3; ++c)
            k_cn_explicit<<<blocks, kT, 0, s>>>(P.nx, P.ny, P.nz, c, P.top_neumann, vel[c], g->dzc, g->dzf,
                                                beta, rhs_prev[c]);
        for (int c = 0; c < 3; ++c)
            k_ab2<<<blocks, kT, 0, s>>>(P.nx, P.ny, P.nz, c, vel[c], rhs_prev[c], nullptr, 1.0, 1.0, 0.0);
        count_launches(6);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g->err = std::string("IMEX explicit part: ") + cudaGetErrorString(e);
        return SLC_E_CUDA;
    }
    rc = slc_internal_zsolve_theta(g, vel[0], vel[1], vel[2], theta * dt, s);
    if (!rc) rc = slc_internal_apply_bc(g, vel[0], vel[1], vel[2], s);
    if (!rc) rc = slc_internal_project(g, vel[0], vel[1], vel[2], p, dt, dt, s);
    return rc;
}
