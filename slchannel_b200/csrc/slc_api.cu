// slc_api.cu -- the C ABI (include/slc_b200.h): handle set-up and the
// entry points that sequence the kernels of the SL-BDF2 step on a stream.
#include <cufft.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/slc_b200.h"
#include "slc_grid.h"

std::atomic<long long> g_slc_launches{0};

namespace {

std::string g_create_err;

struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int fail(slc_grid *g, int code, const std::string &msg)
{
    if (g) g->err = msg;
    else g_create_err = msg;
    return code;
}

int cuda_fail(slc_grid *g, cudaError_t e, const char *what)
{
    return fail(g, SLC_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define SLC_CK(call, what)                                   \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(g, e_, what); \
    } while (0)

#define SLC_FFT(call, what)                                                                   \
    do {                                                                                      \
        cufftResult r_ = (call);                                                              \
        if (r_ != CUFFT_SUCCESS)                                                              \
            return fail(g, SLC_E_CUFFT, std::string(what) + ": cufft error " + std::to_string((int)r_)); \
    } while (0)

template <typename T>
int dalloc(slc_grid *g, T **p, size_t n, const char *what)
{
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T) > 0 ? n * sizeof(T) : 16);
    if (e != cudaSuccess) return fail(g, SLC_E_NOMEM, std::string("cudaMalloc ") + what + ": " + cudaGetErrorString(e));
    g->allocs.push_back(q);
    *p = (T *)q;
    return SLC_OK;
}

template <typename T>
int upload(slc_grid *g, T **p, const std::vector<T> &h, const char *what)
{
    int rc = dalloc(g, p, h.size(), what);
    if (rc) return rc;
    SLC_CK(cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), what);
    return SLC_OK;
}

// semilag.py:102-114: 1 / prod_{l != m}(z[b+m] - z[b+l]), products in ascending l,
// stored node-major (entry (b, m) at m * nb + b).
std::vector<double> denom_table(const std::vector<double> &zn, int order)
{
    const int nb = (int)zn.size() - order + 1;
    std::vector<double> t((size_t)std::max(nb, 0) * order);
    for (int b = 0; b < nb; ++b)
        for (int m = 0; m < order; ++m) {
            double prod = 1.0;
            bool first = true;
            for (int l = 0; l < order; ++l) {
                double d = (l == m) ? 1.0 : zn[b + m] - zn[b + l];
                prod = first ? d : prod * d;
                first = false;
            }
            t[(size_t)m * nb + b] = 1.0 / prod;  // node-major (denom_rows)
        }
    return t;
}

cudaStream_t S(void *stream) { return (cudaStream_t)stream; }

int ensure_zsolve_tables(slc_grid *g, double dt, cudaStream_t s)
{
    if (g->zs_valid && g->zs_dt == dt) return SLC_OK;
    const int nz = g->P.nz;
    SLC_CK(launch_zsolve_tables(g->P, g->dzc, g->dzf, dt, g->zs_tab,
                                g->zs_tab + zsolve_table_doubles(nz) / 2, s),
           "z-solve tables");
    g->zs_dt = dt;
    g->zs_valid = true;
    return SLC_OK;
}

long tim_begin(slc_grid *g, int phase, cudaStream_t s);
void tim_end(slc_grid *g, long slot, cudaStream_t s);

int do_zsolve(slc_grid *g, double *u, double *v, double *w, double dt, cudaStream_t s)
{
    long t = tim_begin(g, SLC_PHASE_ZSOLVE, s);
    int rc = ensure_zsolve_tables(g, dt, s);
    if (rc) return rc;
    SLC_CK(launch_zsolve(g->P, TriMut{u, v, w}, g->zs_tab,
                         g->zs_tab + zsolve_table_doubles(g->P.nz) / 2, s),
           "z-solve");
    tim_end(g, t, s);
    return SLC_OK;
}

int do_project(slc_grid *g, double *u, double *v, double *w, double *p, double dt_div,
               double dt_proj, cudaStream_t s)
{
    long t = tim_begin(g, SLC_PHASE_PROJECT, s);
    SLC_CK(launch_div_pack(g->P, Tri{u, v, w}, g->dzf, dt_div, g->rhs, s), "divergence");
    SLC_FFT(cufftSetStream(g->fwd, s), "cufftSetStream");
    SLC_FFT(cufftExecD2Z(g->fwd, g->rhs, (cufftDoubleComplex *)g->hat), "cufftExecD2Z");
    SLC_CK(launch_thomas_poisson(g->P, g->hat, g->cpw, g->kx2, g->ky2, g->cl, g->cr, s),
           "Poisson Thomas sweep");
    SLC_FFT(cufftSetStream(g->inv, s), "cufftSetStream");
    SLC_FFT(cufftExecZ2D(g->inv, (cufftDoubleComplex *)g->hat, g->rhs), "cufftExecZ2D");
    SLC_CK(launch_project(g->P, g->rhs, TriMut{u, v, w}, p, g->dzc, dt_proj, s), "projection");
    SLC_CK(launch_apply_bc(g->P, u, v, w, p, s), "boundary conditions");
    tim_end(g, t, s);
    return SLC_OK;
}

int ensure_mid(slc_grid *g)
{
    for (int c = 0; c < 3; ++c)
        if (!g->mid[c]) {
            int rc = dalloc(g, &g->mid[c], g->ghost_elems[c], "U* workspace");
            if (rc) return rc;
            SLC_CK(cudaMemset(g->mid[c], 0, g->ghost_elems[c] * sizeof(double)), "memset");
        }
    return SLC_OK;
}

// Padded node copies and tensor maps of the TMA-staged BDF2 gather; state -1
// (L1 gather) when the grid is too shallow for a box or the driver lacks the
// tensor-map entry point.
int ensure_tma(slc_grid *g)
{
    if (g->tma_state) return SLC_OK;
    if (!tma_supported(g->P)) {
        g->tma_state = -1;
        return SLC_OK;
    }
    for (int q = 0; q < 6; ++q) {
        int rc = dalloc(g, &g->tma.pad[q], tma_padded_elems(g->P, q % 3), "padded node copy");
        if (rc) return rc;
    }
    SLC_CK(tma_encode(g->P, g->tma), "tensor map encode");
    g->tma_state = 1;
    return SLC_OK;
}

int ensure_mixed(slc_grid *g);

// Halo-padded FP32 copies and tensor maps of the mixed form's staged gather;
// state -1 (L1 gather) when the grid is too shallow for a box or the driver
// lacks the tensor-map entry point.
int ensure_mixed_tma(slc_grid *g)
{
    if (g->tmx_state) return SLC_OK;
    int rc = ensure_mixed(g);
    if (rc) return rc;
    if (!mixed_tma_supported(g->P)) {
        g->tmx_state = -1;
        return SLC_OK;
    }
    for (int q = 0; q < 6; ++q) {
        const size_t n = mixed_tma_elems(g->P, g->mws, q % 3);
        rc = dalloc(g, &g->tmx.pad[q], n, "padded FP32 copy");
        if (rc) return rc;
        SLC_CK(cudaMemset(g->tmx.pad[q], 0, n * sizeof(float)), "memset");
    }
    if (mixed_tma_encode(g->P, g->mws, g->tmx) != cudaSuccess) {
        g->tmx_state = -1;
        return SLC_OK;
    }
    g->tmx_state = 1;
    return SLC_OK;
}

int ensure_mixed(slc_grid *g)
{
    if (g->mixed_ready) return SLC_OK;
    const SlcParams &P = g->P;
    g->mws.nzp[0] = g->mws.nzp[1] = mixed_nzp(P.nz + 2);
    g->mws.nzp[2] = mixed_nzp(P.nz + 1);
    for (int q = 0; q < 9; ++q) {
        const size_t n = (size_t)P.nx * P.ny * g->mws.nzp[q % 3];
        int rc = dalloc(g, &g->mws.f32[q], n, "mixed FP32 node buffer");
        if (rc) return rc;
        rc = dalloc(g, &g->mws.mean[q], (size_t)P.nz + 2, "mixed plane mean");
        if (rc) return rc;
        rc = dalloc(g, &g->mws.mean32[q], (size_t)P.nz + 2, "mixed plane mean fp32");
        if (rc) return rc;
    }
    int rc = dalloc(g, &g->mws.partials, mixed_partials_doubles(P), "mixed mean partials");
    if (rc) return rc;
    g->mixed_ready = true;
    return SLC_OK;
}

}  // namespace

int slc_grid_ensure_mixed(slc_grid *g) { return ensure_mixed(g); }
int slc_grid_ensure_mid(slc_grid *g) { return ensure_mid(g); }

int slc_grid_ensure_staged(slc_grid *g, bool *ready)
{
    *ready = false;
    int rc;
    if (g->mixed) {
        rc = ensure_mixed_tma(g);
        if (!rc) *ready = g->tmx_state == 1;
    } else {
        rc = ensure_mid(g);
        if (!rc) rc = ensure_tma(g);
        if (!rc) *ready = g->tma_state == 1;
    }
    return rc;
}

// The BDF2 step after its trace+gather: the implicit z diffusion and the
// projection of next (slc_step_bdf2's tail; the host step streams the rest).
int slc_step_bdf2_tail(slc_grid *g, double *const next[3], double *p, double dt, cudaStream_t s)
{
    const double dt_eff = (2.0 / 3.0) * dt;
    int rc = do_zsolve(g, next[0], next[1], next[2], dt_eff, s);
    if (rc) return rc;
    return do_project(g, next[0], next[1], next[2], p, dt_eff, dt_eff, s);
}

namespace {

unsigned long long *counter(slc_grid *g, int64_t *user)
{
    return user ? (unsigned long long *)user : g->ncl_scratch;
}

constexpr size_t kMaxTimedIntervals = 1 << 15;

// Start a timed interval of `phase` on stream s; returns its slot or -1.
long tim_begin(slc_grid *g, int phase, cudaStream_t s)
{
    if (!g->timing || g->ev_used >= kMaxTimedIntervals) return -1;
    const size_t i = g->ev_used;
    if (g->evs.size() < 2 * (i + 1)) {
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess) return -1;
        if (cudaEventCreate(&b) != cudaSuccess) {
            cudaEventDestroy(a);
            return -1;
        }
        g->evs.push_back(a);
        g->evs.push_back(b);
        g->ev_phase.push_back(phase);
    }
    g->ev_phase[i] = phase;
    if (cudaEventRecord(g->evs[2 * i], s) != cudaSuccess) return -1;
    g->ev_used = i + 1;
    return (long)i;
}

void tim_end(slc_grid *g, long slot, cudaStream_t s)
{
    if (slot >= 0) cudaEventRecord(g->evs[2 * slot + 1], s);
}

int do_apply_bc(slc_grid *g, double *u, double *v, double *w, cudaStream_t s)
{
    long t = tim_begin(g, SLC_PHASE_BC, s);
    SLC_CK(launch_apply_bc(g->P, u, v, w, nullptr, s), "boundary conditions");
    tim_end(g, t, s);
    return SLC_OK;
}

// Which trace+gather: the step's choice, the L1 gather, or the TMA-staged one.
enum GatherMode { kGatherDefault, kGatherL1, kGatherStaged };
#ifndef SLC_MIXED_STAGED_DEFAULT  // the mixed step gathers from TMA-staged boxes
#define SLC_MIXED_STAGED_DEFAULT 1
#endif
#ifndef SLC_FP64_STAGED_DEFAULT  // so does the FP64 step at order 6
#define SLC_FP64_STAGED_DEFAULT 1
#endif
#ifndef SLC_FP64_O4_STAGED_DEFAULT  // and at order 4
#define SLC_FP64_O4_STAGED_DEFAULT 0
#endif
// The step keeps gathering from staged boxes while at least this fraction of
// the blocks staged both feet, and otherwise gathers through L1 (whose
// kernel holds more registers per thread, so it is the faster when many
// blocks would fall back), trying the staged gather again every
// kStagedProbeEvery calls.  The two gathers give the same results.
constexpr double kStagedMinFraction = 0.9;
constexpr int kStagedProbeEvery = 50;

bool capturing(cudaStream_t s)
{
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(s, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone;
}

// The default mode's choice, from the staged-box counters of an earlier call
// (copied to pinned host memory behind that call, read here once its event
// has completed: no synchronisation).
bool choose_staged(slc_grid *g, cudaStream_t s)
{
    GatherChoice &c = g->gchoice;
    if (capturing(s)) return c.staged;  // no bookkeeping inside a graph capture
    if (c.pending) {
        const cudaError_t q = cudaEventQuery(c.ev);
        if (q == cudaSuccess) {
            const unsigned long long *h = c.host;
            auto delta = [&](int k) { return h[k] >= c.last[k] ? h[k] - c.last[k] : h[k]; };  // reset between
            const unsigned long long blocks = delta(1), both = std::min(delta(2), delta(3));
            if (blocks > 0) c.staged = (double)both >= kStagedMinFraction * (double)blocks;
            for (int k = 0; k < 4; ++k) c.last[k] = h[k];
            c.pending = false;
        } else if (q == cudaErrorNotReady && cudaPeekAtLastError() == cudaErrorNotReady) {
            cudaGetLastError();  // "not ready" is no error of the caller's
        }
    }
    if (!c.staged && ++c.calls_l1 >= kStagedProbeEvery) {
        c.calls_l1 = 0;
        return true;  // probe: the counters of this call decide again
    }
    return c.staged;
}

// After a staged launch of the default mode: copy the counters behind it.
void note_staged(slc_grid *g, cudaStream_t s)
{
    GatherChoice &c = g->gchoice;
    if (c.pending || capturing(s)) return;
    if (!c.host) {
        void *h = nullptr;
        if (cudaHostAlloc(&h, 4 * sizeof(unsigned long long), cudaHostAllocDefault) != cudaSuccess) return;
        if (cudaEventCreateWithFlags(&c.ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaFreeHost(h);
            return;
        }
        c.host = (unsigned long long *)h;
    }
    if (cudaMemcpyAsync(c.host, g->dev_flags, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s) ==
            cudaSuccess &&
        cudaEventRecord(c.ev, s) == cudaSuccess)
        c.pending = true;
}

int do_trace_gather_bdf2(slc_grid *g, const double *const cur[3], const double *const prev[3],
                         double dt, double *const out[3], int64_t *nclamp, cudaStream_t s,
                         GatherMode mode = kGatherDefault)
{
    if (g->mixed) {
        int rc = ensure_mixed(g);
        if (rc) return rc;
        // at order 4 the mixed step keeps its L1 gather (5.37 against 5.80 ms
        // per tricubic step at 256^3)
        bool want = mode == kGatherStaged ||
                    (mode == kGatherDefault && SLC_MIXED_STAGED_DEFAULT && g->P.order == 6);
        if (want) {
            rc = ensure_mixed_tma(g);
            if (rc) return rc;
            if (mode == kGatherDefault && g->tmx_state == 1) want = choose_staged(g, s);
        }
        if (want && g->tmx_state == 1) {
            long t = tim_begin(g, SLC_PHASE_MID, s);
            SLC_CK(launch_mixed_prepare(g->P, Tri{cur[0], cur[1], cur[2]}, Tri{prev[0], prev[1], prev[2]},
                                        Tri{nullptr, nullptr, nullptr}, g->mws, s, &g->tmx),
                   "mixed-form pack (padded)");
            tim_end(g, t, s);
            unsigned long long *ncl = counter(g, nclamp);
            SLC_CK(cudaMemsetAsync(ncl, 0, sizeof(unsigned long long), s), "memset");
            t = tim_begin(g, SLC_PHASE_SL, s);
            SLC_CK(launch_sl_mixed_tma(g->P, Tri{cur[0], cur[1], cur[2]}, Tri{prev[0], prev[1], prev[2]}, g->mws,
                                       g->tmx, dt, TriMut{out[0], out[1], out[2]}, ncl, g->dev_flags, s),
                   "mixed trace+gather BDF2 (TMA-staged)");
            tim_end(g, t, s);
            if (mode == kGatherDefault) note_staged(g, s);
            return SLC_OK;
        }
        long t = tim_begin(g, SLC_PHASE_MID, s);
        SLC_CK(launch_mixed_prepare(g->P, Tri{cur[0], cur[1], cur[2]}, Tri{prev[0], prev[1], prev[2]},
                                    Tri{nullptr, nullptr, nullptr}, g->mws, s),
               "mixed-form pack");
        tim_end(g, t, s);
        unsigned long long *ncl = counter(g, nclamp);
        SLC_CK(cudaMemsetAsync(ncl, 0, sizeof(unsigned long long), s), "memset");
        t = tim_begin(g, SLC_PHASE_SL, s);
        SLC_CK(launch_sl_mixed(g->P, 2, Tri{cur[0], cur[1], cur[2]}, Tri{prev[0], prev[1], prev[2]},
                               g->mws, dt, TriMut{out[0], out[1], out[2]}, ncl, s),
               "mixed trace+gather BDF2");
        tim_end(g, t, s);
        return SLC_OK;
    }
    // the FP64 staged kernel holds three blocks per SM; at order 4 the L1
    // kernel runs four and stays the faster
    bool staged = mode == kGatherStaged ||
                  (mode == kGatherDefault && (g->P.order == 6 ? SLC_FP64_STAGED_DEFAULT : SLC_FP64_O4_STAGED_DEFAULT));
    int rc = ensure_mid(g);
    if (!rc && staged) rc = ensure_tma(g);
    if (rc) return rc;
    if (staged && mode == kGatherDefault && g->tma_state == 1) staged = choose_staged(g, s);
    if (staged && g->tma_state == 1) {
        long t = tim_begin(g, SLC_PHASE_MID, s);
        SLC_CK(launch_mid_pack(g->P, Tri{cur[0], cur[1], cur[2]}, Tri{prev[0], prev[1], prev[2]},
                               TriMut{g->mid[0], g->mid[1], g->mid[2]}, g->tma, s),
               "U* and padded node copies");
        tim_end(g, t, s);
        unsigned long long *ncl = counter(g, nclamp);
        SLC_CK(cudaMemsetAsync(ncl, 0, sizeof(unsigned long long), s), "memset");
        t = tim_begin(g, SLC_PHASE_SL, s);
        SLC_CK(launch_sl_tma(g->P, Tri{cur[0], cur[1], cur[2]}, Tri{prev[0], prev[1], prev[2]},
                             Tri{g->mid[0], g->mid[1], g->mid[2]}, dt, TriMut{out[0], out[1], out[2]},
                             ncl, g->dev_flags, g->tma, s),
               "trace+gather BDF2 (TMA-staged)");
        tim_end(g, t, s);
        if (mode == kGatherDefault) note_staged(g, s);
        return SLC_OK;
    }
    long t = tim_begin(g, SLC_PHASE_MID, s);
    for (int c = 0; c < 3; ++c)
        SLC_CK(launch_lincomb(cur[c], prev[c], 2.0, -1.0, g->mid[c], (int64_t)g->ghost_elems[c], s),
               "U* = 2V^n - V^{n-1}");
    tim_end(g, t, s);
    unsigned long long *ncl = counter(g, nclamp);
    SLC_CK(cudaMemsetAsync(ncl, 0, sizeof(unsigned long long), s), "memset");
    t = tim_begin(g, SLC_PHASE_SL, s);
    SLC_CK(launch_sl(g->P, 2, Tri{cur[0], cur[1], cur[2]}, Tri{prev[0], prev[1], prev[2]},
                     Tri{g->mid[0], g->mid[1], g->mid[2]}, false, dt, TriMut{out[0], out[1], out[2]},
                     ncl, s),
           "trace+gather BDF2");
    tim_end(g, t, s);
    return SLC_OK;
}

}  // namespace

// Step pieces for the other translation units (eulerian.cu).
int slc_internal_zsolve_theta(slc_grid *g, double *u, double *v, double *w, double dt_implicit, cudaStream_t s)
{
    return do_zsolve(g, u, v, w, dt_implicit, s);
}
int slc_internal_project(slc_grid *g, double *u, double *v, double *w, double *p, double dt_div,
                         double dt_proj, cudaStream_t s)
{
    return do_project(g, u, v, w, p, dt_div, dt_proj, s);
}
int slc_internal_apply_bc(slc_grid *g, double *u, double *v, double *w, cudaStream_t s)
{
    return do_apply_bc(g, u, v, w, s);
}

// Record the message of a failed handle-free call (read with slc_last_error(NULL)).
int slc_report_error(int code, const char *msg)
{
    g_create_err = msg;
    return code;
}

extern "C" {

const char *slc_version(void) { return "slc_b200 0.1"; }

const char *slc_last_error(const slc_grid *g) { return g ? g->err.c_str() : g_create_err.c_str(); }

int slc_grid_create(const slc_grid_desc *d, slc_grid **out)
{
    slc_grid *g = nullptr;
    if (!d || !out) return fail(nullptr, SLC_E_INVALID, "null descriptor or output pointer");
    *out = nullptr;
    if (d->order != 4 && d->order != 6)
        return fail(nullptr, SLC_E_INVALID, "sl.interp_order must be 4 (tricubic) or 6 (triquintic), got " + std::to_string(d->order));
    if (d->traj_order != 2 && d->traj_order != 4)
        return fail(nullptr, SLC_E_INVALID, "sl.traj_interp_order must be 2 (trilinear) or 4 (tricubic), got " + std::to_string(d->traj_order));
    if (d->n_traj_iters < 1)
        return fail(nullptr, SLC_E_INVALID, "sl.n_traj_iters must be >= 1");
    if (d->stretching != 0 && d->stretching != 1)
        return fail(nullptr, SLC_E_INVALID, "stretching must be 0 (symmetric) or 1 (bottom)");
    if (d->precision != SLC_PREC_FP64 && d->precision != SLC_PREC_MIXED)
        return fail(nullptr, SLC_E_INVALID, "unknown precision form");
    if (d->nx < 1 || d->ny < 1 || d->nz < 2)
        return fail(nullptr, SLC_E_INVALID, "grid needs nx, ny >= 1 and nz >= 2");
    if (d->nz + 1 < d->order)
        return fail(nullptr, SLC_E_INVALID, "nz=" + std::to_string(d->nz) + " too small for interpolation order " + std::to_string(d->order));
    if (d->nz > 1024) return fail(nullptr, SLC_E_INVALID, "nz > 1024 is not supported");
    const double big = (double)(d->nx + 2) * (d->ny + 2) * (d->nz + 2);
    if (big >= 2147483647.0)
        return fail(nullptr, SLC_E_INVALID, "grid too large for 32-bit field indexing");
    if (!d->z_f || !d->z_c) return fail(nullptr, SLC_E_INVALID, "z_f / z_c host pointers are null");
    if (!(d->Lx > 0 && d->Ly > 0 && d->Lz > 0 && d->nu >= 0 && d->gamma > 0))
        return fail(nullptr, SLC_E_INVALID, "domain extents, gamma and nu must be positive");

    g = new slc_grid();
    g->device = d->device;
    DeviceGuard dg(d->device);
    if (!dg.ok) {
        delete g;
        return fail(nullptr, SLC_E_CUDA, "cannot select CUDA device " + std::to_string(d->device));
    }
    const int nx = d->nx, ny = d->ny, nz = d->nz;
    SlcParams &P = g->P;
    P.nx = nx;
    P.ny = ny;
    P.nz = nz;
    P.symmetric = d->stretching == 0;
    P.order = d->order;
    P.n_iters = d->n_traj_iters;
    P.traj_order = d->traj_order;
    P.top_neumann = d->top_wall_neumann ? 1 : 0;
    P.xy_lagged = d->xy_rhs_lagged ? 1 : 0;
    g->mixed = d->precision == SLC_PREC_MIXED ? 1 : 0;
    g->Lx = d->Lx;
    g->Ly = d->Ly;
    P.dx = d->Lx / nx;
    P.dy = d->Ly / ny;
    P.inv_dx = 1.0 / P.dx;
    P.inv_dy = 1.0 / P.dy;
    P.inv_dx2 = 1.0 / (P.dx * P.dx);
    P.inv_dy2 = 1.0 / (P.dy * P.dy);
    P.Lz = d->Lz;
    P.two_over_Lz = 2.0 / d->Lz;
    P.inv_Lz = 1.0 / d->Lz;
    P.gamma = d->gamma;
    P.inv_gamma = 1.0 / d->gamma;
    P.tanh_g = std::tanh(d->gamma);
    P.half_nz = 0.5 * nz;
    P.nzd = (double)nz;
    P.nu = d->nu;
    std::vector<double> zf(d->z_f, d->z_f + nz + 1), zc(d->z_c, d->z_c + nz + 2);
    const double eps_z = 1e-12 * d->Lz;  // semilag.py:244-247
    P.z_lo = zf[0] + eps_z;
    P.z_hi = zf[nz] - eps_z;
    for (int o = 2; o <= SLC_MAX_ORDER; o += 2) {
        const int h = o / 2 - 1;
        for (int m = 0; m < o; ++m) {
            double den = 1.0;
            for (int l = 0; l < o; ++l)
                if (l != m) den *= (double)((m - h) - (l - h));
            P.udenom[o][m] = 1.0 / den;
        }
    }
    std::vector<double> dzf(nz), dzc(nz + 1);
    for (int k = 0; k < nz; ++k) dzf[k] = zf[k + 1] - zf[k];
    for (int k = 0; k <= nz; ++k) dzc[k] = zc[k + 1] - zc[k];

    int rc = SLC_OK;
#define CREATE_CK(expr)                        \
    do {                                       \
        rc = (expr);                           \
        if (rc) {                              \
            std::string m_ = g->err;           \
            slc_grid_destroy(g);               \
            return fail(nullptr, rc, m_);      \
        }                                      \
    } while (0)

    CREATE_CK(upload(g, &g->zc, zc, "z_c"));
    CREATE_CK(upload(g, &g->zf, zf, "z_f"));
    CREATE_CK(upload(g, &g->dzc, dzc, "dz_c"));
    CREATE_CK(upload(g, &g->dzf, dzf, "dz_f"));
    {
        std::vector<float> zc32(zc.begin(), zc.end()), zf32(zf.begin(), zf.end());
        CREATE_CK(upload(g, &g->zc32, zc32, "z_c fp32"));
        CREATE_CK(upload(g, &g->zf32, zf32, "z_f fp32"));
    }
    for (int o = 2; o <= SLC_MAX_ORDER; o += 2) {
        if (nz + 2 - o + 1 <= 0) continue;
        std::vector<double> tc = denom_table(zc, o);
        CREATE_CK(upload(g, &g->dinv_c[o], tc, "centre denominators"));
        std::vector<float> tc32(tc.begin(), tc.end());
        CREATE_CK(upload(g, &g->dinv_c32[o], tc32, "centre denominators fp32"));
        if (nz + 1 - o + 1 > 0) {
            std::vector<double> tf = denom_table(zf, o);
            CREATE_CK(upload(g, &g->dinv_f[o], tf, "face denominators"));
            std::vector<float> tf32(tf.begin(), tf.end());
            CREATE_CK(upload(g, &g->dinv_f32[o], tf32, "face denominators fp32"));
        }
    }
    P.zc = g->zc;
    P.zf = g->zf;
    P.zc32 = g->zc32;
    P.zf32 = g->zf32;
    for (int o = 0; o <= SLC_MAX_ORDER; ++o) {
        P.dinv_c[o] = g->dinv_c[o];
        P.dinv_f[o] = g->dinv_f[o];
        P.dinv_c32[o] = g->dinv_c32[o];
        P.dinv_f32[o] = g->dinv_f32[o];
    }

    // Poisson tables (projection.py:47-114): modified wavenumbers and the
    // two z-coupling coefficients.
    const int nky = ny / 2 + 1;
    {
        const double two_pi = 2.0 * M_PI;
        const double ddx = P.dx / two_pi, ddy = P.dy / two_pi;
        const double vx = 1.0 / (nx * ddx), vy = 1.0 / (ny * ddy);
        std::vector<double> kx2(nx), ky2(nky), cl(nz), cr(nz);
        for (int m = 0; m < nx; ++m) {
            const double f = (m < (nx + 1) / 2) ? (double)m : (double)(m - nx);
            const double kx = f * vx;
            const double km = (2.0 / P.dx) * std::sin(kx * P.dx / 2.0);
            kx2[m] = km * km;
        }
        for (int m = 0; m < nky; ++m) {
            const double ky = (double)m * vy;
            const double km = (2.0 / P.dy) * std::sin(ky * P.dy / 2.0);
            ky2[m] = km * km;
        }
        for (int k = 0; k < nz; ++k) {
            cl[k] = 1.0 / (dzc[k] * dzf[k]);
            cr[k] = 1.0 / (dzc[k + 1] * dzf[k]);
        }
        CREATE_CK(upload(g, &g->kx2, kx2, "kx2"));
        CREATE_CK(upload(g, &g->ky2, ky2, "ky2"));
        CREATE_CK(upload(g, &g->cl, cl, "coeff_left"));
        CREATE_CK(upload(g, &g->cr, cr, "coeff_right"));
    }
    const size_t nreal = (size_t)nz * nx * ny, ncplx = (size_t)nz * nx * nky;
    CREATE_CK(dalloc(g, &g->rhs, nreal, "Poisson rhs"));
    CREATE_CK(dalloc(g, &g->hat, 2 * ncplx, "Poisson spectrum"));
    CREATE_CK(dalloc(g, &g->cpw, ncplx, "Poisson Thomas scratch"));
    CREATE_CK(dalloc(g, &g->zs_tab, zsolve_table_doubles(nz), "z-solve tables"));
    CREATE_CK(dalloc(g, &g->partials, (size_t)kBulkBlocks, "bulk partials"));
    CREATE_CK(dalloc(g, &g->scal, (size_t)8, "scalars"));
    CREATE_CK(dalloc(g, &g->dev_flags, (size_t)4, "device flags"));
    if (cudaMemset(g->dev_flags, 0, 4 * sizeof(unsigned long long)) != cudaSuccess) {
        slc_grid_destroy(g);
        return fail(nullptr, SLC_E_CUDA, "memset device flags");
    }
    CREATE_CK(dalloc(g, &g->ncl_scratch, (size_t)1, "clamp counter"));
    for (int c = 0; c < 4; ++c) {
        GhostShape s = ghost_shape(c, nx, ny, nz);
        g->ghost_elems[c] = (size_t)s.X * s.Y * s.Z;
    }
    {
        int dims[2] = {nx, ny};
        if (cufftPlanMany(&g->fwd, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, nz) != CUFFT_SUCCESS) {
            slc_grid_destroy(g);
            return fail(nullptr, SLC_E_CUFFT, "cufftPlanMany D2Z failed");
        }
        if (cufftPlanMany(&g->inv, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, nz) != CUFFT_SUCCESS) {
            cufftDestroy(g->fwd);
            slc_grid_destroy(g);
            return fail(nullptr, SLC_E_CUFFT, "cufftPlanMany Z2D failed");
        }
        g->plans = true;
    }
#undef CREATE_CK
    *out = g;
    return SLC_OK;
}

int slc_grid_destroy(slc_grid *g)
{
    if (!g) return SLC_OK;
    DeviceGuard dg(g->device);
    if (g->plans) {
        cufftDestroy(g->fwd);
        cufftDestroy(g->inv);
    }
    for (cudaEvent_t e : g->evs) cudaEventDestroy(e);
    for (void *p : g->allocs) cudaFree(p);
    if (g->adj) adj_free(g->adj);
    if (g->stats) stats_free(g->stats);
    if (g->host) {
        cudaDeviceSynchronize();  // copies in flight may still use the host buffers
        host_step_free(g->host);
    }
    if (g->gchoice.host) {
        cudaDeviceSynchronize();  // a counter copy may still be in flight
        cudaFreeHost(g->gchoice.host);
    }
    if (g->gchoice.ev) cudaEventDestroy(g->gchoice.ev);
    delete g;
    return SLC_OK;
}

int slc_apply_bc(slc_grid *g, double *u, double *v, double *w, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    DeviceGuard dg(g->device);
    return do_apply_bc(g, u, v, w, S(stream));
}

int slc_face_coord(slc_grid *g, const double *z, int64_t n, double *kf, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (n < 0 || (n > 0 && (!z || !kf))) return fail(g, SLC_E_INVALID, "bad face_coord arguments");
    DeviceGuard dg(g->device);
    SLC_CK(launch_face_coord(g->P, z, n, kf, S(stream)), "face_coord");
    return SLC_OK;
}

int slc_interp_points(slc_grid *g, int comp, int order, const double *nodebuf, const double *x,
                      const double *y, const double *z, int64_t n, int count_clamp, double *out,
                      int64_t *nclamp, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (comp < 0 || comp > 2) return fail(g, SLC_E_INVALID, "comp must be 0 (u), 1 (v) or 2 (w)");
    if (order != 2 && order != 4 && order != 6) return fail(g, SLC_E_INVALID, "order must be 2, 4 or 6");
    const int NZ = comp == 2 ? g->P.nz + 1 : g->P.nz + 2;
    if (NZ < order) return fail(g, SLC_E_INVALID, "grid too small for this order");
    if (n < 0 || (n > 0 && (!nodebuf || !x || !y || !z || !out)))
        return fail(g, SLC_E_INVALID, "bad interp arguments");
    if (count_clamp && !nclamp) return fail(g, SLC_E_INVALID, "count_clamp needs a counter");
    DeviceGuard dg(g->device);
    SLC_CK(launch_interp(g->P, comp, order, nodebuf, x, y, z, n, count_clamp, out,
                         (unsigned long long *)nclamp, S(stream)),
           "interp");
    return SLC_OK;
}

int slc_departure(slc_grid *g, int comp, const double *mid_u, const double *mid_v,
                  const double *mid_w, double dt, double *xd, double *yd, double *zd, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (comp < 0 || comp > 2) return fail(g, SLC_E_INVALID, "comp must be 0 (u), 1 (v) or 2 (w)");
    if (!mid_u || !mid_v || !mid_w || !xd || !yd || !zd) return fail(g, SLC_E_INVALID, "null pointer");
    DeviceGuard dg(g->device);
    SLC_CK(launch_departure(g->P, comp, Tri{mid_u, mid_v, mid_w}, dt, xd, yd, zd, S(stream)),
           "departure");
    return SLC_OK;
}

int slc_advect(slc_grid *g, const double *fu, const double *fv, const double *fw,
               const double *mid_u, const double *mid_v, const double *mid_w, double dt,
               double *ou, double *ov, double *ow, int64_t *nclamp, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!fu || !fv || !fw || !mid_u || !mid_v || !mid_w || !ou || !ov || !ow)
        return fail(g, SLC_E_INVALID, "null pointer");
    DeviceGuard dg(g->device);
    unsigned long long *ncl = counter(g, nclamp);
    cudaStream_t s = S(stream);
    SLC_CK(cudaMemsetAsync(ncl, 0, sizeof(unsigned long long), s), "memset");
    if (g->mixed) {
        int rc = ensure_mixed(g);
        if (rc) return rc;
        SLC_CK(launch_mixed_prepare(g->P, Tri{fu, fv, fw}, Tri{fu, fv, fw}, Tri{mid_u, mid_v, mid_w},
                                    g->mws, s),
               "mixed-form pack");
        long t = tim_begin(g, SLC_PHASE_SL, s);
        SLC_CK(launch_sl_mixed(g->P, 0, Tri{fu, fv, fw}, Tri{fu, fv, fw}, g->mws, dt,
                               TriMut{ou, ov, ow}, ncl, s),
               "mixed advect");
        tim_end(g, t, s);
        return SLC_OK;
    }
    long t = tim_begin(g, SLC_PHASE_SL, s);
    SLC_CK(launch_sl(g->P, 0, Tri{fu, fv, fw}, Tri{fu, fv, fw}, Tri{mid_u, mid_v, mid_w}, false, dt,
                     TriMut{ou, ov, ow}, ncl, s),
           "advect");
    tim_end(g, t, s);
    return SLC_OK;
}

int slc_advect_extra(slc_grid *g, const double *fu, const double *fv, const double *fw,
                     const double *mid_u, const double *mid_v, const double *mid_w, double dt,
                     double *ou, double *ov, double *ow, int n_extra,
                     const double *const *extra_in, double *const *extra_out, int64_t *nclamp,
                     void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!fu || !fv || !fw || !mid_u || !mid_v || !mid_w || !ou || !ov || !ow)
        return fail(g, SLC_E_INVALID, "null pointer");
    if (n_extra < 0 || n_extra > SLC_MAX_EXTRA)
        return fail(g, SLC_E_INVALID, "n_extra must be in [0, " + std::to_string(SLC_MAX_EXTRA) + "]");
    if (n_extra > 0 && (!extra_in || !extra_out)) return fail(g, SLC_E_INVALID, "null extra arrays");
    for (int q = 0; q < 3 * n_extra; ++q)
        if (!extra_in[q] || !extra_out[q]) return fail(g, SLC_E_INVALID, "null extra field pointer");
    DeviceGuard dg(g->device);
    const SlcParams &P = g->P;
    unsigned long long *ncl = counter(g, nclamp);
    cudaStream_t s = S(stream);
    SLC_CK(cudaMemsetAsync(ncl, 0, sizeof(unsigned long long), s), "memset");
    // the extras' arrival-shaped (nx, ny, nzi) outputs, z fastest
    OutMap arr[3];
    for (int c = 0; c < 3; ++c) {
        const long long nzi = c == 2 ? P.nz - 1 : P.nz;
        arr[c] = OutMap{0, (long long)P.ny * nzi, nzi};
    }
    long t = tim_begin(g, SLC_PHASE_SL, s);
    if (g->mixed) {
        // the mixed form packs each triple's FP32 fluctuations in turn; every
        // pack uses the same trajectory velocity, so every triple is gathered
        // at the same FP32-traced feet
        int rc = ensure_mixed(g);
        if (rc) return rc;
        const Tri mid{mid_u, mid_v, mid_w};
        SLC_CK(launch_mixed_prepare(P, Tri{fu, fv, fw}, Tri{fu, fv, fw}, mid, g->mws, s), "mixed-form pack");
        SLC_CK(launch_sl_mixed(P, 0, Tri{fu, fv, fw}, Tri{fu, fv, fw}, g->mws, dt, TriMut{ou, ov, ow},
                               ncl, s),
               "mixed advect");
        for (int e = 0; e < n_extra; ++e) {
            const Tri f{extra_in[3 * e], extra_in[3 * e + 1], extra_in[3 * e + 2]};
            SLC_CK(launch_mixed_prepare(P, f, f, mid, g->mws, s), "mixed-form pack");
            SLC_CK(launch_sl_mixed(P, 0, f, f, g->mws, dt,
                                   TriMut{extra_out[3 * e], extra_out[3 * e + 1], extra_out[3 * e + 2]},
                                   g->ncl_scratch, s, arr),
                   "mixed advect (extra field)");
        }
        tim_end(g, t, s);
        return SLC_OK;
    }
    // FP64: one trace per arrival point for up to kMaxMultiFields fields; the
    // first launch carries the advected triple and counts the clamps
    const double *in[3 * kMaxMultiFields];
    double *out[3 * kMaxMultiFields];
    OutMap maps[3 * kMaxMultiFields];
    const Tri mid{mid_u, mid_v, mid_w};
    int e = 0;
    bool first = true;
    while (first || e < n_extra) {
        int nf = 0;
        if (first) {
            const double *f0[3] = {fu, fv, fw};
            double *o0[3] = {ou, ov, ow};
            for (int c = 0; c < 3; ++c) {
                in[c] = f0[c];
                out[c] = o0[c];
                maps[c] = OutMap{0, 0, 0};
            }
            nf = 1;
        }
        for (; nf < kMaxMultiFields && e < n_extra; ++nf, ++e)
            for (int c = 0; c < 3; ++c) {
                in[3 * nf + c] = extra_in[3 * e + c];
                out[3 * nf + c] = extra_out[3 * e + c];
                maps[3 * nf + c] = arr[c];
            }
        SLC_CK(launch_advect_multi(P, nf, in, out, maps, mid, dt, first ? ncl : nullptr, s),
               "advect with extra fields");
        first = false;
    }
    tim_end(g, t, s);
    return SLC_OK;
}

int slc_trace_gather_bdf2(slc_grid *g, const double *un, const double *vn, const double *wn,
                          const double *unm1, const double *vnm1, const double *wnm1, double dt,
                          double *ou, double *ov, double *ow, int64_t *nclamp, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!un || !vn || !wn || !unm1 || !vnm1 || !wnm1 || !ou || !ov || !ow)
        return fail(g, SLC_E_INVALID, "null pointer");
    DeviceGuard dg(g->device);
    const double *cur[3] = {un, vn, wn}, *prev[3] = {unm1, vnm1, wnm1};
    double *out[3] = {ou, ov, ow};
    return do_trace_gather_bdf2(g, cur, prev, dt, out, nclamp, S(stream), kGatherL1);
}

int slc_trace_gather_bdf2_staged(slc_grid *g, const double *un, const double *vn, const double *wn,
                                 const double *unm1, const double *vnm1, const double *wnm1,
                                 double dt, double *ou, double *ov, double *ow, int64_t *nclamp,
                                 void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!un || !vn || !wn || !unm1 || !vnm1 || !wnm1 || !ou || !ov || !ow)
        return fail(g, SLC_E_INVALID, "null pointer");
    DeviceGuard dg(g->device);
    const double *cur[3] = {un, vn, wn}, *prev[3] = {unm1, vnm1, wnm1};
    double *out[3] = {ou, ov, ow};
    cudaStream_t s = S(stream);
    // time-outs of the bounded mbarrier waits (counter 0), before and after
    unsigned long long before = 0, after = 0;
    SLC_CK(cudaStreamSynchronize(s), "staged gather: synchronise");
    if (g->dev_flags)
        SLC_CK(cudaMemcpy(&before, g->dev_flags, sizeof(before), cudaMemcpyDeviceToHost), "read stats");
    int rc = do_trace_gather_bdf2(g, cur, prev, dt, out, nclamp, s, kGatherStaged);
    if (rc) return rc;
    SLC_CK(cudaStreamSynchronize(s), "staged gather: synchronise");
    if (g->dev_flags)
        SLC_CK(cudaMemcpy(&after, g->dev_flags, sizeof(after), cudaMemcpyDeviceToHost), "read stats");
    if (after != before)
        return fail(g, SLC_E_CUDA,
                    "staged gather: " + std::to_string(after - before) +
                        " bulk copies did not complete within the bounded waits");
    return SLC_OK;
}

int slc_zsolve(slc_grid *g, double *u, double *v, double *w, double dt, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!u || !v || !w) return fail(g, SLC_E_INVALID, "null pointer");
    DeviceGuard dg(g->device);
    return do_zsolve(g, u, v, w, dt, S(stream));
}

int slc_divergence(slc_grid *g, const double *u, const double *v, const double *w, double *div,
                   void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!u || !v || !w || !div) return fail(g, SLC_E_INVALID, "null pointer");
    DeviceGuard dg(g->device);
    SLC_CK(launch_divergence(g->P, Tri{u, v, w}, g->dzf, div, S(stream)), "divergence");
    return SLC_OK;
}

int slc_project(slc_grid *g, double *u, double *v, double *w, double *p, double dt_div,
                double dt_proj, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!u || !v || !w || !p) return fail(g, SLC_E_INVALID, "null pointer");
    if (!(dt_div != 0.0)) return fail(g, SLC_E_INVALID, "dt_div must be nonzero");
    DeviceGuard dg(g->device);
    return do_project(g, u, v, w, p, dt_div, dt_proj, S(stream));
}

int slc_bulk_velocity(slc_grid *g, const double *u, double *out, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!u || !out) return fail(g, SLC_E_INVALID, "null pointer");
    DeviceGuard dg(g->device);
    cudaStream_t s = S(stream);
    SLC_CK(launch_bulk_partials(g->P, (double *)u, g->dzf, nullptr, g->partials, s), "bulk");
    SLC_CK(launch_bulk_finish(g->P, g->partials, g->Lx, g->Ly, 0.0, 1.0, out, nullptr, s), "bulk");
    return SLC_OK;
}

int slc_divergence_raw(int nx, int ny, int nz, double dx, double dy, const double *dz_f,
                       const double *u, const double *v, const double *w, double *div,
                       void *stream)
{
    slc_grid *g = nullptr;
    if (nx < 1 || ny < 1 || nz < 1 || !dz_f || !u || !v || !w || !div)
        return fail(g, SLC_E_INVALID, "bad divergence arguments");
    SlcParams P{};
    P.nx = nx;
    P.ny = ny;
    P.nz = nz;
    P.dx = dx;
    P.dy = dy;
    P.inv_dx = 1.0 / dx;
    P.inv_dy = 1.0 / dy;
    SLC_CK(launch_divergence(P, Tri{u, v, w}, dz_f, div, S(stream)), "divergence");
    return SLC_OK;
}

int slc_bulk_scratch_doubles(void) { return kBulkBlocks; }

int slc_bulk_velocity_raw(int nx, int ny, int nz, const double *u, const double *vol_k,
                          double inv_volume, double *scratch, double *out, void *stream)
{
    slc_grid *g = nullptr;
    if (nx < 1 || ny < 1 || nz < 1 || !u || !vol_k || !scratch || !out)
        return fail(g, SLC_E_INVALID, "bad bulk-velocity arguments");
    SlcParams P{};
    P.nx = nx;
    P.ny = ny;
    P.nz = nz;
    P.dx = 1.0;
    P.dy = 1.0;
    P.Lz = 1.0;
    cudaStream_t s = S(stream);
    SLC_CK(launch_bulk_partials(P, (double *)u, vol_k, nullptr, scratch, s), "bulk");
    // dx*dy/(Lx*Ly*Lz) with dx = dy = Lz = 1 and Lx*Ly = 1/inv_volume
    SLC_CK(launch_bulk_finish(P, scratch, 1.0 / inv_volume, 1.0, 0.0, 1.0, out, nullptr, s), "bulk");
    return SLC_OK;
}

int slc_bulk_shift(slc_grid *g, double *u, double *v, double *w, double U_bulk, double dt,
                   double *out2, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!u || !v || !w || !out2) return fail(g, SLC_E_INVALID, "null pointer");
    if (!(dt != 0.0)) return fail(g, SLC_E_INVALID, "dt must be nonzero");
    DeviceGuard dg(g->device);
    cudaStream_t s = S(stream);
    long t = tim_begin(g, SLC_PHASE_BULK, s);
    SLC_CK(launch_bulk_partials(g->P, u, g->dzf, nullptr, g->partials, s), "bulk");
    SLC_CK(launch_bulk_finish(g->P, g->partials, g->Lx, g->Ly, U_bulk, dt, nullptr, g->scal, s),
           "bulk");
    SLC_CK(launch_bulk_partials(g->P, u, g->dzf, g->scal, g->partials, s), "bulk shift");
    SLC_CK(launch_apply_bc(g->P, u, v, w, nullptr, s), "boundary conditions");
    SLC_CK(launch_bulk_finish(g->P, g->partials, g->Lx, g->Ly, 0.0, 1.0, out2, nullptr, s), "bulk");
    SLC_CK(cudaMemcpyAsync(out2 + 1, g->scal + 1, sizeof(double), cudaMemcpyDeviceToDevice, s),
           "copy forcing");
    tim_end(g, t, s);
    return SLC_OK;
}

int slc_step_bdf1(slc_grid *g, double *const cur[3], double *const next[3], double *p, double dt,
                  int64_t *nclamp, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!cur || !next || !p) return fail(g, SLC_E_INVALID, "null pointer");
    for (int c = 0; c < 3; ++c)
        if (!cur[c] || !next[c]) return fail(g, SLC_E_INVALID, "null field pointer");
    if (!(dt > 0.0)) return fail(g, SLC_E_INVALID, "dt must be positive");
    DeviceGuard dg(g->device);
    cudaStream_t s = S(stream);
    int rc = do_apply_bc(g, cur[0], cur[1], cur[2], s);
    if (rc) return rc;
    unsigned long long *ncl = counter(g, nclamp);
    SLC_CK(cudaMemsetAsync(ncl, 0, sizeof(unsigned long long), s), "memset");
    Tri c3{cur[0], cur[1], cur[2]};
    if (g->mixed) {
        rc = ensure_mixed(g);
        if (rc) return rc;
        long tm = tim_begin(g, SLC_PHASE_MID, s);
        SLC_CK(launch_mixed_prepare(g->P, c3, c3, Tri{nullptr, nullptr, nullptr}, g->mws, s),
               "mixed-form pack");
        tim_end(g, tm, s);
    }
    long t = tim_begin(g, SLC_PHASE_SL, s);
    if (g->mixed)
        SLC_CK(launch_sl_mixed(g->P, 1, c3, c3, g->mws, dt, TriMut{next[0], next[1], next[2]}, ncl, s),
               "mixed trace+gather BDF1");
    else
        SLC_CK(launch_sl(g->P, 1, c3, c3, c3, false, dt, TriMut{next[0], next[1], next[2]}, ncl, s),
               "trace+gather BDF1");
    tim_end(g, t, s);
    rc = do_zsolve(g, next[0], next[1], next[2], dt, s);
    if (rc) return rc;
    return do_project(g, next[0], next[1], next[2], p, dt, dt, s);
}

int slc_step_bdf2(slc_grid *g, double *const cur[3], double *const prev[3], double *const next[3],
                  double *p, double dt, int64_t *nclamp, void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!cur || !prev || !next || !p) return fail(g, SLC_E_INVALID, "null pointer");
    for (int c = 0; c < 3; ++c)
        if (!cur[c] || !prev[c] || !next[c]) return fail(g, SLC_E_INVALID, "null field pointer");
    if (!(dt > 0.0)) return fail(g, SLC_E_INVALID, "dt must be positive");
    DeviceGuard dg(g->device);
    cudaStream_t s = S(stream);
    int rc = do_apply_bc(g, cur[0], cur[1], cur[2], s);
    if (rc) return rc;
    rc = do_trace_gather_bdf2(g, cur, prev, dt, next, nclamp, s);
    if (rc) return rc;
    return slc_step_bdf2_tail(g, next, p, dt, s);
}

int slc_gather_stats(slc_grid *g, int64_t *out4, int reset)
{
    if (!g || !out4) return fail(g, SLC_E_INVALID, "null argument");
    DeviceGuard dg(g->device);
    unsigned long long h[4];
    SLC_CK(cudaMemcpy(h, g->dev_flags, sizeof(h), cudaMemcpyDeviceToHost), "read gather stats");
    for (int q = 0; q < 4; ++q) out4[q] = (int64_t)h[q];
    if (reset) SLC_CK(cudaMemset(g->dev_flags, 0, sizeof(h)), "reset gather stats");
    return SLC_OK;
}

int slc_step_bdf2_inc(slc_grid *g, double *const cur[3], double *const prev[3], double *const next[3],
                      double *p_cur, double *p_prev, int have_prev, double dt, int64_t *nclamp,
                      void *stream)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    if (!cur || !prev || !next || !p_cur || !p_prev) return fail(g, SLC_E_INVALID, "null pointer");
    for (int c = 0; c < 3; ++c)
        if (!cur[c] || !prev[c] || !next[c]) return fail(g, SLC_E_INVALID, "null field pointer");
    if (!(dt > 0.0)) return fail(g, SLC_E_INVALID, "dt must be positive");
    DeviceGuard dg(g->device);
    cudaStream_t s = S(stream);
    const size_t np = g->ghost_elems[3];
    if (!g->p_ext) {
        int rc = dalloc(g, &g->p_ext, np, "extrapolated pressure");
        if (!rc) rc = dalloc(g, &g->phi, np, "pressure increment");
        if (rc) return rc;
    }
    int rc = do_apply_bc(g, cur[0], cur[1], cur[2], s);
    if (rc) return rc;
    rc = do_trace_gather_bdf2(g, cur, prev, dt, next, nclamp, s);
    if (rc) return rc;
    const double dt_eff = (2.0 / 3.0) * dt;
    // p_ext = 2 p^n - p^{n-1}, or p^n on the first BDF2 step after a bootstrap
    if (have_prev)
        SLC_CK(launch_lincomb(p_cur, p_prev, 2.0, -1.0, g->p_ext, (int64_t)np, s), "p_ext");
    else
        SLC_CK(cudaMemcpyAsync(g->p_ext, p_cur, np * sizeof(double), cudaMemcpyDeviceToDevice, s), "p_ext");
    SLC_CK(launch_grad_sub(g->P, g->p_ext, TriMut{next[0], next[1], next[2]}, g->dzc, dt_eff, s),
           "predictor pressure gradient");
    rc = do_zsolve(g, next[0], next[1], next[2], dt_eff, s);
    if (!rc) rc = do_project(g, next[0], next[1], next[2], g->phi, dt_eff, dt_eff, s);
    if (rc) return rc;
    // p^{n-1} <- p^n, p^{n+1} = p_ext + phi (solver.py:1001-1012)
    SLC_CK(cudaMemcpyAsync(p_prev, p_cur, np * sizeof(double), cudaMemcpyDeviceToDevice, s), "p history");
    SLC_CK(launch_lincomb(g->p_ext, g->phi, 1.0, 1.0, p_cur, (int64_t)np, s), "p update");
    return SLC_OK;
}

int slc_timing(slc_grid *g, int enable)
{
    if (!g) return fail(nullptr, SLC_E_INVALID, "null handle");
    g->timing = enable != 0;
    g->ev_used = 0;
    return SLC_OK;
}

int slc_timing_read(slc_grid *g, double *ms, int64_t *count)
{
    if (!g || !ms || !count) return fail(g, SLC_E_INVALID, "null argument");
    DeviceGuard dg(g->device);
    for (int p = 0; p < SLC_NPHASE; ++p) {
        ms[p] = 0.0;
        count[p] = 0;
    }
    for (size_t i = 0; i < g->ev_used; ++i) {
        SLC_CK(cudaEventSynchronize(g->evs[2 * i + 1]), "event synchronize");
        float t = 0.f;
        SLC_CK(cudaEventElapsedTime(&t, g->evs[2 * i], g->evs[2 * i + 1]), "event elapsed");
        const int p = g->ev_phase[i];
        if (p >= 0 && p < SLC_NPHASE) {
            ms[p] += (double)t;
            count[p] += 1;
        }
    }
    g->ev_used = 0;
    return SLC_OK;
}

int64_t slc_kernel_launches(void) { return (int64_t)g_slc_launches.load(); }

}  // extern "C"
