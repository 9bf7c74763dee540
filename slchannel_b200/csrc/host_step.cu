// host_step.cu -- the SL-BDF2 step for callers whose state lives in pinned
// HOST memory (slc_step_bdf2_host).
//
// Every call uploads that step's V^n and V^{n-1}, runs the step with its bulk
// shift on the device, and downloads V^{n+1}, p and (u_bulk, forcing).  The
// transfers are overlapped with each other and with compute:
//  * two copy streams (host-to-device, device-to-host) run concurrently with
//    the internal compute streams.  The caller's stream ends each call
//    waiting for that call's downloads; the next call's compute starts when
//    its inputs are on the device, not when the previous call's p has
//    reached the host;
//  * the device state is double-buffered across calls, so the next call's
//    uploads proceed while this call computes;
//  * copies are cut into pieces with one event each.  An upload whose host
//    source is a range an earlier call is still downloading into waits for
//    the overlapping pieces only, so a caller that feeds each step's V^{n+1}
//    back as the next V^n pipelines the round trip piece by piece.  A
//    download into a host range an earlier upload still reads waits for it;
//  * FP64 handles with nx >= 96 stream the step by x slab.  V^n and V^{n+1}
//    move in slab pieces, the last slab first.  As a slab of V^n lands, its
//    ghosts and its U* = 2 V^n - V^{n-1} are formed, and a slab's BDF2
//    trace+gather starts as soon as the slabs on both sides of it are on the
//    device, provided its feet provably stay within them (SlabGate in
//    slc_internal.h; a slab that fails the check is recomputed once all of
//    V^n is there).  The step's compute then overlaps the V^{n+1} -> host ->
//    V^n round trip instead of waiting for all of it, and the results are
//    those of slc_step_bdf2 (same per-point arithmetic, same U* and ghosts).
// Host buffers must stay untouched until the caller's stream is synchronised.
#include <algorithm>
#include <string>
#include <vector>

#include "slc_bc.cuh"
#include "slc_grid.h"

namespace {

constexpr size_t kChunkBytes = (size_t)16 << 20;
#ifndef SLC_SLAB_NODES
#define SLC_SLAB_NODES 32
#endif
constexpr int kSlabNodes = SLC_SLAB_NODES;  // target slab width in x nodes
constexpr int kSlabMargin = 8;  // nodes of a slab's neighbours kept for stencils and staggering

struct Piece {
    const char *lo, *hi;  // host byte range
    cudaEvent_t ev;       // recorded after the piece's copy
};

// Rows of one prep launch: per component up to two ranges of x planes of
// the ghost-shaped arrays.
struct PrepJob {
    double *cur[3];
    const double *prev[3];
    double *mid[3];
    int nr[3];
    int lo[3][2], hi[3][2];
};

// Slabs of the x nodes; S = 0 when the step is not streamed (fewer than
// three slabs of kSlabNodes).
SlabBounds slab_plan(const SlcParams &P)
{
    SlabBounds sb{};
    const int S = std::min(kMaxSlabs, P.nx / kSlabNodes);
    if (S < 3) return sb;
    sb.S = S;
    for (int s = 0; s <= S; ++s) sb.b[s] = (int)((long long)s * P.nx / S);
    return sb;
}

// x planes [lo, hi) of component c's ghost-shaped array that carry slab s:
// its nodes, plus the x-ghost planes for the first and last slab.
void slab_planes(const SlabBounds &sb, int c, int nx, int s, int &lo, int &hi)
{
    const int ox = c == 0 ? 0 : 1;  // plane of x node 0
    const int X = c == 0 ? nx + 1 : nx + 2;
    lo = s == 0 ? 0 : sb.b[s] + ox;
    hi = s == sb.S - 1 ? X : sb.b[s + 1] + ox;
}

// Slab s's planes without the x-ghost planes (those are filled by the ghost
// job once their interior sources, in the first and last slab, are there).
void slab_interior_planes(const SlabBounds &sb, int c, int nx, int s, int &lo, int &hi)
{
    slab_planes(sb, c, nx, s, lo, hi);
    if (s == 0) lo = 1;
    if (s == sb.S - 1 && c != 0) hi = nx + 1;
}

// Arrival order of the slabs: the last first, then 0, 1, ..., S-2, so slab
// 0's left neighbour (the periodic image) is there before slab 1.
int slab_order(int S, int idx) { return idx == 0 ? S - 1 : idx - 1; }

// Ghosts (from their interior sources) and U* = 2 V^n - V^{n-1} on the rows
// of the job, and max |U*_u| into gate->umax.  One warp per (x, y) row,
// lanes along z.  Only ghost elements of cur are written, and every source
// is an interior element, so the threads never read what another writes.
__global__ void __launch_bounds__(256) k_slab_prep(SlcParams P, PrepJob job, SlabGate *gate)
{
    const int c = blockIdx.y;
    const GhostShape g = ghost_shape(c, P.nx, P.ny, P.nz);
    const int span0 = job.nr[c] > 0 ? (job.hi[c][0] - job.lo[c][0]) * g.Y : 0;
    const int span1 = job.nr[c] > 1 ? (job.hi[c][1] - job.lo[c][1]) * g.Y : 0;
    double *cur = job.cur[c];
    const double *prev = job.prev[c];
    double *mid = job.mid[c];
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    unsigned long long um = 0;
    for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < span0 + span1;
         row += gridDim.x * warps) {
        const int r = row < span0 ? row : row - span0;
        const int I = (row < span0 ? job.lo[c][0] : job.lo[c][1]) + r / g.Y;
        const int J = r % g.Y;
        const size_t base = ((size_t)I * g.Y + J) * g.Z;
        for (int K = lane; K < g.Z; K += 32) {
            double a;
            if (bc_is_ghost(c, P.nx, P.ny, P.nz, I, J, K)) {
                const BcSrc s = bc_src(c, P.nx, P.ny, P.nz, P.top_neumann, I, J, K);
                a = s.zero ? 0.0 : s.sign * cur[((size_t)s.Is * g.Y + s.Js) * g.Z + s.Ks];
                cur[base + K] = a;
            } else {
                a = cur[base + K];
            }
            const double m = 2.0 * a + (-1.0) * prev[base + K];  // k_lincomb's U*, exactly
            mid[base + K] = m;
            if (c == 0) um = max(um, (unsigned long long)__double_as_longlong(fabs(m)));
        }
    }
    if (c != 0) return;
    __shared__ unsigned long long wmax[8];
    for (int o = 16; o > 0; o >>= 1) um = max(um, __shfl_xor_sync(0xffffffffu, um, o));
    if (lane == 0) wmax[threadIdx.x >> 5] = um;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < warps; ++w) um = max(um, wmax[w]);
        atomicMax(&gate->umax, um);
    }
}

}  // namespace

struct HostStep {
    int device = 0;
    cudaStream_t h2d = nullptr, d2h = nullptr, comp = nullptr;
    cudaStream_t sl[3] = {nullptr, nullptr, nullptr};  // slab trace+gather, one per component
    cudaEvent_t entry = nullptr;  // the caller's stream at the first call
    bool started = false;
    double *dev[2][10] = {};  // set -> cur(3), prev(3), next(3), p
    double *scal2[2] = {nullptr, nullptr};
    cudaEvent_t inputs_ready[2] = {}, compute_done[2] = {}, set_free[2] = {};
    bool set_used[2] = {false, false};
    int set = 0;
    // pieces of the previous call ([0]) and of the call before it ([1])
    std::vector<Piece> downloads[2], uploads[2];
    // piece events, one pool per call modulo 3: the two previous calls'
    // events stay untouched while this call still waits on them
    std::vector<cudaEvent_t> pool[3];
    size_t pool_used = 0;
    int gen = 0;
    // the streamed step
    SlabGate *gate = nullptr;
    cudaEvent_t prev_ready = nullptr, slab_ready[kMaxSlabs] = {}, released[kMaxSlabs] = {};
    cudaEvent_t sl_done[3] = {};
    long long n_streamed = 0, n_plain = 0;
    int last_S = 0;
};

namespace {

int hfail(slc_grid *g, int code, const std::string &m)
{
    g->err = m;
    return code;
}

#define HS_CK(call, what)                                                                       \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) return hfail(g, SLC_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
    } while (0)

cudaEvent_t next_event(HostStep *h)
{
    std::vector<cudaEvent_t> &pool = h->pool[h->gen];
    if (h->pool_used == pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
        pool.push_back(e);
    }
    return pool[h->pool_used++];
}

// Make stream s wait for every piece of `pend` that touches host range [lo, hi).
int wait_overlapping(slc_grid *g, const std::vector<Piece> &pend, const char *lo, const char *hi,
                     cudaStream_t s)
{
    for (const Piece &p : pend)
        if (lo < p.hi && p.lo < hi) HS_CK(cudaStreamWaitEvent(s, p.ev, 0), "wait piece");
    return SLC_OK;
}

int ensure_host_step(slc_grid *g)
{
    if (g->host) return SLC_OK;
    HostStep *h = new HostStep();
    h->device = g->device;
    g->host = h;
    HS_CK(cudaStreamCreateWithFlags(&h->h2d, cudaStreamNonBlocking), "copy stream");
    HS_CK(cudaStreamCreateWithFlags(&h->d2h, cudaStreamNonBlocking), "copy stream");
    HS_CK(cudaStreamCreateWithFlags(&h->comp, cudaStreamNonBlocking), "compute stream");
    for (int c = 0; c < 3; ++c) {
        HS_CK(cudaStreamCreateWithFlags(&h->sl[c], cudaStreamNonBlocking), "slab stream");
        HS_CK(cudaEventCreateWithFlags(&h->sl_done[c], cudaEventDisableTiming), "event");
    }
    HS_CK(cudaEventCreateWithFlags(&h->entry, cudaEventDisableTiming), "event");
    HS_CK(cudaEventCreateWithFlags(&h->prev_ready, cudaEventDisableTiming), "event");
    for (int s = 0; s < kMaxSlabs; ++s) {
        HS_CK(cudaEventCreateWithFlags(&h->slab_ready[s], cudaEventDisableTiming), "event");
        HS_CK(cudaEventCreateWithFlags(&h->released[s], cudaEventDisableTiming), "event");
    }
    for (int s = 0; s < 2; ++s) {
        for (int q = 0; q < 10; ++q) {
            const size_t n = q == 9 ? g->ghost_elems[3] : g->ghost_elems[q % 3];
            void *p = nullptr;
            HS_CK(cudaMalloc(&p, n * sizeof(double)), "host-step device state");
            g->allocs.push_back(p);
            HS_CK(cudaMemset(p, 0, n * sizeof(double)), "memset");
            h->dev[s][q] = (double *)p;
        }
        void *p = nullptr;
        HS_CK(cudaMalloc(&p, 2 * sizeof(double)), "host-step scalars");
        g->allocs.push_back(p);
        h->scal2[s] = (double *)p;
        HS_CK(cudaEventCreateWithFlags(&h->inputs_ready[s], cudaEventDisableTiming), "event");
        HS_CK(cudaEventCreateWithFlags(&h->compute_done[s], cudaEventDisableTiming), "event");
        HS_CK(cudaEventCreateWithFlags(&h->set_free[s], cudaEventDisableTiming), "event");
    }
    void *p = nullptr;
    HS_CK(cudaMalloc(&p, sizeof(SlabGate)), "slab gate");
    g->allocs.push_back(p);
    h->gate = (SlabGate *)p;
    return SLC_OK;
}

int launch_prep(slc_grid *g, const PrepJob &job, SlabGate *gate, cudaStream_t s)
{
    int rows = 0;
    for (int c = 0; c < 3; ++c) {
        const GhostShape gs = ghost_shape(c, g->P.nx, g->P.ny, g->P.nz);
        int r = 0;
        for (int q = 0; q < job.nr[c]; ++q) r += (job.hi[c][q] - job.lo[c][q]) * gs.Y;
        rows = std::max(rows, r);
    }
    if (rows == 0) return SLC_OK;
    const unsigned bx = (unsigned)std::min((rows + 7) / 8, 148 * 8);
    k_slab_prep<<<dim3(bx, 3), 256, 0, s>>>(g->P, job, gate);
    count_launches(1);
    HS_CK(cudaGetLastError(), "slab prep");
    return SLC_OK;
}

// The BDF2 step of this call's device set D, streamed by x slab (see the
// file comment).  The V^n slab uploads record slab_ready[s]; V^{n-1} is
// whole when prev_ready is.
int streamed_step(slc_grid *g, HostStep *h, const SlabBounds &sb, double *const *D, double dt)
{
    const SlcParams &P = g->P;
    cudaStream_t cs = h->comp;
    const int S = sb.S;
    int wmin = P.nx;
    for (int s = 0; s < S; ++s) wmin = std::min(wmin, sb.b[s + 1] - sb.b[s]);
    const double limit = (double)(wmin - kSlabMargin);
    const int ncomp = P.nz > 1 ? 3 : 2;
    unsigned long long *ncl = g->ncl_scratch;
    const Tri mid{g->mid[0], g->mid[1], g->mid[2]};
    HS_CK(cudaStreamWaitEvent(cs, h->prev_ready, 0), "wait V^{n-1}");
    HS_CK(cudaMemsetAsync(h->gate, 0, sizeof(SlabGate), cs), "memset");
    HS_CK(cudaMemsetAsync(ncl, 0, sizeof(unsigned long long), cs), "memset");

    PrepJob job{};
    for (int c = 0; c < 3; ++c) {
        job.cur[c] = D[c];
        job.prev[c] = D[3 + c];
        job.mid[c] = g->mid[c];
    }
    // slab s's neighbours are prepared: its launches may run
    auto release = [&](int s) -> int {
        HS_CK(cudaMemcpyAsync(&h->gate->snap[s], &h->gate->umax, sizeof(unsigned long long),
                              cudaMemcpyDeviceToDevice, cs),
              "gate snapshot");
        HS_CK(cudaEventRecord(h->released[s], cs), "record");
        for (int c = 0; c < ncomp; ++c) {
            HS_CK(cudaStreamWaitEvent(h->sl[c], h->released[s], 0), "wait release");
            HS_CK(launch_sl_slab(P, c, D[c], D[3 + c], mid, dt, D[6 + c], ncl, h->gate, s, sb.b[s],
                                 sb.b[s + 1], limit, h->sl[c]),
                  "slab trace+gather BDF2");
        }
        return SLC_OK;
    };
    for (int idx = 0; idx < S; ++idx) {
        const int s = slab_order(S, idx);
        HS_CK(cudaStreamWaitEvent(cs, h->slab_ready[s], 0), "wait slab");
        for (int c = 0; c < 3; ++c) {
            job.nr[c] = 1;
            slab_interior_planes(sb, c, P.nx, s, job.lo[c][0], job.hi[c][0]);
        }
        int rc = launch_prep(g, job, h->gate, cs);
        if (rc) return rc;
        if (s == 0) {  // the x-ghost planes: their sources (planes nx and 1) are here now
            for (int c = 0; c < 3; ++c) {
                job.nr[c] = c == 0 ? 1 : 2;
                job.lo[c][0] = 0;
                job.hi[c][0] = 1;
                job.lo[c][1] = P.nx + 1;
                job.hi[c][1] = P.nx + 2;
            }
            rc = launch_prep(g, job, h->gate, cs);
            if (rc) return rc;
        }
        if (idx >= 2) {
            rc = release(s - 1);
            if (rc) return rc;
        }
    }
    int rc = release(S - 2);
    if (!rc) rc = release(S - 1);
    if (rc) return rc;
    for (int c = 0; c < ncomp; ++c) {
        HS_CK(cudaEventRecord(h->sl_done[c], h->sl[c]), "record");
        HS_CK(cudaStreamWaitEvent(cs, h->sl_done[c], 0), "join slab streams");
    }
    for (int c = 0; c < ncomp; ++c)
        HS_CK(launch_sl_fix(P, c, D[c], D[3 + c], mid, dt, D[6 + c], ncl, h->gate, sb, cs),
              "deferred slabs");
    double *n3[3] = {D[6], D[7], D[8]};
    return slc_step_bdf2_tail(g, n3, D[9], dt, cs);
}

}  // namespace

void host_step_free(HostStep *h)
{
    if (!h) return;
    if (h->h2d) cudaStreamDestroy(h->h2d);
    if (h->d2h) cudaStreamDestroy(h->d2h);
    if (h->comp) cudaStreamDestroy(h->comp);
    for (int c = 0; c < 3; ++c) {
        if (h->sl[c]) cudaStreamDestroy(h->sl[c]);
        if (h->sl_done[c]) cudaEventDestroy(h->sl_done[c]);
    }
    if (h->entry) cudaEventDestroy(h->entry);
    if (h->prev_ready) cudaEventDestroy(h->prev_ready);
    for (int s = 0; s < kMaxSlabs; ++s) {
        if (h->slab_ready[s]) cudaEventDestroy(h->slab_ready[s]);
        if (h->released[s]) cudaEventDestroy(h->released[s]);
    }
    for (int s = 0; s < 2; ++s) {
        if (h->inputs_ready[s]) cudaEventDestroy(h->inputs_ready[s]);
        if (h->compute_done[s]) cudaEventDestroy(h->compute_done[s]);
        if (h->set_free[s]) cudaEventDestroy(h->set_free[s]);
    }
    for (int q = 0; q < 3; ++q)
        for (cudaEvent_t e : h->pool[q]) cudaEventDestroy(e);
    delete h;
}

extern "C" int slc_step_bdf2(slc_grid *g, double *const cur[3], double *const prev[3],
                             double *const next[3], double *p, double dt, int64_t *nclamp,
                             void *stream);
extern "C" int slc_bulk_shift(slc_grid *g, double *u, double *v, double *w, double U_bulk, double dt,
                              double *out2, void *stream);

extern "C" int slc_step_bdf2_host(slc_grid *g, const double *const cur[3], const double *const prev[3],
                                  double *const next[3], double *p, double *bulk_out2, double U_bulk,
                                  double dt, void *stream)
{
    if (!g) return SLC_E_INVALID;
    if (!cur || !prev || !next || !p || !bulk_out2) return hfail(g, SLC_E_INVALID, "null pointer");
    for (int c = 0; c < 3; ++c)
        if (!cur[c] || !prev[c] || !next[c]) return hfail(g, SLC_E_INVALID, "null field pointer");
    if (!(dt > 0.0)) return hfail(g, SLC_E_INVALID, "dt must be positive");
    cudaSetDevice(g->device);
    int rc = ensure_host_step(g);
    if (!rc) rc = slc_grid_ensure_mid(g);
    if (rc) return rc;
    HostStep *h = g->host;
    cudaStream_t s = (cudaStream_t)stream;
    if (!h->started) {  // order the first call after the caller's earlier work on the handle
        HS_CK(cudaEventRecord(h->entry, s), "record");
        HS_CK(cudaStreamWaitEvent(h->comp, h->entry, 0), "wait caller");
        HS_CK(cudaStreamWaitEvent(h->h2d, h->entry, 0), "wait caller");
        h->started = true;
    }
    const int set = h->set;
    double *const *D = h->dev[set];
    h->gen = (h->gen + 1) % 3;  // this call's events: the pool of three calls ago
    h->pool_used = 0;
    const SlabBounds sb = g->mixed ? SlabBounds{} : slab_plan(g->P);
    const bool streamed = sb.S >= 3;
    std::vector<Piece> ups, downs;

    auto upload = [&](const void *src, double *dst, size_t off, size_t nb) -> int {
        const char *lo = (const char *)src + off;
        for (int q = 0; q < 2; ++q) {
            int r = wait_overlapping(g, h->downloads[q], lo, lo + nb, h->h2d);
            if (r) return r;
        }
        HS_CK(cudaMemcpyAsync((char *)dst + off, lo, nb, cudaMemcpyHostToDevice, h->h2d), "upload");
        cudaEvent_t e = next_event(h);
        if (!e) return hfail(g, SLC_E_CUDA, "event pool");
        HS_CK(cudaEventRecord(e, h->h2d), "record");
        ups.push_back(Piece{lo, lo + nb, e});
        return SLC_OK;
    };
    auto upload_chunked = [&](const void *src, double *dst, size_t bytes) -> int {
        for (size_t off = 0; off < bytes; off += kChunkBytes) {
            int r = upload(src, dst, off, std::min(kChunkBytes, bytes - off));
            if (r) return r;
        }
        return SLC_OK;
    };

    // the device set's inputs were last read by the compute of two calls ago
    if (h->set_used[set]) HS_CK(cudaStreamWaitEvent(h->h2d, h->compute_done[set], 0), "wait set");
    // uploads: V^{n-1} first (no dependency on the previous call), then V^n
    for (int c = 0; c < 3 && !rc; ++c)
        rc = upload_chunked(prev[c], D[3 + c], g->ghost_elems[c] * sizeof(double));
    if (rc) return rc;
    HS_CK(cudaEventRecord(h->prev_ready, h->h2d), "record");
    if (streamed) {
        for (int idx = 0; idx < sb.S; ++idx) {
            const int sl = slab_order(sb.S, idx);
            for (int c = 0; c < 3; ++c) {
                const GhostShape gs = ghost_shape(c, g->P.nx, g->P.ny, g->P.nz);
                const size_t plane = (size_t)gs.Y * gs.Z * sizeof(double);
                int lo, hi;
                slab_planes(sb, c, g->P.nx, sl, lo, hi);
                rc = upload(cur[c], D[c], lo * plane, (size_t)(hi - lo) * plane);
                if (rc) return rc;
            }
            HS_CK(cudaEventRecord(h->slab_ready[sl], h->h2d), "record");
        }
    } else {
        for (int c = 0; c < 3 && !rc; ++c) rc = upload_chunked(cur[c], D[c], g->ghost_elems[c] * sizeof(double));
        if (rc) return rc;
    }
    HS_CK(cudaEventRecord(h->inputs_ready[set], h->h2d), "record");

    // compute on the internal streams; next and p of this set were last read
    // by the downloads of two calls ago
    if (h->set_used[set]) HS_CK(cudaStreamWaitEvent(h->comp, h->set_free[set], 0), "wait set");
    if (streamed) {
        rc = streamed_step(g, h, sb, D, dt);
        h->n_streamed++;
    } else {
        HS_CK(cudaStreamWaitEvent(h->comp, h->inputs_ready[set], 0), "wait inputs");
        double *c3[3] = {D[0], D[1], D[2]}, *p3[3] = {D[3], D[4], D[5]}, *n3[3] = {D[6], D[7], D[8]};
        rc = slc_step_bdf2(g, c3, p3, n3, D[9], dt, nullptr, h->comp);
        h->n_plain++;
    }
    h->last_S = streamed ? sb.S : 0;
    if (!rc) rc = slc_bulk_shift(g, D[6], D[7], D[8], U_bulk, dt, h->scal2[set], h->comp);
    if (rc) return rc;
    HS_CK(cudaEventRecord(h->compute_done[set], h->comp), "record");

    // downloads: V^{n+1} (the next call's input, first, in the order the next
    // call uploads it), (u_bulk, forcing), then p; each after any upload
    // still reading its host range
    HS_CK(cudaStreamWaitEvent(h->d2h, h->compute_done[set], 0), "wait compute");
    auto download = [&](void *dst, const double *src, size_t off, size_t nb) -> int {
        char *lo = (char *)dst + off;
        for (int q = 0; q < 2; ++q) {
            int r = wait_overlapping(g, h->uploads[q], lo, lo + nb, h->d2h);
            if (r) return r;
        }
        int r = wait_overlapping(g, ups, lo, lo + nb, h->d2h);
        if (r) return r;
        HS_CK(cudaMemcpyAsync(lo, (const char *)src + off, nb, cudaMemcpyDeviceToHost, h->d2h), "download");
        cudaEvent_t e = next_event(h);
        if (!e) return hfail(g, SLC_E_CUDA, "event pool");
        HS_CK(cudaEventRecord(e, h->d2h), "record");
        downs.push_back(Piece{lo, lo + nb, e});
        return SLC_OK;
    };
    auto download_chunked = [&](void *dst, const double *src, size_t bytes) -> int {
        for (size_t off = 0; off < bytes; off += kChunkBytes) {
            int r = download(dst, src, off, std::min(kChunkBytes, bytes - off));
            if (r) return r;
        }
        return SLC_OK;
    };
    if (streamed) {
        for (int idx = 0; idx < sb.S && !rc; ++idx) {
            const int sl = slab_order(sb.S, idx);
            for (int c = 0; c < 3 && !rc; ++c) {
                const GhostShape gs = ghost_shape(c, g->P.nx, g->P.ny, g->P.nz);
                const size_t plane = (size_t)gs.Y * gs.Z * sizeof(double);
                int lo, hi;
                slab_planes(sb, c, g->P.nx, sl, lo, hi);
                rc = download(next[c], D[6 + c], lo * plane, (size_t)(hi - lo) * plane);
            }
        }
    } else {
        for (int c = 0; c < 3 && !rc; ++c)
            rc = download_chunked(next[c], D[6 + c], g->ghost_elems[c] * sizeof(double));
    }
    if (!rc) rc = download(bulk_out2, h->scal2[set], 0, 2 * sizeof(double));
    if (!rc) rc = download_chunked(p, D[9], g->ghost_elems[3] * sizeof(double));
    if (rc) return rc;
    HS_CK(cudaEventRecord(h->set_free[set], h->d2h), "record");
    h->set_used[set] = true;
    // the caller's stream completes when the results are on the host
    HS_CK(cudaStreamWaitEvent(s, h->set_free[set], 0), "wait downloads");
    h->uploads[1] = std::move(h->uploads[0]);
    h->uploads[0] = std::move(ups);
    h->downloads[1] = std::move(h->downloads[0]);
    h->downloads[0] = std::move(downs);
    h->set ^= 1;
    return SLC_OK;
}

extern "C" int slc_host_step_stats(slc_grid *g, int64_t *out4)
{
    if (!g || !out4) return SLC_E_INVALID;
    out4[0] = out4[1] = out4[2] = out4[3] = 0;
    HostStep *h = g->host;
    if (!h) return SLC_OK;
    cudaSetDevice(g->device);
    out4[0] = h->n_streamed;
    out4[1] = h->n_plain;
    out4[2] = h->last_S;
    if (h->last_S > 0) {
        HS_CK(cudaStreamSynchronize(h->comp), "synchronise");
        int def[kMaxSlabs];
        HS_CK(cudaMemcpy(def, h->gate->deferred, sizeof(def), cudaMemcpyDeviceToHost), "read gate");
        for (int s = 0; s < h->last_S; ++s) out4[3] += def[s] != 0;
    }
    return SLC_OK;
}
