// host_step.cu -- the SL-BDF2 step for callers whose state lives in pinned
// HOST memory (slc_step_bdf2_host).
//
// Every call uploads that step's V^n and V^{n-1}, runs the step with its bulk
// shift on the device, and downloads V^{n+1}, p and (u_bulk, forcing).  The
// transfers are overlapped with each other and with compute:
//  * two copy streams (host-to-device, device-to-host) run concurrently with
//    an internal compute stream.  Compute runs there rather than on the
//    caller's stream, which ends each call waiting for that call's downloads:
//    the next call's compute then starts when its inputs are on the device,
//    not when the previous call's p has reached the host;
//  * the device state is double-buffered across calls, so the next call's
//    uploads proceed while this call computes;
//  * copies are cut into chunks with one event each.  An upload whose host
//    source is a range an earlier call is still downloading into waits for
//    that chunk only, so a caller that feeds each step's V^{n+1} back as the
//    next V^n pipelines the round trip chunk by chunk.  A download into a
//    host range an earlier upload still reads waits for that upload.
// Host buffers must stay untouched until the caller's stream is synchronised.
#include <algorithm>
#include <string>
#include <vector>

#include "slc_grid.h"

namespace {

constexpr size_t kChunkBytes = (size_t)16 << 20;

struct Pending {
    const char *lo = nullptr, *hi = nullptr;  // host byte range
    std::vector<cudaEvent_t> ev;              // per chunk (event i covers chunk i)
    size_t chunk = kChunkBytes;
};

}  // namespace

struct HostStep {
    int device = 0;
    cudaStream_t h2d = nullptr, d2h = nullptr, comp = nullptr;
    cudaEvent_t entry = nullptr;  // the caller's stream at the first call
    bool started = false;
    double *dev[2][10] = {};  // set -> cur(3), prev(3), next(3), p
    double *scal2[2] = {nullptr, nullptr};
    cudaEvent_t inputs_ready[2] = {}, compute_done[2] = {}, set_free[2] = {};
    bool set_used[2] = {false, false};
    int set = 0;
    std::vector<Pending> downloads, uploads;  // of the previous call
    // chunk events, one pool per call parity: the previous call's events stay
    // untouched while this call still waits on them
    std::vector<cudaEvent_t> pool[2];
    size_t pool_used = 0;
    int parity = 0;
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
    std::vector<cudaEvent_t> &pool = h->pool[h->parity];
    if (h->pool_used == pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
        pool.push_back(e);
    }
    return pool[h->pool_used++];
}

bool overlaps(const Pending &p, const char *lo, const char *hi) { return lo < p.hi && p.lo < hi; }

// Make stream s wait for whatever of `pend` touches host range [lo, lo + bytes):
// chunk by chunk when the range is exactly a pending one, else for all of it.
int wait_pending(slc_grid *g, const std::vector<Pending> &pend, const char *lo, size_t bytes,
                 cudaStream_t s, size_t chunk_index, bool per_chunk)
{
    const char *hi = lo + bytes;
    for (const Pending &p : pend) {
        if (!overlaps(p, lo, hi) || p.ev.empty()) continue;
        if (per_chunk && p.lo == lo && p.hi == hi && chunk_index < p.ev.size())
            HS_CK(cudaStreamWaitEvent(s, p.ev[chunk_index], 0), "wait chunk");
        else
            HS_CK(cudaStreamWaitEvent(s, p.ev.back(), 0), "wait range");
    }
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
    HS_CK(cudaEventCreateWithFlags(&h->entry, cudaEventDisableTiming), "event");
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
    return SLC_OK;
}

}  // namespace

void host_step_free(HostStep *h)
{
    if (!h) return;
    if (h->h2d) cudaStreamDestroy(h->h2d);
    if (h->d2h) cudaStreamDestroy(h->d2h);
    if (h->comp) cudaStreamDestroy(h->comp);
    if (h->entry) cudaEventDestroy(h->entry);
    for (int s = 0; s < 2; ++s) {
        if (h->inputs_ready[s]) cudaEventDestroy(h->inputs_ready[s]);
        if (h->compute_done[s]) cudaEventDestroy(h->compute_done[s]);
        if (h->set_free[s]) cudaEventDestroy(h->set_free[s]);
    }
    for (int q = 0; q < 2; ++q)
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
    h->parity ^= 1;  // this call's events: the pool of two calls ago (no longer waited on)
    h->pool_used = 0;

    // the set was last used two calls ago: its downloads must be done
    if (h->set_used[set]) HS_CK(cudaStreamWaitEvent(h->h2d, h->set_free[set], 0), "wait set");

    // uploads: V^{n-1} first (no dependency on the previous call), then V^n
    std::vector<Pending> ups;
    const double *src[6] = {prev[0], prev[1], prev[2], cur[0], cur[1], cur[2]};
    double *dst[6] = {D[3], D[4], D[5], D[0], D[1], D[2]};
    for (int q = 0; q < 6; ++q) {
        const size_t bytes = g->ghost_elems[q % 3] * sizeof(double);
        const char *lo = (const char *)src[q];
        Pending pe;
        pe.lo = lo;
        pe.hi = lo + bytes;
        for (size_t off = 0, k = 0; off < bytes; off += kChunkBytes, ++k) {
            const size_t nb = std::min(kChunkBytes, bytes - off);
            rc = wait_pending(g, h->downloads, lo, bytes, h->h2d, k, true);
            if (rc) return rc;
            HS_CK(cudaMemcpyAsync((char *)dst[q] + off, lo + off, nb, cudaMemcpyHostToDevice, h->h2d),
                  "upload");
            cudaEvent_t e = next_event(h);
            if (!e) return hfail(g, SLC_E_CUDA, "event pool");
            HS_CK(cudaEventRecord(e, h->h2d), "record");
            pe.ev.push_back(e);
        }
        ups.push_back(pe);
    }
    HS_CK(cudaEventRecord(h->inputs_ready[set], h->h2d), "record");

    // compute on the internal stream, after the previous call's compute
    HS_CK(cudaStreamWaitEvent(h->comp, h->inputs_ready[set], 0), "wait inputs");
    double *c3[3] = {D[0], D[1], D[2]}, *p3[3] = {D[3], D[4], D[5]}, *n3[3] = {D[6], D[7], D[8]};
    rc = slc_step_bdf2(g, c3, p3, n3, D[9], dt, nullptr, h->comp);
    if (!rc) rc = slc_bulk_shift(g, D[6], D[7], D[8], U_bulk, dt, h->scal2[set], h->comp);
    if (rc) return rc;
    HS_CK(cudaEventRecord(h->compute_done[set], h->comp), "record");

    // downloads: V^{n+1} (the next call's input, first), (u_bulk, forcing),
    // then p; each after any upload still reading its host range
    HS_CK(cudaStreamWaitEvent(h->d2h, h->compute_done[set], 0), "wait compute");
    std::vector<Pending> downs;
    double *hdst[5] = {next[0], next[1], next[2], bulk_out2, p};
    const double *dsrc[5] = {D[6], D[7], D[8], h->scal2[set], D[9]};
    for (int q = 0; q < 5; ++q) {
        const size_t bytes = q < 3 ? g->ghost_elems[q] * sizeof(double)
                                   : (q == 4 ? g->ghost_elems[3] * sizeof(double) : 2 * sizeof(double));
        char *lo = (char *)hdst[q];
        rc = wait_pending(g, h->uploads, lo, bytes, h->d2h, 0, false);
        if (!rc) rc = wait_pending(g, ups, lo, bytes, h->d2h, 0, false);
        if (rc) return rc;
        Pending pe;
        pe.lo = lo;
        pe.hi = lo + bytes;
        for (size_t off = 0; off < bytes; off += kChunkBytes) {
            const size_t nb = std::min(kChunkBytes, bytes - off);
            HS_CK(cudaMemcpyAsync(lo + off, (const char *)dsrc[q] + off, nb, cudaMemcpyDeviceToHost,
                                  h->d2h),
                  "download");
            cudaEvent_t e = next_event(h);
            if (!e) return hfail(g, SLC_E_CUDA, "event pool");
            HS_CK(cudaEventRecord(e, h->d2h), "record");
            pe.ev.push_back(e);
        }
        downs.push_back(pe);
    }
    HS_CK(cudaEventRecord(h->set_free[set], h->d2h), "record");
    h->set_used[set] = true;
    // the caller's stream completes when the results are on the host
    HS_CK(cudaStreamWaitEvent(s, h->set_free[set], 0), "wait downloads");
    h->uploads = ups;
    h->downloads = downs;
    h->set ^= 1;
    return SLC_OK;
}
