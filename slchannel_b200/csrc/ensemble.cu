// ensemble.cu -- many independent channels of uneven grids advanced together:
// every substep of the SL-BDF2 step is ONE launch over all instances (the
// trace+gather a persistent kernel over an (instance, component, tile) work
// queue, the other substeps one block per (instance, tile) item), the
// Poisson FFTs one cuFFT call per group of instances sharing (nx, ny), and
// the whole step is captured once per time-level phase into a CUDA graph.
//
// Each instance keeps its own slc_grid handle for its tables (and for the
// BDF1 bootstrap and diagnostics through the single-channel entry points).
// Per instance the kernels do the arithmetic of the single-channel step
// (slc_step_bdf2 followed by slc_bulk_shift), so an instance advanced in the
// ensemble matches the same instance advanced on its own.
#include <cufft.h>

#include <algorithm>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "slc_grid.h"

struct slc_ensemble {
    int device = 0;
    int order = 6;
    int traj = 2;  // the instances' common trajectory order, 0 when they differ
    int mixed = 0;  // all instances in the mixed form
    std::vector<slc_grid *> grids;
    std::vector<EnsInst> host_inst;
    std::vector<int> tkl;
    // instances whose trace+gather runs as the single-grid TMA-staged launches
    // (large enough to fill the GPU alone) instead of in the persistent kernel
    std::vector<char> staged;
    bool bound = false;
    std::string err;
    // device copies
    EnsInst *d_inst = nullptr;
    EnsItem *d_items = nullptr;
    unsigned *d_queue = nullptr;
    unsigned long long *d_ncl = nullptr;  // internal counters when the caller passes none
    std::vector<double *> zs_tabs;
    // item ranges inside d_items
    struct Range {
        int off = 0, n = 0;
    } r_bc, r_lin, r_sl, r_div, r_th, r_pr, r_bulk, r_pp, r_pack;
    Range r_zs[kZsChunks];  // z-solve items grouped by chunk size
    int sl_grid = 148;
    int pack_threads = 32;  // k_pack_mixed_ens block size: the largest instance's levels
    // FFT groups (instances sharing nx, ny): pools and plans
    struct Group {
        int nx = 0, ny = 0, planes = 0;
        double *rhs = nullptr, *hat = nullptr;
        cufftHandle fwd = 0, inv = 0;
        bool plans = false;
    };
    std::vector<Group> groups;
    std::vector<void *> allocs;
    // graphs, one per phase
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};
};

// An order-6 instance whose staged trace+gather has at least this many
// blocks per component (a few waves of the GPU) runs it as its own launches.
#ifndef SLC_ENS_STAGED_MIN_BLOCKS
#define SLC_ENS_STAGED_MIN_BLOCKS 2048
#endif

namespace {

std::string g_ens_err;

int efail(slc_ensemble *e, int code, const std::string &msg)
{
    if (e) e->err = msg;
    else g_ens_err = msg;
    return code;
}

#define ENS_CK(call, what)                                                                      \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return efail(e, SLC_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e_));    \
    } while (0)

#define ENS_FFT(call, what)                                                                        \
    do {                                                                                           \
        cufftResult r_ = (call);                                                                   \
        if (r_ != CUFFT_SUCCESS)                                                                   \
            return efail(e, SLC_E_CUFFT, std::string(what) + ": cufft error " + std::to_string((int)r_)); \
    } while (0)

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DevGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

template <typename T>
int ealloc(slc_ensemble *e, T **p, size_t n, const char *what)
{
    void *q = nullptr;
    cudaError_t r = cudaMalloc(&q, n * sizeof(T) > 0 ? n * sizeof(T) : 16);
    if (r != cudaSuccess)
        return efail(e, SLC_E_NOMEM, std::string("cudaMalloc ") + what + ": " + cudaGetErrorString(r));
    e->allocs.push_back(q);
    *p = (T *)q;
    return SLC_OK;
}

void drop_graphs(slc_ensemble *e)
{
    for (auto &x : e->exec)
        if (x) {
            cudaGraphExecDestroy(x);
            x = nullptr;
        }
}

void free_groups(slc_ensemble *e)
{
    for (auto &gr : e->groups)
        if (gr.plans) {
            cufftDestroy(gr.fwd);
            cufftDestroy(gr.inv);
            gr.plans = false;
        }
}

// Work items of every multi-instance kernel, in one array.
void build_items(slc_ensemble *e, std::vector<EnsItem> &items)
{
    items.clear();
    e->pack_threads = 32;
    const int n = (int)e->grids.size();
    auto begin = [&](slc_ensemble::Range &r) { r.off = (int)items.size(); };
    auto end = [&](slc_ensemble::Range &r) { r.n = (int)items.size() - r.off; };
    // boundary conditions: u, v, w and p ghosts, 256 per block
    begin(e->r_bc);
    for (int i = 0; i < n; ++i) {
        const SlcParams &P = e->grids[i]->P;
        long long tot = 0;
        for (int c = 0; c < 4; ++c) {
            const GhostShape g = ghost_shape(c, P.nx, P.ny, P.nz);
            const long long xg = (c == 0) ? 1 : 2, yg = (c == 1) ? 1 : 2;
            tot += xg * g.Y * g.Z + (long long)P.nx * yg * g.Z + (long long)P.nx * P.ny * 2;
        }
        const int nb = (int)((tot + 255) / 256);
        for (int b = 0; b < nb; ++b) items.push_back({i, b, nb, 0});
    }
    end(e->r_bc);
    // U* = 2 V^n - V^{n-1}: 1024 elements per block
    auto st = [&](int i) { return i < (int)e->staged.size() && e->staged[i]; };
    begin(e->r_lin);
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3 && !st(i); ++c) {
            const long long ne = (long long)e->grids[i]->ghost_elems[c];
            const int nb = (int)((ne + 1023) / 1024);
            for (int b = 0; b < nb; ++b) items.push_back({i, c, b, 0});
        }
    end(e->r_lin);
    // trace+gather: (instance, component, x index, (y tile << 16) | z tile)
    begin(e->r_sl);
    for (int i = 0; i < n; ++i) {
        if (st(i)) continue;
        const SlcParams &P = e->grids[i]->P;
        const int tk = 1 << e->tkl[i], tj = 256 / tk;
        for (int c = 0; c < 3; ++c) {
            const int nzi = c == 2 ? P.nz - 1 : P.nz;
            if (nzi <= 0) continue;
            const int nkt = (nzi + tk - 1) / tk, njt = (P.ny + tj - 1) / tj;
            for (int x = 0; x < P.nx; ++x)
                for (int jt = 0; jt < njt; ++jt)
                    for (int kt = 0; kt < nkt; ++kt) items.push_back({i, c, x, (jt << 16) | kt});
        }
    }
    end(e->r_sl);
    // z-solve: blocks of zsolve_ens_warps() columns, grouped by chunk size
    for (int q = 0; q < kZsChunks; ++q) {
        begin(e->r_zs[q]);
        for (int i = 0; i < n; ++i) {
            const SlcParams &P = e->grids[i]->P;
            if (zsolve_chunk(P.nz) != kZsChunkValues[q]) continue;
            const long long warps = 3LL * P.nx * P.ny;
            const int W = zsolve_ens_warps();
            const int nb = (int)((warps + W - 1) / W);
            for (int b = 0; b < nb; ++b) items.push_back({i, b, 0, 0});
        }
        end(e->r_zs[q]);
    }
    // divergence pack and projection: 32 x 32 (k, j) tiles per x index
    begin(e->r_div);
    for (int i = 0; i < n; ++i) {
        const SlcParams &P = e->grids[i]->P;
        for (int z = 0; z < P.nx; ++z)
            for (int y = 0; y < (P.ny + 31) / 32; ++y)
                for (int x = 0; x < (P.nz + 31) / 32; ++x) items.push_back({i, x, y, z});
    }
    end(e->r_div);
    e->r_pr = e->r_div;
    // Poisson Thomas sweep: 4 threads per (kx, ky) column, 256 per block
    begin(e->r_th);
    for (int i = 0; i < n; ++i) {
        const SlcParams &P = e->grids[i]->P;
        const long long nthr = 4LL * P.nx * (P.ny / 2 + 1);
        const int nb = (int)((nthr + 255) / 256);
        for (int b = 0; b < nb; ++b) items.push_back({i, b, 0, 0});
    }
    end(e->r_th);
    // bulk partial sums: the single-channel block decomposition per instance
    begin(e->r_bulk);
    for (int i = 0; i < n; ++i)
        for (int b = 0; b < kBulkBlocks; ++b) items.push_back({i, b, 0, 0});
    end(e->r_bulk);
    // mixed form: plane-mean partials (column group, field) and FP32 packs
    begin(e->r_pp);
    if (e->mixed)
        for (int i = 0; i < n; ++i)
            for (int f = 0; f < 6 && !st(i); ++f)
                for (int b = 0; b < mixed_mean_blocks(); ++b) items.push_back({i, b, f, 0});
    end(e->r_pp);
    begin(e->r_pack);
    if (e->mixed)
        for (int i = 0; i < n; ++i) {
            if (st(i)) continue;
            const SlcParams &P = e->grids[i]->P;
            const MixedWS &ws = e->grids[i]->mws;
            e->pack_threads = std::max(e->pack_threads,
                                       mixed_pack_threads(std::max(ws.nzp[0], ws.nzp[2])));
            const int nj = (P.ny + mixed_pack_cols() - 1) / mixed_pack_cols();
            for (int z = 0; z < 3 * P.nx; ++z)
                for (int jb = 0; jb < nj; ++jb) items.push_back({i, jb, z, 0});
        }
    end(e->r_pack);
}

int upload_tables(slc_ensemble *e)
{
    std::vector<EnsItem> items;
    build_items(e, items);
    if (e->d_items) {
        cudaFree(e->d_items);
        e->allocs.erase(std::remove(e->allocs.begin(), e->allocs.end(), (void *)e->d_items),
                        e->allocs.end());
        e->d_items = nullptr;
    }
    int rc = ealloc(e, &e->d_items, items.size(), "ensemble work items");
    if (rc) return rc;
    ENS_CK(cudaMemcpy(e->d_items, items.data(), items.size() * sizeof(EnsItem),
                      cudaMemcpyHostToDevice),
           "upload work items");
    for (size_t i = 0; i < e->host_inst.size(); ++i) e->host_inst[i].tkl = e->tkl[i];
    ENS_CK(cudaMemcpy(e->d_inst, e->host_inst.data(), e->host_inst.size() * sizeof(EnsInst),
                      cudaMemcpyHostToDevice),
           "upload instance table");
    drop_graphs(e);
    return SLC_OK;
}

const EnsItem *items_at(slc_ensemble *e, const slc_ensemble::Range &r) { return e->d_items + r.off; }

// The step of phase ph on stream s (captured or direct).
int enqueue_step(slc_ensemble *e, int ph, cudaStream_t s)
{
    const int n = (int)e->grids.size();
    const int cur = ens_cur(ph), nxt = ens_next(ph);
    const EnsInst *I = e->d_inst;
    ENS_CK(launch_bc_ens(I, items_at(e, e->r_bc), e->r_bc.n, cur, 0, s), "boundary conditions");
    if (e->mixed)
        ENS_CK(launch_mixed_prepare_ens(I, n, items_at(e, e->r_pp), e->r_pp.n, items_at(e, e->r_pack),
                                        e->r_pack.n, e->pack_threads, ph, s),
               "mixed-form means and packs");
    else
        ENS_CK(launch_lincomb_ens(I, items_at(e, e->r_lin), e->r_lin.n, ph, s), "U* = 2V^n - V^{n-1}");
    for (int i = 0; i < n; ++i)
        ENS_CK(cudaMemsetAsync(e->host_inst[i].ncl, 0, sizeof(unsigned long long), s), "memset");
    ENS_CK(cudaMemsetAsync(e->d_queue, 0, sizeof(unsigned), s), "memset");
    const int prv = ens_prev(ph);
    for (int i = 0; i < n; ++i) {
        if (!e->staged[i]) continue;
        slc_grid *g = e->grids[i];
        const EnsInst &H = e->host_inst[i];
        const Tri a{H.lev[cur][0], H.lev[cur][1], H.lev[cur][2]}, b{H.lev[prv][0], H.lev[prv][1], H.lev[prv][2]};
        const TriMut o{H.lev[nxt][0], H.lev[nxt][1], H.lev[nxt][2]};
        if (e->mixed) {
            ENS_CK(launch_mixed_prepare(g->P, a, b, Tri{nullptr, nullptr, nullptr}, g->mws, s, &g->tmx),
                   "mixed-form pack (padded)");
            ENS_CK(launch_sl_mixed_tma(g->P, a, b, g->mws, g->tmx, H.dt, o, H.ncl, g->dev_flags, s),
                   "mixed trace+gather BDF2 (TMA-staged)");
        } else {
            ENS_CK(launch_mid_pack(g->P, a, b, TriMut{g->mid[0], g->mid[1], g->mid[2]}, g->tma, s),
                   "U* and padded node copies");
            ENS_CK(launch_sl_tma(g->P, a, b, Tri{g->mid[0], g->mid[1], g->mid[2]}, H.dt, o, H.ncl, g->dev_flags,
                                 g->tma, s),
                   "trace+gather BDF2 (TMA-staged)");
        }
    }
    if (e->mixed)
        ENS_CK(launch_sl_mixed_ens(I, items_at(e, e->r_sl), e->r_sl.n, ph, e->order, e->traj, e->d_queue,
                                   e->sl_grid, s),
               "mixed trace+gather BDF2");
    else
        ENS_CK(launch_sl_ens(I, items_at(e, e->r_sl), e->r_sl.n, ph, e->order, e->d_queue, e->sl_grid, s),
               "trace+gather BDF2");
    for (int q = 0; q < kZsChunks; ++q)
        ENS_CK(launch_zsolve_ens(I, items_at(e, e->r_zs[q]), e->r_zs[q].n, nxt, kZsChunkValues[q], s),
               "z-solve");
    ENS_CK(launch_div_pack_ens(I, items_at(e, e->r_div), e->r_div.n, nxt, s), "divergence");
    for (auto &gr : e->groups) {
        ENS_FFT(cufftSetStream(gr.fwd, s), "cufftSetStream");
        ENS_FFT(cufftExecD2Z(gr.fwd, gr.rhs, (cufftDoubleComplex *)gr.hat), "cufftExecD2Z");
    }
    ENS_CK(launch_thomas_ens(I, items_at(e, e->r_th), e->r_th.n, s), "Poisson Thomas sweep");
    for (auto &gr : e->groups) {
        ENS_FFT(cufftSetStream(gr.inv, s), "cufftSetStream");
        ENS_FFT(cufftExecZ2D(gr.inv, (cufftDoubleComplex *)gr.hat, gr.rhs), "cufftExecZ2D");
    }
    ENS_CK(launch_project_ens(I, items_at(e, e->r_pr), e->r_pr.n, nxt, s), "projection");
    ENS_CK(launch_bc_ens(I, items_at(e, e->r_bc), e->r_bc.n, nxt, 1, s), "boundary conditions");
    ENS_CK(launch_bulk_partials_ens(I, items_at(e, e->r_bulk), e->r_bulk.n, nxt, 0, s), "bulk");
    ENS_CK(launch_bulk_finish_ens(I, n, 0, s), "bulk");
    ENS_CK(launch_bulk_partials_ens(I, items_at(e, e->r_bulk), e->r_bulk.n, nxt, 1, s), "bulk shift");
    ENS_CK(launch_bc_ens(I, items_at(e, e->r_bc), e->r_bc.n, nxt, 0, s), "boundary conditions");
    ENS_CK(launch_bulk_finish_ens(I, n, 1, s), "bulk");
    return SLC_OK;
}

}  // namespace

extern "C" {

const char *slc_ensemble_last_error(const slc_ensemble *e)
{
    return e ? e->err.c_str() : g_ens_err.c_str();
}

int slc_ensemble_create(const slc_grid_desc *descs, int n, slc_ensemble **out)
{
    if (!descs || !out || n < 1) return efail(nullptr, SLC_E_INVALID, "need descriptors, n >= 1 and an output pointer");
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (descs[i].precision != descs[0].precision)
            return efail(nullptr, SLC_E_INVALID, "all instances of an ensemble share one precision");
        if (descs[i].order != descs[0].order)
            return efail(nullptr, SLC_E_INVALID, "all instances of an ensemble share one interp_order");
        if (descs[i].device != descs[0].device)
            return efail(nullptr, SLC_E_INVALID, "all instances of an ensemble live on one device");
        if (descs[i].nz < 2)
            return efail(nullptr, SLC_E_INVALID, "ensemble instances need nz >= 2");
    }
    slc_ensemble *e = new slc_ensemble();
    e->device = descs[0].device;
    e->order = descs[0].order;
    e->traj = descs[0].traj_order;
    for (int i = 1; i < n; ++i)
        if (descs[i].traj_order != e->traj) e->traj = 0;  // a mixture: read per instance
    e->mixed = descs[0].precision == SLC_PREC_MIXED ? 1 : 0;
    DevGuard dg(e->device);
    for (int i = 0; i < n; ++i) {
        slc_grid *g = nullptr;
        int rc = slc_grid_create(&descs[i], &g);
        if (rc) {
            g_ens_err = std::string("instance ") + std::to_string(i) + ": " + slc_last_error(nullptr);
            slc_ensemble_destroy(e);
            return rc;
        }
        e->grids.push_back(g);
        e->tkl.push_back(descs[i].nz > 48 ? 6 : 5);
    }
    e->host_inst.resize(n);
    int rc = ealloc(e, &e->d_inst, (size_t)n, "instance table");
    if (!rc) rc = ealloc(e, &e->d_queue, (size_t)1, "work-queue counter");
    if (!rc) rc = ealloc(e, &e->d_ncl, (size_t)n, "clamp counters");
    if (rc) {
        g_ens_err = e->err;
        slc_ensemble_destroy(e);
        return rc;
    }
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, e->device);
    e->sl_grid = dev_sms * (e->mixed ? sl_mixed_ens_blocks_per_sm() : sl_ens_blocks_per_sm());
    *out = e;
    return SLC_OK;
}

int slc_ensemble_destroy(slc_ensemble *e)
{
    if (!e) return SLC_OK;
    DevGuard dg(e->device);
    drop_graphs(e);
    free_groups(e);
    if (e->cap) cudaStreamDestroy(e->cap);
    for (void *p : e->allocs) cudaFree(p);
    for (slc_grid *g : e->grids) slc_grid_destroy(g);
    delete e;
    return SLC_OK;
}

int slc_ensemble_size(const slc_ensemble *e) { return e ? (int)e->grids.size() : 0; }

slc_grid *slc_ensemble_grid(slc_ensemble *e, int i)
{
    if (!e || i < 0 || i >= (int)e->grids.size()) return nullptr;
    return e->grids[i];
}

int slc_ensemble_bind(slc_ensemble *e, double *const *lev, double *const *p, const double *dt,
                      const double *U_bulk, int64_t *nclamp, double *bulk_out)
{
    if (!e) return efail(nullptr, SLC_E_INVALID, "null ensemble");
    if (!lev || !p || !dt || !U_bulk || !bulk_out) return efail(e, SLC_E_INVALID, "null argument");
    const int n = (int)e->grids.size();
    for (int i = 0; i < n; ++i) {
        for (int q = 0; q < 9; ++q)
            if (!lev[i * 9 + q]) return efail(e, SLC_E_INVALID, "null field pointer");
        if (!p[i]) return efail(e, SLC_E_INVALID, "null pressure pointer");
        if (!(dt[i] > 0.0)) return efail(e, SLC_E_INVALID, "dt must be positive");
    }
    DevGuard dg(e->device);
    drop_graphs(e);
    free_groups(e);
    for (void *q : e->allocs)
        if (q != e->d_inst && q != e->d_queue && q != e->d_ncl) cudaFree(q);
    e->allocs.erase(std::remove_if(e->allocs.begin(), e->allocs.end(),
                                   [&](void *q) { return q != e->d_inst && q != e->d_queue && q != e->d_ncl; }),
                    e->allocs.end());
    e->d_items = nullptr;
    e->zs_tabs.assign(n, nullptr);
    e->groups.clear();
    // FFT groups by (nx, ny), instances in index order inside a group
    std::map<std::pair<int, int>, int> gid;
    std::vector<int> group_of(n), plane_off(n);
    for (int i = 0; i < n; ++i) {
        const SlcParams &P = e->grids[i]->P;
        auto key = std::make_pair(P.nx, P.ny);
        auto it = gid.find(key);
        if (it == gid.end()) {
            it = gid.emplace(key, (int)e->groups.size()).first;
            slc_ensemble::Group gr;
            gr.nx = P.nx;
            gr.ny = P.ny;
            e->groups.push_back(gr);
        }
        group_of[i] = it->second;
        plane_off[i] = e->groups[it->second].planes;
        e->groups[it->second].planes += P.nz;
    }
    for (auto &gr : e->groups) {
        const size_t real = (size_t)gr.planes * gr.nx * gr.ny;
        const size_t cplx = (size_t)gr.planes * gr.nx * (gr.ny / 2 + 1);
        int rc = ealloc(e, &gr.rhs, real, "group Poisson rhs");
        if (!rc) rc = ealloc(e, &gr.hat, 2 * cplx, "group Poisson spectrum");
        if (rc) return rc;
        int dims[2] = {gr.nx, gr.ny};
        ENS_FFT(cufftPlanMany(&gr.fwd, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, gr.planes),
                "cufftPlanMany D2Z");
        if (cufftPlanMany(&gr.inv, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, gr.planes) !=
            CUFFT_SUCCESS) {
            cufftDestroy(gr.fwd);
            return efail(e, SLC_E_CUFFT, "cufftPlanMany Z2D failed");
        }
        gr.plans = true;
    }
    for (int i = 0; i < n; ++i) {
        slc_grid *g = e->grids[i];
        const SlcParams &P = g->P;
        EnsInst &I = e->host_inst[i];
        I = EnsInst{};
        I.P = P;
        for (int l = 0; l < 3; ++l)
            for (int c = 0; c < 3; ++c) I.lev[l][c] = lev[i * 9 + l * 3 + c];
        I.p = p[i];
        for (int c = 0; c < 3; ++c) {
            if (!g->mid[c]) {
                void *q = nullptr;
                ENS_CK(cudaMalloc(&q, g->ghost_elems[c] * sizeof(double)), "U* workspace");
                g->allocs.push_back(q);
                g->mid[c] = (double *)q;
                ENS_CK(cudaMemset(q, 0, g->ghost_elems[c] * sizeof(double)), "memset");
            }
            I.mid[c] = g->mid[c];
        }
        I.dzf = g->dzf;
        I.dzc = g->dzc;
        I.kx2 = g->kx2;
        I.ky2 = g->ky2;
        I.cl = g->cl;
        I.cr = g->cr;
        const slc_ensemble::Group &gr = e->groups[group_of[i]];
        I.rhs = gr.rhs + (size_t)plane_off[i] * P.nx * P.ny;
        I.hat = gr.hat + (size_t)2 * plane_off[i] * P.nx * (P.ny / 2 + 1);
        I.cpw = g->cpw;
        double *tab = nullptr;
        int rc = ealloc(e, &tab, zsolve_table_doubles(P.nz), "z-solve tables");
        if (rc) return rc;
        const size_t half = zsolve_table_doubles(P.nz) / 2;
        ENS_CK(launch_zsolve_tables(P, g->dzc, g->dzf, (2.0 / 3.0) * dt[i], tab, tab + half, 0),
               "z-solve tables");
        e->zs_tabs[i] = tab;
        I.zs_uv = tab;
        I.zs_w = tab + half;
        I.partials = g->partials;
        I.scal = g->scal;
        I.ncl = nclamp ? (unsigned long long *)(nclamp + i) : e->d_ncl + i;
        I.bulk_out = bulk_out + 2 * i;
        I.dt = dt[i];
        I.Lx = g->Lx;
        I.Ly = g->Ly;
        I.U_bulk = U_bulk[i];
        I.tkl = e->tkl[i];
        if (e->mixed) {
            int rm = slc_grid_ensure_mixed(g);
            if (rm) return efail(e, rm, std::string("instance ") + std::to_string(i) + ": " + g->err);
            I.mixed = 1;
            I.mws = g->mws;
        }
    }
    // the large order-6 instances gather through the single-grid staged
    // launches (each fills the GPU alone); the rest share the persistent kernel
    e->staged.assign(n, 0);
    if (e->order == 6)
        for (int i = 0; i < n; ++i) {
            const SlcParams &P = e->grids[i]->P;
            const long long blocks = (long long)((P.nz + 31) / 32) * ((P.ny + 3) / 4) * ((P.nx + 1) / 2);
            if (blocks < SLC_ENS_STAGED_MIN_BLOCKS) continue;
            bool ready = false;
            int rs = slc_grid_ensure_staged(e->grids[i], &ready);
            if (rs) return efail(e, rs, std::string("instance ") + std::to_string(i) + ": " + e->grids[i]->err);
            e->staged[i] = ready ? 1 : 0;
        }
    ENS_CK(cudaDeviceSynchronize(), "z-solve tables");
    int rc = upload_tables(e);
    if (rc) return rc;
    e->bound = true;
    return SLC_OK;
}

int slc_ensemble_set_tiles(slc_ensemble *e, const int *tkl)
{
    if (!e || !tkl) return efail(e, SLC_E_INVALID, "null argument");
    for (size_t i = 0; i < e->grids.size(); ++i)
        if (tkl[i] < 3 || tkl[i] > 8) return efail(e, SLC_E_INVALID, "tile log2 z-extent must be in [3, 8]");
    for (size_t i = 0; i < e->grids.size(); ++i) e->tkl[i] = tkl[i];
    if (!e->bound) return SLC_OK;
    DevGuard dg(e->device);
    return upload_tables(e);
}

int slc_ensemble_get_tiles(const slc_ensemble *e, int *tkl)
{
    if (!e || !tkl) return SLC_E_INVALID;
    for (size_t i = 0; i < e->grids.size(); ++i) tkl[i] = e->tkl[i];
    return SLC_OK;
}

int slc_ensemble_step_bdf2(slc_ensemble *e, int phase, int use_graph, void *stream)
{
    if (!e) return efail(nullptr, SLC_E_INVALID, "null ensemble");
    if (!e->bound) return efail(e, SLC_E_INVALID, "slc_ensemble_bind must come first");
    if (phase < 0 || phase > 2) return efail(e, SLC_E_INVALID, "phase must be 0, 1 or 2");
    DevGuard dg(e->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (!use_graph) return enqueue_step(e, phase, s);
    if (!e->exec[phase]) {
        if (!e->cap) ENS_CK(cudaStreamCreateWithFlags(&e->cap, cudaStreamNonBlocking), "capture stream");
        ENS_CK(cudaStreamBeginCapture(e->cap, cudaStreamCaptureModeThreadLocal), "begin capture");
        int rc = enqueue_step(e, phase, e->cap);
        cudaGraph_t graph = nullptr;
        cudaError_t ce = cudaStreamEndCapture(e->cap, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        ENS_CK(ce, "end capture");
        cudaError_t ie = cudaGraphInstantiate(&e->exec[phase], graph, 0);
        cudaGraphDestroy(graph);
        ENS_CK(ie, "graph instantiate");
    }
    ENS_CK(cudaGraphLaunch(e->exec[phase], s), "graph launch");
    return SLC_OK;
}

// Time the trace+gather of the instances with one grid shape for each tile
// candidate and keep the fastest.  Runs U* and the trace+gather of `phase`
// (overwriting the V^{n+1} level and the clamp counters), so call it before
// the step that fills that level.  tkl_out (n ints, may be NULL) receives the
// choice; timings_ms (n * 3 doubles, may be NULL) the time per candidate
// 2^5, 2^6, 2^7 of each instance's shape.
int slc_ensemble_autotune(slc_ensemble *e, int phase, int reps, int *tkl_out, double *timings_ms,
                          void *stream)
{
    if (!e) return efail(nullptr, SLC_E_INVALID, "null ensemble");
    if (!e->bound) return efail(e, SLC_E_INVALID, "slc_ensemble_bind must come first");
    if (phase < 0 || phase > 2 || reps < 1) return efail(e, SLC_E_INVALID, "bad phase or reps");
    DevGuard dg(e->device);
    cudaStream_t s = (cudaStream_t)stream;
    const int n = (int)e->grids.size();
    ENS_CK(launch_bc_ens(e->d_inst, items_at(e, e->r_bc), e->r_bc.n, ens_cur(phase), 0, s), "bc");
    if (e->mixed)
        ENS_CK(launch_mixed_prepare_ens(e->d_inst, n, items_at(e, e->r_pp), e->r_pp.n, items_at(e, e->r_pack),
                                        e->r_pack.n, e->pack_threads, phase, s),
               "mixed prepare");
    else
        ENS_CK(launch_lincomb_ens(e->d_inst, items_at(e, e->r_lin), e->r_lin.n, phase, s), "U*");
    std::map<std::vector<int>, std::vector<int>> shapes;
    for (int i = 0; i < n; ++i) {
        const SlcParams &P = e->grids[i]->P;
        shapes[{P.nx, P.ny, P.nz}].push_back(i);
    }
    const int cand[3] = {5, 6, 7};
    std::vector<int> best(e->tkl);
    cudaEvent_t a, b;
    ENS_CK(cudaEventCreate(&a), "event");
    ENS_CK(cudaEventCreate(&b), "event");
    EnsItem *d_tmp = nullptr;
    int rc = SLC_OK;
    for (auto &kv : shapes) {
        double tbest = 1e30;
        for (int ci = 0; ci < 3 && !rc; ++ci) {
            // items of this shape's instances with candidate tile shape
            std::vector<EnsItem> items;
            for (int i : kv.second) {
                const SlcParams &P = e->grids[i]->P;
                const int tk = 1 << cand[ci], tj = 256 / tk;
                for (int c = 0; c < 3; ++c) {
                    const int nzi = c == 2 ? P.nz - 1 : P.nz;
                    const int nkt = (nzi + tk - 1) / tk, njt = (P.ny + tj - 1) / tj;
                    for (int x = 0; x < P.nx; ++x)
                        for (int jt = 0; jt < njt; ++jt)
                            for (int kt = 0; kt < nkt; ++kt) items.push_back({i, c, x, (jt << 16) | kt});
                }
            }
            for (int i : kv.second) e->host_inst[i].tkl = cand[ci];
            cudaError_t ce = cudaMemcpy(e->d_inst, e->host_inst.data(), n * sizeof(EnsInst),
                                        cudaMemcpyHostToDevice);
            if (ce == cudaSuccess) ce = cudaMalloc(&d_tmp, items.size() * sizeof(EnsItem));
            if (ce == cudaSuccess)
                ce = cudaMemcpy(d_tmp, items.data(), items.size() * sizeof(EnsItem), cudaMemcpyHostToDevice);
            float ms = 0.f;
            for (int r = 0; r <= reps && ce == cudaSuccess; ++r) {  // r == 0 warms up
                ce = cudaMemsetAsync(e->d_queue, 0, sizeof(unsigned), s);
                if (ce == cudaSuccess && r == 1) ce = cudaEventRecord(a, s);
                if (ce == cudaSuccess)
                    ce = e->mixed ? launch_sl_mixed_ens(e->d_inst, d_tmp, (int)items.size(), phase, e->order,
                                                        e->traj, e->d_queue, e->sl_grid, s)
                                  : launch_sl_ens(e->d_inst, d_tmp, (int)items.size(), phase, e->order,
                                                  e->d_queue, e->sl_grid, s);
            }
            if (ce == cudaSuccess) ce = cudaEventRecord(b, s);
            if (ce == cudaSuccess) ce = cudaEventSynchronize(b);
            if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, a, b);
            if (d_tmp) cudaFree(d_tmp);
            d_tmp = nullptr;
            if (ce != cudaSuccess) {
                rc = efail(e, SLC_E_CUDA, std::string("autotune: ") + cudaGetErrorString(ce));
                break;
            }
            const double t = ms / reps;
            if (timings_ms)
                for (int i : kv.second) timings_ms[i * 3 + ci] = t;
            if (t < tbest) {
                tbest = t;
                for (int i : kv.second) best[i] = cand[ci];
            }
        }
        if (rc) break;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) {
        for (int i = 0; i < n; ++i) e->host_inst[i].tkl = e->tkl[i];
        cudaMemcpy(e->d_inst, e->host_inst.data(), n * sizeof(EnsInst), cudaMemcpyHostToDevice);
        return rc;
    }
    e->tkl = best;
    if (tkl_out)
        for (int i = 0; i < n; ++i) tkl_out[i] = best[i];
    return upload_tables(e);
}

}  // extern "C"
