// slc_grid.h -- the handle behind slc_grid_create (private to the library):
// grid tables, cuFFT plans and workspaces of one channel.
#pragma once

#include <cufft.h>

#include <string>
#include <vector>

#include "../../include/slc_b200.h"
#include "slc_internal.h"

struct AdjWS;                 // adjoint workspace (adjoint.cu), allocated on first use
void adj_free(AdjWS *w);
struct HostStep;              // host-state step machinery (host_step.cu), on first use
void host_step_free(HostStep *h);
struct StatsWS;               // diagnostics / statistics workspace (diagnostics.cu), on first use
void stats_free(StatsWS *s);

// The step's choice between the TMA-staged and the L1 gather (slc_api.cu),
// from the staged-box counters of earlier calls, read back asynchronously.
struct GatherChoice {
    bool staged = true;
    bool pending = false;                // a counter copy is in flight behind ev
    unsigned long long *host = nullptr;  // pinned copy of dev_flags
    cudaEvent_t ev = nullptr;
    unsigned long long last[4] = {0, 0, 0, 0};
    int calls_l1 = 0;
};

struct slc_grid {
    SlcParams P{};
    int device = 0;
    double Lx = 0, Ly = 0;
    double *zc = nullptr, *zf = nullptr, *dzc = nullptr, *dzf = nullptr;
    double *dinv_c[SLC_MAX_ORDER + 1] = {}, *dinv_f[SLC_MAX_ORDER + 1] = {};
    float *zc32 = nullptr, *zf32 = nullptr;
    float *dinv_c32[SLC_MAX_ORDER + 1] = {}, *dinv_f32[SLC_MAX_ORDER + 1] = {};
    double *kx2 = nullptr, *ky2 = nullptr, *cl = nullptr, *cr = nullptr;
    double *rhs = nullptr, *hat = nullptr, *cpw = nullptr;
    double *zs_tab = nullptr;
    double zs_dt = 0.0;
    bool zs_valid = false;
    double *partials = nullptr, *scal = nullptr;
    unsigned long long *ncl_scratch = nullptr;
    double *mid[3] = {nullptr, nullptr, nullptr};
    int mixed = 0;          // SLC_PREC_MIXED
    bool mixed_ready = false;
    MixedWS mws{};
    AdjWS *adj = nullptr;
    double *p_ext = nullptr, *phi = nullptr;  // incremental-pressure workspaces
    HostStep *host = nullptr;
    StatsWS *stats = nullptr;
    TmaSL tma{};
    int tma_state = 0;        // 0 not tried, 1 ready, -1 unavailable (L1 gather path)
    TmaMixed tmx{};           // the mixed form's staged gather (padded FP32 copies, tensor maps)
    int tmx_state = 0;        // as tma_state
    unsigned long long *dev_flags = nullptr;  // staged-gather statistics (launch_sl_tma)
    GatherChoice gchoice;
    size_t ghost_elems[4] = {0, 0, 0, 0};
    cufftHandle fwd = 0, inv = 0;
    bool plans = false;
    std::vector<void *> allocs;
    std::string err;
    // per-phase event timing (slc_timing)
    bool timing = false;
    std::vector<cudaEvent_t> evs;  // pairs: [2i] start, [2i+1] end
    std::vector<int> ev_phase;
    size_t ev_used = 0;
};

// Allocate the mixed form's workspace of a mixed-precision handle (slc_api.cu).
int slc_grid_ensure_mixed(slc_grid *g);
// Allocate the U* workspace g->mid (slc_api.cu).
int slc_grid_ensure_mid(slc_grid *g);
// Allocate what the handle's TMA-staged BDF2 gather needs (padded copies,
// tensor maps); *ready tells whether the grid can use it (slc_api.cu).
int slc_grid_ensure_staged(slc_grid *g, bool *ready);
// zsolve + projection of slc_step_bdf2 after its trace+gather (slc_api.cu).
int slc_step_bdf2_tail(slc_grid *g, double *const next[3], double *p, double dt, cudaStream_t s);
