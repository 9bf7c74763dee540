// zsolve.cu -- theta = 1 implicit wall-normal diffusion (I - dt nu Dzz) f = rhs
// on every (i, j) column of u, v and w, in place on the interiors.
//
// The diagonals are the reference's (operators.py:382-630: interior rows from
// dz_c / dz_f, no-slip or free-slip wall closures for u, v; w rows dropping the
// wall couplings).  They are the same for every column, so the Thomas
// factorisation (denominators and c') is computed once per dt by one thread,
// and each column is solved by one warp: lane l owns a contiguous chunk of the
// column in registers, the forward recurrence d'_k = alpha_k d'_{k-1} +
// invden_k d_k and the backward recurrence x_k = -c'_k x_{k+1} + d'_k are
// affine maps, and a 5-step warp scan of the per-chunk maps hands each lane
// its incoming value.  The reference solves the same systems with parallel
// cyclic reduction (tridiag.py:36-61); the results agree to rounding.
#include <string>

#include "../../include/slc_b200.h"
#include "slc_internal.h"

namespace {

// One thread per system (0: u/v, 1: w); sequential factorisation.
__global__ void k_zsolve_tables(SlcParams P, const double *dz_c, const double *dz_f, double dt,
                                double *tab_uv, double *tab_w)
{
    const int which = threadIdx.x;
    if (which > 1) return;
    const double alpha = 1.0 * dt * P.nu;  // theta = 1
    const int nz = P.nz;
    const int n = which == 0 ? nz : nz - 1;
    if (n <= 0) return;
    const int CH = zsolve_chunk(nz), L = 32 * CH;
    double *al = which == 0 ? tab_uv : tab_w;
    double *inv = al + L;
    double *cp = inv + L;
    double cprev = 0.0;
    for (int k = 0; k < n; ++k) {
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
        double a = lower, b = center, c = upper;
        if (k == 0) {
            a = 0.0;
            if (which == 0) b = center - lower;  // u[0] = -u[1]
        }
        if (k == n - 1) {
            c = 0.0;
            if (which == 0) b = P.top_neumann ? center + upper : center - upper;
        }
        const double denom = b - a * cprev;
        const double id = 1.0 / denom;
        const double cpk = c * id;
        const int pos = (k % CH) * 32 + k / CH;  // lane-interleaved
        al[pos] = -a * id;
        inv[pos] = id;
        cp[pos] = cpk;
        cprev = cpk;
    }
}

constexpr int kZWarps = 4;  // warps (columns) per block

__host__ __device__ __forceinline__ int zpad(int k) { return k + (k >> 3); }  // bank skew, 1 per 8

// Column `wid` (component-major over the 3 nx ny columns) solved by the
// calling warp, with `sm` its zpad(32 CH) doubles of shared memory.
template <int CH>
__device__ __forceinline__ void zsolve_warp(const SlcParams &P, double *u, double *v, double *w,
                                            const double *__restrict__ tab_uv,
                                            const double *__restrict__ tab_w, long long wid,
                                            double *sm)
{
    const int lane = threadIdx.x & 31;
    const long long ncol = (long long)P.nx * P.ny;
    if (wid >= 3 * ncol) return;  // whole warps exit together
    const int comp = (int)(wid / ncol);
    const int col = (int)(wid - (long long)comp * ncol);
    const int i = col / P.ny, j = col - (col / P.ny) * P.ny;
    const GhostShape g = ghost_shape(comp, P.nx, P.ny, P.nz);
    double *base = comp == 0 ? u : (comp == 1 ? v : w);
    double *colp = base + (size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z + 1;
    const int n = comp == 2 ? P.nz - 1 : P.nz;
    const double *tab = comp == 2 ? tab_w : tab_uv;
    const double *al = tab, *inv = tab + 32 * CH, *cp = tab + 64 * CH;

    // coalesced column load, transposed through shared memory into per-lane chunks
#pragma unroll
    for (int q = 0; q < CH; ++q) {
        const int k = q * 32 + lane;
        if (k < n) sm[zpad(k)] = colp[k];
    }
    __syncwarp();
    const int s = lane * CH;
    double d[CH];
#pragma unroll
    for (int q = 0; q < CH; ++q) d[q] = (s + q < n) ? sm[zpad(s + q)] : 0.0;

    // forward: chunk map y_out = A y_in + B
    double A = 1.0, B = 0.0;
#pragma unroll
    for (int q = 0; q < CH; ++q) {
        const int k = s + q;
        if (k < n) {
            const double a = __ldg(al + q * 32 + lane);
            B = fma(a, B, __ldg(inv + q * 32 + lane) * d[q]);
            A = a * A;
        }
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double Ap = __shfl_up_sync(0xffffffffu, A, off);
        const double Bp = __shfl_up_sync(0xffffffffu, B, off);
        if (lane >= off) {
            B = fma(A, Bp, B);
            A = A * Ap;
        }
    }
    double y = __shfl_up_sync(0xffffffffu, B, 1);
    if (lane == 0) y = 0.0;
#pragma unroll
    for (int q = 0; q < CH; ++q) {
        const int k = s + q;
        if (k < n) {
            y = fma(__ldg(al + q * 32 + lane), y, __ldg(inv + q * 32 + lane) * d[q]);
            d[q] = y;
        }
    }

    // backward: x_k = -c'_k x_{k+1} + d'_k (c'_{n-1} = 0)
    A = 1.0;
    B = 0.0;
#pragma unroll
    for (int q = CH - 1; q >= 0; --q) {
        const int k = s + q;
        if (k < n) {
            const double gk = -__ldg(cp + q * 32 + lane);
            B = fma(gk, B, d[q]);
            A = gk * A;
        }
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double An = __shfl_down_sync(0xffffffffu, A, off);
        const double Bn = __shfl_down_sync(0xffffffffu, B, off);
        if (lane + off < 32) {
            B = fma(A, Bn, B);
            A = A * An;
        }
    }
    double x = __shfl_down_sync(0xffffffffu, B, 1);
    if (lane == 31) x = 0.0;
#pragma unroll
    for (int q = CH - 1; q >= 0; --q) {
        const int k = s + q;
        if (k < n) {
            x = fma(-__ldg(cp + q * 32 + lane), x, d[q]);
            d[q] = x;
        }
    }
    // back through shared memory for a coalesced store
    __syncwarp();
#pragma unroll
    for (int q = 0; q < CH; ++q)
        if (s + q < n) sm[zpad(s + q)] = d[q];
    __syncwarp();
#pragma unroll
    for (int q = 0; q < CH; ++q) {
        const int k = q * 32 + lane;
        if (k < n) colp[k] = sm[zpad(k)];
    }
}

template <int CH>
__global__ void __launch_bounds__(kZWarps * 32) k_zsolve(SlcParams P, double *u, double *v,
                                                         double *w,
                                                         const double *__restrict__ tab_uv,
                                                         const double *__restrict__ tab_w)
{
    extern __shared__ double zsm[];
    const int wib = threadIdx.x >> 5;
    zsolve_warp<CH>(P, u, v, w, tab_uv, tab_w, (long long)blockIdx.x * kZWarps + wib,
                    zsm + wib * zpad(32 * CH));
}

// Ensemble form: item (inst, block index) over the instances whose chunk
// size is CH (the caller groups them), so each channel is solved exactly as
// on its own, and each launch carries one instantiation's registers and
// shared memory rather than the largest one's.
template <int CH>
__global__ void __launch_bounds__(kZWarps * 32) k_zsolve_ens(const EnsInst *__restrict__ ins,
                                                             const EnsItem *__restrict__ items,
                                                             int lvl)
{
    extern __shared__ double zsm[];
    const EnsItem it = items[blockIdx.x];
    const EnsInst &I = ins[it.inst];
    const int wib = threadIdx.x >> 5;
    const long long wid = (long long)it.a * kZWarps + wib;
    zsolve_warp<CH>(I.P, I.lev[lvl][0], I.lev[lvl][1], I.lev[lvl][2], I.zs_uv, I.zs_w, wid,
                    zsm + wib * zpad(32 * CH));
}

}  // namespace

cudaError_t launch_zsolve_tables(const SlcParams &P, const double *dz_c, const double *dz_f,
                                 double dt, double *tab_uv, double *tab_w, cudaStream_t s)
{
    k_zsolve_tables<<<1, 32, 0, s>>>(P, dz_c, dz_f, dt, tab_uv, tab_w);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_zsolve(const SlcParams &P, TriMut f, const double *tab_uv, const double *tab_w,
                          cudaStream_t s)
{
    const long long warps = 3LL * P.nx * P.ny;
    const unsigned blocks = (unsigned)((warps + kZWarps - 1) / kZWarps);
    const int CH = zsolve_chunk(P.nz);  // chunk length per lane
#define ZS(CHV)                                                                              \
    k_zsolve<CHV><<<blocks, kZWarps * 32, kZWarps * zpad(32 * CHV) * sizeof(double), s>>>( \
        P, f.u, f.v, f.w, tab_uv, tab_w)
    if (P.nz > 1024) return cudaErrorInvalidValue;
    if (CH == 1) ZS(1);
    else if (CH == 2) ZS(2);
    else if (CH == 4) ZS(4);
    else if (CH == 8) ZS(8);
    else if (CH == 12) ZS(12);
    else if (CH == 16) ZS(16);
    else ZS(32);
#undef ZS
    count_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// slc_zsolve_noalloc: the same z-solve for callers that must not allocate
// device memory.  Its only scratch, the Thomas factorisation tables (6 nz
// doubles), lives in this fixed device array instead of a handle's workspace.
// ---------------------------------------------------------------------------

constexpr int kNoAllocMaxNz = 1024;  // 6 * 1024 doubles = 48 KiB per GPU
static __device__ __align__(256) double g_zsolve_noalloc_tables[6 * kNoAllocMaxNz];

namespace {

// Device address of the table array on the current device.  In host code the
// array's name is only a stand-in symbol, so the address is looked up with
// that device current -- on every call: the lookup is cheap, and an address
// cached across calls would dangle after a cudaDeviceReset (the module is
// loaded again, possibly elsewhere).
int noalloc_tables(double **out)
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_zsolve_noalloc_tables);
    if (e != cudaSuccess || !p)
        return slc_report_error(SLC_E_CUDA, (std::string("cudaGetSymbolAddress: ") +
                                             cudaGetErrorString(e)).c_str());
    *out = (double *)p;
    return SLC_OK;
}

}  // namespace

extern "C" int slc_zsolve_noalloc(int nx, int ny, int nz, double nu, int top_wall_neumann,
                                  const double *dz_c, const double *dz_f, double dt, double *u,
                                  double *v, double *w, void *stream)
{
    if (nx < 1 || ny < 1 || nz < 2)
        return slc_report_error(SLC_E_INVALID, "slc_zsolve_noalloc: needs nx, ny >= 1 and nz >= 2");
    if (nz > kNoAllocMaxNz)
        return slc_report_error(SLC_E_INVALID,
                                ("slc_zsolve_noalloc: nz = " + std::to_string(nz) +
                                 " exceeds the fixed table size (nz <= " +
                                 std::to_string(kNoAllocMaxNz) + ")").c_str());
    if (!dz_c || !dz_f || !u || !v || !w)
        return slc_report_error(SLC_E_INVALID, "slc_zsolve_noalloc: null pointer");
    double *tab = nullptr;
    int rc = noalloc_tables(&tab);
    if (rc) return rc;
    SlcParams P{};
    P.nx = nx;
    P.ny = ny;
    P.nz = nz;
    P.nu = nu;
    P.top_neumann = top_wall_neumann ? 1 : 0;
    cudaStream_t s = (cudaStream_t)stream;
    // every entry of the tables the solve reads is rewritten first, so nothing
    // needs clearing between calls
    const size_t half = zsolve_table_doubles(nz) / 2;  // <= 3 * 1024 for nz <= 1024
    cudaError_t e = launch_zsolve_tables(P, dz_c, dz_f, dt, tab, tab + half, s);
    if (e == cudaSuccess) e = launch_zsolve(P, TriMut{u, v, w}, tab, tab + half, s);
    if (e != cudaSuccess)
        return slc_report_error(SLC_E_CUDA, (std::string("slc_zsolve_noalloc: ") +
                                             cudaGetErrorString(e)).c_str());
    return SLC_OK;
}

int zsolve_ens_warps() { return kZWarps; }

namespace {
template <int CH>
cudaError_t launch_zsolve_ens_ch(const EnsInst *ins, const EnsItem *items, int nitems, int lvl,
                                 cudaStream_t s)
{
    const size_t smem = (size_t)kZWarps * zpad(32 * CH) * sizeof(double);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_zsolve_ens<CH>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_zsolve_ens<CH><<<nitems, kZWarps * 32, smem, s>>>(ins, items, lvl);
    count_launches(1);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_zsolve_ens(const EnsInst *ins, const EnsItem *items, int nitems, int lvl,
                              int ch, cudaStream_t s)
{
    if (nitems <= 0) return cudaSuccess;
    switch (ch) {
    case 1: return launch_zsolve_ens_ch<1>(ins, items, nitems, lvl, s);
    case 2: return launch_zsolve_ens_ch<2>(ins, items, nitems, lvl, s);
    case 4: return launch_zsolve_ens_ch<4>(ins, items, nitems, lvl, s);
    case 8: return launch_zsolve_ens_ch<8>(ins, items, nitems, lvl, s);
    case 12: return launch_zsolve_ens_ch<12>(ins, items, nitems, lvl, s);
    case 16: return launch_zsolve_ens_ch<16>(ins, items, nitems, lvl, s);
    default: return launch_zsolve_ens_ch<32>(ins, items, nitems, lvl, s);
    }
}
