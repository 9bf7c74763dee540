// sl_tma.cu -- the BDF2 trace+gather with the gather's source boxes staged
// in shared memory by the Tensor Memory Accelerator (sm_100a).
//
// Why: the order-6 gather issues 216 eight-byte loads per foot per arrival
// point.  A warp's load at one stencil offset covers 32 consecutive z values
// (256 bytes), which from L1 costs about three wavefronts (it straddles three
// 128-byte lines at most alignments) and from shared memory two when its
// lanes read one row of the box.  The kernel is bound by that data pipe.
// Lanes whose foot coordinate floors to the next row in x or y read another
// row; the box depth keeps such lanes on their banks (Box below).
//
// How: a block is a tile of 2 (x) x 4 (y) x 32 (z) arrival points, one warp
// per 32 z.  Every thread traces its feet (the iterated midpoint rule of
// sl_device.cuh, unchanged).  Warp reductions and shared-memory integer
// min/max of the feet's stencil bases give each foot's bounding box.  If it
// fits the order's box (Box<O>), one thread issues a 3-D cp.async.bulk.tensor
// load of the box (no multicast) from a halo-padded node copy of V^n (near
// foot) or V^{n-1} (far foot) onto an mbarrier, and the threads gather from
// shared memory.  A block whose feet spread wider uses the L1 gather.  At
// order 6 the feet go one after the other through one box buffer
// (k_sl_tma_seq); at order 4 both boxes are staged at once (k_sl_tma).  The boxes
// come from padded node copies, written together with U* by k_mid_pack:
// node (i, j, k) at padded (i + q nx, j + r ny, k), x and y extended by one
// box, so a box never wraps.  Weights, the contraction order and the
// epilogue are those of k_sl, so the results are bit-identical to it.
#include <cuda.h>

#include <climits>
#include <mutex>

#include "slc_grid.h"
#include "slc_tma.cuh"

namespace {

constexpr int kThreads = 256;

#include "sl_device.cuh"

constexpr int kTI = 2, kTJ = 4, kTK = 32;    // arrival tile (x, y, z)
// staged box (x, y, z) in nodes.  The z extent sets the row stride in shared
// memory: 48 doubles = 384 bytes, a multiple of the 128-byte bank cycle, so
// lanes whose stencil base moved one row in x or y keep their banks
// (40 doubles gave 3.12 wavefronts per 8-byte load, 48 gives 2.33)
// Staged box (x, y, z) in nodes and resident blocks per SM, per order.  The
// z extent sets the row stride in shared memory: 48 doubles = 384 bytes, a
// multiple of the 128-byte bank cycle, so lanes whose stencil base moved one
// row in x or y keep their banks (40 doubles gave 3.12 wavefronts per 8-byte
// load, 48 gives 2.33).  Order 6 (k_sl_tma_seq, one box per block): 10 x 12
// x 48 doubles = 46 KB at four blocks per SM (64 registers, some spill).
// Measured at 256^3, trace+gather per step: two boxes per block, 10 x 12 at
// two blocks per SM 10.64 ms, 9 x 10 at three 9.88 ms; one box, 9 x 10 at
// three 10.00, at four 9.52, at five 9.71, 10 x 12 at four 9.62 ms (and at
// trajectory CFL 3, 128^3: 1.55 against 1.37 ms, the larger box staging 97 %
// of the far feet instead of 63 %); the L1 gather 10.76 ms.  Order 4
// (k_sl_tma, both boxes at once): 7 x 9 x 48 (24.2 KB) at four blocks.
template <int O>
struct Box {
    static constexpr int X = O == 4 ? 7 : 10;
    static constexpr int Y = O == 4 ? 9 : 12;
    static constexpr int Z = 48;
    static constexpr int elems = X * Y * Z;
    static constexpr size_t bytes = (size_t)elems * sizeof(double);
    static constexpr size_t smem = 2 * bytes + 128;  // both boxes + alignment slack (128-byte starts)
    static constexpr int min_blocks = 4;
};
// the padded copies' halo: the largest box
constexpr int kBX = Box<6>::X > Box<4>::X ? Box<6>::X : Box<4>::X;
constexpr int kBY = Box<6>::Y > Box<4>::Y ? Box<6>::Y : Box<4>::Y;
constexpr int kBZ = 48;
static_assert((kBZ * sizeof(double)) % 16 == 0, "TMA inner box extent");

// Unwrapped stencil base of one coordinate relative to the tile origin
// (NaN or far-out values give a large sentinel that no box fits).
__device__ __forceinline__ int rel_base(double f, int h, int origin)
{
    const double r = f - (double)h - (double)origin;
    if (!(r > -4096.0 && r < 4096.0)) return 1 << 20;
    return (int)r;
}

struct Foot {
    double z;      // clamped z
    double tx, ty;
    int rx, ry;    // unwrapped x, y base (minus O/2 - 1) relative to the tile
    int k0;        // z base
};

template <int C, int O>
__device__ __forceinline__ Foot locate_foot(const SlcParams &P, double xd, double yd, double zd,
                                            int i0, int j0, unsigned &ncl)
{
    constexpr int h = O / 2 - 1;
    if (zd < P.z_lo || zd > P.z_hi) ncl += 1;
    Foot F;
    F.z = clampz(P, zd);
    double s = xd * P.inv_dx + Comp<C>::shift_x;
    double f = floor(s);
    F.tx = s - f;
    F.rx = rel_base(f, h, i0);
    s = yd * P.inv_dy + Comp<C>::shift_y;
    f = floor(s);
    F.ty = s - f;
    F.ry = rel_base(f, h, j0);
    const int NZ = Comp<C>::centers ? P.nz + 2 : P.nz + 1;
    const int m0 = locate_m0(P, Comp<C>::centers, face_cell(P, F.z), F.z);
    F.k0 = min(max(m0 - h, 0), NZ - O);
    return F;
}

// Gather from a staged box: weights and contraction order as gather_sum.
template <int C, int O>
__device__ __forceinline__ double gather_box(const SlcParams &P, const double *box, const Foot &F,
                                             int ox, int oy, int oz)
{
    double wx[O], wy[O], wz[O];
    uniform_weights<O, double>(P, F.tx, wx);
    uniform_weights<O, double>(P, F.ty, wy);
    const double *zn = Comp<C>::centers ? P.zc : P.zf;
    const double *dinv = Comp<C>::centers ? P.dinv_c[O] : P.dinv_f[O];
    z_weights<O, double>(zn, dinv, denom_rows(Comp<C>::centers, P.nz, O), F.k0, F.z, wz);
    const double *b = box + (ox * Box<O>::Y + oy) * Box<O>::Z + oz;
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < O; ++i) {
        double accy = 0.0;
#pragma unroll
        for (int j = 0; j < O; ++j) {
            const double *row = b + (i * Box<O>::Y + j) * Box<O>::Z;
            double accz = 0.0;
#pragma unroll
            for (int k = 0; k < O; ++k) accz = fma(wz[k], row[k], accz);
            accy = fma(wy[j], accz, accy);
        }
        acc = fma(wx[i], accy, acc);
    }
    return acc;
}

// Gather through L1 from the ghost-shaped array (the k_sl path).
template <int C, int O>
__device__ __forceinline__ double gather_global(const SlcParams &P, NodeView<double> V, double xd,
                                                double yd, const Foot &F)
{
    Stencil<O, double> st;
    build_stencil<C, O, double>(P, V.sx, V.sy, xd, yd, F.z, face_cell(P, F.z), st);
    return gather_sum<O, double, double>(V.p, st);
}

template <int C, int O>
__global__ void __launch_bounds__(kThreads, Box<O>::min_blocks)
    k_sl_tma(const __grid_constant__ SlcParams P, const __grid_constant__ Vel3 M, const double *__restrict__ fn, const double *__restrict__ fnm1,
             double dt, double *__restrict__ out, unsigned long long *nclamp, unsigned long long *stats,
             const __grid_constant__ CUtensorMap tmN, const __grid_constant__ CUtensorMap tmM)
{
    extern __shared__ unsigned char smraw[];
    __shared__ __align__(8) unsigned long long mbar[2];
    __shared__ int red[12];  // per foot: min/max of rx, ry, k0
    double *boxN = (double *)(((uintptr_t)smraw + 127) & ~(uintptr_t)127);
    double *boxM = boxN + Box<O>::elems;
    const int tid = threadIdx.x;
    const int i0 = blockIdx.z * kTI, j0 = blockIdx.y * kTJ;
    const int k = blockIdx.x * kTK + (tid & 31);
    const int j = j0 + ((tid >> 5) & (kTJ - 1));
    const int i = i0 + (tid >> 7);
    const int nzi = (C == 2) ? P.nz - 1 : P.nz;
    const bool act = k < nzi && j < P.ny && i < P.nx;
    const unsigned barN = smem_u32(&mbar[0]), barM = smem_u32(&mbar[1]);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            red[2 * q] = INT_MAX;
            red[2 * q + 1] = INT_MIN;
        }
        mbar_init(barN, 1);
        mbar_init(barM, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    unsigned ncl = 0;
    double xa = 0.0, ya = 0.0, za = 0.0, us0 = 0.0, vs0 = 0.0, ws0 = 0.0;
    double xn = 0.0, yn = 0.0, zn = 0.0, xm = 0.0, ym = 0.0, zm = 0.0;
    Foot Fn{}, Fm{};
    if (act) {
        arrival_point<C>(P, i, j, k, xa, ya, za);
        first_sample<C>(P, M, i, j, k, xa, ya, za, us0, vs0, ws0);
        trace_foot(P, M, xa, ya, za, 0.5 * dt, us0, vs0, ws0, xn, yn, zn);
        trace_foot(P, M, xa, ya, za, dt, us0, vs0, ws0, xm, ym, zm);  // half of 2 dt
        Fn = locate_foot<C, O>(P, xn, yn, zn, i0, j0, ncl);
        Fm = locate_foot<C, O>(P, xm, ym, zm, i0, j0, ncl);
        atomicMin(&red[0], Fn.rx);
        atomicMax(&red[1], Fn.rx);
        atomicMin(&red[2], Fn.ry);
        atomicMax(&red[3], Fn.ry);
        atomicMin(&red[4], Fn.k0);
        atomicMax(&red[5], Fn.k0);
        atomicMin(&red[6], Fm.rx);
        atomicMax(&red[7], Fm.rx);
        atomicMin(&red[8], Fm.ry);
        atomicMax(&red[9], Fm.ry);
        atomicMin(&red[10], Fm.k0);
        atomicMax(&red[11], Fm.k0);
    }
    __syncthreads();
    // block-uniform box choice per foot
    bool fit[2];
    int X0[2] = {0, 0}, Y0[2] = {0, 0}, Z0[2] = {0, 0};
#pragma unroll
    for (int f = 0; f < 2; ++f) {
        const int *r = red + 6 * f;
        fit[f] = r[0] <= r[1] && r[1] - r[0] + O <= Box<O>::X && r[3] - r[2] + O <= Box<O>::Y &&
                 r[5] + O - (r[4] & ~1) <= Box<O>::Z;
        if (fit[f]) {  // r[0], r[2] are small here (|.| < 4096)
            int x0 = (i0 + r[0]) % P.nx;
            if (x0 < 0) x0 += P.nx;
            int y0 = (j0 + r[2]) % P.ny;
            if (y0 < 0) y0 += P.ny;
            X0[f] = x0;
            Y0[f] = y0;
            Z0[f] = r[4] & ~1;  // even: 16-byte aligned inner coordinate
        }
    }
    if (tid == 0) {
        // stats: [0] time-outs, [1] blocks, [2] near boxes staged, [3] far boxes staged
        atomicAdd(stats + 1, 1ull);
        if (fit[0]) atomicAdd(stats + 2, 1ull);
        if (fit[1]) atomicAdd(stats + 3, 1ull);
        if (fit[0]) {
            mbar_expect_tx(barN, (unsigned)Box<O>::bytes);
            tma_load_3d(smem_u32(boxN), &tmN, Z0[0], Y0[0], X0[0], barN);
        }
        if (fit[1]) {
            mbar_expect_tx(barM, (unsigned)Box<O>::bytes);
            tma_load_3d(smem_u32(boxM), &tmM, Z0[1], Y0[1], X0[1], barM);
        }
    }
    if (act) {
        double ubar, ubb;
        bool staged = fit[0] && mbar_wait(barN);
        if (fit[0] && !staged) atomicAdd(stats, 1ull);
        if (staged)
            ubar = gather_box<C, O>(P, boxN, Fn, Fn.rx - red[0], Fn.ry - red[2], Fn.k0 - Z0[0]);
        else
            ubar = gather_global<C, O>(P, ghost_view<double>(C, fn, P.nx, P.ny, P.nz), xn, yn, Fn);
        staged = fit[1] && mbar_wait(barM);
        if (fit[1] && !staged) atomicAdd(stats, 1ull);
        if (staged)
            ubb = gather_box<C, O>(P, boxM, Fm, Fm.rx - red[6], Fm.ry - red[8], Fm.k0 - Z0[1]);
        else
            ubb = gather_global<C, O>(P, ghost_view<double>(C, fnm1, P.nx, P.ny, P.nz), xm, ym, Fm);
        const double Rn = xy_diffusion<C>(P, fn, i, j, k);
        const double Rh = P.xy_lagged ? Rn : 2.0 * Rn - xy_diffusion<C>(P, fnm1, i, j, k);
        double res = ubar * (4.0 / 3.0) + ubb * (-1.0 / 3.0);
        res = res + ((2.0 / 3.0) * dt) * Rh;
        const GhostShape g = ghost_shape(C, P.nx, P.ny, P.nz);
        out[(size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z + (k + 1)] = res;
    }
    add_clamps(nclamp, ncl);
    // no copy may still be writing this block's shared memory when it exits;
    // a drain that gives up is counted with the other time-outs (stats[0]),
    // which slc_trace_gather_bdf2_staged turns into an error status
    if (tid == 0) {
        if (fit[0] && !mbar_wait(barN)) atomicAdd(stats, 1ull);
        if (fit[1] && !mbar_wait(barM)) atomicAdd(stats, 1ull);
    }
}

// The same gather with one box buffer (the order-6 form): the near foot is
// traced, located, staged and gathered, then the far foot, so a thread holds
// one foot's state at a time and a block one box; more blocks share an SM,
// and the box can be larger.

__device__ __forceinline__ void block_minmax3(int *red, bool act, int a, int b, int c)
{
    const int v[3] = {a, b, c};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int lo = __reduce_min_sync(0xffffffffu, act ? v[q] : INT_MAX);
        const int hi = __reduce_max_sync(0xffffffffu, act ? v[q] : INT_MIN);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&red[2 * q], lo);
            atomicMax(&red[2 * q + 1], hi);
        }
    }
}

template <int O>
__device__ __forceinline__ bool box_fits(const int *r, int i0, int j0, const SlcParams &P, int &X0, int &Y0,
                                         int &Z0)
{
    const bool fit = r[0] <= r[1] && r[1] - r[0] + O <= Box<O>::X && r[3] - r[2] + O <= Box<O>::Y &&
                     r[5] + O - (r[4] & ~1) <= Box<O>::Z;
    X0 = Y0 = Z0 = 0;
    if (fit) {
        X0 = (i0 + r[0]) % P.nx;
        if (X0 < 0) X0 += P.nx;
        Y0 = (j0 + r[2]) % P.ny;
        if (Y0 < 0) Y0 += P.ny;
        Z0 = r[4] & ~1;
    }
    return fit;
}

template <int C, int O>
__global__ void __launch_bounds__(kThreads, Box<O>::min_blocks)
    k_sl_tma_seq(const __grid_constant__ SlcParams P, const __grid_constant__ Vel3 M, const double *__restrict__ fn,
                 const double *__restrict__ fnm1, double dt, double *__restrict__ out,
                 unsigned long long *nclamp, unsigned long long *stats, const __grid_constant__ CUtensorMap tmN,
                 const __grid_constant__ CUtensorMap tmM)
{
    extern __shared__ unsigned char smraw[];
    __shared__ __align__(8) unsigned long long mbar[2];
    __shared__ int red[12];  // per foot: min/max of rx, ry, k0
    __shared__ int near_lost;  // the near copy did not complete: the box is not reused
    double *box = (double *)(((uintptr_t)smraw + 127) & ~(uintptr_t)127);
    const int tid = threadIdx.x;
    const int i0 = blockIdx.z * kTI, j0 = blockIdx.y * kTJ;
    const int k = blockIdx.x * kTK + (tid & 31);
    const int j = j0 + ((tid >> 5) & (kTJ - 1));
    const int i = i0 + (tid >> 7);
    const int nzi = (C == 2) ? P.nz - 1 : P.nz;
    const bool act = k < nzi && j < P.ny && i < P.nx;
    const unsigned barN = smem_u32(&mbar[0]), barM = smem_u32(&mbar[1]);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            red[2 * q] = INT_MAX;
            red[2 * q + 1] = INT_MIN;
        }
        near_lost = 0;
        mbar_init(barN, 1);
        mbar_init(barM, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    unsigned ncl = 0;
    double xa = 0.0, ya = 0.0, za = 0.0, us0 = 0.0, vs0 = 0.0, ws0 = 0.0, xd = 0.0, yd = 0.0, zd = 0.0;
    Foot F{};
    if (act) {
        arrival_point<C>(P, i, j, k, xa, ya, za);
        first_sample<C>(P, M, i, j, k, xa, ya, za, us0, vs0, ws0);
        trace_foot(P, M, xa, ya, za, 0.5 * dt, us0, vs0, ws0, xd, yd, zd);
        F = locate_foot<C, O>(P, xd, yd, zd, i0, j0, ncl);
    }
    block_minmax3(red, act, F.rx, F.ry, F.k0);
    __syncthreads();
    int X0, Y0, Z0;
    const bool fitN = box_fits<O>(red, i0, j0, P, X0, Y0, Z0);
    if (tid == 0) {
        // stats: [0] time-outs, [1] blocks, [2] near boxes staged, [3] far boxes staged
        atomicAdd(stats + 1, 1ull);
        if (fitN) {
            atomicAdd(stats + 2, 1ull);
            mbar_expect_tx(barN, (unsigned)Box<O>::bytes);
            tma_load_3d(smem_u32(box), &tmN, Z0, Y0, X0, barN);
        }
    }
    double ubar = 0.0;
    if (act) {
        const bool staged = fitN && mbar_wait(barN);
        if (fitN && !staged) atomicAdd(stats, 1ull);
        if (staged)
            ubar = gather_box<C, O>(P, box, F, F.rx - red[0], F.ry - red[2], F.k0 - Z0);
        else
            ubar = gather_global<C, O>(P, ghost_view<double>(C, fn, P.nx, P.ny, P.nz), xd, yd, F);
    }
    __syncthreads();  // every thread is done with the near box
    if (tid == 0 && fitN && !mbar_wait(barN)) {
        atomicAdd(stats, 1ull);
        near_lost = 1;
    }
    if (act) {
        trace_foot(P, M, xa, ya, za, dt, us0, vs0, ws0, xd, yd, zd);  // half of 2 dt
        F = locate_foot<C, O>(P, xd, yd, zd, i0, j0, ncl);
    }
    block_minmax3(red + 6, act, F.rx, F.ry, F.k0);
    __syncthreads();
    const bool fitM = !near_lost && box_fits<O>(red + 6, i0, j0, P, X0, Y0, Z0);
    if (tid == 0 && fitM) {
        atomicAdd(stats + 3, 1ull);
        mbar_expect_tx(barM, (unsigned)Box<O>::bytes);
        tma_load_3d(smem_u32(box), &tmM, Z0, Y0, X0, barM);
    }
    if (act) {
        double ubb;
        const bool staged = fitM && mbar_wait(barM);
        if (fitM && !staged) atomicAdd(stats, 1ull);
        if (staged)
            ubb = gather_box<C, O>(P, box, F, F.rx - red[6], F.ry - red[8], F.k0 - Z0);
        else
            ubb = gather_global<C, O>(P, ghost_view<double>(C, fnm1, P.nx, P.ny, P.nz), xd, yd, F);
        const double Rn = xy_diffusion<C>(P, fn, i, j, k);
        const double Rh = P.xy_lagged ? Rn : 2.0 * Rn - xy_diffusion<C>(P, fnm1, i, j, k);
        double res = ubar * (4.0 / 3.0) + ubb * (-1.0 / 3.0);
        res = res + ((2.0 / 3.0) * dt) * Rh;
        const GhostShape g = ghost_shape(C, P.nx, P.ny, P.nz);
        out[(size_t)(i + 1) * g.Y * g.Z + (size_t)(j + 1) * g.Z + (k + 1)] = res;
    }
    add_clamps(nclamp, ncl);
    if (tid == 0 && fitM && !mbar_wait(barM)) atomicAdd(stats, 1ull);
}

// U* = 2 V^n - V^{n-1} at every node (ghost-shaped, node entries only) and
// the halo-padded node copies of V^n and V^{n-1}.  One warp per padded
// (x, y) row, lanes along z (contiguous in both layouts); the row's source
// (x mod nx, y mod ny) is found once per row.
template <int C>
__global__ void __launch_bounds__(256) k_mid_pack(SlcParams P, const double *__restrict__ a,
                                                  const double *__restrict__ b, double ca, double cb,
                                                  double *__restrict__ mid, double *__restrict__ pa,
                                                  double *__restrict__ pb, int NZp)
{
    const int NZ = C < 2 ? P.nz + 2 : P.nz + 1;
    const int PX = P.nx + kBX, PY = P.ny + kBY;
    const int rows = PX * PY;
    const NodeView<double> Va = ghost_view<double>(C, a, P.nx, P.ny, P.nz);
    const NodeView<double> Vb = ghost_view<double>(C, b, P.nx, P.ny, P.nz);
    double *vm = const_cast<double *>(ghost_view<double>(C, mid, P.nx, P.ny, P.nz).p);
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows;
         r += gridDim.x * (blockDim.x >> 5)) {
        const int x = r / PY, y = r - x * PY;
        const int xi = x % P.nx, yj = y % P.ny;
        const size_t g = (size_t)xi * Va.sx + (size_t)yj * Va.sy;
        const double *ra = Va.p + g, *rb = Vb.p + g;
        double *dm = (x < P.nx && y < P.ny) ? vm + g : nullptr;
        double *da = pa + (size_t)r * NZp, *db = pb + (size_t)r * NZp;
#pragma unroll 4
        for (int z = lane; z < NZp; z += 32) {
            double va = 0.0, vb = 0.0;
            if (z < NZ) {
                va = ra[z];
                vb = rb[z];
                if (dm) dm[z] = ca * va + cb * vb;
            }
            da[z] = va;
            db[z] = vb;
        }
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

template <int O>
cudaError_t launch_tma_t(const SlcParams &P, const Vel3 &M, Tri fn, Tri fnm1, double dt, TriMut out,
                         unsigned long long *ncl, unsigned long long *stats, const TmaSL &T,
                         cudaStream_t s)
{
    const dim3 gc((P.nz + kTK - 1) / kTK, (P.ny + kTJ - 1) / kTJ, (P.nx + kTI - 1) / kTI);
    const dim3 gw((P.nz - 1 + kTK - 1) / kTK, (P.ny + kTJ - 1) / kTJ, (P.nx + kTI - 1) / kTI);
    // the attributes are per device context, so set on every launch (a
    // host-side attribute write)
    if constexpr (O == 6) {  // one box per block
        const size_t sm = Box<O>::bytes + 128;
        cudaError_t e = cudaFuncSetAttribute(k_sl_tma_seq<0, O>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_sl_tma_seq<1, O>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_sl_tma_seq<2, O>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        const CUtensorMap *tq = (const CUtensorMap *)T.maps;
        k_sl_tma_seq<0, O><<<gc, kThreads, sm, s>>>(P, M, fn.u, fnm1.u, dt, out.u, ncl, stats, tq[0], tq[3]);
        k_sl_tma_seq<1, O><<<gc, kThreads, sm, s>>>(P, M, fn.v, fnm1.v, dt, out.v, ncl, stats, tq[1], tq[4]);
        if (P.nz > 1)
            k_sl_tma_seq<2, O><<<gw, kThreads, sm, s>>>(P, M, fn.w, fnm1.w, dt, out.w, ncl, stats, tq[2], tq[5]);
        count_launches(P.nz > 1 ? 3 : 2);
        return cudaGetLastError();
    } else {  // both boxes at once
        cudaError_t attr = cudaFuncSetAttribute(k_sl_tma<0, O>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Box<O>::smem);
        if (attr == cudaSuccess)
            attr = cudaFuncSetAttribute(k_sl_tma<1, O>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Box<O>::smem);
        if (attr == cudaSuccess)
            attr = cudaFuncSetAttribute(k_sl_tma<2, O>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Box<O>::smem);
        if (attr != cudaSuccess) return attr;
        const CUtensorMap *tm = (const CUtensorMap *)T.maps;
        k_sl_tma<0, O><<<gc, kThreads, Box<O>::smem, s>>>(P, M, fn.u, fnm1.u, dt, out.u, ncl, stats, tm[0], tm[3]);
        k_sl_tma<1, O><<<gc, kThreads, Box<O>::smem, s>>>(P, M, fn.v, fnm1.v, dt, out.v, ncl, stats, tm[1], tm[4]);
        if (P.nz > 1)
            k_sl_tma<2, O><<<gw, kThreads, Box<O>::smem, s>>>(P, M, fn.w, fnm1.w, dt, out.w, ncl, stats, tm[2], tm[5]);
        count_launches(P.nz > 1 ? 3 : 2);
        return cudaGetLastError();
    }
}

}  // namespace

int tma_padded_nz(int NZ) { return (NZ + 1) & ~1; }

// Boxes must fit inside the padded arrays in every dimension.
bool tma_supported(const SlcParams &P) { return P.nz + 1 >= kBZ && encode_fn() != nullptr; }

size_t tma_padded_elems(const SlcParams &P, int comp)
{
    const int NZ = comp < 2 ? P.nz + 2 : P.nz + 1;
    return (size_t)(P.nx + kBX) * (P.ny + kBY) * tma_padded_nz(NZ);
}

// Tensor maps of the six padded node copies (slot comp + 3 * which).
cudaError_t tma_encode(const SlcParams &P, TmaSL &T)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    static_assert(sizeof(CUtensorMap) * 6 <= sizeof(T.maps), "tensor-map storage");
    CUtensorMap *tm = (CUtensorMap *)T.maps;
    for (int q = 0; q < 6; ++q) {
        const int comp = q % 3;
        const int NZ = comp < 2 ? P.nz + 2 : P.nz + 1;
        const cuuint64_t nzp = (cuuint64_t)tma_padded_nz(NZ);
        const cuuint64_t dims[3] = {nzp, (cuuint64_t)(P.ny + kBY), (cuuint64_t)(P.nx + kBX)};
        const cuuint64_t strides[2] = {nzp * 8, nzp * 8 * (cuuint64_t)(P.ny + kBY)};
        const bool o4 = P.order == 4;
        const cuuint32_t box[3] = {(cuuint32_t)kBZ, (cuuint32_t)(o4 ? Box<4>::Y : Box<6>::Y),
                                   (cuuint32_t)(o4 ? Box<4>::X : Box<6>::X)};
        const cuuint32_t estr[3] = {1, 1, 1};
        CUresult r = enc(&tm[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)T.pad[q], dims, strides, box,
                         estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}

cudaError_t launch_mid_pack(const SlcParams &P, Tri cur, Tri prev, TriMut mid, const TmaSL &T,
                            cudaStream_t s)
{
    for (int c = 0; c < 3; ++c) {
        const int NZ = c < 2 ? P.nz + 2 : P.nz + 1;
        const int nzp = tma_padded_nz(NZ);
        const long long rows = (long long)(P.nx + kBX) * (P.ny + kBY);
        long long blocks = (rows + 7) / 8;  // 8 warps, one padded row each
        if (blocks > 148 * 16) blocks = 148 * 16;
        const double *a = c == 0 ? cur.u : (c == 1 ? cur.v : cur.w);
        const double *b = c == 0 ? prev.u : (c == 1 ? prev.v : prev.w);
        double *m = c == 0 ? mid.u : (c == 1 ? mid.v : mid.w);
        if (c == 0) k_mid_pack<0><<<(unsigned)blocks, 256, 0, s>>>(P, a, b, 2.0, -1.0, m, T.pad[c], T.pad[c + 3], nzp);
        else if (c == 1) k_mid_pack<1><<<(unsigned)blocks, 256, 0, s>>>(P, a, b, 2.0, -1.0, m, T.pad[c], T.pad[c + 3], nzp);
        else k_mid_pack<2><<<(unsigned)blocks, 256, 0, s>>>(P, a, b, 2.0, -1.0, m, T.pad[c], T.pad[c + 3], nzp);
    }
    count_launches(3);
    return cudaGetLastError();
}

cudaError_t launch_sl_tma(const SlcParams &P, Tri fn, Tri fnm1, Tri mid, double dt, TriMut out,
                          unsigned long long *nclamp, unsigned long long *stats, const TmaSL &T,
                          cudaStream_t s)
{
    Vel3 M;
    M.u = ghost_view<double>(0, mid.u, P.nx, P.ny, P.nz);
    M.v = ghost_view<double>(1, mid.v, P.nx, P.ny, P.nz);
    M.w = ghost_view<double>(2, mid.w, P.nx, P.ny, P.nz);
    if (P.order == 4) return launch_tma_t<4>(P, M, fn, fnm1, dt, out, nclamp, stats, T, s);
    return launch_tma_t<6>(P, M, fn, fnm1, dt, out, nclamp, stats, T, s);
}

// One 3-D tiled tensor map (z innermost, no swizzle, zero fill) over a node
// array: FP32 or FP64 elements, dims (z, y, x), the y and x strides in
// bytes, and the box (z, y, x) in elements.
cudaError_t tma_encode_3d(void *map128, bool fp32, const void *base, const unsigned long long dims[3],
                          const unsigned long long strides[2], const unsigned box[3])
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    const cuuint64_t d[3] = {dims[0], dims[1], dims[2]};
    const cuuint64_t st[2] = {strides[0], strides[1]};
    const cuuint32_t bx[3] = {box[0], box[1], box[2]};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc((CUtensorMap *)map128, fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                     3, const_cast<void *>(base), d, st, bx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}
