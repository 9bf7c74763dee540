// gather_probe.cu -- a measurement, not on the step path: the order-6
// Lagrange gather of an FP32 field (the mixed form's fluctuation gather) done
// two ways on the same synthetic field and feet, for the record of whether
// the tensor cores pay for it.
//   scalar: one thread per point, 216 FP32 loads and FMAs (the mixed
//           kernel's way; 64 registers, four blocks per SM);
//   tensor: the z-contraction of a group of 16 points (8 z x 2 y) as
//           mma.sync m16n8k16 over the union of the group's stencil rows,
//           FP16x3 (fluctuation and weights each split into FP16 hi + lo,
//           hi*hi + hi*lo + lo*hi, FP32 accumulation); the x and y
//           contraction per thread on the accumulator fragments, the sum
//           over rows by warp shuffles.
// Uniform z nodes (integer node coordinates): the loads and the arithmetic
// have the structure of the product gather.  slc_gather_probe allocates its
// own buffers and is synchronous.
#include <cuda_fp16.h>

#include <cstring>
#include <string>

#include "../../include/slc_b200.h"
#include "slc_internal.h"

namespace {

struct ProbeGrid {
    int NX, NY, NZ, NZP, NZH, PZ;  // nodes, FP32 row, FP16 row (>= NZ + 10), points per column
};

__device__ __forceinline__ void foot(const ProbeGrid &G, int i, int j, int k, float &sx, float &sy, float &sz)
{
    // smooth displacements in index units; dy changes sign
    const float dx = 0.3f + 0.1f * __sinf(6.2831853f * (j / 64.f + k / 128.f));
    const float dy = 0.12f * __sinf(6.2831853f * (i / 80.f) + 6.2831853f * k / 90.f);
    const float dz = 0.4f * __sinf(6.2831853f * (i + j) / 70.f) * (float)(k * (G.PZ + 1 - k)) / (0.25f * (G.PZ + 1) * (G.PZ + 1));
    sx = (float)i - dx;
    sy = (float)j - dy;
    sz = (float)(k + 1) - dz;  // arrival at node k+1
}

__device__ __forceinline__ void uw6(float t, float (&w)[6])
{
    // Lagrange weights on offsets -2..3 at t in [0,1)
    const float den[6] = {-120.f, 24.f, -12.f, 12.f, -24.f, 120.f};
    float d[6];
#pragma unroll
    for (int l = 0; l < 6; ++l) d[l] = t - (float)(l - 2);
    float pre[6];
    pre[0] = 1.f;
#pragma unroll
    for (int l = 1; l < 6; ++l) pre[l] = pre[l - 1] * d[l - 1];
    float suf = 1.f;
#pragma unroll
    for (int m = 5; m >= 0; --m) {
        w[m] = pre[m] * suf / den[m];
        suf *= d[m];
    }
}

__device__ __forceinline__ int wrapi(int v, int n) { v %= n; return v < 0 ? v + n : v; }

struct Stn {
    int bx, by, k0;  // first stencil node in each direction (x, y unwrapped)
    float wx[6], wy[6], wz[6];
};

__device__ __forceinline__ void stencil(const ProbeGrid &G, float sx, float sy, float sz, Stn &s)
{
    float fx = floorf(sx), fy = floorf(sy), fz = floorf(sz);
    s.bx = (int)fx - 2;
    s.by = (int)fy - 2;
    int k0 = (int)fz - 2;
    k0 = min(max(k0, 0), G.NZ - 6);
    s.k0 = k0;
    uw6(sx - fx, s.wx);
    uw6(sy - fy, s.wy);
    // z weights on the actual six nodes k0..k0+5 (uniform: offsets from sz)
    float d[6];
#pragma unroll
    for (int l = 0; l < 6; ++l) d[l] = sz - (float)(k0 + l);
    const float den[6] = {-120.f, 24.f, -12.f, 12.f, -24.f, 120.f};
    float pre[6];
    pre[0] = 1.f;
#pragma unroll
    for (int l = 1; l < 6; ++l) pre[l] = pre[l - 1] * d[l - 1];
    float suf = 1.f;
#pragma unroll
    for (int m = 5; m >= 0; --m) {
        s.wz[m] = pre[m] * suf / den[m];
        suf *= d[m];
    }
}

__device__ __forceinline__ float gather_scalar(const ProbeGrid &G, const float *__restrict__ F, const Stn &s)
{
    float acc = 0.f;
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        const int x = wrapi(s.bx + a, G.NX);
        float accy = 0.f;
#pragma unroll
        for (int b = 0; b < 6; ++b) {
            const int y = wrapi(s.by + b, G.NY);
            const float *row = F + ((size_t)x * G.NY + y) * G.NZP + s.k0;
            float accz = 0.f;
#pragma unroll
            for (int c = 0; c < 6; ++c) accz = fmaf(s.wz[c], __ldg(row + c), accz);
            accy = fmaf(s.wy[b], accz, accy);
        }
        acc = fmaf(s.wx[a], accy, acc);
    }
    return acc;
}

// S: block = 64 z x 4 y at one x (as the product kernel)
__global__ void __launch_bounds__(256, 4) k_probe_gather_scalar(const ProbeGrid G, const float *__restrict__ F, float *__restrict__ out)
{
    const int k = blockIdx.x * 64 + (threadIdx.x & 63);
    const int j = blockIdx.y * 4 + (threadIdx.x >> 6);
    const int i = blockIdx.z;
    float sx, sy, sz;
    foot(G, i, j, k, sx, sy, sz);
    Stn s;
    stencil(G, sx, sy, sz, s);
    out[((size_t)i * G.NY + j) * G.PZ + k] = gather_scalar(G, F, s);
}

__device__ __forceinline__ void mma16816(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned pack2(__half lo, __half hi)
{
    return (unsigned)__half_as_ushort(lo) | ((unsigned)__half_as_ushort(hi) << 16);
}

__device__ __forceinline__ float sel6(const float (&w)[6], int q)
{
    float r = 0.f;
#pragma unroll
    for (int m = 0; m < 6; ++m) r = (q == m) ? w[m] : r;
    return r;
}

// T: block = 32 z x 8 y at one x; warp w = 8 z x 4 y (z0 = 8 (w & 3), y0 = 4 (w >> 2));
// lane l: z = z0 + (l & 7), y = y0 + (l >> 3).  Group h (lanes 16h..16h+15) = 8 z x 2 y.
__global__ void __launch_bounds__(256, 2) k_probe_gather_tensor(const ProbeGrid G, const float *__restrict__ F, const __half *__restrict__ Hh,
                                               const __half *__restrict__ Hl, float *__restrict__ out,
                                               unsigned *nfallback)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int k = blockIdx.x * 32 + 8 * (w & 3) + (lane & 7);
    const int j = blockIdx.y * 8 + 4 * (w >> 2) + (lane >> 3);
    const int i = blockIdx.z;
    float sx, sy, sz;
    foot(G, i, j, k, sx, sy, sz);
    Stn s;
    stencil(G, sx, sy, sz, s);
    const int g = lane >> 2, tig = lane & 3;
    float result = 0.f;
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
        // group bounds over lanes 16h..16h+15
        int bxl = s.bx, bxh = s.bx, byl = s.by, byh = s.by, kl = s.k0, kh = s.k0;
#pragma unroll
        for (int m = 1; m < 16; m <<= 1) {
            bxl = min(bxl, __shfl_xor_sync(0xffffffffu, bxl, m));
            bxh = max(bxh, __shfl_xor_sync(0xffffffffu, bxh, m));
            byl = min(byl, __shfl_xor_sync(0xffffffffu, byl, m));
            byh = max(byh, __shfl_xor_sync(0xffffffffu, byh, m));
            kl = min(kl, __shfl_xor_sync(0xffffffffu, kl, m));
            kh = max(kh, __shfl_xor_sync(0xffffffffu, kh, m));
        }
        const int src = 16 * h;
        bxl = __shfl_sync(0xffffffffu, bxl, src);
        bxh = __shfl_sync(0xffffffffu, bxh, src);
        byl = __shfl_sync(0xffffffffu, byl, src);
        byh = __shfl_sync(0xffffffffu, byh, src);
        kl = __shfl_sync(0xffffffffu, kl, src);
        kh = __shfl_sync(0xffffffffu, kh, src);
        const int a = kl & ~1;
        const bool fit = (bxh - bxl) <= 2 && (byh - byl) <= 2 && (kh + 5 - a) <= 15;
        if (!fit) {
            if ((lane >> 4) == h) result = gather_scalar(G, F, s);
            if (lane == 0) atomicAdd(nfallback, 1u);
            continue;
        }
        float acc[2][2] = {{0.f, 0.f}, {0.f, 0.f}};  // [nb][e]
        // B fragments of the two column blocks, and the x/y weights this
        // thread applies: points p = 2 tig + e of column block nb
        unsigned bh[2][2], bl[2][2];
        float wxu[2][2][8], wyg[2][2];
#pragma unroll
        for (int nb = 0; nb < 2; ++nb) {
            const int Lb = 16 * h + 8 * nb + g;  // owner of column g
            float wz[6];
#pragma unroll
            for (int m = 0; m < 6; ++m) wz[m] = __shfl_sync(0xffffffffu, s.wz[m], Lb);
            const int o = __shfl_sync(0xffffffffu, s.k0, Lb) - a;
            float q[4];
            q[0] = sel6(wz, 2 * tig - o);
            q[1] = sel6(wz, 2 * tig + 1 - o);
            q[2] = sel6(wz, 2 * tig + 8 - o);
            q[3] = sel6(wz, 2 * tig + 9 - o);
            __half hq[4], lq[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                hq[r] = __float2half_rn(q[r]);
                lq[r] = __float2half_rn(q[r] - __half2float(hq[r]));
            }
            bh[nb][0] = pack2(hq[0], hq[1]);
            bh[nb][1] = pack2(hq[2], hq[3]);
            bl[nb][0] = pack2(lq[0], lq[1]);
            bl[nb][1] = pack2(lq[2], lq[3]);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int Lp = 16 * h + 8 * nb + 2 * tig + e;
                const float px = __shfl_sync(0xffffffffu, sx, Lp);
                const float py = __shfl_sync(0xffffffffu, sy, Lp);
                const float fx = floorf(px), fy = floorf(py);
                const int ox = (int)fx - 2 - bxl, oy = (int)fy - 2 - byl;
                float wx[6], wy[6];
                uw6(px - fx, wx);
                uw6(py - fy, wy);
#pragma unroll
                for (int ix = 0; ix < 8; ++ix) wxu[nb][e][ix] = sel6(wx, ix - ox);
                wyg[nb][e] = sel6(wy, g - oy);
            }
        }
        // rows: r = ix * 8 + iy; m-block mb holds ix = 2 mb (rows 0-7) and 2 mb + 1 (rows 8-15)
        const int y = wrapi(byl + g, G.NY);
        const int nmb = (bxh - bxl + 6 + 1) / 2;  // x union 6..8 -> 3 or 4 row blocks
#pragma unroll
        for (int mb = 0; mb < 4; ++mb) {
            if (mb < nmb) {
                const int x0 = wrapi(bxl + 2 * mb, G.NX), x1 = wrapi(bxl + 2 * mb + 1, G.NX);
                const size_t r0 = ((size_t)x0 * G.NY + y) * G.NZH + a + 2 * tig;
                const size_t r1 = ((size_t)x1 * G.NY + y) * G.NZH + a + 2 * tig;
                unsigned ah[4], al[4];
                ah[0] = *(const unsigned *)(Hh + r0);
                ah[1] = *(const unsigned *)(Hh + r1);
                ah[2] = *(const unsigned *)(Hh + r0 + 8);
                ah[3] = *(const unsigned *)(Hh + r1 + 8);
                al[0] = *(const unsigned *)(Hl + r0);
                al[1] = *(const unsigned *)(Hl + r1);
                al[2] = *(const unsigned *)(Hl + r0 + 8);
                al[3] = *(const unsigned *)(Hl + r1 + 8);
#pragma unroll
                for (int nb = 0; nb < 2; ++nb) {
                    float c[4] = {0.f, 0.f, 0.f, 0.f};
                    mma16816(c, ah, bh[nb][0], bh[nb][1]);
                    mma16816(c, ah, bl[nb][0], bl[nb][1]);
                    mma16816(c, al, bh[nb][0], bh[nb][1]);
                    // c0,c1: row g (ix 2mb, iy g), points 2tig, 2tig+1; c2,c3: row g+8 (ix 2mb+1)
#pragma unroll
                    for (int e = 0; e < 2; ++e)
                        acc[nb][e] = fmaf(wxu[nb][e][2 * mb], c[e],
                                          fmaf(wxu[nb][e][2 * mb + 1], c[2 + e], acc[nb][e]));
                }
            }
        }
        // y weight of row iy = g, then the sum over g (lanes with the same tig)
        float v[2][2];
#pragma unroll
        for (int nb = 0; nb < 2; ++nb)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                float t = acc[nb][e] * wyg[nb][e];
                t += __shfl_xor_sync(0xffffffffu, t, 4);
                t += __shfl_xor_sync(0xffffffffu, t, 8);
                t += __shfl_xor_sync(0xffffffffu, t, 16);
                v[nb][e] = t;
            }
        // the owner lane 16h + 8nb + n takes point n = 2 tig' + e from lane tig'
        const int n = lane & 7, nbo = (lane >> 3) & 1;
        float r00 = __shfl_sync(0xffffffffu, v[0][0], n >> 1);
        float r01 = __shfl_sync(0xffffffffu, v[0][1], n >> 1);
        float r10 = __shfl_sync(0xffffffffu, v[1][0], n >> 1);
        float r11 = __shfl_sync(0xffffffffu, v[1][1], n >> 1);
        if ((lane >> 4) == h) {
            const float r0 = (n & 1) ? r01 : r00, r1 = (n & 1) ? r11 : r10;
            result = nbo ? r1 : r0;
        }
    }
    out[((size_t)i * G.NY + j) * G.PZ + k] = result;
}

// The synthetic fluctuation field (FP32 rows of NZP, zero padding) and its
// FP16 hi/lo planes (rows of NZH, zero padding).
__global__ void k_probe_field(const ProbeGrid G, float *F, __half *Hh, __half *Hl)
{
    const size_t n = (size_t)G.NX * G.NY * G.NZH;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(t % G.NZH);
        const size_t col = t / G.NZH;
        const int x = (int)(col / G.NY), y = (int)(col % G.NY);
        float v = 0.f;
        if (z < G.NZ)
            v = 0.2f * __sinf(0.11f * x + 0.0007f * y * y + 0.05f * z) + 0.05f * __cosf(0.3f * z + 0.2f * x) +
                0.01f * __sinf(1.7f * x + 2.3f * y + 3.1f * z);
        if (z < G.NZP) F[col * G.NZP + z] = v;
        const __half hv = __float2half_rn(v);
        Hh[t] = hv;
        Hl[t] = __float2half_rn(v - __half2float(hv));
    }
}

// max |a - b| and max |a| (as ordered integer bit patterns of non-negative floats)
__global__ void k_probe_diff(const float *a, const float *b, size_t n, unsigned *res)
{
    unsigned md = 0, ma = 0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        md = max(md, __float_as_uint(fabsf(a[t] - b[t])));
        ma = max(ma, __float_as_uint(fabsf(a[t])));
    }
    atomicMax(res, md);
    atomicMax(res + 1, ma);
}

}  // namespace

extern "C" int slc_gather_probe(int n, int reps, double *out4, void *stream)
{
    if (!out4) return slc_report_error(SLC_E_INVALID, "slc_gather_probe: null output");
    if (n < 64 || n > 256 || n % 64 != 0 || reps < 1)
        return slc_report_error(SLC_E_INVALID, "slc_gather_probe: n must be 64, 128, 192 or 256 and reps >= 1");
    ProbeGrid G;
    G.NX = G.NY = n;
    G.NZ = n + 2;
    G.PZ = n;
    G.NZP = (G.NZ + 3) & ~3;
    G.NZH = G.NZ + 10;
    while (G.NZH % 64 != 8 && G.NZH % 64 != 24 && G.NZH % 64 != 40 && G.NZH % 64 != 56) G.NZH += 2;
    const size_t nF = (size_t)G.NX * G.NY * G.NZP, nH = (size_t)G.NX * G.NY * G.NZH;
    const size_t nO = (size_t)G.NX * G.NY * G.PZ;
    cudaStream_t s = (cudaStream_t)stream;
    float *F = nullptr, *o1 = nullptr, *o2 = nullptr;
    __half *Hh = nullptr, *Hl = nullptr;
    unsigned *cnt = nullptr;
    auto cleanup = [&]() {
        cudaFree(F); cudaFree(o1); cudaFree(o2); cudaFree(Hh); cudaFree(Hl); cudaFree(cnt);
    };
    if (cudaMalloc(&F, nF * 4) != cudaSuccess || cudaMalloc(&o1, nO * 4) != cudaSuccess ||
        cudaMalloc(&o2, nO * 4) != cudaSuccess || cudaMalloc(&Hh, nH * 2) != cudaSuccess ||
        cudaMalloc(&Hl, nH * 2) != cudaSuccess || cudaMalloc(&cnt, 16) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        return slc_report_error(SLC_E_NOMEM, "slc_gather_probe: device allocation failed");
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_probe_field<<<148 * 8, 256, 0, s>>>(G, F, Hh, Hl);
    cudaMemsetAsync(cnt, 0, 16, s);
    const dim3 gs(G.PZ / 64, G.NY / 4, G.NX), gt(G.PZ / 32, G.NY / 8, G.NX);
    k_probe_gather_scalar<<<gs, 256, 0, s>>>(G, F, o1);  // warm-up
    k_probe_gather_tensor<<<gt, 256, 0, s>>>(G, F, Hh, Hl, o2, cnt + 2);
    float ms_s = 0.f, ms_t = 0.f;
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps; ++r) k_probe_gather_scalar<<<gs, 256, 0, s>>>(G, F, o1);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms_s, e0, e1);
    cudaMemsetAsync(cnt + 2, 0, 4, s);
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps; ++r) k_probe_gather_tensor<<<gt, 256, 0, s>>>(G, F, Hh, Hl, o2, cnt + 2);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms_t, e0, e1);
    k_probe_diff<<<148 * 4, 256, 0, s>>>(o1, o2, nO, cnt);
    count_launches(4 + 2 * reps);
    unsigned h[3] = {0, 0, 0};
    cudaError_t err = cudaMemcpyAsync(h, cnt, 12, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err == cudaSuccess) err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cleanup();
    if (err != cudaSuccess)
        return slc_report_error(SLC_E_CUDA, (std::string("slc_gather_probe: ") + cudaGetErrorString(err)).c_str());
    float md, ma;
    memcpy(&md, &h[0], 4);
    memcpy(&ma, &h[1], 4);
    out4[0] = ms_s / reps;
    out4[1] = ms_t / reps;
    out4[2] = ma > 0.f ? (double)md / (double)ma : 0.0;
    out4[3] = (double)h[2] / reps;
    return SLC_OK;
}
