// slc_bc.cuh -- where each ghost element of a ghost-shaped array takes its
// value from (solver.py:70-107; projection.py:180-195 for p).  Every ghost is
// a copy, a negated copy or a zero of ONE interior element, so ghosts can be
// filled in any order and any subset at a time.
#pragma once

#include "slc_common.cuh"

__device__ __host__ inline int n_xghost(int C) { return C == 0 ? 1 : 2; }
__device__ __host__ inline int n_yghost(int C) { return C == 1 ? 1 : 2; }

// true when (I, J, K) is a ghost element of component C (0 u, 1 v, 2 w, 3 p)
__host__ __device__ inline bool bc_is_ghost(int C, int nx, int ny, int nz, int I, int J, int K)
{
    const bool gx = I == 0 || (C != 0 && I == nx + 1);
    const bool gy = J == 0 || (C != 1 && J == ny + 1);
    const bool gz = C == 2 ? (K == 0 || K == nz) : (K == 0 || K == nz + 1);
    return gx || gy || gz;
}

// Source of ghost element (I, J, K): value = sign * f[Is][Js][Ks], or 0.0
// when zero (w on the walls).
struct BcSrc {
    int Is, Js, Ks;
    double sign;
    bool zero;
};

__host__ __device__ inline BcSrc bc_src(int C, int nx, int ny, int nz, int top_neumann, int I, int J, int K)
{
    BcSrc r{I, J, K, 1.0, false};
    // periodic sources in x and y
    if (C == 0) {
        if (I == 0) r.Is = nx;
    } else {
        if (I == 0) r.Is = nx;
        else if (I == nx + 1) r.Is = 1;
    }
    if (C == 1) {
        if (J == 0) r.Js = ny;
    } else {
        if (J == 0) r.Js = ny;
        else if (J == ny + 1) r.Js = 1;
    }
    if (C == 2) {
        if (K == 0 || K == nz) r.zero = true;  // impermeable walls
    } else if (C == 3) {  // pressure: Neumann copies in z
        r.Ks = K == 0 ? 1 : (K == nz + 1 ? nz : K);
    } else if (K == 0) {
        r.Ks = 1;
        r.sign = -1.0;
    } else if (K == nz + 1) {
        r.Ks = nz;
        r.sign = top_neumann ? 1.0 : -1.0;
    }
    return r;
}
