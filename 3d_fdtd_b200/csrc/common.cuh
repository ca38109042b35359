// common.cuh -- device-side types and arithmetic shared by the FDTD kernels.
//
// Layout in HBM: structure of arrays.  Component m (0..5 = Ex Ey Ez Hx Hy Hz)
// of cell (i,j,k) lives at f[m][i + nx*(j + ny*k)]: x is the fastest axis,
// the reference's own axis order (timefield3d.c:1553), so a warp reads 32
// consecutive x cells of one component in one or two 128-byte lines.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fdtd {

// -------------------------------------------------------------------------
// Arithmetic.  The FP64 path reproduces the reference's double arithmetic
// operation for operation: every product and sum is rounded on its own, as
// the reference's x86-64 build computes them (no FMA).  The *_rn intrinsics
// are never contracted by the compiler.  The FP32 path uses plain operators
// and lets the compiler fuse multiply-adds.
// -------------------------------------------------------------------------
template <typename T> struct Ar;

template <> struct Ar<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double sqrt_(double a) { return __dsqrt_rn(a); }
};

template <> struct Ar<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
    static __device__ __forceinline__ float add(float a, float b) { return a + b; }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
    static __device__ __forceinline__ float div(float a, float b) { return a / b; }
    static __device__ __forceinline__ float sqrt_(float a) { return sqrtf(a); }
};

// exact double helpers for host-shaped reductions (always unfused)
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

constexpr int kMaxSourcePlanes = 4;

// Sources are kept as z-planes: a plane at index k holds the six source
// components of every (i,j) of that plane, component-major:
// p[m*nx*ny + i + nx*j].  A full-grid source array would add 24 bytes per
// cell to every step for values that are zero everywhere but one plane.
struct SourcePlanes {
    int n;
    int k[kMaxSourcePlanes];
    const float *p[kMaxSourcePlanes];
};

template <typename T>
struct GridView {
    int nx, ny, nz;
    long long n;
    T *f[6];
    T *old[6];              // Mur snapshot (full grid, only the shell is written)
    const float *ep[3];
    const float *mu[3];
    const float *sig[6];    // null when every value is zero
};

// CPML state.  Slab of axis a holds cells with index in [0,L) or [N-L,N) on
// that axis; psi[a][0..1] are the two E auxiliaries, psi[a][2..3] the two H
// ones, in the component order of the curl terms that differentiate along a:
//   a = x: (Ey, Ez) / (Hy, Hz);  a = y: (Ex, Ez) / (Hx, Hz);  a = z: (Ex, Ey) / (Hx, Hy).
// prof[w][a] are 1-D tables along axis a: w = 0 b_E, 1 a_E, 2 1/kappa_E,
// 3 b_H, 4 a_H, 5 1/kappa_H.
template <typename T>
struct CpmlView {
    int L;
    T *psi[3][4];
    const T *prof[6][3];
};

__device__ __forceinline__ int slab_local(int idx, int N, int L)
{
    return idx < L ? idx : (idx >= N - L ? idx - N + 2 * L : -1);
}

}  // namespace fdtd
