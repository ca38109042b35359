// yee_flat.cu -- FP32 Yee step as two flat, fully parallel kernels.
//
// One thread per cell, no z-loop: the E kernel updates E from H (read-only in
// that kernel), the H kernel updates H from the new E, both in place.  Every
// neighbour a thread reads is also read by the thread next to it, so the
// neighbour loads are served by L1/L2 and DRAM sees each component about once
// per kernel: ~48 B per cell for E (E read + written, H read, 3 coefficients)
// and ~36 B for H, plus the CPML auxiliaries in the slabs.  With tens of
// thousands of blocks in flight the GPU hides memory latency by occupancy,
// which the plane-streaming fused kernels could not (they stay resident
// for a whole z-chunk and stall on each plane's dependency chain).
//
// Arithmetic is the fused kernels' (FP32, raw curl differences):
//   E' = ca E + cb (curl_H + dx (psi_a - psi_b) - dx J)
//   H' = H - hb (curl_E + dx (psi_a - psi_b) + dx M),   hb = dt/dx
// with psi' = b psi + a (difference / dx) inside the CPML slabs, the units of the
// split FP64 kernels and the CPU restatement.
#include "common.cuh"
#include "kernels.h"

namespace fdtd {

constexpr int kFX = 32, kFY = 8;

__device__ __forceinline__ float src_comp(const SourcePlanes &s, int k, int m, long long nxy, long long ij)
{
    for (int t = 0; t < s.n; t++)
        if (s.k[t] == k) return s.p[t][m * nxy + ij];
    return 0.f;
}

template <bool CPML, bool LOSSY>
__global__ void __launch_bounds__(kFX *kFY) k_flat_E(FlatArgs a)
{
    const int i = blockIdx.x * kFX + threadIdx.x;
    const int j = blockIdx.y * kFY + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2 || k < 1 || k > nz - 2) return;
    const long long nxy = (long long)nx * ny;
    const long long ij = i + (long long)nx * j;
    const long long q = ij + nxy * k;
    const float *__restrict__ Hx = a.f[3], *__restrict__ Hy = a.f[4], *__restrict__ Hz = a.f[5];
    const float hx = __ldg(Hx + q), hy = __ldg(Hy + q), hz = __ldg(Hz + q);
    const float dHz_dy = hz - __ldg(Hz + q - nx);
    const float dHy_dz = hy - __ldg(Hy + q - nxy);
    const float dHx_dz = hx - __ldg(Hx + q - nxy);
    const float dHz_dx = hz - __ldg(Hz + q - 1);
    const float dHy_dx = hy - __ldg(Hy + q - 1);
    const float dHx_dy = hx - __ldg(Hx + q - nx);
    const float dx = a.dx;
    float cx, cy, cz;
    if (!CPML) {
        cx = dHz_dy - dHy_dz;
        cy = dHx_dz - dHz_dx;
        cz = dHy_dx - dHx_dy;
    } else {
        const int L = a.L;
        const float div = 1.0f / dx;
        const int si = slab_local(i, nx, L), sj = slab_local(j, ny, L), sk = slab_local(k, nz, L);
        float kx = 1.f, ky = 1.f, kz = 1.f;
        float pxy = 0.f, pxz = 0.f, pyx = 0.f, pyz = 0.f, pzx = 0.f, pzy = 0.f;
        if (si >= 0) {
            const long long s = si + 2LL * L * (j + (long long)ny * k);
            const float b = __ldg(a.prof[0][0] + i), c = __ldg(a.prof[1][0] + i);
            kx = __ldg(a.prof[2][0] + i);
            pyx = b * a.psi[0][0][s] + c * (dHz_dx * div);
            pzx = b * a.psi[0][1][s] + c * (dHy_dx * div);
            a.psi[0][0][s] = pyx;
            a.psi[0][1][s] = pzx;
        }
        if (sj >= 0) {
            const long long s = i + (long long)nx * (sj + 2LL * L * k);
            const float b = __ldg(a.prof[0][1] + j), c = __ldg(a.prof[1][1] + j);
            ky = __ldg(a.prof[2][1] + j);
            pxy = b * a.psi[1][0][s] + c * (dHz_dy * div);
            pzy = b * a.psi[1][1][s] + c * (dHx_dy * div);
            a.psi[1][0][s] = pxy;
            a.psi[1][1][s] = pzy;
        }
        if (sk >= 0) {
            const long long s = ij + nxy * sk;
            const float b = __ldg(a.prof[0][2] + k), c = __ldg(a.prof[1][2] + k);
            kz = __ldg(a.prof[2][2] + k);
            pxz = b * a.psi[2][0][s] + c * (dHy_dz * div);
            pyz = b * a.psi[2][1][s] + c * (dHx_dz * div);
            a.psi[2][0][s] = pxz;
            a.psi[2][1][s] = pyz;
        }
        cx = ky * dHz_dy - kz * dHy_dz + dx * (pxy - pxz);
        cy = kz * dHx_dz - kx * dHz_dx + dx * (pyz - pyx);
        cz = kx * dHy_dx - ky * dHx_dy + dx * (pzx - pzy);
    }
    if (a.src.n) {
        cx -= dx * src_comp(a.src, k, 0, nxy, ij);
        cy -= dx * src_comp(a.src, k, 1, nxy, ij);
        cz -= dx * src_comp(a.src, k, 2, nxy, ij);
    }
    float *__restrict__ Ex = a.f[0], *__restrict__ Ey = a.f[1], *__restrict__ Ez = a.f[2];
    if (LOSSY) {
        Ex[q] = __ldg(a.ca[0] + q) * Ex[q] + __ldg(a.cb[0] + q) * cx;
        Ey[q] = __ldg(a.ca[1] + q) * Ey[q] + __ldg(a.cb[1] + q) * cy;
        Ez[q] = __ldg(a.ca[2] + q) * Ez[q] + __ldg(a.cb[2] + q) * cz;
    } else {
        Ex[q] = Ex[q] + __ldg(a.cb[0] + q) * cx;
        Ey[q] = Ey[q] + __ldg(a.cb[1] + q) * cy;
        Ez[q] = Ez[q] + __ldg(a.cb[2] + q) * cz;
    }
}

template <bool CPML>
__global__ void __launch_bounds__(kFX *kFY) k_flat_H(FlatArgs a)
{
    const int i = blockIdx.x * kFX + threadIdx.x;
    const int j = blockIdx.y * kFY + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2 || k < 1 || k > nz - 2) return;
    const long long nxy = (long long)nx * ny;
    const long long ij = i + (long long)nx * j;
    const long long q = ij + nxy * k;
    const float *__restrict__ Ex = a.f[0], *__restrict__ Ey = a.f[1], *__restrict__ Ez = a.f[2];
    const float ex = __ldg(Ex + q), ey = __ldg(Ey + q), ez = __ldg(Ez + q);
    const float dEz_dy = __ldg(Ez + q + nx) - ez;
    const float dEy_dz = __ldg(Ey + q + nxy) - ey;
    const float dEx_dz = __ldg(Ex + q + nxy) - ex;
    const float dEz_dx = __ldg(Ez + q + 1) - ez;
    const float dEy_dx = __ldg(Ey + q + 1) - ey;
    const float dEx_dy = __ldg(Ex + q + nx) - ex;
    const float dx = a.dx;
    float cx, cy, cz;
    if (!CPML) {
        cx = dEz_dy - dEy_dz;
        cy = dEx_dz - dEz_dx;
        cz = dEy_dx - dEx_dy;
    } else {
        const int L = a.L;
        const float div = 1.0f / dx;
        const int si = slab_local(i, nx, L), sj = slab_local(j, ny, L), sk = slab_local(k, nz, L);
        float kx = 1.f, ky = 1.f, kz = 1.f;
        float pxy = 0.f, pxz = 0.f, pyx = 0.f, pyz = 0.f, pzx = 0.f, pzy = 0.f;
        if (si >= 0) {
            const long long s = si + 2LL * L * (j + (long long)ny * k);
            const float b = __ldg(a.prof[3][0] + i), c = __ldg(a.prof[4][0] + i);
            kx = __ldg(a.prof[5][0] + i);
            pyx = b * a.psi[0][2][s] + c * (dEz_dx * div);
            pzx = b * a.psi[0][3][s] + c * (dEy_dx * div);
            a.psi[0][2][s] = pyx;
            a.psi[0][3][s] = pzx;
        }
        if (sj >= 0) {
            const long long s = i + (long long)nx * (sj + 2LL * L * k);
            const float b = __ldg(a.prof[3][1] + j), c = __ldg(a.prof[4][1] + j);
            ky = __ldg(a.prof[5][1] + j);
            pxy = b * a.psi[1][2][s] + c * (dEz_dy * div);
            pzy = b * a.psi[1][3][s] + c * (dEx_dy * div);
            a.psi[1][2][s] = pxy;
            a.psi[1][3][s] = pzy;
        }
        if (sk >= 0) {
            const long long s = ij + nxy * sk;
            const float b = __ldg(a.prof[3][2] + k), c = __ldg(a.prof[4][2] + k);
            kz = __ldg(a.prof[5][2] + k);
            pxz = b * a.psi[2][2][s] + c * (dEy_dz * div);
            pyz = b * a.psi[2][3][s] + c * (dEx_dz * div);
            a.psi[2][2][s] = pxz;
            a.psi[2][3][s] = pyz;
        }
        cx = ky * dEz_dy - kz * dEy_dz + dx * (pxy - pxz);
        cy = kz * dEx_dz - kx * dEz_dx + dx * (pyz - pyx);
        cz = kx * dEy_dx - ky * dEx_dy + dx * (pzx - pzy);
    }
    if (a.src.n) {
        cx += dx * src_comp(a.src, k, 3, nxy, ij);
        cy += dx * src_comp(a.src, k, 4, nxy, ij);
        cz += dx * src_comp(a.src, k, 5, nxy, ij);
    }
    float *__restrict__ Hx = a.f[3], *__restrict__ Hy = a.f[4], *__restrict__ Hz = a.f[5];
    const float hb = a.hb;
    Hx[q] = Hx[q] - hb * cx;
    Hy[q] = Hy[q] - hb * cy;
    Hz[q] = Hz[q] - hb * cz;
}

void launch_flat_step(const FlatArgs &a, cudaStream_t st, cudaEvent_t mid)
{
    dim3 grid((a.nx + kFX - 1) / kFX, (a.ny + kFY - 1) / kFY, a.nz), block(kFX, kFY);
    const bool cpml = a.L > 0, lossy = a.ca[0] != nullptr;
    note_launch(2);
    if (cpml) {
        if (lossy) k_flat_E<true, true><<<grid, block, 0, st>>>(a);
        else k_flat_E<true, false><<<grid, block, 0, st>>>(a);
        k_flat_H<true><<<grid, block, 0, st>>>(a);
    } else {
        if (lossy) k_flat_E<false, true><<<grid, block, 0, st>>>(a);
        else k_flat_E<false, false><<<grid, block, 0, st>>>(a);
        k_flat_H<false><<<grid, block, 0, st>>>(a);
    }
    (void)mid;
}

}  // namespace fdtd
