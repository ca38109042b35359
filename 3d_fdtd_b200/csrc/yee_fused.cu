// yee_fused.cu -- FP32 single-pass Yee step: E^{n+1} and H^{n+1/2} in one
// kernel launch per time step.
//
// Why fused: the split E and H kernels each read the other field set, so a step
// moves ~84 B per cell plus coefficients; one pass that keeps the freshly
// computed E plane on chip for the H update moves 60 B per cell (6 components
// read and written once, 3 E coefficients read), the algorithmic minimum.
//
// Data flow.  Fields ping-pong between two buffer sets (read `in`, write
// `out`), so blocks never race on a neighbour's halo.  A block owns a TX x TY
// tile of (x, y) columns and a chunk [z0, z1) of z planes and streams along z:
//   iteration k: load H_in(k) (tile + 1-cell halo on every side) into shared
//                memory; compute E_new(k) on the tile plus the +x column and
//                +y row (those two are owned by neighbours and only recomputed
//                here); store the owned E_new(k); then compute H_new(k-1) from
//                E_new(k-1), E_new(k) and H_in(k-1), all on chip.
// The chunk computes E_new(z1) once more than it stores (the next chunk owns
// it).  Cells on the outer shell (index 0 or N-1 on any axis) are never updated,
// as in the reference's interior-only update (timefield3d.c:1679-1837); they
// are equal in both buffer sets, so the kernel never writes them.
//
// Arithmetic (FP32, reference operation order not required):
//   E' = ca E + cb (curl_H + dx (psi_a - psi_b) - dx J),  cb = main/dx, ca = 1 when lossless
//   H' = H - hb (curl_E + dx (psi_a - psi_b) + dx M),    hb = dt/dx (mu = 1, no magnetic loss)
// where curl terms are raw neighbour differences scaled by 1/kappa inside the
// CPML slabs and psi' = b psi + a (difference/dx), the same units the split
// kernels and the CPU restatement use, so either path can continue the other.
#include "common.cuh"
#include "kernels.h"

namespace fdtd {

template <int TX, int TY>
struct FusedSmem {
    float h[2][3][TY + 2][TX + 2];   // H_in planes k-1 / k, halo -1 .. T on both axes
    float e[2][3][TY + 1][TX + 1];   // E_new planes k-1 / k, tile + the +1 column / row
};

__device__ __forceinline__ float ldg(const float *p) { return __ldg(p); }

template <int TX, int TY, bool CPML, bool LOSSY>
__global__ void __launch_bounds__(TX *TY)
k_fused_step(FusedArgs a, int zc)
{
    __shared__ FusedSmem<TX, TY> sm;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long long nxy = (long long)nx * ny;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int X0 = blockIdx.x * TX, Y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, nz);
    if (z0 >= nz) return;
    const float dx = a.dx, hb = a.hb;
    const int L = a.L;

    // H_in plane k (tile + halo) -> sm.h[p]
    auto load_h = [&](int k, int p) {
        constexpr int W = TX + 2, H = TY + 2;
        for (int t = tid; t < W * H; t += TX * TY) {
            int ly = t / W - 1, lx = t % W - 1;
            int gi = X0 + lx, gj = Y0 + ly;
            float hx = 0.f, hy = 0.f, hz = 0.f;
            if (k >= 0 && k < nz && gi >= 0 && gi < nx && gj >= 0 && gj < ny) {
                long long q = gi + (long long)nx * gj + nxy * k;
                hx = ldg(a.f_in[3] + q);
                hy = ldg(a.f_in[4] + q);
                hz = ldg(a.f_in[5] + q);
            }
            sm.h[p][0][ly + 1][lx + 1] = hx;
            sm.h[p][1][ly + 1][lx + 1] = hy;
            sm.h[p][2][ly + 1][lx + 1] = hz;
        }
    };

    // E_new at tile cell (lx, ly) of plane k -> sm.e[p]; store if owned
    auto e_cell = [&](int lx, int ly, int k, int p, bool owned) {
        const int gi = X0 + lx, gj = Y0 + ly;
        float ex = 0.f, ey = 0.f, ez = 0.f;
        if (gi < nx && gj < ny) {
            const long long ij = gi + (long long)nx * gj;
            const long long q = ij + nxy * k;
            ex = ldg(a.f_in[0] + q);
            ey = ldg(a.f_in[1] + q);
            ez = ldg(a.f_in[2] + q);
            const bool interior = gi >= 1 && gi <= nx - 2 && gj >= 1 && gj <= ny - 2 && k >= 1 && k <= nz - 2;
            if (interior) {
                const int pm = p ^ 1;
                const int sx = lx + 1, sy = ly + 1;
                float hx0 = sm.h[p][0][sy][sx], hy0 = sm.h[p][1][sy][sx], hz0 = sm.h[p][2][sy][sx];
                float dHz_dy = hz0 - sm.h[p][2][sy - 1][sx];
                float dHy_dz = hy0 - sm.h[pm][1][sy][sx];
                float dHx_dz = hx0 - sm.h[pm][0][sy][sx];
                float dHz_dx = hz0 - sm.h[p][2][sy][sx - 1];
                float dHy_dx = hy0 - sm.h[p][1][sy][sx - 1];
                float dHx_dy = hx0 - sm.h[p][0][sy - 1][sx];
                float cx, cy, cz;
                if (!CPML) {
                    cx = dHz_dy - dHy_dz;
                    cy = dHx_dz - dHz_dx;
                    cz = dHy_dx - dHx_dy;
                } else {
                    const float div = 1.0f / dx;
                    const int si = slab_local(gi, nx, L), sj = slab_local(gj, ny, L), sk = slab_local(k, nz, L);
                    float kx = 1.f, ky = 1.f, kz = 1.f;
                    float pxy = 0.f, pxz = 0.f, pyx = 0.f, pyz = 0.f, pzx = 0.f, pzy = 0.f;
                    if (si >= 0) {
                        const long long s = si + 2LL * L * (gj + (long long)ny * k);
                        const float b = ldg(a.prof[0][0] + gi), c = ldg(a.prof[1][0] + gi);
                        kx = ldg(a.prof[2][0] + gi);
                        pyx = b * ldg(a.psi_in[0][0] + s) + c * (dHz_dx * div);
                        pzx = b * ldg(a.psi_in[0][1] + s) + c * (dHy_dx * div);
                        if (owned) { a.psi_out[0][0][s] = pyx; a.psi_out[0][1][s] = pzx; }
                    }
                    if (sj >= 0) {
                        const long long s = gi + (long long)nx * (sj + 2LL * L * k);
                        const float b = ldg(a.prof[0][1] + gj), c = ldg(a.prof[1][1] + gj);
                        ky = ldg(a.prof[2][1] + gj);
                        pxy = b * ldg(a.psi_in[1][0] + s) + c * (dHz_dy * div);
                        pzy = b * ldg(a.psi_in[1][1] + s) + c * (dHx_dy * div);
                        if (owned) { a.psi_out[1][0][s] = pxy; a.psi_out[1][1][s] = pzy; }
                    }
                    if (sk >= 0) {
                        const long long s = ij + nxy * sk;
                        const float b = ldg(a.prof[0][2] + k), c = ldg(a.prof[1][2] + k);
                        kz = ldg(a.prof[2][2] + k);
                        pxz = b * ldg(a.psi_in[2][0] + s) + c * (dHy_dz * div);
                        pyz = b * ldg(a.psi_in[2][1] + s) + c * (dHx_dz * div);
                        if (owned) { a.psi_out[2][0][s] = pxz; a.psi_out[2][1][s] = pyz; }
                    }
                    cx = ky * dHz_dy - kz * dHy_dz + dx * (pxy - pxz);
                    cy = kz * dHx_dz - kx * dHz_dx + dx * (pyz - pyx);
                    cz = kx * dHy_dx - ky * dHx_dy + dx * (pzx - pzy);
                }
                for (int t = 0; t < a.src.n; t++)
                    if (a.src.k[t] == k) {
                        const float *sp = a.src.p[t];
                        cx -= dx * sp[ij];
                        cy -= dx * sp[nxy + ij];
                        cz -= dx * sp[2 * nxy + ij];
                    }
                const float bx = ldg(a.cb[0] + q), by = ldg(a.cb[1] + q), bz = ldg(a.cb[2] + q);
                if (LOSSY) {
                    ex = ldg(a.ca[0] + q) * ex + bx * cx;
                    ey = ldg(a.ca[1] + q) * ey + by * cy;
                    ez = ldg(a.ca[2] + q) * ez + bz * cz;
                } else {
                    ex = ex + bx * cx;
                    ey = ey + by * cy;
                    ez = ez + bz * cz;
                }
                if (owned) {
                    a.f_out[0][q] = ex;
                    a.f_out[1][q] = ey;
                    a.f_out[2][q] = ez;
                }
            }
        }
        sm.e[p][0][ly][lx] = ex;
        sm.e[p][1][ly][lx] = ey;
        sm.e[p][2][ly][lx] = ez;
    };

    const int gi = X0 + tx, gj = Y0 + ty;
    const bool col_in = gi < nx && gj < ny;
    const bool col_interior = gi >= 1 && gi <= nx - 2 && gj >= 1 && gj <= ny - 2;
    const long long ij = gi + (long long)nx * gj;

    load_h(z0 - 1, (z0 - 1) & 1);
    for (int k = z0; k <= z1; k++) {
        const int p = k & 1, pm = p ^ 1;
        if (k < nz) load_h(k, p);
        __syncthreads();
        if (k < nz) {
            // the tile (stored when k is this chunk's), then the +x column and +y row
            e_cell(tx, ty, k, p, k < z1);
            for (int t = tid; t < TX + TY; t += TX * TY) {
                if (t < TY) e_cell(TX, t, k, p, false);
                else e_cell(t - TY, TY, k, p, false);
            }
        }
        __syncthreads();
        // H_new(k-1) on the tile
        const int km = k - 1;
        if (km >= z0 && km >= 1 && km <= nz - 2 && col_in && col_interior) {
            const int sx = tx + 1, sy = ty + 1;
            float ex0 = sm.e[pm][0][ty][tx], ey0 = sm.e[pm][1][ty][tx], ez0 = sm.e[pm][2][ty][tx];
            float dEz_dy = sm.e[pm][2][ty + 1][tx] - ez0;
            float dEy_dz = sm.e[p][1][ty][tx] - ey0;
            float dEx_dz = sm.e[p][0][ty][tx] - ex0;
            float dEz_dx = sm.e[pm][2][ty][tx + 1] - ez0;
            float dEy_dx = sm.e[pm][1][ty][tx + 1] - ey0;
            float dEx_dy = sm.e[pm][0][ty + 1][tx] - ex0;
            float cx, cy, cz;
            if (!CPML) {
                cx = dEz_dy - dEy_dz;
                cy = dEx_dz - dEz_dx;
                cz = dEy_dx - dEx_dy;
            } else {
                const float div = 1.0f / dx;
                const int si = slab_local(gi, nx, L), sj = slab_local(gj, ny, L), sk = slab_local(km, nz, L);
                float kx = 1.f, ky = 1.f, kz = 1.f;
                float pxy = 0.f, pxz = 0.f, pyx = 0.f, pyz = 0.f, pzx = 0.f, pzy = 0.f;
                if (si >= 0) {
                    const long long s = si + 2LL * L * (gj + (long long)ny * km);
                    const float b = ldg(a.prof[3][0] + gi), c = ldg(a.prof[4][0] + gi);
                    kx = ldg(a.prof[5][0] + gi);
                    pyx = b * ldg(a.psi_in[0][2] + s) + c * (dEz_dx * div);
                    pzx = b * ldg(a.psi_in[0][3] + s) + c * (dEy_dx * div);
                    a.psi_out[0][2][s] = pyx;
                    a.psi_out[0][3][s] = pzx;
                }
                if (sj >= 0) {
                    const long long s = gi + (long long)nx * (sj + 2LL * L * km);
                    const float b = ldg(a.prof[3][1] + gj), c = ldg(a.prof[4][1] + gj);
                    ky = ldg(a.prof[5][1] + gj);
                    pxy = b * ldg(a.psi_in[1][2] + s) + c * (dEz_dy * div);
                    pzy = b * ldg(a.psi_in[1][3] + s) + c * (dEx_dy * div);
                    a.psi_out[1][2][s] = pxy;
                    a.psi_out[1][3][s] = pzy;
                }
                if (sk >= 0) {
                    const long long s = ij + nxy * sk;
                    const float b = ldg(a.prof[3][2] + km), c = ldg(a.prof[4][2] + km);
                    kz = ldg(a.prof[5][2] + km);
                    pxz = b * ldg(a.psi_in[2][2] + s) + c * (dEy_dz * div);
                    pyz = b * ldg(a.psi_in[2][3] + s) + c * (dEx_dz * div);
                    a.psi_out[2][2][s] = pxz;
                    a.psi_out[2][3][s] = pyz;
                }
                cx = ky * dEz_dy - kz * dEy_dz + dx * (pxy - pxz);
                cy = kz * dEx_dz - kx * dEz_dx + dx * (pyz - pyx);
                cz = kx * dEy_dx - ky * dEx_dy + dx * (pzx - pzy);
            }
            for (int t = 0; t < a.src.n; t++)
                if (a.src.k[t] == km) {
                    const float *sp = a.src.p[t];
                    cx += dx * sp[3 * nxy + ij];
                    cy += dx * sp[4 * nxy + ij];
                    cz += dx * sp[5 * nxy + ij];
                }
            const long long q = ij + nxy * km;
            a.f_out[3][q] = sm.h[pm][0][sy][sx] - hb * cx;
            a.f_out[4][q] = sm.h[pm][1][sy][sx] - hb * cy;
            a.f_out[5][q] = sm.h[pm][2][sy][sx] - hb * cz;
        }
        __syncthreads();
    }
}

// tile shape and z-chunk; chosen so the grid covers the 148 SMs several times
constexpr int kFTX = 32, kFTY = 8;

static int zchunk_for(int nx, int ny, int nz)
{
    long long tiles = (long long)((nx + kFTX - 1) / kFTX) * ((ny + kFTY - 1) / kFTY);
    // aim for ~8 resident-block waves worth of blocks, chunks of >= 16 planes
    long long want = 148LL * 8;
    long long chunks = (want + tiles - 1) / tiles;
    if (chunks < 1) chunks = 1;
    int zc = (int)((nz + chunks - 1) / chunks);
    if (zc < 16) zc = 16;
    return zc;
}

int fused_supported(int nx, int ny, int nz) { return nx >= 4 && ny >= 4 && nz >= 4; }

void launch_fused_step(const FusedArgs &a, cudaStream_t st)
{
    const int zc = zchunk_for(a.nx, a.ny, a.nz);
    dim3 grid((a.nx + kFTX - 1) / kFTX, (a.ny + kFTY - 1) / kFTY, (a.nz + zc - 1) / zc);
    dim3 block(kFTX, kFTY);
    note_launch();
    const bool lossy = a.ca[0] != nullptr;
    if (a.L > 0) {
        if (lossy) k_fused_step<kFTX, kFTY, true, true><<<grid, block, 0, st>>>(a, zc);
        else k_fused_step<kFTX, kFTY, true, false><<<grid, block, 0, st>>>(a, zc);
    } else {
        if (lossy) k_fused_step<kFTX, kFTY, false, true><<<grid, block, 0, st>>>(a, zc);
        else k_fused_step<kFTX, kFTY, false, false><<<grid, block, 0, st>>>(a, zc);
    }
}

}  // namespace fdtd
