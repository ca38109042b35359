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
//   iteration k: E_new(k) on the tile plus the +x column and +y row (those two
//                belong to neighbours and are only recomputed here), store the
//                tile's E_new(k); then H_new(k-1) from E_new(k-1), E_new(k) and
//                H_in(k-1), all on chip.
// Inputs arrive through a cp.async pipeline: while plane k computes, plane
// k+1's H tile (with its 1-cell halo), E and coefficient tiles stream into
// shared memory, so each block always has one plane of loads in flight.  The
// chunk computes E_new(z1) once more than it stores (the next chunk owns it).
// Cells on the outer shell (index 0 or N-1 on any axis) are never updated, as
// in the reference's interior-only update (timefield3d.c:1679-1837); they are
// equal in both buffer sets, so the kernel never writes them.
//
// Arithmetic (FP32, operation order differs from the reference's FP64):
//   E' = ca E + cb (curl_H + dx (psi_a - psi_b) - dx J),  cb = main/dx, ca = 1 when lossless
//   H' = H - hb (curl_E + dx (psi_a - psi_b) + dx M),    hb = dt/dx (mu = 1, no magnetic loss)
// where curl terms are raw neighbour differences scaled by 1/kappa inside the
// CPML slabs and psi' = b psi + a (difference/dx), the same units the split
// kernels and the CPU restatement use, so either path can continue the other.
#include "common.cuh"
#include "kernels.h"

namespace fdtd {

__device__ __forceinline__ float ldg(const float *p) { return __ldg(p); }

// 4-byte asynchronous global -> shared copy; pred false writes 0 and reads nothing
__device__ __forceinline__ void cp_async4(float *smem, const float *gmem, bool pred)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(pred ? 4 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int TX, int TY, bool LOSSY>
struct FusedSmem {
    static constexpr int NC = LOSSY ? 6 : 3;      // coefficient arrays staged
    float h[3][3][TY + 2][TX + 2];                // H_in planes, ring of 3 (k-1, k, k+1), halo -1 .. T
    float eo[2][3][TY + 1][TX + 1];               // E_in planes k, k+1 (tile + the +1 column/row)
    float co[2][NC][TY + 1][TX + 1];              // cb (and ca) planes k, k+1
    float e[2][3][TY + 1][TX + 1];                // E_new planes k-1, k
};

template <int TX, int TY, bool CPML, bool LOSSY>
__global__ void __launch_bounds__(TX *TY)
k_fused_step(FusedArgs a, int zc)
{
    using S = FusedSmem<TX, TY, LOSSY>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S &sm = *reinterpret_cast<S *>(smem_raw);
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long long nxy = (long long)nx * ny;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int X0 = blockIdx.x * TX, Y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, nz);
    if (z0 >= nz) return;
    const float dx = a.dx, hb = a.hb;
    const int L = a.L;
    const float *zero_src = a.f_in[0];   // valid address for zero-fill copies

    // issue the copies of H_in plane k into ring slot k % 3
    auto fetch_h = [&](int k) {
        constexpr int W = TX + 2, H = TY + 2;
        const int slot = (k + 3) % 3;
        const bool kin = k >= 0 && k < nz;
        for (int t = tid; t < W * H; t += TX * TY) {
            const int ly = t / W - 1, lx = t % W - 1;
            const int gi = X0 + lx, gj = Y0 + ly;
            const bool ok = kin && gi >= 0 && gi < nx && gj >= 0 && gj < ny;
            const long long q = ok ? gi + (long long)nx * gj + nxy * k : 0;
#pragma unroll
            for (int c = 0; c < 3; c++)
                cp_async4(&sm.h[slot][c][ly + 1][lx + 1], ok ? a.f_in[3 + c] + q : zero_src, ok);
        }
    };
    // E_in and coefficients of plane k (tile + halo column/row) into slot k % 2
    auto fetch_e = [&](int k) {
        constexpr int W = TX + 1, H = TY + 1;
        const int slot = k & 1;
        const bool kin = k >= 0 && k < nz;
        for (int t = tid; t < W * H; t += TX * TY) {
            const int ly = t / W, lx = t % W;
            const int gi = X0 + lx, gj = Y0 + ly;
            const bool ok = kin && gi < nx && gj < ny;
            const long long q = ok ? gi + (long long)nx * gj + nxy * k : 0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                cp_async4(&sm.eo[slot][c][ly][lx], ok ? a.f_in[c] + q : zero_src, ok);
                cp_async4(&sm.co[slot][c][ly][lx], ok ? a.cb[c] + q : zero_src, ok);
                if (LOSSY) cp_async4(&sm.co[slot][3 + c][ly][lx], ok ? a.ca[c] + q : zero_src, ok);
            }
        }
    };

    // E_new at tile cell (lx, ly) of plane k -> sm.e[k % 2]; store if owned
    auto e_cell = [&](int lx, int ly, int k, bool owned) {
        const int gi = X0 + lx, gj = Y0 + ly;
        const int p3 = k % 3, pm3 = (k + 2) % 3, p2 = k & 1;
        float ex = sm.eo[p2][0][ly][lx], ey = sm.eo[p2][1][ly][lx], ez = sm.eo[p2][2][ly][lx];
        const bool interior = gi >= 1 && gi <= nx - 2 && gj >= 1 && gj <= ny - 2 && k >= 1 && k <= nz - 2;
        if (interior) {
            const long long ij = gi + (long long)nx * gj;
            const int sx = lx + 1, sy = ly + 1;
            const float hx0 = sm.h[p3][0][sy][sx], hy0 = sm.h[p3][1][sy][sx], hz0 = sm.h[p3][2][sy][sx];
            const float dHz_dy = hz0 - sm.h[p3][2][sy - 1][sx];
            const float dHy_dz = hy0 - sm.h[pm3][1][sy][sx];
            const float dHx_dz = hx0 - sm.h[pm3][0][sy][sx];
            const float dHz_dx = hz0 - sm.h[p3][2][sy][sx - 1];
            const float dHy_dx = hy0 - sm.h[p3][1][sy][sx - 1];
            const float dHx_dy = hx0 - sm.h[p3][0][sy - 1][sx];
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
            const float bx = sm.co[p2][0][ly][lx], by = sm.co[p2][1][ly][lx], bz = sm.co[p2][2][ly][lx];
            if (LOSSY) {
                ex = sm.co[p2][3][ly][lx] * ex + bx * cx;
                ey = sm.co[p2][4][ly][lx] * ey + by * cy;
                ez = sm.co[p2][5][ly][lx] * ez + bz * cz;
            } else {
                ex = ex + bx * cx;
                ey = ey + by * cy;
                ez = ez + bz * cz;
            }
            if (owned) {
                const long long q = ij + nxy * k;
                a.f_out[0][q] = ex;
                a.f_out[1][q] = ey;
                a.f_out[2][q] = ez;
            }
        }
        sm.e[p2][0][ly][lx] = ex;
        sm.e[p2][1][ly][lx] = ey;
        sm.e[p2][2][ly][lx] = ez;
    };

    const int gi = X0 + tx, gj = Y0 + ty;
    const bool col_ok = gi >= 1 && gi <= nx - 2 && gj >= 1 && gj <= ny - 2;
    const long long ij = gi + (long long)nx * gj;

    // prologue: H(z0-1), H(z0), E/coefficients(z0)
    fetch_h(z0 - 1);
    fetch_h(z0);
    fetch_e(z0);
    cp_async_commit();
    for (int k = z0; k <= z1; k++) {
        // stream plane k+1 while plane k computes
        if (k + 1 <= z1 && k + 1 < nz) {
            fetch_h(k + 1);
            fetch_e(k + 1);
        }
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        if (k < nz) {
            e_cell(tx, ty, k, k < z1);
            for (int t = tid; t < TX + TY; t += TX * TY) {
                if (t < TY) e_cell(TX, t, k, false);
                else e_cell(t - TY, TY, k, false);
            }
        }
        __syncthreads();
        // H_new(k-1) on the tile
        const int km = k - 1;
        if (km >= z0 && km >= 1 && km <= nz - 2 && col_ok) {
            const int p2 = k & 1, pm2 = p2 ^ 1, pm3 = (k + 2) % 3;
            const int sx = tx + 1, sy = ty + 1;
            const float ex0 = sm.e[pm2][0][ty][tx], ey0 = sm.e[pm2][1][ty][tx], ez0 = sm.e[pm2][2][ty][tx];
            const float dEz_dy = sm.e[pm2][2][ty + 1][tx] - ez0;
            const float dEy_dz = sm.e[p2][1][ty][tx] - ey0;
            const float dEx_dz = sm.e[p2][0][ty][tx] - ex0;
            const float dEz_dx = sm.e[pm2][2][ty][tx + 1] - ez0;
            const float dEy_dx = sm.e[pm2][1][ty][tx + 1] - ey0;
            const float dEx_dy = sm.e[pm2][0][ty + 1][tx] - ex0;
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
            a.f_out[3][q] = sm.h[pm3][0][sy][sx] - hb * cx;
            a.f_out[4][q] = sm.h[pm3][1][sy][sx] - hb * cy;
            a.f_out[5][q] = sm.h[pm3][2][sy][sx] - hb * cz;
        }
        __syncthreads();
    }
    cp_async_wait<0>();
}

constexpr int kFTX = 32, kFTY = 8;

// z-chunk length: every block is resident at once when the tiles fit in the
// SMs' block slots (no partial last wave); large grids fall back to one chunk
// per tile column and full waves.
static int zchunk_for(int nx, int ny, int nz, int slots)
{
    long long tiles = (long long)((nx + kFTX - 1) / kFTX) * ((ny + kFTY - 1) / kFTY);
    long long chunks = slots > 0 ? slots / tiles : 1;
    if (chunks < 1) chunks = 1;
    int zc = (int)((nz + chunks - 1) / chunks);
    if (zc < 8) zc = 8;
    return zc;
}

int fused_supported(int nx, int ny, int nz) { return nx >= 4 && ny >= 4 && nz >= 4; }

template <bool CPML, bool LOSSY>
static void launch_variant(const FusedArgs &a, cudaStream_t st)
{
    auto kern = k_fused_step<kFTX, kFTY, CPML, LOSSY>;
    const size_t smem = sizeof(FusedSmem<kFTX, kFTY, LOSSY>);
    static int slots = -1;
    if (slots < 0) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int per_sm = 0, dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kFTX * kFTY, smem);
        slots = per_sm * sms;
    }
    const int zc = zchunk_for(a.nx, a.ny, a.nz, slots);
    dim3 grid((a.nx + kFTX - 1) / kFTX, (a.ny + kFTY - 1) / kFTY, (a.nz + zc - 1) / zc);
    kern<<<grid, dim3(kFTX, kFTY), smem, st>>>(a, zc);
}

void launch_fused_step(const FusedArgs &a, cudaStream_t st)
{
    note_launch();
    const bool lossy = a.ca[0] != nullptr;
    if (a.L > 0) {
        if (lossy) launch_variant<true, true>(a, st);
        else launch_variant<true, false>(a, st);
    } else {
        if (lossy) launch_variant<false, true>(a, st);
        else launch_variant<false, false>(a, st);
    }
}

}  // namespace fdtd
