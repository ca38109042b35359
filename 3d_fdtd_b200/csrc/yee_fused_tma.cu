// yee_fused_tma.cu -- the FP32 single-pass Yee step with TMA staging.
//
// Same data flow and arithmetic as yee_fused.cu (see there), but every input
// tile of a z-plane is brought into shared memory by the tensor memory
// accelerator: one thread issues, per plane, three H boxes (tile plus a 1-cell
// halo on every side, hardware zero fill outside the grid), three E boxes and
// three (six if lossy) coefficient boxes, all completing on one mbarrier.  A
// ring of three plane stages (k-1, k, k+1) keeps the next plane's copies in
// flight while plane k computes.  This removes the per-element copy issue that
// made the cp.async variant instruction-bound.
//
// TMA rules observed: every box starts at an x coordinate that is a multiple
// of 4 floats (16 bytes), so the H box starts at X0-4 and is TX+8 wide; strides
// are multiples of 16 bytes, which needs nx % 4 == 0 (other widths use the
// cp.async kernel).  Loads only (no TMA stores), no multicast.
//
// Waits on the mbarriers are bounded.  A wait that gives up sets the grid's
// device error flag and a block-wide abort flag; the block then finishes its
// loop without waiting (results are garbage, the host reports
// FDTD_ERR_TIMEOUT) instead of hanging.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "kernels.h"

namespace fdtd {

constexpr int TX = 32, TY = 8;
constexpr int HW = TX + 8;   // H box width: x from X0-4 to X0+TX+3
constexpr int EW = TX + 4;   // E / coefficient box width: x from X0 to X0+TX+3
constexpr int HOFF = 4;      // smem x index of tile column 0 in an H box
constexpr unsigned kWaitLimit = 1u << 22;

// every TMA destination starts on a 128-byte boundary: box buffers are padded
constexpr int pad128f(int nfloats) { return ((nfloats * 4 + 127) / 128) * 32; }
constexpr int HBOX = (TY + 2) * HW, EBOX = (TY + 1) * EW;
constexpr int HBOXP = pad128f(HBOX), EBOXP = pad128f(EBOX);

template <bool LOSSY>
struct alignas(128) TmaStage {
    static constexpr int NC = LOSSY ? 6 : 3;
    float h[3][HBOXP];     // H box c: [TY+2][HW], x fastest
    float e[3][EBOXP];     // E box c: [TY+1][EW]
    float c[NC][EBOXP];    // cb (and ca) boxes
    static constexpr unsigned kBytes = 3u * HBOX * 4 + (3u + NC) * EBOX * 4;
};
static_assert((HBOXP * 4) % 128 == 0 && (EBOXP * 4) % 128 == 0, "TMA box buffers must keep 128-byte alignment");

template <bool LOSSY>
struct TmaSmem {
    TmaStage<LOSSY> st[3];
    float en[2][3][TY + 1][TX + 1];   // E_new planes k-1, k
    unsigned long long bar[3];
    int abort;
};
// dynamic shared memory requested: the struct plus room to align its base to 128 bytes
template <bool LOSSY> constexpr size_t tma_smem_bytes() { return sizeof(TmaSmem<LOSSY>) + 128; }

__device__ __forceinline__ float Hat(const float *box, int lx, int ly) { return box[(ly + 1) * HW + lx + HOFF]; }
__device__ __forceinline__ float Eat(const float *box, int lx, int ly) { return box[ly * EW + lx]; }

// ---- PTX wrappers ----------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// ---- per-cell CPML data along x or y (loop invariant for a column) ---------
struct SlabE {
    long long base;   // psi index without the k term, or -1 outside the slab
    float b, a, kinv;
};

template <bool LOSSY>
__device__ __forceinline__ void issue_plane(TmaSmem<LOSSY> &sm, const FusedMaps &m, int k, int X0, int Y0)
{
    const int slot = (k + 3) % 3;
    TmaStage<LOSSY> &s = sm.st[slot];
    unsigned long long *bar = &sm.bar[slot];
    fence_async_shared();
    mbar_expect_tx(bar, TmaStage<LOSSY>::kBytes);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        tma_load_3d(&s.h[c][0], &m.h[c], X0 - HOFF, Y0 - 1, k, bar);
        tma_load_3d(&s.e[c][0], &m.e[c], X0, Y0, k, bar);
        tma_load_3d(&s.c[c][0], &m.cb[c], X0, Y0, k, bar);
        if (LOSSY) tma_load_3d(&s.c[3 + c][0], &m.ca[c], X0, Y0, k, bar);
    }
}

// true when every TMA destination is 128-byte aligned and every mbarrier 8-byte aligned
template <bool LOSSY>
__device__ __forceinline__ bool tma_layout_ok(const TmaSmem<LOSSY> &sm)
{
    for (int s = 0; s < 3; s++) {
        for (int c = 0; c < 3; c++)
            if ((smem_u32(&sm.st[s].h[c][0]) & 127u) || (smem_u32(&sm.st[s].e[c][0]) & 127u)) return false;
        for (int c = 0; c < TmaStage<LOSSY>::NC; c++)
            if (smem_u32(&sm.st[s].c[c][0]) & 127u) return false;
        if (smem_u32(&sm.bar[s]) & 7u) return false;
    }
    return true;
}

template <bool LOSSY>
__device__ __forceinline__ void wait_plane(TmaSmem<LOSSY> &sm, int k, int z0, int *err)
{
    const int slot = (k + 3) % 3;
    const unsigned parity = (unsigned)(((k - z0 + 1) / 3) & 1);
    volatile int *abort = &sm.abort;
    for (unsigned it = 0; it < kWaitLimit; it++) {
        if (*abort) return;   // checked first: after a refused start the barriers were never set up
        if (mbar_try_wait(&sm.bar[slot], parity)) return;
    }
    *abort = 1;
    atomicExch(err, 1);
}

template <bool CPML, bool LOSSY>
__global__ void __launch_bounds__(TX *TY)
k_fused_tma(FusedArgs a, const __grid_constant__ FusedMaps maps, int zc, int *err)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // align the base explicitly: TMA destinations need 128-byte alignment
    const unsigned pad = (128u - (smem_u32(smem_raw) & 127u)) & 127u;
    TmaSmem<LOSSY> &sm = *reinterpret_cast<TmaSmem<LOSSY> *>(smem_raw + pad);
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long long nxy = (long long)nx * ny;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int X0 = blockIdx.x * TX, Y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, nz);
    if (z0 >= nz) return;
    const float dx = a.dx, hb = a.hb, div = 1.0f / a.dx;
    const int L = a.L;

    if (tid == 0) {
        // self-check before any copy is issued: a misaligned destination would
        // fault, so refuse (error flag, abort) instead
        const bool layout_ok = tma_layout_ok<LOSSY>(sm);
        if (layout_ok)
            for (int s = 0; s < 3; s++) mbar_init(&sm.bar[s], 1);
        sm.abort = layout_ok ? 0 : 1;
        if (!layout_ok) atomicExch(err, 2);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    const bool live = sm.abort == 0;
    if (tid == 0 && live) {
        issue_plane<LOSSY>(sm, maps, z0 - 1, X0, Y0);
        issue_plane<LOSSY>(sm, maps, z0, X0, Y0);
    }

    // loop-invariant per-column data of this thread's tile cell
    const int gi = X0 + tx, gj = Y0 + ty;
    const bool col_ok = gi >= 1 && gi <= nx - 2 && gj >= 1 && gj <= ny - 2;
    const long long ij = gi + (long long)nx * gj;
    SlabE ex_{-1, 1.f, 0.f, 1.f}, ey_{-1, 1.f, 0.f, 1.f}, hx_{-1, 1.f, 0.f, 1.f}, hy_{-1, 1.f, 0.f, 1.f};
    if (CPML && col_ok) {
        const int si = slab_local(gi, nx, L), sj = slab_local(gj, ny, L);
        if (si >= 0) {
            ex_ = {si + 2LL * L * gj, __ldg(a.prof[0][0] + gi), __ldg(a.prof[1][0] + gi), __ldg(a.prof[2][0] + gi)};
            hx_ = {si + 2LL * L * gj, __ldg(a.prof[3][0] + gi), __ldg(a.prof[4][0] + gi), __ldg(a.prof[5][0] + gi)};
        }
        if (sj >= 0) {
            ey_ = {gi + (long long)nx * sj, __ldg(a.prof[0][1] + gj), __ldg(a.prof[1][1] + gj), __ldg(a.prof[2][1] + gj)};
            hy_ = {gi + (long long)nx * sj, __ldg(a.prof[3][1] + gj), __ldg(a.prof[4][1] + gj), __ldg(a.prof[5][1] + gj)};
        }
    }
    const long long xstride = 2LL * L * ny;     // psi x-slab stride per z plane
    const long long ystride = (long long)nx * 2 * L;

    // E_new at tile cell (lx, ly) of plane k (slot p3, previous H plane in pm3)
    auto e_cell = [&](int lx, int ly, int k, bool owned, const SlabE &sx, const SlabE &sy) {
        const int ggi = X0 + lx, ggj = Y0 + ly;
        const int p3 = k % 3, pm3 = (k + 2) % 3, p2 = k & 1;
        const TmaStage<LOSSY> &S = sm.st[p3];
        float ex = Eat(S.e[0], lx, ly), ey = Eat(S.e[1], lx, ly), ez = Eat(S.e[2], lx, ly);
        const bool interior = ggi >= 1 && ggi <= nx - 2 && ggj >= 1 && ggj <= ny - 2 && k >= 1 && k <= nz - 2;
        if (interior) {
            const TmaStage<LOSSY> &Sm = sm.st[pm3];
            const float hx0 = Hat(S.h[0], lx, ly), hy0 = Hat(S.h[1], lx, ly), hz0 = Hat(S.h[2], lx, ly);
            const float dHz_dy = hz0 - Hat(S.h[2], lx, ly - 1);
            const float dHy_dz = hy0 - Hat(Sm.h[1], lx, ly);
            const float dHx_dz = hx0 - Hat(Sm.h[0], lx, ly);
            const float dHz_dx = hz0 - Hat(S.h[2], lx - 1, ly);
            const float dHy_dx = hy0 - Hat(S.h[1], lx - 1, ly);
            const float dHx_dy = hx0 - Hat(S.h[0], lx, ly - 1);
            float cx, cy, cz;
            const long long cij = ggi + (long long)nx * ggj;
            if (!CPML) {
                cx = dHz_dy - dHy_dz;
                cy = dHx_dz - dHz_dx;
                cz = dHy_dx - dHx_dy;
            } else {
                float pxy = 0.f, pxz = 0.f, pyx = 0.f, pyz = 0.f, pzx = 0.f, pzy = 0.f, kz = 1.f;
                if (sx.base >= 0) {
                    const long long s = sx.base + xstride * k;
                    pyx = sx.b * __ldg(a.psi_in[0][0] + s) + sx.a * (dHz_dx * div);
                    pzx = sx.b * __ldg(a.psi_in[0][1] + s) + sx.a * (dHy_dx * div);
                    if (owned) { a.psi_out[0][0][s] = pyx; a.psi_out[0][1][s] = pzx; }
                }
                if (sy.base >= 0) {
                    const long long s = sy.base + ystride * k;
                    pxy = sy.b * __ldg(a.psi_in[1][0] + s) + sy.a * (dHz_dy * div);
                    pzy = sy.b * __ldg(a.psi_in[1][1] + s) + sy.a * (dHx_dy * div);
                    if (owned) { a.psi_out[1][0][s] = pxy; a.psi_out[1][1][s] = pzy; }
                }
                const int sk = slab_local(k, nz, L);
                if (sk >= 0) {
                    const long long s = cij + nxy * sk;
                    const float b = __ldg(a.prof[0][2] + k), c = __ldg(a.prof[1][2] + k);
                    kz = __ldg(a.prof[2][2] + k);
                    pxz = b * __ldg(a.psi_in[2][0] + s) + c * (dHy_dz * div);
                    pyz = b * __ldg(a.psi_in[2][1] + s) + c * (dHx_dz * div);
                    if (owned) { a.psi_out[2][0][s] = pxz; a.psi_out[2][1][s] = pyz; }
                }
                cx = sy.kinv * dHz_dy - kz * dHy_dz + dx * (pxy - pxz);
                cy = kz * dHx_dz - sx.kinv * dHz_dx + dx * (pyz - pyx);
                cz = sx.kinv * dHy_dx - sy.kinv * dHx_dy + dx * (pzx - pzy);
            }
            for (int t = 0; t < a.src.n; t++)
                if (a.src.k[t] == k) {
                    const float *sp = a.src.p[t];
                    cx -= dx * sp[cij];
                    cy -= dx * sp[nxy + cij];
                    cz -= dx * sp[2 * nxy + cij];
                }
            if (LOSSY) {
                ex = Eat(S.c[3], lx, ly) * ex + Eat(S.c[0], lx, ly) * cx;
                ey = Eat(S.c[4], lx, ly) * ey + Eat(S.c[1], lx, ly) * cy;
                ez = Eat(S.c[5], lx, ly) * ez + Eat(S.c[2], lx, ly) * cz;
            } else {
                ex = ex + Eat(S.c[0], lx, ly) * cx;
                ey = ey + Eat(S.c[1], lx, ly) * cy;
                ez = ez + Eat(S.c[2], lx, ly) * cz;
            }
            if (owned) {
                const long long q = cij + nxy * k;
                a.f_out[0][q] = ex;
                a.f_out[1][q] = ey;
                a.f_out[2][q] = ez;
            }
        }
        sm.en[p2][0][ly][lx] = ex;
        sm.en[p2][1][ly][lx] = ey;
        sm.en[p2][2][ly][lx] = ez;
    };

    // CPML column data of a halo cell (computed on the fly; 40 of 296 cells)
    auto slab_of = [&](int lx, int ly, bool xaxis) -> SlabE {
        SlabE r{-1, 1.f, 0.f, 1.f};
        if (!CPML) return r;
        const int ggi = X0 + lx, ggj = Y0 + ly;
        if (ggi < 1 || ggi > nx - 2 || ggj < 1 || ggj > ny - 2) return r;
        if (xaxis) {
            const int si = slab_local(ggi, nx, L);
            if (si >= 0) r = {si + 2LL * L * ggj, __ldg(a.prof[0][0] + ggi), __ldg(a.prof[1][0] + ggi), __ldg(a.prof[2][0] + ggi)};
        } else {
            const int sj = slab_local(ggj, ny, L);
            if (sj >= 0) r = {ggi + (long long)nx * sj, __ldg(a.prof[0][1] + ggj), __ldg(a.prof[1][1] + ggj), __ldg(a.prof[2][1] + ggj)};
        }
        return r;
    };

    for (int k = z0; k <= z1; k++) {
        if (tid == 0 && live && k + 1 <= z1 && k + 1 < nz) issue_plane<LOSSY>(sm, maps, k + 1, X0, Y0);
        if (k < nz) {
            if (k == z0) wait_plane<LOSSY>(sm, z0 - 1, z0, err);
            wait_plane<LOSSY>(sm, k, z0, err);
            e_cell(tx, ty, k, k < z1, ex_, ey_);
            for (int t = tid; t < TX + TY; t += TX * TY) {
                const int lx = t < TY ? TX : t - TY, ly = t < TY ? t : TY;
                e_cell(lx, ly, k, false, slab_of(lx, ly, true), slab_of(lx, ly, false));
            }
        }
        __syncthreads();
        const int km = k - 1;
        if (km >= z0 && km >= 1 && km <= nz - 2 && col_ok) {
            const int p2 = k & 1, pm2 = p2 ^ 1;
            const TmaStage<LOSSY> &Sm = sm.st[(k + 2) % 3];
            const float ex0 = sm.en[pm2][0][ty][tx], ey0 = sm.en[pm2][1][ty][tx], ez0 = sm.en[pm2][2][ty][tx];
            const float dEz_dy = sm.en[pm2][2][ty + 1][tx] - ez0;
            const float dEy_dz = sm.en[p2][1][ty][tx] - ey0;
            const float dEx_dz = sm.en[p2][0][ty][tx] - ex0;
            const float dEz_dx = sm.en[pm2][2][ty][tx + 1] - ez0;
            const float dEy_dx = sm.en[pm2][1][ty][tx + 1] - ey0;
            const float dEx_dy = sm.en[pm2][0][ty + 1][tx] - ex0;
            float cx, cy, cz;
            if (!CPML) {
                cx = dEz_dy - dEy_dz;
                cy = dEx_dz - dEz_dx;
                cz = dEy_dx - dEx_dy;
            } else {
                float pxy = 0.f, pxz = 0.f, pyx = 0.f, pyz = 0.f, pzx = 0.f, pzy = 0.f, kz = 1.f;
                if (hx_.base >= 0) {
                    const long long s = hx_.base + xstride * km;
                    pyx = hx_.b * __ldg(a.psi_in[0][2] + s) + hx_.a * (dEz_dx * div);
                    pzx = hx_.b * __ldg(a.psi_in[0][3] + s) + hx_.a * (dEy_dx * div);
                    a.psi_out[0][2][s] = pyx;
                    a.psi_out[0][3][s] = pzx;
                }
                if (hy_.base >= 0) {
                    const long long s = hy_.base + ystride * km;
                    pxy = hy_.b * __ldg(a.psi_in[1][2] + s) + hy_.a * (dEz_dy * div);
                    pzy = hy_.b * __ldg(a.psi_in[1][3] + s) + hy_.a * (dEx_dy * div);
                    a.psi_out[1][2][s] = pxy;
                    a.psi_out[1][3][s] = pzy;
                }
                const int sk = slab_local(km, nz, L);
                if (sk >= 0) {
                    const long long s = ij + nxy * sk;
                    const float b = __ldg(a.prof[3][2] + km), c = __ldg(a.prof[4][2] + km);
                    kz = __ldg(a.prof[5][2] + km);
                    pxz = b * __ldg(a.psi_in[2][2] + s) + c * (dEy_dz * div);
                    pyz = b * __ldg(a.psi_in[2][3] + s) + c * (dEx_dz * div);
                    a.psi_out[2][2][s] = pxz;
                    a.psi_out[2][3][s] = pyz;
                }
                cx = hy_.kinv * dEz_dy - kz * dEy_dz + dx * (pxy - pxz);
                cy = kz * dEx_dz - hx_.kinv * dEz_dx + dx * (pyz - pyx);
                cz = hx_.kinv * dEy_dx - hy_.kinv * dEx_dy + dx * (pzx - pzy);
            }
            for (int t = 0; t < a.src.n; t++)
                if (a.src.k[t] == km) {
                    const float *sp = a.src.p[t];
                    cx += dx * sp[3 * nxy + ij];
                    cy += dx * sp[4 * nxy + ij];
                    cz += dx * sp[5 * nxy + ij];
                }
            const long long q = ij + nxy * km;
            a.f_out[3][q] = Hat(Sm.h[0], tx, ty) - hb * cx;
            a.f_out[4][q] = Hat(Sm.h[1], tx, ty) - hb * cy;
            a.f_out[5][q] = Hat(Sm.h[2], tx, ty) - hb * cz;
        }
        __syncthreads();
    }
    // all issued planes were waited for in the loop; nothing is left in flight
}

// ---- host side ---------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        cudaGetLastError();
    }
    return fn;
}

int fused_tma_supported(int nx, int ny, int nz) { return nx % 4 == 0 && nx >= 8 && ny >= 4 && nz >= 4 && encode_fn(); }

static bool encode(CUtensorMap *m, const float *base, int nx, int ny, int nz, int box_x, int box_y)
{
    cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    cuuint64_t strides[2] = {(cuuint64_t)nx * 4, (cuuint64_t)nx * ny * 4};
    cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, 1};
    cuuint32_t elem[3] = {1, 1, 1};
    CUresult r = encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)base, dims, strides, box, elem,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool fused_make_maps(FusedMaps *m, const float *const f[6], const float *const cb[3], const float *const ca[3],
                     int nx, int ny, int nz)
{
    if (!encode_fn()) return false;
    for (int c = 0; c < 3; c++) {
        if (!encode(&m->h[c], f[3 + c], nx, ny, nz, HW, TY + 2)) return false;
        if (!encode(&m->e[c], f[c], nx, ny, nz, EW, TY + 1)) return false;
        if (!encode(&m->cb[c], cb[c], nx, ny, nz, EW, TY + 1)) return false;
        if (ca && ca[c]) {
            if (!encode(&m->ca[c], ca[c], nx, ny, nz, EW, TY + 1)) return false;
        } else {
            m->ca[c] = m->cb[c];
        }
    }
    return true;
}

template <bool CPML, bool LOSSY>
static void launch_tma(const FusedArgs &a, const FusedMaps &m, int *err, cudaStream_t st)
{
    auto kern = k_fused_tma<CPML, LOSSY>;
    const size_t smem = tma_smem_bytes<LOSSY>();
    static int slots = -1;
    if (slots < 0) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int per_sm = 0, dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TX * TY, smem);
        slots = per_sm * sms;
    }
    long long tiles = (long long)((a.nx + TX - 1) / TX) * ((a.ny + TY - 1) / TY);
    long long chunks = slots > 0 ? slots / tiles : 1;
    if (chunks < 1) chunks = 1;
    int zc = (int)((a.nz + chunks - 1) / chunks);
    if (zc < 8) zc = 8;
    dim3 grid((a.nx + TX - 1) / TX, (a.ny + TY - 1) / TY, (a.nz + zc - 1) / zc);
    kern<<<grid, dim3(TX, TY), smem, st>>>(a, m, zc, err);
}

void launch_fused_step_tma(const FusedArgs &a, const FusedMaps &m, int *err, cudaStream_t st)
{
    note_launch();
    const bool lossy = a.ca[0] != nullptr;
    if (a.L > 0) {
        if (lossy) launch_tma<true, true>(a, m, err, st);
        else launch_tma<true, false>(a, m, err, st);
    } else {
        if (lossy) launch_tma<false, true>(a, m, err, st);
        else launch_tma<false, false>(a, m, err, st);
    }
}

}  // namespace fdtd
