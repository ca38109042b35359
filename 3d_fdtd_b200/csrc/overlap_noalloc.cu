// overlap_noalloc.cu -- mode overlap of one field plane with no device
// allocation: fdtd_mode_overlap_plane_noalloc.
//
// The regular overlap path reduces into per-grid scratch that the library
// cudaMalloc's when a grid is first used.  Some callers can never allocate:
// code running while a stream is being captured into a CUDA graph (allocation
// is not capturable), host applications that hand this library a fixed budget
// of memory they own and forbid it to grow, and latency-critical loops where
// cudaMalloc's implicit device synchronisation is not acceptable.  For them
// this entry point takes every input and the output as caller-owned device
// pointers and keeps its scratch in a file-scope __device__ array of fixed
// size: one partial sum per row of the plane, at most kMaxRows rows.
//
// The array is a module global: every GPU that loads the library holds its
// 128 KiB until the process exits, and every call on that GPU shares it.  Each
// call overwrites rows [0, ny) before reading them, so nothing needs clearing,
// but two calls whose kernels overlap on the GPU (different streams, no
// ordering between them) race on the array and may return wrong sums.
#include <cstdint>
#include <mutex>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"

namespace fdtd {

constexpr int kMaxRows = 8192;
static __device__ __align__(256) double2 g_overlap_rows[kMaxRows];

// Row j of the plane: sum over i of Hx mEy - Hy mEx + Ey mHx - Ex mHy for cells
// with a mode sample (timefield3d.c:3176-3233), mode H -> -conj(H) when reverse.
// One warp per row, lanes strided over i, fixed-shape warp reduction.
template <typename T>
__global__ void k_overlap_rows(const T *ex, const T *ey, const T *hx, const T *hy, int nx, int ny, int cx, int cy,
                               const double2 *mode, int mi, int mj, double ratio, int reverse, double2 *rows)
{
    const int lane = threadIdx.x & 31;
    const int warps = (blockDim.x >> 5) * gridDim.x;
    for (int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); j < ny; j += warps) {
        double sre = 0.0, sim = 0.0;
        const int my = (int)dmul((double)(j - cy), ratio) + mj / 2;
        if (my >= 0 && my < mj) {
            for (int i = lane; i < nx; i += 32) {
                const int mx = (int)dmul((double)(i - cx), ratio) + mi / 2;
                if (mx < 0 || mx >= mi) continue;
                const double2 *e = mode + 6LL * (mx + (long long)mi * my);
                double2 mEx = e[0], mEy = e[1], mHx = e[3], mHy = e[4];
                if (reverse) {
                    mHx.x = -mHx.x;
                    mHy.x = -mHy.x;
                }
                const long long q = i + (long long)nx * j;
                const double vex = (double)ex[q], vey = (double)ey[q], vhx = (double)hx[q], vhy = (double)hy[q];
                sre = dadd(sre, dadd(dsub(dmul(vhx, mEy.x), dmul(vhy, mEx.x)), dsub(dmul(vey, mHx.x), dmul(vex, mHy.x))));
                sim = dadd(sim, dadd(dsub(dmul(vhx, mEy.y), dmul(vhy, mEx.y)), dsub(dmul(vey, mHx.y), dmul(vex, mHy.y))));
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            sre = dadd(sre, __shfl_down_sync(0xffffffffu, sre, o));
            sim = dadd(sim, __shfl_down_sync(0xffffffffu, sim, o));
        }
        if (lane == 0) rows[j] = make_double2(sre, sim);
    }
}

// rows[0..ny) -> scale * sum, in row order (one thread; ny <= kMaxRows)
__global__ void k_overlap_rows_total(const double2 *rows, int ny, double scale, double2 *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double sre = 0.0, sim = 0.0;
    for (int j = 0; j < ny; j++) {
        sre = dadd(sre, rows[j].x);
        sim = dadd(sim, rows[j].y);
    }
    *out = make_double2(dmul(scale, sre), dmul(scale, sim));
}

// device address of g_overlap_rows per device, looked up once per device
static double2 *rows_address(int dev)
{
    static std::mutex mu;
    static double2 *addr[64] = {};
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        if (!cuda_ok(cudaGetSymbolAddress(&p, g_overlap_rows), "cudaGetSymbolAddress(g_overlap_rows)")) return nullptr;
        addr[dev] = (double2 *)p;
    }
    return addr[dev];
}

}  // namespace fdtd

using namespace fdtd;

extern "C" int fdtd_mode_overlap_plane_noalloc(const void *ex, const void *ey, const void *hx, const void *hy,
                                               int precision, int nx, int ny, int center_x, int center_y,
                                               const complex *mode_fields, int mode_i, int mode_j, double ratio,
                                               int reverse, double disc, complex *result, void *stream)
{
    if (!ex || !ey || !hx || !hy || !mode_fields || !result || nx <= 0 || ny <= 0 || mode_i <= 0 || mode_j <= 0 ||
        !(ratio > 0) || !(disc > 0) || (precision != FDTD_F64 && precision != FDTD_F32)) {
        set_error(FDTD_ERR_ARG, "fdtd_mode_overlap_plane_noalloc: invalid argument");
        return FDTD_ERR_ARG;
    }
    // the mode and the result are read and written as double2 (16-byte
    // accesses); a misaligned pointer would fault the kernel and poison the
    // caller's context, so it is refused here, before any launch
    const size_t esz = precision == FDTD_F64 ? sizeof(double) : sizeof(float);
    if (((uintptr_t)mode_fields | (uintptr_t)result) % 16 != 0 ||
        ((uintptr_t)ex | (uintptr_t)ey | (uintptr_t)hx | (uintptr_t)hy) % esz != 0) {
        set_error(FDTD_ERR_ARG,
                  "fdtd_mode_overlap_plane_noalloc: mode_fields and result must be 16-byte aligned and the field "
                  "planes aligned to their element size");
        return FDTD_ERR_ARG;
    }
    if (ny > kMaxRows) {
        set_error(FDTD_ERR_ARG, "fdtd_mode_overlap_plane_noalloc: plane has %d rows; the fixed scratch holds at most %d",
                  ny, kMaxRows);
        return FDTD_ERR_ARG;
    }
    if (!device_available()) return FDTD_ERR_NO_DEVICE;
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice")) return FDTD_ERR_CUDA;
    double2 *rows = rows_address(dev);
    if (!rows) return fdtd_last_error() ? fdtd_last_error() : FDTD_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    const int warps_per_block = 8;
    int blocks = (ny + warps_per_block - 1) / warps_per_block;
    if (blocks > 1024) blocks = 1024;
    const double2 *md = (const double2 *)mode_fields;
    note_launch(2);
    if (precision == FDTD_F64)
        k_overlap_rows<double><<<blocks, 32 * warps_per_block, 0, st>>>(
            (const double *)ex, (const double *)ey, (const double *)hx, (const double *)hy, nx, ny, center_x,
            center_y, md, mode_i, mode_j, ratio, reverse == 1, rows);
    else
        k_overlap_rows<float><<<blocks, 32 * warps_per_block, 0, st>>>(
            (const float *)ex, (const float *)ey, (const float *)hx, (const float *)hy, nx, ny, center_x, center_y,
            md, mode_i, mode_j, ratio, reverse == 1, rows);
    k_overlap_rows_total<<<1, 32, 0, st>>>(rows, ny, (-0.5 * disc * disc), (double2 *)result);
    return cuda_ok(cudaGetLastError(), "fdtd_mode_overlap_plane_noalloc") ? FDTD_OK : FDTD_ERR_CUDA;
}
