// yee_split.cu -- separate E and H passes and the Mur boundary.
//
// This is the path that reproduces the reference step
// timefield3d_apply_timestep_omp_full (timefield3d.c:2787-2849) exactly:
//   shell snapshot -> E interior -> E Mur faces -> H interior -> H Mur faces.
// In FP64 every interior and boundary value is bit-identical to the
// reference's (same operations, same order, no FMA).  It also carries the
// CPML terms for grids that use FP64 or the non-fused FP32 path.
//
// Thread layout: a 32 x 4 block of (x, y) columns; each thread walks a chunk
// of z planes, carrying the previous plane's H (E pass) or next plane's E
// (H pass) in registers so that the z-neighbour is read once.
#include "common.cuh"
#include "kernels.h"

namespace fdtd {

constexpr int kBX = 32, kBY = 4, kZChunk = 16;

template <typename T>
__device__ __forceinline__ T src_at(const SourcePlanes &s, int k, int m, long long nxy, long long ij)
{
    for (int t = 0; t < s.n; t++)
        if (s.k[t] == k) return (T)s.p[t][m * nxy + ij];
    return (T)0;
}

// ---------------------------------------------------------------------------
// E interior.  Semi-implicit form: timefield3d_apply_E_timestep_zsection
// (timefield3d.c:1759-1837); explicit form: timefield3d_apply_E_timestep
// (timefield3d.c:1607-1677).
// ---------------------------------------------------------------------------
template <typename T, bool SIG, bool CPML, bool EXPL>
__global__ void __launch_bounds__(kBX *kBY)
k_update_E(GridView<T> g, CpmlView<T> c, SourcePlanes src, T dt, T divisor, int k_lo, int k_hi)
{
    using A = Ar<T>;
    const int i = blockIdx.x * kBX + threadIdx.x;
    const int j = blockIdx.y * kBY + threadIdx.y;
    if (i < 1 || i > g.nx - 2 || j < 1 || j > g.ny - 2) return;
    const long long nxy = (long long)g.nx * g.ny;
    const long long ij = i + (long long)g.nx * j;
    int k0 = max(k_lo, 1) + blockIdx.z * kZChunk;
    int k1 = min(min(k_hi, g.nz - 1), k0 + kZChunk);
    if (k0 >= k1) return;
    const T *Hx = g.f[3], *Hy = g.f[4], *Hz = g.f[5];
    long long q = ij + nxy * k0;
    T hx_m = Hx[q - nxy], hy_m = Hy[q - nxy];
    for (int k = k0; k < k1; k++, q += nxy) {
        T hx = Hx[q], hy = Hy[q], hz = Hz[q];
        T dHz_dy = A::sub(hz, Hz[q - g.nx]);
        T dHy_dz = A::sub(hy, hy_m);
        T dHx_dz = A::sub(hx, hx_m);
        T dHz_dx = A::sub(hz, Hz[q - 1]);
        T dHy_dx = A::sub(hy, Hy[q - 1]);
        T dHx_dy = A::sub(hx, Hx[q - g.nx]);
        hx_m = hx;
        hy_m = hy;
        T curl_x, curl_y, curl_z;
        if (!CPML) {
            curl_x = A::mul(divisor, A::sub(dHz_dy, dHy_dz));
            curl_y = A::mul(divisor, A::sub(dHx_dz, dHz_dx));
            curl_z = A::mul(divisor, A::sub(dHy_dx, dHx_dy));
        } else {
            const int L = c.L;
            int sx = slab_local(i, g.nx, L), sy = slab_local(j, g.ny, L), sz = slab_local(k, g.nz, L);
            T kx = sx >= 0 ? c.prof[2][0][i] : (T)1;
            T ky = sy >= 0 ? c.prof[2][1][j] : (T)1;
            T kz = sz >= 0 ? c.prof[2][2][k] : (T)1;
            T pxy = 0, pxz = 0, pyx = 0, pyz = 0, pzx = 0, pzy = 0;
            if (sx >= 0) {
                long long s = sx + 2LL * L * (j + (long long)g.ny * k);
                T b = c.prof[0][0][i], a = c.prof[1][0][i];
                pyx = A::add(A::mul(b, c.psi[0][0][s]), A::mul(a, A::mul(dHz_dx, divisor)));
                pzx = A::add(A::mul(b, c.psi[0][1][s]), A::mul(a, A::mul(dHy_dx, divisor)));
                c.psi[0][0][s] = pyx;
                c.psi[0][1][s] = pzx;
            }
            if (sy >= 0) {
                long long s = i + (long long)g.nx * (sy + 2LL * L * k);
                T b = c.prof[0][1][j], a = c.prof[1][1][j];
                pxy = A::add(A::mul(b, c.psi[1][0][s]), A::mul(a, A::mul(dHz_dy, divisor)));
                pzy = A::add(A::mul(b, c.psi[1][1][s]), A::mul(a, A::mul(dHx_dy, divisor)));
                c.psi[1][0][s] = pxy;
                c.psi[1][1][s] = pzy;
            }
            if (sz >= 0) {
                long long s = ij + nxy * sz;
                T b = c.prof[0][2][k], a = c.prof[1][2][k];
                pxz = A::add(A::mul(b, c.psi[2][0][s]), A::mul(a, A::mul(dHy_dz, divisor)));
                pyz = A::add(A::mul(b, c.psi[2][1][s]), A::mul(a, A::mul(dHx_dz, divisor)));
                c.psi[2][0][s] = pxz;
                c.psi[2][1][s] = pyz;
            }
            curl_x = A::add(A::mul(divisor, A::sub(A::mul(dHz_dy, ky), A::mul(dHy_dz, kz))), A::sub(pxy, pxz));
            curl_y = A::add(A::mul(divisor, A::sub(A::mul(dHx_dz, kz), A::mul(dHz_dx, kx))), A::sub(pyz, pyx));
            curl_z = A::add(A::mul(divisor, A::sub(A::mul(dHy_dx, kx), A::mul(dHx_dy, ky))), A::sub(pzx, pzy));
        }
        T curl[3] = {curl_x, curl_y, curl_z};
#pragma unroll
        for (int m = 0; m < 3; m++) {
            T e = g.f[m][q];
            T ep = (T)g.ep[m][q];
            T sig = SIG ? (T)g.sig[m][q] : (T)0;
            T J = src_at<T>(src, k, m, nxy, ij);
            T out;
            if (EXPL) {
                T Jt = A::add(J, A::mul(e, sig));
                out = A::add(e, A::div(A::mul(dt, A::sub(curl[m], Jt)), ep));
            } else if (SIG) {
                T main_coeff = A::div((T)1, A::add(A::div(ep, dt), A::mul((T)0.5, sig)));
                T e_coeff = A::sub(A::div(ep, dt), A::mul((T)0.5, sig));
                out = A::mul(main_coeff, A::sub(A::add(A::mul(e_coeff, e), curl[m]), J));
            } else {
                T e_coeff = A::div(ep, dt);
                T main_coeff = A::div((T)1, e_coeff);
                out = A::mul(main_coeff, A::sub(A::add(A::mul(e_coeff, e), curl[m]), J));
            }
            g.f[m][q] = out;
        }
    }
}

// ---------------------------------------------------------------------------
// H interior.  Semi-implicit: timefield3d_apply_H_timestep_zsection
// (timefield3d.c:1679-1757), magnetic current = source + sig_m H
// (timefield3d.c:1705-1707); explicit: timefield3d_apply_H_timestep
// (timefield3d.c:1537-1605).
// ---------------------------------------------------------------------------
template <typename T, bool SIG, bool MU, bool CPML, bool EXPL>
__global__ void __launch_bounds__(kBX *kBY)
k_update_H(GridView<T> g, CpmlView<T> c, SourcePlanes src, T dt, T divisor, int k_lo, int k_hi)
{
    using A = Ar<T>;
    const int i = blockIdx.x * kBX + threadIdx.x;
    const int j = blockIdx.y * kBY + threadIdx.y;
    if (i < 1 || i > g.nx - 2 || j < 1 || j > g.ny - 2) return;
    const long long nxy = (long long)g.nx * g.ny;
    const long long ij = i + (long long)g.nx * j;
    int k0 = max(k_lo, 1) + blockIdx.z * kZChunk;
    int k1 = min(min(k_hi, g.nz - 1), k0 + kZChunk);
    if (k0 >= k1) return;
    const T *Ex = g.f[0], *Ey = g.f[1], *Ez = g.f[2];
    long long q = ij + nxy * k0;
    T ex = Ex[q], ey = Ey[q];
    for (int k = k0; k < k1; k++, q += nxy) {
        T ez = Ez[q];
        T ex_p = Ex[q + nxy], ey_p = Ey[q + nxy];
        T dEz_dy = A::sub(Ez[q + g.nx], ez);
        T dEy_dz = A::sub(ey_p, ey);
        T dEx_dz = A::sub(ex_p, ex);
        T dEz_dx = A::sub(Ez[q + 1], ez);
        T dEy_dx = A::sub(Ey[q + 1], ey);
        T dEx_dy = A::sub(Ex[q + g.nx], ex);
        ex = ex_p;
        ey = ey_p;
        T curl_x, curl_y, curl_z;
        if (!CPML) {
            curl_x = A::mul(divisor, A::sub(dEz_dy, dEy_dz));
            curl_y = A::mul(divisor, A::sub(dEx_dz, dEz_dx));
            curl_z = A::mul(divisor, A::sub(dEy_dx, dEx_dy));
        } else {
            const int L = c.L;
            int sx = slab_local(i, g.nx, L), sy = slab_local(j, g.ny, L), sz = slab_local(k, g.nz, L);
            T kx = sx >= 0 ? c.prof[5][0][i] : (T)1;
            T ky = sy >= 0 ? c.prof[5][1][j] : (T)1;
            T kz = sz >= 0 ? c.prof[5][2][k] : (T)1;
            T pxy = 0, pxz = 0, pyx = 0, pyz = 0, pzx = 0, pzy = 0;
            if (sx >= 0) {
                long long s = sx + 2LL * L * (j + (long long)g.ny * k);
                T b = c.prof[3][0][i], a = c.prof[4][0][i];
                pyx = A::add(A::mul(b, c.psi[0][2][s]), A::mul(a, A::mul(dEz_dx, divisor)));
                pzx = A::add(A::mul(b, c.psi[0][3][s]), A::mul(a, A::mul(dEy_dx, divisor)));
                c.psi[0][2][s] = pyx;
                c.psi[0][3][s] = pzx;
            }
            if (sy >= 0) {
                long long s = i + (long long)g.nx * (sy + 2LL * L * k);
                T b = c.prof[3][1][j], a = c.prof[4][1][j];
                pxy = A::add(A::mul(b, c.psi[1][2][s]), A::mul(a, A::mul(dEz_dy, divisor)));
                pzy = A::add(A::mul(b, c.psi[1][3][s]), A::mul(a, A::mul(dEx_dy, divisor)));
                c.psi[1][2][s] = pxy;
                c.psi[1][3][s] = pzy;
            }
            if (sz >= 0) {
                long long s = ij + nxy * sz;
                T b = c.prof[3][2][k], a = c.prof[4][2][k];
                pxz = A::add(A::mul(b, c.psi[2][2][s]), A::mul(a, A::mul(dEy_dz, divisor)));
                pyz = A::add(A::mul(b, c.psi[2][3][s]), A::mul(a, A::mul(dEx_dz, divisor)));
                c.psi[2][2][s] = pxz;
                c.psi[2][3][s] = pyz;
            }
            curl_x = A::add(A::mul(divisor, A::sub(A::mul(dEz_dy, ky), A::mul(dEy_dz, kz))), A::sub(pxy, pxz));
            curl_y = A::add(A::mul(divisor, A::sub(A::mul(dEx_dz, kz), A::mul(dEz_dx, kx))), A::sub(pyz, pyx));
            curl_z = A::add(A::mul(divisor, A::sub(A::mul(dEy_dx, kx), A::mul(dEx_dy, ky))), A::sub(pzx, pzy));
        }
        T curl[3] = {curl_x, curl_y, curl_z};
#pragma unroll
        for (int m = 0; m < 3; m++) {
            T h = g.f[3 + m][q];
            T mu = MU ? (T)g.mu[m][q] : (T)1;
            T sig = SIG ? (T)g.sig[3 + m][q] : (T)0;
            T M = src_at<T>(src, k, 3 + m, nxy, ij);
            if (SIG) M = A::add(M, A::mul(h, sig));
            T out;
            if (EXPL) {
                out = A::sub(h, A::div(A::mul(dt, A::add(curl[m], M)), mu));
            } else if (SIG) {
                T main_coeff = A::div((T)1, A::add(A::div(mu, dt), A::mul((T)0.5, sig)));
                T h_coeff = A::sub(A::div(mu, dt), A::mul((T)0.5, sig));
                out = A::mul(main_coeff, A::sub(A::sub(A::mul(h_coeff, h), curl[m]), M));
            } else {
                T h_coeff = A::div(mu, dt);
                T main_coeff = A::div((T)1, h_coeff);
                out = A::mul(main_coeff, A::sub(A::sub(A::mul(h_coeff, h), curl[m]), M));
            }
            g.f[3 + m][q] = out;
        }
    }
}

// ---------------------------------------------------------------------------
// Shell snapshot: timefield3d_update_old_edge_fields (timefield3d.c:246-346),
// the 2-cell shell of all six components.  One block per z plane: planes
// 0,1,nz-2,nz-1 entirely, other planes only their 2-cell ring.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_save_shell(GridView<T> g)
{
    const int k = blockIdx.x;
    const long long nxy = (long long)g.nx * g.ny;
    const long long base = nxy * k;
    const bool full = k <= 1 || k >= g.nz - 2;
    if (full) {
        for (long long t = threadIdx.x; t < nxy; t += blockDim.x)
#pragma unroll
            for (int m = 0; m < 6; m++) g.old[m][base + t] = g.f[m][base + t];
        return;
    }
    // ring: rows 0,1,ny-2,ny-1 whole; other rows columns 0,1,nx-2,nx-1
    const int nrow_full = 4 * g.nx;
    const int nring = nrow_full + 4 * (g.ny - 4);
    for (int t = threadIdx.x; t < nring; t += blockDim.x) {
        int i, j;
        if (t < nrow_full) {
            int r = t / g.nx;
            i = t - r * g.nx;
            j = r < 2 ? r : g.ny - 4 + r;
        } else {
            int u = t - nrow_full;
            int r = u >> 2, cidx = u & 3;
            j = 2 + r;
            i = cidx < 2 ? cidx : g.nx - 4 + cidx;
        }
        long long q = base + i + (long long)g.nx * j;
#pragma unroll
        for (int m = 0; m < 6; m++) g.old[m][q] = g.f[m][q];
    }
}

// ---------------------------------------------------------------------------
// Mur first-order ABC, E (timefield3d.c:2499-2721) or H (2275-2497) faces.
// Faces run in the reference's order x=0, y=0, z=0, x=end, y=end, z=end and
// later faces read what earlier ones wrote on shared edges, so the order is
// kept inside a block.  x and y faces only couple cells of one z plane, so a
// block owns one plane; the first block also owns plane 1 and runs the z=0
// face after that plane's x=0/y=0 faces (its inner cells), the last block
// likewise for the z=end face.  Tangential components of a face normal to a:
// x: (y,z), y: (x,z), z: (x,y); for E component c v = 1/sqrt(ep_c mu_t), for
// H component c v = 1/sqrt(ep_t mu_c), t the third axis.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void mur_cell(GridView<T> &g, int efield, int axis, long long qb, long long qi,
                                          T dt, T dx)
{
    using A = Ar<T>;
    const int c1 = axis == 0 ? 1 : 0, c2 = axis == 2 ? 1 : 2;
#pragma unroll
    for (int w = 0; w < 2; w++) {
        int c = w ? c2 : c1;
        int t = 3 - axis - c;
        T ep = efield ? (T)g.ep[c][qb] : (T)g.ep[t][qb];
        T mu = efield ? (T)g.mu[t][qb] : (T)g.mu[c][qb];
        int m = efield ? c : 3 + c;
        T F_old = g.old[m][qb];
        T F_inner = g.f[m][qi];
        T F_inner_old = g.old[m][qi];
        T speed = A::div((T)1, A::sqrt_(A::mul(ep, mu)));
        T sdt = A::mul(speed, dt);
        T scalar = A::div(A::sub(sdt, dx), A::add(sdt, dx));
        g.f[m][qb] = A::add(F_inner_old, A::mul(scalar, A::sub(F_inner, F_old)));
    }
}

template <typename T>
__global__ void k_mur(GridView<T> g, T dt, T dx, int efield, int ks, int ke)
{
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long nxy = (long long)nx * ny;
    const int lo = ks == 0, hi = ke == nz;
    const int mid0 = lo ? 2 : ks, mid1 = hi ? nz - 2 : ke;
    const int nblk = lo + max(0, mid1 - mid0) + hi;
    const int b = blockIdx.x;
    if (b >= nblk) return;
    int p0, p1, zface = -1;
    if (lo && b == 0) { p0 = 0; p1 = min(2, ke); zface = 0; }
    else if (hi && b == nblk - 1) { p0 = nz - 2; p1 = nz; zface = 1; }
    else { p0 = mid0 + b - lo; p1 = p0 + 1; }
    const int np = p1 - p0;
    for (int high = 0; high < 2; high++) {
        // x face
        {
            int ib = high ? nx - 1 : 0, ii = high ? nx - 2 : 1;
            for (int t = threadIdx.x; t < ny * np; t += blockDim.x) {
                int j = t % ny, k = p0 + t / ny;
                long long r = (long long)nx * j + nxy * k;
                mur_cell(g, efield, 0, r + ib, r + ii, dt, dx);
            }
        }
        __syncthreads();
        // y face
        {
            int jb = high ? ny - 1 : 0, ji = high ? ny - 2 : 1;
            for (int t = threadIdx.x; t < nx * np; t += blockDim.x) {
                int i = t % nx, k = p0 + t / nx;
                long long r = i + nxy * k;
                mur_cell(g, efield, 1, r + (long long)nx * jb, r + (long long)nx * ji, dt, dx);
            }
        }
        __syncthreads();
        // z face
        if (zface == high) {
            int kb = high ? nz - 1 : 0, ki = high ? nz - 2 : 1;
            for (long long t = threadIdx.x; t < nxy; t += blockDim.x)
                mur_cell(g, efield, 2, t + nxy * kb, t + nxy * ki, dt, dx);
        }
        __syncthreads();
    }
}

// AoS double (reference layout) -> SoA T, whole grid
template <typename T>
__global__ void k_aos_to_soa(const double *aos, T *d0, T *d1, T *d2, T *d3, T *d4, T *d5, long long n)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const double *a = aos + 6 * q;
        d0[q] = (T)a[0]; d1[q] = (T)a[1]; d2[q] = (T)a[2];
        d3[q] = (T)a[3]; d4[q] = (T)a[4]; d5[q] = (T)a[5];
    }
}

// SoA T -> AoS double
template <typename T>
__global__ void k_soa_to_aos(double *aos, const T *s0, const T *s1, const T *s2, const T *s3, const T *s4,
                             const T *s5, long long n)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        double *a = aos + 6 * q;
        a[0] = (double)s0[q]; a[1] = (double)s1[q]; a[2] = (double)s2[q];
        a[3] = (double)s3[q]; a[4] = (double)s4[q]; a[5] = (double)s5[q];
    }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static dim3 grid_for(int nx, int ny, int k_lo, int k_hi, int nz)
{
    int a = k_lo < 1 ? 1 : k_lo, b = k_hi > nz - 1 ? nz - 1 : k_hi;
    int nk = b > a ? b - a : 0;
    return dim3((nx + kBX - 1) / kBX, (ny + kBY - 1) / kBY, (nk + kZChunk - 1) / kZChunk);
}

template <typename T>
void launch_update_E(const GridView<T> &g, const CpmlView<T> &c, const SourcePlanes &s, T dt, T divisor,
                     int k_lo, int k_hi, bool sig, bool cpml, bool expl, cudaStream_t st)
{
    dim3 grd = grid_for(g.nx, g.ny, k_lo, k_hi, g.nz), blk(kBX, kBY);
    if (grd.z == 0) return;
    note_launch();
    if (expl) k_update_E<T, true, false, true><<<grd, blk, 0, st>>>(g, c, s, dt, divisor, k_lo, k_hi);
    else if (cpml) {
        if (sig) k_update_E<T, true, true, false><<<grd, blk, 0, st>>>(g, c, s, dt, divisor, k_lo, k_hi);
        else k_update_E<T, false, true, false><<<grd, blk, 0, st>>>(g, c, s, dt, divisor, k_lo, k_hi);
    } else {
        if (sig) k_update_E<T, true, false, false><<<grd, blk, 0, st>>>(g, c, s, dt, divisor, k_lo, k_hi);
        else k_update_E<T, false, false, false><<<grd, blk, 0, st>>>(g, c, s, dt, divisor, k_lo, k_hi);
    }
}

template <typename T>
void launch_update_H(const GridView<T> &g, const CpmlView<T> &c, const SourcePlanes &s, T dt, T divisor,
                     int k_lo, int k_hi, bool sig, bool mu, bool cpml, bool expl, cudaStream_t st)
{
    dim3 grd = grid_for(g.nx, g.ny, k_lo, k_hi, g.nz), blk(kBX, kBY);
    if (grd.z == 0) return;
    note_launch();
    if (expl) { k_update_H<T, true, true, false, true><<<grd, blk, 0, st>>>(g, c, s, dt, divisor, k_lo, k_hi); return; }
#define FDTD_H(SG, MU_, CP) k_update_H<T, SG, MU_, CP, false><<<grd, blk, 0, st>>>(g, c, s, dt, divisor, k_lo, k_hi)
    if (sig) {
        if (cpml) FDTD_H(true, true, true); else FDTD_H(true, true, false);
    } else if (mu) {
        if (cpml) FDTD_H(false, true, true); else FDTD_H(false, true, false);
    } else {
        if (cpml) FDTD_H(false, false, true); else FDTD_H(false, false, false);
    }
#undef FDTD_H
}

template <typename T>
void launch_save_shell(const GridView<T> &g, cudaStream_t st)
{
    note_launch();
    k_save_shell<T><<<g.nz, 256, 0, st>>>(g);
}

template <typename T>
void launch_mur(const GridView<T> &g, T dt, T dx, int efield, int ks, int ke, cudaStream_t st)
{
    const int lo = ks == 0, hi = ke == g.nz;
    const int mid0 = lo ? 2 : ks, mid1 = hi ? g.nz - 2 : ke;
    int nblk = lo + (mid1 > mid0 ? mid1 - mid0 : 0) + hi;
    if (nblk > 0) {
        note_launch();
        k_mur<T><<<nblk, 256, 0, st>>>(g, dt, dx, efield, ks, ke);
    }
}

template <typename T>
void launch_aos_to_soa(const double *aos, T *const d[6], long long n, cudaStream_t st)
{
    int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    note_launch();
    k_aos_to_soa<T><<<blocks, 256, 0, st>>>(aos, d[0], d[1], d[2], d[3], d[4], d[5], n);
}

template <typename T>
void launch_soa_to_aos(double *aos, T *const s[6], long long n, cudaStream_t st)
{
    int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    note_launch();
    k_soa_to_aos<T><<<blocks, 256, 0, st>>>(aos, s[0], s[1], s[2], s[3], s[4], s[5], n);
}

#define FDTD_INST(T)                                                                                          \
    template void launch_update_E<T>(const GridView<T> &, const CpmlView<T> &, const SourcePlanes &, T, T, int, \
                                     int, bool, bool, bool, cudaStream_t);                                     \
    template void launch_update_H<T>(const GridView<T> &, const CpmlView<T> &, const SourcePlanes &, T, T, int, \
                                     int, bool, bool, bool, bool, cudaStream_t);                               \
    template void launch_save_shell<T>(const GridView<T> &, cudaStream_t);                                    \
    template void launch_mur<T>(const GridView<T> &, T, T, int, int, int, cudaStream_t);                       \
    template void launch_aos_to_soa<T>(const double *, T *const[6], long long, cudaStream_t);                  \
    template void launch_soa_to_aos<T>(double *, T *const[6], long long, cudaStream_t);
FDTD_INST(float)
FDTD_INST(double)
#undef FDTD_INST

}  // namespace fdtd
