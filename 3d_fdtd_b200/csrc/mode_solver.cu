// mode_solver.cu -- waveguide eigenmodes on the GPU in FP64: the reference's
// restarted Arnoldi iteration on the beta^2 operator (mode.c:3461-3616).
//
// A `mode` holds 6 complex components per cell of the cross-section, index
// 6*(i + mi*j) + m, m = Ex Ey Ez Hx Hy Hz, with complex ep, mu (3 per cell)
// and PML stretch factors sx, sy (2 per cell).  The solver looks for the mode
// with the largest real beta^2.  Per restart:
//   orthogonalise psi against previous modes (H inner product), boundary
//   condition, optional lateral symmetrisation, zero the PML cells; Krylov
//   basis k_0 = psi/|psi|, k_i = B k_{i-1} with modified Gram-Schmidt into an
//   upper Hessenberg H; the eigenvalue of H with the largest real part, its
//   eigenvector y; psi = sum_j y_j k_j; n_eff = sqrt(lambda)/omega.
// It stops when |n_eff| changes by less than tol, then forms Hz from
// div B = 0 and E from curl H and H-normalises the mode.
//
// Inside the loop only Hx and Hy matter: the operator reads and writes only
// them, the inner products use only them, Hz stays zero and E is recomputed
// from H before any use.  So the device vectors hold (Hx, Hy) per cell and
// the other four components are formed once at the end.
//
// Device arithmetic uses the reference's complex formulas (complex.c:75-149)
// with round-to-nearest intrinsics and no FMA, so one operator application
// equals mode_apply_beta_squared_operator (mode.c:2796-2943) bit for bit.
// Inner products are FP64 tree sums (the reference sums sequentially).  The
// small eigenproblem runs on the host: shifted QR on the Hessenberg matrix for
// the eigenvalues (the reference runs Householder QL sweeps to a 1e-3
// off-diagonal ratio, matrix.c:672-871), and the eigenvector from the
// reference's bordered system (matrix.c:1114-1158): H - lambda I with its
// last row replaced by ones, right-hand side n e_n.  The reference stores the
// last Arnoldi norm one element past its size x size matrix
// (mode.c:3542-3544 with i = size); that value is never read and is not kept.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "host_ref.h"

namespace fdtd {

using cd = std::complex<double>;

// ---- device complex arithmetic (complex.c), no FMA -------------------------
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(dadd(a.x, b.x), dadd(a.y, b.y)); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(dsub(a.x, b.x), dsub(a.y, b.y)); }
__device__ __forceinline__ double2 csmul(double s, double2 a) { return make_double2(dmul(s, a.x), dmul(s, a.y)); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(dsub(dmul(a.x, b.x), dmul(a.y, b.y)), dadd(dmul(a.x, b.y), dmul(a.y, b.x)));
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double cmag(double2 a) { return __dsqrt_rn(dadd(dmul(a.x, a.x), dmul(a.y, a.y))); }
__device__ __forceinline__ double2 cdiv(double2 x, double2 y)
{
    const double2 num = cmul(x, cconj(y));
    const double m = cmag(y);
    return csmul(__ddiv_rn(1.0, dmul(m, m)), num);
}
__device__ __forceinline__ double2 crecip(double2 x) { return cdiv(make_double2(1.0, 0.0), x); }

// material and PML of the cross-section, reference layout
struct MsGeom {
    int mi, mj;
    double disc, omega2;
    const double2 *ep, *mu, *pml;   // 3, 3, 2 per cell
    const double2 *inv_epz, *inv_muz; // 1 per cell
};

// per-cell 1/ep_z and 1/mu_z (complex_reciprocal)
__global__ void k_ms_inverses(MsGeom g, double2 *inv_epz, double2 *inv_muz)
{
    const int n = g.mi * g.mj;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        inv_epz[c] = crecip(g.ep[3 * c + 2]);
        inv_muz[c] = crecip(g.mu[3 * c + 2]);
    }
}

// out = B in on interior cells (mode.c:2796-2943), 0 on the window edge.
// Vectors: v[2c] = Hx, v[2c+1] = Hy.
__global__ void k_ms_beta2(MsGeom g, const double2 *__restrict__ in, double2 *__restrict__ out)
{
    const int mi = g.mi, mj = g.mj, n = mi * mj;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % mi, j = c / mi;
        if (i < 1 || i > mi - 2 || j < 1 || j > mj - 2) {
            out[2 * c] = make_double2(0.0, 0.0);
            out[2 * c + 1] = make_double2(0.0, 0.0);
            continue;
        }
        const double d = 1.0 / g.disc;
        const int r = c + 1, l = c - 1, u = c + mi, dn = c - mi, dr = c - mi + 1, ul = c + mi - 1;
        const double2 Hx = in[2 * c], Hx_r = in[2 * r], Hx_l = in[2 * l], Hx_u = in[2 * u], Hx_d = in[2 * dn],
                      Hx_dr = in[2 * dr];
        const double2 Hy = in[2 * c + 1], Hy_r = in[2 * r + 1], Hy_l = in[2 * l + 1], Hy_u = in[2 * u + 1],
                      Hy_d = in[2 * dn + 1], Hy_ul = in[2 * ul + 1];
        const double2 Bx = cmul(g.mu[3 * c], Hx), Bx_r = cmul(g.mu[3 * r], Hx_r), Bx_l = cmul(g.mu[3 * l], Hx_l),
                      Bx_d = cmul(g.mu[3 * dn], Hx_d), Bx_dr = cmul(g.mu[3 * dr], Hx_dr);
        const double2 By = cmul(g.mu[3 * c + 1], Hy), By_u = cmul(g.mu[3 * u + 1], Hy_u),
                      By_d = cmul(g.mu[3 * dn + 1], Hy_d), By_l = cmul(g.mu[3 * l + 1], Hy_l),
                      By_ul = cmul(g.mu[3 * ul + 1], Hy_ul);
        const double2 imz = g.inv_muz[c], imz_l = g.inv_muz[l], imz_d = g.inv_muz[dn];
        const double2 iez = g.inv_epz[c], iez_r = g.inv_epz[r], iez_u = g.inv_epz[u];
        const double2 sx = g.pml[2 * c], sx_u = g.pml[2 * u], sx_d = g.pml[2 * dn], sx_r = g.pml[2 * r],
                      sx_l = g.pml[2 * l];
        const double2 sy = g.pml[2 * c + 1], sy_u = g.pml[2 * u + 1], sy_d = g.pml[2 * dn + 1],
                      sy_r = g.pml[2 * r + 1], sy_l = g.pml[2 * l + 1];
        (void)sx_d;
        const double2 Bx_dx = cdiv(csmul(d, csub(Bx_r, Bx)), sx);
        const double2 Bx_dx_l = cdiv(csmul(d, csub(Bx, Bx_l)), sx_l);
        const double2 Bx_dx_d = cdiv(csmul(d, csub(Bx_dr, Bx_d)), sx_d);
        const double2 By_dy = cdiv(csmul(d, csub(By_u, By)), sy);
        const double2 By_dy_d = cdiv(csmul(d, csub(By, By_d)), sy_d);
        const double2 By_dy_l = cdiv(csmul(d, csub(By_ul, By_l)), sy_l);
        const double2 Hx_dy = cdiv(csmul(d, csub(Hx, Hx_d)), sy);
        const double2 Hx_dy_u = cdiv(csmul(d, csub(Hx_u, Hx)), sy_u);
        const double2 Hx_dy_r = cdiv(csmul(d, csub(Hx_r, Hx_dr)), sy_r);
        const double2 Hy_dx = cdiv(csmul(d, csub(Hy, Hy_l)), sx);
        const double2 Hy_dx_r = cdiv(csmul(d, csub(Hy_r, Hy)), sx_r);
        const double2 Hy_dx_u = cdiv(csmul(d, csub(Hy_u, Hy_ul)), sx_u);
        const double2 epx = g.ep[3 * c], epy = g.ep[3 * c + 1];
        const double2 x1 = cdiv(csmul(d, csub(cmul(imz, Bx_dx), cmul(imz_l, Bx_dx_l))), sx);
        const double2 x2 = cdiv(csmul(d, csub(cmul(imz, By_dy), cmul(imz_l, By_dy_l))), sx);
        const double2 x3 = cdiv(cmul(csmul(-d, epy), csub(cmul(iez_u, Hy_dx_u), cmul(iez, Hy_dx))), sy);
        const double2 x4 = cdiv(cmul(csmul(d, epy), csub(cmul(iez_u, Hx_dy_u), cmul(iez, Hx_dy))), sy);
        const double2 x5 = csmul(g.omega2, cmul(cmul(epy, g.mu[3 * c]), Hx));
        const double2 y1 = cdiv(csmul(d, csub(cmul(imz, Bx_dx), cmul(imz_d, Bx_dx_d))), sy);
        const double2 y2 = cdiv(csmul(d, csub(cmul(imz, By_dy), cmul(imz_d, By_dy_d))), sy);
        const double2 y3 = cdiv(cmul(csmul(d, epx), csub(cmul(iez_r, Hy_dx_r), cmul(iez, Hy_dx))), sx);
        const double2 y4 = cdiv(cmul(csmul(-d, epx), csub(cmul(iez_r, Hx_dy_r), cmul(iez, Hx_dy))), sx);
        const double2 y5 = csmul(g.omega2, cmul(cmul(epx, g.mu[3 * c + 1]), Hy));
        out[2 * c] = cadd(cadd(cadd(x1, x2), cadd(x3, x4)), x5);
        out[2 * c + 1] = cadd(cadd(cadd(y1, y2), cadd(y3, y4)), y5);
    }
}

// ---- inner products: disc^2 * sum conj(a) b over (Hx, Hy) -----------------
// Blocks write partials; the last block to finish (completion count after a
// fence) adds them in block order and writes *out (optionally also
// sqrt(|out|) to *norm_out) and resets the count.  Deterministic.
constexpr int kDotBlocks = 148, kDotThreads = 256;

__global__ void __launch_bounds__(kDotThreads) k_ms_dot(const double2 *a, const double2 *b, int n2, double disc2,
                                                      double2 *partials, unsigned *done, double2 *out,
                                                      double *norm_out)
{
    double sre = 0.0, sim = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += gridDim.x * blockDim.x) {
        const double2 p = cmul(cconj(a[t]), b[t]);
        sre = dadd(sre, p.x);
        sim = dadd(sim, p.y);
    }
    for (int o = 16; o > 0; o >>= 1) {
        sre = dadd(sre, __shfl_down_sync(0xffffffffu, sre, o));
        sim = dadd(sim, __shfl_down_sync(0xffffffffu, sim, o));
    }
    __shared__ double2 ws[kDotThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) ws[warp] = make_double2(sre, sim);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 v = ws[0];
        for (int w = 1; w < kDotThreads / 32; w++) v = cadd(v, ws[w]);
        partials[blockIdx.x] = v;
    }
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double2 s = partials[0];
    for (int p = 1; p < (int)gridDim.x; p++) s = cadd(s, partials[p]);
    s = csmul(disc2, s);
    *out = s;
    if (norm_out) *norm_out = __dsqrt_rn(cmag(s));
    *done = 0u;
}

// y -= (*coef) x
__global__ void k_ms_axpy(double2 *y, const double2 *x, const double2 *coef, int n2)
{
    const double2 c = *coef;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += gridDim.x * blockDim.x)
        y[t] = csub(y[t], cmul(c, x[t]));
}

// y *= 1 / *norm (mode_H_normalize: divisor = 1/norm)
__global__ void k_ms_scale(double2 *y, const double *norm, int n2)
{
    const double s = 1.0 / *norm;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += gridDim.x * blockDim.x) y[t] = csmul(s, y[t]);
}

// boundary condition (mode.c:1381-1632): confinement 2 zeroes the window edge;
// confinement 1 zeroes rows 0 and mj-1 (columns 1..mi-2) and copies the
// neighbour column into columns 0 and mi-1 (every row)
__global__ void k_ms_bc(double2 *v, int mi, int mj, int confinement)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const double2 z = make_double2(0.0, 0.0);
    if (confinement == 2) {
        // left/right columns (all rows), then top/bottom rows (inner columns)
        if (t < mj) {
            const int cr = (t + 1) * mi - 1, cl = t * mi;
            v[2 * cr] = z; v[2 * cr + 1] = z;
            v[2 * cl] = z; v[2 * cl + 1] = z;
        }
        if (t >= 1 && t < mi - 1) {
            const int ct = t + (mj - 1) * mi, cb = t;
            v[2 * ct] = z; v[2 * ct + 1] = z;
            v[2 * cb] = z; v[2 * cb + 1] = z;
        }
    }
}

// confinement 1 in two ordered launches: vertical zero first, then the
// horizontal zero-gradient copy (which reads the already-zeroed rows)
__global__ void k_ms_bc1_vertical(double2 *v, int mi, int mj)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 1 && t < mi - 1) {
        const double2 z = make_double2(0.0, 0.0);
        const int ct = t + (mj - 1) * mi, cb = t;
        v[2 * ct] = z; v[2 * ct + 1] = z;
        v[2 * cb] = z; v[2 * cb + 1] = z;
    }
}

__global__ void k_ms_bc1_horizontal(double2 *v, int mi, int mj)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < mj) {
        const int cr = (t + 1) * mi - 1, cl = t * mi;
        v[2 * cr] = v[2 * (cr - 1)]; v[2 * cr + 1] = v[2 * (cr - 1) + 1];
        v[2 * cl] = v[2 * (cl + 1)]; v[2 * cl + 1] = v[2 * (cl + 1) + 1];
    }
}

// zero the cells whose PML stretch has an imaginary part (mode.c:1587-1612)
__global__ void k_ms_zero_pml(double2 *v, const double2 *pml, int n)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        if (pml[2 * c].y > 1e-9 || pml[2 * c + 1].y > 1e-9) {
            v[2 * c] = make_double2(0.0, 0.0);
            v[2 * c + 1] = make_double2(0.0, 0.0);
        }
    }
}

// reflection x -> mi-1-x with Hx -> -Hx (mode.c:4494-4527)
__global__ void k_ms_reflect(const double2 *v, double2 *r, int mi, int mj)
{
    const int n = mi * mj;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % mi, j = c / mi;
        const int s = (mi - 1 - i) + j * mi;
        r[2 * s] = csub(make_double2(0.0, 0.0), v[2 * c]);
        r[2 * s + 1] = v[2 * c + 1];
    }
}

// v += (+1 or -1 by the sign of Re *ip) r
__global__ void k_ms_symmetrise(double2 *v, const double2 *r, const double2 *ip, int n2)
{
    const double2 s = make_double2(ip->x > 0 ? 1.0 : -1.0, 0.0);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += gridDim.x * blockDim.x)
        v[t] = cadd(v[t], cmul(s, r[t]));
}

// psi = sum_j y_j k_j, j = 0..m-1 in order (k_j at basis + j*n2)
__global__ void k_ms_combine(double2 *psi, const double2 *basis, const double2 *y, int m, int n2)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += gridDim.x * blockDim.x) {
        double2 s = make_double2(0.0, 0.0);
        for (int j = 0; j < m; j++) s = cadd(s, cmul(y[j], basis[(long long)j * n2 + t]));
        psi[t] = s;
    }
}

// final fields in the reference layout: Hx, Hy from v; Hz = -i/beta (dBx/dx +
// dBy/dy) on interior cells (mode.c:3350-3395); then the boundary condition;
// then E = (-i/omega) ep^-1 curl H on interior cells (mode.c:2330-2397)
__global__ void k_ms_fields_h(MsGeom g, const double2 *v, double2 *f, double2 beta)
{
    const int mi = g.mi, mj = g.mj, n = mi * mj;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        double2 *o = f + 6 * c;
        o[3] = v[2 * c];
        o[4] = v[2 * c + 1];
        o[0] = o[1] = o[2] = o[5] = make_double2(0.0, 0.0);
    }
}

__global__ void k_ms_hz(MsGeom g, double2 *f, double2 beta)
{
    const int mi = g.mi, mj = g.mj, n = mi * mj;
    const double d = 1.0 / g.disc;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % mi, j = c / mi;
        if (i < 1 || i > mi - 2 || j < 1 || j > mj - 2) continue;
        const int r = c + 1, u = c + mi;
        const double2 Bx = cmul(g.mu[3 * c], f[6 * c + 3]), By = cmul(g.mu[3 * c + 1], f[6 * c + 4]);
        const double2 Bx_r = cmul(g.mu[3 * r], f[6 * r + 3]), By_u = cmul(g.mu[3 * u + 1], f[6 * u + 4]);
        const double2 Bx_dx = cdiv(csmul(d, csub(Bx_r, Bx)), g.pml[2 * c]);
        const double2 By_dy = cdiv(csmul(d, csub(By_u, By)), g.pml[2 * c + 1]);
        f[6 * c + 5] = cmul(cdiv(make_double2(0.0, -1.0), beta), cadd(Bx_dx, By_dy));
    }
}

// boundary condition on all 6 components of the final fields
__global__ void k_ms_bc_full(double2 *f, int mi, int mj, int confinement, int pass)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const double2 z = make_double2(0.0, 0.0);
    if (confinement == 2) {
        if (t < mj) {
            const int cr = (t + 1) * mi - 1, cl = t * mi;
            for (int m = 0; m < 6; m++) { f[6 * cr + m] = z; f[6 * cl + m] = z; }
        }
        if (t >= 1 && t < mi - 1) {
            const int ct = t + (mj - 1) * mi, cb = t;
            for (int m = 0; m < 6; m++) { f[6 * ct + m] = z; f[6 * cb + m] = z; }
        }
    } else if (pass == 0) {
        if (t >= 1 && t < mi - 1) {
            const int ct = t + (mj - 1) * mi, cb = t;
            for (int m = 0; m < 6; m++) { f[6 * ct + m] = z; f[6 * cb + m] = z; }
        }
    } else {
        if (t < mj) {
            const int cr = (t + 1) * mi - 1, cl = t * mi;
            for (int m = 0; m < 6; m++) { f[6 * cr + m] = f[6 * (cr - 1) + m]; f[6 * cl + m] = f[6 * (cl + 1) + m]; }
        }
    }
}

__global__ void k_ms_e(MsGeom g, double2 *f, double2 beta, double omega)
{
    const int mi = g.mi, mj = g.mj, n = mi * mj;
    const double d = 1.0 / g.disc;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % mi, j = c / mi;
        if (i < 1 || i > mi - 2 || j < 1 || j > mj - 2) continue;
        const int l = c - 1, dn = c - mi;
        const double2 Hx = f[6 * c + 3], Hy = f[6 * c + 4], Hz = f[6 * c + 5];
        const double2 Hy_l = f[6 * l + 4], Hz_l = f[6 * l + 5];
        const double2 Hx_d = f[6 * dn + 3], Hz_d = f[6 * dn + 5];
        const double2 sx = g.pml[2 * c], sy = g.pml[2 * c + 1];
        const double2 dx_Hy = cdiv(csmul(d, csub(Hy, Hy_l)), sx);
        const double2 dx_Hz = cdiv(csmul(d, csub(Hz, Hz_l)), sx);
        const double2 dy_Hx = cdiv(csmul(d, csub(Hx, Hx_d)), sy);
        const double2 dy_Hz = cdiv(csmul(d, csub(Hz, Hz_d)), sy);
        const double2 iex = crecip(g.ep[3 * c]), iey = crecip(g.ep[3 * c + 1]), iez = g.inv_epz[c];
        const double2 mi_om = csmul(1.0 / omega, make_double2(0.0, -1.0));
        const double2 ib = cmul(make_double2(0.0, 1.0), beta);
        f[6 * c + 0] = cmul(mi_om, cmul(iex, cadd(dy_Hz, cmul(ib, Hy))));
        f[6 * c + 1] = cmul(mi_om, csmul(-1.0, cmul(iey, cadd(dx_Hz, cmul(ib, Hx)))));
        f[6 * c + 2] = cmul(mi_om, cmul(iez, csub(dx_Hy, dy_Hx)));
    }
}

// final H normalisation over all 6 components by 1/|H| (mode_H_normalize)
__global__ void k_ms_scale_full(double2 *f, const double *norm, int n6)
{
    const double s = 1.0 / *norm;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n6; t += gridDim.x * blockDim.x) f[t] = csmul(s, f[t]);
}

// H inner product over the Hx, Hy entries of 6-component fields: gather them first
__global__ void k_ms_gather_h(const double2 *f, double2 *v, int n)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        v[2 * c] = f[6 * c + 3];
        v[2 * c + 1] = f[6 * c + 4];
    }
}

// ============================================================================
// host side
// ============================================================================
namespace {

int grid_blocks(long long n, int threads = 256)
{
    long long b = (n + threads - 1) / threads;
    return (int)(b < 1184 ? (b < 1 ? 1 : b) : 1184);
}

// eigenvalues of an upper Hessenberg complex matrix (row-major n x n) by
// single-shift QR with Wilkinson shifts and deflation (Givens rotations)
bool hessenberg_eigenvalues(std::vector<cd> A, int n, std::vector<cd> &ev)
{
    ev.assign(n, cd(0, 0));
    auto at = [&](int r, int c) -> cd & { return A[(size_t)r * n + c]; };
    int hi = n - 1, iter = 0, total = 0;
    const double eps = 1e-15;
    while (hi >= 0) {
        if (hi == 0) {
            ev[0] = at(0, 0);
            break;
        }
        int l = hi;
        while (l > 0) {
            const double s = std::abs(at(l - 1, l - 1)) + std::abs(at(l, l));
            if (std::abs(at(l, l - 1)) <= eps * (s > 0 ? s : 1.0)) break;
            l--;
        }
        if (l == hi) {
            ev[hi] = at(hi, hi);
            hi--;
            iter = 0;
            continue;
        }
        if (++total > 100000) return false;
        // Wilkinson shift from the trailing 2x2 of the active block
        const cd a = at(hi - 1, hi - 1), b = at(hi - 1, hi), c = at(hi, hi - 1), d = at(hi, hi);
        const cd tr = a + d, det = a * d - b * c;
        const cd disc = std::sqrt(tr * tr / 4.0 - det);
        const cd m1 = tr / 2.0 + disc, m2 = tr / 2.0 - disc;
        cd mu = std::abs(m1 - d) < std::abs(m2 - d) ? m1 : m2;
        if (iter > 0 && iter % 12 == 0) mu = d + std::abs(c);   // exceptional shift
        iter++;
        // QR step on rows/columns l..hi of A - mu I
        for (int k = l; k <= hi; k++) at(k, k) -= mu;
        std::vector<cd> cs(hi - l), sn(hi - l);
        for (int k = l; k < hi; k++) {
            const cd x = at(k, k), y = at(k + 1, k);
            const double r = std::sqrt(std::norm(x) + std::norm(y));
            cd cc = 1.0, ss = 0.0;
            if (r > 0) { cc = x / r; ss = y / r; }
            cs[k - l] = cc; sn[k - l] = ss;
            // rows k, k+1 <- G^H [row k; row k+1]
            for (int col = k; col < n; col++) {
                const cd t1 = at(k, col), t2 = at(k + 1, col);
                at(k, col) = std::conj(cc) * t1 + std::conj(ss) * t2;
                at(k + 1, col) = -ss * t1 + cc * t2;
            }
        }
        for (int k = l; k < hi; k++) {
            const cd cc = cs[k - l], ss = sn[k - l];
            // columns k, k+1 <- [col k, col k+1] G
            for (int row = 0; row <= std::min(k + 2, hi); row++) {
                const cd t1 = at(row, k), t2 = at(row, k + 1);
                at(row, k) = t1 * cc + t2 * ss;
                at(row, k + 1) = -t1 * std::conj(ss) + t2 * std::conj(cc);
            }
        }
        for (int k = l; k <= hi; k++) at(k, k) += mu;
    }
    return true;
}

// solve B x = b (row-major n x n) by Gaussian elimination with partial pivoting
bool linear_solve(std::vector<cd> B, std::vector<cd> b, int n, std::vector<cd> &x)
{
    for (int k = 0; k < n; k++) {
        int p = k;
        for (int r = k + 1; r < n; r++)
            if (std::abs(B[(size_t)r * n + k]) > std::abs(B[(size_t)p * n + k])) p = r;
        if (std::abs(B[(size_t)p * n + k]) == 0.0) return false;
        if (p != k) {
            for (int c = 0; c < n; c++) std::swap(B[(size_t)k * n + c], B[(size_t)p * n + c]);
            std::swap(b[k], b[p]);
        }
        for (int r = k + 1; r < n; r++) {
            const cd f = B[(size_t)r * n + k] / B[(size_t)k * n + k];
            if (f == cd(0, 0)) continue;
            for (int c = k; c < n; c++) B[(size_t)r * n + c] -= f * B[(size_t)k * n + c];
            b[r] -= f * b[k];
        }
    }
    x.assign(n, cd(0, 0));
    for (int r = n - 1; r >= 0; r--) {
        cd s = b[r];
        for (int c = r + 1; c < n; c++) s -= B[(size_t)r * n + c] * x[c];
        x[r] = s / B[(size_t)r * n + r];
    }
    return true;
}

// complex_sqrt of complex.c:151-167 (angle with the 11-digit pi of complex.c,
// exponential by the same power series)
cd reference_sqrt(cd x)
{
    const double pi = 3.14159265359;
    const double mag = std::sqrt(std::sqrt(x.real() * x.real() + x.imag() * x.imag()));
    double angle = std::atan(x.imag() / x.real());
    if (x.real() < 0) angle += pi;
    else if (x.imag() < 0) angle += 2 * pi;
    if (angle > pi) angle -= 2 * pi;
    angle /= 2;
    double re, im;
    cexp_series(angle, &re, &im);
    return cd(mag * re, mag * im);
}

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

template <typename T> bool dev_alloc(DevBuf &b, size_t count, T **out)
{
    if (!cuda_ok(cudaMalloc(&b.p, count * sizeof(T) + 16), "cudaMalloc(mode solver)")) return false;
    *out = (T *)b.p;
    return true;
}

#define MSK(call)                                      \
    do {                                               \
        if (!cuda_ok((call), #call)) return false;     \
    } while (0)

struct Solver {
    int mi = 0, mj = 0, n = 0, n2 = 0;
    double disc = 0, omega = 0;
    cudaStream_t st = nullptr;
    DevBuf b_ep, b_mu, b_pml, b_iez, b_imz, b_psi, b_basis, b_tmp, b_part, b_done, b_scal, b_norm, b_y, b_prev, b_f;
    double2 *ep = nullptr, *mu = nullptr, *pml = nullptr, *iez = nullptr, *imz = nullptr;
    double2 *psi = nullptr, *basis = nullptr, *tmp = nullptr, *part = nullptr, *scal = nullptr, *y = nullptr;
    double2 *prev = nullptr, *f = nullptr;
    double *norm = nullptr;
    unsigned *done = nullptr;
    MsGeom g{};

    ~Solver()
    {
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    }

    bool setup(const mode &m, double om, int basis_vectors, int nprev)
    {
        mi = m.i; mj = m.j; n = mi * mj; n2 = 2 * n;
        disc = m.disc; omega = om;
        MSK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        if (!dev_alloc(b_ep, 3 * (size_t)n, &ep) || !dev_alloc(b_mu, 3 * (size_t)n, &mu) ||
            !dev_alloc(b_pml, 2 * (size_t)n, &pml) || !dev_alloc(b_iez, n, &iez) || !dev_alloc(b_imz, n, &imz) ||
            !dev_alloc(b_psi, n2, &psi) || !dev_alloc(b_basis, (size_t)basis_vectors * n2, &basis) ||
            !dev_alloc(b_tmp, n2, &tmp) || !dev_alloc(b_part, kDotBlocks, &part) ||
            !dev_alloc(b_done, 1, &done) || !dev_alloc(b_scal, (size_t)(basis_vectors + 1) * (basis_vectors + 1) + 8, &scal) ||
            !dev_alloc(b_norm, (size_t)basis_vectors + 8, &norm) || !dev_alloc(b_y, basis_vectors + 1, &y) ||
            !dev_alloc(b_prev, (size_t)(nprev > 0 ? nprev : 1) * n2, &prev) || !dev_alloc(b_f, 6 * (size_t)n, &f))
            return false;
        MSK(cudaMemsetAsync(done, 0, sizeof(unsigned), st));
        static_assert(sizeof(complex) == sizeof(double2), "complex layout");
        MSK(cudaMemcpyAsync(ep, m.ep.m, 3 * (size_t)n * sizeof(double2), cudaMemcpyHostToDevice, st));
        MSK(cudaMemcpyAsync(mu, m.mu.m, 3 * (size_t)n * sizeof(double2), cudaMemcpyHostToDevice, st));
        MSK(cudaMemcpyAsync(pml, m.pml.m, 2 * (size_t)n * sizeof(double2), cudaMemcpyHostToDevice, st));
        g.mi = mi; g.mj = mj; g.disc = disc; g.omega2 = om * om;
        g.ep = ep; g.mu = mu; g.pml = pml; g.inv_epz = iez; g.inv_muz = imz;
        note_launch();
        k_ms_inverses<<<grid_blocks(n), 256, 0, st>>>(g, iez, imz);
        return cuda_ok(cudaGetLastError(), "mode solver setup");
    }

    // *out = <a, b>_H (and *nrm = sqrt|<a,b>| when nrm)
    void dot(const double2 *a, const double2 *b, double2 *out, double *nrm)
    {
        note_launch();
        k_ms_dot<<<kDotBlocks, kDotThreads, 0, st>>>(a, b, n2, disc * disc, part, done, out, nrm);
    }
    void axpy(double2 *v, const double2 *x, const double2 *coef)
    {
        note_launch();
        k_ms_axpy<<<grid_blocks(n2), 256, 0, st>>>(v, x, coef, n2);
    }
    void scale(double2 *v, const double *nrm)
    {
        note_launch();
        k_ms_scale<<<grid_blocks(n2), 256, 0, st>>>(v, nrm, n2);
    }
    void normalize(double2 *v)
    {
        dot(v, v, scal, norm);
        scale(v, norm);
    }
    void bc(double2 *v, int confinement)
    {
        const int len = mi > mj ? mi : mj;
        note_launch();
        if (confinement == 2) {
            k_ms_bc<<<(len + 255) / 256, 256, 0, st>>>(v, mi, mj, 2);
        } else {
            k_ms_bc1_vertical<<<(len + 255) / 256, 256, 0, st>>>(v, mi, mj);
            note_launch();
            k_ms_bc1_horizontal<<<(len + 255) / 256, 256, 0, st>>>(v, mi, mj);
        }
    }
    void apply(const double2 *in, double2 *out)
    {
        note_launch();
        k_ms_beta2<<<grid_blocks(n), 256, 0, st>>>(g, in, out);
    }
};

}  // namespace

bool mode_apply_beta2_device(const mode &in, double omega, mode &out)
{
    Solver s;
    if (!s.setup(in, omega, 1, 0)) return false;
    std::vector<double2> h((size_t)s.n2);
    for (int c = 0; c < s.n; c++) {
        h[2 * c] = make_double2(in.fields.m[6 * c + 3].re, in.fields.m[6 * c + 3].im);
        h[2 * c + 1] = make_double2(in.fields.m[6 * c + 4].re, in.fields.m[6 * c + 4].im);
    }
    MSK(cudaMemcpyAsync(s.psi, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice, s.st));
    s.apply(s.psi, s.tmp);
    MSK(cudaGetLastError());
    MSK(cudaMemcpyAsync(h.data(), s.tmp, h.size() * sizeof(double2), cudaMemcpyDeviceToHost, s.st));
    MSK(cudaStreamSynchronize(s.st));
    for (int c = 0; c < s.n; c++) {
        for (int m = 0; m < 6; m++) out.fields.m[6 * c + m] = complex{0.0, 0.0};
        out.fields.m[6 * c + 3] = complex{h[2 * c].x, h[2 * c].y};
        out.fields.m[6 * c + 4] = complex{h[2 * c + 1].x, h[2 * c + 1].y};
    }
    return true;
}

bool mode_solve_device(mode *psi, double omega, double tol, const mode *prev, int nprev, int size, int confinement,
                       int lateral_symmetry, int max_restarts, cd *beta_out, int *restarts_out)
{
    const int K = size;
    Solver s;
    if (!s.setup(*psi, omega, K + 1, nprev)) return false;
    const int n = s.n, n2 = s.n2;
    // start vector: mode_initialize_rand (mode.c:1192-1206), Hx then Hy per cell
    std::vector<double2> h((size_t)n2);
    for (int c = 0; c < n; c++) {
        h[2 * c] = make_double2((double)rand(), 0.0);
        h[2 * c + 1] = make_double2((double)rand(), 0.0);
    }
    MSK(cudaMemcpyAsync(s.psi, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice, s.st));
    for (int p = 0; p < nprev; p++) {
        for (int c = 0; c < n; c++) {
            h[2 * c] = make_double2(prev[p].fields.m[6 * c + 3].re, prev[p].fields.m[6 * c + 3].im);
            h[2 * c + 1] = make_double2(prev[p].fields.m[6 * c + 4].re, prev[p].fields.m[6 * c + 4].im);
        }
        MSK(cudaMemcpyAsync(s.prev + (size_t)p * n2, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice,
                            s.st));
        MSK(cudaStreamSynchronize(s.st));   // h is reused
    }
    s.normalize(s.psi);   // mode_H_normalize after the random start
    // scalar slots on the device: scal[0] scratch, scal[1 + r*K + c] = H(r, c)
    double2 *Hd = s.scal + 1;
    std::vector<double2> Hh((size_t)K * K);
    std::vector<cd> H((size_t)K * K), ev, yv;
    cd beta(0, 0);
    double n_mag = 100.0, n_diff = 100.0;
    int restarts = 0;
    while (std::fabs(n_diff) > tol) {
        if (restarts >= max_restarts) {
            set_error(FDTD_ERR_TIMEOUT, "mode solver: |n_eff| still changing by %.3g after %d restarts", n_diff,
                      restarts);
            return false;
        }
        // orthogonalise against previous modes (one pass), normalising in between
        s.normalize(s.psi);
        for (int p = nprev - 1; p >= 0; p--) {
            s.dot(s.prev + (size_t)p * n2, s.psi, s.scal, nullptr);
            s.axpy(s.psi, s.prev + (size_t)p * n2, s.scal);
            s.normalize(s.psi);
        }
        s.bc(s.psi, confinement);   // after mode_apply_H_curl, which only changes E
        if (lateral_symmetry) {
            note_launch();
            k_ms_reflect<<<grid_blocks(n), 256, 0, s.st>>>(s.psi, s.tmp, s.mi, s.mj);
            s.dot(s.psi, s.tmp, s.scal, nullptr);
            note_launch();
            k_ms_symmetrise<<<grid_blocks(n2), 256, 0, s.st>>>(s.psi, s.tmp, s.scal, n2);
        }
        note_launch();
        k_ms_zero_pml<<<grid_blocks(n), 256, 0, s.st>>>(s.psi, s.pml, n);
        // Krylov basis k_0..k_K
        double2 *k0 = s.basis;
        MSK(cudaMemcpyAsync(k0, s.psi, (size_t)n2 * sizeof(double2), cudaMemcpyDeviceToDevice, s.st));
        s.normalize(k0);
        s.bc(k0, confinement);
        MSK(cudaMemsetAsync(Hd, 0, (size_t)K * K * sizeof(double2), s.st));
        for (int i = 1; i <= K; i++) {
            double2 *ki = s.basis + (size_t)i * n2;
            s.apply(s.basis + (size_t)(i - 1) * n2, ki);
            s.bc(ki, confinement);
            for (int j = 0; j < i; j++) {
                double2 *hji = Hd + (size_t)j * K + (i - 1);
                s.dot(s.basis + (size_t)j * n2, ki, hji, nullptr);
                s.axpy(ki, s.basis + (size_t)j * n2, hji);
            }
            if (i < K) {
                // subdiagonal H(i, i-1) = |k_i|, then normalise
                s.dot(ki, ki, s.scal, s.norm + i);
                note_launch();
                k_ms_scale<<<grid_blocks(n2), 256, 0, s.st>>>(ki, s.norm + i, n2);
            }
        }
        MSK(cudaGetLastError());
        std::vector<double> sub((size_t)K + 8);
        MSK(cudaMemcpyAsync(Hh.data(), Hd, Hh.size() * sizeof(double2), cudaMemcpyDeviceToHost, s.st));
        MSK(cudaMemcpyAsync(sub.data(), s.norm, (size_t)K * sizeof(double), cudaMemcpyDeviceToHost, s.st));
        MSK(cudaStreamSynchronize(s.st));
        for (int r = 0; r < K; r++)
            for (int c = 0; c < K; c++) H[(size_t)r * K + c] = cd(Hh[(size_t)r * K + c].x, Hh[(size_t)r * K + c].y);
        for (int i = 1; i < K; i++) H[(size_t)i * K + (i - 1)] = cd(sub[i], 0.0);
        // eigenvalue with the largest real part (index 0 unless some real part > 0)
        if (!hessenberg_eigenvalues(H, K, ev)) {
            set_error(FDTD_ERR_CUDA, "mode solver: Hessenberg QR did not converge");
            return false;
        }
        int best = 0;
        double bmax = 0.0;
        for (int i = 0; i < K; i++)
            if (ev[i].real() > bmax) { bmax = ev[i].real(); best = i; }
        const cd lam = ev[best];
        // eigenvector from (H - lambda I) with the last row replaced by ones, rhs n e_n
        std::vector<cd> B(H), rhs((size_t)K, cd(0, 0));
        for (int i = 0; i < K; i++) B[(size_t)i * K + i] -= lam;
        for (int c = 0; c < K; c++) B[(size_t)(K - 1) * K + c] = cd(1, 0);
        rhs[K - 1] = cd((double)K, 0);
        if (!linear_solve(B, rhs, K, yv)) {
            set_error(FDTD_ERR_CUDA, "mode solver: singular eigenvector system");
            return false;
        }
        double yn = 0;
        for (auto &v : yv) yn += std::norm(v);
        yn = std::sqrt(yn);
        std::vector<double2> yd((size_t)K);
        for (int i = 0; i < K; i++) yd[i] = make_double2(yv[i].real() / yn, yv[i].imag() / yn);
        MSK(cudaMemcpyAsync(s.y, yd.data(), yd.size() * sizeof(double2), cudaMemcpyHostToDevice, s.st));
        note_launch();
        k_ms_combine<<<grid_blocks(n2), 256, 0, s.st>>>(s.psi, s.basis, s.y, K, n2);
        MSK(cudaGetLastError());
        MSK(cudaStreamSynchronize(s.st));   // yd is a host temporary
        beta = reference_sqrt(lam);
        const cd n_eff = beta / omega;
        const double n_old = n_mag;
        n_mag = std::abs(n_eff);
        n_diff = n_mag - n_old;
        restarts++;
    }
    // final fields: Hz from div B, boundary, E from curl H, boundary, H-normalise
    const double2 b2 = make_double2(beta.real(), beta.imag());
    note_launch();
    k_ms_fields_h<<<grid_blocks(n), 256, 0, s.st>>>(s.g, s.psi, s.f, b2);
    note_launch();
    k_ms_hz<<<grid_blocks(n), 256, 0, s.st>>>(s.g, s.f, b2);
    const int len = s.mi > s.mj ? s.mi : s.mj;
    for (int pass = 0; pass < (confinement == 2 ? 1 : 2); pass++) {
        note_launch();
        k_ms_bc_full<<<(len + 255) / 256, 256, 0, s.st>>>(s.f, s.mi, s.mj, confinement, pass);
    }
    note_launch();
    k_ms_e<<<grid_blocks(n), 256, 0, s.st>>>(s.g, s.f, b2, omega);
    for (int pass = 0; pass < (confinement == 2 ? 1 : 2); pass++) {
        note_launch();
        k_ms_bc_full<<<(len + 255) / 256, 256, 0, s.st>>>(s.f, s.mi, s.mj, confinement, pass);
    }
    note_launch();
    k_ms_gather_h<<<grid_blocks(n), 256, 0, s.st>>>(s.f, s.tmp, n);
    s.dot(s.tmp, s.tmp, s.scal, s.norm);
    note_launch();
    k_ms_scale_full<<<grid_blocks(6LL * n), 256, 0, s.st>>>(s.f, s.norm, 6 * n);
    MSK(cudaGetLastError());
    MSK(cudaMemcpyAsync(psi->fields.m, s.f, 6 * (size_t)n * sizeof(double2), cudaMemcpyDeviceToHost, s.st));
    MSK(cudaStreamSynchronize(s.st));
    if (beta_out) *beta_out = beta;
    if (restarts_out) *restarts_out = restarts;
    return true;
}

}  // namespace fdtd
