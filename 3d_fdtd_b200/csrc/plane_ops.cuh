// plane_ops.cuh -- per-cell and per-block pieces of the plane work around the
// stencil (mode source values, mode overlap partials, per-frequency
// accumulation), shared by the per-step kernels (aux_kernels.cu) and the
// multi-step wavefront kernel (yee_wave.cu) so that both compute the same
// values bit for bit.
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace fdtd {

// ---------------------------------------------------------------------------
// Mode plane source, timefield3d_mode_source (timefield3d.c:2977-3026):
//   src[m<3]  = A ep_m (Re cos(phase) + Im sin(phase))
//   src[m>=3] = -M_sign A mu_m (Re cos(phase) + Im sin(phase)),  M_sign = 2 reverse - 1
// from the mode sample at ((int)((i-cx) r) + mi/2, (int)((j-cy) r) + mj/2),
// r = disc / mode.disc; cells whose sample falls outside the mode keep their
// value.  Adjoint variant, timefield3d_mode_source_adjoint
// (timefield3d.c:3028-3068): J = (Hy_m, -Hx_m, 0), M = (-M_sign Ey_m, M_sign Ex_m, 0).
// cos/sin of the phase are computed on the host with the C library, like the
// reference, and passed in; sched != null selects per-step values indexed by
// the device step counter.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void schedule_values(const SourceJob &sj, long long n, double &A, double &c, double &s)
{
    if (n < 0 || n >= sj.nsched) {
        A = 0.0; c = 0.0; s = 0.0;   // outside the schedule: zero source
    } else {
        A = sj.sched[3 * n]; c = sj.sched[3 * n + 1]; s = sj.sched[3 * n + 2];
    }
}

// amplitude and phase of a source plane: entry n of the schedule, and for the
// exact adjoint (adjoint 2) also entry n+1, which drives the H components
struct SrcStep {
    double A, c, s;       // J (E components); all six components otherwise
    double A1, c1, s1;    // M (H components) of the exact adjoint
};

__device__ __forceinline__ SrcStep schedule_step(const SourceJob &sj, long long n)
{
    SrcStep v;
    schedule_values(sj, n, v.A, v.c, v.s);
    if (sj.adjoint == 2) schedule_values(sj, n + 1, v.A1, v.c1, v.s1);
    else { v.A1 = 0.0; v.c1 = 0.0; v.s1 = 0.0; }
    return v;
}

__device__ __forceinline__ SrcStep fixed_step(double A, double c, double s)
{
    SrcStep v;
    v.A = A; v.c = c; v.s = s; v.A1 = 0.0; v.c1 = 0.0; v.s1 = 0.0;
    return v;
}

// Re(w m e^{i phi}) for a mode sample m, with (c, s) = (cos phi, sin phi)
__device__ __forceinline__ double weighted_proj(const SourceJob &sj, double2 m, double c, double s)
{
    const double zr = dsub(dmul(sj.wre, m.x), dmul(sj.wim, m.y));
    const double zi = dadd(dmul(sj.wre, m.y), dmul(sj.wim, m.x));
    return dsub(dmul(zr, c), dmul(zi, s));
}

// the six source values of cell (i, j); false when the cell has no mode
// sample (the plane keeps its value there)
//   adjoint 0: timefield3d_mode_source (timefield3d.c:2977-3026)
//   adjoint 1: timefield3d_mode_source_adjoint (timefield3d.c:3028-3068)
//   adjoint 2: the exact discrete adjoint of an overlap monitor
//     O = sum_n e^{i omega n dt} o_n, o_n = -disc^2/2 sum (Hx mEy - Hy mEx + Ey mHx - Ex mHy)
//     (mode H -> -conj(H) when reverse) for the objective Re(w O): with
//     kappa = disc^2 / (2 dt), the E-update current
//       Jx = -kappa Re(w mHy e^{i phi_n}), Jy = kappa Re(w mHx e^{i phi_n})
//     adds exactly the monitor's E weights (divided by eps) to E, and the
//     H-update current of entry n+1
//       Mx = -kappa Re(w mEy e^{i phi_n+1}), My = kappa Re(w mEx e^{i phi_n+1})
//     adds minus its H weights at the end of the step, i.e. before the next
//     step's E update (the transposed leapfrog step is the same step with H
//     negated, so the adjoint is this forward run; see
//     timefield3d_set_exact_adjoint_schedule).
__device__ __forceinline__ bool mode_source_cell(const SourceJob &sj, int i, int j, const SrcStep &st, float v[6])
{
    const long long t = i + (long long)sj.nx * j;
    const int M_sign = -1 + 2 * sj.reverse;
    double xd = dmul((double)(i - sj.cx), sj.ratio);
    double yd = dmul((double)(j - sj.cy), sj.ratio);
    int mx = (int)xd + sj.mi / 2, my = (int)yd + sj.mj / 2;
    if (mx < 0 || mx >= sj.mi || my < 0 || my >= sj.mj) return false;
    const double2 *e = sj.mode + 6LL * (mx + (long long)sj.mi * my);
    const double A = st.A, c = st.c, s = st.s;
    if (sj.adjoint == 0) {
#pragma unroll
        for (int m = 0; m < 6; m++) {
            double proj = dadd(dmul(e[m].x, c), dmul(e[m].y, s));
            double w;
            if (m < 3) w = dmul(dmul(A, (double)sj.ep[m][t]), proj);
            else w = dmul(dmul(dmul((double)(-M_sign), A), (double)sj.mu[m - 3][t]), proj);
            v[m] = __double2float_rn(w);
        }
    } else if (sj.adjoint == 1) {
        v[0] = __double2float_rn(dmul(1.0, dadd(dmul(e[4].x, c), dmul(e[4].y, s))));
        v[1] = __double2float_rn(dmul(-1.0, dadd(dmul(e[3].x, c), dmul(e[3].y, s))));
        v[2] = 0.0f;
        v[3] = __double2float_rn(dmul((double)(-1 * M_sign), dadd(dmul(e[1].x, c), dmul(e[1].y, s))));
        v[4] = __double2float_rn(dmul((double)(1 * M_sign), dadd(dmul(e[0].x, c), dmul(e[0].y, s))));
        v[5] = 0.0f;
    } else {
        double2 mHx = e[3], mHy = e[4];
        if (sj.reverse) {
            mHx.x = -mHx.x;
            mHy.x = -mHy.x;
        }
        const double k0 = dmul(sj.kappa, A), k1 = dmul(sj.kappa, st.A1);
        v[0] = __double2float_rn(-dmul(k0, weighted_proj(sj, mHy, c, s)));
        v[1] = __double2float_rn(dmul(k0, weighted_proj(sj, mHx, c, s)));
        v[2] = 0.0f;
        v[3] = __double2float_rn(-dmul(k1, weighted_proj(sj, e[1], st.c1, st.s1)));
        v[4] = __double2float_rn(dmul(k1, weighted_proj(sj, e[0], st.c1, st.s1)));
        v[5] = 0.0f;
    }
    return true;
}

// the source plane over the mode window, cells first, first + stride, ...
__device__ __forceinline__ void mode_source_cells(const SourceJob &sj, long long first, long long stride,
                                                  const SrcStep &st)
{
    const long long nxy = (long long)sj.nx * sj.ny;
    const long long cells = (long long)sj.win.wni * sj.win.wnj;
    for (long long u = first; u < cells; u += stride) {
        const int i = sj.win.wi + (int)(u % sj.win.wni), j = sj.win.wj + (int)(u / sj.win.wni);
        const long long t = i + (long long)sj.nx * j;
        float v[6];
        if (!mode_source_cell(sj, i, j, st, v)) continue;
#pragma unroll
        for (int m = 0; m < 6; m++) sj.plane[m * nxy + t] = v[m];
    }
}

// ---------------------------------------------------------------------------
// Mode overlap (timefield3d.c:3176-3233): per cell with a mode sample,
//   Hx mEy - Hy mEx + Ey mHx - Ex mHy   (mode H -> -conj(H) when reverse)
// summed over the plane in FP64.  One grid covers several monitors
// (blockIdx.y); each block writes one partial; the finalize kernel adds the
// partials in a fixed order (deterministic), scales by -dx^2/2 and, for
// monitors, accumulates e^{i omega n dt} o(n) per frequency with Kahan
// compensation.
// ---------------------------------------------------------------------------
// the sums of thread vt of a bdim-thread block computing partial `part` of
// `nparts` of one job's plane sum: window cells part*bdim + vt, strided by
// nparts*bdim
template <typename T>
__device__ __forceinline__ void overlap_thread_sum(const T *const *Ex_, int nx, int ny, const OverlapJob &jb, int vt,
                                                   int bdim, int part, int nparts, double &sre, double &sim)
{
    const long long nxy = (long long)nx * ny;
    const T *Ex = Ex_[0], *Ey = Ex_[1], *Hx = Ex_[3], *Hy = Ex_[4];
    const long long base = nxy * jb.cz;
    const long long cells = (long long)jb.win.wni * jb.win.wnj;
    sre = 0.0;
    sim = 0.0;
    for (long long u = part * (long long)bdim + vt; u < cells; u += (long long)nparts * bdim) {
        const int i = jb.win.wi + (int)(u % jb.win.wni), j = jb.win.wj + (int)(u / jb.win.wni);
        const long long t = i + (long long)nx * j;
        double xd = dmul((double)(i - jb.cx), jb.ratio);
        double yd = dmul((double)(j - jb.cy), jb.ratio);
        int mx = (int)xd + jb.mi / 2, my = (int)yd + jb.mj / 2;
        if (mx < 0 || mx >= jb.mi || my < 0 || my >= jb.mj) continue;
        const double2 *e = jb.mode + 6LL * (mx + (long long)jb.mi * my);
        double2 mEx = e[0], mEy = e[1], mHx = e[3], mHy = e[4];
        if (jb.reverse) {
            mHx.x = -mHx.x;
            mHy.x = -mHy.x;
        }
        double ex = (double)Ex[base + t], ey = (double)Ey[base + t];
        double hx = (double)Hx[base + t], hy = (double)Hy[base + t];
        double re = dadd(dsub(dmul(hx, mEy.x), dmul(hy, mEx.x)), dsub(dmul(ey, mHx.x), dmul(ex, mHy.x)));
        double im = dadd(dsub(dmul(hx, mEy.y), dmul(hy, mEx.y)), dsub(dmul(ey, mHx.y), dmul(ex, mHy.y)));
        sre = dadd(sre, re);
        sim = dadd(sim, im);
    }
}

// fixed-shape warp sum (the result is in lane 0)
__device__ __forceinline__ void overlap_warp_reduce(double &sre, double &sim)
{
    for (int o = 16; o > 0; o >>= 1) {
        sre = dadd(sre, __shfl_down_sync(0xffffffffu, sre, o));
        sim = dadd(sim, __shfl_down_sync(0xffffffffu, sim, o));
    }
}

// partial `part` of `nparts` of one job's plane sum, written to *out (all
// threads of the block call it): thread sums, warp sums, then warp 0 adds the
// warp sums with the same fixed shape
template <typename T>
__device__ __forceinline__ void overlap_block(const T *const *Ex_, int nx, int ny, const OverlapJob &jb, int part,
                                              int nparts, double2 *out)
{
    double sre, sim;
    overlap_thread_sum<T>(Ex_, nx, ny, jb, threadIdx.x, blockDim.x, part, nparts, sre, sim);
    overlap_warp_reduce(sre, sim);
    __shared__ double2 ws[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) ws[warp] = make_double2(sre, sim);
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        double2 v = lane < nw ? ws[lane] : make_double2(0.0, 0.0);
        overlap_warp_reduce(v.x, v.y);
        if (lane == 0) *out = v;
    }
}

// the same partial as overlap_block with a 256-thread block, computed by ONE
// warp: the eight warps' sums one after another, then the same final stage
// (all lanes of the warp call it; lane 0 writes *out)
template <typename T>
__device__ __forceinline__ void overlap_warp(const T *const *Ex_, int nx, int ny, const OverlapJob &jb, int part,
                                             int nparts, double2 *out)
{
    const int lane = threadIdx.x & 31;
    double2 mine = make_double2(0.0, 0.0);
    for (int v = 0; v < 8; v++) {
        double sre, sim;
        overlap_thread_sum<T>(Ex_, nx, ny, jb, v * 32 + lane, 256, part, nparts, sre, sim);
        overlap_warp_reduce(sre, sim);
        sre = __shfl_sync(0xffffffffu, sre, 0);
        sim = __shfl_sync(0xffffffffu, sim, 0);
        if (lane == v) mine = make_double2(sre, sim);
    }
    overlap_warp_reduce(mine.x, mine.y);
    if (lane == 0) *out = mine;
}

// reduce_phase: phase - (int)(phase/(2 pi)) 2 pi with the reference's 9-digit pi
// (timefield3d.c:3,3235)
__device__ __forceinline__ double reduce_phase(double ph)
{
    const double two_pi = dmul(2.0, 3.141592652);
    double q = (double)(int)__ddiv_rn(ph, two_pi);
    return dsub(ph, dmul(q, two_pi));
}

// acc[2f] += e^{i omega_f n dt} o with Kahan compensation in acc[2f+1]
// e^{i omega_f n dt} o
__device__ __forceinline__ double2 frequency_term(const OverlapJob &jb, int f, double2 o, double dt, long long n)
{
    double ph = reduce_phase(dmul(dmul((double)n, dt), jb.omega[f]));
    double s, c;
    sincos(ph, &s, &c);
    return make_double2(dsub(dmul(c, o.x), dmul(s, o.y)), dadd(dmul(c, o.y), dmul(s, o.x)));
}

// sum += add with Kahan compensation comp
__device__ __forceinline__ void kahan_add(double2 &sum, double2 &comp, double2 add)
{
    double yr = dsub(add.x, comp.x), yi = dsub(add.y, comp.y);
    double tr = dadd(sum.x, yr), ti = dadd(sum.y, yi);
    comp.x = dsub(dsub(tr, sum.x), yr);
    comp.y = dsub(dsub(ti, sum.y), yi);
    sum = make_double2(tr, ti);
}

__device__ __forceinline__ void accumulate_frequency(const OverlapJob &jb, int f, double2 o, double dt, long long n)
{
    const double2 add = frequency_term(jb, f, o, dt, n);
    double2 sum = jb.acc[2 * f], comp = jb.acc[2 * f + 1];
    kahan_add(sum, comp, add);
    jb.acc[2 * f] = sum;
    jb.acc[2 * f + 1] = comp;
}

}  // namespace fdtd
