// aux_kernels.cu -- plane-sized work around the stencil: mode sources, mode
// overlap monitors, running DFTs, probes and the taper edge store/gradient.
//
// All of it touches one z-plane (or a list of edge cells) per step, so it is
// a small fraction of a step's HBM traffic; what matters is that it stays on
// the device (no per-step host round trip) and that the reductions are FP64.
#include "plane_ops.cuh"

namespace fdtd {

// fixed amplitude and phase, or (sched != null) the schedule entry of step *step + offset
__global__ void k_mode_source(SourceJob sj, double amplitude, double cph, double sph, const long long *step,
                              int step_offset)
{
    const SrcStep v = sj.sched ? schedule_step(sj, *step + step_offset) : fixed_step(amplitude, cph, sph);
    mode_source_cells(sj, blockIdx.x * (long long)blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x, v);
}

__global__ void k_set_value(float *p, long long idx, float v) { p[idx] = v; }

template <typename T>
__global__ void k_overlap_partial(const T *const *Ex_, int nx, int ny, const OverlapJob *jobs, double2 *partials,
                                  int nparts)
{
    const OverlapJob jb = jobs[blockIdx.y];
    overlap_block<T>(Ex_, nx, ny, jb, blockIdx.x, nparts, partials + (long long)blockIdx.y * nparts + blockIdx.x);
}

// sum one job's partials in order, scale, store the instantaneous value and
// accumulate e^{i omega n dt} o per frequency (all threads of the block call it)
__device__ __forceinline__ void overlap_finalize_job(const OverlapJob &jb, const double2 *partials, int nparts,
                                                     double scale, double dt, long long n)
{
    __shared__ double2 tot;
    if (threadIdx.x == 0) {
        double sre = 0.0, sim = 0.0;
        for (int p = 0; p < nparts; p++) {
            double2 v = partials[p];
            sre = dadd(sre, v.x);
            sim = dadd(sim, v.y);
        }
        tot = make_double2(dmul(scale, sre), dmul(scale, sim));
        if (jb.inst) *jb.inst = tot;
    }
    __syncthreads();
    if (!jb.acc) return;
    const double2 o = tot;
    // one thread per frequency
    for (int f = threadIdx.x; f < jb.nfreq; f += blockDim.x) accumulate_frequency(jb, f, o, dt, n);
}

__global__ void k_overlap_finalize(const OverlapJob *jobs, int njobs, const double2 *partials, int nparts,
                                   double scale, double dt, const long long *step, int step_offset)
{
    const int jid = blockIdx.x;
    if (jid >= njobs) return;
    const OverlapJob jb = jobs[jid];
    overlap_finalize_job(jb, partials + (long long)jid * nparts, nparts, scale, dt, *step + step_offset);
}

// ---------------------------------------------------------------------------
// End of one step of a run, in one launch: blocks [0, njobs*nparts) compute
// the overlap partials of the fields just updated, the next `src_blocks`
// write the scheduled source plane of the NEXT step (step counter + 1).  The
// last block to finish (completion count, after a memory fence) adds the
// partials of every job in order -- the order of k_overlap_finalize, so the
// monitors are bit-identical to the separate kernels -- accumulates the
// frequencies, advances the step counter and resets the count for the next
// launch.  Nothing waits on anything: blocks only count themselves out.
// ---------------------------------------------------------------------------
constexpr int kTailJobs = 64;

template <typename T>
__global__ void __launch_bounds__(256) k_step_tail(TailArgs a)
{
    // Programmatic dependent launch (no-ops in a plain launch): wait until the
    // H update has completed and its stores are visible -- that also orders the
    // source plane write after the E update that read it -- then let the next
    // step's E update start scheduling; its blocks wait for this grid in turn.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int nov = a.njobs * a.nparts;
    const int b = blockIdx.x;
    if (b < nov) {
        const int jid = b / a.nparts, part = b - jid * a.nparts;
        const OverlapJob jb = a.jobs[jid];
        overlap_block<T>((const T *const *)a.f, a.nx, a.ny, jb, part, a.nparts, a.partials + b);
    } else {
        const SrcStep v = schedule_step(a.src, *a.step + 1);
        mode_source_cells(a.src, (b - nov) * (long long)blockDim.x + threadIdx.x,
                          (long long)a.src_blocks * blockDim.x, v);
    }
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(a.done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const long long n = *a.step;
    // stage every partial in shared memory, then one thread per job adds its
    // partials in order (the order of k_overlap_finalize)
    constexpr int kStage = 1024;
    __shared__ double2 part[kStage];
    __shared__ double2 tot[kTailJobs];
    const int np = a.njobs * a.nparts;
    const bool staged = np <= kStage && a.njobs <= kTailJobs;
    if (staged) {
        for (int i = threadIdx.x; i < np; i += blockDim.x) part[i] = a.partials[i];
        __syncthreads();
        if (threadIdx.x < a.njobs) {
            const int jid = threadIdx.x;
            double sre = 0.0, sim = 0.0;
            for (int p = 0; p < a.nparts; p++) {
                const double2 v = part[jid * a.nparts + p];
                sre = dadd(sre, v.x);
                sim = dadd(sim, v.y);
            }
            tot[jid] = make_double2(dmul(a.scale, sre), dmul(a.scale, sim));
            const OverlapJob jb = a.jobs[jid];
            if (jb.inst) *jb.inst = tot[jid];
        }
        __syncthreads();
        // one warp per job, one lane per frequency: the jobs' loads, phases
        // and stores overlap instead of following one another
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for (int jid = warp; jid < a.njobs; jid += blockDim.x >> 5) {
            const OverlapJob jb = a.jobs[jid];
            if (!jb.acc) continue;
            for (int f = lane; f < jb.nfreq; f += 32) accumulate_frequency(jb, f, tot[jid], a.dt, n);
        }
    } else {
        for (int jid = 0; jid < a.njobs; jid++) {
            const OverlapJob jb = a.jobs[jid];
            overlap_finalize_job(jb, a.partials + (long long)jid * a.nparts, a.nparts, a.scale, a.dt, n);
            __syncthreads();
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *a.step = n + 1;
        *a.done = 0u;
    }
}

template <typename T>
__global__ void k_dft(const T *const *f, int nx, int ny, int nz, int slice, int k_lo, int k_hi, double tr,
                      double ti, double2 *acc)
{
    const long long nxy = (long long)nx * ny;
    long long cnt = slice >= 0 ? (long long)nx * (k_hi - k_lo) : nxy * (k_hi - k_lo);
    const long long accn = slice >= 0 ? (long long)nx * nz : nxy * nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cnt; t += (long long)gridDim.x * blockDim.x) {
        long long q, a;
        if (slice >= 0) {
            int i = (int)(t % nx);
            int k = k_lo + (int)(t / nx);
            q = i + (long long)nx * slice + nxy * k;
            a = i + (long long)nx * k;
        } else {
            q = nxy * k_lo + t;
            a = q;
        }
#pragma unroll
        for (int m = 0; m < 6; m++) {
            double v = (double)f[m][q];
            double2 s = acc[m * accn + a];
            s.x = dadd(s.x, dmul(v, tr));
            s.y = dadd(s.y, dmul(v, ti));
            acc[m * accn + a] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// Probes: buf[p*cap + count[p]] = f[m_p][q_p] after each step.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_probes(const T *const *f, const ProbeJob *probes, int np, double *buf, int cap, int *count)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    int c = count[p];
    if (c < cap) buf[(long long)p * cap + c] = (double)f[probes[p].m][probes[p].q];
    count[p] = c + 1;
}

__global__ void k_step_advance(long long *step) { *step += 1; }

// ---------------------------------------------------------------------------
// Taper edge store (adjoint3d.c:259-337): gather E (3 components) at the
// rasterised edge pixels of every (edge, j, k); store[t][cell][3].
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_taper_store(const T *const *f, const long long *cells, int ncell, T *store, int t_index,
                              const long long *step, int t0, int dir, int duration)
{
    int t = t_index;
    if (step) t = t0 + dir * (int)(*step);
    if (t < 0 || t >= duration) return;
    T *dst = store + (long long)t * ncell * 3;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        long long q = cells[c];
        dst[3 * c + 0] = f[0][q];
        dst[3 * c + 1] = f[1][q];
        dst[3 * c + 2] = f[2][q];
    }
}

// ep-gradient, adjoint3d_taper_calculate_ep_gradient (adjoint3d.c:339-373):
// g[cell] = sum_t sum_{m<3} fwd * adj, FP64, time-ordered like the reference.
template <typename T>
__global__ void k_ep_gradient(const T *fwd, const T *adj, int ncell, int duration, double *grad)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    double sum = 0.0;
    for (int t = 0; t < duration; t++) {
        const long long o = ((long long)t * ncell + c) * 3;
#pragma unroll
        for (int m = 0; m < 3; m++) sum = dadd(sum, dmul((double)fwd[o + m], (double)adj[o + m]));
    }
    grad[c] = sum;
}

// Exact discrete-adjoint ep-gradient: dF/deps of each stored cell (summed over
// its 3 E components) for a forward store fwd[n] = E after forward step n and
// an adjoint store adj[n] = the exact adjoint's E at forward index n (see
// timefield3d_set_exact_adjoint_schedule):
//   g = -sum_{n=0}^{T-1} adj[n] (fwd[n] - fwd[n-1]),  fwd[-1] = 0.
// A change deps of a cell changes its E update in forward step n by
// -(deps/eps)(E^{n+1} - E^n); the objective's sensitivity to a change of E made
// during step n is eps times the adjoint E of index n (the state before step
// n), so eps cancels.
template <typename T>
__global__ void k_ep_gradient_exact(const T *fwd, const T *adj, int ncell, int duration, double *grad)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    double sum = 0.0;
    for (int t = 0; t < duration; t++) {
        const long long o = ((long long)t * ncell + c) * 3, om = o - 3LL * ncell;
#pragma unroll
        for (int m = 0; m < 3; m++) {
            const double d = t > 0 ? dsub((double)fwd[o + m], (double)fwd[om + m]) : (double)fwd[o + m];
            sum = dadd(sum, dmul((double)adj[o + m], d));
        }
    }
    grad[c] = -sum;
}

template <typename T> void launch_ep_gradient_exact(const T *fwd, const T *adj, int ncell, int duration, double *grad,
                                                    cudaStream_t st)
{
    note_launch();
    k_ep_gradient_exact<T><<<(ncell + 127) / 128, 128, 0, st>>>(fwd, adj, ncell, duration, grad);
}
template void launch_ep_gradient_exact<float>(const float *, const float *, int, int, double *, cudaStream_t);
template void launch_ep_gradient_exact<double>(const double *, const double *, int, int, double *, cudaStream_t);

// ---------------------------------------------------------------------------
// materials: finite check (one flag), and FP32 update coefficients
// ---------------------------------------------------------------------------
__global__ void k_check_finite(const float *a, long long n, int *bad)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        if (!isfinite(a[q])) { *bad = 1; return; }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static int source_blocks(const ModeWindow &w)
{
    const long long cells = (long long)w.wni * w.wnj;
    const long long blocks = (cells + 255) / 256;
    return blocks < 1 ? 1 : blocks > 1184 ? 1184 : (int)blocks;
}

void launch_mode_source(float *plane, const float *const ep_plane[3], const float *const mu_plane[3], int nx, int ny,
                        int cx, int cy, const double2 *mode, int mi, int mj, double ratio, double amplitude,
                        double cph, double sph, const double *sched, const long long *step, int nsched, int reverse,
                        int adjoint, cudaStream_t st)
{
    SourceJob sj{};
    sj.plane = plane;
    for (int c = 0; c < 3; c++) { sj.ep[c] = ep_plane[c]; sj.mu[c] = mu_plane[c]; }
    sj.nx = nx; sj.ny = ny; sj.cx = cx; sj.cy = cy;
    sj.mode = mode; sj.mi = mi; sj.mj = mj; sj.ratio = ratio;
    sj.sched = sched; sj.nsched = nsched; sj.reverse = reverse; sj.adjoint = adjoint;
    launch_mode_source_job(sj, amplitude, cph, sph, step, 0, st);
}

void launch_mode_source_job(const SourceJob &sj_in, double amplitude, double cph, double sph, const long long *step,
                            int step_offset, cudaStream_t st)
{
    SourceJob sj = sj_in;
    sj.win = mode_window(sj.nx, sj.ny, sj.cx, sj.cy, sj.mi, sj.mj, sj.ratio);
    note_launch();
    k_mode_source<<<source_blocks(sj.win), 256, 0, st>>>(sj, amplitude, cph, sph, step, step_offset);
}

template <typename T>
void launch_step_tail(TailArgs a, cudaStream_t st)
{
    a.nparts = a.njobs > 0 ? overlap_parts(a.cells) : 0;
    if (a.src.plane) {
        a.src.win = mode_window(a.src.nx, a.src.ny, a.src.cx, a.src.cy, a.src.mi, a.src.mj, a.src.ratio);
        a.src_blocks = source_blocks(a.src.win);
    } else {
        a.src_blocks = 0;
    }
    const int blocks = a.njobs * a.nparts + a.src_blocks;
    note_launch();
    if (blocks == 0) {
        k_step_advance<<<1, 1, 0, st>>>(a.step);
        return;
    }
    // launched with a programmatic dependency on the preceding kernel (see k_step_tail)
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_step_tail<T>, a);
}
template void launch_step_tail<float>(TailArgs, cudaStream_t);
template void launch_step_tail<double>(TailArgs, cudaStream_t);

void launch_set_value(float *p, long long idx, float v, cudaStream_t st)
{
    note_launch();
    k_set_value<<<1, 1, 0, st>>>(p, idx, v);
}

// partials per overlap job: one 256-thread block per 256 window cells, 1 to 64
int overlap_parts(long long cells)
{
    const long long b = (cells + 255) / 256;
    return (int)(b < 1 ? 1 : b > 64 ? 64 : b);
}

template <typename T>
void launch_overlap(const T *const *f_dev, int nx, int ny, const OverlapJob *jobs_dev, int njobs, long long cells,
                    double2 *partials, double scale, double dt, const long long *step, int step_offset,
                    cudaStream_t st)
{
    if (njobs <= 0) return;
    const int parts = overlap_parts(cells);
    note_launch();
    k_overlap_partial<T><<<dim3(parts, njobs), 256, 0, st>>>(f_dev, nx, ny, jobs_dev, partials, parts);
    note_launch();
    k_overlap_finalize<<<njobs, 32, 0, st>>>(jobs_dev, njobs, partials, parts, scale, dt, step, step_offset);
}

template <typename T>
void launch_dft(const T *const *f_dev, int nx, int ny, int nz, int slice, int k_lo, int k_hi, double tr, double ti,
                double2 *acc, cudaStream_t st)
{
    if (k_hi <= k_lo) return;
    long long cnt = slice >= 0 ? (long long)nx * (k_hi - k_lo) : (long long)nx * ny * (k_hi - k_lo);
    int blocks = (int)((cnt + 255) / 256);
    if (blocks > 4736) blocks = 4736;
    note_launch();
    k_dft<T><<<blocks, 256, 0, st>>>(f_dev, nx, ny, nz, slice, k_lo, k_hi, tr, ti, acc);
}

template <typename T>
void launch_probes(const T *const *f_dev, const ProbeJob *probes, int np, double *buf, int cap, int *count,
                   cudaStream_t st)
{
    if (np <= 0) return;
    note_launch();
    k_probes<T><<<(np + 127) / 128, 128, 0, st>>>(f_dev, probes, np, buf, cap, count);
}

void launch_step_advance(long long *step, cudaStream_t st)
{
    note_launch();
    k_step_advance<<<1, 1, 0, st>>>(step);
}

template <typename T>
void launch_taper_store(const T *const *f_dev, const long long *cells, int ncell, T *store, int t_index,
                        const long long *step, int t0, int dir, int duration, cudaStream_t st)
{
    if (ncell <= 0) return;
    int blocks = (ncell + 255) / 256;
    if (blocks > 592) blocks = 592;
    note_launch();
    k_taper_store<T><<<blocks, 256, 0, st>>>(f_dev, cells, ncell, store, t_index, step, t0, dir, duration);
}

template <typename T>
void launch_ep_gradient(const T *fwd, const T *adj, int ncell, int duration, double *grad, cudaStream_t st)
{
    if (ncell <= 0) return;
    note_launch();
    k_ep_gradient<T><<<(ncell + 127) / 128, 128, 0, st>>>(fwd, adj, ncell, duration, grad);
}

void launch_check_finite(const float *a, long long n, int *bad, cudaStream_t st)
{
    int blocks = (int)((n + 255) / 256);
    if (blocks > 2368) blocks = 2368;
    if (blocks > 0) {
        note_launch();
        k_check_finite<<<blocks, 256, 0, st>>>(a, n, bad);
    }
}

#define FDTD_INST(T)                                                                                               \
    template void launch_overlap<T>(const T *const *, int, int, const OverlapJob *, int, long long, double2 *,     \
                                    double, double, const long long *, int, cudaStream_t);                         \
    template void launch_dft<T>(const T *const *, int, int, int, int, int, int, double, double, double2 *,         \
                                cudaStream_t);                                                                     \
    template void launch_probes<T>(const T *const *, const ProbeJob *, int, double *, int, int *, cudaStream_t);   \
    template void launch_taper_store<T>(const T *const *, const long long *, int, T *, int, const long long *, int, \
                                        int, int, cudaStream_t);                                                   \
    template void launch_ep_gradient<T>(const T *, const T *, int, int, double *, cudaStream_t);
FDTD_INST(float)
FDTD_INST(double)
#undef FDTD_INST

}  // namespace fdtd
