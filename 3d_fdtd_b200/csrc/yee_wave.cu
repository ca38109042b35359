// yee_wave.cu -- a run of S time steps of the FP32 flat update (E, H, CPML,
// source planes, mode-overlap monitors) in ONE persistent launch, ordered as
// a wavefront in z so that the planes in use stay in the 126 MB L2.
//
// The per-step path (yee_flat4.cu + k_step_tail) streams the whole grid from
// HBM twice per step: ~1.1 GB for the 200 x 160 x 400 CPML grid.  Here steps
// run in sweeps of SW steps; inside a sweep step ls+1 trails step ls by a few
// planes, so a sweep touches a window of about 4 SW planes at a time and each
// plane comes from HBM about once per sweep instead of once per step.
//
// Work items.  (step ls, field E|H, plane k) is one plane item of nb(k)
// blocks of work: the blocks of the per-field launch, with the same thread
// slots and per-cell code (flat4_cells.cuh), so the fields are bit-identical
// to the per-step path.  (step ls, plane z) of a monitor plane is one overlap
// item of parts(z) blocks, one overlap partial each, with the partition and
// reduction tree of the per-step kernels (plane_ops.cuh).  A ticket is up to
// `group` consecutive blocks of work of one item.  Dependencies, per plane, on
// counts of finished tickets (the updates are in place, so reads after writes
// and writes after reads coincide):
//   E(ls, k)        after H(ls-1, k), H(ls-1, k-1), overlaps(ls-1, k)
//   H(ls, k)        after E(ls, k), E(ls, k+1)
//   overlaps(ls, z) after H(ls, z)
// Items get the key
//   E: q P + k + 4 l,   H: q P + k + 4 l + 2,   overlaps: q P + z + 4 l + 3
// (sweep q = ls / SW, l = ls % SW, P = max(nz, 4 SW)); every dependency has a
// smaller key, so tickets numbered in key order are a topological order.
// Blocks take tickets in increasing order from a grid-wide counter and the
// launch is cooperative (all blocks resident), so the smallest unfinished
// ticket can always run: the launch always makes progress (k_wave).
//
// Synchronisation: a finished ticket is a block barrier then one
// `red.release.gpu` add on its item's counter; lane 0 of warp 0 polls the
// counters of the next ticket with relaxed loads and takes an acquire fence
// once they are complete, then the block barrier orders the other threads
// after it.  Field loads inside the launch are plain coherent loads (the
// read-only path is not coherent with writes of the same launch).  Every wait
// is bounded by %globaltimer: past the limit the block sets the grid's error
// flag, and once the flag is set no wait blocks any more, so the launch ends
// and the host reports a timeout.
//
// Around the launch: k_wave_ring writes the scheduled source plane of every
// step of the run into a ring (the plane's cells outside the mode keep the
// plane buffer's values, as the per-step path leaves them); k_wave_finalize
// adds each step's overlap partials in order and accumulates the monitors
// exactly as the per-step tail does, writes the next step's source into the
// plane buffer and advances the device step counter by S.
#include <algorithm>
#include <climits>
#include <vector>

#include "flat4_cells.cuh"
#include "plane_ops.cuh"

namespace fdtd {

constexpr int kWaveE = 0, kWaveH = 1, kWaveM = 2;

__host__ __device__ inline int wave_desc(int kind, int k, int ls) { return kind | (k << 2) | (ls << 17); }

__device__ __forceinline__ unsigned long long wave_clock()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_relaxed(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_relaxed_s(const int *p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release(unsigned *p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int wave_counter(const WaveArgs &w, int kind, int k, int ls)
{
    return kind == kWaveM ? 2 * w.steps * w.nz + ls * w.nz + k : (ls * 2 + kind) * w.nz + k;
}

// one thread: wait until every dependency of `it` is complete, bounded by
// w.wait_ns; then an acquire fence
__device__ void wave_wait(const WaveItem &it, const WaveArgs &w)
{
    unsigned long long t0 = 0;
    unsigned ns = 32;
    for (;;) {
        bool done = true;
#pragma unroll
        for (int d = 0; d < 3; d++)
            if (it.dep[d].x >= 0 && ld_relaxed(w.cnt + it.dep[d].x) < (unsigned)it.dep[d].y) done = false;
        if (done || ld_relaxed_s(w.err) != 0) break;
        const unsigned long long now = wave_clock();
        if (t0 == 0) {
            t0 = now;
        } else if (now - t0 > w.wait_ns) {
            atomicCAS(w.err, 0, 1);
            break;
        }
        __nanosleep(ns);
        if (ns < 128) ns <<= 1;
    }
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
}

// the cells of block lb of plane item (field, k): block lb of the per-field
// launch, laid out by the regions of flat4_plan
template <bool LOSSY>
__device__ __forceinline__ void wave_cells(const FlatArgs &a, const Plan4 &p, bool efield, int k, int lb, int ls)
{
    const int s = lb * kBlock4 + threadIdx.x;
    int g, j, kk;
    bool live;
    if (p.L == 0) {
        locate<0>(p.zs, a.nx / 4, a.ny, s, k - 1, g, j, kk, live);
        if (efield) e_cells<4, 0, LOSSY, true>(a, g, j, kk, live, ls);
        else h_cells<4, 0, true>(a, g, j, kk, live, ls);
    } else if (k < p.L || k >= a.nz - p.L) {
        const int by = k < p.L ? k - 1 : (p.L - 1) + (k - (a.nz - p.L));
        locate<0>(p.zs, a.nx / 2, a.ny, s, by, g, j, kk, live);
        if (efield) e_cells<2, 7, LOSSY, true>(a, g, j, kk, live, ls);
        else h_cells<2, 7, true>(a, g, j, kk, live, ls);
    } else if (lb < p.nb_box) {
        locate<1>(p.box, a.nx / 4, a.ny, s, k - p.L, g, j, kk, live);
        if (efield) e_cells<4, 0, LOSSY, true>(a, g, j, kk, live, ls);
        else h_cells<4, 0, true>(a, g, j, kk, live, ls);
    } else if (lb < p.nb_box + p.nb_y) {
        locate<3>(p.yrows, a.nx / 2, a.ny, s - p.nb_box * kBlock4, k - p.L, g, j, kk, live);
        if (efield) e_cells<2, 2, LOSSY, true>(a, g, j, kk, live, ls);
        else h_cells<2, 2, true>(a, g, j, kk, live, ls);
    } else {
        locate<4>(p.xcols, a.nx / 2, a.ny, s - (p.nb_box + p.nb_y) * kBlock4, k - p.L, g, j, kk, live);
        if (efield) e_cells<2, 3, LOSSY, true>(a, g, j, kk, live, ls);
        else h_cells<2, 3, true>(a, g, j, kk, live, ls);
    }
}

// block lb of the overlap item of plane z, step ls: partial (lb % nparts) of
// the (lb / nparts)-th monitor on plane z
__device__ __forceinline__ void wave_overlap(const FlatArgs &a, const WaveArgs &w, int z, int lb, int ls)
{
    int want = lb / w.nparts;
    const int part = lb - want * w.nparts;
    int jid = -1;
    for (int q = 0; q < w.njobs; q++) {
        if (w.jobs[q].cz != z) continue;
        if (want == 0) {
            jid = q;
            break;
        }
        want--;
    }
    if (jid < 0) return;
    const OverlapJob jb = w.jobs[jid];
    const float *fp[6] = {a.f[0], a.f[1], a.f[2], a.f[3], a.f[4], a.f[5]};
    overlap_block<float>(fp, a.nx, a.ny, jb, part, w.nparts,
                         w.partials + ((long long)ls * w.njobs + jid) * w.nparts + part);
}

// Blocks take tickets in increasing order from a grid-wide counter (lane 0 of
// warp 0 fetches the next one while the block works on the current one); a
// ticket is up to w.group consecutive blocks of work of one item, done one
// after another, so the ticket's decode, waits and release are paid once per
// group.  Progress: the smallest unfinished ticket is either some block's
// current ticket (its dependencies are smaller, hence finished) or some
// block's fetched next ticket, whose current ticket is smaller and therefore
// finished.
template <bool LOSSY>
__global__ void __launch_bounds__(kBlock4, 3) k_wave(FlatArgs a, Plan4 p, WaveArgs w)
{
    __shared__ int s_desc, s_u, s_n;
    const int tid = threadIdx.x, lane = tid & 31;
    int cursor = 0;  // warp 0: item of the block's previous ticket
    int t_next = 0;  // lane 0 of warp 0: the block's next ticket
    if (tid == 0) t_next = (int)atomicAdd(w.next, 1u);
    for (;;) {
        if (tid < 32) {
            const int t = __shfl_sync(0xffffffffu, t_next, 0);
            if (t >= w.tickets) {
                if (lane == 0) s_desc = -1;
            } else {
                if (lane == 0) t_next = (int)atomicAdd(w.next, 1u);
                // the item holding ticket t: the last item whose first ticket is <= t
                for (;;) {
                    const int i = cursor + lane;
                    const int t0 = i < w.nitems ? w.items[i].t0 : INT_MAX;
                    const unsigned le = __ballot_sync(0xffffffffu, t0 <= t);
                    if (le == 0xffffffffu) {
                        cursor += 32;
                        continue;
                    }
                    cursor += __popc(le) - 1;
                    break;
                }
                if (lane == 0) {
                    const WaveItem it = w.items[cursor];
                    wave_wait(it, w);
                    s_desc = it.desc;
                    s_u = t - it.t0;
                    s_n = it.nblocks;
                }
            }
        }
        __syncthreads();
        const int desc = s_desc, u = s_u, nblocks = s_n;
        if (desc < 0) break;
        const int kind = desc & 3, k = (desc >> 2) & 0x7fff, ls = desc >> 17;
        const int lb0 = u * w.group, lb1 = min(lb0 + w.group, nblocks);
        for (int lb = lb0; lb < lb1; lb++) {
            if (kind == kWaveM) {
                wave_overlap(a, w, k, lb, ls);
                __syncthreads();   // overlap_block's shared scratch
            } else {
                wave_cells<LOSSY>(a, p, kind == kWaveE, k, lb, ls);
            }
        }
        __syncthreads();
        // warp 1 signals, so its release fence overlaps warp 0's next decode
        if (tid == 32) red_release(w.cnt + wave_counter(w, kind, k, ls), 1u);
    }
}

// ring[ls] = the scheduled source plane of step (*step + ls): the mode's
// values where a cell has a sample, the plane buffer's elsewhere
__global__ void k_wave_ring(SourceJob sj, float *ring, long long stride, const long long *step)
{
    const int ls = blockIdx.y;
    const SrcStep sv = schedule_step(sj, *step + ls);
    const long long nxy = (long long)sj.nx * sj.ny;
    float *dst = ring + ls * stride;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nxy; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % sj.nx), j = (int)(t / sj.nx);
        float v[6];
        if (!mode_source_cell(sj, i, j, sv, v)) {
#pragma unroll
            for (int m = 0; m < 6; m++) v[m] = sj.plane[m * nxy + t];
        }
#pragma unroll
        for (int m = 0; m < 6; m++) dst[m * nxy + t] = v[m];
    }
}

// blocks 0..njobs-1: one monitor each.  Per chunk of 32 steps, the step
// totals (partials added in order, scaled) in parallel, then the terms
// e^{i omega_f n dt} o(n) of every (step, frequency) in parallel, then per
// frequency the Kahan additions in step order, the sums kept in registers
// (the per-step tail's arithmetic and order).  Blocks njobs..: the scheduled
// source of step n0 + S into the plane buffer.  The last block to finish
// advances the step counter.
__global__ void __launch_bounds__(256) k_wave_finalize(WaveFinal f)
{
    constexpr int CH = 32;   // steps per chunk, frequencies per pass
    const long long n0 = *f.step;
    const int tid = threadIdx.x;
    if ((int)blockIdx.x < f.njobs) {
        __shared__ double2 tot[CH];
        __shared__ double2 term[CH][CH];
        const OverlapJob jb = f.jobs[blockIdx.x];
        const double2 *pj = f.partials + (long long)blockIdx.x * f.nparts;
        const long long pstride = (long long)f.njobs * f.nparts;   // one step further
        for (int fb = 0; fb == 0 || (jb.acc && fb < jb.nfreq); fb += CH) {
            const int fq = fb + tid;
            const bool mine = tid < CH && jb.acc && fq < jb.nfreq;
            double2 sum = make_double2(0.0, 0.0), comp = sum;
            if (mine) {
                sum = jb.acc[2 * fq];
                comp = jb.acc[2 * fq + 1];
            }
            for (int c0 = 0; c0 < f.steps; c0 += CH) {
                const int nl = min(CH, f.steps - c0);
                if (tid < nl) {
                    const double2 *pp = pj + (long long)(c0 + tid) * pstride;
                    double sre = 0.0, sim = 0.0;
                    for (int q = 0; q < f.nparts; q++) {
                        const double2 v = pp[q];
                        sre = dadd(sre, v.x);
                        sim = dadd(sim, v.y);
                    }
                    tot[tid] = make_double2(dmul(f.scale, sre), dmul(f.scale, sim));
                }
                __syncthreads();
                if (jb.acc)
                    for (int q = tid; q < CH * CH; q += blockDim.x) {
                        const int l = q / CH, fi = q % CH;
                        if (l < nl && fb + fi < jb.nfreq) term[l][fi] = frequency_term(jb, fb + fi, tot[l], f.dt, n0 + c0 + l);
                    }
                __syncthreads();
                if (mine)
                    for (int l = 0; l < nl; l++) kahan_add(sum, comp, term[l][tid]);
                if (tid == 0 && fb == 0 && jb.inst && c0 + nl == f.steps) *jb.inst = tot[nl - 1];
                __syncthreads();
            }
            if (mine) {
                jb.acc[2 * fq] = sum;
                jb.acc[2 * fq + 1] = comp;
            }
        }
    } else if (f.src.plane) {
        const SrcStep sv = schedule_step(f.src, n0 + f.steps);
        mode_source_cells(f.src, (blockIdx.x - f.njobs) * (long long)blockDim.x + tid,
                          (long long)(gridDim.x - f.njobs) * blockDim.x, sv);
    }
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(f.done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last && tid == 0) {
        *f.step = n0 + f.steps;
        *f.done = 0u;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int wave_items(const Plan4 &p, int nz, int steps, int sweep, int group, const int *job_z, int njobs, int nparts,
               std::vector<WaveItem> &out, int &tickets)
{
    out.clear();
    tickets = 0;
    if (nz < 3 || steps < 1 || sweep < 1 || group < 1 || steps >= (1 << 14) || nz >= (1 << 15)) return -1;
    const int P = std::max(nz, 4 * sweep);
    // blocks of work of a plane item: the blocks of the per-field launch
    auto nb = [&](int k) { return p.L == 0 ? p.nbz : (k < p.L || k >= nz - p.L ? p.nbz : p.nbm); };
    std::vector<int> parts(nz, 0);
    for (int q = 0; q < njobs; q++) {
        if (job_z[q] < 1 || job_z[q] > nz - 2) return -1;
        parts[job_z[q]] += nparts;
    }
    struct Entry {
        long long key;
        int ls, kind, k;
    };
    std::vector<Entry> e;
    e.reserve((size_t)steps * (nz - 2) * 2);
    for (int ls = 0; ls < steps; ls++) {
        const long long base = (long long)(ls / sweep) * P + 4LL * (ls % sweep);
        for (int k = 1; k <= nz - 2; k++) {
            e.push_back({base + k, ls, kWaveE, k});
            e.push_back({base + k + 2, ls, kWaveH, k});
            if (parts[k]) e.push_back({base + k + 3, ls, kWaveM, k});
        }
    }
    std::sort(e.begin(), e.end(), [](const Entry &x, const Entry &y) {
        if (x.key != y.key) return x.key < y.key;
        if (x.ls != y.ls) return x.ls < y.ls;
        return x.kind < y.kind;
    });
    // tickets of an item of `blocks` blocks of work
    auto tk = [&](int blocks) { return (blocks + group - 1) / group; };
    auto counter = [&](int kind, int k, int ls) {
        return kind == kWaveM ? 2 * steps * nz + ls * nz + k : (ls * 2 + kind) * nz + k;
    };
    long long t = 0;
    out.reserve(e.size());
    for (const Entry &x : e) {
        WaveItem it{};
        it.t0 = (int)t;
        it.desc = wave_desc(x.kind, x.k, x.ls);
        for (int d = 0; d < 3; d++) it.dep[d] = make_int2(-1, 0);
        int nd = 0;
        if (x.kind == kWaveE) {
            if (x.ls > 0) {
                it.dep[nd++] = make_int2(counter(kWaveH, x.k, x.ls - 1), tk(nb(x.k)));
                if (x.k - 1 >= 1) it.dep[nd++] = make_int2(counter(kWaveH, x.k - 1, x.ls - 1), tk(nb(x.k - 1)));
                if (parts[x.k]) it.dep[nd++] = make_int2(counter(kWaveM, x.k, x.ls - 1), tk(parts[x.k]));
            }
        } else if (x.kind == kWaveH) {
            it.dep[nd++] = make_int2(counter(kWaveE, x.k, x.ls), tk(nb(x.k)));
            if (x.k + 1 <= nz - 2) it.dep[nd++] = make_int2(counter(kWaveE, x.k + 1, x.ls), tk(nb(x.k + 1)));
        } else {
            it.dep[nd++] = make_int2(counter(kWaveH, x.k, x.ls), tk(nb(x.k)));
        }
        it.nblocks = x.kind == kWaveM ? parts[x.k] : nb(x.k);
        out.push_back(it);
        t += tk(it.nblocks);
        if (t > INT_MAX / 2) return -1;
    }
    tickets = (int)t;
    return 0;
}

int wave_counters(int nz, int steps) { return 3 * steps * nz; }

int wave_grid(bool lossy)
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    const cudaError_t e = lossy ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wave<true>, kBlock4, 0)
                                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wave<false>, kBlock4, 0);
    if (e != cudaSuccess) return 0;
    return sms * per_sm;
}

cudaError_t launch_wave(const FlatArgs &a, const Plan4 &p, const WaveArgs &w, int grid, const SourceJob *sched,
                        float *ring, const WaveFinal &fin, cudaStream_t st)
{
    const long long nxy = (long long)a.nx * a.ny;
    // the counters and, after them, the ticket counter
    cudaError_t e = cudaMemsetAsync(w.cnt, 0, ((size_t)wave_counters(a.nz, w.steps) + 1) * sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    if (sched) {
        note_launch();
        const int bx = (int)std::min<long long>((nxy + 255) / 256, 256);
        k_wave_ring<<<dim3(bx, w.steps), 256, 0, st>>>(*sched, ring, 6 * nxy, fin.step);
    }
    FlatArgs aw = a;
    if (sched) {
        aw.ring = ring;
        aw.ring_stride = 6 * nxy;
    } else {
        aw.ring = nullptr;
    }
    Plan4 pp = p;
    WaveArgs ww = w;
    void *args[] = {&aw, &pp, &ww};
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kBlock4);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    note_launch();
    e = a.ca[0] ? cudaLaunchKernelExC(&cfg, (const void *)k_wave<true>, args)
                : cudaLaunchKernelExC(&cfg, (const void *)k_wave<false>, args);
    if (e != cudaSuccess) return e;
    WaveFinal ff = fin;
    int fin_blocks = ff.njobs;
    if (ff.src.plane) {
        ff.src.win = mode_window(ff.src.nx, ff.src.ny, ff.src.cx, ff.src.cy, ff.src.mi, ff.src.mj, ff.src.ratio);
        const long long cells = (long long)ff.src.win.wni * ff.src.win.wnj;
        fin_blocks += (int)std::min<long long>(std::max<long long>(1, (cells + 255) / 256), 1184);
    }
    fin_blocks = std::max(fin_blocks, 1);   // one block at least, to advance the counter
    note_launch();
    k_wave_finalize<<<fin_blocks, 256, 0, st>>>(ff);
    return cudaGetLastError();
}

}  // namespace fdtd

// ---------------------------------------------------------------------------
// schedule inspection (host only; no device work)
// ---------------------------------------------------------------------------
extern "C" int fdtd_wave_schedule(int nx, int ny, int nz, int cpml_cells, int steps, int sweep, int group,
                                  const int *job_z, int njobs, int nparts, int *out, int cap, int *tickets)
{
    using namespace fdtd;
    if (nx < 8 || nx % 4 != 0 || ny < 3 || nz < 3 || cpml_cells < 0 || njobs < 0 || nparts < 1 || !tickets ||
        (njobs > 0 && !job_z))
        return -1;
    FlatArgs a{};
    a.nx = nx; a.ny = ny; a.nz = nz; a.L = cpml_cells;
    if (a.L > 0 && !flat4_split_supported(a)) return -1;
    const Plan4 p = flat4_plan(a);
    std::vector<WaveItem> items;
    int t = 0;
    if (wave_items(p, nz, steps, sweep, group, job_z, njobs, nparts, items, t) != 0) return -1;
    *tickets = t;
    if (out) {
        if (cap < (int)items.size()) return -1;
        for (size_t i = 0; i < items.size(); i++) {
            int *o = out + 9 * i;
            o[0] = items[i].t0;
            o[1] = items[i].desc;
            o[2] = items[i].nblocks;
            for (int d = 0; d < 3; d++) {
                o[3 + 2 * d] = items[i].dep[d].x;
                o[4 + 2 * d] = items[i].dep[d].y;
            }
        }
    }
    return (int)items.size();
}
