// yee_sweep.cu -- many grids (taper candidates of uneven length) advanced
// together by one persistent launch per chunk of steps.
//
// The reference simulates one design at a time (3d_fdtd.c:93-202).  An
// optimisation sweep runs many independent candidates; here every resident
// candidate advances inside ONE cooperative launch of S steps (one block per
// SM, all co-resident), each candidate for at most its own remaining steps.
// Per step, three phases separated by grid barriers where needed:
//   A  the one-pass FP32 Yee update (yee_stream.cu) of every candidate still
//      running: all candidates' (band, chunk) tiles in one list ordered by
//      estimated cost, longest first, each block taking the next tile from a
//      per-step counter when it finishes one (tiles of candidates of every
//      length, so dealing them out statically left the blocks' phase times
//      up to 2x apart);
//   -- barrier --
//   B  each candidate's step tail: the overlap partials of its monitors (one
//      warp per partial, the same partial as the per-step tail's 256-thread
//      block) and its scheduled source plane for the next step;
//   -- barrier --
//   C  the monitors of the step: partials added in order, accumulated per
//      frequency with Kahan compensation at step base + s (one warp per
//      monitor).  Partials are double-buffered by step parity, so phase C of
//      step s runs beside phase A of step s+1 without a barrier between them.
// Every candidate's fields, auxiliaries and monitors are those of the same
// candidate run alone with FDTD_YEE_STREAM, bit for bit: the tile split does
// not change any cell's arithmetic and the reductions keep their order.
//
// Memory: loads of data written inside the launch (fields through the
// L2-only cp.async path, CPML auxiliaries, source planes, partials) are
// coherent; every grid barrier is arrival (release) then a bounded poll
// (acquire).  A barrier that waits longer than its limit sets the sweep's
// error flag; the flag stops every later wait, the launch ends, and the grids
// report FDTD_ERR_TIMEOUT at their next synchronising call.
#include "stream_cells.cuh"
#include "plane_ops.cuh"
#include "engine.h"

#include <algorithm>

#define CK_RET(call)                               \
    do {                                           \
        if (!cuda_ok((call), #call)) return false; \
    } while (0)

namespace fdtd {

__device__ __forceinline__ unsigned long long sweep_clock()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_relaxed_i32(const int *p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// grid barrier number k (1, 2, ...): every block arrives once; true when all
// a.arrivals arrived, false when the wait gave up (or another block's did)
__device__ bool sweep_barrier(const SweepArgs &a, unsigned k, int *abort_s)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        int ab = 0;
        __threadfence();
        atomicAdd(a.bar, 1u);
        const unsigned target = k * a.arrivals;
        unsigned long long t0 = 0;
        unsigned ns = 32;
        for (;;) {
            if (ld_acquire_u32(a.bar) >= target) break;
            if (ld_relaxed_i32(a.err) != 0) {
                ab = 1;
                break;
            }
            const unsigned long long now = sweep_clock();
            if (t0 == 0) {
                t0 = now;
            } else if (now - t0 > a.wait_ns) {
                atomicCAS(a.err, 0, 1);
                ab = 1;
                break;
            }
            __nanosleep(ns);
            if (ns < 256) ns <<= 1;
        }
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        *abort_s = ab;
    }
    __syncthreads();
    return *abort_s == 0;
}

// The tile arguments of every grid of a sweep (grid g, input set p at 2g + p)
// in constant memory, as a kernel's parameters are for the per-step launch:
// read from a global-memory copy the tile held its dozens of pointers in
// registers and spilled, and its planes took twice as long.
__constant__ StreamArgs c_sweep_args[2 * kSweepMaxGrids];
static_assert(sizeof(c_sweep_args) <= 60 * 1024, "sweep tile arguments must fit constant memory");

// One tile, out of line, so that the persistent loop's state and the phase
// B/C code do not share the tile's registers.
template <bool CPML, bool LOSSY, int TPC>
__device__ __forceinline__ void sweep_tile(int idx, int t, float *sm)
{
    const StreamArgs &sa = c_sweep_args[idx];
    stream_tile<CPML, LOSSY, true, TPC>(sa, sa.tiles[t], sm);
}

// TPC: the staged rows of every grid's tiles when they agree and are one of
// 5..8 (what the plan gives grids 128 cells wide or more), else 0 (run time)
template <bool CPML, bool LOSSY, int TPC>
__global__ void __launch_bounds__(kStreamMaxThreads, 1) k_sweep(SweepArgs a)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ int abort_s, item_s;
    const int G = gridDim.x, warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gw = blockIdx.x * warps + warp, nw = G * warps;
    unsigned nbar = 0;
    for (int s = 0; s < a.steps; s++) {
        // ---- A: Yee tiles of the running grids, handed out one at a time
        //      from a list ordered by cost (longest first), so the blocks
        //      finish the step together whatever the grids' lengths
        for (;;) {
            __syncthreads();   // the block's previous tile no longer reads shared memory; item_s is free
            if (threadIdx.x == 0) item_s = (int)atomicAdd(a.next + s, 1u);
            __syncthreads();
            const int idx = item_s;
            if (idx >= a.nitems) break;
            const int2 it = a.items[idx];
            const SweepGrid &sg = a.grids[it.x];
            if (s >= sg.steps) continue;
            sweep_tile<CPML, LOSSY, TPC>(2 * it.x + ((sg.p0 + s) & 1), it.y, sm);
        }
        if (!sweep_barrier(a, ++nbar, &abort_s)) return;
        // ---- B: overlap partials of step s, scheduled source of step s+1
        int w = 0;
        for (int g = 0; g < a.ngrids; g++) {
            const SweepGrid &sg = a.grids[g];
            if (s >= sg.steps) continue;
            const int nov = sg.njobs * sg.nparts;
            const float *const *f = sg.fout[(sg.p0 + s) & 1];
            for (int i = (gw - w % nw + nw) % nw; i < nov; i += nw) {
                const int jid = i / sg.nparts, part = i - jid * sg.nparts;
                overlap_warp<float>(f, sg.nx, sg.ny, sg.jobs[jid], part, sg.nparts,
                                    sg.partials + (size_t)(s & 1) * nov + i);
            }
            w += nov;
            if (sg.src.plane) {
                const SrcStep v = schedule_step(sg.src, sg.base + s + 1);
                for (int i = (gw - w % nw + nw) % nw; i < sg.src_warps; i += nw)
                    mode_source_cells(sg.src, (long long)i * 32 + lane, (long long)sg.src_warps * 32, v);
                w += sg.src_warps;
            }
        }
        if (!sweep_barrier(a, ++nbar, &abort_s)) return;
        // ---- C: the monitors of step s (no barrier after: the partials of the
        //      next step go to the other buffer)
        w = 0;
        for (int g = 0; g < a.ngrids; g++) {
            const SweepGrid &sg = a.grids[g];
            if (s >= sg.steps) continue;
            const int nov = sg.njobs * sg.nparts;
            for (int jid = (gw - w % nw + nw) % nw; jid < sg.njobs; jid += nw) {
                const double2 *pp = sg.partials + (size_t)(s & 1) * nov + (size_t)jid * sg.nparts;
                double sre = 0.0, sim = 0.0;
                for (int p = 0; p < sg.nparts; p++) {
                    const double2 v = pp[p];
                    sre = dadd(sre, v.x);
                    sim = dadd(sim, v.y);
                }
                const double2 tot = make_double2(dmul(sg.scale, sre), dmul(sg.scale, sim));
                const OverlapJob jb = sg.jobs[jid];
                if (jb.inst && lane == 0) *jb.inst = tot;
                if (jb.acc)
                    for (int f = lane; f < jb.nfreq; f += 32) accumulate_frequency(jb, f, tot, sg.dt, sg.base + s);
            }
            w += sg.njobs;
        }
    }
    // device step counters: the block that owns each grid's last monitor work
    // is irrelevant here; block 0 writes them once every phase C is issued
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (int g = 0; g < a.ngrids; g++) *a.grids[g].step = a.grids[g].base + a.grids[g].steps;
}

// a timed-out sweep marks every grid it ran (their next synchronising call
// reports FDTD_ERR_TIMEOUT)
__global__ void k_sweep_err_to_grid(const int *sweep, int *grid)
{
    if (*sweep) *grid = 1;
}

void launch_sweep_err_to_grid(const int *sweep, int *grid, cudaStream_t st)
{
    note_launch(1);
    k_sweep_err_to_grid<<<1, 1, 0, st>>>(sweep, grid);
}

// A barrier that nothing completes (arrivals one more than the grid): every
// block's wait gives up after the limit and the flag is set.
__global__ void k_sweep_barrier_selftest(SweepArgs a)
{
    __shared__ int abort_s;
    sweep_barrier(a, 1, &abort_s);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

struct SweepContext {
    cudaStream_t st = nullptr;
    int dev = -1, nsm = 0;
    unsigned *d_bar = nullptr;
    unsigned *d_next = nullptr;   // per step of a launch, the next tile item (kSweepMaxSteps)
    int2 *d_items = nullptr;
    size_t items_cap = 0;
    int *d_err = nullptr;
    SweepGrid *d_grids = nullptr;
    size_t grids_cap = 0;
    StreamTile *d_tiles = nullptr;
    size_t tiles_cap = 0;
    double2 *d_partials = nullptr;
    size_t partials_cap = 0;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev = nullptr;
};

SweepContext &ctx()
{
    static SweepContext c;
    return c;
}

template <typename P> bool grow(P **p, size_t &cap, size_t need)
{
    if (*p && cap >= need) return true;
    if (*p) cudaFree(*p);
    *p = nullptr;
    cap = 0;
    if (!cuda_ok(cudaMalloc((void **)p, need ? need : 16), "cudaMalloc(sweep)")) return false;
    cap = need;
    return true;
}

}  // namespace

using SweepKernel = void (*)(SweepArgs);

template <bool CPML, bool LOSSY> static SweepKernel sweep_kernel(int tp)
{
    switch (tp) {
    case 5: return k_sweep<CPML, LOSSY, 5>;
    case 6: return k_sweep<CPML, LOSSY, 6>;
    case 7: return k_sweep<CPML, LOSSY, 7>;
    case 8: return k_sweep<CPML, LOSSY, 8>;
    default: return k_sweep<CPML, LOSSY, 0>;
    }
}

static SweepKernel sweep_kernel(bool cpml, bool lossy, int tp)
{
    if (cpml) return lossy ? sweep_kernel<true, true>(tp) : sweep_kernel<true, false>(tp);
    return lossy ? sweep_kernel<false, true>(tp) : sweep_kernel<false, false>(tp);
}

bool sweep_setup(int *nsm_out)
{
    SweepContext &c = ctx();
    int dev = 0;
    CK_RET(cudaGetDevice(&dev));
    if (c.dev != dev) {
        if (c.st) cudaStreamDestroy(c.st);
        c = SweepContext{};
        c.dev = dev;
        CK_RET(cudaDeviceGetAttribute(&c.nsm, cudaDevAttrMultiProcessorCount, dev));
        CK_RET(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
        CK_RET(cudaEventCreateWithFlags(&c.ev, cudaEventDisableTiming));
        CK_RET(cudaMalloc(&c.d_bar, sizeof(unsigned)));
        CK_RET(cudaMalloc(&c.d_next, 4096 * sizeof(unsigned)));   // steps_per_launch <= 4096
        CK_RET(cudaMalloc(&c.d_err, sizeof(int)));
        CK_RET(cudaMemset(c.d_err, 0, sizeof(int)));
    }
    *nsm_out = c.nsm;
    return true;
}

// Runs the launches described by `launches` (each a list of SweepGrid, one per
// grid) on the sweep stream as one captured graph.  Tile tables and partial
// buffers are the caller's (already uploaded to `tiles`/`partials`).
bool sweep_launch(const std::vector<std::vector<SweepGrid>> &launches, const std::vector<int> &steps,
                  const std::vector<int2> &items, bool cpml, bool lossy, int tpc, int threads, size_t smem,
                  unsigned long long wait_ns)
{
    SweepContext &c = ctx();
    const int ng = launches.empty() ? 0 : (int)launches[0].size();
    const size_t per = (size_t)ng;
    std::vector<SweepGrid> flat;
    for (auto &l : launches) flat.insert(flat.end(), l.begin(), l.end());
    if (ng > kSweepMaxGrids) {
        set_error(FDTD_ERR_ARG, "sweep: more than %d grids", kSweepMaxGrids);
        return false;
    }
    CK_RET(cudaStreamSynchronize(c.st));   // no sweep of this context reads the constant arguments now
    {
        std::vector<StreamArgs> args;
        for (int g = 0; g < ng; g++)
            for (int p = 0; p < 2; p++) args.push_back(launches[0][g].args[p]);
        if (!args.empty())
            CK_RET(cudaMemcpyToSymbolAsync(c_sweep_args, args.data(), args.size() * sizeof(StreamArgs), 0,
                                           cudaMemcpyHostToDevice, c.st));
        CK_RET(cudaStreamSynchronize(c.st));
    }
    CK_RET(cudaMemsetAsync(c.d_err, 0, sizeof(int), c.st));
    if (c.exec) {
        cudaGraphExecDestroy(c.exec);
        c.exec = nullptr;
    }
    if (!grow(&c.d_grids, c.grids_cap, flat.size() * sizeof(SweepGrid))) return false;
    CK_RET(cudaMemcpyAsync(c.d_grids, flat.data(), flat.size() * sizeof(SweepGrid), cudaMemcpyHostToDevice, c.st));
    if (!grow(&c.d_items, c.items_cap, std::max<size_t>(items.size(), 1) * sizeof(int2))) return false;
    if (!items.empty())
        CK_RET(cudaMemcpyAsync(c.d_items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice, c.st));
    const SweepKernel kern = sweep_kernel(cpml, lossy, tpc);
    const void *fn = (const void *)kern;
    CK_RET(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CK_RET(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
    if (per_sm < 1) {
        set_error(FDTD_ERR_CUDA, "sweep: a block of %d threads with %zu bytes of shared memory cannot be resident",
                  threads, smem);
        return false;
    }
    cudaGraph_t gr;
    CK_RET(cudaStreamBeginCapture(c.st, cudaStreamCaptureModeThreadLocal));
    bool ok = true;
    for (size_t l = 0; l < launches.size() && ok; l++) {
        SweepArgs a{};
        a.grids = c.d_grids + l * per;
        a.ngrids = ng;
        a.steps = steps[l];
        a.items = c.d_items;
        a.nitems = (int)items.size();
        a.next = c.d_next;
        a.bar = c.d_bar;
        a.err = c.d_err;
        a.wait_ns = wait_ns;
        a.arrivals = (unsigned)c.nsm;
        ok = cudaMemsetAsync(c.d_bar, 0, sizeof(unsigned), c.st) == cudaSuccess &&
             cudaMemsetAsync(c.d_next, 0, (size_t)std::max(1, steps[l]) * sizeof(unsigned), c.st) == cudaSuccess;
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)c.nsm);
        cfg.blockDim = dim3((unsigned)threads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = c.st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        note_launch(1);
        if (ok) {
            ok = cudaLaunchKernelEx(&cfg, kern, a) == cudaSuccess;
        }
    }
    cudaError_t ce = cudaStreamEndCapture(c.st, &gr);
    if (!ok) {
        if (ce == cudaSuccess) cudaGraphDestroy(gr);
        return cuda_ok(cudaGetLastError(), "sweep capture") && false;
    }
    CK_RET(ce);
    cudaError_t ie = cudaGraphInstantiate(&c.exec, gr, 0);
    cudaGraphDestroy(gr);
    CK_RET(ie);
    CK_RET(cudaGraphLaunch(c.exec, c.st));
    return true;
}

cudaStream_t sweep_stream() { return ctx().st; }
cudaEvent_t sweep_event() { return ctx().ev; }
int *sweep_err() { return ctx().d_err; }
StreamTile **sweep_tiles(size_t need)
{
    SweepContext &c = ctx();
    if (!grow(&c.d_tiles, c.tiles_cap, need)) return nullptr;
    return &c.d_tiles;
}
double2 **sweep_partials(size_t need)
{
    SweepContext &c = ctx();
    if (!grow(&c.d_partials, c.partials_cap, need)) return nullptr;
    return &c.d_partials;
}

bool sweep_barrier_selftest(unsigned long long limit_ns, int *timed_out)
{
    int nsm = 0;
    if (!sweep_setup(&nsm)) return false;
    SweepContext &c = ctx();
    CK_RET(cudaMemsetAsync(c.d_bar, 0, sizeof(unsigned), c.st));
    int *d_err = nullptr;
    CK_RET(cudaMalloc(&d_err, sizeof(int)));
    CK_RET(cudaMemsetAsync(d_err, 0, sizeof(int), c.st));
    SweepArgs a{};
    a.bar = c.d_bar;
    a.err = d_err;
    a.wait_ns = limit_ns;
    a.arrivals = 2;   // one block, two arrivals expected: never complete
    note_launch(1);
    k_sweep_barrier_selftest<<<1, 32, 0, c.st>>>(a);
    bool ok = cuda_ok(cudaGetLastError(), "sweep barrier self-test") &&
              cuda_ok(cudaMemcpyAsync(timed_out, d_err, sizeof(int), cudaMemcpyDeviceToHost, c.st), "D2H") &&
              cuda_ok(cudaStreamSynchronize(c.st), "sync");
    cudaFree(d_err);
    return ok;
}

}  // namespace fdtd
