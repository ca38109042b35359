// yee_stream.cu -- FP32 Yee step in one pass: E^{n+1} and H^{n+3/2} of every
// cell in a single launch, streaming z-planes through shared memory.
//
// Why one pass.  Updating E and H in two launches reads each field set twice
// per step (the E launch reads H, the H launch reads the new E), about 84 B per
// cell against the 60 B algorithmic minimum (6 components read and written
// once, 3 E coefficients read).  Here a block keeps the new E of the plane it
// just computed on chip and updates H of the plane below from it, so every
// value crosses HBM once per step.
//
// Tiles.  The interior rows 1..ny-2 are cut into bands of at most `ty` rows
// and the interior planes 1..nz-2 into chunks; one block owns one (band, chunk)
// tile, all tiles are resident at once (one block per SM) and advance through
// z in lockstep, so the rows a band reads from its neighbours were fetched
// from HBM by the neighbour a moment earlier and are still in L2.  Bands are
// cut at the y-slab edges; each band gets chunks of planes by a cost model of
// a plane's pass fitted to per-tile times (stream_plan).
//
// Data flow.  Fields and CPML auxiliaries ping-pong between two sets (read
// `in`, write `out`), so no block reads a value another block has already
// replaced.  A band of R rows j0..j0+R-1 runs R+1 rows of threads: row R (the
// halo row j0+R, owned by the next band) only recomputes its new E, which the
// H update of row j0+R-1 needs.  Iteration it of a tile [k0, k1) handles plane
// k = k0 + it:
//   E_new(k)   for rows j0..j0+R (stored for owned rows and planes < k1)
//   H_new(k-1) for rows j0..j0+R-1 (it >= 1)
// so it runs k1 - k0 + 1 iterations, the last one computing E_new(k1) only for
// the H update of plane k1-1.  Cells on the outer shell (index 0 or N-1 on any
// axis) are never updated, as in the reference's interior-only update
// (timefield3d.c:1679-1837); both sets hold the same shell values, and a
// recomputed row or plane on the shell passes its E through unchanged.
//
// Pipeline.  Interior threads own 4 consecutive x cells (a quad) of one row;
// on a CPML grid every cell of the row-end quads that reach into an x slab has
// a thread of its own (stream_cells.cuh, StreamRoles).  Quads move with
// 16-byte cp.async copies into a ring of 3 shared-memory stages: right after
// the plane's barrier each thread reads its own slots of plane k-1's stage
// (old H, the H update's x-slab auxiliaries) into registers and issues plane
// k+2 into that stage, so planes k+1 and k+2 are in flight while plane k
// computes.  A thread copies only slots that it (or, for an x-slab quad, a
// lane of its warp, after a warp barrier) reads.  One block barrier per
// plane: the new E of a plane goes to a double-buffered shared array read by
// the next iteration's H update (own cells, neighbour rows and columns).
// Threads of row 0 also stage Hx, Hz of row j0-1 (the E update's j-1
// neighbours); x neighbours come from the same shared rows.  x-slab CPML
// auxiliaries are staged with the plane; y- and z-slab ones and source planes
// are read from global memory where a cell needs them, and the slab cells'
// 1-D profiles sit in a shared table.  Cell indices are 32-bit (grids below
// 2^31 cells).
//
// Arithmetic: exactly the per-cell expressions of the flat kernels
// (flat4_cells.cuh: same curl differences, same CPML recursion in
// cpml_curl, same coefficient forms), so results match them to the bit as
// long as the compiler contracts the same products.
#include "stream_cells.cuh"

namespace fdtd {

// TPC: staged rows a block's tile has (a.ty + 1), as a constant for 2..8,
// 0 when only known at run time
template <bool CPML, bool LOSSY, int TPC>
__global__ void __launch_bounds__(kStreamMaxThreads, 1) k_yee_stream(StreamArgs a)
{
    // programmatic dependent launch, as the flat kernels (see k_flat4_merged)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    extern __shared__ __align__(16) float sm[];
    stream_tile<CPML, LOSSY, false, TPC>(a, a.tiles[blockIdx.x], sm);
}

using StreamKernel = void (*)(StreamArgs);

template <bool CPML, bool LOSSY> static StreamKernel stream_kernel(int tp)
{
    switch (tp) {
    case 2: return k_yee_stream<CPML, LOSSY, 2>;
    case 3: return k_yee_stream<CPML, LOSSY, 3>;
    case 4: return k_yee_stream<CPML, LOSSY, 4>;
    case 5: return k_yee_stream<CPML, LOSSY, 5>;
    case 6: return k_yee_stream<CPML, LOSSY, 6>;
    case 7: return k_yee_stream<CPML, LOSSY, 7>;
    case 8: return k_yee_stream<CPML, LOSSY, 8>;
    default: return k_yee_stream<CPML, LOSSY, 0>;
    }
}

static StreamKernel stream_kernel(bool cpml, bool lossy, int tp)
{
    if (cpml) return lossy ? stream_kernel<true, true>(tp) : stream_kernel<true, false>(tp);
    return lossy ? stream_kernel<false, true>(tp) : stream_kernel<false, false>(tp);
}

// ---------------------------------------------------------------------------
// host side: the tile plan
// ---------------------------------------------------------------------------
static size_t stream_smem_floats(int nx, int ty, bool lossy, int L)
{
    const int NA = lossy ? 12 : 9;
    return ((size_t)kStreamStages * NA * (ty + 1) + 2 * kStreamStages + 6 * (size_t)(ty + 1)) * nx +
           (size_t)kStreamStages * 4 * (ty + 1) * stream_xpsi_stride(L) + (L > 0 ? 36 * (size_t)L : 0);
}

// split items 0..n-1 of cost c[] into at most `parts` contiguous runs of at
// most `maxlen` items each, a run starting at every item t with brk[t] set
// (brk may be empty), minimising the largest run cost (binary search on that
// cost); returns the run starts (size = runs actually used) or empty
static std::vector<int> split_runs(const std::vector<double> &c, int parts, int maxlen,
                                   const std::vector<char> &brk = {})
{
    const int n = (int)c.size();
    auto greedy = [&](double cap, std::vector<int> *starts) {
        int runs = 0, len = 0;
        double acc = 0;
        for (int t = 0; t < n; t++) {
            if (len == 0 || acc + c[t] > cap || len >= maxlen || (!brk.empty() && brk[t])) {
                if (len > 0 || runs == 0) {
                    runs++;
                    if (starts) starts->push_back(t);
                }
                acc = 0;
                len = 0;
            }
            acc += c[t];
            len++;
        }
        return runs;
    };
    double lo = 0, hi = 0;
    for (double x : c) { lo = std::max(lo, x); hi += x; }
    if (greedy(hi, nullptr) > parts) return {};   // maxlen alone needs more runs
    for (int iter = 0; iter < 60; iter++) {
        const double mid = 0.5 * (lo + hi);
        if (greedy(mid, nullptr) <= parts) hi = mid; else lo = mid;
    }
    std::vector<int> starts;
    greedy(hi, &starts);
    return starts;
}

int stream_supported(int nx, int ny, int nz, bool lossy, int L)
{
    if (nx % 4 != 0 || nx < 8 || ny < 3 || nz < 3 || L < 0) return 0;
    if ((long long)nx * ny * nz >= (1LL << 31)) return 0;   // cell indices are 32-bit (sidx_t)
    if (stream_roles(nx, L, 2).threads > kStreamMaxThreads) return 0;   // at least one row plus its halo row
    return stream_smem_floats(nx, 1, lossy, L) * sizeof(float) <= kStreamSmemBudget;
}

// Time of a band's pass over one plane (us; only ratios matter): rows
// [j0, j0 + rows) with its halo row j0 + rows.  See stream_plan.
static double band_plane_cost(int nx, int ny, int L, int j0, int rows)
{
    const double sx = nx / 200.0;
    const int jh = j0 + rows;
    const bool yb = L > 0 && (j0 < L || jh - 1 >= ny - L);
    double c = yb ? 1.88 + 0.32 * sx * rows : 0.90 + 0.22 * sx * rows;
    if (!yb && L > 0 && jh >= ny - L && jh < ny - 1) c += 0.8;
    return c;
}

static double plane_weight(int nz, int L, int k) { return L > 0 && (k < L || k >= nz - L) ? 1.67 : 1.0; }

double stream_tile_cost(int nx, int ny, int nz, int L, const StreamTile &t)
{
    double w = 0;
    for (int k = t.k0; k < t.k1; k++) w += plane_weight(nz, L, k);
    return band_plane_cost(nx, ny, L, t.j0, t.rows) * w;
}

bool stream_plan(int nx, int ny, int nz, int L, bool lossy, int nsm, StreamPlan *out, int ty_cap)
{
    if (!stream_supported(nx, ny, nz, lossy, L) || nsm <= 0 || ty_cap < 0) return false;
    const int QX = nx / 4, rows = ny - 2, planes = nz - 2;
    int ty_max = kStreamMaxThreads / QX - 1;
    if (ty_cap > 0) ty_max = std::min(ty_max, ty_cap);
    while (ty_max > 1 && (stream_smem_floats(nx, ty_max, lossy, L) * sizeof(float) > kStreamSmemBudget ||
                          stream_roles(nx, L, ty_max + 1).threads > kStreamMaxThreads))
        ty_max--;
    ty_max = std::min(ty_max, rows);
    // Cost of a tile: its band's time a plane x (sum of its planes' weights).
    // A plane's pass is bound by the latency of the update chain as well as
    // by the bytes, so a band's plane time is a fixed part plus a part a row:
    // 0.90 + 0.22 R us for interior bands and 1.88 + 0.32 R us for bands in
    // a y slab (their updates carry the CPML recursion on every cell), with
    // 0.8 us more when a band's halo row lies in a y slab (those threads run
    // the CPML update; the band cuts avoid that), and the row part scaled by
    // nx / 200; a z-slab plane
    // weighs 1.67.  Fitted to per-tile times (%globaltimer per block) on the
    // 200 x 160 x 400 grid with a 12-cell CPML; only the ratios matter.
    std::vector<double> pc(planes);
    std::vector<char> brk(rows, 0);
    for (int t = 0; t < rows; t++) {
        const int jj = 1 + t;
        // bands split where the y slabs begin, so that interior bands hold no
        // y-slab row; above the interior the cut is one row early, so that no
        // interior band's halo row (the row above its last) lies in the slab
        brk[t] = L > 0 && (jj == L || jj == ny - L - 1);
    }
    for (int t = 0; t < planes; t++) pc[t] = plane_weight(nz, L, 1 + t);
    // bands: as few as the row limit allows between the slab boundaries, of
    // even size there (a band's plane time hardly shrinks with fewer rows, so
    // a thin remainder band would be the slowest); then chunks of planes per
    // band, handed out one at a time to the band whose tiles are the most
    // expensive, up to `nsm` tiles, none shorter than 8 planes (shorter
    // chunks re-read their boundary planes too often).  With fewer than one
    // SM a band (a share of a multi-grid sweep) every band is one tile.
    std::vector<int> bs;
    for (int t0 = 0; t0 < rows;) {
        int t1 = t0 + 1;
        while (t1 < rows && !brk[t1]) t1++;
        const int len = t1 - t0, parts = (len + ty_max - 1) / ty_max;
        for (int p = 0; p < parts; p++) bs.push_back(t0 + (int)((long long)len * p / parts));
        t0 = t1;
    }
    const int nbands = (int)bs.size();
    const int nc_max = std::max(1, planes / 8);
    std::vector<double> bcost(nbands);
    std::vector<int> nchunk(nbands, 1);
    for (int b = 0; b < nbands; b++) {
        const int r0 = bs[b], r1 = b + 1 < nbands ? bs[b + 1] : rows;
        bcost[b] = band_plane_cost(nx, ny, L, 1 + r0, r1 - r0);
    }
    for (int used = nbands; used < nsm; used++) {
        int best = -1;
        for (int b = 0; b < nbands; b++)
            if (nchunk[b] < nc_max && (best < 0 || bcost[b] / nchunk[b] > bcost[best] / nchunk[best])) best = b;
        if (best < 0) break;
        nchunk[best]++;
    }
    out->tiles.clear();
    out->ty = 0;
    for (int b = 0; b < nbands; b++) {
        const int r0 = bs[b], r1 = b + 1 < nbands ? bs[b + 1] : rows;
        out->ty = std::max(out->ty, r1 - r0);
        const std::vector<int> cs = split_runs(pc, nchunk[b], planes);
        if (cs.empty()) return false;
        for (size_t c = 0; c < cs.size(); c++) {
            const int p0 = cs[c], p1 = c + 1 < cs.size() ? cs[c + 1] : planes;
            out->tiles.push_back(StreamTile{1 + r0, r1 - r0, 1 + p0, 1 + p1});
        }
    }
    out->threads = stream_roles(nx, L, out->ty + 1).threads;
    out->smem = stream_smem_floats(nx, out->ty, lossy, L) * sizeof(float);
    return true;
}

bool stream_configure(size_t smem, int threads)
{
    if (smem > kStreamSmemBudget) return false;
    for (int v = 0; v < 4; v++)
        for (int tp = 1; tp <= 8; tp++) {   // 1: the run-time-rows kernel
            const void *f = (const void *)stream_kernel((v & 2) != 0, (v & 1) != 0, tp);
            if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
                return false;
            cudaFuncAttributes at{};
            if (cudaFuncGetAttributes(&at, f) != cudaSuccess || at.maxThreadsPerBlock < threads) return false;
        }
    return true;
}

void launch_yee_stream(const StreamArgs &a, const StreamPlan &p, cudaStream_t st)
{
    note_launch(1);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)p.tiles.size());
    cfg.blockDim = dim3((unsigned)p.threads);
    cfg.dynamicSmemBytes = p.smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, stream_kernel(a.L > 0, a.ca[0] != nullptr, a.ty + 1), a);
}

}  // namespace fdtd

// ---------------------------------------------------------------------------
// plan inspection (host only; no device work)
// ---------------------------------------------------------------------------
extern "C" int fdtd_stream_plan(int nx, int ny, int nz, int cpml_cells, int lossy, int nsm, int *tiles, int cap,
                                int *ty, int *threads, long long *smem_bytes)
{
    using namespace fdtd;
    if (cpml_cells < 0 || nsm <= 0 || !ty || !threads || !smem_bytes) return -1;
    StreamPlan p;
    if (!stream_plan(nx, ny, nz, cpml_cells, lossy != 0, nsm, &p, 0)) return -1;
    *ty = p.ty;
    *threads = p.threads;
    *smem_bytes = (long long)p.smem;
    if (tiles) {
        if (cap < (int)p.tiles.size()) return -1;
        for (size_t t = 0; t < p.tiles.size(); t++) {
            tiles[4 * t + 0] = p.tiles[t].j0;
            tiles[4 * t + 1] = p.tiles[t].rows;
            tiles[4 * t + 2] = p.tiles[t].k0;
            tiles[4 * t + 3] = p.tiles[t].k1;
        }
    }
    return (int)p.tiles.size();
}
