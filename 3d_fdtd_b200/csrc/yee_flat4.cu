// yee_flat4.cu -- the flat FP32 E and H kernels, W consecutive x cells per thread.
//
// Same arithmetic as yee_flat.cu.  A thread owns W (4 or 2) consecutive x cells
// of one row and moves every array with W-float vector loads and stores.  Each
// kernel runs in three phases: every load the thread needs (fields, neighbours,
// coefficients, source plane, CPML auxiliaries and profiles) is issued first,
// then the arithmetic, then every store.  Issuing the auxiliaries after the
// first stores would chain a DRAM round trip per dependent load-store pair (the
// compiler cannot prove the arrays apart), and almost every warp of a CPML
// grid holds some x-slab cells; with the loads up front each warp waits for
// memory once.
//
// The x-neighbour (i-1 for E, i+1 for H) comes from the adjacent lane by a warp
// shuffle when that lane holds the neighbouring group of the same row, else
// from one scalar load.  Needs nx % 4 == 0 (rows start on 16-byte boundaries);
// other widths use yee_flat.cu.
//
// Regions.  Threads are laid out per z-plane over (group, row) slots.  A grid
// without CPML runs whole planes k = 1..nz-2 with W = 4 (kind 0).  With a CPML
// the slab code holds far more state (auxiliaries, profiles), yet inside the
// box [L, N-L) of every axis it computes exactly what the plain code computes
// (kappa = 1, auxiliaries 0).  So a CPML grid splits every update into four
// launches, each compiled with only the slab terms its cells need (template
// mask SLABS: 1 x, 2 y, 4 z):
//   z-slab planes 1..L-1, nz-L..nz-2, whole        kind 0, SLABS 7, W 2
//   middle planes, y-slab rows x box columns        kind 3, SLABS 2, W 4
//   middle planes, all rows x x-slab columns        kind 4, SLABS 3, W 2
//   middle planes, interior box                     kind 1, SLABS 0, W 4
// W = 2 where the x-slab state (per element) would not fit two resident
// blocks per SM at W = 4.  The shell launches run on a second stream beside
// the box.
//
// CPML auxiliaries: the y- and z-slab ones are contiguous in x and move as
// vectors; the x-slab ones (the groups at each end of a row) per element.
#include "flat4_cells.cuh"

namespace fdtd {

template <int W, int SLABS, bool LOSSY, int KIND>
__global__ void __launch_bounds__(kBlock4, W == 4 ? (SLABS ? 2 : (LOSSY ? 3 : 4)) : 3) k_flat4_E(FlatArgs a, Region4 r)
{
    int g, j, k;
    bool live;
    locate<KIND>(r, a.nx / W, a.ny, blockIdx.x * kBlock4 + threadIdx.x, blockIdx.y, g, j, k, live);
    e_cells<W, SLABS, LOSSY>(a, g, j, k, live);
}

template <int W, int SLABS, int KIND>
__global__ void __launch_bounds__(kBlock4, W == 4 ? (SLABS ? 2 : 4) : 3) k_flat4_H(FlatArgs a, Region4 r)
{
    int g, j, k;
    bool live;
    // planes in descending order: see k_flat4_merged
    locate<KIND>(r, a.nx / W, a.ny, blockIdx.x * kBlock4 + threadIdx.x, gridDim.y - 1 - blockIdx.y, g, j, k, live);
    h_cells<W, SLABS>(a, g, j, k, live);
}

// One launch per field over a CPML grid: blocks in plane order, each plane's
// blocks split between the regions present in it (block-uniform branch).
//   planes 1..L-1, nz-L..nz-2: nbz blocks of the z-slab region (W 2, SLABS 7)
//   planes L..nz-L-1: nb_box box blocks (W 4, plain), nb_y y-slab-row blocks
//   (W 2, SLABS 2), nb_x x-slab-column blocks (W 2, SLABS 3)
// The E launch walks the planes upwards and the H launch downwards: the E
// planes the H launch reads first are the ones the E launch wrote last (still
// in the 126 MB L2), and the H planes the next E launch reads first are the
// ones the H launch wrote last.  Block order does not change any result.
template <bool E_FIELD, bool LOSSY>
__global__ void __launch_bounds__(kBlock4, E_FIELD ? 3 : 4) k_flat4_merged(FlatArgs a, Plan4 p)
{
    // Programmatic dependent launch: every block first waits until the
    // preceding grid of the stream (the previous step's tail or H update, or
    // the E update for H) has completed and its stores are visible, then lets
    // the next launch start scheduling, so its blocks fill SMs freed by this
    // grid's last wave and wait there in turn.  Both are no-ops in a launch
    // without the attribute.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    int b = E_FIELD ? (int)blockIdx.x : (int)(gridDim.x - 1 - blockIdx.x);
    const int nzs = (p.L - 1) * p.nbz, nmb = p.nmid * p.nbm;
    int plane, lb;
    bool zslab;
    if (b < nzs) {
        zslab = true;
        plane = b / p.nbz;
        lb = b - plane * p.nbz;
    } else if (b < nzs + nmb) {
        zslab = false;
        b -= nzs;
        plane = b / p.nbm;
        lb = b - plane * p.nbm;
    } else {
        zslab = true;
        b -= nzs + nmb;
        const int q = b / p.nbz;
        lb = b - q * p.nbz;
        plane = (p.L - 1) + q;  // index into zs (its second plane range)
    }
    const int t = threadIdx.x;
    int g, j, k;
    bool live;
    if (zslab) {
        locate<0>(p.zs, a.nx / 2, a.ny, lb * kBlock4 + t, plane, g, j, k, live);
        if (E_FIELD) e_cells<2, 7, LOSSY>(a, g, j, k, live);
        else h_cells<2, 7>(a, g, j, k, live);
    } else if (lb < p.nb_box) {
        locate<1>(p.box, a.nx / 4, a.ny, lb * kBlock4 + t, plane, g, j, k, live);
        if (E_FIELD) e_cells<4, 0, LOSSY>(a, g, j, k, live);
        else h_cells<4, 0>(a, g, j, k, live);
    } else if (lb < p.nb_box + p.nb_y) {
        locate<3>(p.yrows, a.nx / 2, a.ny, (lb - p.nb_box) * kBlock4 + t, plane, g, j, k, live);
        if (E_FIELD) e_cells<2, 2, LOSSY>(a, g, j, k, live);
        else h_cells<2, 2>(a, g, j, k, live);
    } else {
        locate<4>(p.xcols, a.nx / 2, a.ny, (lb - p.nb_box - p.nb_y) * kBlock4 + t, plane, g, j, k, live);
        if (E_FIELD) e_cells<2, 3, LOSSY>(a, g, j, k, live);
        else h_cells<2, 3>(a, g, j, k, live);
    }
}

int flat4_supported(int nx, int nz) { return nx % 4 == 0 && nx >= 8 && nz >= 3; }

static Region4 planes_region(int kA, int nA, int kB, int count)
{
    Region4 r{};
    r.kA = kA; r.nA = nA; r.kB = kB; r.count = count;
    return r;
}

// kernel instantiation per launch kind; kind 0 is the CPML z-slab planes (or
// whole planes of a CPML grid that does not split) when `cpml`, else the whole
// planes of a grid without CPML
template <bool LOSSY>
static void launch_E(const FlatArgs &a, const Region4 &r, dim3 grid, int kind, bool cpml, cudaStream_t st)
{
    switch (kind) {
    case 1: k_flat4_E<4, 0, LOSSY, 1><<<grid, kBlock4, 0, st>>>(a, r); break;
    case 3: k_flat4_E<4, 2, LOSSY, 3><<<grid, kBlock4, 0, st>>>(a, r); break;
    case 4: k_flat4_E<2, 3, LOSSY, 4><<<grid, kBlock4, 0, st>>>(a, r); break;
    default:
        if (cpml) k_flat4_E<2, 7, LOSSY, 0><<<grid, kBlock4, 0, st>>>(a, r);
        else k_flat4_E<4, 0, LOSSY, 0><<<grid, kBlock4, 0, st>>>(a, r);
    }
}

static void launch_H(const FlatArgs &a, const Region4 &r, dim3 grid, int kind, bool cpml, cudaStream_t st)
{
    switch (kind) {
    case 1: k_flat4_H<4, 0, 1><<<grid, kBlock4, 0, st>>>(a, r); break;
    case 3: k_flat4_H<4, 2, 3><<<grid, kBlock4, 0, st>>>(a, r); break;
    case 4: k_flat4_H<2, 3, 4><<<grid, kBlock4, 0, st>>>(a, r); break;
    default:
        if (cpml) k_flat4_H<2, 7, 0><<<grid, kBlock4, 0, st>>>(a, r);
        else k_flat4_H<4, 0, 0><<<grid, kBlock4, 0, st>>>(a, r);
    }
}

static void launch_phase(bool e_phase, const FlatArgs &a, const Region4 &r, int nplanes, int kind, bool cpml,
                         cudaStream_t st)
{
    if (r.count <= 0 || nplanes <= 0) return;
    note_launch(1);
    const dim3 grid((r.count + kBlock4 - 1) / kBlock4, nplanes);
    if (!e_phase) launch_H(a, r, grid, kind, cpml, st);
    else if (a.ca[0]) launch_E<true>(a, r, grid, kind, cpml, st);
    else launch_E<false>(a, r, grid, kind, cpml, st);
}

Plan4 flat4_plan(const FlatArgs &a)
{
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    auto nblk = [](int count) { return (count + kBlock4 - 1) / kBlock4; };
    Plan4 p{};
    if (a.L == 0) {
        p.zs = planes_region(1, nz - 2, 0, (nx / 4) * ny);
        p.nbz = nblk(p.zs.count);
        return p;
    }
    const int L = a.L, ng2 = nx / 2, nmid = nz - 2 * L;
    const int gL = (L + 3) / 4, gR = (nx - L) / 4;  // box columns in 4-cell groups
    p.L = L;
    p.nmid = nmid;
    p.zs = planes_region(1, L - 1, nz - L, ng2 * ny);
    p.box = planes_region(L, nmid, 0, (gR - gL) * (ny - 2 * L));
    p.box.gL = gL; p.box.gR = gR; p.box.L = L;
    // shell columns in 2-cell groups: [2 gL, 2 gR) for the y-slab rows, the rest for the x-slab columns
    p.yrows = planes_region(L, nmid, 0, 2 * (L - 1) * (2 * gR - 2 * gL));
    p.yrows.gL = 2 * gL; p.yrows.gR = 2 * gR; p.yrows.L = L;
    p.xcols = planes_region(L, nmid, 0, (ny - 2) * (2 * gL + ng2 - 2 * gR));
    p.xcols.gL = 2 * gL; p.xcols.gR = 2 * gR; p.xcols.L = L;
    p.nbz = nblk(p.zs.count);
    p.nb_box = nblk(p.box.count);
    p.nb_y = nblk(p.yrows.count);
    p.nbm = p.nb_box + p.nb_y + nblk(p.xcols.count);
    return p;
}

bool flat4_split_supported(const FlatArgs &a)
{
    const int L = a.L;
    if (L < 2 || a.ny <= 2 * L || a.nz <= 2 * L) return false;
    const int gL = (L + 3) / 4, gR = (a.nx - L) / 4;
    return gR > gL;
}

void launch_flat4_step(const FlatArgs &a, cudaStream_t st, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join)
{
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const bool cpml = a.L > 0;
    if (!cpml) {
        const Region4 r = planes_region(1, nz - 2, 0, (nx / 4) * ny);
        launch_phase(true, a, r, nz - 2, 0, false, st);
        launch_phase(false, a, r, nz - 2, 0, false, st);
        return;
    }
    if (!side || !flat4_split_supported(a)) {
        // CPML code (W = 2) over whole planes
        const Region4 r = planes_region(1, nz - 2, 0, (nx / 2) * ny);
        launch_phase(true, a, r, nz - 2, 0, true, st);
        launch_phase(false, a, r, nz - 2, 0, true, st);
        return;
    }
    const Plan4 p = flat4_plan(a);
    const int L = a.L, nmid = nz - 2 * L;
    const long long blocks = 2LL * (L - 1) * p.nbz + (long long)nmid * p.nbm;
    const bool lossy = a.ca[0] != nullptr;
    note_launch(2);
    // both launches carry a programmatic dependency on the kernel before them
    // (see k_flat4_merged)
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(kBlock4);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (lossy) {
        cudaLaunchKernelEx(&cfg, k_flat4_merged<true, true>, a, p);
        cudaLaunchKernelEx(&cfg, k_flat4_merged<false, true>, a, p);
    } else {
        cudaLaunchKernelEx(&cfg, k_flat4_merged<true, false>, a, p);
        cudaLaunchKernelEx(&cfg, k_flat4_merged<false, false>, a, p);
    }
    (void)side; (void)fork; (void)join;
}

}  // namespace fdtd
