// libmdgpu: the C-ABI (include/md_b200.h) over the sm_100a kernels. Host orchestration only: handles own
// their device buffers and one CUDA stream per system; every kernel is in the md_*.cuh headers.
#include "md_b200.h"

#include "md_adjoint.cuh"
#include "md_batch.cuh"
#include "md_cells.cuh"
#include "md_common.cuh"
#include "md_fp32.cuh"
#include "md_fp64.cuh"
#include "md_fx32.cuh"
#include "md_fx64.cuh"
#include "md_graph.cuh"
#include "md_nlist.cuh"
#include "md_scan.cuh"
#include "md_tiles.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <vector>

using namespace md;

namespace {

thread_local std::string g_error;
thread_local uint64_t* g_launches = nullptr;  // launch counter of the system the current call works on
// While md_run captures a chunk graph: the graph's profiling events (force kernels are bracketed by external
// event records) and the flag a tile force kernel sets when its tile outgrows the recorded shared memory
thread_local std::vector<cudaEvent_t>* g_capture_prof = nullptr;
thread_local size_t g_capture_prof_next = 0;  // next unused event of *g_capture_prof (created before capture)
thread_local int* g_graph_overflow = nullptr;
thread_local bool g_capturing = false;  // function attributes are set before a capture, not inside it
std::atomic<uint64_t> g_serial{1};  // serial numbers of force fields and lists (md_run's graphs record them)

md_status fail(md_status s, const std::string& msg) {
    g_error = msg;
    return s;
}

#define MD_CUDA(call)                                                                                  \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(MD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// After k kernel launches: surface launch errors and count the launches
#define MD_CHECK_LAUNCH_N(k)                    \
    do {                                        \
        MD_CUDA(cudaGetLastError());            \
        if (g_launches) *g_launches += (k);     \
    } while (0)
#define MD_CHECK_LAUNCH() MD_CHECK_LAUNCH_N(1)
// exclusive_scan launches three kernels
#define MD_CHECK_SCAN() MD_CHECK_LAUNCH_N(3)

#define MD_TRY(expr)                       \
    do {                                   \
        md_status s_ = (expr);             \
        if (s_ != MD_OK) return s_;        \
    } while (0)

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t count = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        count = 0;
    }
    // Grow to at least n elements (contents are not kept)
    cudaError_t reserve(size_t n) {
        if (n <= count && p) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) count = std::max<size_t>(n, 1);
        return e;
    }
};

template <typename T>
void swap_buffers(DevBuf<T>& a, DevBuf<T>& b) {
    std::swap(a.p, b.p);
    std::swap(a.count, b.count);
}

inline unsigned blocks_for(long long n, int threads) {
    return static_cast<unsigned>((n + threads - 1) / threads);
}

constexpr int kThreads = 256;
// Dynamic shared memory above this gets the opt-in attribute: static shared memory (at most 16 KB in these
// kernels) counts against the same 48 KB default, so the threshold leaves room for it.
constexpr size_t kSmemNoOptIn = 32 * 1024;

// Opt a kernel in to `bytes` of dynamic shared memory (not while md_run captures a graph: it sets them first)
template <typename K>
cudaError_t allow_smem(K kernel, size_t bytes) {
    if (g_capturing || bytes <= kSmemNoOptIn) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

// Slots of md_system::scal (device scalars)
constexpr int kScalFactor = 1;  // [1] velocity scale factor, [2] 1 to apply it / 0 to skip
constexpr int kScalKE = 4;      // [4] kinetic energy ([5] scratch of the blocked sum)
constexpr int kScalR1 = 6;      // [6] r1, [7] chi2 of one Bussi step

}  // namespace

// ---- handles ---------------------------------------------------------------------------------------------

// One chunk graph of md_run (md_run_graph.inl)
struct RunGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaEvent_t> prof;  // (before, after) each force kernel, when recorded with profiling on
    int rdf_samples = 0;            // g(r) samples per launch
    uint64_t kernels = 0;           // kernels per launch outside the rebuild bodies
    uint64_t body_kernels = 0;      // kernels of one rebuild body
};

struct md_system {
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t n = 0;
    Box box{};
    DevBuf<double4> pos, pos2;
    DevBuf<double> vel, vel2, force, force2, mass, mass2;
    DevBuf<uint64_t> ids, ids2;
    DevBuf<double2> ke_blocks;
    DevBuf<double> scal;         // device scalars, indexed by the kScal* constants
    double* host_scal = nullptr; // pinned mirror of scal
    uint64_t layout = 0;         // bumps whenever the particle order changes
    uint64_t launches = 0;       // kernels launched on this system
    // md_profile_*: events around each list force kernel of md_run
    bool profile = false;
    std::vector<cudaEvent_t> events;
    size_t events_used = 0;
    double profile_ms = 0.0;
    int64_t profile_count = 0;
    // md_system_frame_by_id: id-ordered staging buffer, its copy stream and the event that orders them
    DevBuf<double> frame;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t frame_ready = nullptr;
    // resident grid of k_force_fp32_resident<fixed, energy> (blocks that fit on the SMs at once), 0 until known
    unsigned fp32_resident[2][2] = {{0, 0}, {0, 0}};
    unsigned fx32_resident[2] = {0, 0};  // likewise for k_force_fx32<energy>
    // md_run's chunk graphs (md_run_graph.inl): the cache, chunk length (0: host loop), test flags, the stream
    // the rebuild bodies are captured on, device counters ([0] rebuilds, [1] overflow), per-chunk records and
    // Bussi draws, the snapshot a chunk restarts from, and the canonical buffer of each double-buffered array
    std::map<std::string, RunGraph> graphs;
    int graph_chunk = 64;
    int graph_flags = 0;
    cudaStream_t body_stream = nullptr;
    DevBuf<int> graph_state, snap_flag;
    DevBuf<double> chunk_rec, chunk_noise;
    DevBuf<double4> snap_pos, snap_ref, pos_save;
    DevBuf<double> snap_vel, snap_force, snap_mass;
    DevBuf<uint64_t> snap_ids;
    DevBuf<unsigned long long> snap_hist;
    void* canon[7] = {};
    uint64_t graph_launches = 0, graph_recoveries = 0;
    int64_t prepared_steps = -1;  // run length md_run_prepare last captured graphs for
};

void drop_run_graphs(md_system* s) {
    for (auto& g : s->graphs) {
        if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
        for (cudaEvent_t e : g.second.prof) cudaEventDestroy(e);
    }
    s->graphs.clear();
}

// After k_permute: the permuted arrays become the system's, the old ones its reorder buffers. No device
// pointer of a system outlives a call, so the swap is invisible outside the library.
inline void swap_reordered(md_system* s) {
    swap_buffers(s->pos, s->pos2);
    swap_buffers(s->vel, s->vel2);
    swap_buffers(s->force, s->force2);
    swap_buffers(s->mass, s->mass2);
    swap_buffers(s->ids, s->ids2);
}

struct CellGrid {
    int ncps = 0, ncells = 0;
    DevBuf<int> cell_of, count, start, cursor;
    DevBuf<uint32_t> bucket, order;
    DevBuf<long long> tiles;
};

struct md_cells {
    double min_size = 0.0;
    int device = -1;
    int64_t n = 0;
    CellGrid g;
};

struct md_nlist {
    uint64_t serial = g_serial++;
    double rc = 0, skin = 0, rl = 0, rl2 = 0, max_disp2 = 0;
    bool reverse = false;
    int device = -1;
    const md_system* sys = nullptr;
    uint64_t layout = 0;  // sys->layout right after our last build
    int64_t n = -1;
    CellGrid grid;
    int cap = 0;
    bool use_cells = false;
    DevBuf<uint32_t> rows;
    DevBuf<int2> counts;
    DevBuf<int> tmp_counts, cell_sorted, flags;  // flags: [0] stale, [1] max row, [2] device rebuild count
    DevBuf<long long> half_off, rev_off, tiles;
    DevBuf<double4> ref_pos;
    DevBuf<float4> frames;  // per-particle float coordinates for the float kernels (n + 1, sentinel last)
    DevBuf<float4> frames2; // the frames a force kernel with the fused next drift writes (then swapped in)
    DevBuf<int4> iframes;   // fixed-point frames of MD_PREC_FX64 (n)
    DevBuf<int4> iframes2;  // the fixed-point frames a FX64 force kernel with the fused next drift writes
    bool use_tiles = false; // shared-memory tile kernels (3+ cells per side and tiles that fit)
    TileGeom tiles_geom{};
    int build_kernel = -1;  // list build of the last rebuild: 0 thread per particle, 1 tiles
    int build_pin = -1;     // set by md_nlist_set_build_variant (-1: tiles where available)
    int variant[5] = {-1, -1, -1, -1, -1};  // force kernel per precision (0 global gathers, 1 tile; -1 untuned)
    int pinned[5] = {-1, -1, -1, -1, -1};   // set by md_nlist_set_force_variant
    uint64_t builds = 0;                    // list builds so far (names the rows of the last one)
    // MD_PREC_FX32's near rows and then far rows (k_rows_split) and their (near groups, far groups) counts, for
    // build nf_build with the near radius^2 nf_near2
    DevBuf<uint32_t> rows_nf;
    DevBuf<int2> counts_nf;
    uint64_t nf_build = 0;
    double nf_near2 = -1.0;
    int rebuilds = 0;
    uint64_t pairs = 0;
    bool pairs_ready = false;  // half_off and pairs match the last build
    bool built = false;
};

struct md_forcefield {
    uint64_t serial = g_serial++;
    double eps = 1, sigma = 1, rc = 2.5;
    LJ lj{};
    int precision = MD_PREC_FP64;
    bool deterministic = false;
    double virial = 0.0, inside = 0.0;
    int device = -1;
    // FP64 energies: r^2 of every own pair, in pair order, in two buffers used in turn. The ordered sums of one
    // step run on two more streams while the next step's force kernel fills the other buffer: the 1024-pair block
    // sums on `side`, the chain over the block sums (one warp) on `chain`, with the block sums in two buffers too,
    // so that the next step's block sums never wait for this step's chain. Both streams have the device's highest
    // priority, so that their blocks are not queued behind the next step's force kernel.
    DevBuf<double> pair_r2[2];
    DevBuf<double2> eblocks[2];
    DevBuf<long long> epairs;   // [b]: the pair count of the records in pair_r2[b], copied when the step fills them
    DevBuf<int> enblocks;       // [e]: the block count of eblocks[e]
    int side_priority = 0;      // of the two streams (the device's highest), also given to their kernels in graphs
    int ew_next = 0, eb_next = 0;
    cudaStream_t side = nullptr, chain = nullptr;
    cudaEvent_t ev_force = nullptr, ev_done = nullptr, ev_read[2] = {nullptr, nullptr}, ev_chain[2] = {nullptr, nullptr};
    bool read_pending[2] = {false, false};   // ev_read[b] marks the last block sums that read pair_r2[b]
    bool chain_pending[2] = {false, false};  // ev_chain[e] marks the last chain that read eblocks[e]
    bool side_pending = false;               // ev_done marks energy sums the system's stream has not joined
    DevBuf<double> out;  // [0] pe, [1] virial, [2] inside
    DevBuf<unsigned long long> inside_count;
    DevBuf<long long> fx_acc;  // fixed-point accumulators of the float kernels: pe, virial
    double* host_out = nullptr;
};

struct md_rdf {
    double rmax = 0, bin_width = 0;
    int bins = 0;
    int samples = 0;
    double particles = 0, density = 0;
    int device = -1;
    DevBuf<unsigned long long> hist;
};

namespace {

md_status use_device(int device) {
    MD_CUDA(cudaSetDevice(device));
    return MD_OK;
}

// Select the system's device and count the call's launches on it
md_status use_system(md_system* s) {
    g_launches = &s->launches;
    MD_CUDA(cudaSetDevice(s->device));
    return MD_OK;
}

md_status sync(md_system* s) {
    MD_CUDA(cudaStreamSynchronize(s->stream));
    MD_CUDA(cudaGetLastError());
    return MD_OK;
}

// Kinetic energy into s->scal[0] with the reference's blocked order (no host sync)
md_status kinetic_async(md_system* s) {
    const int n = static_cast<int>(s->n);
    const int nb = (n + kChunk - 1) / kChunk;
    if (nb == 0) {
        MD_CUDA(cudaMemsetAsync(s->scal.p + kScalKE, 0, sizeof(double), s->stream));
        return MD_OK;
    }
    MD_CUDA(s->ke_blocks.reserve(nb));
    const size_t smem = kEnergyWarps * kChunk * sizeof(double);
    k_kinetic_blocks<<<blocks_for(nb, kEnergyWarps), kEnergyWarps * 32, smem, s->stream>>>(s->vel.p, s->mass.p, n,
                                                                                          s->ke_blocks.p, nb);
    MD_CHECK_LAUNCH();
    k_sum_blocks<<<1, 32, 0, s->stream>>>(s->ke_blocks.p, nb, s->scal.p + kScalKE);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

md_status scale_async(md_system* s) {
    const long long count = 3 * s->n;
    if (count == 0) return MD_OK;
    const unsigned g = std::min<unsigned>(blocks_for(count, kThreads), 148u * 16u);
    k_scale_velocities<<<g, kThreads, 0, s->stream>>>(s->vel.p, count, s->scal.p + kScalFactor);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

double dof_of(int64_t n) { return 3.0 * static_cast<double>(n) - 3.0; }

// src/Forcefield.cpp:8-15 and the constant factors of pairTerms (:25-36)
LJ lj_constants(double epsilon, double sigma, double cutoff) {
    const double sr6 = std::pow(sigma / cutoff, 6);
    const double sr12 = sr6 * sr6;
    LJ lj{};
    lj.shift = 4.0 * epsilon * (sr12 - sr6);
    lj.sig2 = sigma * sigma;
    lj.eps24 = 24.0 * epsilon;
    lj.eps4 = 4.0 * epsilon;
    lj.rc2 = cutoff * cutoff;
    return lj;
}

// Counting sort by cell (src/CellList.cpp:9-52) into g.start / g.order; returns ncps
md_status cell_sort(CellGrid& g, md_system* s, double min_size) {
    const int n = static_cast<int>(s->n);
    const double L = s->box.L;
    g.ncps = std::max(1, static_cast<int>(L / min_size));  // src/CellList.cpp:14
    const long long nc = static_cast<long long>(g.ncps) * g.ncps * g.ncps;
    if (nc > (1ll << 30)) return fail(MD_ERR_INVALID, "cell grid too large");
    g.ncells = static_cast<int>(nc);
    const double inv_cell = g.ncps / L;  // src/CellList.cpp:18
    MD_CUDA(g.cell_of.reserve(n));
    MD_CUDA(g.count.reserve(g.ncells));
    MD_CUDA(g.cursor.reserve(g.ncells));
    MD_CUDA(g.start.reserve(g.ncells + 1));
    MD_CUDA(g.bucket.reserve(n));
    MD_CUDA(g.order.reserve(n));
    MD_CUDA(g.tiles.reserve(scan_tiles_needed(g.ncells)));
    MD_CUDA(cudaMemsetAsync(g.count.p, 0, sizeof(int) * g.ncells, s->stream));
    MD_CUDA(cudaMemsetAsync(g.cursor.p, 0, sizeof(int) * g.ncells, s->stream));
    if (n > 0) {
        k_cell_assign<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(s->pos.p, n, inv_cell, g.ncps, g.cell_of.p,
                                                                           g.count.p);
        MD_CHECK_LAUNCH();
    }
    exclusive_scan<int, int>(g.count.p, g.ncells, g.start.p, g.tiles.p, s->stream);
    MD_CHECK_SCAN();
    if (n > 0) {
        k_cell_scatter<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(g.cell_of.p, n, g.start.p, g.cursor.p,
                                                                            g.bucket.p);
        MD_CHECK_LAUNCH();
        k_cell_rank<<<blocks_for(static_cast<long long>(g.ncells) * 32, kThreads), kThreads, 0, s->stream>>>(
            g.start.p, g.ncells, g.bucket.p, g.order.p);
        MD_CHECK_LAUNCH();
    }
    return MD_OK;
}

int initial_capacity(const md_nlist* nl, const md_system* s) {
    const double vol = s->box.L * s->box.L * s->box.L;
    const double rho = static_cast<double>(s->n) / vol;
    double est = 4.18879020478639 * nl->rl2 * nl->rl * rho;  // full sphere of radius r_l
    est = std::min(est, static_cast<double>(s->n));
    int cap = static_cast<int>(1.35 * est) + 24;
    return (cap + 7) & ~7;
}

// Defined in md_abi_float.inl
md_status frames_async(md_system* s, md_nlist* nl);
CellOffsets cell_offsets(const md_nlist* nl, const md_system* s);

#ifndef MD_TILE_HOME_TARGET
#define MD_TILE_HOME_TARGET 96.0
#endif
constexpr double kTileHomeTarget = MD_TILE_HOME_TARGET;  // home particles per tile block aimed at

// Segment length and shared-memory size of the tile kernels for this build. Segments aim at ~96 home
// particles per block. The largest staged tile of the geometry is measured on the device (the cells only
// change at rebuilds, so it holds until the next one); it must fit 3072 slots (96 KB of double4 for the
// FP64 kernel), shrinking kk down to one cell. Beyond 6000 slots the global-gather kernels are used instead.
md_status tile_geometry(md_nlist* nl, md_system* s, bool* use) {
    *use = false;
    const int nc = nl->grid.ncps;
    if (nc < 3 || s->n == 0) return MD_OK;
    const double avg = static_cast<double>(s->n) / (static_cast<double>(nc) * nc * nc);
    int kk = static_cast<int>(std::lround(kTileHomeTarget / std::max(avg, 1.0)));
    kk = std::clamp(kk, 1, std::min(kMaxSegment, nc - 2));
    TileGeom& g = nl->tiles_geom;
    for (;;) {
        g.ncps = nc;
        g.kk = kk;
        g.nseg = (nc + kk - 1) / kk;
        g.cell = s->box.L / nc;
        g.box = s->box;
        MD_CUDA(cudaMemsetAsync(nl->flags.p + 2, 0, sizeof(int), s->stream));
        const long long segs = static_cast<long long>(nc) * nc * g.nseg;
        k_tile_max_staged<<<blocks_for(segs, 128), 128, 0, s->stream>>>(nl->grid.start.p, g, nl->flags.p + 2);
        MD_CHECK_LAUNCH();
        int staged = 0;
        MD_CUDA(cudaMemcpyAsync(&staged, nl->flags.p + 2, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        MD_TRY(sync(s));
        g.max_staged = std::max(staged, 1);
        if (staged <= 3072 || kk == 1) {
            *use = staged <= 6000;
            return MD_OK;
        }
        --kk;
    }
}

unsigned tile_blocks(const TileGeom& g) { return static_cast<unsigned>(g.ncps) * g.ncps * g.nseg; }

// NeighbourList::build (src/NeighbourList.cpp:55-134) on the device. The reference builds the cell list,
// reorders the system, and builds the cell list again; the second build only recomputes the cells of the
// already sorted particles (same positions, identity order), which k_permute writes directly.
md_status nlist_build(md_nlist* nl, md_system* s) {
    if (2.0 * nl->rl > s->box.L) return fail(MD_ERR_LIST_RADIUS, "Cutoff + skin must be less than half the box length");
    const int n = static_cast<int>(s->n);
    nl->device = s->device;
    MD_TRY(cell_sort(nl->grid, s, nl->rl));
    MD_CUDA(s->pos2.reserve(n));
    MD_CUDA(s->vel2.reserve(3 * static_cast<size_t>(n)));
    MD_CUDA(s->force2.reserve(3 * static_cast<size_t>(n)));
    MD_CUDA(s->mass2.reserve(n));
    MD_CUDA(s->ids2.reserve(n));
    MD_CUDA(nl->cell_sorted.reserve(n));
    MD_CUDA(nl->ref_pos.reserve(n));
    if (n > 0) {
        k_permute<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(
            nl->grid.order.p, n, s->pos.p, s->vel.p, s->force.p, s->mass.p, s->ids.p, s->pos2.p, s->vel2.p,
            s->force2.p, s->mass2.p, s->ids2.p, nl->grid.cell_of.p, nl->cell_sorted.p, nl->ref_pos.p);
        MD_CHECK_LAUNCH();
        swap_reordered(s);
    }
    s->layout++;
    nl->use_cells = nl->grid.ncps >= 3;  // src/NeighbourList.cpp:69
    if (nl->cap == 0 || nl->n != s->n) {
        nl->cap = initial_capacity(nl, s);
        for (int& v : nl->variant) v = -1;  // a new system: tune the force kernels again
    }
    MD_CUDA(nl->counts.reserve(n));
    MD_CUDA(nl->flags.reserve(4));
    MD_CUDA(nl->half_off.reserve(n + 1));
    MD_CUDA(nl->tmp_counts.reserve(n));
    MD_CUDA(nl->tiles.reserve(scan_tiles_needed(n)));
    nl->use_tiles = false;
    if (nl->use_cells && n > 0) {
        MD_TRY(frames_async(s, nl));  // float frames of the new cells (the tile build's prefilter reads them)
        MD_TRY(tile_geometry(nl, s, &nl->use_tiles));
    }
    const uint32_t sentinel = static_cast<uint32_t>(n) | (kSentinelCode << kCodeShift);
    for (int attempt = 0; attempt < 4; ++attempt) {
        MD_CUDA(nl->rows.reserve(row_buffer_entries(n, nl->cap)));
        MD_CUDA(cudaMemsetAsync(nl->flags.p, 0, 4 * sizeof(int), s->stream));
        if (n > 0 && nl->use_tiles && nl->build_pin != 0) {
            const TileGeom& tg = nl->tiles_geom;
            const double margin = 1e-5 * nl->rl2 + 1e-4;  // float r^2 error is below 1e-5 here
            BuildParams bp{nl->rl2, static_cast<float>(nl->rl2 - margin), static_cast<float>(nl->rl2 + margin),
                           nl->cap, static_cast<uint32_t>(n)};
            const size_t smem = sizeof(float4) * tg.max_staged;
            MD_CUDA(allow_smem(k_nlist_build_tile, smem));
            k_nlist_build_tile<<<tile_blocks(tg), kTileThreads, smem, s->stream>>>(
                nl->frames.p, s->pos.p, nl->grid.start.p, nl->cell_sorted.p, tg, bp, cell_offsets(nl, s), nl->rows.p,
                nl->counts.p, nl->flags.p + 1);
            MD_CHECK_LAUNCH();
            nl->build_kernel = 1;
        } else if (n > 0) {
            ListGeom geo{s->box, nl->rl2, nl->grid.ncps, nl->use_cells ? 1 : 0, nl->cap, sentinel};
            k_nlist_build<<<blocks_for(n, 128), 128, 0, s->stream>>>(s->pos.p, n, geo, nl->cell_sorted.p,
                                                                      nl->grid.start.p, nl->rows.p, nl->counts.p,
                                                                      nl->flags.p + 1);
            MD_CHECK_LAUNCH();
            nl->build_kernel = 0;
        }
        int maxrow = 0;
        MD_CUDA(cudaMemcpyAsync(&maxrow, nl->flags.p + 1, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        MD_TRY(sync(s));
        if (maxrow <= nl->cap) break;
        nl->cap = ((maxrow + maxrow / 4 + 16) + 7) & ~7;
        if (attempt == 3) return fail(MD_ERR_CAPACITY, "neighbour row capacity could not be met");
    }
    nl->pairs_ready = false;  // the half-list offsets and pair count are computed when first needed
    nl->builds++;
    nl->n = s->n;
    nl->sys = s;
    nl->layout = s->layout;
    nl->built = true;
    nl->rebuilds++;
    return MD_OK;
}

// The half-list offsets (half_off) and the pair count of the last build: an exclusive scan of the own counts,
// computed on first use after a build (the FP64 energies, the pair count, the download); float runs never need it
md_status ensure_pairs(md_nlist* nl) {
    if (nl->pairs_ready || !nl->built) return MD_OK;
    md_system* s = const_cast<md_system*>(nl->sys);
    const int n = static_cast<int>(nl->n);
    if (n > 0) {
        k_own_counts<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(nl->counts.p, n, nl->tmp_counts.p);
        MD_CHECK_LAUNCH();
    }
    exclusive_scan<int, long long>(nl->tmp_counts.p, n, nl->half_off.p, nl->tiles.p, s->stream);
    MD_CHECK_SCAN();
    long long pairs = 0;
    MD_CUDA(cudaMemcpyAsync(&pairs, nl->half_off.p + n, sizeof(long long), cudaMemcpyDeviceToHost, s->stream));
    MD_TRY(sync(s));
    nl->pairs = static_cast<uint64_t>(pairs);
    nl->pairs_ready = true;
    return MD_OK;
}

bool nlist_current(const md_nlist* nl, const md_system* s) {
    return nl->built && nl->sys == s && nl->n == s->n && nl->layout == s->layout;
}

// Defined in md_abi_float.inl and below
md_status forces_list_float_async(md_forcefield* ff, md_system* s, md_nlist* nl, bool want_energy, double kick_dt,
                                  bool frames_fresh, bool* fused_ke, bool fuse_drift, bool fixed_fresh);
md_status rdf_sample_async(md_rdf* r, md_system* s, md_nlist* nl);
md_status run_steps(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps,
                    const md_run_options& o, double* pe, double* ke, double* virial);

md_status check_cutoff(const md_forcefield* ff, const md_system* s) {
    if (2.0 * ff->rc > s->box.L) return fail(MD_ERR_CUTOFF, "Cutoff must be less than half the box length");
    return MD_OK;
}

// md_profile_*: a CUDA event on the system's stream before and after each list force kernel
md_status profile_mark(md_system* s) {
    if (!s->profile) return MD_OK;
    if (g_capture_prof) {  // inside a graph capture: an event record node, recorded at every launch
        if (g_capture_prof_next >= g_capture_prof->size()) return fail(MD_ERR_STATE, "graph profile events exhausted");
        MD_CUDA(cudaEventRecordWithFlags((*g_capture_prof)[g_capture_prof_next++], s->stream, cudaEventRecordExternal));
        return MD_OK;
    }
    if (s->events_used == s->events.size()) {
        cudaEvent_t e;
        MD_CUDA(cudaEventCreate(&e));
        s->events.push_back(e);
    }
    MD_CUDA(cudaEventRecord(s->events[s->events_used++], s->stream));
    return MD_OK;
}

// Sum the (start, end) event pairs recorded so far; the stream must have been synchronised
md_status profile_collect(md_system* s) {
    for (size_t k = 0; k + 1 < s->events_used; k += 2) {
        float ms = 0.f;
        MD_CUDA(cudaEventElapsedTime(&ms, s->events[k], s->events[k + 1]));
        s->profile_ms += ms;
        s->profile_count++;
    }
    s->events_used = 0;
    return MD_OK;
}

// Autotuner of the list force kernel: with tiles available, the first force call of a list (per precision)
// times the global-gather kernel (variant 0) and the shared-memory tile kernel (variant 1) on the current
// state, two launches each after a warm-up, and keeps the faster. Both variants give the same bits, so the
// choice never changes a result. md_nlist_set_force_variant pins a variant instead.
template <typename Launch>
md_status choose_variant(md_system* s, md_nlist* nl, int prec, Launch&& launch) {
    // variants available: 0 always, 1 with tiles; for FP64 2 (branch-free quads); for the float modes 2, 3
    // and 4 (prefetching global gathers; the second with capped registers, the third on a resident grid)
    unsigned mask = 1u | (nl->use_tiles ? 2u : 0u) | (prec == MD_PREC_FP32FX || prec == MD_PREC_FP32 ? 28u : 0u) |
                    (prec == MD_PREC_FP64 ? 4u : 0u);
    if (nl->variant[prec] >= 0 && ((mask >> nl->variant[prec]) & 1u)) return MD_OK;
    if (mask == 1u) {
        nl->variant[prec] = 0;
        return MD_OK;
    }
    if (nl->pinned[prec] >= 0 && ((mask >> nl->pinned[prec]) & 1u)) {
        nl->variant[prec] = nl->pinned[prec];
        return MD_OK;
    }
    cudaEvent_t e0, e1;
    MD_CUDA(cudaEventCreate(&e0));
    MD_CUDA(cudaEventCreate(&e1));
    float best = 0.f;
    int pick = -1;
    for (int v = 0; v < 5; ++v) {
        if (!((mask >> v) & 1u)) continue;
        MD_TRY(launch(v));
        MD_CUDA(cudaEventRecord(e0, s->stream));
        MD_TRY(launch(v));
        MD_TRY(launch(v));
        MD_CUDA(cudaEventRecord(e1, s->stream));
        MD_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        MD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (pick < 0 || ms < best) {
            best = ms;
            pick = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    nl->variant[prec] = pick;
    return MD_OK;
}

// A step's force stage. What it leaves behind:
//   - list forces in s->force;
//   - with want_energy, (pe, virial) in ff->out and the inside-cutoff count in ff->inside_count;
//   - with kick_dt > 0, the closing half kick (VelocityVerletIntegrator::kick) applied to the velocities.
// frames_fresh tells the float kernels that the frames already match the positions (the fused drift wrote
// them). Returns through *fused_ke whether the fused kick also left the step's kinetic energy in
// s->scal[kScalKE] (float tile kernels only; fixed-point, not the reference's summation order).
md_status kick_async(md_system* s, double dt);
// Lists with fewer pairs than this keep each pair's (E, W) for the FP64 energy sums, larger ones its r^2
// (store_pair_rec)
constexpr long long kTermsMaxPairs = 4'000'000;

// A kernel launch carrying a scheduling priority: the launch keeps it when a CUDA graph records it (a graph's
// nodes do not take the priority of the stream they were captured from)
template <typename... P, typename... A>
md_status launch_priority(void (*kernel)(P...), unsigned grid, unsigned block, cudaStream_t st, int priority,
                          A&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = priority;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MD_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
    MD_CHECK_LAUNCH();
    return MD_OK;
}

// The FP64 energy sums' two streams and their events, created on the first force call that records energies
md_status energy_streams(md_forcefield* ff) {
    int least = 0, greatest = 0;
    MD_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    MD_CUDA(cudaStreamCreateWithPriority(&ff->side, cudaStreamNonBlocking, greatest));
    MD_CUDA(cudaStreamCreateWithPriority(&ff->chain, cudaStreamNonBlocking, greatest));
    ff->side_priority = greatest;
    for (cudaEvent_t* e : {&ff->ev_force, &ff->ev_done, &ff->ev_read[0], &ff->ev_read[1], &ff->ev_chain[0],
                           &ff->ev_chain[1]})
        MD_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    MD_CUDA(ff->epairs.reserve(2));
    MD_CUDA(ff->enblocks.reserve(2));
    return MD_OK;
}

// Waits for every energy sum queued on the two streams; afterwards no buffer is being read and the buffers are used
// from the first pair again (what a CUDA graph's capture starts from and what its run leaves behind)
md_status energy_quiesce(md_forcefield* ff) {
    if (ff->side) {
        MD_CUDA(cudaStreamSynchronize(ff->side));
        MD_CUDA(cudaStreamSynchronize(ff->chain));
    }
    ff->read_pending[0] = ff->read_pending[1] = false;
    ff->chain_pending[0] = ff->chain_pending[1] = false;
    ff->side_pending = false;
    ff->ew_next = ff->eb_next = 0;
    return MD_OK;
}

// Both pairs of energy buffers for at least `pairs` pair records of either form (two doubles each; call with
// nothing queued on the streams)
md_status reserve_energy_records(md_forcefield* ff, long long pairs) {
    const size_t blocks = static_cast<size_t>((pairs + kChunk - 1) / kChunk) + 1;
    for (DevBuf<double>& r : ff->pair_r2) MD_CUDA(r.reserve(2 * static_cast<size_t>(pairs)));
    for (DevBuf<double2>& e : ff->eblocks) MD_CUDA(e.reserve(blocks));
    return MD_OK;
}

// The system's stream waits for the FP64 energy sums queued on the force field's side streams (every reader or
// writer of ff->out on the system's stream calls this first)
md_status join_energy(md_forcefield* ff, md_system* s) {
    if (ff->side_pending) {
        MD_CUDA(cudaStreamWaitEvent(s->stream, ff->ev_done, 0));
        ff->side_pending = false;
    }
    return MD_OK;
}

// The stream on which ff->out is final after the last force call: the chain stream while its sums are pending
cudaStream_t energy_stream(const md_forcefield* ff, const md_system* s) {
    return ff->side_pending ? ff->chain : s->stream;
}

// With fuse_drift (float modes on a tiled list, with the closing kick) the kernel also performs the next step's
// opening kick and drift (KickArgs), leaving the new positions and frames in place and the half-skin flag in
// nl->flags[0].
md_status forces_list_async(md_forcefield* ff, md_system* s, md_nlist* nl, bool want_energy, double kick_dt = 0.0,
                            bool frames_fresh = false, bool* fused_ke = nullptr, bool fuse_drift = false,
                            bool fixed_fresh = false) {
    const int n = static_cast<int>(s->n);
    if (fused_ke) *fused_ke = false;
    if (ff->precision != MD_PREC_FP64) MD_TRY(join_energy(ff, s));
    MD_CUDA(ff->out.reserve(4));
    MD_CUDA(ff->inside_count.reserve(1));
    MD_CUDA(cudaMemsetAsync(ff->inside_count.p, 0, sizeof(unsigned long long), s->stream));
    if (ff->precision == MD_PREC_FP64) {
        // Inside a CUDA graph's capture (g_capturing) the pair count of a list the graph rebuilt is known only on
        // the device (half_off[n]): the buffers were sized before the capture (graph_prepare_buffers), the record
        // stores stop at their size, and the sums read the count from the device.
        const bool capturing = g_capturing;
        if (n > 0 && !capturing) MD_TRY(ensure_pairs(nl));
        const long long pairs = n > 0 && !capturing ? static_cast<long long>(nl->pairs) : 0;
        const int nb = static_cast<int>((pairs + kChunk - 1) / kChunk);
        // the r^2 record buffer this step fills: free once the block sums that last read it are done
        const int b = ff->ew_next;
        const bool sums = want_energy && (capturing ? n > 0 : nb > 0);
        if (sums) {
            if (!capturing) {
                if (!ff->side) MD_TRY(energy_streams(ff));
                const auto small = [&](size_t r2, size_t blocks) {
                    return r2 < 2 * static_cast<size_t>(pairs) || blocks < static_cast<size_t>(nb);
                };
                if (small(ff->pair_r2[0].count, ff->eblocks[0].count) ||
                    small(ff->pair_r2[1].count, ff->eblocks[1].count)) {
                    // buffers are about to be replaced: no sums may read them; both pairs grow together (so that
                    // the second buffer is not allocated in the middle of a run), with headroom, since the pair
                    // count drifts up and down from one rebuild to the next
                    MD_TRY(energy_quiesce(ff));
                    MD_TRY(reserve_energy_records(ff, pairs + pairs / 8));
                }
            }
            if (ff->read_pending[b]) MD_CUDA(cudaStreamWaitEvent(s->stream, ff->ev_read[b], 0));
        }
        const long long rec_cap = sums ? static_cast<long long>(ff->pair_r2[b].count / 2) : 0;
        const bool terms = (capturing ? rec_cap : pairs) < kTermsMaxPairs;  // the records' form
        if (n > 0) {
            // variant 0: global gathers; 1: shared-memory tile; 2: global gathers a quad of entries at a time,
            // branch-free (all bit-identical). With want_energy the kernel also stores every own pair's r^2 in
            // pair order for the blocked sums below.
            auto launch_form = [&](int variant, bool kick, double* ew, auto form) -> md_status {
                constexpr bool kTerms = decltype(form)::value;
                if (variant == 1) {
                    const TileGeom& tg = nl->tiles_geom;
                    const size_t smem = sizeof(double4) * tg.max_staged;
                    MD_CUDA(allow_smem(k_force_fp64_tile<kTerms>, smem));
                    const KickArgs ka{kick ? s->vel.p : nullptr, s->mass.p, 0.5 * kick_dt};
                    k_force_fp64_tile<kTerms><<<tile_blocks(tg), kTileThreads, smem, s->stream>>>(
                        s->pos.p, n, nl->grid.start.p, nl->cell_sorted.p, tg, ff->lj, nl->rows.p, nl->cap,
                        nl->counts.p, s->force.p, ff->inside_count.p, ka, nl->half_off.p, ew, rec_cap);
                } else if (variant == 2) {
                    k_force_fp64_quads<kTerms><<<blocks_for(n, 128), 128, 0, s->stream>>>(
                        s->pos.p, n, s->box, ff->lj, nl->rows.p, nl->cap, nl->counts.p, s->force.p, ff->inside_count.p,
                        kick ? s->vel.p : nullptr, s->mass.p, 0.5 * kick_dt, nl->half_off.p, ew, rec_cap);
                } else {
                    k_force_fp64<kTerms><<<blocks_for(n, 128), 128, 0, s->stream>>>(
                        s->pos.p, n, s->box, ff->lj, nl->rows.p, nl->cap, nl->counts.p, s->force.p, ff->inside_count.p,
                        kick ? s->vel.p : nullptr, s->mass.p, 0.5 * kick_dt, nl->half_off.p, ew, rec_cap);
                }
                MD_CHECK_LAUNCH();
                return MD_OK;
            };
            auto launch = [&](int variant, bool kick, double* ew) -> md_status {
                return terms ? launch_form(variant, kick, ew, std::true_type{})
                             : launch_form(variant, kick, ew, std::false_type{});
            };
            MD_TRY(choose_variant(s, nl, MD_PREC_FP64, [&](int v) { return launch(v, false, nullptr); }));
            MD_CUDA(cudaMemsetAsync(ff->inside_count.p, 0, sizeof(unsigned long long), s->stream));
            MD_TRY(profile_mark(s));
            MD_TRY(launch(nl->variant[MD_PREC_FP64], kick_dt > 0.0, sums ? ff->pair_r2[b].p : nullptr));
            MD_TRY(profile_mark(s));
        }
        if (want_energy) {
            if (sums) {
                // the ordered sums on the side streams, after this step's force kernel; the next step goes on
                const int eb = ff->eb_next;
                const int grid_blocks = capturing ? static_cast<int>((rec_cap + kChunk - 1) / kChunk) : nb;
                // the sums' pair count: on the host path the host's (passed as their record capacity); in a graph
                // the device's, copied to a slot kept with the records (a rebuild for the next step rewrites
                // half_off). Measured: the copy on every host step made 2000-step runs at 4M a quarter slower.
                const long long* count = nullptr;
                long long sum_cap = pairs;
                if (capturing) {
                    k_copy_count<<<1, 1, 0, s->stream>>>(nl->half_off.p + n, ff->epairs.p + b);
                    MD_CHECK_LAUNCH();
                    count = ff->epairs.p + b;
                    sum_cap = rec_cap;
                }
                MD_CUDA(cudaEventRecord(ff->ev_force, s->stream));
                MD_CUDA(cudaStreamWaitEvent(ff->side, ff->ev_force, 0));
                if (ff->chain_pending[eb]) MD_CUDA(cudaStreamWaitEvent(ff->side, ff->ev_chain[eb], 0));
                if (terms)
                    MD_TRY(launch_priority(k_pair_block_sums_terms, blocks_for(grid_blocks, 32 * kPairSumWarpsTerms),
                                           32 * kPairSumWarpsTerms, ff->side, ff->side_priority,
                                           reinterpret_cast<const double2*>(ff->pair_r2[b].p), count, sum_cap,
                                           ff->eblocks[eb].p, ff->enblocks.p + eb));
                else
                    MD_TRY(launch_priority(k_pair_block_sums, blocks_for(grid_blocks, 32 * kPairSumWarps),
                                           32 * kPairSumWarps, ff->side, ff->side_priority, ff->pair_r2[b].p,
                                           count, sum_cap, ff->lj, ff->eblocks[eb].p, ff->enblocks.p + eb));
                MD_CUDA(cudaEventRecord(ff->ev_read[b], ff->side));
                ff->read_pending[b] = true;
                ff->ew_next = b ^ 1;
                MD_CUDA(cudaStreamWaitEvent(ff->chain, ff->ev_read[b], 0));
                MD_TRY(launch_priority(k_sum_pair_blocks, 1, 32, ff->chain, ff->side_priority, ff->eblocks[eb].p,
                                       ff->enblocks.p + eb, ff->out.p));
                MD_CUDA(cudaEventRecord(ff->ev_chain[eb], ff->chain));
                ff->chain_pending[eb] = true;
                ff->eb_next = eb ^ 1;
                MD_CUDA(cudaEventRecord(ff->ev_done, ff->chain));
                ff->side_pending = true;
            } else {
                MD_TRY(join_energy(ff, s));
                MD_CUDA(cudaMemsetAsync(ff->out.p, 0, 2 * sizeof(double), s->stream));
            }
        }
    } else {
        MD_TRY(forces_list_float_async(ff, s, nl, want_energy, kick_dt, frames_fresh, fused_ke, fuse_drift,
                                       fixed_fresh));
    }
    return MD_OK;
}

md_status read_energy(md_forcefield* ff, md_system* s, double* pe, double* virial, double* inside) {
    MD_TRY(join_energy(ff, s));
    unsigned long long ins = 0;
    double out[2] = {0, 0};
    MD_CUDA(cudaMemcpyAsync(out, ff->out.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MD_CUDA(cudaMemcpyAsync(&ins, ff->inside_count.p, sizeof(ins), cudaMemcpyDeviceToHost, s->stream));
    MD_TRY(sync(s));
    ff->virial = out[1];
    ff->inside = static_cast<double>(ins);
    if (pe) *pe = out[0];
    if (virial) *virial = out[1];
    if (inside) *inside = ff->inside;
    return MD_OK;
}

// Half kick + drift + wrap; with check_skin also the list's half-skin test into nl->flags[0]; with
// write_frames also the float frames of the new positions (the list must be current and use tiles).
md_status kick_drift_async(md_system* s, md_nlist* nl, double dt, bool check_skin, bool write_frames = false) {
    const int n = static_cast<int>(s->n);
    if (n == 0) return MD_OK;
    if (check_skin) MD_CUDA(cudaMemsetAsync(nl->flags.p, 0, sizeof(int), s->stream));
    if (write_frames) {
        const TileGeom& tg = nl->tiles_geom;
        k_kick_drift_frames<<<blocks_for(n + 1, kThreads), kThreads, 0, s->stream>>>(
            s->pos.p, s->vel.p, s->force.p, s->mass.p, n, 0.5 * dt, dt, s->box, check_skin ? nl->ref_pos.p : nullptr,
            nl->max_disp2, check_skin ? nl->flags.p : nullptr, nl->cell_sorted.p, tg.ncps, tg.cell, nl->frames.p);
    } else {
        k_kick_drift<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(
            s->pos.p, s->vel.p, s->force.p, s->mass.p, n, 0.5 * dt, dt, s->box, check_skin ? nl->ref_pos.p : nullptr,
            nl ? nl->max_disp2 : 0.0, check_skin ? nl->flags.p : nullptr);
    }
    MD_CHECK_LAUNCH();
    return MD_OK;
}

// The first half of VelocityVerletIntegrator::step (src/Integrator.cpp:18-30): kick, drift and wrap, then
// NeighbourList::update. The staleness flag is read back (one 4-byte copy); a stale or never-built list is
// rebuilt. Afterwards the float frames match the positions whenever the list uses tiles.
md_status drift_and_update(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, bool* rebuilt) {
    const bool current = nlist_current(nl, s);
    const bool frames = current && nl->use_tiles &&
                        (ff->precision == MD_PREC_FP32FX || ff->precision == MD_PREC_FP32 || ff->precision == MD_PREC_FX32);
    MD_TRY(kick_drift_async(s, nl, dt, current, frames));
    bool stale = true;
    if (current) {
        int flag = 0;
        MD_CUDA(cudaMemcpyAsync(&flag, nl->flags.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        MD_TRY(sync(s));
        stale = flag != 0;
    }
    if (stale) MD_TRY(nlist_build(nl, s));
    *rebuilt = stale;
    return MD_OK;
}

md_status kick_async(md_system* s, double dt) {
    const int n = static_cast<int>(s->n);
    if (n == 0) return MD_OK;
    k_kick<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(s->vel.p, s->force.p, s->mass.p, n, 0.5 * dt);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

}  // namespace

#include "md_abi_float.inl"
#include "md_run_graph.inl"

// ---- library ---------------------------------------------------------------------------------------------

extern "C" {

const char* md_last_error(void) { return g_error.c_str(); }

const char* md_version(void) { return "md-b200 0.1 (sm_100a)"; }

int md_device_count(void) {
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return c;
}

// ---- System ------------------------------------------------------------------------------------------------

md_status md_system_create(int64_t n, double box_length, int device, md_system** out) {
    if (!out || n < 0 || n > kMaxParticles || !(box_length > 0.0)) return fail(MD_ERR_INVALID, "md_system_create: bad arguments");
    if (md_device_count() <= device || device < 0) return fail(MD_ERR_NO_DEVICE, "no CUDA device " + std::to_string(device));
    MD_TRY(use_device(device));
    auto* s = new md_system;
    s->device = device;
    s->n = n;
    s->box = Box{box_length, 1.0 / box_length, 0.25 * box_length};
    md_status st = MD_OK;
    auto chk = [&](cudaError_t e) {
        if (e != cudaSuccess && st == MD_OK) st = fail(MD_ERR_CUDA, cudaGetErrorString(e));
    };
    chk(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    chk(s->pos.reserve(n));
    chk(s->vel.reserve(3 * n));
    chk(s->force.reserve(3 * n));
    chk(s->mass.reserve(n));
    chk(s->ids.reserve(n));
    chk(s->scal.reserve(8));
    chk(cudaMallocHost(reinterpret_cast<void**>(&s->host_scal), 8 * sizeof(double)));
    if (st == MD_OK && n > 0) {
        chk(cudaMemsetAsync(s->pos.p, 0, sizeof(double4) * n, s->stream));
        chk(cudaMemsetAsync(s->vel.p, 0, sizeof(double) * 3 * n, s->stream));
        chk(cudaMemsetAsync(s->force.p, 0, sizeof(double) * 3 * n, s->stream));
        std::vector<double> ones(n, 1.0);
        std::vector<uint64_t> ids(n);
        for (int64_t i = 0; i < n; ++i) ids[i] = static_cast<uint64_t>(i);
        chk(cudaMemcpyAsync(s->mass.p, ones.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
        chk(cudaMemcpyAsync(s->ids.p, ids.data(), sizeof(uint64_t) * n, cudaMemcpyHostToDevice, s->stream));
        chk(cudaStreamSynchronize(s->stream));
    }
    if (st != MD_OK) {
        md_system_destroy(s);
        return st;
    }
    *out = s;
    return MD_OK;
}

md_status md_system_destroy(md_system* s) {
    if (!s) return MD_OK;
    if (g_launches == &s->launches) g_launches = nullptr;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    for (cudaEvent_t e : s->events) cudaEventDestroy(e);
    if (s->frame_ready) cudaEventDestroy(s->frame_ready);
    if (s->host_scal) cudaFreeHost(s->host_scal);
    drop_run_graphs(s);
    if (s->body_stream) cudaStreamDestroy(s->body_stream);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return MD_OK;
}

// Trajectory.cpp:4-25's frame in id order: a device scatter through the ids (the inverse of the list's
// permutation) into a staging buffer, then one copy to the host on a second stream, so the system's stream
// can go on stepping while the frame travels and the host formats the previous one.
md_status md_system_frame_by_id(md_system* s, double* out6, int wait) {
    if (!s || !out6) return fail(MD_ERR_INVALID, "md_system_frame_by_id: bad arguments");
    MD_TRY(use_system(s));
    const int n = static_cast<int>(s->n);
    if (!s->copy_stream) MD_CUDA(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
    if (!s->frame_ready) MD_CUDA(cudaEventCreateWithFlags(&s->frame_ready, cudaEventDisableTiming));
    // the previous frame's copy must be done with the staging buffer
    MD_CUDA(cudaStreamSynchronize(s->copy_stream));
    MD_CUDA(s->frame.reserve(6 * static_cast<size_t>(n)));
    if (n > 0) {
        k_frame_by_id<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(s->pos.p, s->vel.p, s->ids.p, n, s->frame.p);
        MD_CHECK_LAUNCH();
    }
    MD_CUDA(cudaEventRecord(s->frame_ready, s->stream));
    MD_CUDA(cudaStreamWaitEvent(s->copy_stream, s->frame_ready, 0));
    MD_CUDA(cudaMemcpyAsync(out6, s->frame.p, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, s->copy_stream));
    if (wait) MD_CUDA(cudaStreamSynchronize(s->copy_stream));
    return MD_OK;
}

md_status md_system_frame_wait(md_system* s) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    MD_TRY(use_system(s));
    if (s->copy_stream) MD_CUDA(cudaStreamSynchronize(s->copy_stream));
    return MD_OK;
}

md_status md_system_size(const md_system* s, int64_t* n, double* box_length) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    if (n) *n = s->n;
    if (box_length) *box_length = s->box.L;
    return MD_OK;
}

md_status md_system_upload(md_system* s, const double* pos4, const double* vel3, const double* force3,
                           const double* mass, const uint64_t* ids) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    MD_TRY(use_system(s));
    const size_t n = static_cast<size_t>(s->n);
    if (n == 0) return MD_OK;
    if (pos4) MD_CUDA(cudaMemcpyAsync(s->pos.p, pos4, sizeof(double4) * n, cudaMemcpyHostToDevice, s->stream));
    if (vel3) MD_CUDA(cudaMemcpyAsync(s->vel.p, vel3, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s->stream));
    if (force3) MD_CUDA(cudaMemcpyAsync(s->force.p, force3, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s->stream));
    if (mass) MD_CUDA(cudaMemcpyAsync(s->mass.p, mass, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
    if (ids) MD_CUDA(cudaMemcpyAsync(s->ids.p, ids, sizeof(uint64_t) * n, cudaMemcpyHostToDevice, s->stream));
    // New positions keep the particle order, so a list built before stays usable until update() says it is
    // stale, as with System::setPosition in the reference
    return sync(s);
}

md_status md_system_download(md_system* s, double* pos4, double* vel3, double* force3, double* mass, uint64_t* ids) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    MD_TRY(use_system(s));
    const size_t n = static_cast<size_t>(s->n);
    if (n == 0) return MD_OK;
    if (pos4) MD_CUDA(cudaMemcpyAsync(pos4, s->pos.p, sizeof(double4) * n, cudaMemcpyDeviceToHost, s->stream));
    if (vel3) MD_CUDA(cudaMemcpyAsync(vel3, s->vel.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s->stream));
    if (force3) MD_CUDA(cudaMemcpyAsync(force3, s->force.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s->stream));
    if (mass) MD_CUDA(cudaMemcpyAsync(mass, s->mass.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    if (ids) MD_CUDA(cudaMemcpyAsync(ids, s->ids.p, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, s->stream));
    return sync(s);
}

md_status md_system_reorder(md_system* s, const uint64_t* order) {
    if (!s || (!order && s->n)) return fail(MD_ERR_INVALID, "md_system_reorder: bad arguments");
    MD_TRY(use_system(s));
    const int n = static_cast<int>(s->n);
    if (n == 0) return MD_OK;
    std::vector<uint32_t> o(n);
    std::vector<char> seen(n, 0);
    for (int k = 0; k < n; ++k) {
        if (order[k] >= static_cast<uint64_t>(n) || seen[order[k]]) return fail(MD_ERR_INVALID, "order is not a permutation");
        seen[order[k]] = 1;
        o[k] = static_cast<uint32_t>(order[k]);
    }
    DevBuf<uint32_t> d;
    MD_CUDA(d.reserve(n));
    MD_CUDA(cudaMemcpyAsync(d.p, o.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s->stream));
    MD_CUDA(s->pos2.reserve(n));
    MD_CUDA(s->vel2.reserve(3 * static_cast<size_t>(n)));
    MD_CUDA(s->force2.reserve(3 * static_cast<size_t>(n)));
    MD_CUDA(s->mass2.reserve(n));
    MD_CUDA(s->ids2.reserve(n));
    k_permute<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(d.p, n, s->pos.p, s->vel.p, s->force.p, s->mass.p,
                                                                   s->ids.p, s->pos2.p, s->vel2.p, s->force2.p,
                                                                   s->mass2.p, s->ids2.p, nullptr, nullptr, nullptr);
    MD_CHECK_LAUNCH();
    swap_reordered(s);
    s->layout++;
    return sync(s);
}

md_status md_fcc_lattice(int cells, double a, double* pos4) {
    if (cells < 0 || (!pos4 && cells > 0)) return fail(MD_ERR_INVALID, "md_fcc_lattice: bad arguments");
    // src/Initialisation.cpp:7-44: basis atoms of the cubic cell, offset by a quarter cell
    static constexpr double basis[4][3] = {{0.0, 0.0, 0.0}, {0.5, 0.5, 0.0}, {0.5, 0.0, 0.5}, {0.0, 0.5, 0.5}};
    size_t p = 0;
    for (int ix = 0; ix < cells; ++ix)
        for (int iy = 0; iy < cells; ++iy)
            for (int iz = 0; iz < cells; ++iz)
                for (const auto& b : basis) {
                    pos4[4 * p + 0] = (ix + b[0] + 0.25) * a;
                    pos4[4 * p + 1] = (iy + b[1] + 0.25) * a;
                    pos4[4 * p + 2] = (iz + b[2] + 0.25) * a;
                    pos4[4 * p + 3] = 0.0;
                    ++p;
                }
    return MD_OK;
}

md_status md_initialize_velocities(md_system* s, double temperature, uint32_t seed) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    const size_t n = static_cast<size_t>(s->n);
    std::vector<double> mass(n), vel(3 * n);
    MD_TRY(md_system_download(s, nullptr, nullptr, nullptr, mass.data(), nullptr));
    // src/Initialisation.cpp:47-76: one normal_distribution(0, sqrt(T / m)) per particle, drawn x, y, z
    std::mt19937 rng(seed);
    double momentum[3] = {0.0, 0.0, 0.0};
    double total_mass = 0.0;
    for (size_t i = 0; i < n; ++i) {
        std::normal_distribution<double> dist(0.0, std::sqrt(temperature / mass[i]));
        for (int k = 0; k < 3; ++k) {
            const double v = dist(rng);
            vel[k * n + i] = v;
            momentum[k] += mass[i] * v;
        }
        total_mass += mass[i];
    }
    for (int k = 0; k < 3; ++k)
        for (size_t i = 0; i < n; ++i) vel[k * n + i] -= momentum[k] / total_mass;
    MD_TRY(md_system_upload(s, nullptr, vel.data(), nullptr, nullptr, nullptr));
    return md_rescale_velocities(s, temperature);
}

md_status md_system_stream(md_system* s, void** stream) {
    if (!s || !stream) return fail(MD_ERR_INVALID, "md_system_stream: bad arguments");
    *stream = s->stream;
    return MD_OK;
}

md_status md_system_synchronize(md_system* s) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    MD_TRY(use_system(s));
    return sync(s);
}

md_status md_system_launch_count(const md_system* s, uint64_t* launches) {
    if (!s || !launches) return fail(MD_ERR_INVALID, "md_system_launch_count: bad arguments");
    *launches = s->launches;
    return MD_OK;
}

md_status md_profile_enable(md_system* s, int enable) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    MD_TRY(use_system(s));
    MD_TRY(sync(s));
    s->profile = enable != 0;
    s->events_used = 0;
    s->profile_ms = 0.0;
    s->profile_count = 0;
    return MD_OK;
}

md_status md_profile_read(md_system* s, double* force_ms, int64_t* force_launches) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    MD_TRY(use_system(s));
    MD_TRY(sync(s));
    MD_TRY(profile_collect(s));
    if (force_ms) *force_ms = s->profile_ms;
    if (force_launches) *force_launches = s->profile_count;
    return MD_OK;
}

md_status md_kinetic_energy(md_system* s, double* out) {
    if (!s || !out) return fail(MD_ERR_INVALID, "md_kinetic_energy: bad arguments");
    MD_TRY(use_system(s));
    MD_TRY(kinetic_async(s));
    MD_CUDA(cudaMemcpyAsync(s->host_scal, s->scal.p + kScalKE, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MD_TRY(sync(s));
    *out = s->host_scal[0];
    return MD_OK;
}

md_status md_temperature(md_system* s, double* out) {
    double ke = 0.0;
    MD_TRY(md_kinetic_energy(s, &ke));
    *out = 2.0 * ke / dof_of(s->n);  // src/System.cpp:79-82
    return MD_OK;
}

md_status md_state_hash(md_system* s, uint64_t* out) {
    if (!s || !out) return fail(MD_ERR_INVALID, "md_state_hash: bad arguments");
    const size_t n = static_cast<size_t>(s->n);
    std::vector<double> pos(4 * n), vel(3 * n);
    MD_TRY(md_system_download(s, pos.data(), vel.data(), nullptr, nullptr, nullptr));
    // FNV-1a over (x, vx, y, vy, z, vz) per particle (src/System.cpp:85-105)
    uint64_t h = 14695981039346656037ull;
    auto mix = [&h](double v) {
        uint64_t bits;
        std::memcpy(&bits, &v, 8);
        for (unsigned b = 0; b < 8; ++b) {
            h ^= (bits >> (8u * b)) & 0xffu;
            h *= 1099511628211ull;
        }
    };
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            mix(pos[4 * i + k]);
            mix(vel[k * n + i]);
        }
    *out = h;
    return MD_OK;
}

md_status md_scale_velocities(md_system* s, double scale) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    MD_TRY(use_system(s));
    s->host_scal[kScalFactor] = scale;
    s->host_scal[kScalFactor + 1] = 1.0;
    MD_CUDA(cudaMemcpyAsync(s->scal.p + kScalFactor, s->host_scal + kScalFactor, 2 * sizeof(double),
                            cudaMemcpyHostToDevice, s->stream));
    MD_TRY(scale_async(s));
    return sync(s);
}

md_status md_rescale_velocities(md_system* s, double target) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    MD_TRY(use_system(s));
    MD_TRY(kinetic_async(s));
    k_rescale_factor<<<1, 1, 0, s->stream>>>(s->scal.p + kScalKE, dof_of(s->n), target, s->scal.p + kScalFactor);
    MD_CHECK_LAUNCH();
    MD_TRY(scale_async(s));
    return sync(s);
}

md_status md_bussi_apply(md_system* s, double temperature, double tau, double dt, double r1, double chi2) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    MD_TRY(use_system(s));
    const double c = std::exp(-dt / tau);  // src/Thermostat.cpp:46
    s->host_scal[kScalR1] = r1;
    s->host_scal[kScalR1 + 1] = chi2;
    MD_CUDA(cudaMemcpyAsync(s->scal.p + kScalR1, s->host_scal + kScalR1, 2 * sizeof(double), cudaMemcpyHostToDevice,
                            s->stream));
    MD_TRY(kinetic_async(s));
    k_bussi_factor<<<1, 1, 0, s->stream>>>(s->scal.p + kScalKE, dof_of(s->n), temperature, c, s->scal.p + kScalR1,
                                           s->scal.p + kScalR1 + 1, s->scal.p + kScalFactor);
    MD_CHECK_LAUNCH();
    MD_TRY(scale_async(s));
    return sync(s);
}

md_status md_bussi_noise(uint64_t seed, int64_t n, int64_t count, double* r1, double* chi2) {
    if ((count > 0 && (!r1 || !chi2)) || count < 0 || n < 2) return fail(MD_ERR_INVALID, "md_bussi_noise: bad arguments");
    std::mt19937_64 rng(seed);
    const double dof = dof_of(n);
    for (int64_t k = 0; k < count; ++k) {
        // fresh distributions per call, as BussiThermostat::apply constructs them (src/Thermostat.cpp:48-51)
        std::normal_distribution<double> gaussian(0.0, 1.0);
        std::gamma_distribution<double> gamma(0.5 * (dof - 1.0), 2.0);
        r1[k] = gaussian(rng);
        chi2[k] = gamma(rng);
    }
    return MD_OK;
}

// ---- CellList ----------------------------------------------------------------------------------------------

md_status md_cells_create(double min_cell_size, md_cells** out) {
    if (!out || !(min_cell_size > 0.0)) return fail(MD_ERR_INVALID, "md_cells_create: bad arguments");
    auto* c = new md_cells;
    c->min_size = min_cell_size;
    *out = c;
    return MD_OK;
}

md_status md_cells_destroy(md_cells* c) {
    if (c && c->device >= 0) cudaSetDevice(c->device);
    delete c;
    return MD_OK;
}

md_status md_cells_build(md_cells* c, md_system* s, int* cells_per_side) {
    if (!c || !s) return fail(MD_ERR_INVALID, "md_cells_build: bad arguments");
    MD_TRY(use_system(s));
    c->device = s->device;
    c->n = s->n;
    MD_TRY(cell_sort(c->g, s, c->min_size));
    MD_TRY(sync(s));
    if (cells_per_side) *cells_per_side = c->g.ncps;
    return MD_OK;
}

md_status md_cells_download(md_cells* c, int* particle_cell, uint64_t* cell_start, uint64_t* cell_particles) {
    if (!c || c->device < 0) return fail(MD_ERR_STATE, "cell list not built");
    MD_TRY(use_device(c->device));
    const size_t n = static_cast<size_t>(c->n);
    if (particle_cell && n) MD_CUDA(cudaMemcpy(particle_cell, c->g.cell_of.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    if (cell_start) {
        std::vector<int> st(c->g.ncells + 1);
        MD_CUDA(cudaMemcpy(st.data(), c->g.start.p, sizeof(int) * st.size(), cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < st.size(); ++k) cell_start[k] = static_cast<uint64_t>(st[k]);
    }
    if (cell_particles && n) {
        std::vector<uint32_t> o(n);
        MD_CUDA(cudaMemcpy(o.data(), c->g.order.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < n; ++k) cell_particles[k] = o[k];
    }
    return MD_OK;
}

// ---- NeighbourList -----------------------------------------------------------------------------------------

md_status md_nlist_create(double cutoff, double skin, int reverse_index, md_nlist** out) {
    if (!out || !(cutoff > 0.0) || !(skin >= 0.0)) return fail(MD_ERR_INVALID, "md_nlist_create: bad arguments");
    auto* nl = new md_nlist;
    // src/NeighbourList.cpp:5-8
    nl->rc = cutoff;
    nl->skin = skin;
    nl->rl = cutoff + skin;
    nl->rl2 = (cutoff + skin) * (cutoff + skin);
    nl->max_disp2 = 0.25 * skin * skin;
    nl->reverse = reverse_index != 0;
    *out = nl;
    return MD_OK;
}

md_status md_nlist_destroy(md_nlist* nl) {
    if (nl && nl->device >= 0) cudaSetDevice(nl->device);
    delete nl;
    return MD_OK;
}

md_status md_nlist_build(md_nlist* nl, md_system* s) {
    if (!nl || !s) return fail(MD_ERR_INVALID, "md_nlist_build: bad arguments");
    MD_TRY(use_system(s));
    return nlist_build(nl, s);
}

md_status md_nlist_update(md_nlist* nl, md_system* s, int* rebuilt) {
    if (!nl || !s) return fail(MD_ERR_INVALID, "md_nlist_update: bad arguments");
    MD_TRY(use_system(s));
    bool stale = true;
    // A list never built for this many particles is stale (src/NeighbourList.cpp:14-18)
    if (nl->built && nl->n == s->n && nl->sys == s) {
        const int n = static_cast<int>(s->n);
        MD_CUDA(cudaMemsetAsync(nl->flags.p, 0, sizeof(int), s->stream));
        if (n > 0) {
            k_skin_check<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(s->pos.p, n, s->box, nl->ref_pos.p,
                                                                              nl->max_disp2, nl->flags.p);
            MD_CHECK_LAUNCH();
        }
        int flag = 0;
        MD_CUDA(cudaMemcpyAsync(&flag, nl->flags.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        MD_TRY(sync(s));
        stale = flag != 0;
    }
    if (stale) MD_TRY(nlist_build(nl, s));
    if (rebuilt) *rebuilt = stale ? 1 : 0;
    return MD_OK;
}

md_status md_nlist_info(const md_nlist* nl, uint64_t* pair_count, int* rebuild_count, int* cells_per_side,
                        int* reverse_index) {
    if (!nl) return fail(MD_ERR_INVALID, "null list");
    if (pair_count) {
        if (nl->built) {
            MD_TRY(use_system(const_cast<md_system*>(nl->sys)));
            MD_TRY(ensure_pairs(const_cast<md_nlist*>(nl)));
        }
        *pair_count = nl->pairs;
    }
    if (rebuild_count) *rebuild_count = nl->rebuilds;
    if (cells_per_side) *cells_per_side = nl->grid.ncps;
    if (reverse_index) *reverse_index = nl->reverse ? 1 : 0;
    return MD_OK;
}

md_status md_nlist_set_force_variant(md_nlist* nl, int precision, int variant) {
    if (!nl || precision < MD_PREC_FP64 || precision > MD_PREC_FX32 || variant < -1 || variant > 4 ||
        (precision >= MD_PREC_FX64 && variant >= 1) || (precision == MD_PREC_FP64 && variant >= 3))
        return fail(MD_ERR_INVALID, "md_nlist_set_force_variant: bad arguments");
    nl->pinned[precision] = variant;
    nl->variant[precision] = -1;
    return MD_OK;
}

md_status md_nlist_force_variant(const md_nlist* nl, int precision, int* variant) {
    if (!nl || !variant || precision < MD_PREC_FP64 || precision > MD_PREC_FX32)
        return fail(MD_ERR_INVALID, "md_nlist_force_variant: bad arguments");
    *variant = nl->variant[precision];
    return MD_OK;
}

md_status md_nlist_set_build_variant(md_nlist* nl, int variant) {
    if (!nl || variant < -1 || variant > 1) return fail(MD_ERR_INVALID, "md_nlist_set_build_variant: bad arguments");
    nl->build_pin = variant;
    return MD_OK;
}

md_status md_nlist_build_variant(const md_nlist* nl, int* variant) {
    if (!nl || !variant) return fail(MD_ERR_INVALID, "md_nlist_build_variant: bad arguments");
    *variant = nl->build_kernel;
    return MD_OK;
}

md_status md_nlist_layout(const md_nlist* nl, int* use_tiles, int* segment_cells, int* segments_per_column,
                          int* max_staged, int* row_capacity) {
    if (!nl) return fail(MD_ERR_INVALID, "null list");
    if (use_tiles) *use_tiles = nl->use_tiles ? 1 : 0;
    if (segment_cells) *segment_cells = nl->tiles_geom.kk;
    if (segments_per_column) *segments_per_column = nl->tiles_geom.nseg;
    if (max_staged) *max_staged = nl->tiles_geom.max_staged;
    if (row_capacity) *row_capacity = nl->cap;
    return MD_OK;
}

md_status md_nlist_download(md_nlist* nl, uint64_t* offsets, uint64_t* neighbours, uint64_t* rev_offsets,
                            uint64_t* rev_pairs) {
    if (!nl) return fail(MD_ERR_INVALID, "null list");
    if (!nl->built) return fail(MD_ERR_STATE, "neighbour list not built");
    MD_TRY(use_system(const_cast<md_system*>(nl->sys)));
    MD_TRY(ensure_pairs(nl));
    const int n = static_cast<int>(nl->n);
    cudaStream_t st = nl->sys->stream;
    const size_t P = nl->pairs;
    if (offsets) {
        std::vector<long long> o(n + 1);
        MD_CUDA(cudaMemcpyAsync(o.data(), nl->half_off.p, sizeof(long long) * (n + 1), cudaMemcpyDeviceToHost, st));
        MD_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i <= n; ++i) offsets[i] = static_cast<uint64_t>(o[i]);
    }
    if (neighbours && P) {
        DevBuf<uint64_t> d;
        MD_CUDA(d.reserve(P));
        k_half_csr<<<blocks_for(n, kThreads), kThreads, 0, st>>>(nl->rows.p, n, nl->cap, nl->counts.p, nl->half_off.p, d.p);
        MD_CHECK_LAUNCH();
        MD_CUDA(cudaMemcpyAsync(neighbours, d.p, sizeof(uint64_t) * P, cudaMemcpyDeviceToHost, st));
        MD_CUDA(cudaStreamSynchronize(st));
    }
    if ((rev_offsets || rev_pairs) && nl->reverse) {
        MD_CUDA(nl->rev_off.reserve(n + 1));
        k_rev_counts<<<blocks_for(std::max(n, 1), kThreads), kThreads, 0, st>>>(nl->counts.p, n, nl->tmp_counts.p);
        MD_CHECK_LAUNCH();
        exclusive_scan<int, long long>(nl->tmp_counts.p, n, nl->rev_off.p, nl->tiles.p, st);
        MD_CHECK_SCAN();
        if (rev_offsets) {
            std::vector<long long> o(n + 1);
            MD_CUDA(cudaMemcpyAsync(o.data(), nl->rev_off.p, sizeof(long long) * (n + 1), cudaMemcpyDeviceToHost, st));
            MD_CUDA(cudaStreamSynchronize(st));
            for (int i = 0; i <= n; ++i) rev_offsets[i] = static_cast<uint64_t>(o[i]);
        }
        if (rev_pairs && P) {
            DevBuf<uint64_t> d;
            MD_CUDA(d.reserve(P));
            k_reverse_pairs<<<blocks_for(n, kThreads), kThreads, 0, st>>>(nl->rows.p, n, nl->cap, nl->counts.p,
                                                                          nl->half_off.p, nl->rev_off.p, d.p);
            MD_CHECK_LAUNCH();
            MD_CUDA(cudaMemcpyAsync(rev_pairs, d.p, sizeof(uint64_t) * P, cudaMemcpyDeviceToHost, st));
            MD_CUDA(cudaStreamSynchronize(st));
        }
    }
    MD_CUDA(cudaGetLastError());
    return MD_OK;
}

md_status md_nlist_fx32_rows(md_nlist* nl, uint32_t* near_rows, uint32_t* far_rows, int32_t* groups, double* near2) {
    if (!nl) return fail(MD_ERR_INVALID, "null list");
    if (!nl->built || nl->nf_build != nl->builds || !(nl->nf_near2 > 0.0))
        return fail(MD_ERR_STATE, "md_nlist_fx32_rows: the last build has no MD_PREC_FX32 split (compute its forces first)");
    MD_TRY(use_system(const_cast<md_system*>(nl->sys)));
    const long long n = static_cast<long long>(nl->n);
    const int cap = nl->cap;
    cudaStream_t st = nl->sys->stream;
    if (near2) *near2 = nl->nf_near2;
    // rows_nf: the near rows (capacity kFx32NearCap), then the far rows (capacity cap), both interleaved (entry s
    // of row i at ((i >> 5) * (c >> 2) + (s >> 2)) * 128 + (i & 31) * 4 + (s & 3) for capacity c)
    auto copy_rows = [&](size_t first, int c, uint32_t* out) -> md_status {
        std::vector<uint32_t> raw(row_buffer_entries(n, c));
        if (raw.empty()) return MD_OK;
        MD_CUDA(cudaMemcpyAsync(raw.data(), nl->rows_nf.p + first, sizeof(uint32_t) * raw.size(), cudaMemcpyDeviceToHost, st));
        MD_CUDA(cudaStreamSynchronize(st));
        for (long long i = 0; i < n; ++i)
            for (int s = 0; s < c; ++s)
                out[i * c + s] = raw[((static_cast<size_t>(i >> 5) * (c >> 2) + (s >> 2)) * 32 + (i & 31)) * 4 + (s & 3)];
        return MD_OK;
    };
    if (near_rows) MD_TRY(copy_rows(0, kFx32NearCap, near_rows));
    if (far_rows) MD_TRY(copy_rows(fx32_near_entries(n), cap, far_rows));
    if (groups && n > 0) {
        MD_CUDA(cudaMemcpyAsync(groups, nl->counts_nf.p, sizeof(int2) * n, cudaMemcpyDeviceToHost, st));
        MD_CUDA(cudaStreamSynchronize(st));
    }
    return MD_OK;
}

// ---- LennardJonesForceField --------------------------------------------------------------------------------

md_status md_forcefield_create(double epsilon, double sigma, double cutoff, md_forcefield** out) {
    if (!out || !(cutoff > 0.0)) return fail(MD_ERR_INVALID, "md_forcefield_create: bad arguments");
    auto* ff = new md_forcefield;
    ff->eps = epsilon;
    ff->sigma = sigma;
    ff->rc = cutoff;
    ff->lj = lj_constants(epsilon, sigma, cutoff);
    *out = ff;
    return MD_OK;
}

md_status md_forcefield_destroy(md_forcefield* ff) {
    if (ff && ff->device >= 0) cudaSetDevice(ff->device);
    if (ff && ff->host_out) cudaFreeHost(ff->host_out);
    if (ff && ff->side) {
        cudaStreamSynchronize(ff->side);
        cudaStreamSynchronize(ff->chain);
        for (cudaEvent_t e : {ff->ev_force, ff->ev_done, ff->ev_read[0], ff->ev_read[1], ff->ev_chain[0], ff->ev_chain[1]})
            if (e) cudaEventDestroy(e);
        cudaStreamDestroy(ff->side);
        cudaStreamDestroy(ff->chain);
    }
    delete ff;
    return MD_OK;
}

md_status md_forcefield_shift(const md_forcefield* ff, double* shift) {
    if (!ff || !shift) return fail(MD_ERR_INVALID, "md_forcefield_shift: bad arguments");
    *shift = ff->lj.shift;
    return MD_OK;
}

md_status md_forcefield_set_precision(md_forcefield* ff, int precision) {
    if (!ff || precision < MD_PREC_FP64 || precision > MD_PREC_FX32) return fail(MD_ERR_INVALID, "bad precision");
    ff->precision = precision;
    return MD_OK;
}

md_status md_forcefield_set_deterministic(md_forcefield* ff, int deterministic) {
    if (!ff) return fail(MD_ERR_INVALID, "null force field");
    ff->deterministic = deterministic != 0;
    return MD_OK;
}

md_status md_forces_list(md_forcefield* ff, md_system* s, md_nlist* nl, double* pe, double* virial, double* inside) {
    if (!ff || !s || !nl) return fail(MD_ERR_INVALID, "md_forces_list: bad arguments");
    MD_TRY(use_system(s));
    MD_TRY(check_cutoff(ff, s));
    if (ff->deterministic && !nl->reverse)
        return fail(MD_ERR_NO_REVERSE_INDEX, "Deterministic forces need a NeighbourList built with reverseIndex = true");
    if (!nlist_current(nl, s)) return fail(MD_ERR_STATE, "the neighbour list was not built for this system's current order");
    ff->device = s->device;
    MD_TRY(forces_list_async(ff, s, nl, true));
    return read_energy(ff, s, pe, virial, inside);
}

md_status md_forcefield_results(const md_forcefield* ff, double* virial, double* inside) {
    if (!ff) return fail(MD_ERR_INVALID, "null force field");
    if (virial) *virial = ff->virial;
    if (inside) *inside = ff->inside;
    return MD_OK;
}

md_status md_forces_all_pairs(md_forcefield* ff, md_system* s, double* pe, double* virial, double* inside) {
    if (!ff || !s) return fail(MD_ERR_INVALID, "md_forces_all_pairs: bad arguments");
    MD_TRY(use_system(s));
    MD_TRY(check_cutoff(ff, s));
    ff->device = s->device;
    const int n = static_cast<int>(s->n);
    MD_TRY(join_energy(ff, s));
    MD_CUDA(ff->out.reserve(4));
    if (n > 0) {
        k_force_all_pairs<<<blocks_for(n, 128), 128, 0, s->stream>>>(s->pos.p, n, s->box, ff->lj, s->force.p);
        MD_CHECK_LAUNCH();
        k_energy_all_pairs<<<1, 32, 0, s->stream>>>(s->pos.p, n, s->box, ff->lj, ff->out.p);
        MD_CHECK_LAUNCH();
    } else {
        MD_CUDA(cudaMemsetAsync(ff->out.p, 0, 3 * sizeof(double), s->stream));
    }
    double out[3];
    MD_CUDA(cudaMemcpyAsync(out, ff->out.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MD_TRY(sync(s));
    ff->virial = out[1];
    ff->inside = out[2];
    if (pe) *pe = out[0];
    if (virial) *virial = out[1];
    if (inside) *inside = out[2];
    return MD_OK;
}

// ---- VelocityVerletIntegrator ------------------------------------------------------------------------------

md_status md_step_list(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, double* pe, int* rebuilt) {
    if (!s || !ff || !nl) return fail(MD_ERR_INVALID, "md_step_list: bad arguments");
    MD_TRY(use_system(s));
    MD_TRY(check_cutoff(ff, s));
    if (ff->deterministic && !nl->reverse)
        return fail(MD_ERR_NO_REVERSE_INDEX, "Deterministic forces need a NeighbourList built with reverseIndex = true");
    ff->device = s->device;
    bool stale = true;
    MD_TRY(drift_and_update(s, ff, nl, dt, &stale));
    if (rebuilt) *rebuilt = stale ? 1 : 0;
    MD_TRY(forces_list_async(ff, s, nl, true, dt, true));
    return read_energy(ff, s, pe, nullptr, nullptr);
}

md_status md_step_all_pairs(md_system* s, md_forcefield* ff, double dt, double* pe) {
    if (!s || !ff) return fail(MD_ERR_INVALID, "md_step_all_pairs: bad arguments");
    MD_TRY(use_system(s));
    MD_TRY(check_cutoff(ff, s));
    MD_TRY(kick_drift_async(s, nullptr, dt, false));
    MD_TRY(md_forces_all_pairs(ff, s, pe, nullptr, nullptr));
    MD_TRY(kick_async(s, dt));
    return sync(s);
}

// ---- RadialDistribution --------------------------------------------------------------------------------------

md_status md_rdf_create(double r_max, int bins, md_rdf** out) {
    if (!out || !(r_max > 0.0) || bins <= 0 || bins > (1 << 20)) return fail(MD_ERR_INVALID, "md_rdf_create: bad arguments");
    auto* r = new md_rdf;
    r->rmax = r_max;
    r->bins = bins;
    r->bin_width = r_max / bins;  // src/RadialDistribution.cpp:6-7
    *out = r;
    return MD_OK;
}

md_status md_rdf_destroy(md_rdf* r) {
    if (r && r->device >= 0) cudaSetDevice(r->device);
    delete r;
    return MD_OK;
}

md_status md_rdf_sample(md_rdf* r, md_system* s, md_nlist* nl) {
    if (!r || !s || !nl) return fail(MD_ERR_INVALID, "md_rdf_sample: bad arguments");
    MD_TRY(use_system(s));
    if (!nlist_current(nl, s)) return fail(MD_ERR_STATE, "the neighbour list was not built for this system's current order");
    if (r->device >= 0 && r->device != s->device) return fail(MD_ERR_INVALID, "histogram lives on another device");
    MD_TRY(rdf_sample_async(r, s, nl));
    return sync(s);
}

md_status md_rdf_histogram(md_rdf* r, double* hist) {
    if (!r || !hist) return fail(MD_ERR_INVALID, "md_rdf_histogram: bad arguments");
    if (r->device < 0) {
        for (int b = 0; b < r->bins; ++b) hist[b] = 0.0;
        return MD_OK;
    }
    MD_TRY(use_device(r->device));
    std::vector<unsigned long long> h(r->bins);
    MD_CUDA(cudaMemcpy(h.data(), r->hist.p, sizeof(unsigned long long) * r->bins, cudaMemcpyDeviceToHost));
    for (int b = 0; b < r->bins; ++b) hist[b] = static_cast<double>(h[b]);
    return MD_OK;
}

md_status md_rdf_values(md_rdf* r, double* radii, double* g, int* samples) {
    if (!r) return fail(MD_ERR_INVALID, "null rdf");
    std::vector<double> h(r->bins);
    MD_TRY(md_rdf_histogram(r, h.data()));
    for (int b = 0; b < r->bins; ++b) {
        if (radii) radii[b] = (static_cast<double>(b) + 0.5) * r->bin_width;  // src/RadialDistribution.cpp:32-38
        if (g) {
            if (r->samples == 0) {
                g[b] = 0.0;
                continue;
            }
            // src/RadialDistribution.cpp:42-54
            const double lo = static_cast<double>(b) * r->bin_width;
            const double hi = lo + r->bin_width;
            const double shell = 4.0 / 3.0 * 3.14159265358979323846 * (hi * hi * hi - lo * lo * lo);
            g[b] = h[b] / (r->samples * 0.5 * r->particles * r->density * shell);
        }
    }
    if (samples) *samples = r->samples;
    return MD_OK;
}

// ---- device-resident run -------------------------------------------------------------------------------------

md_status md_run(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps, const md_run_options* opts,
                 double* pe, double* ke, double* virial) {
    if (!s || !ff || !nl || n_steps < 0) return fail(MD_ERR_INVALID, "md_run: bad arguments");
    MD_TRY(use_system(s));
    MD_TRY(check_cutoff(ff, s));
    if (ff->deterministic && !nl->reverse)
        return fail(MD_ERR_NO_REVERSE_INDEX, "Deterministic forces need a NeighbourList built with reverseIndex = true");
    md_run_options o{};
    if (opts) o = *opts;
    if (o.thermostat == 2 && n_steps > 0 && (!o.bussi_r1 || !o.bussi_chi2))
        return fail(MD_ERR_INVALID, "Bussi run needs r1 and chi2 draws");
    if (o.thermostat == 1 && o.rescale_every <= 0) return fail(MD_ERR_INVALID, "rescale_every must be positive");
    if (o.rdf && o.rdf_every <= 0) return fail(MD_ERR_INVALID, "rdf_every must be positive");
    ff->device = s->device;
    return run_steps(s, ff, nl, dt, n_steps, o, pe, ke, virial);
}

md_status md_run_prepare(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps,
                         const md_run_options* opts, int record) {
    if (!s || !ff || !nl || n_steps < 0) return fail(MD_ERR_INVALID, "md_run_prepare: bad arguments");
    MD_TRY(use_system(s));
    MD_TRY(check_cutoff(ff, s));
    md_run_options o{};
    if (opts) o = *opts;
    if (o.thermostat == 1 && o.rescale_every <= 0) return fail(MD_ERR_INVALID, "rescale_every must be positive");
    if (o.rdf && o.rdf_every <= 0) return fail(MD_ERR_INVALID, "rdf_every must be positive");
    ff->device = s->device;
    if (!graph_mode_ok(s, ff, nl, n_steps)) return MD_OK;  // md_run would take the host path: nothing to prepare
    MD_TRY(graph_prepare(s, ff, nl, dt, n_steps, o, (record & 1) != 0, (record & 2) != 0));
    s->prepared_steps = n_steps;
    return sync(s);
}

md_status md_system_set_graph(md_system* s, int chunk_steps, int flags) {
    if (!s || chunk_steps < 0 || chunk_steps > 1024 || (flags & ~MD_GRAPH_TEST_RERUN))
        return fail(MD_ERR_INVALID, "md_system_set_graph: bad arguments");
    MD_TRY(use_system(s));
    MD_TRY(sync(s));
    drop_run_graphs(s);
    s->graph_chunk = chunk_steps;
    s->graph_flags = flags;
    return MD_OK;
}

md_status md_system_graph_info(const md_system* s, int* chunk_steps, uint64_t* graphs, uint64_t* launches,
                               uint64_t* recoveries) {
    if (!s) return fail(MD_ERR_INVALID, "null system");
    if (chunk_steps) *chunk_steps = s->graph_chunk;
    if (graphs) *graphs = s->graphs.size();
    if (launches) *launches = s->graph_launches;
    if (recoveries) *recoveries = s->graph_recoveries;
    return MD_OK;
}

}  // extern "C"

// ---- kinetic energy without allocation ---------------------------------------------------------------------
//
// For callers that own every byte of device memory themselves and may not allocate: an embedding runtime
// with its own pool, or a process that must not call cudaMalloc/cudaFree once running. The block partial
// sums live in this fixed array instead of an allocation. Every GPU that loads the library holds it (256 KB)
// until the process exits.
namespace {

constexpr int64_t kNoAllocMaxBlocks = 16384;  // 1024-particle blocks: up to 16,777,216 particles
// kNoAllocMaxBlocks block partials, then one slot for the result
static __device__ __align__(256) double2 g_noalloc_ke_blocks[kNoAllocMaxBlocks + 1];

// Host code must not take g_noalloc_ke_blocks' address directly (it names a host-side shadow): the device
// address comes from cudaGetSymbolAddress, once per device, with that device current. The address is kept
// with the context it was looked up in: after a device reset the primary context is a new one, the module is
// loaded again at another address, and the address is looked up again.
constexpr int kNoAllocMaxDevices = 64;
struct NoAllocScratch {
    void* context = nullptr;  // CUcontext current when ptr was looked up
    double2* ptr = nullptr;
};
NoAllocScratch g_noalloc[kNoAllocMaxDevices] = {};
std::mutex g_noalloc_mutex;

// The calling thread's current CUcontext, through the runtime's driver entry point (no link against libcuda)
md_status current_context(void** ctx) {
    using GetCurrent = int (*)(void**);
    static GetCurrent get = nullptr;
    if (!get) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        MD_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q));
        if (!fn || q != cudaDriverEntryPointSuccess) return fail(MD_ERR_CUDA, "cuCtxGetCurrent is unavailable");
        get = reinterpret_cast<GetCurrent>(fn);
    }
    *ctx = nullptr;
    if (get(ctx) != 0) return fail(MD_ERR_CUDA, "cuCtxGetCurrent failed");
    return MD_OK;
}

md_status noalloc_scratch(int device, double2** out) {
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(MD_ERR_INVALID, "device index out of range");
    // NULL until the runtime has made the device's primary context current on this thread, which the
    // symbol lookup below does
    void* ctx = nullptr;
    MD_TRY(current_context(&ctx));
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoAllocScratch& e = g_noalloc[device];
    if (!e.ptr || !ctx || e.context != ctx) {
        void* p = nullptr;
        MD_CUDA(cudaGetSymbolAddress(&p, g_noalloc_ke_blocks));
        MD_TRY(current_context(&ctx));
        e.ptr = static_cast<double2*>(p);
        e.context = ctx;
    }
    *out = e.ptr;
    return MD_OK;
}

}  // namespace

extern "C" md_status md_kinetic_energy_noalloc(const double* vel3, const double* mass, int64_t n, double* out,
                                               void* stream) {
    if (n < 0 || (n > 0 && (!vel3 || !mass)) || !out) return fail(MD_ERR_INVALID, "md_kinetic_energy_noalloc: bad arguments");
    const int64_t nb = (n + kChunk - 1) / kChunk;
    if (nb > kNoAllocMaxBlocks)
        return fail(MD_ERR_INVALID, "md_kinetic_energy_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
                                        std::to_string(kNoAllocMaxBlocks * kChunk) + " particles");
    int device = 0;
    MD_CUDA(cudaGetDevice(&device));
    double2* scratch = nullptr;
    MD_TRY(noalloc_scratch(device, &scratch));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    g_launches = nullptr;
    double* result = reinterpret_cast<double*>(scratch + kNoAllocMaxBlocks);
    // Every block partial that the sum reads is written first by k_kinetic_blocks, and the result slot is
    // written whole by k_sum_blocks, so nothing left by an earlier call is read and nothing needs clearing.
    if (nb > 0) {
        const size_t smem = kEnergyWarps * kChunk * sizeof(double);
        k_kinetic_blocks<<<blocks_for(nb, kEnergyWarps), kEnergyWarps * 32, smem, st>>>(
            vel3, mass, static_cast<int>(n), scratch, static_cast<int>(nb));
        MD_CHECK_LAUNCH();
    }
    // (sum of the .x partials, sum of the .y partials) into the result slot; .x is the kinetic energy
    k_sum_blocks<<<1, 32, 0, st>>>(scratch, static_cast<int>(nb), result);
    MD_CHECK_LAUNCH();
    MD_CUDA(cudaMemcpyAsync(out, result, sizeof(double), cudaMemcpyDeviceToDevice, st));
    return MD_OK;
}

#include "md_batch.inl"
#include "md_adjoint.inl"
