// Shared-memory cell tiles for the list build and the list force kernels (boxes of at least 3 cells per side).
//
// Work decomposition: one thread block per "segment" = kk consecutive cells along z of one (x, y) cell
// column. The block stages into shared memory every particle its home atoms can pair with: the 9 columns
// (x + dx, y + dy), dx, dy in {-1, 0, 1}, over the z cells [z0 - 1, z0 + kk], wrapped periodically. Cells are
// sorted x-major, so each staged column is one or two contiguous particle ranges and the home atoms are one
// contiguous range. Pair gathers then come from shared memory instead of scattered global loads.
//
// Row entries keep global indices (j | code << 27). Inside a block, particle j of the staged cell that code
// names, relative to a home atom at z offset t, sits at shared slot j + delta[t][code]; a per-block table
// holds that delta together with the cell's float image offset -d * cell.
//
// Rows are stored "uint4-interleaved" per group of 32 consecutive particles: the 4 entries [4q, 4q + 4) of
// particle i are the uint4 at ((i >> 5) * cap / 4 + q) * 32 + (i & 31), so a warp reading one uint4 per lane
// touches 512 contiguous bytes.
#pragma once

#include "md_common.cuh"
#include "md_fp32.cuh"
#include "md_fp64.cuh"

namespace md {

constexpr int kTileThreads = 128;
#ifndef MD_TILE_MAX_SEGMENT
#define MD_TILE_MAX_SEGMENT 10
#endif
constexpr int kMaxSegment = MD_TILE_MAX_SEGMENT;     // kk <= kMaxSegment cells per segment
constexpr int kMaxStagedCells = 9 * (kMaxSegment + 2);
constexpr int kScanPerLane = (kMaxStagedCells + 31) / 32;  // staged-cell counts per lane in tile_tables' scan
struct TileGeom {
    int ncps;       // cells per side (>= 3)
    int kk;         // cells per segment along z
    int nseg;       // segments per column = ceil(ncps / kk)
    int max_staged; // bound on staged particles per block (shared slots; one more holds the sentinel)
    double cell;    // cell side L / ncps
    Box box;
};

// ---- staging tables --------------------------------------------------------------------------------------

struct TileTables {
    int ncell;                    // staged cells: 9 * (kk + 2)
    int gstart[kMaxStagedCells];  // first particle of each staged cell
    int count[kMaxStagedCells];
    int off[kMaxStagedCells];     // its first shared slot
    int total;                    // staged particles
    int z0, kk;                   // home z range [z0, z0 + kk)
    int cx, cy;
    int home_begin, home_end;     // home particles [home_begin, home_end)
};

// Fills the staged-cell table of this block: one thread per staged cell reads its range, warp 0 turns the
// counts into shared-memory offsets. Ends with __syncthreads.
__device__ __forceinline__ void tile_tables(const TileGeom& g, const int* __restrict__ cell_start, TileTables& t) {
    const int n = g.ncps;
    const int seg = blockIdx.x % g.nseg;
    const int col = blockIdx.x / g.nseg;
    const int cx = col / n, cy = col % n, z0 = seg * g.kk;
    const int kk = min(g.kk, n - z0);
    const int span = kk + 2;
    const int ncell = 9 * span;
    for (int k = threadIdx.x; k < ncell; k += blockDim.x) {
        const int c = k / span, u = k % span;
        const int x = (cx + c / 3 - 1 + n) % n;
        const int y = (cy + c % 3 - 1 + n) % n;
        const int z = (z0 - 1 + u + n) % n;
        const int cell = (x * n + y) * n + z;
        const int s = cell_start[cell];
        t.gstart[k] = s;
        t.count[k] = cell_start[cell + 1] - s;
    }
    if (threadIdx.x == 0) {
        t.cx = cx;
        t.cy = cy;
        t.z0 = z0;
        t.kk = kk;
        t.ncell = ncell;
        const int hc0 = (cx * n + cy) * n + z0;
        t.home_begin = cell_start[hc0];
        t.home_end = cell_start[hc0 + kk];
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // exclusive scan of up to kMaxStagedCells counts, kScanPerLane per lane
        const int lane = threadIdx.x;
        int v[kScanPerLane], s = 0;
#pragma unroll
        for (int q = 0; q < kScanPerLane; ++q) {
            const int k = lane * kScanPerLane + q;
            v[q] = k < ncell ? t.count[k] : 0;
            s += v[q];
        }
        int inc = s;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        int run = inc - s;
#pragma unroll
        for (int q = 0; q < kScanPerLane; ++q) {
            const int k = lane * kScanPerLane + q;
            if (k < ncell) t.off[k] = run;
            run += v[q];
        }
        if (lane == 31) t.total = inc;
    }
    __syncthreads();
}

// Copy every staged cell's particles into shared memory with asynchronous 16-byte copies (cp.async), so all of
// a block's loads are in flight at once; warps take cells in turn. The caller waits (cp_async_wait) and
// synchronises before reading the tile.
template <typename T>
__device__ __forceinline__ void stage_tile(const T* __restrict__ src, T* dst, const TileTables& t) {
    static_assert(sizeof(T) % 16 == 0, "staged records are whole 16-byte units");
    constexpr int kUnits = sizeof(T) / 16;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int k = warp; k < t.ncell; k += nwarps) {
        const char* g = reinterpret_cast<const char*>(src + t.gstart[k]);
        const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst + t.off[k]));
        for (int u = lane; u < t.count[k] * kUnits; u += 32)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s + 16u * u), "l"(g + 16 * u) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Largest staged particle count over all segments of this geometry (one thread per segment); sizes the
// shared tile until the next rebuild, since the cell contents only change at rebuilds.
__global__ void k_tile_max_staged(const int* __restrict__ cell_start, TileGeom g, int* __restrict__ out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = g.ncps;
    if (b >= n * n * g.nseg) return;
    const int seg = b % g.nseg, col = b / g.nseg;
    const int cx = col / n, cy = col % n, z0 = seg * g.kk;
    const int span = min(g.kk, n - z0) + 2;
    int total = 0;
    for (int c = 0; c < 9; ++c) {
        const int x = (cx + c / 3 - 1 + n) % n, y = (cy + c % 3 - 1 + n) % n;
        for (int u = 0; u < span; ++u) {
            const int cell = (x * n + y) * n + (z0 - 1 + u + n) % n;
            total += cell_start[cell + 1] - cell_start[cell];
        }
    }
    atomicMax(out, total);
}

// Staged cell of code (dx, dy, dz) seen from home z offset h (0-based in the segment)
__device__ __forceinline__ int staged_cell(int code, int h, int span) {
    const int dxy = code / 3;        // (dx + 1) * 3 + (dy + 1)
    const int dz = code % 3 - 1;
    return dxy * span + h + 1 + dz;
}

// ---- list build -------------------------------------------------------------------------------------------

// NeighbourList::build pass 1 (src/NeighbourList.cpp:75-111) on a tile. Candidates come from staged float
// frames; a candidate is accepted when float r^2 < r_l^2 - margin, rejected when float r^2 > r_l^2 + margin,
// and otherwise decided by the reference's exact double test on the global positions (a thin shell of
// candidates). margin bounds the float error of r^2 (frames are within 1.6 cells' half width of their cell
// centre, so each coordinate carries under 4e-7 absolute error), which keeps the list bit-identical.
// Row order: own pairs (j > i) in the reference's candidate order, then the j < i that list i, ascending.
struct BuildParams {
    double rl2;
    float rl2_lo, rl2_hi;  // (r_l^2 - margin, r_l^2 + margin) in float
    int cap;
    uint32_t sentinel;     // index of the sentinel particle (n)
};

// The reference's list test in double (src/NeighbourList.cpp:38-52), kept out of line: only candidates within
// float rounding of r_l reach it
__device__ __noinline__ bool exact_within(const double4& pi, const double4& pj, const Box& box, double rl2) {
    const double ex = min_image(dsub(pi.x, pj.x), box);
    const double ey = min_image(dsub(pi.y, pj.y), box);
    const double ez = min_image(dsub(pi.z, pj.z), box);
    return norm2(ex, ey, ez) < rl2;
}

// The exact pass of scan_cell: candidates [u0, u1) decided as the float scan does, except those in the thin shell,
// which the reference's double test decides; appended from the row length cnt on
__device__ __noinline__ void rescan_cell_exact(const float4* q, int jbase, int u0, int u1, const float4 qo,
                                               uint32_t code, float lo, float hi, double rl2, int cap,
                                               const double4 pi, const double4* __restrict__ pos, const Box box,
                                               uint32_t* row, int& cnt) {
    for (int u = u0; u < u1; ++u) {
        const float4 qj = q[u];
        const float dx = qo.x - qj.x;
        const float dy = qo.y - qj.y;
        const float dz = qo.z - qj.z;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        bool take = r2 < lo;
        if (!take && r2 <= hi) take = exact_within(pi, pos[jbase + u], box, rl2);
        if (take) {
            if (cnt < cap) row[(cnt >> 2) * 128 + (cnt & 3)] = static_cast<uint32_t>(jbase + u) | (code << kCodeShift);
            ++cnt;
        }
    }
}

// Appends to a row the candidates u in [u0, u1) of one cell that are within r_l of particle i: candidate u has
// the float frame q[u] and the index jbase + u, qo = q_i + the cell's image offset (the margin covers the
// rounding of that hoisted sum), row is particle i's interleaved row (entry s at row[(s >> 2) * 128 + (s & 3)])
// and cnt its length. The loop runs branch-free: a candidate whose float r^2 is below lo = r_l^2 - margin is
// appended with a predicated store, one above hi = r_l^2 + margin is dropped. If any candidate of the cell falls
// in the thin shell between, the cell is scanned again from its first slot with the reference's exact double
// test (src/NeighbourList.cpp:38-52) deciding the shell, rewriting the same slots. Entries past cap are counted
// and not written. kOutOfLine keeps that re-scan in a separate function (fewer registers in the tiled build's
// loop; the batch build is faster with it inline).
template <bool kOutOfLine>
__device__ __forceinline__ void scan_cell(const float4* q, int jbase, int u0, int u1, const float4& qo, uint32_t code,
                                          float lo, float hi, double rl2, int cap, const double4& pi,
                                          const double4* __restrict__ pos, const Box& box, uint32_t* row, int& cnt) {
    const int cnt0 = cnt;
    bool shell = false;
    const uint32_t vbase = static_cast<uint32_t>(jbase) | (code << kCodeShift);  // entry of candidate u: vbase + u
    // q_j - qo: the negation of qo - q_j in every bit (round-to-nearest is symmetric), x and y in one packed add
    const float2 nxy = make_float2(-qo.x, -qo.y);
    const float nz = -qo.z;
    if (cnt + (u1 - u0) <= cap) {  // every candidate fits: no capacity test per candidate
        for (int u = u0; u < u1; ++u) {
            const float4 qj = q[u];
            const float2 d = __fadd2_rn(make_float2(qj.x, qj.y), nxy);
            const float dz = __fadd_rn(qj.z, nz);
            const float r2 = fmaf(d.x, d.x, fmaf(d.y, d.y, dz * dz));
            const bool take = r2 < lo;
            shell |= !take && r2 <= hi;
            uint32_t* p = row + (cnt + 31 * (cnt & ~3));  // (cnt >> 2) * 128 + (cnt & 3)
            asm volatile("{\n\t.reg .pred t;\n\tsetp.ne.u32 t, %2, 0;\n\t@t st.global.u32 [%0], %1;\n\t}"
                         :: "l"(p), "r"(vbase + static_cast<uint32_t>(u)), "r"(static_cast<unsigned>(take)) : "memory");
            cnt += take ? 1 : 0;
        }
    } else {
        for (int u = u0; u < u1; ++u) {
            const float4 qj = q[u];
            const float2 d = __fadd2_rn(make_float2(qj.x, qj.y), nxy);
            const float dz = __fadd_rn(qj.z, nz);
            const float r2 = fmaf(d.x, d.x, fmaf(d.y, d.y, dz * dz));
            const bool take = r2 < lo;
            shell |= !take && r2 <= hi;
            if (take && cnt < cap) row[(cnt >> 2) * 128 + (cnt & 3)] = vbase + static_cast<uint32_t>(u);
            cnt += take ? 1 : 0;
        }
    }
    if (shell) {
        cnt = cnt0;
        if (kOutOfLine) {
            rescan_cell_exact(q, jbase, u0, u1, qo, code, lo, hi, rl2, cap, pi, pos, box, row, cnt);
        } else {
            for (int u = u0; u < u1; ++u) {
                const float4 qj = q[u];
                const float dx = qo.x - qj.x;
                const float dy = qo.y - qj.y;
                const float dz = qo.z - qj.z;
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                bool take = r2 < lo;
                if (!take && r2 <= hi) take = exact_within(pi, pos[jbase + u], box, rl2);
                if (take) {
                    if (cnt < cap) row[(cnt >> 2) * 128 + (cnt & 3)] = static_cast<uint32_t>(jbase + u) | (code << kCodeShift);
                    ++cnt;
                }
            }
        }
    }
}

__global__ void __launch_bounds__(kTileThreads) k_nlist_build_tile(
    const float4* __restrict__ frames, const double4* __restrict__ pos, const int* __restrict__ cell_start,
    const int* __restrict__ cell_sorted, TileGeom g, BuildParams bp, CellOffsets offs, uint32_t* __restrict__ rows,
    int2* __restrict__ counts, int* __restrict__ max_count) {
    extern __shared__ float4 s_q[];
    __shared__ TileTables t;
    tile_tables(g, cell_start, t);
    if (t.total > g.max_staged) {  // the host's bound was wrong: report a full row so it rebuilds bigger
        if (threadIdx.x == 0) atomicMax(max_count, 1 << 30);
        return;
    }
    stage_tile(frames, s_q, t);
    cp_async_wait();
    __syncthreads();
    const int n = g.ncps;
    const int span = t.kk + 2;
    for (int i = t.home_begin + threadIdx.x; i < t.home_end; i += blockDim.x) {
        const float4 qi = frames[i];
        const double4 pi = pos[i];
        const int z = cell_sorted[i] % n;
        const int h = (z - t.z0 + n) % n;
        int cnt = 0;
        // this particle's interleaved row: entry s at row[(s >> 2) * 128 + (s & 3)]
        uint32_t* row = rows + static_cast<size_t>(i >> 5) * (bp.cap >> 2) * 128 + (i & 31) * 4;
        auto scan = [&](const float4* q, int gs, int u0, int u1, const float4& qo, uint32_t code) {
            scan_cell<true>(q, gs, u0, u1, qo, code, bp.rl2_lo, bp.rl2_hi, bp.rl2, bp.cap, pi, pos, g.box, row, cnt);
        };
        // own pairs: 27 cells in (dx, dy, dz) order, increasing j inside each (src/CellList.cpp:55-83)
        for (uint32_t code = 0; code < 27; ++code) {
            const int sc = staged_cell(static_cast<int>(code), h, span);
            const float4 o = offs.off[code];
            const float4 qo = make_float4(qi.x + o.x, qi.y + o.y, qi.z + o.z, 0.0f);
            const int gs = t.gstart[sc];
            scan(s_q + t.off[sc], gs, max(0, i + 1 - gs), t.count[sc], qo, code);
        }
        const int own = cnt;
        // the j < i that list i, increasing j: cells in increasing cell id
        const int cx = t.cx, cy = t.cy;
        int ox[3], oy[3], oz[3];
        auto asc = [n](int c, int* d) {
            if (c == 0) { d[0] = 0; d[1] = 1; d[2] = -1; }
            else if (c == n - 1) { d[0] = 1; d[1] = -1; d[2] = 0; }
            else { d[0] = -1; d[1] = 0; d[2] = 1; }
        };
        asc(cx, ox);
        asc(cy, oy);
        asc(z, oz);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int d = 0; d < 3; ++d) {
                    const uint32_t code = (ox[a] + 1) * 9 + (oy[b] + 1) * 3 + (oz[d] + 1);
                    const int sc = staged_cell(static_cast<int>(code), h, span);
                    const float4 o = offs.off[code];
                    const float4 qo = make_float4(qi.x + o.x, qi.y + o.y, qi.z + o.z, 0.0f);
                    const int gs = t.gstart[sc];
                    scan(s_q + t.off[sc], gs, 0, min(t.count[sc], i - gs), qo, code);
                }
        // a row past the capacity keeps counts within it (the entries written), so kernels that read the rows
        // before the host sees max_count stay in bounds; max_count reports the full length
        const int own_c = min(own, bp.cap), cnt_c = min(cnt, bp.cap);
        counts[i] = make_int2(own_c, cnt_c - own_c);
        const int padded = (cnt + 7) & ~7;
        for (int s = cnt; s < padded && s < bp.cap; ++s) row[(s >> 2) * 128 + (s & 3)] = bp.sentinel | (kSentinelCode << kCodeShift);
        atomicMax(max_count, padded);
    }
}

// ---- float forces -----------------------------------------------------------------------------------------

// Per-block table entry for (home z offset, code): image offset -d * cell in x, y, z and the shared slot delta
// (as int bits) of the staged cell that code names.
template <bool kFixed, bool kEnergy>
__global__ void __launch_bounds__(kTileThreads) k_force_fp32_tile(
    const float4* __restrict__ frames, const double4* __restrict__ pos, int n_atoms, const int* __restrict__ cell_start,
    const int* __restrict__ cell_sorted, TileGeom g, FloatLJ lj, CellOffsets offs, const uint32_t* __restrict__ rows,
    int cap, const int2* __restrict__ counts, double* __restrict__ force, unsigned long long* __restrict__ acc,
    KickArgs kick) {
    extern __shared__ float4 s_q[];
    __shared__ TileTables t;
    __shared__ float4 s_tab[kMaxSegment][32];
    if (kick.frames_out && blockIdx.x == 0 && threadIdx.x == 0)
        kick.frames_out[n_atoms] = make_float4(kSentinelCoord, kSentinelCoord, kSentinelCoord, 0.0f);
    tile_tables(g, cell_start, t);
    const int span = t.kk + 2;
    const int sentinel_slot = g.max_staged;
    if (t.total > g.max_staged) {  // the bound recorded in a graph was outgrown: the host reruns the chunk
        if (kick.overflow && threadIdx.x == 0) *kick.overflow = 1;
        return;
    }
    stage_tile(frames, s_q, t);
    if (threadIdx.x == 0) s_q[sentinel_slot] = make_float4(kSentinelCoord, kSentinelCoord, kSentinelCoord, 0.f);
    for (int e = threadIdx.x; e < t.kk * 32; e += blockDim.x) {
        const int h = e / 32, code = e % 32;
        float4 o;
        int delta;
        if (code < 27) {
            const int sc = staged_cell(code, h, span);
            o = offs.off[code];
            delta = t.off[sc] - t.gstart[sc];
        } else {
            o = make_float4(0.f, 0.f, 0.f, 0.f);
            delta = sentinel_slot - n_atoms;  // the sentinel entry is j = n_atoms
        }
        o.w = __int_as_float(delta);
        s_tab[h][code] = o;
    }
    cp_async_wait();
    __syncthreads();
    long long e_fx = 0, w_fx = 0, k_fx = 0;
    unsigned ins = 0;
    const int n = g.ncps;
    for (int i = t.home_begin + threadIdx.x; i < t.home_end; i += blockDim.x) {
        const int h = (cell_sorted[i] % n - t.z0 + n) % n;
        const float4* tab = s_tab[h];
        const float4 qi = frames[i];
        const int2 c = counts[i];
        const int groups = (c.x + c.y + 7) >> 3;  // rows are padded with sentinels to a multiple of 8
        FloatAcc<kFixed, kEnergy> a;
        for (int gi = 0; gi < groups; ++gi) {
            const uint4 e0 = row_quad(rows, i, 2 * gi, cap);
            const uint4 e1 = row_quad(rows, i, 2 * gi + 1, cap);
            const float4* sq = s_q;
            const Box box = g.box;
            const GroupSums gs = float_group<kEnergy>(
                e0, e1, lj,
                [=](uint32_t e, float& dx, float& dy, float& dz) {
                    const float4 o = tab[e >> kCodeShift];
                    const unsigned slot = min(static_cast<unsigned>((e & kIndexMask) + __float_as_int(o.w)),
                                              static_cast<unsigned>(sentinel_slot));
                    return float_separation(qi, sq[slot], o, dx, dy, dz);
                },
                [=](uint32_t e) { return exact_inside(pos[i], pos[e & kIndexMask], box, lj.rc2d); }, ins);
            a.add_group(gs.x, gs.y, gs.z, gs.e, gs.w, e_fx, w_fx);
        }
        k_fx += a.finish(i, n_atoms, force, kick);
    }
    if (kEnergy || kick.vel) flush_sums(e_fx, w_fx, ins, k_fx, acc);
}

// ---- double-precision forces ------------------------------------------------------------------------------

// k_force_fp64 on a tile: the same per-particle order (own pairs in list order, then the pairs where the
// particle is second, in increasing j) and the same double operation sequence, with neighbour positions
// read from the staged tile. Optionally fuses the closing half kick (bit-identical to k_kick).
template <bool kTerms>
__global__ void __launch_bounds__(kTileThreads) k_force_fp64_tile(
    const double4* __restrict__ pos, int n_atoms, const int* __restrict__ cell_start,
    const int* __restrict__ cell_sorted, TileGeom g, LJ lj, const uint32_t* __restrict__ rows, int cap,
    const int2* __restrict__ counts, double* __restrict__ force, unsigned long long* __restrict__ inside,
    KickArgs kick, const long long* __restrict__ half_off, double* __restrict__ pair_r2, long long rec_cap) {
    extern __shared__ double4 s_p[];
    __shared__ TileTables t;
    __shared__ int s_delta[kMaxSegment][32];
    tile_tables(g, cell_start, t);
    const int span = t.kk + 2;
    if (t.total > g.max_staged) return;
    stage_tile(pos, s_p, t);
    for (int e = threadIdx.x; e < t.kk * 32; e += blockDim.x) {
        const int h = e / 32, code = e % 32;
        int delta = 0;
        if (code < 27) {
            const int sc = staged_cell(code, h, span);
            delta = t.off[sc] - t.gstart[sc];
        }
        s_delta[h][code] = delta;
    }
    cp_async_wait();
    __syncthreads();
    const int n = g.ncps;
    const unsigned last_slot = static_cast<unsigned>(g.max_staged - 1);
    unsigned long long ins = 0;
    for (int i = t.home_begin + threadIdx.x; i < t.home_end; i += blockDim.x) {
        const int h = (cell_sorted[i] % n - t.z0 + n) % n;
        const int* delta = s_delta[h];
        const double4 pi = s_p[i + delta[13]];  // code 13 = (0, 0, 0): the home cell
        const int2 c = counts[i];
        const long long pb = pair_r2 ? half_off[i] : 0;
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int s = 0; s < c.x + c.y; ++s) {
            const uint32_t e = rows[row_index(i, s, cap)];
            const unsigned slot = min(static_cast<unsigned>((e & kIndexMask) + delta[e >> kCodeShift]), last_slot);
            const double4 pj = s_p[slot];
            const bool own = s < c.x;
            const double4& a = own ? pi : pj;  // the pair's first particle
            const double4& b = own ? pj : pi;
            const double dx = min_image(dsub(a.x, b.x), g.box);
            const double dy = min_image(dsub(a.y, b.y), g.box);
            const double dz = min_image(dsub(a.z, b.z), g.box);
            const double r2 = norm2(dx, dy, dz);
            if (!(r2 < lj.rc2)) {
                if (own && pair_r2) store_pair_rec<kTerms>(pair_r2, pb + s, r2, 0.0, 0.0, false, rec_cap);
                continue;
            }
            double f, en;
            pair_terms(r2, lj, f, en);
            if (own) {
                if (pair_r2) store_pair_rec<kTerms>(pair_r2, pb + s, r2, f, en, true, rec_cap);
                fx = dadd(fx, dmul(f, dx));
                fy = dadd(fy, dmul(f, dy));
                fz = dadd(fz, dmul(f, dz));
                ++ins;
            } else {
                fx = dsub(fx, dmul(f, dx));
                fy = dsub(fy, dmul(f, dy));
                fz = dsub(fz, dmul(f, dz));
            }
        }
        const double F[3] = {fx, fy, fz};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const size_t o = static_cast<size_t>(k) * n_atoms + i;
            force[o] = F[k];
            if (kick.vel) kick.vel[o] = dadd(kick.vel[o], ddiv(dmul(kick.half_dt, F[k]), kick.mass[i]));
        }
    }
    ins = warp_sum_u64(ins);
    if ((threadIdx.x & 31) == 0 && ins) atomicAdd(inside, ins);
}

// ---- fixed-point kinetic energy -----------------------------------------------------------------------------

// 0.5 m v^2 per particle rounded to 2^-32 units and summed as integers: the same value the float force kernels
// fuse with the closing kick, independent of the launch shape (not the reference's summation order).
__global__ void k_kinetic_fixed(const double* __restrict__ vel, const double* __restrict__ mass, int n,
                                unsigned long long* __restrict__ acc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    long long v = 0;
    if (i < n) {
        double ke = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double x = vel[static_cast<size_t>(k) * n + i];
            ke = dadd(ke, dmul(x, x));
        }
        v = __double2ll_rn(dmul(dmul(dmul(0.5, mass[i]), ke), kKineticScale));  // as FloatAcc::finish
    }
    v = warp_sum_i64(v);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(acc, static_cast<unsigned long long>(v));
}

__global__ void k_fixed_to_double(const unsigned long long* __restrict__ acc, double unit, double* __restrict__ out) {
    *out = static_cast<double>(static_cast<long long>(*acc)) * unit;
}

// ---- fused drift ------------------------------------------------------------------------------------------

// kickAndDrift (src/Integrator.cpp:32-53) + NeighbourList::update's half-skin test (src/NeighbourList.cpp:24-30)
// + the float frame of the new position (float kernels only). Same double sequence as k_kick_drift.
__global__ void k_kick_drift_frames(double4* __restrict__ pos, double* __restrict__ vel,
                                    const double* __restrict__ force, const double* __restrict__ mass, int n,
                                    double half_dt, double dt, Box box, const double4* __restrict__ ref_pos,
                                    double max_disp2, int* __restrict__ stale, const int* __restrict__ cell_sorted,
                                    int ncps, double cell, float4* __restrict__ frames) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (frames && i == 0) frames[n] = make_float4(kSentinelCoord, kSentinelCoord, kSentinelCoord, 0.0f);
    if (i >= n) return;
    const double m = mass[i];
    double4 p = pos[i];
    double* pc[3] = {&p.x, &p.y, &p.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const size_t o = static_cast<size_t>(k) * n + i;
        const double v = dadd(vel[o], ddiv(dmul(half_dt, force[o]), m));
        vel[o] = v;
        *pc[k] = wrap(dadd(*pc[k], dmul(dt, v)), box);
    }
    pos[i] = p;
    if (ref_pos) {
        const double4 r = ref_pos[i];
        const double dx = min_image(dsub(p.x, r.x), box);
        const double dy = min_image(dsub(p.y, r.y), box);
        const double dz = min_image(dsub(p.z, r.z), box);
        if (norm2(dx, dy, dz) > max_disp2) *stale = 1;
    }
    if (frames) frames[i] = frame_of(p, cell_sorted[i], ncps, cell, box);
}

}  // namespace md
