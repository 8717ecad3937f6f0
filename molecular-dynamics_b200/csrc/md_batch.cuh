// Batched replicas: many independent Lennard-Jones systems of uneven size, density and temperature advanced by
// the same kernel launches, each replica following the reference's single-system step (src/Integrator.cpp:18-30,
// src/NeighbourList.cpp:11-134, src/Forcefield.cpp:214-326, src/Thermostat.cpp:17-58) on its own box.
//
// Layout. Replica r owns the particle slots [off_r, off_r + n_r), off_r a multiple of kTile, so every tile of
// kTile slots (and every thread block over one) belongs to exactly one replica; tile_rep[t] names it. Positions,
// masses, ids, frames and neighbour rows are indexed by slot. Velocities and forces keep each replica's
// component-major arrays contiguous: component k of slot a sits at 3 off_r + k np_r + (a - off_r), np_r being n_r
// rounded up to kTile. The cell arrays are concatenated the same way (cell_off_r; the cell starts of replica r
// take ncells_r + 1 entries from cell_off_r + r).
//
// Rebuilds are decided on the device: the drift kernel flags a replica whose particle moved more than half the
// skin, k_b_stale_lists turns the flags into a list of stale replicas and of their tiles, and the rebuild kernels
// loop over those lists with a fixed grid, so a step needs no host decision and a run of steps can be one CUDA
// graph. Each replica's cell sort, reorder, list and sums repeat the single-system kernels' operation sequences,
// so a replica's trajectory is bit-identical to the same system run alone.
#pragma once

#include "md_cells.cuh"
#include "md_common.cuh"
#include "md_fp32.cuh"
#include "md_tiles.cuh"
#include "md_fp64.cuh"
#include "md_nlist.cuh"

namespace md {

constexpr int kTile = 128;          // slots per tile; replicas start on tile boundaries
constexpr int kListThreads = 1024;  // k_b_stale_lists block
constexpr int kRepScanThreads = 256;   // per-replica scans

struct BRep {
    Box box;
    double inv_cell;     // cells per side / L (src/CellList.cpp:18)
    double cell;         // L / cells per side
    double dof;          // 3 n - 3 (src/System.cpp:79-82)
    double temperature;  // thermostat target
    int off;             // first slot
    int n;               // particles
    int np;              // n rounded up to kTile: component stride of velocities and forces
    int ncps;            // cells per side
    int ncells;          // ncps^3
    int cell_off;        // first cell of the count/cursor arrays
    int use_cells;       // ncps >= 3 (src/NeighbourList.cpp:69)
    int tile_off;        // first tile
    int chunk_off;       // first 1024-particle block of the kinetic-energy sums
};

// Index of component k of slot a in the velocity and force arrays
__device__ __forceinline__ size_t bvec(const BRep& d, int k, int a) {
    return 3 * static_cast<size_t>(d.off) + static_cast<size_t>(k) * d.np + (a - d.off);
}

__device__ __forceinline__ int inclusive_warp_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int x = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += x;
    }
    return v;
}

// Exclusive block scan of v with a running carry (kRepScanThreads threads); returns the exclusive prefix and adds
// the block's total to *carry after a barrier
__device__ __forceinline__ int block_scan_carry(int v, int* s_warp, int* carry) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = inclusive_warp_scan(v);
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int y = lane < kRepScanThreads / 32 ? s_warp[lane] : 0;
        y = inclusive_warp_scan(y);
        if (lane < kRepScanThreads / 32) s_warp[lane] = y;
    }
    __syncthreads();
    const int excl = *carry + (warp ? s_warp[warp - 1] : 0) + x - v;
    __syncthreads();
    if (threadIdx.x == kRepScanThreads - 1) *carry = excl + v;
    __syncthreads();
    return excl;
}

// ---- integration --------------------------------------------------------------------------------------------

// One tile per block. A pending thermostat scale (scale[r].y != 0) is applied first, as scaleVelocities would
// have at the end of the previous step (src/Thermostat.cpp:7-14), then kickAndDrift (src/Integrator.cpp:32-53),
// the half-skin test (src/NeighbourList.cpp:24-30) that flags the replica stale, and with kFrames the float
// frame of the new position.
template <bool kFrames>
__global__ void __launch_bounds__(kTile)
    k_b_kick_drift(const BRep* __restrict__ reps, const int* __restrict__ tile_rep, double4* __restrict__ pos,
                   double* __restrict__ vel, const double* __restrict__ force, const double* __restrict__ mass,
                   double half_dt, double dt, const double4* __restrict__ ref_pos, double max_disp2,
                   int* __restrict__ stale, const double2* __restrict__ scale, const int* __restrict__ cell_sorted,
                   float4* __restrict__ frames) {
    const int r = tile_rep[blockIdx.x];
    const BRep d = reps[r];
    const int i = (blockIdx.x - d.tile_off) * kTile + threadIdx.x;
    if (i >= d.n) return;
    const int a = d.off + i;
    const double2 sc = scale[r];
    const double m = mass[a];
    double4 p = pos[a];
    double* pc[3] = {&p.x, &p.y, &p.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const size_t o = bvec(d, k, a);
        double v = vel[o];
        if (sc.y != 0.0) v = dmul(v, sc.x);
        v = dadd(v, ddiv(dmul(half_dt, force[o]), m));
        vel[o] = v;
        *pc[k] = wrap(dadd(*pc[k], dmul(dt, v)), d.box);
    }
    pos[a] = p;
    const double4 q = ref_pos[a];
    const double dx = min_image(dsub(p.x, q.x), d.box);
    const double dy = min_image(dsub(p.y, q.y), d.box);
    const double dz = min_image(dsub(p.z, q.z), d.box);
    if (norm2(dx, dy, dz) > max_disp2) stale[r] = 1;
    if (kFrames) frames[a] = frame_of(p, cell_sorted[a], d.ncps, d.cell, d.box);
}

// Applies and clears the pending thermostat scales (end of a run), one tile per block; k_b_clear_scale follows.
__global__ void __launch_bounds__(kTile) k_b_apply_scale(const BRep* __restrict__ reps, const int* __restrict__ tile_rep,
                                                         double* __restrict__ vel, const double2* __restrict__ scale) {
    const int r = tile_rep[blockIdx.x];
    const BRep d = reps[r];
    const int i = (blockIdx.x - d.tile_off) * kTile + threadIdx.x;
    const double2 sc = scale[r];
    if (i >= d.n || sc.y == 0.0) return;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const size_t o = bvec(d, k, d.off + i);
        vel[o] = dmul(vel[o], sc.x);
    }
}

__global__ void k_b_clear_scale(int R, double2* __restrict__ scale) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < R) scale[r] = make_double2(1.0, 0.0);
}

// ---- rebuild ------------------------------------------------------------------------------------------------

// One block. Reads and clears the stale flags, lists the stale replicas and their tiles in replica order
// (work[0] replicas, work[1] tiles) and counts each replica's rebuild.
__global__ void __launch_bounds__(kListThreads)
    k_b_stale_lists(const BRep* __restrict__ reps, int R, int* __restrict__ stale, int* __restrict__ stale_reps,
                    int* __restrict__ stale_tiles, int* __restrict__ work, unsigned long long* __restrict__ rebuilds) {
    __shared__ int s_warp[2][32];
    __shared__ int s_base[2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kWarps = kListThreads / 32;
    if (threadIdx.x == 0) s_base[0] = s_base[1] = 0;
    __syncthreads();
    for (int r0 = 0; r0 < R; r0 += kListThreads) {
        const int r = r0 + threadIdx.x;
        int f = 0, nt = 0, t0 = 0;
        if (r < R && stale[r]) {
            stale[r] = 0;
            const BRep d = reps[r];
            f = 1;
            nt = d.np / kTile;
            t0 = d.tile_off;
        }
        const int sf = inclusive_warp_scan(f), st = inclusive_warp_scan(nt);
        if (lane == 31) {
            s_warp[0][warp] = sf;
            s_warp[1][warp] = st;
        }
        __syncthreads();
        if (warp == 0) {
            const int a = inclusive_warp_scan(s_warp[0][lane]);
            const int b = inclusive_warp_scan(s_warp[1][lane]);
            s_warp[0][lane] = a;
            s_warp[1][lane] = b;
        }
        __syncthreads();
        if (f) {
            const int pf = s_base[0] + (warp ? s_warp[0][warp - 1] : 0) + sf - 1;
            const int pt = s_base[1] + (warp ? s_warp[1][warp - 1] : 0) + st - nt;
            stale_reps[pf] = r;
            for (int k = 0; k < nt; ++k) stale_tiles[pt + k] = t0 + k;
            rebuilds[r] += 1;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_base[0] += s_warp[0][kWarps - 1];
            s_base[1] += s_warp[1][kWarps - 1];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        work[0] = s_base[0];
        work[1] = s_base[1];
    }
}

// The particle of this thread in the w-th stale tile: returns false past the replica's end
__device__ __forceinline__ bool stale_slot(const BRep* __restrict__ reps, const int* __restrict__ tile_rep,
                                           const int* __restrict__ stale_tiles, int w, int& r, BRep& d, int& a) {
    const int t = stale_tiles[w];
    r = tile_rep[t];
    d = reps[r];
    const int i = (t - d.tile_off) * kTile + threadIdx.x;
    a = d.off + i;
    return i < d.n;
}

// CellList::build's cell index and histogram (src/CellList.cpp:25-40) for the stale replicas
__global__ void __launch_bounds__(kTile)
    k_b_cell_assign(const BRep* __restrict__ reps, const int* __restrict__ tile_rep, const int* __restrict__ stale_tiles,
                    const int* __restrict__ work, const double4* __restrict__ pos, int* __restrict__ cell_of,
                    int* __restrict__ count) {
    const int nw = work[1];
    for (int w = blockIdx.x; w < nw; w += gridDim.x) {
        int r, a;
        BRep d;
        if (!stale_slot(reps, tile_rep, stale_tiles, w, r, d, a)) continue;
        const double4 p = pos[a];
        const int c = (cell_coord(p.x, d.inv_cell, d.ncps) * d.ncps + cell_coord(p.y, d.inv_cell, d.ncps)) * d.ncps +
                      cell_coord(p.z, d.inv_cell, d.ncps);
        cell_of[a] = c;
        atomicAdd(&count[d.cell_off + c], 1);
    }
}

// Exclusive prefix sum of each stale replica's cell histogram into slot numbers (src/CellList.cpp:42-46); the
// histogram is cleared for the next rebuild. One block per stale replica.
__global__ void __launch_bounds__(kRepScanThreads)
    k_b_cell_scan(const BRep* __restrict__ reps, const int* __restrict__ stale_reps, const int* __restrict__ work,
                  int* __restrict__ count, int* __restrict__ start) {
    __shared__ int s_warp[32];
    __shared__ int s_carry;
    const int nr = work[0];
    for (int w = blockIdx.x; w < nr; w += gridDim.x) {
        const int r = stale_reps[w];
        const BRep d = reps[r];
        int* st = start + d.cell_off + r;
        if (threadIdx.x == 0) s_carry = d.off;
        __syncthreads();
        for (int c0 = 0; c0 < d.ncells; c0 += kRepScanThreads) {
            const int c = c0 + threadIdx.x;
            const int v = c < d.ncells ? count[d.cell_off + c] : 0;
            const int e = block_scan_carry(v, s_warp, &s_carry);
            if (c < d.ncells) {
                st[c] = e;
                count[d.cell_off + c] = 0;
            }
        }
        if (threadIdx.x == 0) st[d.ncells] = d.off + d.n;
        __syncthreads();
    }
}

// Scatter into the cell buckets in any order (k_cell_scatter)
__global__ void __launch_bounds__(kTile)
    k_b_cell_scatter(const BRep* __restrict__ reps, const int* __restrict__ tile_rep,
                     const int* __restrict__ stale_tiles, const int* __restrict__ work, const int* __restrict__ cell_of,
                     const int* __restrict__ start, int* __restrict__ cursor, uint32_t* __restrict__ bucket) {
    const int nw = work[1];
    for (int w = blockIdx.x; w < nw; w += gridDim.x) {
        int r, a;
        BRep d;
        if (!stale_slot(reps, tile_rep, stale_tiles, w, r, d, a)) continue;
        const int c = cell_of[a];
        bucket[start[d.cell_off + r + c] + atomicAdd(&cursor[d.cell_off + c], 1)] = static_cast<uint32_t>(a);
    }
}

// Stable order inside each cell: a particle's rank is the number of smaller slots in its bucket, as in the
// reference's serial scatter (src/CellList.cpp:48-51). Clears the scatter cursors for the next rebuild.
__global__ void __launch_bounds__(kTile)
    k_b_cell_rank(const BRep* __restrict__ reps, const int* __restrict__ tile_rep, const int* __restrict__ stale_tiles,
                  const int* __restrict__ work, const int* __restrict__ cell_of, const int* __restrict__ start,
                  int* __restrict__ cursor, const uint32_t* __restrict__ bucket, uint32_t* __restrict__ order) {
    const int nw = work[1];
    for (int w = blockIdx.x; w < nw; w += gridDim.x) {
        int r, a;
        BRep d;
        if (!stale_slot(reps, tile_rep, stale_tiles, w, r, d, a)) continue;
        const int c = cell_of[a];
        const int s = start[d.cell_off + r + c], e = start[d.cell_off + r + c + 1];
        int rank = 0;
        for (int f = s; f < e; ++f) rank += bucket[f] < static_cast<uint32_t>(a);
        order[s + rank] = static_cast<uint32_t>(a);
        cursor[d.cell_off + c] = 0;
    }
}

// new[a] = old[order[a]] inside each stale replica (src/System.cpp:42-64), into the scratch arrays; the sorted
// particles' cells go straight to cell_sorted
__global__ void __launch_bounds__(kTile)
    k_b_permute(const BRep* __restrict__ reps, const int* __restrict__ tile_rep, const int* __restrict__ stale_tiles,
                const int* __restrict__ work, const uint32_t* __restrict__ order, const int* __restrict__ cell_of,
                const double4* __restrict__ pos, const double* __restrict__ vel, const double* __restrict__ force,
                const double* __restrict__ mass, const uint64_t* __restrict__ ids, double4* __restrict__ pos2,
                double* __restrict__ vel2, double* __restrict__ force2, double* __restrict__ mass2,
                uint64_t* __restrict__ ids2, int* __restrict__ cell_sorted) {
    const int nw = work[1];
    for (int w = blockIdx.x; w < nw; w += gridDim.x) {
        int r, a;
        BRep d;
        if (!stale_slot(reps, tile_rep, stale_tiles, w, r, d, a)) continue;
        const int o = static_cast<int>(order[a]);
        pos2[a] = pos[o];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            vel2[bvec(d, k, a)] = vel[bvec(d, k, o)];
            force2[bvec(d, k, a)] = force[bvec(d, k, o)];
        }
        mass2[a] = mass[o];
        ids2[a] = ids[o];
        cell_sorted[a] = cell_of[o];
    }
}

// Copies the permuted arrays back and records the list's reference positions (src/NeighbourList.cpp:129-132)
// and the frames of the new order
__global__ void __launch_bounds__(kTile)
    k_b_commit(const BRep* __restrict__ reps, const int* __restrict__ tile_rep, const int* __restrict__ stale_tiles,
               const int* __restrict__ work, const double4* __restrict__ pos2, const double* __restrict__ vel2,
               const double* __restrict__ force2, const double* __restrict__ mass2, const uint64_t* __restrict__ ids2,
               const int* __restrict__ cell_sorted, double4* __restrict__ pos, double* __restrict__ vel,
               double* __restrict__ force, double* __restrict__ mass, uint64_t* __restrict__ ids,
               double4* __restrict__ ref_pos, float4* __restrict__ frames) {
    const int nw = work[1];
    for (int w = blockIdx.x; w < nw; w += gridDim.x) {
        int r, a;
        BRep d;
        if (!stale_slot(reps, tile_rep, stale_tiles, w, r, d, a)) continue;
        const double4 p = pos2[a];
        pos[a] = p;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            vel[bvec(d, k, a)] = vel2[bvec(d, k, a)];
            force[bvec(d, k, a)] = force2[bvec(d, k, a)];
        }
        mass[a] = mass2[a];
        ids[a] = ids2[a];
        ref_pos[a] = p;
        frames[a] = frame_of(p, cell_sorted[a], d.ncps, d.cell, d.box);
    }
}

struct BBuild {
    double rl2;      // (r_c + skin)^2
    float lo, hi;    // float r^2 below lo: inside, above hi: outside, between: decided in double
    int cap;         // row capacity
    uint32_t sentinel;
};

__device__ __forceinline__ bool within_rl(const double4& a, const double4& b, const Box& box, double rl2) {
    const double dx = min_image(dsub(a.x, b.x), box);
    const double dy = min_image(dsub(a.y, b.y), box);
    const double dz = min_image(dsub(a.z, b.z), box);
    return norm2(dx, dy, dz) < rl2;
}

// k_nlist_build for the stale replicas, with slots for indices: the same rows (own pairs in the reference's
// candidate order, then reverse partners ascending, then sentinels). With cells, candidates are screened with
// the float frames and only those within rounding of r_l are tested in double, which gives the double test's
// answer for every pair.
__global__ void __launch_bounds__(kTile)
    k_b_nlist_build(const BRep* __restrict__ reps, const int* __restrict__ tile_rep, const int* __restrict__ stale_tiles,
                    const int* __restrict__ work, const double4* __restrict__ pos, const float4* __restrict__ frames,
                    const int* __restrict__ cell_sorted, const int* __restrict__ start, BBuild bp,
                    uint32_t* __restrict__ rows, int2* __restrict__ counts, int* __restrict__ max_count) {
    const int nw = work[1];
    for (int w = blockIdx.x; w < nw; w += gridDim.x) {
        int r, a;
        BRep d;
        if (!stale_slot(reps, tile_rep, stale_tiles, w, r, d, a)) continue;
        const double4 pi = pos[a];
        int cnt = 0;
        auto push = [&](int j, uint32_t code) {
            if (cnt < bp.cap) rows[row_index(a, cnt, bp.cap)] = static_cast<uint32_t>(j) | (code << kCodeShift);
            ++cnt;
        };
        int own;
        if (d.use_cells) {
            const float4 qi = frames[a];
            const float cellf = static_cast<float>(d.cell);
            const int* st = start + d.cell_off + r;
            uint32_t* row = rows + row_index(a, 0, bp.cap);
            // candidates [j0, j1) of one cell (scan_cell: branch-free float screen, exact shell re-scan);
            // qo = q_i + the cell's image offset, computed once per candidate cell
            auto take = [&](int j0, int j1, uint32_t code, const float4& qo) {
                scan_cell<false>(frames + j0, j0, 0, j1 - j0, qo, code, bp.lo, bp.hi, bp.rl2, bp.cap, pi, pos, d.box, row,
                                 cnt);
            };
            auto shifted = [&](uint32_t code) {
                const float4 o = code_offset(static_cast<int>(code), cellf);
                return make_float4(qi.x + o.x, qi.y + o.y, qi.z + o.z, 0.0f);
            };
            const int nc = d.ncps;
            const int c = cell_sorted[a];
            const int cx = c / (nc * nc), cy = (c / nc) % nc, cz = c % nc;
            for (int dx = -1; dx <= 1; ++dx) {
                const int x = (cx + dx + nc) % nc;
                for (int dy = -1; dy <= 1; ++dy) {
                    const int y = (cy + dy + nc) % nc;
                    for (int dz = -1; dz <= 1; ++dz) {
                        const int cell = (x * nc + y) * nc + (cz + dz + nc) % nc;
                        const uint32_t code = (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
                        const int e = st[cell + 1];
                        const int j0 = st[cell] > a + 1 ? st[cell] : a + 1;
                        if (j0 < e) take(j0, e, code, shifted(code));
                    }
                }
            }
            own = cnt;
            int ox[3], oy[3], oz[3];
            ascending_offsets(cx, nc, ox);
            ascending_offsets(cy, nc, oy);
            ascending_offsets(cz, nc, oz);
            for (int u = 0; u < 3; ++u) {
                const int x = (cx + ox[u] + nc) % nc;
                for (int v = 0; v < 3; ++v) {
                    const int y = (cy + oy[v] + nc) % nc;
                    for (int q = 0; q < 3; ++q) {
                        const int cell = (x * nc + y) * nc + (cz + oz[q] + nc) % nc;
                        const uint32_t code = (ox[u] + 1) * 9 + (oy[v] + 1) * 3 + (oz[q] + 1);
                        const int e = st[cell + 1] < a ? st[cell + 1] : a;
                        if (st[cell] < e) take(st[cell], e, code, shifted(code));
                    }
                }
            }
        } else {
            // under 3 cells per side every particle of the replica is a candidate (src/NeighbourList.cpp:45-50)
            const int end = d.off + d.n;
            for (int j = a + 1; j < end; ++j)
                if (within_rl(pi, pos[j], d.box, bp.rl2)) push(j, 13u);
            own = cnt;
            for (int j = d.off; j < a; ++j)
                if (within_rl(pi, pos[j], d.box, bp.rl2)) push(j, 13u);
        }
        // a row past the capacity keeps counts within it (so every reader stays in bounds) and reports its
        // length: the host restores the chunk's starting state and runs it again with a larger capacity
        const int own_c = own < bp.cap ? own : bp.cap;
        const int all_c = cnt < bp.cap ? cnt : bp.cap;
        counts[a] = make_int2(own_c, all_c - own_c);
        const int padded = (cnt + 7) & ~7;
        for (int s = cnt; s < padded && s < bp.cap; ++s) rows[row_index(a, s, bp.cap)] = bp.sentinel;
        atomicMax(max_count, padded);
    }
}

// ---- forces -------------------------------------------------------------------------------------------------

// computeForcesDeterministic's per-particle sums (k_force_fp64) per replica, with the closing half kick and
// the replica's inside-cutoff count into acc[4 r + 2]
__global__ void __launch_bounds__(kTile)
    k_b_force_fp64(const BRep* __restrict__ reps, const int* __restrict__ tile_rep, const double4* __restrict__ pos,
                   LJ lj, const uint32_t* __restrict__ rows, int cap, const int2* __restrict__ counts,
                   double* __restrict__ force, unsigned long long* __restrict__ acc, double* __restrict__ kick_vel,
                   const double* __restrict__ mass, double half_dt) {
    const int r = tile_rep[blockIdx.x];
    const BRep d = reps[r];
    const int i = (blockIdx.x - d.tile_off) * kTile + threadIdx.x;
    unsigned long long ins = 0;
    if (i < d.n) {
        const int a = d.off + i;
        const double4 pi = pos[a];
        const int2 c = counts[a];
        const int m = c.x + c.y;
        const int quads = (m + 3) >> 2;
        double fx = 0.0, fy = 0.0, fz = 0.0;
        // k_force_fp64_quads' loop: a quad of row entries at a time, the next one in flight, every entry evaluated
        // and masked, the reverse pairs in the own form (the same bits as the reference's two loops)
        const uint4* rq = reinterpret_cast<const uint4*>(rows) + static_cast<size_t>(a >> 5) * (cap >> 2) * 32 + (a & 31);
        uint4 nq = make_uint4(0, 0, 0, 0);
        if (quads > 0) nq = __ldcs(rq);
        for (int q = 0; q < quads; ++q) {
            const uint4 eq = nq;
            if (q + 1 < quads) nq = __ldcs(rq + 32 * (q + 1));
            const uint32_t ent[4] = {eq.x, eq.y, eq.z, eq.w};
            double4 pj[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) pj[u] = pos[4 * q + u < m ? static_cast<int>(ent[u] & kIndexMask) : a];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int sl = 4 * q + u;
                const double dx = min_image(dsub(pi.x, pj[u].x), d.box);
                const double dy = min_image(dsub(pi.y, pj[u].y), d.box);
                const double dz = min_image(dsub(pi.z, pj[u].z), d.box);
                const double r2 = norm2(dx, dy, dz);
                const bool in = sl < m && r2 < lj.rc2;
                double f, e;
                pair_terms(in ? r2 : 1.0, lj, f, e);
                fx = dadd(fx, in ? dmul(f, dx) : 0.0);
                fy = dadd(fy, in ? dmul(f, dy) : 0.0);
                fz = dadd(fz, in ? dmul(f, dz) : 0.0);
                ins += (in && sl < c.x) ? 1u : 0u;
            }
        }
        const double F[3] = {fx, fy, fz};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const size_t o = bvec(d, k, a);
            force[o] = F[k];
            if (kick_vel) kick_vel[o] = dadd(kick_vel[o], ddiv(dmul(half_dt, F[k]), mass[a]));
        }
    }
    ins = warp_sum_u64(ins);
    if ((threadIdx.x & 31) == 0 && ins) atomicAdd(&acc[4 * r + 2], ins);
}

// The float list forces per replica (k_force_fp32_rows and, for replicas under 3 cells per side,
// k_force_fp32_small), with the same pinned pair sequence and 8-entry groups (kPrefetch: rows one group ahead).
// Each block covers `apb`
// consecutive particles of one tile with kTPA threads per particle; thread u of a particle takes groups
// u, u + kTPA, ... and the threads' fixed-point sums are added as integers, so every (apb, kTPA) gives the same
// bits (kTPA > 1 only with fixed point). Per-replica sums go to acc[4 r .. 4 r + 3] (energy, virial, inside
// count, kinetic energy after the fused kick).
template <bool kFixed, bool kEnergy, int kTPA, bool kPrefetch = false>
__global__ void __launch_bounds__(256)
    k_b_force_fp32(const BRep* __restrict__ reps, const int* __restrict__ tile_rep, int apb,
                   const float4* __restrict__ frames, const double4* __restrict__ pos, FloatLJ lj,
                   const uint32_t* __restrict__ rows, int cap, const int2* __restrict__ counts,
                   double* __restrict__ force, unsigned long long* __restrict__ acc, double* __restrict__ kick_vel,
                   const double* __restrict__ mass, double half_dt) {
    static_assert(kFixed || kTPA == 1, "float accumulation keeps one thread per particle");
    // the replica's cell-code offsets as a table of (x, y) pairs and one of z: an 8- and a 4-byte shared load
    // per entry instead of one of 16 (fewer shared-memory wavefronts in the L1 data pipe)
    __shared__ __align__(16) float s_o[4][32];
    const int parts = kTile / apb;
    const int t = blockIdx.x / parts, part = blockIdx.x - t * parts;
    const int r = tile_rep[t];
    const BRep d = reps[r];
    if (threadIdx.x < 32) {
        const float4 o = code_offset(threadIdx.x, static_cast<float>(d.cell));
        reinterpret_cast<float2*>(s_o[0])[threadIdx.x] = make_float2(o.x, o.y);
        s_o[2][threadIdx.x] = o.z;
    }
    __syncthreads();
    const int sub = threadIdx.x % kTPA;
    const int i = (t - d.tile_off) * kTile + part * apb + threadIdx.x / kTPA;
    const bool active = i < d.n;
    const int a = d.off + i;
    long long e_fx = 0, w_fx = 0, k_fx = 0;
    unsigned ins = 0;
    FloatAcc<kFixed, kEnergy> acc_i;
    if (active) {
        const int2 c = counts[a];
        const int m = c.x + c.y;
        const int groups = (m + 7) >> 3;
        if (d.use_cells) {
            const float4 qi = frames[a];
            // with kPrefetch (one thread per particle) the next group's row quads are in flight while this
            // group's frames are gathered, as in k_force_fp32_rows
            uint4 n0 = make_uint4(0, 0, 0, 0), n1 = n0;
            if (kPrefetch && sub < groups) {
                n0 = row_quad_stream(rows, a, 2 * sub, cap);
                n1 = row_quad_stream(rows, a, 2 * sub + 1, cap);
            }
            for (int g = sub; g < groups; g += kTPA) {
                uint4 e0, e1;
                if (kPrefetch) {
                    e0 = n0;
                    e1 = n1;
                    if (g + kTPA < groups) {
                        n0 = row_quad_stream(rows, a, 2 * (g + kTPA), cap);
                        n1 = row_quad_stream(rows, a, 2 * (g + kTPA) + 1, cap);
                    }
                } else {
                    e0 = row_quad(rows, a, 2 * g, cap);
                    e1 = row_quad(rows, a, 2 * g + 1, cap);
                }
                const float2* s_xy = reinterpret_cast<const float2*>(s_o[0]);
                const float* s_z = s_o[2];
                const Box box = d.box;
                const GroupSums gs = float_group<kEnergy>(
                    e0, e1, lj,
                    [=](uint32_t e, float& dx, float& dy, float& dz) {
                        const uint32_t k = e >> kCodeShift;
                        const float2 oxy = s_xy[k];
                        return float_separation(qi, frames[e & kIndexMask], make_float4(oxy.x, oxy.y, s_z[k], 0.0f),
                                                dx, dy, dz);
                    },
                    [=](uint32_t e) { return exact_inside(pos[a], pos[e & kIndexMask], box, lj.rc2d); }, ins);
                acc_i.add_group(gs.x, gs.y, gs.z, gs.e, gs.w, e_fx, w_fx);
            }
        } else {
            const double4 pi = pos[a];
            for (int g = sub; g < groups; g += kTPA) {
                float gx = 0.f, gy = 0.f, gz = 0.f, ge = 0.f, gw = 0.f;
                for (int s = 8 * g; s < 8 * g + 8 && s < m; ++s) {
                    const double4 pj = pos[rows[row_index(a, s, cap)] & kIndexMask];
                    const double ddx = min_image(dsub(pi.x, pj.x), d.box);
                    const double ddy = min_image(dsub(pi.y, pj.y), d.box);
                    const double ddz = min_image(dsub(pi.z, pj.z), d.box);
                    const float dx = static_cast<float>(ddx), dy = static_cast<float>(ddy), dz = static_cast<float>(ddz);
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, __fmul_rn(dz, dz)));
                    const bool in = norm2(ddx, ddy, ddz) < lj.rc2d;
                    float_pair<kEnergy>(dx, dy, dz, in, r2, lj, gx, gy, gz, ge, gw, ins);
                }
                acc_i.add_group(gx, gy, gz, ge, gw, e_fx, w_fx);
            }
        }
    }
    if (kTPA > 1) {
#pragma unroll
        for (int o = 1; o < kTPA; o <<= 1) {
            acc_i.ax += __shfl_xor_sync(0xffffffffu, acc_i.ax, o);
            acc_i.ay += __shfl_xor_sync(0xffffffffu, acc_i.ay, o);
            acc_i.az += __shfl_xor_sync(0xffffffffu, acc_i.az, o);
        }
    }
    if (active && sub == 0) {
        const double F[3] = {kFixed ? static_cast<double>(acc_i.ax) * kForceUnit : static_cast<double>(acc_i.fx),
                             kFixed ? static_cast<double>(acc_i.ay) * kForceUnit : static_cast<double>(acc_i.fy),
                             kFixed ? static_cast<double>(acc_i.az) * kForceUnit : static_cast<double>(acc_i.fz)};
        double ke = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const size_t o = bvec(d, k, a);
            force[o] = F[k];
            if (kick_vel) {  // as FloatAcc::finish
                const double v = dadd(kick_vel[o], ddiv(dmul(half_dt, F[k]), mass[a]));
                kick_vel[o] = v;
                ke = dadd(ke, dmul(v, v));
            }
        }
        if (kick_vel) k_fx = __double2ll_rn(dmul(dmul(dmul(0.5, mass[a]), ke), kKineticScale));
    }
    if (kEnergy || kick_vel) flush_sums(e_fx, w_fx, ins, k_fx, acc + 4 * r);
}

// Per replica: the fixed-point sums of the float kernels as doubles (k_finish_float_energy's conversions), the
// kinetic energy into ke[r] when `kinetic`, energy and virial into pe_out/w_out when given; clears acc
__global__ void k_b_finish_float(int R, unsigned long long* __restrict__ acc, bool kinetic, double* __restrict__ ke,
                                 double* __restrict__ pe_out, double* __restrict__ w_out,
                                 unsigned long long* __restrict__ inside) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    unsigned long long* s = acc + 4 * r;
    if (pe_out) pe_out[r] = 0.5 * static_cast<double>(static_cast<long long>(s[0])) * kEnergyUnit;
    if (w_out) w_out[r] = 0.5 * static_cast<double>(static_cast<long long>(s[1])) * kEnergyUnit;
    if (inside) inside[r] = s[2] / 2;
    if (kinetic) ke[r] = static_cast<double>(static_cast<long long>(s[3])) * (1.0 / kKineticScale);
    s[0] = s[1] = s[2] = s[3] = 0;
}

// Inside-cutoff counts of the FP64 kernel (acc[4 r + 2]) into inside[r]; clears acc
__global__ void k_b_finish_fp64(int R, unsigned long long* __restrict__ acc, unsigned long long* __restrict__ inside) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    unsigned long long* s = acc + 4 * r;
    if (inside) inside[r] = s[2];
    s[0] = s[1] = s[2] = s[3] = 0;
}

// The inside-cutoff count of every replica's last force evaluation into a record row (doubles)
__global__ void k_b_record_inside(int R, const unsigned long long* __restrict__ inside, double* __restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < R) out[r] = static_cast<double>(inside[r]);
}

// ---- kinetic energy and thermostats ---------------------------------------------------------------------------

// System::kineticEnergy's blocked sum (k_kinetic_blocks) per replica: one warp per 1024-particle block of a
// replica; with `scale` the pending thermostat scale is applied to each velocity first (the kinetic energy
// after scaleVelocities).
__global__ void k_b_kinetic_blocks(const BRep* __restrict__ reps, const int* __restrict__ chunk_rep, int nchunks,
                                   const double* __restrict__ vel, const double* __restrict__ mass,
                                   const double2* __restrict__ scale, double* __restrict__ chunk_sums) {
    extern __shared__ double sm_kb[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int blk = blockIdx.x * kEnergyWarps + warp;
    if (blk >= nchunks) return;
    const int r = chunk_rep[blk];
    const BRep d = reps[r];
    double* v = sm_kb + warp * kChunk;
    const int i0 = (blk - d.chunk_off) * kChunk;
    const int m = d.n - i0 < kChunk ? d.n - i0 : kChunk;
    const double2 sc = scale ? scale[r] : make_double2(1.0, 0.0);
    for (int t = lane; t < m; t += 32) {
        const int a = d.off + i0 + t;
        double c[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            c[k] = vel[bvec(d, k, a)];
            if (sc.y != 0.0) c[k] = dmul(c[k], sc.x);
        }
        v[t] = dmul(dmul(0.5, mass[a]), norm2(c[0], c[1], c[2]));
    }
    __syncwarp();
    if (lane == 0) {
        double s = 0.0;
        for (int t = 0; t < m; ++t) s = dadd(s, v[t]);
        chunk_sums[blk] = s;
    }
}

// deterministicSum's outer loop per replica: its block sums added in order; one warp per replica
__global__ void k_b_sum_chunks(const BRep* __restrict__ reps, int R, const double* __restrict__ chunk_sums,
                               double* __restrict__ out) {
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= R) return;
    const BRep d = reps[r];
    const int nb = (d.n + kChunk - 1) / kChunk;
    double s = 0.0;
    for (int b0 = 0; b0 < nb; b0 += 32) {
        const double v = b0 + lane < nb ? chunk_sums[d.chunk_off + b0 + lane] : 0.0;
        const int m = nb - b0 < 32 ? nb - b0 : 32;
        for (int t = 0; t < m; ++t) {
            const double x = __shfl_sync(0xffffffffu, v, t);
            if (lane == 0) s = dadd(s, x);
        }
    }
    if (lane == 0) out[r] = s;
}

// Fixed-point kinetic energy per replica (k_kinetic_fixed) with the pending scale applied, into acc[4 r + 3]
__global__ void __launch_bounds__(kTile)
    k_b_kinetic_fixed(const BRep* __restrict__ reps, const int* __restrict__ tile_rep, const double* __restrict__ vel,
                      const double* __restrict__ mass, const double2* __restrict__ scale,
                      unsigned long long* __restrict__ acc) {
    const int r = tile_rep[blockIdx.x];
    const BRep d = reps[r];
    const int i = (blockIdx.x - d.tile_off) * kTile + threadIdx.x;
    long long v = 0;
    if (i < d.n) {
        const int a = d.off + i;
        const double2 sc = scale[r];
        double ke = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double x = vel[bvec(d, k, a)];
            if (sc.y != 0.0) x = dmul(x, sc.x);
            ke = dadd(ke, dmul(x, x));
        }
        v = __double2ll_rn(dmul(dmul(dmul(0.5, mass[a]), ke), kKineticScale));
    }
    v = warp_sum_i64(v);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&acc[4 * r + 3], static_cast<unsigned long long>(v));
}

// Thermostat factors per replica into scale[r] = (factor, 1), or (1, 0) to leave the replica alone.
// mode 1: rescaleVelocities to the replica's temperature (src/Thermostat.cpp:17-30); mode 2: Bussi with the
// step's draws r1[r], chi2[r] (src/Thermostat.cpp:36-58).
__global__ void k_b_thermostat(const BRep* __restrict__ reps, int R, int mode, const double* __restrict__ ke, double c,
                               const double* __restrict__ r1, const double* __restrict__ chi2,
                               double2* __restrict__ scale) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    const BRep d = reps[r];
    const double kinetic = ke[r];
    double2 out = make_double2(1.0, 0.0);
    if (mode == 1) {
        const double t = ddiv(dmul(2.0, kinetic), d.dof);
        if (t > 0.0) out = make_double2(__dsqrt_rn(ddiv(d.temperature, t)), 1.0);
    } else if (kinetic > 0.0) {
        out = make_double2(bussi_scale(kinetic, d.dof, d.temperature, c, r1[r], chi2[r]), 1.0);
    }
    scale[r] = out;
}

// ---- FP64 energy and virial in the reference's pair order ----------------------------------------------------

// Exclusive prefix of each replica's own-pair counts (the half-list CSR offsets, src/NeighbourList.cpp:116-127)
// into half_off[slot] and the replica's pair count into pairs[r]; one block per replica
__global__ void __launch_bounds__(kRepScanThreads)
    k_b_half_offsets(const BRep* __restrict__ reps, int R, const int2* __restrict__ counts, int* __restrict__ half_off,
                     int* __restrict__ pairs) {
    __shared__ int s_warp[32];
    __shared__ int s_carry;
    for (int r = blockIdx.x; r < R; r += gridDim.x) {
        const BRep d = reps[r];
        if (threadIdx.x == 0) s_carry = 0;
        __syncthreads();
        for (int i0 = 0; i0 < d.n; i0 += kRepScanThreads) {
            const int i = i0 + threadIdx.x;
            const int v = i < d.n ? counts[d.off + i].x : 0;
            const int e = block_scan_carry(v, s_warp, &s_carry);
            if (i < d.n) half_off[d.off + i] = e;
        }
        if (threadIdx.x == 0) pairs[r] = s_carry;
        __syncthreads();
    }
}

// item_off[r] = number of 1024-pair blocks of the replicas before r; item_off[R] the total. One block.
__global__ void __launch_bounds__(kRepScanThreads) k_b_pair_items(int R, const int* __restrict__ pairs,
                                                               int* __restrict__ item_off) {
    __shared__ int s_warp[32];
    __shared__ int s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int r0 = 0; r0 < R; r0 += kRepScanThreads) {
        const int r = r0 + threadIdx.x;
        const int v = r < R ? (pairs[r] + kChunk - 1) / kChunk : 0;
        const int e = block_scan_carry(v, s_warp, &s_carry);
        if (r < R) item_off[r] = e;
    }
    if (threadIdx.x == 0) item_off[R] = s_carry;
}

// Per replica: energy and virial of each 1024-pair block of the half list in the reference's pair order, summed
// from 0.0 one after another (deterministicSum's inner loop, include/Parallel.hpp:43-46; pairEnergy/pairVirial
// of src/Forcefield.cpp:288-296). Each warp takes blocks (items) of all replicas in turn: the lanes evaluate the
// block's pairs into shared memory, lane 0 adds them in order.
__global__ void k_b_energy_blocks(const BRep* __restrict__ reps, int R, const int* __restrict__ item_off,
                                  const int* __restrict__ pairs, const int* __restrict__ half_off,
                                  const double4* __restrict__ pos, LJ lj, const uint32_t* __restrict__ rows, int cap,
                                  double2* __restrict__ item_sums) {
    extern __shared__ double2 sm_bew[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double2* ew = sm_bew + warp * kChunk;
    const int total = item_off[R];
    for (int item = blockIdx.x * kEnergyWarps + warp; item < total; item += gridDim.x * kEnergyWarps) {
        int lo = 0, hi = R;  // the replica: last r with item_off[r] <= item
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (item_off[mid] <= item) lo = mid; else hi = mid;
        }
        const int r = lo;
        const BRep d = reps[r];
        const int np = pairs[r];
        const int k0 = (item - item_off[r]) * kChunk;
        const int k1 = k0 + kChunk < np ? k0 + kChunk : np;
        int i = 0;  // first particle whose pairs reach k0
        if (lane == 0) {
            int l = 0, h = d.n;
            while (h - l > 1) {
                const int mid = (l + h) >> 1;
                if (half_off[d.off + mid] <= k0) l = mid; else h = mid;
            }
            i = l;
        }
        i = __shfl_sync(0xffffffffu, i, 0);
        for (; i < d.n && half_off[d.off + i] < k1; ++i) {
            const int a = d.off + i;
            const int b = half_off[a];
            const int kb = b > k0 ? b : k0;
            const int e_i = i + 1 < d.n ? half_off[a + 1] : np;
            const int ke = e_i < k1 ? e_i : k1;
            const double4 pi = pos[a];
            for (int k = kb + lane; k < ke; k += 32) {
                const double4 pj = pos[rows[row_index(a, k - b, cap)] & kIndexMask];
                const double dx = min_image(dsub(pi.x, pj.x), d.box);
                const double dy = min_image(dsub(pi.y, pj.y), d.box);
                const double dz = min_image(dsub(pi.z, pj.z), d.box);
                const double r2 = norm2(dx, dy, dz);
                double f, e;
                pair_terms(r2, lj, f, e);
                const bool in = r2 < lj.rc2;
                f = in ? f : 0.0;
                ew[k - k0] = make_double2(in ? e : 0.0, dmul(f, r2));
            }
        }
        __syncwarp();
        if (lane == 0) {
            double se = 0.0, sw = 0.0;
            for (int t = 0; t < k1 - k0; ++t) {
                const double2 v = ew[t];
                se = dadd(se, v.x);
                sw = dadd(sw, v.y);
            }
            item_sums[item] = make_double2(se, sw);
        }
        __syncwarp();
    }
}

// The replica's block sums added in order (k_sum_blocks); one warp per replica
__global__ void k_b_sum_items(int R, const int* __restrict__ item_off, const double2* __restrict__ item_sums,
                              double* __restrict__ pe_out, double* __restrict__ w_out) {
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= R) return;
    const int b = item_off[r], nb = item_off[r + 1] - b;
    double se = 0.0, sw = 0.0;
    for (int b0 = 0; b0 < nb; b0 += 32) {
        const double2 v = b0 + lane < nb ? item_sums[b + b0 + lane] : make_double2(0.0, 0.0);
        const int m = nb - b0 < 32 ? nb - b0 : 32;
        for (int t = 0; t < m; ++t) {
            const double x = __shfl_sync(0xffffffffu, v.x, t);
            const double y = __shfl_sync(0xffffffffu, v.y, t);
            if (lane == 0) {
                se = dadd(se, x);
                sw = dadd(sw, y);
            }
        }
    }
    if (lane == 0) {
        pe_out[r] = se;
        w_out[r] = sw;
    }
}

// Moves row entries from a capacity-`cap0` buffer to a capacity-`cap1` one (cap1 > cap0), one thread per slot
__global__ void k_b_relayout_rows(int slots, const int2* __restrict__ counts, const uint32_t* __restrict__ src, int cap0,
                                  uint32_t* __restrict__ dst, int cap1) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= slots) return;
    const int2 c = counts[a];
    const int m = (c.x + c.y + 7) & ~7;
    for (int s = 0; s < m && s < cap0; ++s) dst[row_index(a, s, cap1)] = src[row_index(a, s, cap0)];
}

}  // namespace md
