// Verlet neighbour list build on the cell-sorted system (src/NeighbourList.cpp:55-134).
//
// Device layout: one fixed-capacity row of `cap` 32-bit entries per particle, stored uint4-interleaved
// (row_index in md_common.cuh). Row i holds, in order:
//   1. its own pairs j > i in the reference's candidate order (27 cells in (dx, dy, dz) order,
//      src/CellList.cpp:55-83, then increasing j inside each cell, src/NeighbourList.cpp:38-52) — exactly
//      neighboursOf(i);
//   2. the particles j < i that list i as a neighbour, in increasing j — the pairs pairsAsSecond(i) of the
//      reference's reverse index, in the same order (a pair's global index grows with its first particle);
//   3. sentinel entries (n | kSentinelCode << 27) up to a multiple of 8.
// Each entry is j | (cell code << 27), the code being (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1) of the
// neighbour cell, used by the float kernels to rebuild the periodic image. A pair is in the list when its
// minimum-image r^2 < (r_c + skin)^2 in the reference's double arithmetic; the test is symmetric in (i, j)
// bit for bit, so part 2 needs no second pass over the reference order.
#pragma once

#include "md_common.cuh"

namespace md {

struct ListGeom {
    Box box;
    double rl2;     // (cut_off + skin)^2 (src/NeighbourList.cpp:6)
    int ncps;       // cells per side
    int use_cells;  // ncps >= 3 (src/NeighbourList.cpp:69)
    int cap;        // row capacity (multiple of 8)
    uint32_t sentinel;
};

__device__ __forceinline__ bool within_list(const double4& a, const double4& b, const ListGeom& g) {
    const double dx = min_image(dsub(a.x, b.x), g.box);
    const double dy = min_image(dsub(a.y, b.y), g.box);
    const double dz = min_image(dsub(a.z, b.z), g.box);
    return norm2(dx, dy, dz) < g.rl2;
}

// The three wrapped offsets along one axis in increasing wrapped-cell order: for c = 0 the cells are
// {0, 1, n-1}, for c = n-1 {0, n-2, n-1}, otherwise {c-1, c, c+1}.
__device__ __forceinline__ void ascending_offsets(int c, int n, int* d) {
    if (c == 0) {
        d[0] = 0; d[1] = 1; d[2] = -1;
    } else if (c == n - 1) {
        d[0] = 1; d[1] = -1; d[2] = 0;
    } else {
        d[0] = -1; d[1] = 0; d[2] = 1;
    }
}

// One thread per particle. counts[i] = (own, reverse); rows beyond `cap` are not written, and max_count
// records the longest row so the host can grow `cap` and rebuild.
__global__ void k_nlist_build(const double4* __restrict__ pos, int n, ListGeom g, const int* __restrict__ cell_of,
                              const int* __restrict__ cell_start, uint32_t* __restrict__ rows,
                              int2* __restrict__ counts, int* __restrict__ max_count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 pi = pos[i];
    int cnt = 0;
    auto push = [&](int j, uint32_t code) {
        if (cnt < g.cap) rows[row_index(i, cnt, g.cap)] = static_cast<uint32_t>(j) | (code << kCodeShift);
        ++cnt;
    };
    int own;
    if (g.use_cells) {
        const int nc = g.ncps;
        const int c = cell_of[i];
        const int cx = c / (nc * nc), cy = (c / nc) % nc, cz = c % nc;
        for (int dx = -1; dx <= 1; ++dx) {
            const int x = (cx + dx + nc) % nc;
            for (int dy = -1; dy <= 1; ++dy) {
                const int y = (cy + dy + nc) % nc;
                for (int dz = -1; dz <= 1; ++dz) {
                    const int cell = (x * nc + y) * nc + (cz + dz + nc) % nc;
                    const uint32_t code = (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
                    const int e = cell_start[cell + 1];
                    for (int j = cell_start[cell] > i + 1 ? cell_start[cell] : i + 1; j < e; ++j)
                        if (within_list(pi, pos[j], g)) push(j, code);
                }
            }
        }
        own = cnt;
        int ox[3], oy[3], oz[3];
        ascending_offsets(cx, nc, ox);
        ascending_offsets(cy, nc, oy);
        ascending_offsets(cz, nc, oz);
        for (int a = 0; a < 3; ++a) {
            const int x = (cx + ox[a] + nc) % nc;
            for (int b = 0; b < 3; ++b) {
                const int y = (cy + oy[b] + nc) % nc;
                for (int d = 0; d < 3; ++d) {
                    const int cell = (x * nc + y) * nc + (cz + oz[d] + nc) % nc;
                    const uint32_t code = (ox[a] + 1) * 9 + (oy[b] + 1) * 3 + (oz[d] + 1);
                    const int s = cell_start[cell];
                    const int e = cell_start[cell + 1] < i ? cell_start[cell + 1] : i;
                    for (int j = s; j < e; ++j)
                        if (within_list(pi, pos[j], g)) push(j, code);
                }
            }
        }
    } else {
        // Box under 3 cells per side: every particle is a candidate (src/NeighbourList.cpp:45-50)
        for (int j = i + 1; j < n; ++j)
            if (within_list(pi, pos[j], g)) push(j, 13u);
        own = cnt;
        for (int j = 0; j < i; ++j)
            if (within_list(pi, pos[j], g)) push(j, 13u);
    }
    counts[i] = make_int2(own, cnt - own);
    const int padded = (cnt + 7) & ~7;
    for (int s = cnt; s < padded && s < g.cap; ++s) rows[row_index(i, s, g.cap)] = g.sentinel;
    atomicMax(max_count, padded);
}

__global__ void k_own_counts(const int2* __restrict__ counts, int n, int* __restrict__ own) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) own[i] = counts[i].x;
}

__global__ void k_rev_counts(const int2* __restrict__ counts, int n, int* __restrict__ rev) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rev[i] = counts[i].y;
}

// Half CSR for download: neighbours[half_off[i] + s] = own entry s of row i
__global__ void k_half_csr(const uint32_t* __restrict__ rows, int n, int cap, const int2* __restrict__ counts,
                           const long long* __restrict__ half_off, uint64_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long b = half_off[i];
    for (int s = 0; s < counts[i].x; ++s) out[b + s] = rows[row_index(i, s, cap)] & kIndexMask;
}

// Reverse CSR for download (pairsAsSecond): the r-th partner j < i of i is the pair whose global index is
// half_off[j] plus the position of i in j's own entries.
__global__ void k_reverse_pairs(const uint32_t* __restrict__ rows, int n, int cap, const int2* __restrict__ counts,
                                const long long* __restrict__ half_off, const long long* __restrict__ rev_off,
                                uint64_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 c = counts[i];
    const long long b = rev_off[i];
    for (int r = 0; r < c.y; ++r) {
        const int j = static_cast<int>(rows[row_index(i, c.x + r, cap)] & kIndexMask);
        const int own_j = counts[j].x;
        int pos = 0;
        while (pos < own_j && (rows[row_index(j, pos, cap)] & kIndexMask) != static_cast<uint32_t>(i)) ++pos;
        out[b + r] = static_cast<uint64_t>(half_off[j] + pos);
    }
}

}  // namespace md
