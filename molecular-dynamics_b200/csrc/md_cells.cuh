// Cell list: counting sort of particles into cubic cells, stable in particle index, and the particle reorder
// that NeighbourList::build performs on every rebuild.
//
// Reference: src/CellList.cpp:9-52 (cell id, histogram, prefix sum, stable scatter) and src/System.cpp:42-64
// (reorder). The stable scatter is done GPU-style: an atomic scatter into each cell's bucket (any order),
// then one warp per cell ranks its bucket by particle index, which restores the reference's order exactly.
#pragma once

#include "md_common.cuh"

namespace md {

// std::min(static_cast<int>(x * inverseCellSize), cellsPerSide - 1) (src/CellList.cpp:34). The lower clamp
// only matters for a coordinate below -1 cell, which the reference does not handle (it would index out of
// range); it keeps the device in bounds.
__device__ __forceinline__ int cell_coord(double x, double inv_cell, int ncps) {
    int c = __double2int_rz(dmul(x, inv_cell));
    c = c < ncps - 1 ? c : ncps - 1;
    return c > 0 ? c : 0;
}

__global__ void k_cell_assign(const double4* __restrict__ pos, int n, double inv_cell, int ncps,
                              int* __restrict__ cell_of, int* __restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = pos[i];
    const int c = (cell_coord(p.x, inv_cell, ncps) * ncps + cell_coord(p.y, inv_cell, ncps)) * ncps +
                  cell_coord(p.z, inv_cell, ncps);
    cell_of[i] = c;
    atomicAdd(&count[c], 1);
}

// bucket[start[c] + k] for k < count[c] receives the particles of cell c in arbitrary order
__global__ void k_cell_scatter(const int* __restrict__ cell_of, int n, const int* __restrict__ start,
                               int* __restrict__ cursor, uint32_t* __restrict__ bucket) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = cell_of[i];
    bucket[start[c] + atomicAdd(&cursor[c], 1)] = static_cast<uint32_t>(i);
}

// One warp per cell: each particle's rank in its cell is the number of smaller indices in the bucket, so
// order[] lists every cell's particles in increasing index, as the reference's serial scatter does
// (src/CellList.cpp:48-51). A cell of up to 32 particles is ranked from registers (one index per lane, compared
// through shuffles); larger cells compare against the bucket in memory.
__global__ void k_cell_rank(const int* __restrict__ start, int ncells, const uint32_t* __restrict__ bucket,
                            uint32_t* __restrict__ order) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= ncells) return;
    const int s = start[warp];
    const int m = start[warp + 1] - s;
    if (m <= 32) {
        const uint32_t v = lane < m ? bucket[s + lane] : 0xffffffffu;
        int rank = 0;
        for (int f = 0; f < m; ++f) rank += __shfl_sync(0xffffffffu, v, f) < v;
        if (lane < m) order[s + rank] = v;
        return;
    }
    for (int e = lane; e < m; e += 32) {
        const uint32_t v = bucket[s + e];
        int rank = 0;
        for (int f = 0; f < m; ++f) rank += bucket[s + f] < v;
        order[s + rank] = v;
    }
}

// new[k] = old[order[k]] for every per-particle array (src/System.cpp:42-64); the caller swaps the buffers.
// With cell_of_old, also the list's per-particle cell (cell_of of the sorted order) and its reference positions
// (src/NeighbourList.cpp:129-132).
__global__ void k_permute(const uint32_t* __restrict__ order, int n, const double4* __restrict__ pos,
                          const double* __restrict__ vel, const double* __restrict__ force,
                          const double* __restrict__ mass, const uint64_t* __restrict__ ids,
                          double4* __restrict__ pos2, double* __restrict__ vel2, double* __restrict__ force2,
                          double* __restrict__ mass2, uint64_t* __restrict__ ids2, const int* __restrict__ cell_of_old,
                          int* __restrict__ cell_sorted, double4* __restrict__ ref_pos) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t o = order[k];
    const double4 p = pos[o];
    pos2[k] = p;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        vel2[static_cast<size_t>(c) * n + k] = vel[static_cast<size_t>(c) * n + o];
        force2[static_cast<size_t>(c) * n + k] = force[static_cast<size_t>(c) * n + o];
    }
    mass2[k] = mass[o];
    ids2[k] = ids[o];
    if (cell_of_old) {
        cell_sorted[k] = cell_of_old[o];
        ref_pos[k] = p;
    }
}

// out[6 id + k] = (x, y, z, vx, vy, vz)[k] of the particle whose id is `id` (ids are a permutation of 0..n-1;
// an id out of range is skipped)
__global__ void k_frame_by_id(const double4* __restrict__ pos, const double* __restrict__ vel,
                              const uint64_t* __restrict__ ids, int n, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t id = ids[i];
    if (id >= static_cast<uint64_t>(n)) return;
    double* o = out + 6 * id;
    const double4 p = pos[i];
    o[0] = p.x;
    o[1] = p.y;
    o[2] = p.z;
    o[3] = vel[i];
    o[4] = vel[static_cast<size_t>(n) + i];
    o[5] = vel[2 * static_cast<size_t>(n) + i];
}

}  // namespace md
