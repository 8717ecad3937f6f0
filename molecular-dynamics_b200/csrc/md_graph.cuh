// Small kernels of md_run's graph mode: the device-side rebuild decision and the pieces of a list rebuild that
// the host path does with buffer swaps or host reads.
#pragma once

#include "md_common.cuh"

namespace md {

// The rebuild decision of a step: the conditional node that holds the list rebuild runs when the half-skin test
// of the last drift flagged a particle (NeighbourList::update, src/NeighbourList.cpp:11-36)
__global__ void k_set_rebuild(cudaGraphConditionalHandle handle, const int* __restrict__ stale) {
    cudaGraphSetConditional(handle, *stale != 0 ? 1u : 0u);
}

// Zero two int arrays (the cell counts and cursors of a counting sort)
__global__ void k_zero_ints(int* __restrict__ a, int na, int* __restrict__ b, int nb) {
    const int stride = gridDim.x * blockDim.x;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < na || k < nb; k += stride) {
        if (k < na) a[k] = 0;
        if (k < nb) b[k] = 0;
    }
}

// After a permute into the spare arrays: copy them back, so the system's arrays keep their addresses (the
// graph's kernels were recorded with them)
__global__ void k_copy_back(int n, const double4* __restrict__ pos2, const double* __restrict__ vel2,
                            const double* __restrict__ force2, const double* __restrict__ mass2,
                            const uint64_t* __restrict__ ids2, double4* __restrict__ pos, double* __restrict__ vel,
                            double* __restrict__ force, double* __restrict__ mass, uint64_t* __restrict__ ids) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    pos[k] = pos2[k];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        vel[static_cast<size_t>(c) * n + k] = vel2[static_cast<size_t>(c) * n + k];
        force[static_cast<size_t>(c) * n + k] = force2[static_cast<size_t>(c) * n + k];
    }
    mass[k] = mass2[k];
    ids[k] = ids2[k];
}

// After a device-side list build: count the rebuild (state[0]) and flag a row that outgrew the capacity or a
// staged tile that outgrew its shared memory (state[1]); the host reruns the chunk on its own path then.
// report_always flags every rebuild (md_system_set_graph's test flag for that path).
__global__ void k_build_done(int* __restrict__ max_count, int cap, int* __restrict__ state, bool report_always) {
    state[0] += 1;
    if (*max_count > cap || report_always) state[1] = 1;
    *max_count = 0;
}

}  // namespace md
