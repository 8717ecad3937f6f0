// Double-precision kernels that reproduce the reference bit for bit: list forces in the deterministic
// summation order, the blocked energy/virial/kinetic sums, velocity Verlet, the half-skin check, thermostats
// and the g(r) histogram.
#pragma once

#include "md_common.cuh"

namespace md {

// ---- forces -----------------------------------------------------------------------------------------

// computeForcesDeterministic's per-particle sum (src/Forcefield.cpp:264-320): particle i adds F(i, j) over
// its own pairs in list order, then subtracts F(j, i) over the pairs where it is second, in increasing pair
// index. Pairs outside the cutoff contribute an exact zero in the reference and are skipped here. The
// inside-cutoff count is the number of own pairs with r^2 < r_c^2 (a sum of whole numbers, exact).
// With kick_vel set it also applies the closing half kick, v += (half_dt F) / m, with k_kick's sequence.
// With pair_r2 set, own pair s of particle i also stores its record for the ordered energy sums at index
// half_off[i] + s: with `terms`, its (pairEnergy, pairVirial) as a double2, E and (F/r) r^2 inside the cutoff,
// (0, 0) outside (src/Forcefield.cpp:288-296), which k_pair_block_sums_terms adds; without, its r^2, from which
// k_pair_block_sums recomputes the two terms with the same pair_terms call (the same operations on the same r^2,
// so the same bits). The r^2 record halves the traffic, which pays for large lists; for small ones the recomputation
// lengthens the sums (each lane evaluates its block's 1024 pairs in turn), so they keep the terms. Records past
// rec_cap, the buffer's size in records, are dropped: only a list rebuilt inside a CUDA graph can outgrow the
// buffer, and the graph's run then reports the overflow and repeats its steps on the host path.
template <bool kTerms>
__device__ __forceinline__ void store_pair_rec(double* rec, long long k, double r2, double f, double e, bool in,
                                               long long rec_cap) {
    if (k >= rec_cap) return;
    if (kTerms)
        reinterpret_cast<double2*>(rec)[k] = in ? make_double2(e, dmul(f, r2)) : make_double2(0.0, 0.0);
    else
        rec[k] = r2;  // the energy term is then never used, and the compiler leaves it out
}

template <bool kTerms>
__global__ void k_force_fp64(const double4* __restrict__ pos, int n, Box box, LJ lj, const uint32_t* __restrict__ rows,
                             int cap, const int2* __restrict__ counts, double* __restrict__ force,
                             unsigned long long* __restrict__ inside, double* __restrict__ kick_vel,
                             const double* __restrict__ mass, double half_dt, const long long* __restrict__ half_off,
                             double* __restrict__ pair_r2, long long rec_cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long ins = 0;
    if (i < n) {
        const double4 pi = pos[i];
        const int2 c = counts[i];
        const long long pb = pair_r2 ? half_off[i] : 0;
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int s = 0; s < c.x; ++s) {
            const double4 pj = pos[rows[row_index(i, s, cap)] & kIndexMask];
            const double dx = min_image(dsub(pi.x, pj.x), box);
            const double dy = min_image(dsub(pi.y, pj.y), box);
            const double dz = min_image(dsub(pi.z, pj.z), box);
            const double r2 = norm2(dx, dy, dz);
            if (!(r2 < lj.rc2)) {
                if (pair_r2) store_pair_rec<kTerms>(pair_r2, pb + s, r2, 0.0, 0.0, false, rec_cap);
                continue;
            }
            double f, e;
            pair_terms(r2, lj, f, e);
            if (pair_r2) store_pair_rec<kTerms>(pair_r2, pb + s, r2, f, e, true, rec_cap);
            fx = dadd(fx, dmul(f, dx));
            fy = dadd(fy, dmul(f, dy));
            fz = dadd(fz, dmul(f, dz));
            ++ins;
        }
        for (int s = c.x; s < c.x + c.y; ++s) {
            const double4 pj = pos[rows[row_index(i, s, cap)] & kIndexMask];
            const double dx = min_image(dsub(pj.x, pi.x), box);
            const double dy = min_image(dsub(pj.y, pi.y), box);
            const double dz = min_image(dsub(pj.z, pi.z), box);
            const double r2 = norm2(dx, dy, dz);
            if (!(r2 < lj.rc2)) continue;
            double f, e;
            pair_terms(r2, lj, f, e);
            fx = dsub(fx, dmul(f, dx));
            fy = dsub(fy, dmul(f, dy));
            fz = dsub(fz, dmul(f, dz));
        }
        const double F[3] = {fx, fy, fz};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const size_t o = static_cast<size_t>(k) * n + i;
            force[o] = F[k];
            if (kick_vel) kick_vel[o] = dadd(kick_vel[o], ddiv(dmul(half_dt, F[k]), mass[i]));
        }
    }
    ins = warp_sum_u64(ins);
    if ((threadIdx.x & 31) == 0 && ins) atomicAdd(inside, ins);
}

// Variant 2 of k_force_fp64, the same sums without a branch per entry: the row is read a quad (4 entries) at a
// time, one quad ahead with the streaming hint, the quad's four neighbour positions are gathered together, and
// every entry's terms are evaluated and masked (an exact 0.0 outside r_c and for the row's padding). Own and
// reverse entries take one form: the reverse pair's -F(j, i) dx(j, i) equals +F dx(i, j), since min_image is
// odd (round() and the |d| <= L/4 shortcut are symmetric) and IEEE subtraction antisymmetric, so each sum sees
// the reference's nonzero terms in the reference's order; a masked 0.0 leaves a sum unchanged because a sum
// that starts at +0.0 never becomes -0.0.
template <bool kTerms>
__global__ void __launch_bounds__(128) k_force_fp64_quads(const double4* __restrict__ pos, int n, Box box, LJ lj,
                                                          const uint32_t* __restrict__ rows, int cap,
                                                          const int2* __restrict__ counts, double* __restrict__ force,
                                                          unsigned long long* __restrict__ inside,
                                                          double* __restrict__ kick_vel, const double* __restrict__ mass,
                                                          double half_dt, const long long* __restrict__ half_off,
                                                          double* __restrict__ pair_r2, long long rec_cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long ins = 0;
    if (i < n) {
        const double4 pi = pos[i];
        const int2 c = counts[i];
        const int m = c.x + c.y;
        const int quads = (m + 3) >> 2;
        const long long pb = pair_r2 ? half_off[i] : 0;
        double fx = 0.0, fy = 0.0, fz = 0.0;
        const uint4* rq = reinterpret_cast<const uint4*>(rows) + static_cast<size_t>(i >> 5) * (cap >> 2) * 32 + (i & 31);
        uint4 nq = make_uint4(0, 0, 0, 0);
        if (quads > 0) nq = __ldcs(rq);
        for (int q = 0; q < quads; ++q) {
            const uint4 eq = nq;
            if (q + 1 < quads) nq = __ldcs(rq + 32 * (q + 1));
            const uint32_t ent[4] = {eq.x, eq.y, eq.z, eq.w};
            double4 pj[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) pj[u] = pos[4 * q + u < m ? static_cast<int>(ent[u] & kIndexMask) : 0];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int sl = 4 * q + u;
                const double dx = min_image(dsub(pi.x, pj[u].x), box);
                const double dy = min_image(dsub(pi.y, pj[u].y), box);
                const double dz = min_image(dsub(pi.z, pj[u].z), box);
                const double r2 = norm2(dx, dy, dz);
                const bool in = sl < m && r2 < lj.rc2;
                double f, e;
                pair_terms(in ? r2 : 1.0, lj, f, e);
                fx = dadd(fx, in ? dmul(f, dx) : 0.0);
                fy = dadd(fy, in ? dmul(f, dy) : 0.0);
                fz = dadd(fz, in ? dmul(f, dz) : 0.0);
                if (sl < c.x) {
                    ins += in ? 1u : 0u;
                    if (pair_r2) store_pair_rec<kTerms>(pair_r2, pb + sl, r2, f, e, in, rec_cap);
                }
            }
        }
        const double F[3] = {fx, fy, fz};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const size_t o = static_cast<size_t>(k) * n + i;
            force[o] = F[k];
            if (kick_vel) kick_vel[o] = dadd(kick_vel[o], ddiv(dmul(half_dt, F[k]), mass[i]));
        }
    }
    ins = warp_sum_u64(ins);
    if ((threadIdx.x & 31) == 0 && ins) atomicAdd(inside, ins);
}

constexpr int kEnergyWarps = 4;  // warps per block of the blocked kinetic-energy sums

// The inner loop of deterministicSum (include/Parallel.hpp:43-46) over the (pairEnergy, pairVirial) array, whose
// terms are recomputed here from the r^2 records the force kernel stored: block b sums pairs
// [1024 b, 1024 b + 1024) from 0.0 one after another, a pair outside the cutoff adding 0.0 as the reference's
// zero entries do. One lane per block, so a warp advances 32 blocks' ordered sums together; the warp stages 32
// consecutive records of each of its blocks in shared memory at a time (coalesced 256-byte loads), and each lane
// then evaluates and adds its block's 32 (the evaluations are independent of the sums, so they overlap).
constexpr int kPairSumWarps = 4;
// The pair count is rec_cap, or, in a CUDA graph (where it is known only on the device), read from *pair_count
// (the step's copy of the list's count, so a rebuild for the next step cannot change it under the sums) and capped
// at rec_cap, the records' buffer size; the grid then covers rec_cap. The block count goes to *nblocks_out for
// k_sum_pair_blocks.
__global__ void __launch_bounds__(32 * kPairSumWarps) k_pair_block_sums(const double* __restrict__ pair_r2,
                                                                        const long long* __restrict__ pair_count,
                                                                        long long rec_cap, LJ lj,
                                                                        double2* __restrict__ block_sums,
                                                                        int* __restrict__ nblocks_out) {
    __shared__ double tile[kPairSumWarps][32][33];
    const long long count = pair_count ? *pair_count : rec_cap;
    const long long pairs = count < rec_cap ? count : rec_cap;
    const int nblocks = static_cast<int>((pairs + kChunk - 1) / kChunk);
    if (blockIdx.x == 0 && threadIdx.x == 0) *nblocks_out = nblocks;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b0 = (blockIdx.x * kPairSumWarps + warp) * 32;  // this warp's first block
    if (b0 >= nblocks) return;
    double(*t)[33] = tile[warp];
    const int b = b0 + lane;
    const long long k0 = static_cast<long long>(b) * kChunk;
    const int m = b < nblocks ? static_cast<int>(pairs - k0 < kChunk ? pairs - k0 : kChunk) : 0;
    double se = 0.0, sw = 0.0;
    for (int c = 0; c < kChunk; c += 32) {
        __syncwarp();
        for (int r = 0; r < 32; ++r) {  // row r: records [c, c + 32) of block b0 + r, lane = record
            const long long k = static_cast<long long>(b0 + r) * kChunk + c + lane;
            t[r][lane] = b0 + r < nblocks && k < pairs ? __ldcs(pair_r2 + k) : lj.rc2;
        }
        __syncwarp();
        const int e = m - c < 32 ? m - c : 32;
#pragma unroll 4
        for (int u = 0; u < e; ++u) {
            const double r2 = t[lane][u];
            const bool in = r2 < lj.rc2;
            double f, en;
            pair_terms(in ? r2 : 1.0, lj, f, en);
            se = dadd(se, in ? en : 0.0);
            sw = dadd(sw, in ? dmul(f, r2) : 0.0);
        }
    }
    if (b < nblocks) block_sums[b] = make_double2(se, sw);
}

// k_pair_block_sums over (pairEnergy, pairVirial) records (the force kernels' `terms` form): the same ordered
// block sums, each lane adding its block's staged terms, with the same device pair count and block-count report.
constexpr int kPairSumWarpsTerms = 2;
__global__ void __launch_bounds__(32 * kPairSumWarpsTerms) k_pair_block_sums_terms(
    const double2* __restrict__ pair_ew, const long long* __restrict__ pair_count, long long rec_cap,
    double2* __restrict__ block_sums, int* __restrict__ nblocks_out) {
    __shared__ double2 tile[kPairSumWarpsTerms][32][33];
    const long long count = pair_count ? *pair_count : rec_cap;
    const long long pairs = count < rec_cap ? count : rec_cap;
    const int nblocks = static_cast<int>((pairs + kChunk - 1) / kChunk);
    if (blockIdx.x == 0 && threadIdx.x == 0) *nblocks_out = nblocks;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b0 = (blockIdx.x * kPairSumWarpsTerms + warp) * 32;  // this warp's first block
    if (b0 >= nblocks) return;
    double2(*t)[33] = tile[warp];
    const int b = b0 + lane;
    const long long k0 = static_cast<long long>(b) * kChunk;
    const int m = b < nblocks ? static_cast<int>(pairs - k0 < kChunk ? pairs - k0 : kChunk) : 0;
    double se = 0.0, sw = 0.0;
    for (int c = 0; c < kChunk; c += 32) {
        __syncwarp();
        for (int r = 0; r < 32; ++r) {  // row r: records [c, c + 32) of block b0 + r, lane = record
            const long long k = static_cast<long long>(b0 + r) * kChunk + c + lane;
            t[r][lane] = b0 + r < nblocks && k < pairs ? pair_ew[k] : make_double2(0.0, 0.0);
        }
        __syncwarp();
        const int e = m - c < 32 ? m - c : 32;
        for (int u = 0; u < e; ++u) {
            const double2 x = t[lane][u];
            se = dadd(se, x.x);
            sw = dadd(sw, x.y);
        }
    }
    if (b < nblocks) block_sums[b] = make_double2(se, sw);
}

// The outer loop of deterministicSum (include/Parallel.hpp:52-56): block sums added in order from 0.0.
// One warp: the lanes stage 256 values at a time in shared memory (the next chunk's loads in flight while
// lane 0 adds the current one, one value after another, reading eight ahead of the adds).
__device__ __forceinline__ void sum_blocks(const double2* __restrict__ block_sums, int nblocks,
                                           double* __restrict__ out) {
    constexpr int kStage = 256;
    __shared__ double2 stage[kStage];
    const int lane = threadIdx.x & 31;
    double2 next[kStage / 32];
    auto fetch = [&](int c) {
#pragma unroll
        for (int q = 0; q < kStage / 32; ++q) {
            const int k = c * kStage + q * 32 + lane;
            next[q] = k < nblocks ? block_sums[k] : make_double2(0.0, 0.0);
        }
    };
    double se = 0.0, sw = 0.0;
    const int chunks = (nblocks + kStage - 1) / kStage;
    if (chunks > 0) fetch(0);
    for (int c = 0; c < chunks; ++c) {
        __syncwarp();
#pragma unroll
        for (int q = 0; q < kStage / 32; ++q) stage[q * 32 + lane] = next[q];
        __syncwarp();
        if (c + 1 < chunks) fetch(c + 1);
        if (lane == 0) {
            const int m = nblocks - c * kStage < kStage ? nblocks - c * kStage : kStage;
            int t = 0;
            for (; t + 8 <= m; t += 8) {
                double2 x[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) x[u] = stage[t + u];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    se = dadd(se, x[u].x);
                    sw = dadd(sw, x[u].y);
                }
            }
            for (; t < m; ++t) {
                const double2 x = stage[t];
                se = dadd(se, x.x);
                sw = dadd(sw, x.y);
            }
        }
    }
    if (lane == 0) {
        out[0] = se;
        out[1] = sw;
    }
}

__global__ void k_sum_blocks(const double2* __restrict__ block_sums, int nblocks, double* __restrict__ out) {
    sum_blocks(block_sums, nblocks, out);
}

// sum_blocks over the 1024-pair blocks of k_pair_block_sums, as many as it reported
__global__ void k_sum_pair_blocks(const double2* __restrict__ block_sums, const int* __restrict__ nblocks,
                                  double* __restrict__ out) {
    sum_blocks(block_sums, *nblocks, out);
}

// The step's pair count into the slot its energy sums read
__global__ void k_copy_count(const long long* __restrict__ from, long long* __restrict__ to) { *to = *from; }

// In a CUDA graph's list rebuild: the new list's pair count must fit the energy records' buffer, else the graph's
// run repeats its steps on the host path (state[1], as k_build_done reports a row overflow)
__global__ void k_pairs_fit(const long long* __restrict__ pair_count, long long rec_cap, int* __restrict__ state) {
    if (*pair_count > rec_cap) state[1] = 1;
}

// ---- kinetic energy -----------------------------------------------------------------------------------

// 0.5 * m * (vx^2 + vy^2 + vz^2) over particles [1024 b, 1024 b + 1024) summed in order (src/System.cpp:67-76)
__global__ void k_kinetic_blocks(const double* __restrict__ vel, const double* __restrict__ mass, int n,
                                 double2* __restrict__ block_sums, int nblocks) {
    extern __shared__ double2 sm_ke[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int blk = blockIdx.x * kEnergyWarps + warp;
    if (blk >= nblocks) return;
    double* v = reinterpret_cast<double*>(sm_ke + warp * (kChunk / 2));
    const int i0 = blk * kChunk;
    const int m = n - i0 < kChunk ? n - i0 : kChunk;
    for (int t = lane; t < m; t += 32) {
        const int i = i0 + t;
        const double vx = vel[i], vy = vel[static_cast<size_t>(n) + i], vz = vel[2 * static_cast<size_t>(n) + i];
        v[t] = dmul(dmul(0.5, mass[i]), norm2(vx, vy, vz));
    }
    __syncwarp();
    if (lane == 0) {
        double s = 0.0;
        for (int t = 0; t < m; ++t) s = dadd(s, v[t]);
        block_sums[blk] = make_double2(s, 0.0);
    }
}

// ---- integration --------------------------------------------------------------------------------------

// VelocityVerletIntegrator::kickAndDrift (src/Integrator.cpp:32-53): v += (dt/2) f / m, then
// r = wrap(r + dt v). Fused with NeighbourList::update's staleness test (src/NeighbourList.cpp:24-30) against
// the reference positions of the last build, which sets *stale when any |d|^2 > skin^2 / 4.
__global__ void k_kick_drift(double4* __restrict__ pos, double* __restrict__ vel, const double* __restrict__ force,
                             const double* __restrict__ mass, int n, double half_dt, double dt, Box box,
                             const double4* __restrict__ ref_pos, double max_disp2, int* __restrict__ stale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
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
}

// NeighbourList::update's test on its own (src/NeighbourList.cpp:24-30)
__global__ void k_skin_check(const double4* __restrict__ pos, int n, Box box, const double4* __restrict__ ref_pos,
                             double max_disp2, int* __restrict__ stale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = pos[i], r = ref_pos[i];
    const double dx = min_image(dsub(p.x, r.x), box);
    const double dy = min_image(dsub(p.y, r.y), box);
    const double dz = min_image(dsub(p.z, r.z), box);
    if (norm2(dx, dy, dz) > max_disp2) *stale = 1;
}

// VelocityVerletIntegrator::kick (src/Integrator.cpp:55-71)
__global__ void k_kick(double* __restrict__ vel, const double* __restrict__ force, const double* __restrict__ mass,
                       int n, double half_dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double m = mass[i];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const size_t o = static_cast<size_t>(k) * n + i;
        vel[o] = dadd(vel[o], ddiv(dmul(half_dt, force[o]), m));
    }
}

// ---- thermostats ----------------------------------------------------------------------------------------

// Scale factors computed on the device from the device kinetic energy, so no host round trip is needed.
// scale[0] = factor, scale[1] = 1 to apply or 0 to leave the velocities alone.
// rescaleVelocities (src/Thermostat.cpp:17-30)
__global__ void k_rescale_factor(const double* __restrict__ ke, double dof, double target, double* __restrict__ scale) {
    const double t = ddiv(dmul(2.0, ke[0]), dof);  // System::temperature (src/System.cpp:79-82)
    if (t <= 0.0) {
        scale[1] = 0.0;
        return;
    }
    scale[0] = __dsqrt_rn(ddiv(target, t));
    scale[1] = 1.0;
}

// BussiThermostat::apply's velocity scale, equation A7 (src/Thermostat.cpp:40-57), for kinetic > 0
__device__ __forceinline__ double bussi_scale(double kinetic, double dof, double temperature, double c, double r1,
                                              double chi2) {
    const double target = dmul(dmul(0.5, dof), temperature);
    const double omc = dsub(1.0, c);
    const double t1 = dmul(omc, dsub(ddiv(dmul(target, dadd(chi2, dmul(r1, r1))), dof), kinetic));
    const double t2 = dmul(dmul(2.0, r1), __dsqrt_rn(dmul(dmul(dmul(ddiv(target, dof), kinetic), omc), c)));
    const double nk = dadd(dadd(kinetic, t1), t2);
    return __dsqrt_rn(ddiv(nk, kinetic));
}

// BussiThermostat::apply (src/Thermostat.cpp:36-58), with r1 and chi2 given
__global__ void k_bussi_factor(const double* __restrict__ ke, double dof, double temperature, double c,
                               const double* __restrict__ r1p, const double* __restrict__ chi2p,
                               double* __restrict__ scale) {
    const double kinetic = ke[0];
    if (kinetic <= 0.0) {
        scale[1] = 0.0;
        return;
    }
    scale[0] = bussi_scale(kinetic, dof, temperature, c, r1p[0], chi2p[0]);
    scale[1] = 1.0;
}

__global__ void k_scale_velocities(double* __restrict__ vel, long long count, const double* __restrict__ scale) {
    if (scale[1] == 0.0) return;
    const double s = scale[0];
    for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < count;
         t += static_cast<long long>(gridDim.x) * blockDim.x)
        vel[t] = dmul(vel[t], s);
}

// ---- g(r) -------------------------------------------------------------------------------------------------

// RadialDistribution::sample (src/RadialDistribution.cpp:11-30): every half-list pair with r^2 < r_max^2
// adds one to bin (size_t)(sqrt(r^2) / binWidth). Counts are integers, so atomics keep the result exact.
// A bin index of `bins` or more (possible only through rounding at r just under r_max) is dropped: the
// reference would write past its histogram there.
__global__ void k_rdf_sample(const double4* __restrict__ pos, int n, Box box, const uint32_t* __restrict__ rows,
                             int cap, const int2* __restrict__ counts, double rmax2, double bin_width, int bins,
                             unsigned long long* __restrict__ hist) {
    extern __shared__ unsigned int sm_hist[];
    for (int b = threadIdx.x; b < bins; b += blockDim.x) sm_hist[b] = 0;
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double4 pi = pos[i];
        const int own = counts[i].x;
        for (int s = 0; s < own; ++s) {
            const double4 pj = pos[rows[row_index(i, s, cap)] & kIndexMask];
            const double dx = min_image(dsub(pi.x, pj.x), box);
            const double dy = min_image(dsub(pi.y, pj.y), box);
            const double dz = min_image(dsub(pi.z, pj.z), box);
            const double r2 = norm2(dx, dy, dz);
            if (r2 < rmax2) {
                const unsigned long long b = __double2ull_rz(ddiv(__dsqrt_rn(r2), bin_width));
                if (b < static_cast<unsigned long long>(bins)) atomicAdd(&sm_hist[b], 1u);
            }
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < bins; b += blockDim.x)
        if (sm_hist[b]) atomicAdd(&hist[b], static_cast<unsigned long long>(sm_hist[b]));
}

// ---- O(N^2) forces ----------------------------------------------------------------------------------------

// computeForces(System&) (src/Forcefield.cpp:39-78). Particle p receives, in the reference's loop order,
// -F(i, p) for i = 0 .. p-1 and then +F(p, j) for j = p+1 .. n-1; pairs at or beyond the cutoff are skipped.
__global__ void k_force_all_pairs(const double4* __restrict__ pos, int n, Box box, LJ lj, double* __restrict__ force) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double4 pp = pos[p];
    double f[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < n; ++i) {
        if (i == p) continue;
        const double4 a = i < p ? pos[i] : pp;
        const double4 b = i < p ? pp : pos[i];
        const double dx = min_image(dsub(a.x, b.x), box);
        const double dy = min_image(dsub(a.y, b.y), box);
        const double dz = min_image(dsub(a.z, b.z), box);
        const double r2 = norm2(dx, dy, dz);
        if (r2 >= lj.rc2) continue;
        double fr, e;
        pair_terms(r2, lj, fr, e);
        if (i < p) {
            f[0] = dsub(f[0], dmul(fr, dx));
            f[1] = dsub(f[1], dmul(fr, dy));
            f[2] = dsub(f[2], dmul(fr, dz));
        } else {
            f[0] = dadd(f[0], dmul(fr, dx));
            f[1] = dadd(f[1], dmul(fr, dy));
            f[2] = dadd(f[2], dmul(fr, dz));
        }
    }
    force[p] = f[0];
    force[static_cast<size_t>(n) + p] = f[1];
    force[2 * static_cast<size_t>(n) + p] = f[2];
}

// The all-pairs potential, virial and inside count: one sequential sum over pairs (i, j > i) in the
// reference's loop order, started from 0.0. One warp: lanes evaluate 32 pairs at a time, lane 0 adds them.
__global__ void k_energy_all_pairs(const double4* __restrict__ pos, int n, Box box, LJ lj, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    double pe = 0.0, w = 0.0, ins = 0.0;
    for (int i = 0; i < n; ++i) {
        const double4 pi = pos[i];
        for (int j0 = i + 1; j0 < n; j0 += 32) {
            const int j = j0 + lane;
            double e = 0.0, vir = 0.0;
            bool in = false;
            if (j < n) {
                const double4 pj = pos[j];
                const double dx = min_image(dsub(pi.x, pj.x), box);
                const double dy = min_image(dsub(pi.y, pj.y), box);
                const double dz = min_image(dsub(pi.z, pj.z), box);
                const double r2 = norm2(dx, dy, dz);
                if (r2 < lj.rc2) {
                    double fr;
                    pair_terms(r2, lj, fr, e);
                    vir = dmul(fr, r2);
                    in = true;
                }
            }
            const unsigned mask = __ballot_sync(0xffffffffu, in);
            const int m = n - j0 < 32 ? n - j0 : 32;
            for (int t = 0; t < m; ++t) {
                const double et = __shfl_sync(0xffffffffu, e, t);
                const double wt = __shfl_sync(0xffffffffu, vir, t);
                if (lane == 0 && ((mask >> t) & 1u)) {
                    pe = dadd(pe, et);
                    w = dadd(w, wt);
                    ins = dadd(ins, 1.0);
                }
            }
        }
    }
    if (lane == 0) {
        out[0] = pe;
        out[1] = w;
        out[2] = ins;
    }
}

}  // namespace md
