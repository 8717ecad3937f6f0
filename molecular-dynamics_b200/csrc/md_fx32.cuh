// MD_PREC_FX32: float pair terms for the pairs whose force is small, double pair terms on exact fixed-point
// separations for the close pairs, 64-bit fixed-point sums.
//
// Why the split: a float pair term carries a relative error of a few 1e-7 (the force goes as r^-14, so the
// rounding of r^2 alone is amplified sevenfold). That is below 1e-6 of a particle's net force only where the
// pair force itself is small. Pairs beyond 1.2 sigma have |F| <= 2.4 eps/sigma; the few closer pairs (about one in
// six of a row) carry forces up to 1e2 and, evaluated in float, leave 60 % of particles above 1e-6 relative
// error. So every row is reordered once per list build: entries whose pair was closer than (1.2 sigma + skin)
// at the build come first, and its first two groups of 8 are evaluated in double on the 32-bit fixed-point frames
// (2^-28 units) of MD_PREC_FX64, whose integer differences are exact separations; the rest are evaluated in float
// on the float frames of MD_PREC_FP32FX, with its pinned operation sequence. Between rebuilds every particle
// stays within skin/2 of its build position, so a pair evaluated in float is never closer than near_sigma sigma.
//
// Sums: every group of 8 entries is added into 64-bit fixed point (forces at 2^-32, energy and virial at 2^-30),
// so the result does not depend on the launch shape.
#pragma once

#include "md_common.cuh"
#include "md_fp32.cuh"
#include "md_fx64.cuh"

namespace md {

constexpr int kFx32NearGroups = 2;  // row groups of 8 entries evaluated in double

// Near-first rows. For particle i: the entries of its row whose pair was closer than sqrt(near2) at the list
// build, in their row order, then sentinel entries up to the next multiple of 8 that the remaining entries do not
// fill, then the remaining entries in reverse row order; counts_nf[i] = (the first kFx32NearGroups groups, or all
// of a shorter row; all groups). Every row gets the same number of double groups, so the warps of the force kernel
// never split between the two paths; a row with more than 8 kFx32NearGroups near entries keeps the closest ones
// there and moves the farthest to the float groups (rare: about 12 pairs lie closer than 1.5 sigma at liquid
// density, and those moved are the farthest of them).
// The classification uses ref_frames, the float frames of the list's reference positions (the positions of the
// build), with the float offsets of the entries' cell codes. Rows keep the interleaved layout and capacity of the
// list's rows. A warp builds the rows of its 32 particles in shared memory (stride cap + 1 entries, so the lanes'
// rows start in different banks) and writes them out a quad per lane at a time, which is one 512-byte store per
// warp and quad.
__global__ void k_rows_near_first(const float4* __restrict__ ref_frames, int n, CellOffsets offs, float near2,
                                  const uint32_t* __restrict__ rows, int cap, const int2* __restrict__ counts,
                                  uint32_t* __restrict__ rows_nf, int2* __restrict__ counts_nf) {
    extern __shared__ uint32_t s_rows[];
    __shared__ float4 s_off[32];
    if (threadIdx.x < 32) s_off[threadIdx.x] = offs.off[threadIdx.x];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = (blockIdx.x * (blockDim.x >> 5) + warp) * 32 + lane;
    uint32_t* my = s_rows + static_cast<size_t>(threadIdx.x) * (cap + 1);
    int m = 0, front = 0;
    if (i < n) {
        const float4 qi = ref_frames[i];
        const int2 c = counts[i];
        m = c.x + c.y;
        int back = (m + 7) & ~7;
        for (int s = 0; s < m; s += 4) {
            const uint4 q = row_quad(rows, i, s >> 2, cap);
            const uint32_t ent[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (s + u >= m) break;
                const uint32_t e = ent[u];
                float dx, dy, dz;
                const float r2 = float_separation(qi, ref_frames[e & kIndexMask], s_off[e >> kCodeShift], dx, dy, dz);
                if (r2 < near2)
                    my[front++] = e;
                else
                    my[--back] = e;
            }
        }
        // more near entries than the double groups hold: move the farthest to the float part, one at a time
        while (front > 8 * kFx32NearGroups) {
            int far_k = 0;
            float far_r2 = -1.0f;
            for (int k = 0; k < front; ++k) {
                const uint32_t e = my[k];
                float dx, dy, dz;
                const float r2 = float_separation(qi, ref_frames[e & kIndexMask], s_off[e >> kCodeShift], dx, dy, dz);
                if (r2 > far_r2) {
                    far_r2 = r2;
                    far_k = k;
                }
            }
            const uint32_t e = my[far_k];
            my[far_k] = my[--front];
            my[--back] = e;
        }
        const uint32_t pad = static_cast<uint32_t>(n) | (kSentinelCode << kCodeShift);
        for (int s = front; s < back; ++s) my[s] = pad;
        const int groups = ((m + 7) & ~7) >> 3;
        counts_nf[i] = make_int2(groups < kFx32NearGroups ? groups : kFx32NearGroups, groups);
    }
    __syncwarp();
    const int quads = ((m + 7) & ~7) >> 2;
    uint4* out = reinterpret_cast<uint4*>(rows_nf);
    for (int q = 0; q < quads; ++q)
        out[(static_cast<size_t>(i >> 5) * (cap >> 2) + q) * 32 + (i & 31)] =
            make_uint4(my[4 * q], my[4 * q + 1], my[4 * q + 2], my[4 * q + 3]);
}

// Thread per particle over its near-first row on a resident grid (each thread takes particles i, i + grid, ...):
// groups [0, near_groups) in double on the fixed-point frames (fx64_group, MD_PREC_FX64's sequence), the rest in
// float on the float frames (float_group, MD_PREC_FP32FX's sequence); row quads prefetched a group ahead with
// streaming loads; the fused closing kick, kinetic energy and, with kick.pos_out, the next step's kick and drift
// writing both kinds of frames, as in the other float modes.
template <bool kEnergy>
__global__ void __launch_bounds__(128, 5) k_force_fx32(const int4* __restrict__ iframes, const float4* __restrict__ frames,
                                                    const double4* __restrict__ pos, int n, Box box, Fx64LJ dlj,
                                                    FloatLJ flj, FixedOffsets ioffs, CellOffsets foffs,
                                                    const uint32_t* __restrict__ rows, int cap,
                                                    const int2* __restrict__ counts, double* __restrict__ force,
                                                    unsigned long long* __restrict__ acc, KickArgs kick) {
    // the 32 codes' image offsets: fixed-point (x, y) pairs and z, float (x, y) pairs and z
    __shared__ __align__(16) int s_io[4][32];
    __shared__ __align__(16) float s_fo[4][32];
    if (threadIdx.x < 32) {
        const int4 o = ioffs.off[threadIdx.x];
        reinterpret_cast<int2*>(s_io[0])[threadIdx.x] = make_int2(o.x, o.y);
        s_io[2][threadIdx.x] = o.z;
        const float4 f = foffs.off[threadIdx.x];
        reinterpret_cast<float2*>(s_fo[0])[threadIdx.x] = make_float2(f.x, f.y);
        s_fo[2][threadIdx.x] = f.z;
    }
    __syncthreads();
    if (kick.frames_out && blockIdx.x == 0 && threadIdx.x == 0)
        kick.frames_out[n] = make_float4(kSentinelCoord, kSentinelCoord, kSentinelCoord, 0.0f);
    const int2* s_ixy = reinterpret_cast<const int2*>(s_io[0]);
    const int* s_iz = s_io[2];
    const float2* s_fxy = reinterpret_cast<const float2*>(s_fo[0]);
    const float* s_fz = s_fo[2];
    long long e_fx = 0, w_fx = 0, k_fx = 0;
    unsigned ins = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int4 qi = iframes[i];
        const float4 fi = frames[i];
        const int2 c = counts[i];
        const int near_groups = c.x, groups = c.y;
        FloatAcc<true, kEnergy> a;
        const uint4* rq = reinterpret_cast<const uint4*>(rows) + static_cast<size_t>(i >> 5) * (cap >> 2) * 32 + (i & 31);
        uint4 n0 = make_uint4(0, 0, 0, 0), n1 = n0;
        if (groups > 0) {
            n0 = __ldcs(rq);
            n1 = __ldcs(rq + 32);
        }
        for (int g = 0; g < groups; ++g) {
            const uint4 e0 = n0, e1 = n1;
            rq += 64;
            if (g + 1 < groups) {
                n0 = __ldcs(rq);
                n1 = __ldcs(rq + 32);
            }
            if (g < near_groups) {
                unsigned gin = 0;
                bool shell = false;
                DoubleGroupSums gs =
                    fx64_group<kEnergy, false>(e0, e1, qi, iframes, s_ixy, s_iz, pos, i, box, dlj, gin, &shell);
                if (shell) gs = fx64_group_exact<kEnergy>(e0, e1, qi, iframes, s_ixy, s_iz, pos, i, box, dlj, &gin);
                ins += gin;
                a.add_group(gs.x, gs.y, gs.z, gs.e, gs.w, e_fx, w_fx);
            } else {
                const GroupSums gs = float_group<kEnergy>(
                    e0, e1, flj,
                    [=](uint32_t e, float& dx, float& dy, float& dz) {
                        const uint32_t k = e >> kCodeShift;
                        const float2 oxy = s_fxy[k];
                        return float_separation(fi, frames[e & kIndexMask], make_float4(oxy.x, oxy.y, s_fz[k], 0.0f),
                                                dx, dy, dz);
                    },
                    [=](uint32_t e) { return exact_inside(pos[i], pos[e & kIndexMask], box, flj.rc2d); }, ins);
                a.add_group_fine(gs.x, gs.y, gs.z, gs.e, gs.w, e_fx, w_fx);
            }
        }
        k_fx += a.finish(i, n, force, kick);
    }
    if (kEnergy || kick.vel) flush_sums(e_fx, w_fx, ins, k_fx, acc);
}

}  // namespace md
