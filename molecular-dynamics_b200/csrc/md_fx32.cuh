// MD_PREC_FX32: exact fixed-point separations, float pair terms for the pairs whose force is small, double pair
// terms for the close pairs, 64-bit fixed-point sums.
//
// Why the split: a float pair term carries a relative error of a few 1e-7 (the force goes as r^-14, so the
// rounding of r^2 alone is amplified sevenfold). That is below 1e-6 of a particle's net force only where the
// pair force itself is small. Pairs beyond about 1.3 sigma have |F| <= 2.3 eps/sigma; the few closer pairs (about
// one in six of a row) carry forces up to 1e2 and, evaluated in float, leave 60 % of particles above 1e-6
// relative error. So every row is reordered once per list build: entries whose pair was closer than
// (near_sigma sigma + skin) at the build come first and are evaluated in double (as MD_PREC_FX64 does), the rest
// in float. Between rebuilds every particle stays within skin/2 of its build position, so a pair evaluated in
// float is never closer than near_sigma sigma.
//
// Separations of both kinds come from the 32-bit fixed-point frames (2^-28 units) of MD_PREC_FX64 by integer
// subtraction, so they are exact; the float path rounds each component once when it converts it. Sums: every
// group of 8 entries is added into 64-bit fixed point (forces at 2^-32, energy and virial at 2^-30), so the
// result does not depend on the launch shape.
#pragma once

#include "md_common.cuh"
#include "md_fp32.cuh"
#include "md_fx64.cuh"

namespace md {

// Near-first rows: for particle i, the entries of its row whose pair was within sqrt(near2) at the list build
// (the reference positions ref_pos, with the reference's minimum image) in their row order, then sentinel
// entries up to the next multiple of 8 that the remaining entries do not fill, then the remaining entries in
// reverse row order. counts_nf[i] = (groups holding a near entry, all groups). Rows keep the interleaved layout and
// capacity of the list's rows (the row length, padded to a multiple of 8, is unchanged).
__global__ void k_rows_near_first(const double4* __restrict__ ref_pos, int n, Box box, double near2,
                                  const uint32_t* __restrict__ rows, int cap, const int2* __restrict__ counts,
                                  uint32_t* __restrict__ rows_nf, int2* __restrict__ counts_nf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 pi = ref_pos[i];
    const int2 c = counts[i];
    const int m = c.x + c.y;
    const int padded = (m + 7) & ~7;
    int front = 0, back = padded;
    for (int s = 0; s < m; s += 4) {
        const uint4 q = row_quad(rows, i, s >> 2, cap);
        const uint32_t ent[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (s + u >= m) break;
            const uint32_t e = ent[u];
            const double4 pj = ref_pos[e & kIndexMask];
            const double dx = min_image(dsub(pi.x, pj.x), box);
            const double dy = min_image(dsub(pi.y, pj.y), box);
            const double dz = min_image(dsub(pi.z, pj.z), box);
            if (norm2(dx, dy, dz) < near2)
                rows_nf[row_index(i, front++, cap)] = e;
            else
                rows_nf[row_index(i, --back, cap)] = e;
        }
    }
    const uint32_t pad = static_cast<uint32_t>(n) | (kSentinelCode << kCodeShift);
    for (int s = front; s < back; ++s) rows_nf[row_index(i, s, cap)] = pad;
    counts_nf[i] = make_int2((front + 7) >> 3, padded >> 3);
}

// One 8-entry group in float from fixed-point frames: the exact integer separation (q_i - q_j) + offset, each
// component rounded once to float (__int2float_rn) and kept in frame units, then float_pair with constants in
// frame units (frame_units_lj): r^2 and 1/r^2 are the length-unit values times 2^56 and 2^-56 exactly, the pair's
// F/r times 2^-56 and its force times 2^-28, its energy and virial unchanged. Pairs in
// the shell around r_c where the float r^2 could misclassify them are flagged through *shell; the caller then runs
// the group again with kExact, where the reference's exact double test decides them (the same operations in the
// same order either way).
template <bool kEnergy, bool kExact>
__device__ __forceinline__ GroupSums fx32_float_group(const uint4& e0, const uint4& e1, const int4& qi,
                                                      const int4* __restrict__ frames, const int2* s_xy, const int* s_z,
                                                      const double4* __restrict__ pos, int i, const Box& box,
                                                      const FloatLJ& lj, unsigned& c, bool* shell) {
    const uint32_t ent[8] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
    GroupSums g;
    bool sh = false;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const uint32_t e = ent[u];
        const uint32_t code = e >> kCodeShift;
        const bool pad = code == kSentinelCode;
        const int j = pad ? 0 : static_cast<int>(e & kIndexMask);
        const int4 qj = frames[j];
        const int2 oxy = s_xy[code];
        const int sx = static_cast<int>(static_cast<unsigned>(qi.x) - static_cast<unsigned>(qj.x) + static_cast<unsigned>(oxy.x));
        const int sy = static_cast<int>(static_cast<unsigned>(qi.y) - static_cast<unsigned>(qj.y) + static_cast<unsigned>(oxy.y));
        const int sz = static_cast<int>(static_cast<unsigned>(qi.z) - static_cast<unsigned>(qj.z) + static_cast<unsigned>(s_z[code]));
        // in frame units (2^-28): lj holds sigma^2, r_c^2 and the band scaled by 2^56, so every product below
        // has the mantissa it would have in length units, scaled by an exact power of two
        const float dx = __int2float_rn(sx);
        const float dy = __int2float_rn(sy);
        const float dz = __int2float_rn(sz);
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, __fmul_rn(dz, dz)));
        bool in = !pad && r2 < lj.rc2;
        const bool near = !pad && fabsf(r2 - lj.rc2) < lj.band;
        if (kExact) {
            if (near) in = exact_inside(pos[i], pos[j], box, lj.rc2d);
        } else {
            sh |= near;
        }
        float_pair<kEnergy>(dx, dy, dz, in, pad ? 1.0f : r2, lj, g.x, g.y, g.z, g.e, g.w, c);
    }
    if (!kExact) *shell = sh;
    return g;
}

template <bool kEnergy>
__device__ __noinline__ GroupSums fx32_float_group_exact(const uint4 e0, const uint4 e1, const int4 qi,
                                                         const int4* __restrict__ frames, const int2* s_xy,
                                                         const int* s_z, const double4* __restrict__ pos, int i,
                                                         const Box box, const FloatLJ lj, unsigned* c) {
    unsigned k = 0;
    const GroupSums g = fx32_float_group<kEnergy, true>(e0, e1, qi, frames, s_xy, s_z, pos, i, box, lj, k, nullptr);
    *c = k;
    return g;
}

// Thread per particle over its near-first row on a resident grid (each thread takes particles i, i + grid, ...):
// groups [0, near_groups) in double (fx64_group, the MD_PREC_FX64 sequence), the rest in float
// (fx32_float_group); row quads prefetched a group ahead with streaming loads; the fused closing kick, kinetic
// energy and, with kick.pos_out, the next step's kick and drift writing fixed-point frames, as in the other
// float modes.
template <bool kEnergy>
__global__ void __launch_bounds__(128) k_force_fx32(const int4* __restrict__ frames, const double4* __restrict__ pos,
                                                    int n, Box box, Fx64LJ dlj, FloatLJ flj, FixedOffsets offs,
                                                    const uint32_t* __restrict__ rows, int cap,
                                                    const int2* __restrict__ counts, double* __restrict__ force,
                                                    unsigned long long* __restrict__ acc, KickArgs kick) {
    __shared__ __align__(16) int s_o[4][32];  // s_o[0..1]: the 32 codes' (x, y) offsets; s_o[2]: z
    if (threadIdx.x < 32) {
        const int4 o = offs.off[threadIdx.x];
        reinterpret_cast<int2*>(s_o[0])[threadIdx.x] = make_int2(o.x, o.y);
        s_o[2][threadIdx.x] = o.z;
    }
    __syncthreads();
    const int2* s_xy = reinterpret_cast<const int2*>(s_o[0]);
    const int* s_z = s_o[2];
    long long e_fx = 0, w_fx = 0, k_fx = 0;
    unsigned ins = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int4 qi = frames[i];
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
            unsigned gin = 0;
            bool shell = false;
            if (g < near_groups) {
                DoubleGroupSums gs =
                    fx64_group<kEnergy, false>(e0, e1, qi, frames, s_xy, s_z, pos, i, box, dlj, gin, &shell);
                if (shell) gs = fx64_group_exact<kEnergy>(e0, e1, qi, frames, s_xy, s_z, pos, i, box, dlj, &gin);
                a.add_group(gs.x, gs.y, gs.z, gs.e, gs.w, e_fx, w_fx);
            } else {
                GroupSums gs =
                    fx32_float_group<kEnergy, false>(e0, e1, qi, frames, s_xy, s_z, pos, i, box, flj, gin, &shell);
                if (shell) gs = fx32_float_group_exact<kEnergy>(e0, e1, qi, frames, s_xy, s_z, pos, i, box, flj, &gin);
                a.add_group_frame(gs.x, gs.y, gs.z, gs.e, gs.w, e_fx, w_fx);
            }
            ins += gin;
        }
        k_fx += a.finish(i, n, force, kick);
    }
    if (kEnergy || kick.vel) flush_sums(e_fx, w_fx, ins, k_fx, acc);
}

}  // namespace md
