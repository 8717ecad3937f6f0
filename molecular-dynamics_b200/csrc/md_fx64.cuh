// MD_PREC_FX64: exact separations from 32-bit fixed-point frames, pair terms in double, 64-bit fixed-point
// force sums. The float modes lose most of their accuracy to the rounding of the separation (the force goes
// as r^-14, so a relative error e of r becomes about 14 e of the force); here the separation of a pair is an
// integer difference of frames in units of 2^-28 (exact, wrapping modulo 2^32 like the hardware adds) and only
// its conversion to double rounds, so the per-particle force error against the FP64 path falls from about
// 1e-6 to about 2e-8 of the force. Frames are still gathered as 16 bytes per neighbour.
#pragma once

#include "md_common.cuh"
#include "md_fp32.cuh"

namespace md {

__global__ void k_frames_fixed(const double4* __restrict__ pos, int n, const int* __restrict__ cell_sorted, int ncps,
                               double cell, Box box, int4* __restrict__ frames) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    frames[i] = fixed_frame_of(pos[i], cell_sorted[i], ncps, cell, box);
}

// -d * cell for the 27 codes in frame units (zero for the others); cellq = round(cell * 2^28) on the host
struct FixedOffsets {
    int4 off[32];
};

struct Fx64LJ {
    LJ lj;
    double eps48;  // 48 eps
    double band;   // |r^2 - r_c^2| below this: decide inside/outside with the reference's exact test
};

// s * 2^-28 in double, exactly, without the conversion unit: the double with high word 0x43300000 and low word
// s ^ 0x80000000 is 2^52 + 2^31 + s, and one FMA scales it by 2^-28 and removes (2^52 + 2^31) 2^-28 = 16777224
// (every step exact, so the result is the exact value the int-to-double conversion and the scaling give)
__device__ __forceinline__ double fixed_to_double(int s) {
    const double m = __hiloint2double(0x43300000, s ^ static_cast<int>(0x80000000u));
    return __fma_rn(m, kFrameUnit, -16777224.0);
}

// Separation of a row entry from fixed-point frames: (q_i - q_j) + offset in wrapping 32-bit arithmetic, then
// exactly scaled to double; returns r^2
__device__ __forceinline__ double fixed_separation(const int4& qi, const int4& qj, const int4& o, double& dx, double& dy,
                                                   double& dz) {
    const int sx = static_cast<int>(static_cast<unsigned>(qi.x) - static_cast<unsigned>(qj.x) + static_cast<unsigned>(o.x));
    const int sy = static_cast<int>(static_cast<unsigned>(qi.y) - static_cast<unsigned>(qj.y) + static_cast<unsigned>(o.y));
    const int sz = static_cast<int>(static_cast<unsigned>(qi.z) - static_cast<unsigned>(qj.z) + static_cast<unsigned>(o.z));
    dx = fixed_to_double(sx);
    dy = fixed_to_double(sy);
    dz = fixed_to_double(sz);
    return __fma_rn(dx, dx, __fma_rn(dy, dy, dmul(dz, dz)));
}

// The hardware's approximate double reciprocal (PTX rcp.approx.ftz.f64), the seed of 1/r^2
__device__ __forceinline__ double rcp_approx64(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return y;
}

// One pair's terms in double with a pinned operation sequence: 1/r^2 from the approximate double reciprocal
// (relative error below 2^-19.9, measured on B200 over r^2 in [0.5, 8.5]) refined by two Newton steps (quadratic
// convergence leaves only the double roundings; one step would already be far below what the 2^-28 frames leave
// in the force, but measured 11 % slower as compiled, and the cubic form inv (1 + e + e^2) from one residual e,
// one FMA fewer, 2 % slower), then F/r = (48 eps sr6 - 24 eps) sr6 / r^2 and
// E = 4 eps sr6 (sr6 - 1) - shift
template <bool kEnergy>
__device__ __forceinline__ void fx64_pair(double dx, double dy, double dz, bool in, double r2, const Fx64LJ& p,
                                          double& gx, double& gy, double& gz, double& ge, double& gw,
                                          unsigned& ins) {
    double inv = rcp_approx64(r2);
    inv = __fma_rn(inv, __fma_rn(-r2, inv, 1.0), inv);
    inv = __fma_rn(inv, __fma_rn(-r2, inv, 1.0), inv);
    const double sr2 = dmul(p.lj.sig2, inv);
    const double sr6 = dmul(dmul(sr2, sr2), sr2);
    double fr = dmul(dmul(__fma_rn(p.eps48, sr6, -p.lj.eps24), sr6), inv);
    fr = in ? fr : 0.0;
    gx = __fma_rn(fr, dx, gx);
    gy = __fma_rn(fr, dy, gy);
    gz = __fma_rn(fr, dz, gz);
    if (kEnergy) {
        const double en = __fma_rn(dmul(p.lj.eps4, sr6), dsub(sr6, 1.0), -p.lj.shift);
        ge = dadd(ge, in ? en : 0.0);
        gw = __fma_rn(fr, r2, gw);
        ins += in ? 1u : 0u;
    }
}

// Sums of one 8-entry group in double
struct DoubleGroupSums {
    double x = 0.0, y = 0.0, z = 0.0, e = 0.0, w = 0.0;
};

// One 8-entry group of a row from fixed-point frames through fx64_pair (the image offset of code c is
// (s_xy[c], s_z[c])). Row padding entries carry code 31 and
// are masked (the sentinel's index is n: particle 0's frame is read instead). With kExact the pairs in the
// shell around r_c take the reference's exact test; without it the group runs branch-free and reports through
// *shell whether it holds such a pair, in which case the caller runs it again with kExact (the same sequence
// with the exact decision, so the same sums as a single exact pass).
template <bool kEnergy, bool kExact>
__device__ __forceinline__ DoubleGroupSums fx64_group(const uint4& e0, const uint4& e1, const int4& qi,
                                                      const int4* __restrict__ frames, const int2* s_xy, const int* s_z,
                                                      const double4* __restrict__ pos, int i, const Box& box,
                                                      const Fx64LJ& lj, unsigned& c, bool* shell) {
    const uint32_t ent[8] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
    DoubleGroupSums g;
    bool sh = false;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const uint32_t e = ent[u];
        const uint32_t code = e >> kCodeShift;
        const bool pad = code == kSentinelCode;
        const int j = pad ? 0 : static_cast<int>(e & kIndexMask);
        double dx, dy, dz;
        const int2 oxy = s_xy[code];
        const double r2 = fixed_separation(qi, frames[j], make_int4(oxy.x, oxy.y, s_z[code], 0), dx, dy, dz);
        bool in = !pad && r2 < lj.lj.rc2;
        const bool near = !pad && fabs(dsub(r2, lj.lj.rc2)) < lj.band;
        if (kExact) {
            if (near) in = exact_inside(pos[i], pos[j], box, lj.lj.rc2);
        } else {
            sh |= near;
        }
        fx64_pair<kEnergy>(dx, dy, dz, in, pad ? 1.0 : r2, lj, g.x, g.y, g.z, g.e, g.w, c);
    }
    if (!kExact) *shell = sh;
    return g;
}

template <bool kEnergy>
__device__ __noinline__ DoubleGroupSums fx64_group_exact(const uint4 e0, const uint4 e1, const int4 qi,
                                                         const int4* __restrict__ frames, const int2* s_xy, const int* s_z,
                                                         const double4* __restrict__ pos, int i, const Box box,
                                                         const Fx64LJ lj, unsigned* c) {
    unsigned k = 0;
    const DoubleGroupSums g = fx64_group<kEnergy, true>(e0, e1, qi, frames, s_xy, s_z, pos, i, box, lj, k, nullptr);
    *c = k;
    return g;
}

// Thread per particle over its row (the layout of k_force_fp32_rows) with the next group's row quads prefetched
// (streaming loads), frames gathered from global memory; groups run branch-free, a group with a pair in the
// cutoff shell runs again out of line with the exact test.
template <bool kEnergy>
__global__ void __launch_bounds__(128) k_force_fx64_rows(const int4* __restrict__ frames, const double4* __restrict__ pos,
                                                         int n, Box box, Fx64LJ lj, FixedOffsets offs,
                                                         const uint32_t* __restrict__ rows, int cap,
                                                         const int2* __restrict__ counts, double* __restrict__ force,
                                                         unsigned long long* __restrict__ acc, KickArgs kick) {
    // the 32 codes' fixed-point image offsets as a table of (x, y) pairs (s_o[0..1]) and one of z (s_o[2]): an
    // 8- and a 4-byte shared load per entry instead of one of 16 (fewer shared-memory wavefronts in the L1 data
    // pipe, which the gathers keep busy)
    __shared__ __align__(16) int s_o[4][32];
    if (threadIdx.x < 32) {
        const int4 o = offs.off[threadIdx.x];
        reinterpret_cast<int2*>(s_o[0])[threadIdx.x] = make_int2(o.x, o.y);
        s_o[2][threadIdx.x] = o.z;
    }
    __syncthreads();
    const int2* s_xy = reinterpret_cast<const int2*>(s_o[0]);
    const int* s_z = s_o[2];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    long long e_fx = 0, w_fx = 0, k_fx = 0;
    unsigned ins = 0;
    if (i < n) {
        const int4 qi = frames[i];
        const int2 c = counts[i];
        const int groups = (c.x + c.y + 7) >> 3;
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
            DoubleGroupSums gs = fx64_group<kEnergy, false>(e0, e1, qi, frames, s_xy, s_z, pos, i, box, lj, gin, &shell);
            if (shell) gs = fx64_group_exact<kEnergy>(e0, e1, qi, frames, s_xy, s_z, pos, i, box, lj, &gin);
            ins += gin;
            a.add_group(gs.x, gs.y, gs.z, gs.e, gs.w, e_fx, w_fx);
        }
        k_fx = a.finish(i, n, force, kick);
    }
    if (kEnergy || kick.vel) flush_sums(e_fx, w_fx, ins, k_fx, acc);
}

// Boxes under 3 cells per side: separations from the double positions with the reference's minimum image
// (as k_force_fp32_small), the same double pair terms and fixed-point sums
template <bool kEnergy>
__global__ void k_force_fx64_small(const double4* __restrict__ pos, int n, Box box, Fx64LJ lj,
                                   const uint32_t* __restrict__ rows, int cap, const int2* __restrict__ counts,
                                   double* __restrict__ force, unsigned long long* __restrict__ acc, KickArgs kick) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    long long e_fx = 0, w_fx = 0, k_fx = 0;
    unsigned ins = 0;
    if (i < n) {
        const double4 pi = pos[i];
        const int2 c = counts[i];
        const int m = c.x + c.y;
        FloatAcc<true, kEnergy> a;
        for (int g0 = 0; g0 < m; g0 += 8) {
            double gx = 0.0, gy = 0.0, gz = 0.0, ge = 0.0, gw = 0.0;
            for (int s = g0; s < g0 + 8 && s < m; ++s) {
                const double4 pj = pos[rows[row_index(i, s, cap)] & kIndexMask];
                const double dx = min_image(dsub(pi.x, pj.x), box);
                const double dy = min_image(dsub(pi.y, pj.y), box);
                const double dz = min_image(dsub(pi.z, pj.z), box);
                const double r2 = norm2(dx, dy, dz);
                fx64_pair<kEnergy>(dx, dy, dz, r2 < lj.lj.rc2, r2, lj, gx, gy, gz, ge, gw, ins);
            }
            a.add_group(gx, gy, gz, ge, gw, e_fx, w_fx);
        }
        k_fx = a.finish(i, n, force, kick);
    }
    if (kEnergy || kick.vel) flush_sums(e_fx, w_fx, ins, k_fx, acc);
}

}  // namespace md
