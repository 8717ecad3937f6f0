// Float pair arithmetic for the list forces (precision modes MD_PREC_FP32FX and MD_PREC_FP32).
//
// Positions enter the pair loop as float offsets from the centre of each particle's cell at the last list
// build (a "frame"), refreshed from the double positions every step. A pair's separation is
// q_i - q_j - d * cell, d being the neighbour cell offset coded in the list entry, so the float
// subtraction never sees coordinates of the box's size and min-image needs no rounding step. With cells of at
// least r_c + skin and every particle within skin/2 of its build position, the coded image is the minimum
// image of every pair that can be inside the cutoff.
//
// FP32FX accumulates each particle's force in 64-bit fixed point: the float partial sum over every group of 8
// row entries is rounded to a multiple of 2^-32 and added as an integer. The groups are fixed by the row
// layout, integers add associatively, so the result does not depend on the launch shape. FP32 keeps one float
// sum per component over the whole row (the reference's mixed path accumulates per particle in float too,
// src/Forcefield.cpp:388-412).
#pragma once

#include "md_common.cuh"

namespace md {

constexpr float kForceScale = 4294967296.0f;        // 2^32: fixed-point units per unit force
constexpr double kForceUnit = 1.0 / 4294967296.0;
constexpr float kEnergyScale = 16777216.0f;         // 2^24 for energy and virial sums
constexpr double kEnergyUnit = 1.0 / 16777216.0;
constexpr float kSentinelCoord = 1.0e15f;           // frame of the sentinel particle: never inside the cutoff

struct FloatLJ {
    float sig2;    // sigma^2
    float eps24;   // 24 eps
    float eps48;   // 48 eps
    float eps4;    // 4 eps
    float shift;   // energy shift
    float rc2;     // cut_off^2
};

struct CellOffsets {
    float4 off[27];  // -d * cell for the 27 codes (d in {-1, 0, 1}^3)
};

// Frames: q = minimum-image (r - centre of the particle's build cell), in float. frames[n] is the sentinel.
__global__ void k_frames(const double4* __restrict__ pos, int n, const int* __restrict__ cell_sorted, int ncps,
                         double cell, Box box, float4* __restrict__ frames) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) frames[n] = make_float4(kSentinelCoord, kSentinelCoord, kSentinelCoord, 0.0f);
    if (i >= n) return;
    const int c = cell_sorted[i];
    const int cx = c / (ncps * ncps), cy = (c / ncps) % ncps, cz = c % ncps;
    const double4 p = pos[i];
    double dx = p.x - (cx + 0.5) * cell, dy = p.y - (cy + 0.5) * cell, dz = p.z - (cz + 0.5) * cell;
    dx -= box.L * rint(dx * box.invL);
    dy -= box.L * rint(dy * box.invL);
    dz -= box.L * rint(dz * box.invL);
    frames[i] = make_float4(static_cast<float>(dx), static_cast<float>(dy), static_cast<float>(dz), 0.0f);
}

// One thread per particle over its full row (own and reverse partners, padded with sentinels to a multiple
// of 8). kFixed selects FP32FX; kEnergy adds the energy, virial and inside-pair sums (every pair is seen
// twice, from both ends, so the host halves them).
template <bool kFixed, bool kEnergy>
__global__ void __launch_bounds__(128) k_force_fp32(const float4* __restrict__ frames, int n, FloatLJ lj,
                                                     CellOffsets offs, const uint32_t* __restrict__ rows, int cap,
                                                     const int2* __restrict__ counts, double* __restrict__ force,
                                                     unsigned long long* __restrict__ acc) {
    __shared__ float4 s_off[27];
    if (threadIdx.x < 27) s_off[threadIdx.x] = offs.off[threadIdx.x];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    long long e_fx = 0, w_fx = 0;
    unsigned long long ins = 0;
    if (i < n) {
        const float4 qi = frames[i];
        const uint4* row = reinterpret_cast<const uint4*>(rows + static_cast<size_t>(i) * cap);
        const int2 c = counts[i];
        const int groups = (c.x + c.y + 7) >> 3;
        long long ax = 0, ay = 0, az = 0;
        float fx = 0.f, fy = 0.f, fz = 0.f;
        for (int g = 0; g < groups; ++g) {
            const uint4 e0 = row[2 * g], e1 = row[2 * g + 1];
            const uint32_t ent[8] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
            float gx = 0.f, gy = 0.f, gz = 0.f, ge = 0.f, gw = 0.f;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const uint32_t e = ent[t];
                const float4 qj = frames[e & kIndexMask];
                const float4 o = s_off[e >> kCodeShift];
                const float dx = (qi.x - qj.x) + o.x;
                const float dy = (qi.y - qj.y) + o.y;
                const float dz = (qi.z - qj.z) + o.z;
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const bool in = r2 < lj.rc2;
                const float inv = __frcp_rn(r2);
                const float sr2 = lj.sig2 * inv;
                const float sr6 = sr2 * sr2 * sr2;
                float fr = (lj.eps48 * sr6 - lj.eps24) * sr6 * inv;
                fr = in ? fr : 0.0f;
                gx = fmaf(fr, dx, gx);
                gy = fmaf(fr, dy, gy);
                gz = fmaf(fr, dz, gz);
                if (kEnergy) {
                    const float en = fmaf(lj.eps4 * sr6, sr6 - 1.0f, -lj.shift);
                    ge += in ? en : 0.0f;
                    gw = fmaf(fr, r2, gw);
                    ins += in ? 1u : 0u;
                }
            }
            if (kFixed) {
                ax += __float2ll_rn(gx * kForceScale);
                ay += __float2ll_rn(gy * kForceScale);
                az += __float2ll_rn(gz * kForceScale);
            } else {
                fx += gx;
                fy += gy;
                fz += gz;
            }
            if (kEnergy) {
                e_fx += __float2ll_rn(ge * kEnergyScale);
                w_fx += __float2ll_rn(gw * kEnergyScale);
            }
        }
        double Fx, Fy, Fz;
        if (kFixed) {
            Fx = static_cast<double>(ax) * kForceUnit;
            Fy = static_cast<double>(ay) * kForceUnit;
            Fz = static_cast<double>(az) * kForceUnit;
        } else {
            Fx = fx;
            Fy = fy;
            Fz = fz;
        }
        force[i] = Fx;
        force[static_cast<size_t>(n) + i] = Fy;
        force[2 * static_cast<size_t>(n) + i] = Fz;
    }
    if (kEnergy) {
        e_fx = warp_sum_i64(e_fx);
        w_fx = warp_sum_i64(w_fx);
        ins = warp_sum_u64(ins);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&acc[0], static_cast<unsigned long long>(e_fx));
            atomicAdd(&acc[1], static_cast<unsigned long long>(w_fx));
            atomicAdd(&acc[2], ins);
        }
    }
}

// Boxes under 3 cells per side (all-pairs candidates): separations come from the double positions with the
// reference's minimum image, then narrow to float (the reference's mixed path does the same,
// src/Forcefield.cpp:373-386).
template <bool kFixed, bool kEnergy>
__global__ void k_force_fp32_small(const double4* __restrict__ pos, int n, Box box, FloatLJ lj,
                                   const uint32_t* __restrict__ rows, int cap, const int2* __restrict__ counts,
                                   double* __restrict__ force, unsigned long long* __restrict__ acc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    long long e_fx = 0, w_fx = 0;
    unsigned long long ins = 0;
    if (i < n) {
        const double4 pi = pos[i];
        const uint32_t* row = rows + static_cast<size_t>(i) * cap;
        const int2 c = counts[i];
        const int m = c.x + c.y;
        long long ax = 0, ay = 0, az = 0;
        float fx = 0.f, fy = 0.f, fz = 0.f;
        for (int g0 = 0; g0 < m; g0 += 8) {
            float gx = 0.f, gy = 0.f, gz = 0.f, ge = 0.f, gw = 0.f;
            for (int s = g0; s < g0 + 8 && s < m; ++s) {
                const double4 pj = pos[row[s] & kIndexMask];
                double ddx = pi.x - pj.x, ddy = pi.y - pj.y, ddz = pi.z - pj.z;
                ddx -= box.L * round(ddx * box.invL);
                ddy -= box.L * round(ddy * box.invL);
                ddz -= box.L * round(ddz * box.invL);
                const float dx = static_cast<float>(ddx), dy = static_cast<float>(ddy), dz = static_cast<float>(ddz);
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const bool in = r2 < lj.rc2;
                const float inv = __frcp_rn(r2);
                const float sr2 = lj.sig2 * inv;
                const float sr6 = sr2 * sr2 * sr2;
                float fr = (lj.eps48 * sr6 - lj.eps24) * sr6 * inv;
                fr = in ? fr : 0.0f;
                gx = fmaf(fr, dx, gx);
                gy = fmaf(fr, dy, gy);
                gz = fmaf(fr, dz, gz);
                if (kEnergy) {
                    const float en = fmaf(lj.eps4 * sr6, sr6 - 1.0f, -lj.shift);
                    ge += in ? en : 0.0f;
                    gw = fmaf(fr, r2, gw);
                    ins += in ? 1u : 0u;
                }
            }
            if (kFixed) {
                ax += __float2ll_rn(gx * kForceScale);
                ay += __float2ll_rn(gy * kForceScale);
                az += __float2ll_rn(gz * kForceScale);
            } else {
                fx += gx;
                fy += gy;
                fz += gz;
            }
            if (kEnergy) {
                e_fx += __float2ll_rn(ge * kEnergyScale);
                w_fx += __float2ll_rn(gw * kEnergyScale);
            }
        }
        force[i] = kFixed ? static_cast<double>(ax) * kForceUnit : static_cast<double>(fx);
        force[static_cast<size_t>(n) + i] = kFixed ? static_cast<double>(ay) * kForceUnit : static_cast<double>(fy);
        force[2 * static_cast<size_t>(n) + i] = kFixed ? static_cast<double>(az) * kForceUnit : static_cast<double>(fz);
    }
    if (kEnergy) {
        e_fx = warp_sum_i64(e_fx);
        w_fx = warp_sum_i64(w_fx);
        ins = warp_sum_u64(ins);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&acc[0], static_cast<unsigned long long>(e_fx));
            atomicAdd(&acc[1], static_cast<unsigned long long>(w_fx));
            atomicAdd(&acc[2], ins);
        }
    }
}

// Converts the fixed-point energy sums to (pe, virial) doubles, halving the double-counted pairs; the
// inside count goes to *inside as an integer.
__global__ void k_finish_float_energy(const unsigned long long* __restrict__ acc, double* __restrict__ out,
                                      unsigned long long* __restrict__ inside) {
    out[0] = 0.5 * static_cast<double>(static_cast<long long>(acc[0])) * kEnergyUnit;
    out[1] = 0.5 * static_cast<double>(static_cast<long long>(acc[1])) * kEnergyUnit;
    *inside = acc[2] / 2;
}

}  // namespace md
