// Float pair arithmetic for the list forces (precision modes MD_PREC_FP32FX and MD_PREC_FP32): frames, the
// shared pair/epilogue helpers, the global-gather kernel and the small-box kernel. The shared-memory tile
// kernel is in md_tiles.cuh; both evaluate every pair with the same pinned float operation sequence
// (float_pair), so either one gives the same bits.
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
constexpr float kEnergyScale = 16777216.0f;         // 2^24 for energy and virial sums of float groups
constexpr double kEnergyUnit = 1.0 / 16777216.0;
constexpr double kEnergyScale64 = 1073741824.0;     // 2^30 for energy and virial sums of double groups (FX64)
constexpr double kEnergyUnit64 = 1.0 / 1073741824.0;
constexpr double kKineticScale = 4294967296.0;      // 2^32: fixed-point units of the fused kinetic energy
constexpr float kSentinelCoord = 1.0e15f;           // frame of the sentinel particle: never inside the cutoff

struct FloatLJ {
    float sig2;    // sigma^2
    float eps24;   // 24 eps
    float eps48;   // 48 eps
    float eps4;    // 4 eps
    float shift;   // energy shift
    float rc2;     // cut_off^2
    float band;    // |float r^2 - r_c^2| below this: decide inside/outside with the exact double test
    double rc2d;   // cut_off^2 in double
};

// The frame of a position: minimum-image (r - centre of cell c), narrowed to float. Every kernel that writes
// frames calls this, with explicit roundings, so all of them produce the same bits.
__device__ __forceinline__ float4 frame_of(const double4& p, int c, int ncps, double cell, const Box& box) {
    const int cx = c / (ncps * ncps), cy = (c / ncps) % ncps, cz = c % ncps;
    double d[3] = {dsub(p.x, dmul(cx + 0.5, cell)), dsub(p.y, dmul(cy + 0.5, cell)), dsub(p.z, dmul(cz + 0.5, cell))};
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = dsub(d[k], dmul(box.L, rint(dmul(d[k], box.invL))));
    return make_float4(static_cast<float>(d[0]), static_cast<float>(d[1]), static_cast<float>(d[2]), 0.0f);
}

constexpr double kFrameScale = 268435456.0;  // 2^28 fixed-point frame units per unit length
constexpr double kFrameUnit = 1.0 / 268435456.0;

// frame_of in fixed point: round(q * 2^28) per component (|q| stays below a cell plus half the skin, far
// inside the int32 range)
__device__ __forceinline__ int4 fixed_frame_of(const double4& p, int c, int ncps, double cell, const Box& box) {
    const int cx = c / (ncps * ncps), cy = (c / ncps) % ncps, cz = c % ncps;
    double d[3] = {dsub(p.x, dmul(cx + 0.5, cell)), dsub(p.y, dmul(cy + 0.5, cell)), dsub(p.z, dmul(cz + 0.5, cell))};
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = dsub(d[k], dmul(box.L, rint(dmul(d[k], box.invL))));
    return make_int4(__double2int_rn(dmul(d[0], kFrameScale)), __double2int_rn(dmul(d[1], kFrameScale)),
                     __double2int_rn(dmul(d[2], kFrameScale)), 0);
}

struct CellOffsets {
    float4 off[32];  // -d * cell for the 27 codes (d in {-1, 0, 1}^3); zero for the sentinel code
};

// The closing half kick fused into a force kernel (vel == nullptr: forces only). With pos_out set, the next
// step's opening kick and drift are fused too (a step whose velocities nothing else touches in between): the
// kernel writes v + (half_dt F) / m once more, the new positions into pos_out and their float frames into
// frames_out (the force loop still reads the old ones), and runs the half-skin test against ref_pos into
// *stale, with k_kick_drift_frames' operation sequence.
struct KickArgs {
    double* vel;
    const double* mass;
    double half_dt;
    const double4* pos_in = nullptr;
    double4* pos_out = nullptr;
    float4* frames_out = nullptr;  // float frames of the new positions (float modes)
    int4* iframes_out = nullptr;   // fixed-point frames of the new positions (MD_PREC_FX64)
    const double4* ref_pos = nullptr;
    double max_disp2 = 0.0;
    int* stale = nullptr;
    const int* cell_sorted = nullptr;
    int ncps = 0;
    double cell = 0.0;
    double dt = 0.0;
    Box box{};
    int* overflow = nullptr;  // set to 1 by a tile kernel whose staged tile outgrew its shared memory
};

// The truncated potential's force jumps by |F(r_c)| at the cutoff, so a pair whose float r^2 sits within
// rounding of r_c^2 must be classified as the reference classifies it: min-image r^2 < r_c^2 in double
// (src/Forcefield.cpp:366). Only pairs in a thin shell take this branch.
__device__ __forceinline__ bool exact_inside(const double4& a, const double4& b, const Box& box, double rc2) {
    const double dx = min_image(dsub(a.x, b.x), box);
    const double dy = min_image(dsub(a.y, b.y), box);
    const double dz = min_image(dsub(a.z, b.z), box);
    return norm2(dx, dy, dz) < rc2;
}

// The hardware's approximate reciprocal (PTX rcp.approx.ftz.f32: one instruction, within 1 ulp); deterministic,
// so every kernel that calls it gets the same bits
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// One pair in float with a pinned operation sequence (explicit roundings and FMAs), shared by every float
// kernel. Adds its force to (gx, gy, gz) and, with kEnergy, its energy, virial and inside count (a per-thread
// 32-bit count: a thread visits far fewer than 2^32 row entries).
template <bool kEnergy>
__device__ __forceinline__ void float_pair(float dx, float dy, float dz, bool in, float r2, const FloatLJ& lj,
                                           float& gx, float& gy, float& gz, float& ge, float& gw, unsigned& ins) {
    const float inv = rcp_approx(r2);
    const float sr2 = __fmul_rn(lj.sig2, inv);
    const float sr6 = __fmul_rn(__fmul_rn(sr2, sr2), sr2);
    float fr = __fmul_rn(__fmul_rn(fmaf(lj.eps48, sr6, -lj.eps24), sr6), inv);
    fr = in ? fr : 0.0f;
    gx = fmaf(fr, dx, gx);
    gy = fmaf(fr, dy, gy);
    gz = fmaf(fr, dz, gz);
    if (kEnergy) {
        const float en = fmaf(__fmul_rn(lj.eps4, sr6), __fadd_rn(sr6, -1.0f), -lj.shift);
        ge = __fadd_rn(ge, in ? en : 0.0f);
        gw = fmaf(fr, r2, gw);
        ins += in ? 1u : 0u;
    }
}

// Separation of a row entry's pair from the frames: (q_i - q_j) + image offset, and its float r^2. x and y go
// through one packed add of -q_j and one packed add of the offset (__fadd2_rn: the same two round-to-nearest
// operations per component as the scalar sequence, so the same bits, in half the instructions).
__device__ __forceinline__ float float_separation(const float4& qi, const float4& qj, const float4& o, float& dx,
                                                  float& dy, float& dz) {
    const float2 d = __fadd2_rn(__fadd2_rn(make_float2(qi.x, qi.y), make_float2(-qj.x, -qj.y)), make_float2(o.x, o.y));
    dx = d.x;
    dy = d.y;
    dz = __fadd_rn(__fsub_rn(qi.z, qj.z), o.z);
    return fmaf(dx, dx, fmaf(dy, dy, __fmul_rn(dz, dz)));
}

// Sums of one 8-entry group: force, energy, virial
struct GroupSums {
    float x = 0.f, y = 0.f, z = 0.f, e = 0.f, w = 0.f;
};

// One 8-entry group of a row (entries e0, e1 in order) through float_pair. sep(e, dx, dy, dz) returns the float
// r^2 of entry e and its separation. The group runs branch-free with the float cutoff test; a pair in the
// thin shell around r_c (about one group in a thousand has one) sends the whole group through
// float_group_exact, the same sequence with the reference's exact test (exact(e)) deciding the shell pairs, so
// the sums see the same operations in the same order either way. Adds the group's inside count to *ins.
template <bool kEnergy, typename Sep, typename Exact>
__device__ __noinline__ GroupSums float_group_exact(const uint4 e0, const uint4 e1, const FloatLJ lj, Sep sep,
                                                    Exact exact, unsigned* gin) {
    const uint32_t ent[8] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
    GroupSums g;
    unsigned c = 0;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        float dx, dy, dz;
        const float r2 = sep(ent[u], dx, dy, dz);
        bool in = r2 < lj.rc2;
        if (fabsf(r2 - lj.rc2) < lj.band) in = exact(ent[u]);
        float_pair<kEnergy>(dx, dy, dz, in, r2, lj, g.x, g.y, g.z, g.e, g.w, c);
    }
    *gin = c;
    return g;
}

template <bool kEnergy, typename Sep, typename Exact>
__device__ __forceinline__ GroupSums float_group(const uint4& e0, const uint4& e1, const FloatLJ& lj, Sep sep,
                                                 Exact exact, unsigned& ins) {
    const uint32_t ent[8] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
    GroupSums g;
    unsigned c = 0;
    bool shell = false;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        float dx, dy, dz;
        const float r2 = sep(ent[u], dx, dy, dz);
        shell |= fabsf(r2 - lj.rc2) < lj.band;
        float_pair<kEnergy>(dx, dy, dz, r2 < lj.rc2, r2, lj, g.x, g.y, g.z, g.e, g.w, c);
    }
    if (shell) g = float_group_exact<kEnergy>(e0, e1, lj, sep, exact, &c);
    ins += c;
    return g;
}

// Per-particle accumulators of the float kernels: a group of 8 row entries goes into fixed point (FP32FX) or
// into the running float sum (FP32)
template <bool kFixed, bool kEnergy>
struct FloatAcc {
    long long ax = 0, ay = 0, az = 0;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    __device__ __forceinline__ void add_group(float gx, float gy, float gz, float ge, float gw, long long& e_fx,
                                              long long& w_fx) {
        if (kFixed) {
            ax += __float2ll_rn(gx * kForceScale);
            ay += __float2ll_rn(gy * kForceScale);
            az += __float2ll_rn(gz * kForceScale);
        } else {
            fx = __fadd_rn(fx, gx);
            fy = __fadd_rn(fy, gy);
            fz = __fadd_rn(fz, gz);
        }
        if (kEnergy) {
            e_fx += __float2ll_rn(ge * kEnergyScale);
            w_fx += __float2ll_rn(gw * kEnergyScale);
        }
    }
    // A float group whose energy and virial go into the finer 2^-30 units of the double groups (MD_PREC_FX32,
    // whose rows hold both kinds); forces in the same 2^-32 units (the products with 2^32 and 2^30 are exact)
    __device__ __forceinline__ void add_group_fine(float gx, float gy, float gz, float ge, float gw, long long& e_fx,
                                                   long long& w_fx) {
        static_assert(kFixed, "fine groups accumulate in fixed point");
        ax += __float2ll_rn(gx * kForceScale);
        ay += __float2ll_rn(gy * kForceScale);
        az += __float2ll_rn(gz * kForceScale);
        if (kEnergy) {
            e_fx += __float2ll_rn(ge * static_cast<float>(kEnergyScale64));
            w_fx += __float2ll_rn(gw * static_cast<float>(kEnergyScale64));
        }
    }
    // A group summed in double (MD_PREC_FX64): the same fixed-point units, rounded from double
    __device__ __forceinline__ void add_group(double gx, double gy, double gz, double ge, double gw, long long& e_fx,
                                              long long& w_fx) {
        static_assert(kFixed, "double groups accumulate in fixed point");
        ax += __double2ll_rn(dmul(gx, static_cast<double>(kForceScale)));
        ay += __double2ll_rn(dmul(gy, static_cast<double>(kForceScale)));
        az += __double2ll_rn(dmul(gz, static_cast<double>(kForceScale)));
        if (kEnergy) {
            e_fx += __double2ll_rn(dmul(ge, kEnergyScale64));
            w_fx += __double2ll_rn(dmul(gw, kEnergyScale64));
        }
    }
    // Write the force (double, component-major) and apply the fused closing kick; returns the particle's
    // fixed-point kinetic energy after the kick (0 without a kick)
    __device__ __forceinline__ long long finish(int i, int n, double* __restrict__ force, const KickArgs& kick) const {
        const double F[3] = {kFixed ? static_cast<double>(ax) * kForceUnit : static_cast<double>(fx),
                             kFixed ? static_cast<double>(ay) * kForceUnit : static_cast<double>(fy),
                             kFixed ? static_cast<double>(az) * kForceUnit : static_cast<double>(fz)};
        double ke = 0.0;
        double vn[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const size_t o = static_cast<size_t>(k) * n + i;
            force[o] = F[k];
            if (kick.vel) {  // VelocityVerletIntegrator::kick (src/Integrator.cpp:55-71)
                const double v = dadd(kick.vel[o], ddiv(dmul(kick.half_dt, F[k]), kick.mass[i]));
                ke = dadd(ke, dmul(v, v));
                if (kick.pos_out) {  // the next step's kickAndDrift (src/Integrator.cpp:32-53)
                    vn[k] = dadd(v, ddiv(dmul(kick.half_dt, F[k]), kick.mass[i]));
                    kick.vel[o] = vn[k];
                } else {
                    kick.vel[o] = v;
                }
            }
        }
        if (kick.vel && kick.pos_out) {
            double4 p = kick.pos_in[i];
            p.x = wrap(dadd(p.x, dmul(kick.dt, vn[0])), kick.box);
            p.y = wrap(dadd(p.y, dmul(kick.dt, vn[1])), kick.box);
            p.z = wrap(dadd(p.z, dmul(kick.dt, vn[2])), kick.box);
            kick.pos_out[i] = p;
            const double4 r = kick.ref_pos[i];  // NeighbourList::update (src/NeighbourList.cpp:24-30)
            const double dx = min_image(dsub(p.x, r.x), kick.box);
            const double dy = min_image(dsub(p.y, r.y), kick.box);
            const double dz = min_image(dsub(p.z, r.z), kick.box);
            if (norm2(dx, dy, dz) > kick.max_disp2) *kick.stale = 1;
            if (kick.frames_out) kick.frames_out[i] = frame_of(p, kick.cell_sorted[i], kick.ncps, kick.cell, kick.box);
            if (kick.iframes_out)
                kick.iframes_out[i] = fixed_frame_of(p, kick.cell_sorted[i], kick.ncps, kick.cell, kick.box);
        }
        return kick.vel ? __double2ll_rn(dmul(dmul(dmul(0.5, kick.mass[i]), ke), kKineticScale)) : 0;
    }
};

// Block-level sums of the fixed-point energy, virial, inside count and kinetic energy into acc[0..3]
__device__ __forceinline__ void flush_sums(long long e_fx, long long w_fx, unsigned long long ins, long long k_fx,
                                           unsigned long long* __restrict__ acc) {
    e_fx = warp_sum_i64(e_fx);
    w_fx = warp_sum_i64(w_fx);
    k_fx = warp_sum_i64(k_fx);
    ins = warp_sum_u64(ins);
    if ((threadIdx.x & 31) == 0) {
        if (e_fx) atomicAdd(&acc[0], static_cast<unsigned long long>(e_fx));
        if (w_fx) atomicAdd(&acc[1], static_cast<unsigned long long>(w_fx));
        if (ins) atomicAdd(&acc[2], ins);
        if (k_fx) atomicAdd(&acc[3], static_cast<unsigned long long>(k_fx));
    }
}

// The image offset -d * cell of a neighbour-cell code (d in {-1, 0, 1}^3), zero for codes above 26: the same
// floats the host writes into CellOffsets (-d * cell in double is exact, so only the narrowing rounds)
__device__ __forceinline__ float4 code_offset(int code, float cell) {
    if (code > 26) return make_float4(0.f, 0.f, 0.f, 0.f);
    const int d[3] = {code / 9 - 1, (code / 3) % 3 - 1, code % 3 - 1};
    float o[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) o[k] = d[k] == 0 ? 0.0f : (d[k] > 0 ? -cell : cell);
    return make_float4(o[0], o[1], o[2], 0.0f);
}

// Frames: q = minimum-image (r - centre of the particle's build cell), in float. frames[n] is the sentinel.
__global__ void k_frames(const double4* __restrict__ pos, int n, const int* __restrict__ cell_sorted, int ncps,
                         double cell, Box box, float4* __restrict__ frames) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) frames[n] = make_float4(kSentinelCoord, kSentinelCoord, kSentinelCoord, 0.0f);
    if (i >= n) return;
    frames[i] = frame_of(pos[i], cell_sorted[i], ncps, cell, box);
}

// Thread per particle over its row with neighbour frames gathered from global memory (L1/L2); rows are read
// as interleaved uint4, coalesced across the warp.
// kPrefetch (variants 2, 3 and 4): row quads are loaded one group ahead with the streaming cache hint, so the next
// group's entries are in flight while the current group's frames are gathered, and the streamed rows do not
// displace the frames from L1/L2. kMinBlocks > 1 (variant 3) caps the registers so that many blocks stay resident
// on an SM. Same arithmetic, same bits.
// The row loop of one particle: adds its energy, virial and inside count to the thread's sums and returns its
// fixed-point kinetic energy after the fused kick.
template <bool kFixed, bool kEnergy, bool kPrefetch>
__device__ __forceinline__ long long fp32_row(int i, const float4* __restrict__ frames, const double4* __restrict__ pos,
                                              int n, const Box& box, const FloatLJ& lj, const float4* s_off,
                                              const uint32_t* __restrict__ rows, int cap,
                                              const int2* __restrict__ counts, double* __restrict__ force,
                                              const KickArgs& kick, long long& e_fx, long long& w_fx, unsigned& ins) {
    const float4 qi = frames[i];
    const int2 c = counts[i];
    const int groups = (c.x + c.y + 7) >> 3;  // rows are padded with sentinels to a multiple of 8
    FloatAcc<kFixed, kEnergy> a;
    // quad q of this particle's interleaved row is rq[32 q]; a group is two quads
    const uint4* rq = reinterpret_cast<const uint4*>(rows) + static_cast<size_t>(i >> 5) * (cap >> 2) * 32 + (i & 31);
    uint4 n0 = make_uint4(0, 0, 0, 0), n1 = n0;
    if (kPrefetch && groups > 0) {
        n0 = __ldcs(rq);
        n1 = __ldcs(rq + 32);
    }
    for (int g = 0; g < groups; ++g) {
        uint4 e0, e1;
        if (kPrefetch) {
            e0 = n0;
            e1 = n1;
            rq += 64;
            if (g + 1 < groups) {
                n0 = __ldcs(rq);
                n1 = __ldcs(rq + 32);
            }
        } else {
            e0 = rq[64 * g];
            e1 = rq[64 * g + 32];
        }
        const GroupSums gs = float_group<kEnergy>(
            e0, e1, lj,
            [=](uint32_t e, float& dx, float& dy, float& dz) {
                return float_separation(qi, frames[e & kIndexMask], s_off[e >> kCodeShift], dx, dy, dz);
            },
            [=](uint32_t e) { return exact_inside(pos[i], pos[e & kIndexMask], box, lj.rc2d); }, ins);
        a.add_group(gs.x, gs.y, gs.z, gs.e, gs.w, e_fx, w_fx);
    }
    return a.finish(i, n, force, kick);
}

// The row loop of fp32_row with the prefetch, the image offsets read from a table of (x, y) pairs and a table of
// z (an 8- and a 4-byte shared load per entry instead of one of 16 bytes: fewer shared-memory wavefronts in the
// L1 data pipe, which the gathers keep busy). Same operations, same bits.
template <bool kFixed, bool kEnergy>
__device__ __forceinline__ long long fp32_row_split(int i, const float4* __restrict__ frames,
                                                    const double4* __restrict__ pos, int n, const Box& box,
                                                    const FloatLJ& lj, const float2* s_xy, const float* s_z,
                                                    const uint32_t* __restrict__ rows, int cap,
                                                    const int2* __restrict__ counts, double* __restrict__ force,
                                                    const KickArgs& kick, long long& e_fx, long long& w_fx,
                                                    unsigned& ins) {
    const float4 qi = frames[i];
    const int2 c = counts[i];
    const int groups = (c.x + c.y + 7) >> 3;
    FloatAcc<kFixed, kEnergy> a;
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
        const GroupSums gs = float_group<kEnergy>(
            e0, e1, lj,
            [=](uint32_t e, float& dx, float& dy, float& dz) {
                const uint32_t k = e >> kCodeShift;
                const float2 oxy = s_xy[k];
                return float_separation(qi, frames[e & kIndexMask], make_float4(oxy.x, oxy.y, s_z[k], 0.0f), dx,
                                        dy, dz);
            },
            [=](uint32_t e) { return exact_inside(pos[i], pos[e & kIndexMask], box, lj.rc2d); }, ins);
        a.add_group(gs.x, gs.y, gs.z, gs.e, gs.w, e_fx, w_fx);
    }
    return a.finish(i, n, force, kick);
}

// Variant 4: fp32_row_split on a resident grid (as many blocks as fit on the SMs at once, each thread taking
// particles i, i + grid, ...: no block turnover, no partial last wave, one flush of the sums per thread).
template <bool kFixed, bool kEnergy>
__global__ void __launch_bounds__(128) k_force_fp32_resident(const float4* __restrict__ frames,
                                                             const double4* __restrict__ pos, int n, Box box,
                                                             FloatLJ lj, CellOffsets offs,
                                                             const uint32_t* __restrict__ rows, int cap,
                                                             const int2* __restrict__ counts, double* __restrict__ force,
                                                             unsigned long long* __restrict__ acc, KickArgs kick) {
    __shared__ __align__(16) float s_o[4][32];  // s_o[0..1]: the 32 (x, y) pairs; s_o[2]: z
    if (threadIdx.x < 32) {
        const float4 o = offs.off[threadIdx.x];
        reinterpret_cast<float2*>(s_o[0])[threadIdx.x] = make_float2(o.x, o.y);
        s_o[2][threadIdx.x] = o.z;
    }
    __syncthreads();
    if (kick.frames_out && blockIdx.x == 0 && threadIdx.x == 0)
        kick.frames_out[n] = make_float4(kSentinelCoord, kSentinelCoord, kSentinelCoord, 0.0f);
    long long e_fx = 0, w_fx = 0, k_fx = 0;
    unsigned ins = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        k_fx += fp32_row_split<kFixed, kEnergy>(i, frames, pos, n, box, lj, reinterpret_cast<const float2*>(s_o[0]),
                                                s_o[2], rows, cap, counts, force, kick, e_fx, w_fx, ins);
    if (kEnergy || kick.vel) flush_sums(e_fx, w_fx, ins, k_fx, acc);
}

template <bool kFixed, bool kEnergy, bool kPrefetch = false, int kMinBlocks = 1>
__global__ void __launch_bounds__(128, kMinBlocks) k_force_fp32_rows(const float4* __restrict__ frames,
                                                         const double4* __restrict__ pos, int n, Box box,
                                                         FloatLJ lj, CellOffsets offs,
                                                         const uint32_t* __restrict__ rows, int cap,
                                                         const int2* __restrict__ counts, double* __restrict__ force,
                                                         unsigned long long* __restrict__ acc, KickArgs kick) {
    __shared__ float4 s_off[32];
    if (threadIdx.x < 32) s_off[threadIdx.x] = offs.off[threadIdx.x];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (kick.frames_out && i == 0) kick.frames_out[n] = make_float4(kSentinelCoord, kSentinelCoord, kSentinelCoord, 0.0f);
    long long e_fx = 0, w_fx = 0, k_fx = 0;
    unsigned ins = 0;
    if (i < n)
        k_fx = fp32_row<kFixed, kEnergy, kPrefetch>(i, frames, pos, n, box, lj, s_off, rows, cap, counts, force, kick,
                                                    e_fx, w_fx, ins);
    if (kEnergy || kick.vel) flush_sums(e_fx, w_fx, ins, k_fx, acc);
}

// Boxes under 3 cells per side (all-pairs candidates): separations come from the double positions with the
// reference's minimum image, then narrow to float (the reference's mixed path does the same,
// src/Forcefield.cpp:373-386); the cutoff test uses the double r^2.
template <bool kFixed, bool kEnergy>
__global__ void k_force_fp32_small(const double4* __restrict__ pos, int n, Box box, FloatLJ lj,
                                   const uint32_t* __restrict__ rows, int cap, const int2* __restrict__ counts,
                                   double* __restrict__ force, unsigned long long* __restrict__ acc, KickArgs kick) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    long long e_fx = 0, w_fx = 0, k_fx = 0;
    unsigned ins = 0;
    if (i < n) {
        const double4 pi = pos[i];
        const int2 c = counts[i];
        const int m = c.x + c.y;
        FloatAcc<kFixed, kEnergy> a;
        for (int g0 = 0; g0 < m; g0 += 8) {
            float gx = 0.f, gy = 0.f, gz = 0.f, ge = 0.f, gw = 0.f;
            for (int s = g0; s < g0 + 8 && s < m; ++s) {
                const double4 pj = pos[rows[row_index(i, s, cap)] & kIndexMask];
                const double ddx = min_image(dsub(pi.x, pj.x), box);
                const double ddy = min_image(dsub(pi.y, pj.y), box);
                const double ddz = min_image(dsub(pi.z, pj.z), box);
                const float dx = static_cast<float>(ddx), dy = static_cast<float>(ddy), dz = static_cast<float>(ddz);
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, __fmul_rn(dz, dz)));
                const bool in = norm2(ddx, ddy, ddz) < lj.rc2d;  // the reference's cutoff test, in double
                float_pair<kEnergy>(dx, dy, dz, in, r2, lj, gx, gy, gz, ge, gw, ins);
            }
            a.add_group(gx, gy, gz, ge, gw, e_fx, w_fx);
        }
        k_fx = a.finish(i, n, force, kick);
    }
    if (kEnergy || kick.vel) flush_sums(e_fx, w_fx, ins, k_fx, acc);
}

// Converts the fixed-point sums to doubles: (pe, virial) in `energy_unit`s with the double-counted pairs halved
// into out[0..1], the inside count (halved, an integer) into *inside, and, when ke_out is set, the fused kinetic
// energy (2^-32 units) into *ke_out.
__global__ void k_finish_float_energy(const unsigned long long* __restrict__ acc, double* __restrict__ out,
                                      unsigned long long* __restrict__ inside, double* __restrict__ ke_out,
                                      double kinetic_unit, double energy_unit = kEnergyUnit) {
    out[0] = 0.5 * static_cast<double>(static_cast<long long>(acc[0])) * energy_unit;
    out[1] = 0.5 * static_cast<double>(static_cast<long long>(acc[1])) * energy_unit;
    *inside = acc[2] / 2;
    if (ke_out) *ke_out = static_cast<double>(static_cast<long long>(acc[3])) * kinetic_unit;
}

}  // namespace md
