// MD_PREC_FX32: float pair terms for the pairs whose force is small, double pair terms on exact fixed-point
// separations for the close pairs, 64-bit fixed-point sums.
//
// Why the split: a float pair term carries a relative error of a few 1e-7 (the force goes as r^-14, so the
// rounding of r^2 alone is amplified sevenfold). That is below 1e-6 of a particle's net force only where the
// pair force itself is small. Pairs beyond 1.2 sigma have |F| <= 2.4 eps/sigma; the few closer pairs (about one in
// six of a row) carry forces up to 1e2 and, evaluated in float, leave 60 % of particles above 1e-6 relative
// error. So every row is split once per list build into a near row and a far row. The near row holds the entries
// whose pair was closer than (1.2 sigma + skin) at the build (at most 16, the closest), evaluated in double on the
// 32-bit fixed-point frames (2^-28 units) of MD_PREC_FX64, whose integer differences are exact separations; the
// far row holds the rest, evaluated in float on the float frames of MD_PREC_FP32FX with its pinned operation
// sequence. Between rebuilds every particle stays within skin/2 of its build position, so a pair evaluated in
// float is never closer than 1.2 sigma unless its row had more than 16 near entries.
//
// Sums: every group of 8 entries is added into 64-bit fixed point (forces at 2^-32, energy and virial at 2^-30),
// so the result does not depend on the launch shape.
#pragma once

#include "md_common.cuh"
#include "md_fp32.cuh"
#include "md_fx64.cuh"

namespace md {

constexpr int kFx32NearCap = 16;     // near-row capacity (two groups of 8)
constexpr int kFx32FixNear = 48;     // near entries a row with more than kFx32NearCap of them chooses from

// Entries of the near rows: the same interleaved layout as the list's rows with capacity kFx32NearCap
inline size_t fx32_near_entries(long long n) { return row_buffer_entries(n, kFx32NearCap); }

__device__ __forceinline__ void quad_put(uint4& b, int k, uint32_t e) {
    b.x = k == 0 ? e : b.x;
    b.y = k == 1 ? e : b.y;
    b.z = k == 2 ? e : b.z;
    b.w = k == 3 ? e : b.w;
}

// Appends entry e to a row being written a quad at a time: b holds the open quad, len the row length, q the row's
// first quad (quad k at q[32 k], the interleaved layout)
__device__ __forceinline__ void row_append(uint4& b, int& len, uint4* q, uint32_t e) {
    quad_put(b, len & 3, e);
    if ((++len & 3) == 0) q[((len >> 2) - 1) * 32] = b;
}

// Pads a row written by row_append with sentinel entries to a multiple of 8 and returns its group count
__device__ __forceinline__ int row_close(uint4& b, int& len, uint4* q, uint32_t pad) {
    const int padded = (len + 7) & ~7;
    while (len < padded) row_append(b, len, q, pad);
    return padded >> 3;
}

// The split test: the pair of entry e was closer than sqrt(near2) at the build, on the float frames of the build's
// positions (ref_frames) and the float offsets of the entry's cell code
__device__ __forceinline__ float split_r2(const float4& qi, const float4* __restrict__ ref_frames,
                                          const float4* s_off, uint32_t e) {
    float dx, dy, dz;
    return float_separation(qi, ref_frames[e & kIndexMask], s_off[e >> kCodeShift], dx, dy, dz);
}

// The split rule. Near row: the entries whose pair was closer than sqrt(near2) at the build, in row order (the
// kFx32NearCap closest when there are more), then the last entries of the far part in row order up to the next
// multiple of 8 (where there are enough), then sentinels to that multiple. Far row: every other entry in row order,
// then sentinels to a multiple of 8. counts_nf[i] = (near groups, far groups).
//
// k_rows_split applies it in one pass over each row, thread per particle, 8 entries a step with their 8 gathers
// issued together and the next two row quads prefetched. Each warp stages its 32 rows' outputs in shared memory,
// transposed ([slot][lane]: lanes never share a bank): the near row whole, the far row in a ring of 16 entries
// whose complete quads go out to global memory two quads behind the head, so that at the row's end the last far
// entries are still at hand to fill the near row. Every global store is a whole 16-byte quad with the streaming
// hint, and the staging is kept small (17 KB a block) so that L1 keeps room for the gathered frames. A row with
// more near entries than kFx32NearCap is marked (near groups = -1) for k_rows_split_fix, which chooses the closest.
constexpr int kSplitThreads = 128;
constexpr int kSplitRing = 16;  // far entries staged per lane: at most 11 after a drain (the 8 held back and 3 of an
                                // open quad) and 4 arriving before the next
__global__ void __launch_bounds__(kSplitThreads) k_rows_split(const float4* __restrict__ ref_frames, int n,
                                                              CellOffsets offs, float near2,
                                                              const uint32_t* __restrict__ rows, int cap,
                                                              const int2* __restrict__ counts,
                                                              uint32_t* __restrict__ near_rows,
                                                              uint32_t* __restrict__ far_rows, int2* __restrict__ counts_nf) {
    __shared__ float4 s_off[32];
    __shared__ uint32_t s_near[kSplitThreads / 32][kFx32NearCap][32];
    __shared__ uint32_t s_far[kSplitThreads / 32][kSplitRing][32];
    if (threadIdx.x < 32) s_off[threadIdx.x] = offs.off[threadIdx.x];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    uint32_t(*sn)[32] = s_near[w];
    uint32_t(*sf)[32] = s_far[w];
    const float4 qi = ref_frames[i];
    const int2 c = counts[i];
    const int m = c.x + c.y;
    const size_t lane = static_cast<size_t>(l);
    const uint4* rq = reinterpret_cast<const uint4*>(rows) + static_cast<size_t>(i >> 5) * (cap >> 2) * 32 + lane;
    uint4* nq = reinterpret_cast<uint4*>(near_rows) + static_cast<size_t>(i >> 5) * (kFx32NearCap >> 2) * 32 + lane;
    uint4* fq = reinterpret_cast<uint4*>(far_rows) + static_cast<size_t>(i >> 5) * (cap >> 2) * 32 + lane;
    int nn = 0, nf = 0, fw = 0;  // near entries, far entries, far entries written out
    bool over = false;
    // 8 entries (two quads) per step, the next two quads prefetched; rows are padded with sentinels to a multiple
    // of 8, so every entry of a step can be loaded and only the real ones (s + u < m) are kept
    uint4 p0 = make_uint4(0, 0, 0, 0), p1 = p0;
    if (m > 0) {
        p0 = __ldcs(rq);
        p1 = __ldcs(rq + 32);
    }
    for (int s = 0; s < m; s += 8) {
        const uint32_t ent[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
        if (s + 8 < m) {
            p0 = __ldcs(rq + ((s >> 2) + 2) * 32);
            p1 = __ldcs(rq + ((s >> 2) + 3) * 32);
        }
        float4 fj[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) fj[u] = ref_frames[ent[u] & kIndexMask];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const uint32_t e = ent[u];
            float dx, dy, dz;
            const bool near = float_separation(qi, fj[u], s_off[e >> kCodeShift], dx, dy, dz) < near2;
            const bool real = s + u < m;
            const bool to_near = real && near && nn < kFx32NearCap;
            over |= real && near && !to_near;
            uint32_t* dst = to_near ? &sn[nn][l] : &sf[nf & (kSplitRing - 1)][l];
            if (real) *dst = e;
            nn += to_near ? 1 : 0;
            nf += real && !to_near ? 1 : 0;
            if ((u & 3) == 3 && nf - fw >= 12) {  // a complete quad beyond the 8 held back
                const int r = fw & (kSplitRing - 1);
                __stcs(fq + (fw >> 2) * 32, make_uint4(sf[r][l], sf[r + 1][l], sf[r + 2][l], sf[r + 3][l]));
                fw += 4;
            }
        }
    }
    const uint32_t pad = static_cast<uint32_t>(n) | (kSentinelCode << kCodeShift);
    // the near row: its entries, the last far entries up to a multiple of 8, sentinels
    const int near_len = (nn + 7) & ~7;
    const int take = min(near_len - nn, nf);
    for (int k = 0; k < take; ++k) sn[nn + k][l] = sf[(nf - take + k) & (kSplitRing - 1)][l];
    for (int k = nn + take; k < near_len; ++k) sn[k][l] = pad;
    for (int k = 0; k < near_len; k += 4)
        __stcs(nq + (k >> 2) * 32, make_uint4(sn[k][l], sn[k + 1][l], sn[k + 2][l], sn[k + 3][l]));
    // the far row's rest: the entries still staged and not taken, then sentinels
    const int far_len = nf - take;
    const int far_padded = (far_len + 7) & ~7;
    for (int k = fw; k < far_padded; k += 4) {
        uint32_t v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = k + u < far_len ? sf[(k + u) & (kSplitRing - 1)][l] : pad;
        __stcs(fq + (k >> 2) * 32, make_uint4(v[0], v[1], v[2], v[3]));
    }
    counts_nf[i] = make_int2(over ? -1 : near_len >> 3, far_padded >> 3);
}

// The rows k_rows_split marked, by the same rule: the near part is the kFx32NearCap closest near entries (of the
// first kFx32FixNear in row order; the farthest are dropped one at a time, the later of equal ones first).
// Grid-stride over all particles; only marked rows do work.
__global__ void __launch_bounds__(128) k_rows_split_fix(const float4* __restrict__ ref_frames, int n, CellOffsets offs,
                                                        float near2, const uint32_t* __restrict__ rows, int cap,
                                                        const int2* __restrict__ counts, uint32_t* __restrict__ near_rows,
                                                        uint32_t* __restrict__ far_rows, int2* __restrict__ counts_nf) {
    static_assert(kFx32FixNear < 64, "the kept near entries are a 64-bit mask");
    __shared__ float4 s_off[32];
    if (threadIdx.x < 32) s_off[threadIdx.x] = offs.off[threadIdx.x];
    __syncthreads();
    auto entry = [&](int i, int s) {
        const uint4 q = row_quad(rows, i, s >> 2, cap);
        return (s & 3) == 0 ? q.x : (s & 3) == 1 ? q.y : (s & 3) == 2 ? q.z : q.w;
    };
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (counts_nf[i].x >= 0) continue;
        const float4 qi = ref_frames[i];
        const int2 c = counts[i];
        const int m = c.x + c.y;
        float r2s[kFx32FixNear];
        int slots[kFx32FixNear];
        int k = 0;
        for (int s = 0; s < m && k < kFx32FixNear; ++s) {
            const float r2 = split_r2(qi, ref_frames, s_off, entry(i, s));
            if (r2 < near2) {
                r2s[k] = r2;
                slots[k] = s;
                ++k;
            }
        }
        unsigned long long keep = (1ull << k) - 1;
        int kept = k;
        for (; kept > kFx32NearCap; --kept) {
            int far_t = 0;
            float far_r2 = -1.0f;
            for (int t = 0; t < k; ++t)
                if (((keep >> t) & 1) && r2s[t] >= far_r2) {
                    far_r2 = r2s[t];
                    far_t = t;
                }
            keep &= ~(1ull << far_t);
        }
        // near part in row order; the last `take` entries of the far part move to the near row
        const int near_len = (kept + 7) & ~7;
        const int far_all = m - kept;
        const int take = min(near_len - kept, far_all);
        const size_t lane = static_cast<size_t>(i & 31);
        uint4* nq = reinterpret_cast<uint4*>(near_rows) + static_cast<size_t>(i >> 5) * (kFx32NearCap >> 2) * 32 + lane;
        uint4* fq = reinterpret_cast<uint4*>(far_rows) + static_cast<size_t>(i >> 5) * (cap >> 2) * 32 + lane;
        uint4 nb = make_uint4(0, 0, 0, 0), fb = nb;
        uint32_t moved[8];
        int nn = 0, nf = 0, f = 0, t = 0;
        for (int s = 0; s < m; ++s) {
            const uint32_t e = entry(i, s);
            bool sel = false;
            if (t < k && slots[t] == s) sel = (keep >> t++) & 1;
            if (sel) {
                row_append(nb, nn, nq, e);
            } else {
                if (f >= far_all - take) moved[f - (far_all - take)] = e;
                else row_append(fb, nf, fq, e);
                ++f;
            }
        }
        for (int u = 0; u < take; ++u) row_append(nb, nn, nq, moved[u]);
        const uint32_t pad = static_cast<uint32_t>(n) | (kSentinelCode << kCodeShift);
        const int ng = row_close(nb, nn, nq, pad);
        const int fg = row_close(fb, nf, fq, pad);
        counts_nf[i] = make_int2(ng, fg);
    }
}

// Thread per particle over its near row and then its far row on a resident grid (each thread takes particles i,
// i + grid, ...): the near groups in double on the fixed-point frames (fx64_group, MD_PREC_FX64's sequence), the
// far groups in float on the float frames (float_group, MD_PREC_FP32FX's sequence); row quads prefetched a group
// ahead with streaming loads; the fused closing kick, kinetic energy and, with kick.pos_out, the next step's kick
// and drift writing both kinds of frames, as in the other float modes.
template <bool kEnergy>
__global__ void __launch_bounds__(128, 5) k_force_fx32(const int4* __restrict__ iframes, const float4* __restrict__ frames,
                                                    const double4* __restrict__ pos, int n, Box box, Fx64LJ dlj,
                                                    FloatLJ flj, FixedOffsets ioffs, CellOffsets foffs,
                                                    const uint4* __restrict__ rows_q, unsigned far_q0, int cap,
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
        const int near_groups = c.x, groups = c.x + c.y;
        FloatAcc<true, kEnergy> a;
        // quad indices into rows_q: the near rows first, the far rows from far_q0 (interleaved layouts)
        const unsigned far_q = far_q0 + static_cast<unsigned>(i >> 5) * (cap >> 2) * 32 + (i & 31);
        unsigned rq = near_groups > 0 ? static_cast<unsigned>(i >> 5) * (kFx32NearCap >> 2) * 32 + (i & 31) : far_q;
        uint4 n0 = make_uint4(0, 0, 0, 0), n1 = n0;
        if (groups > 0) {
            n0 = __ldcs(rows_q + rq);
            n1 = __ldcs(rows_q + rq + 32);
        }
        for (int g = 0; g < groups; ++g) {
            const uint4 e0 = n0, e1 = n1;
            rq = g + 1 == near_groups ? far_q : rq + 64;
            if (g + 1 < groups) {
                n0 = __ldcs(rows_q + rq);
                n1 = __ldcs(rows_q + rq + 32);
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
