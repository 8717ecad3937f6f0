// Shared device helpers for libmdgpu (sm_100a).
//
// FP64 parity: every double-precision operation on a path that must reproduce the reference bit for bit
// goes through the explicit round-to-nearest intrinsics below. nvcc never contracts __dmul_rn/__dadd_rn
// into an FMA, so the operation sequence is exactly the one the reference's C++ spells out.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace md {

constexpr int kCodeShift = 27;                       // neighbour entry: j in bits 0..26, cell code in 27..31
constexpr uint32_t kIndexMask = (1u << kCodeShift) - 1u;
constexpr int kMaxParticles = (1 << kCodeShift) - 2; // one slot is the sentinel
constexpr int kChunk = 1024;                         // deterministicSum block (include/Parallel.hpp:34)
constexpr uint32_t kSentinelCode = 31u;              // cell code of row padding entries (j = n, the sentinel)

// Neighbour rows are "uint4-interleaved" per group of 32 consecutive particles: entries [4q, 4q + 4) of
// particle i form the uint4 at index ((i >> 5) * cap / 4 + q) * 32 + (i & 31), so a warp of consecutive
// particles reading one uint4 each touches 512 contiguous bytes. cap is a multiple of 8. The row buffer
// must hold ceil(n / 32) * 32 * cap entries.
__host__ __device__ __forceinline__ size_t row_index(int i, int s, int cap) {
    return ((static_cast<size_t>(i >> 5) * (cap >> 2) + (s >> 2)) * 32 + (i & 31)) * 4 + (s & 3);
}
__device__ __forceinline__ uint4 row_quad(const uint32_t* __restrict__ rows, int i, int q, int cap) {
    return reinterpret_cast<const uint4*>(rows)[(static_cast<size_t>(i >> 5) * (cap >> 2) + q) * 32 + (i & 31)];
}
// row_quad with the streaming (evict-first) cache hint
__device__ __forceinline__ uint4 row_quad_stream(const uint32_t* __restrict__ rows, int i, int q, int cap) {
    return __ldcs(reinterpret_cast<const uint4*>(rows) + (static_cast<size_t>(i >> 5) * (cap >> 2) + q) * 32 + (i & 31));
}
inline size_t row_buffer_entries(long long n, int cap) { return static_cast<size_t>((n + 31) / 32) * 32 * cap; }

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Box constants of one system
struct Box {
    double L;        // box length
    double invL;     // 1 / L (src/System.cpp:10)
    double quarterL; // |d| <= L/4 implies round(d / L) == 0
};

// System::minimumImageDistance, one component (include/System.hpp:86-96): d - L * round(d * invL).
// When |d| <= L/4 the product rounds to +-0 and the reference's result is d itself, so the subtraction
// is skipped without changing a bit.
__device__ __forceinline__ double min_image(double d, const Box& b) {
    if (fabs(d) <= b.quarterL) return d;
    return dsub(d, dmul(b.L, round(dmul(d, b.invL))));
}

// System::wrapCoordinate (include/System.hpp:110-112): x - L * floor(x * invL)
__device__ __forceinline__ double wrap(double x, const Box& b) {
    return dsub(x, dmul(b.L, floor(dmul(x, b.invL))));
}

// dx^2 + dy^2 + dz^2 in the reference's left-to-right order
__device__ __forceinline__ double norm2(double dx, double dy, double dz) {
    return dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
}

// a1 b1 + a2 b2 + a3 b3 in left-to-right order
__device__ __forceinline__ double norm2p(double a1, double b1, double a2, double b2, double a3, double b3) {
    return dadd(dadd(dmul(a1, b1), dmul(a2, b2)), dmul(a3, b3));
}

// Lennard-Jones constants, precomputed on the host with the reference's expressions
// (src/Forcefield.cpp:8-15 and :25-36)
struct LJ {
    double sig2;   // sigma * sigma
    double eps24;  // 24 * epsilon
    double eps4;   // 4 * epsilon
    double shift;  // 4 eps ((s/rc)^12 - (s/rc)^6)
    double rc2;    // cut_off^2
};

// LennardJonesForceField::pairTerms (src/Forcefield.cpp:25-36): F/r and the shifted energy
__device__ __forceinline__ void pair_terms(double r2, const LJ& p, double& f_over_r, double& energy) {
    const double inv_r2 = ddiv(1.0, r2);
    const double sr2 = dmul(p.sig2, inv_r2);
    const double sr6 = dmul(dmul(sr2, sr2), sr2);
    const double sr12 = dmul(sr6, sr6);
    f_over_r = dmul(dmul(p.eps24, dsub(dmul(2.0, sr12), sr6)), inv_r2);
    energy = dsub(dmul(p.eps4, dsub(sr12, sr6)), p.shift);
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ long long warp_sum_i64(long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace md
