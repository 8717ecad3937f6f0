// Adjoint of the FP64 velocity-Verlet trajectory (md_adjoint_* in include/md_b200.h): gradients of the
// trajectory averages of the potential energy and the virial pressure with respect to epsilon, sigma and the
// initial positions and velocities.
//
// The trajectory is the reference's NVE step (src/Integrator.cpp:18-71) with the truncated and shifted pair
// terms (src/Forcefield.cpp:25-36), minimum image and wrap (include/System.hpp:86-112) and blocked sums
// (include/Parallel.hpp:32-57), with two choices that make forward runs, recomputations and the CPU adjoint give
// the same bits: particles are never reordered (the list is built from a stable cell sort of indices), and each
// particle's row holds all its partners within r_c + skin in the reference's candidate order, so every
// per-particle sum runs over that whole row in that order. Every double operation is an explicit
// round-to-nearest intrinsic (no contraction).
//
// For a pair with separation d, r2 = |d|^2, s6 = (sigma^2 / r2)^3, s12 = s6^2:
//   F/r  = fr  = 24 eps (2 s12 - s6) / r2          d fr / d r2  = frp = 24 eps (4 s6 - 14 s12) / r2^2
//   e    = 4 eps (s12 - s6) - shift                 d fr / d sig = frs = 24 eps (24 s12 - 6 s6) / (r2 sig)
//   d e / d sig = es = 4 eps (12 s12 - 6 s6) / sig - d shift / d sig
// The force Jacobian block of a pair is B = fr I + 2 frp d d^T, so (H w)_i = sum_j B_ij (w_i - w_j).
#pragma once

#include "md_common.cuh"

namespace md {

struct AdjConsts {
    Box box;
    double sig2, eps24, eps4, shift, rc2;
    double eps, inv_sigma, shift_sigma;
};

struct AdjPair {
    double dx, dy, dz, r2, fr, e, frp, frs, es;
};

// The pair (i, j) at positions a, b; false at or beyond the cutoff. kDeriv adds frp, frs, es.
template <bool kDeriv>
__device__ __forceinline__ bool adj_pair(const double4& a, const double4& b, const AdjConsts& c, AdjPair& q) {
    q.dx = min_image(dsub(a.x, b.x), c.box);
    q.dy = min_image(dsub(a.y, b.y), c.box);
    q.dz = min_image(dsub(a.z, b.z), c.box);
    q.r2 = norm2(q.dx, q.dy, q.dz);
    if (!(q.r2 < c.rc2)) return false;
    const double inv = ddiv(1.0, q.r2);
    const double s2 = dmul(c.sig2, inv);
    const double s6 = dmul(dmul(s2, s2), s2);
    const double s12 = dmul(s6, s6);
    q.fr = dmul(dmul(c.eps24, dsub(dmul(2.0, s12), s6)), inv);
    q.e = dsub(dmul(c.eps4, dsub(s12, s6)), c.shift);
    if (kDeriv) {
        const double inv2 = dmul(inv, inv);
        q.frp = dmul(dmul(c.eps24, dsub(dmul(4.0, s6), dmul(14.0, s12))), inv2);
        q.frs = dmul(dmul(c.eps24, dsub(dmul(24.0, s12), dmul(6.0, s6))), dmul(inv, c.inv_sigma));
        q.es = dsub(dmul(dmul(c.eps4, dsub(dmul(12.0, s12), dmul(6.0, s6))), c.inv_sigma), c.shift_sigma);
    }
    return true;
}

// Full rows (every partner within r_c + skin, the particle itself excluded) in the reference's candidate
// order from a stable cell sort (order[start[c] .. start[c + 1]) lists cell c's particles by index); under 3
// cells per side, every particle by index. counts[i] is kept within cap; max_count gets the true longest row.
__global__ void k_adj_rows(const double4* __restrict__ pos, int n, Box box, double rl2, int ncps,
                           const int* __restrict__ cell_of, const int* __restrict__ start,
                           const uint32_t* __restrict__ order, int cap, uint32_t* __restrict__ rows,
                           int* __restrict__ counts, int* __restrict__ max_count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 pi = pos[i];
    int cnt = 0;
    auto take = [&](int j) {
        if (j == i) return;
        const double4 pj = pos[j];
        const double dx = min_image(dsub(pi.x, pj.x), box);
        const double dy = min_image(dsub(pi.y, pj.y), box);
        const double dz = min_image(dsub(pi.z, pj.z), box);
        if (!(norm2(dx, dy, dz) < rl2)) return;
        if (cnt < cap) rows[row_index(i, cnt, cap)] = static_cast<uint32_t>(j);
        ++cnt;
    };
    if (ncps < 3) {
        for (int j = 0; j < n; ++j) take(j);
    } else {
        const int c = cell_of[i];
        const int cx = c / (ncps * ncps), cy = (c / ncps) % ncps, cz = c % ncps;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    const int nb = (((cx + dx + ncps) % ncps) * ncps + (cy + dy + ncps) % ncps) * ncps +
                                   (cz + dz + ncps) % ncps;
                    for (int t = start[nb]; t < start[nb + 1]; ++t) take(static_cast<int>(order[t]));
                }
    }
    counts[i] = cnt < cap ? cnt : cap;
    atomicMax(max_count, cnt);
}

// Forces (3 x n, component-major) and the row sums of pair energy and virial
__global__ void k_adj_forces(const double4* __restrict__ pos, int n, AdjConsts c, const uint32_t* __restrict__ rows,
                             int cap, const int* __restrict__ counts, double* __restrict__ force,
                             double* __restrict__ u, double* __restrict__ w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 pi = pos[i];
    double fx = 0.0, fy = 0.0, fz = 0.0, ui = 0.0, wi = 0.0;
    AdjPair q;
    const int m = counts[i];
    for (int s = 0; s < m; ++s) {
        if (!adj_pair<false>(pi, pos[rows[row_index(i, s, cap)]], c, q)) continue;
        fx = dadd(fx, dmul(q.fr, q.dx));
        fy = dadd(fy, dmul(q.fr, q.dy));
        fz = dadd(fz, dmul(q.fr, q.dz));
        ui = dadd(ui, q.e);
        wi = dadd(wi, dmul(q.fr, q.r2));
    }
    force[i] = fx;
    force[static_cast<size_t>(n) + i] = fy;
    force[2 * static_cast<size_t>(n) + i] = fz;
    u[i] = ui;
    w[i] = wi;
}

// Blocked sums of two per-particle arrays into (sum a, sum b) block partials (k_kinetic_blocks' layout), for
// k_sum_blocks
__global__ void k_adj_blocks2(const double* __restrict__ a, const double* __restrict__ b, int n,
                              double2* __restrict__ block_sums, int nblocks) {
    extern __shared__ double2 sm_ab[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int blk = blockIdx.x * 4 + warp;
    if (blk >= nblocks) return;
    double2* v = sm_ab + warp * kChunk;
    const int i0 = blk * kChunk;
    const int m = n - i0 < kChunk ? n - i0 : kChunk;
    for (int t = lane; t < m; t += 32) v[t] = make_double2(a[i0 + t], b ? b[i0 + t] : 0.0);
    __syncwarp();
    if (lane == 0) {
        double sa = 0.0, sb = 0.0;
        for (int t = 0; t < m; ++t) {
            sa = dadd(sa, v[t].x);
            sb = dadd(sb, v[t].y);
        }
        block_sums[blk] = make_double2(sa, sb);
    }
}

// After step k of the forward pass: U_k = 0.5 sum u, W_k = 0.5 sum w, KE_k, and the running sums of U and
// P = (2 KE + W) / 3V in run[0], run[1]
__global__ void k_adj_record(const double* __restrict__ uw, const double* __restrict__ ke, double volume, int k,
                             double* __restrict__ U, double* __restrict__ W, double* __restrict__ KE,
                             double* __restrict__ run) {
    const double u = dmul(0.5, uw[0]), w = dmul(0.5, uw[1]), kin = ke[0];
    U[k] = u;
    W[k] = w;
    KE[k] = kin;
    run[0] = dadd(run[0], u);
    run[1] = dadd(run[1], ddiv(dadd(dmul(2.0, kin), w), dmul(3.0, volume)));
}

// av += (aK m) v: the objective's kinetic-energy term at a state
__global__ void k_adj_obj_v(double* __restrict__ av, const double* __restrict__ vel, const double* __restrict__ mass,
                            int n, double aK) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * n) return;
    const int i = t % n;
    av[t] = dadd(av[t], dmul(dmul(aK, mass[i]), vel[t]));
}

// wv = (half_dt av) / m: the weights of a half kick's backward pass
__global__ void k_adj_weights(const double* __restrict__ av, const double* __restrict__ mass, int n, double half_dt,
                              double* __restrict__ wv) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * n) return;
    wv[t] = ddiv(dmul(half_dt, av[t]), mass[t % n]);
}

// av += dt ar: the drift's backward
__global__ void k_adj_drift_back(double* __restrict__ av, const double* __restrict__ ar, int n, double dt) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 3 * n) av[t] = dadd(av[t], dmul(dt, ar[t]));
}

// One backward pass at positions pos with weights wv: ar_i += -aU F_i + aW dW/dr_i + (H w)_i, and per particle
// the parameter-gradient terms: pe = w_i . F_i, ps = w_i . dF_i/dsig, us = sum es, ws = sum frs r2,
// ue = sum e, we = sum fr r2 (the last four for the objective's own parameter derivatives)
__global__ void k_adj_pass(const double4* __restrict__ pos, int n, AdjConsts c, const uint32_t* __restrict__ rows,
                           int cap, const int* __restrict__ counts, const double* __restrict__ wv, double aU,
                           double aW, double* __restrict__ ar, double* __restrict__ pe, double* __restrict__ ps,
                           double* __restrict__ us, double* __restrict__ ws, double* __restrict__ ue,
                           double* __restrict__ we) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t N = static_cast<size_t>(n);
    const double4 pi = pos[i];
    const double wix = wv[i], wiy = wv[N + i], wiz = wv[2 * N + i];
    double fx = 0.0, fy = 0.0, fz = 0.0, hx = 0.0, hy = 0.0, hz = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    double psi = 0.0, usi = 0.0, wsi = 0.0, uei = 0.0, wei = 0.0;
    AdjPair q;
    const int m = counts[i];
    for (int s = 0; s < m; ++s) {
        const int j = static_cast<int>(rows[row_index(i, s, cap)]);
        if (!adj_pair<true>(pi, pos[j], c, q)) continue;
        fx = dadd(fx, dmul(q.fr, q.dx));
        fy = dadd(fy, dmul(q.fr, q.dy));
        fz = dadd(fz, dmul(q.fr, q.dz));
        const double dwx = dsub(wix, wv[j]), dwy = dsub(wiy, wv[N + j]), dwz = dsub(wiz, wv[2 * N + j]);
        const double t = dmul(dmul(2.0, q.frp), norm2p(q.dx, dwx, q.dy, dwy, q.dz, dwz));
        hx = dadd(hx, dadd(dmul(q.fr, dwx), dmul(t, q.dx)));
        hy = dadd(hy, dadd(dmul(q.fr, dwy), dmul(t, q.dy)));
        hz = dadd(hz, dadd(dmul(q.fr, dwz), dmul(t, q.dz)));
        const double g = dmul(2.0, dadd(q.fr, dmul(q.r2, q.frp)));
        gx = dadd(gx, dmul(g, q.dx));
        gy = dadd(gy, dmul(g, q.dy));
        gz = dadd(gz, dmul(g, q.dz));
        psi = dadd(psi, dmul(q.frs, norm2p(q.dx, wix, q.dy, wiy, q.dz, wiz)));
        usi = dadd(usi, q.es);
        wsi = dadd(wsi, dmul(q.frs, q.r2));
        uei = dadd(uei, q.e);
        wei = dadd(wei, dmul(q.fr, q.r2));
    }
    const double F[3] = {fx, fy, fz}, H[3] = {hx, hy, hz}, G[3] = {gx, gy, gz};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const size_t o = k * N + i;
        ar[o] = dadd(dadd(dadd(ar[o], dmul(-aU, F[k])), dmul(aW, G[k])), H[k]);
    }
    pe[i] = norm2p(wix, fx, wiy, fy, wiz, fz);
    ps[i] = psi;
    us[i] = usi;
    ws[i] = wsi;
    ue[i] = uei;
    we[i] = wei;
}

// The pass's parameter gradients from its six blocked sums (sums[0..5] = pe, ps, us, ws, ue, we):
// theta[0] += sum pe / eps (+ (aU U + aW W) / eps), theta[1] += sum ps (+ aU dU/dsig + aW dW/dsig)
__global__ void k_adj_theta(const double* __restrict__ sums, double eps, double aU, double aW, bool objective,
                            double* __restrict__ theta) {
    double geps = ddiv(sums[0], eps);
    double gsig = sums[1];
    if (objective) {
        const double Uk = dmul(0.5, sums[4]), Wk = dmul(0.5, sums[5]);
        geps = dadd(geps, ddiv(dadd(dmul(aU, Uk), dmul(aW, Wk)), eps));
        gsig = dadd(dadd(gsig, dmul(aU, dmul(0.5, sums[2]))), dmul(aW, dmul(0.5, sums[3])));
    }
    theta[0] = dadd(theta[0], geps);
    theta[1] = dadd(theta[1], gsig);
}

}  // namespace md
