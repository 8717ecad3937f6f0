// ORACLE — test infrastructure only: the serial FP64 CPU adjoint that the CUDA adjoint (md_adjoint_* in
// libmdgpu) is checked against bit for bit. Only tests/ load it; the product never calls it.
//
// The reference has no adjoint. The trajectory differentiated here is the reference's velocity-Verlet NVE step
// (src/Integrator.cpp:18-71: kick, drift and wrap, list update on half the skin, forces, kick) with the
// truncated and shifted Lennard-Jones pair terms (src/Forcefield.cpp:25-36), the minimum image and wrap of
// include/System.hpp:86-112 and the blocked summation of include/Parallel.hpp:32-57. Two choices differ from
// the reference and are made so that forward, recomputation and both implementations give the same bits:
//   - particles are never reordered: the Verlet list is built from a stable cell sort of particle indices
//     (src/CellList.cpp:9-52) and every particle's row holds all its partners within r_c + skin in the
//     reference's candidate order (27 cells in (dx, dy, dz) order, increasing index in a cell; all particles
//     in increasing index under 3 cells per side, src/NeighbourList.cpp:38-52 and :69);
//   - per-particle sums run over the whole row, so U = 0.5 sum_i sum_j e_ij and W = 0.5 sum_i sum_j f_ij r_ij^2.
// Objective (central finite differences through the reference library test it):
//   J = g_U * mean_k U_k + g_P * mean_k P_k over the steps k = 1..K, P_k = (2 KE_k + W_k) / (3 V).
// The backward pass is the discrete adjoint of that step sequence, with checkpoints of (positions,
// velocities, list reference positions) every `every` steps and recomputation of each segment.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

constexpr std::size_t kChunk = 1024;

template <typename F>
double blocked(std::size_t n, F&& f) {
    double total = 0.0;
    for (std::size_t b = 0; b * kChunk < n; ++b) {
        const std::size_t end = std::min(n, (b + 1) * kChunk);
        double s = 0.0;
        for (std::size_t i = b * kChunk; i < end; ++i) s += f(i);
        total += s;
    }
    return total;
}

struct Adj {
    std::size_t n = 0;
    double L = 0, invL = 0, quarterL = 0, V = 0;
    double eps = 1, sigma = 1, rc = 2.5, skin = 0.3, dt = 0.005;
    double sig2 = 0, eps24 = 0, eps4 = 0, shift = 0, rc2 = 0, rl2 = 0, half_dt = 0, inv_sigma = 0, shift_sigma = 0;
    int steps = 0, every = 0;
    std::vector<double> mass;
    std::vector<double> pos0, vel0;  // pos: 4 per particle; vel: component-major
    // list
    int ncps = 1;
    std::vector<double> ref;  // reference positions of the current list (4 per particle)
    std::vector<std::vector<std::size_t>> rows;
    // forward results
    std::vector<double> U, W, KE;
    std::vector<std::vector<double>> ck_pos, ck_vel, ck_ref;
    double meanU = 0, meanP = 0;

    double minImage(double d) const {
        if (std::fabs(d) <= quarterL) return d;
        return d - L * std::round(d * invL);
    }
    double wrap(double x) const { return x - L * std::floor(x * invL); }

    // Verlet list at `p` (becomes the reference positions)
    void build(const std::vector<double>& p) {
        ref = p;
        ncps = std::max(1, static_cast<int>(L / (rc + skin)));
        const double inv_cell = ncps / L;
        auto coord = [&](double x) {
            int c = static_cast<int>(x * inv_cell);
            c = c < ncps - 1 ? c : ncps - 1;
            return c > 0 ? c : 0;
        };
        const std::size_t nc = static_cast<std::size_t>(ncps) * ncps * ncps;
        std::vector<int> cell(n);
        std::vector<std::size_t> start(nc + 1, 0), order(n);
        for (std::size_t i = 0; i < n; ++i) {
            cell[i] = (coord(p[4 * i]) * ncps + coord(p[4 * i + 1])) * ncps + coord(p[4 * i + 2]);
            start[cell[i] + 1]++;
        }
        for (std::size_t c = 0; c < nc; ++c) start[c + 1] += start[c];
        std::vector<std::size_t> cur(start.begin(), start.end() - 1);
        for (std::size_t i = 0; i < n; ++i) order[cur[cell[i]]++] = i;
        rows.assign(n, {});
        auto within = [&](std::size_t i, std::size_t j) {
            const double dx = minImage(p[4 * i] - p[4 * j]);
            const double dy = minImage(p[4 * i + 1] - p[4 * j + 1]);
            const double dz = minImage(p[4 * i + 2] - p[4 * j + 2]);
            return dx * dx + dy * dy + dz * dz < rl2;
        };
        for (std::size_t i = 0; i < n; ++i) {
            auto& row = rows[i];
            if (ncps < 3) {
                for (std::size_t j = 0; j < n; ++j)
                    if (j != i && within(i, j)) row.push_back(j);
                continue;
            }
            const int c = cell[i], cx = c / (ncps * ncps), cy = (c / ncps) % ncps, cz = c % ncps;
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz) {
                        const int nb = (((cx + dx + ncps) % ncps) * ncps + (cy + dy + ncps) % ncps) * ncps +
                                       (cz + dz + ncps) % ncps;
                        for (std::size_t t = start[nb]; t < start[nb + 1]; ++t) {
                            const std::size_t j = order[t];
                            if (j != i && within(i, j)) row.push_back(j);
                        }
                    }
        }
    }

    bool stale(const std::vector<double>& p) const {
        for (std::size_t i = 0; i < n; ++i) {
            const double dx = minImage(p[4 * i] - ref[4 * i]);
            const double dy = minImage(p[4 * i + 1] - ref[4 * i + 1]);
            const double dz = minImage(p[4 * i + 2] - ref[4 * i + 2]);
            if (dx * dx + dy * dy + dz * dz > 0.25 * skin * skin) return true;
        }
        return false;
    }

    struct Pair {
        double dx, dy, dz, r2, fr, e, frp, frs, es;
    };
    // Pair terms of (i, j) at p; false beyond the cutoff
    bool pair(const std::vector<double>& p, std::size_t i, std::size_t j, Pair& q) const {
        q.dx = minImage(p[4 * i] - p[4 * j]);
        q.dy = minImage(p[4 * i + 1] - p[4 * j + 1]);
        q.dz = minImage(p[4 * i + 2] - p[4 * j + 2]);
        q.r2 = q.dx * q.dx + q.dy * q.dy + q.dz * q.dz;
        if (!(q.r2 < rc2)) return false;
        const double inv = 1.0 / q.r2;
        const double s2 = sig2 * inv;
        const double s6 = s2 * s2 * s2;
        const double s12 = s6 * s6;
        q.fr = eps24 * (2.0 * s12 - s6) * inv;                         // F/r (src/Forcefield.cpp:25-36)
        q.e = eps4 * (s12 - s6) - shift;
        const double inv2 = inv * inv;
        q.frp = eps24 * (4.0 * s6 - 14.0 * s12) * inv2;                 // d(F/r)/d(r^2)
        q.frs = eps24 * (24.0 * s12 - 6.0 * s6) * (inv * inv_sigma);    // d(F/r)/d(sigma)
        q.es = eps4 * (12.0 * s12 - 6.0 * s6) * inv_sigma - shift_sigma;  // d(e)/d(sigma), shift included
        return true;
    }

    // Forces, per-particle energy and virial row sums at p
    void forces(const std::vector<double>& p, std::vector<double>& f, std::vector<double>& u, std::vector<double>& w) const {
        for (std::size_t i = 0; i < n; ++i) {
            double fx = 0, fy = 0, fz = 0, ui = 0, wi = 0;
            Pair q;
            for (std::size_t j : rows[i]) {
                if (!pair(p, i, j, q)) continue;
                fx += q.fr * q.dx;
                fy += q.fr * q.dy;
                fz += q.fr * q.dz;
                ui += q.e;
                wi += q.fr * q.r2;
            }
            f[i] = fx;
            f[n + i] = fy;
            f[2 * n + i] = fz;
            u[i] = ui;
            w[i] = wi;
        }
    }

    double kinetic(const std::vector<double>& v) const {
        return blocked(n, [&](std::size_t i) {
            return 0.5 * mass[i] * (v[i] * v[i] + v[n + i] * v[n + i] + v[2 * n + i] * v[2 * n + i]);
        });
    }

    void kick(std::vector<double>& v, const std::vector<double>& f) const {
        for (int k = 0; k < 3; ++k)
            for (std::size_t i = 0; i < n; ++i) v[k * n + i] = v[k * n + i] + half_dt * f[k * n + i] / mass[i];
    }
    void drift(std::vector<double>& p, const std::vector<double>& v) const {
        for (std::size_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) p[4 * i + k] = wrap(p[4 * i + k] + dt * v[k * n + i]);
    }

    // One step from (p, v, f); returns U, W of the new state through the row sums u, w
    void step(std::vector<double>& p, std::vector<double>& v, std::vector<double>& f, std::vector<double>& u,
              std::vector<double>& w) {
        kick(v, f);
        drift(p, v);
        if (stale(p)) build(p);
        forces(p, f, u, w);
        kick(v, f);
    }

    void forward() {
        std::vector<double> p = pos0, v = vel0, f(3 * n), u(n), w(n);
        build(p);
        forces(p, f, u, w);
        U.assign(steps + 1, 0.0);
        W.assign(steps + 1, 0.0);
        KE.assign(steps + 1, 0.0);
        ck_pos.clear();
        ck_vel.clear();
        ck_ref.clear();
        double su = 0.0, sp = 0.0;
        for (int k = 1; k <= steps; ++k) {
            if ((k - 1) % every == 0) {
                ck_pos.push_back(p);
                ck_vel.push_back(v);
                ck_ref.push_back(ref);
            }
            step(p, v, f, u, w);
            U[k] = 0.5 * blocked(n, [&](std::size_t i) { return u[i]; });
            W[k] = 0.5 * blocked(n, [&](std::size_t i) { return w[i]; });
            KE[k] = kinetic(v);
            su += U[k];
            sp += (2.0 * KE[k] + W[k]) / (3.0 * V);
        }
        meanU = su / steps;
        meanP = sp / steps;
    }

    // One backward pair pass at p with weights w (3 x n): adds H(p) w (+ the objective's position gradient when
    // aU, aW are non-zero) to ar, and returns the parameter gradient terms
    void pass(const std::vector<double>& p, const std::vector<double>& wv, double aU, double aW, std::vector<double>& ar,
              double& geps, double& gsig) const {
        std::vector<double> pe(n), ps(n), us(n), ws(n), ue(n), we(n);
        for (std::size_t i = 0; i < n; ++i) {
            double fx = 0, fy = 0, fz = 0, hx = 0, hy = 0, hz = 0, gx = 0, gy = 0, gz = 0;
            double psi = 0, usi = 0, wsi = 0, uei = 0, wei = 0;
            const double wix = wv[i], wiy = wv[n + i], wiz = wv[2 * n + i];
            Pair q;
            for (std::size_t j : rows[i]) {
                if (!pair(p, i, j, q)) continue;
                fx += q.fr * q.dx;
                fy += q.fr * q.dy;
                fz += q.fr * q.dz;
                const double dwx = wix - wv[j], dwy = wiy - wv[n + j], dwz = wiz - wv[2 * n + j];
                const double t = 2.0 * q.frp * (q.dx * dwx + q.dy * dwy + q.dz * dwz);
                hx += q.fr * dwx + t * q.dx;
                hy += q.fr * dwy + t * q.dy;
                hz += q.fr * dwz + t * q.dz;
                const double g = 2.0 * (q.fr + q.r2 * q.frp);
                gx += g * q.dx;
                gy += g * q.dy;
                gz += g * q.dz;
                psi += q.frs * (q.dx * wix + q.dy * wiy + q.dz * wiz);
                usi += q.es;
                wsi += q.frs * q.r2;
                uei += q.e;
                wei += q.fr * q.r2;
            }
            ar[i] = ar[i] + -aU * fx + aW * gx + hx;
            ar[n + i] = ar[n + i] + -aU * fy + aW * gy + hy;
            ar[2 * n + i] = ar[2 * n + i] + -aU * fz + aW * gz + hz;
            pe[i] = wix * fx + wiy * fy + wiz * fz;
            ps[i] = psi;
            us[i] = usi;
            ws[i] = wsi;
            ue[i] = uei;
            we[i] = wei;
        }
        auto sum = [&](const std::vector<double>& a) { return blocked(n, [&](std::size_t i) { return a[i]; }); };
        // d/d eps: w . F / eps, and the objective's (aU U + aW W) / eps (U, W linear in eps)
        geps = sum(pe) / eps;
        gsig = sum(ps);
        if (aU != 0.0 || aW != 0.0) {
            const double Uk = 0.5 * sum(ue), Wk = 0.5 * sum(we);
            geps = geps + (aU * Uk + aW * Wk) / eps;
            gsig = gsig + aU * (0.5 * sum(us)) + aW * (0.5 * sum(ws));
        }
    }

    void weights(const std::vector<double>& av, std::vector<double>& wv) const {
        for (int k = 0; k < 3; ++k)
            for (std::size_t i = 0; i < n; ++i) wv[k * n + i] = half_dt * av[k * n + i] / mass[i];
    }

    void backward(double gU, double gP, double& deps, double& dsig, std::vector<double>& ar, std::vector<double>& av) {
        const double aU = gU / steps;
        const double aW = gP / (3.0 * V * steps);
        const double aK = 2.0 * aW;
        ar.assign(3 * n, 0.0);
        av.assign(3 * n, 0.0);
        deps = 0.0;
        dsig = 0.0;
        std::vector<double> wv(3 * n), f(3 * n), u(n), w(n);
        const int segments = static_cast<int>(ck_pos.size());
        for (int sgi = segments - 1; sgi >= 0; --sgi) {
            const int k0 = sgi * every, k1 = std::min(steps, k0 + every);
            // recompute the segment, keeping every state and its list's reference positions
            std::vector<std::vector<double>> P(k1 - k0 + 1), Vv(k1 - k0 + 1), R(k1 - k0 + 1);
            std::vector<double> p = ck_pos[sgi], v = ck_vel[sgi];
            build(ck_ref[sgi]);
            forces(p, f, u, w);
            P[0] = p;
            Vv[0] = v;
            R[0] = ref;
            for (int k = k0 + 1; k <= k1; ++k) {
                step(p, v, f, u, w);
                P[k - k0] = p;
                Vv[k - k0] = v;
                R[k - k0] = ref;
            }
            for (int j = k1; j > k0; --j) {
                const auto& pj = P[j - k0];
                const auto& vj = Vv[j - k0];
                // objective at s_j: velocity part, then the second half kick's pass at r_j with it
                for (int k = 0; k < 3; ++k)
                    for (std::size_t i = 0; i < n; ++i) av[k * n + i] = av[k * n + i] + aK * mass[i] * vj[k * n + i];
                weights(av, wv);
                if (ref != R[j - k0]) build(R[j - k0]);
                double ge = 0, gs = 0;
                pass(pj, wv, aU, aW, ar, ge, gs);
                deps = deps + ge;
                dsig = dsig + gs;
                // drift
                for (std::size_t t = 0; t < 3 * n; ++t) av[t] = av[t] + dt * ar[t];
                // first half kick: pass at r_{j-1}
                weights(av, wv);
                if (ref != R[j - 1 - k0]) build(R[j - 1 - k0]);
                pass(P[j - 1 - k0], wv, 0.0, 0.0, ar, ge, gs);
                deps = deps + ge;
                dsig = dsig + gs;
            }
        }
    }
};

}  // namespace

extern "C" {

void* orc_adj_create(std::int64_t n, double box, const double* pos4, const double* vel3, const double* mass,
                     double eps, double sigma, double rc, double skin, double dt, int steps, int every) {
    auto* a = new Adj;
    a->n = static_cast<std::size_t>(n);
    a->L = box;
    a->invL = 1.0 / box;
    a->quarterL = 0.25 * box;
    a->V = box * box * box;
    a->eps = eps;
    a->sigma = sigma;
    a->rc = rc;
    a->skin = skin;
    a->dt = dt;
    a->steps = steps;
    a->every = every;
    a->sig2 = sigma * sigma;
    a->eps24 = 24.0 * eps;
    a->eps4 = 4.0 * eps;
    const double sr6 = std::pow(sigma / rc, 6);
    const double sr12 = sr6 * sr6;
    a->shift = 4.0 * eps * (sr12 - sr6);
    a->rc2 = rc * rc;
    a->rl2 = (rc + skin) * (rc + skin);
    a->half_dt = 0.5 * dt;
    a->inv_sigma = 1.0 / sigma;
    a->shift_sigma = 4.0 * eps * (12.0 * sr12 - 6.0 * sr6) / sigma;
    a->pos0.assign(pos4, pos4 + 4 * n);
    a->vel0.assign(vel3, vel3 + 3 * n);
    a->mass.assign(n, 1.0);
    if (mass) a->mass.assign(mass, mass + n);
    return a;
}

void orc_adj_destroy(void* a) { delete static_cast<Adj*>(a); }

void orc_adj_forward(void* h, double* mean_pe, double* mean_p, double* pe_steps, double* w_steps, double* ke_steps) {
    auto* a = static_cast<Adj*>(h);
    a->forward();
    *mean_pe = a->meanU;
    *mean_p = a->meanP;
    for (int k = 1; k <= a->steps; ++k) {
        if (pe_steps) pe_steps[k - 1] = a->U[k];
        if (w_steps) w_steps[k - 1] = a->W[k];
        if (ke_steps) ke_steps[k - 1] = a->KE[k];
    }
}

void orc_adj_backward(void* h, double g_pe, double g_p, double* d_eps, double* d_sigma, double* d_pos3, double* d_vel3) {
    auto* a = static_cast<Adj*>(h);
    std::vector<double> ar, av;
    a->backward(g_pe, g_p, *d_eps, *d_sigma, ar, av);
    if (d_pos3) std::copy(ar.begin(), ar.end(), d_pos3);
    if (d_vel3) std::copy(av.begin(), av.end(), d_vel3);
}

}  // extern "C"
