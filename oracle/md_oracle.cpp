// ORACLE — test infrastructure only. This is a serial CPU restatement of the Lennard-Jones hot path of
// nhantran1711/molecular-dynamics, written from the reference's behaviour (every function cites the
// reference file:line it follows). It is the checker for the CUDA library: only tests/, the smoke check
// and bench.py's cpu_baseline / reference legs load it. The product never calls it.
//
// Parity pinning: tests/test_oracle_golden.py checks this file against golden vectors that
// tests/golden/make_golden.py generated by running the reference itself (compiled from its own sources
// by oracle/Makefile into oracle/_ref/).
//
// All floating point follows the reference's operation order with IEEE double rounding and no FMA
// contraction (built with -ffp-contract=off), so FP64 results are bit-identical to the reference.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numbers>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

std::string g_error;

// deterministicSum: 1024-element blocks summed in order, then the block sums in order
// (reference include/Parallel.hpp:32-57, blockSize at :34)
template <typename F>
double blockedSum(std::size_t n, F&& f) {
    constexpr std::size_t block = 1024;
    double total = 0.0;
    for (std::size_t b = 0; b * block < n; ++b) {
        const std::size_t end = std::min(n, (b + 1) * block);
        double s = 0.0;
        for (std::size_t i = b * block; i < end; ++i) {
            s += f(i);
        }
        total += s;
    }
    return total;
}

struct Sys {
    std::size_t n = 0;
    double L = 0.0;
    double invL = 0.0;
    std::vector<double> pos;  // 4 per particle (x, y, z, pad), include/System.hpp:22
    std::vector<double> vel[3];
    std::vector<double> force[3];
    std::vector<double> mass;
    std::vector<std::uint64_t> id;

    // include/System.hpp:86-96
    void minimumImage(const double* ri, const double* rj, double* dr) const {
        for (int k = 0; k < 3; ++k) {
            double d = ri[k] - rj[k];
            d -= L * std::round(d * invL);
            dr[k] = d;
        }
    }
    // include/System.hpp:110-112
    double wrap(double x) const {
        return x - L * std::floor(x * invL);
    }
    // src/System.cpp:42-64
    void reorder(const std::vector<std::size_t>& order) {
        std::vector<double> p(pos.size());
        for (std::size_t k = 0; k < n; ++k) {
            for (int c = 0; c < 4; ++c) {
                p[4 * k + c] = pos[4 * order[k] + c];
            }
        }
        pos.swap(p);
        auto perm = [&](auto& v) {
            std::remove_reference_t<decltype(v)> s(v.size());
            for (std::size_t k = 0; k < n; ++k) {
                s[k] = v[order[k]];
            }
            v.swap(s);
        };
        for (int k = 0; k < 3; ++k) {
            perm(vel[k]);
            perm(force[k]);
        }
        perm(mass);
        perm(id);
    }
    // src/System.cpp:67-76
    double kinetic() const {
        return blockedSum(n, [&](std::size_t i) {
            return 0.5 * mass[i] * (vel[0][i] * vel[0][i] + vel[1][i] * vel[1][i] + vel[2][i] * vel[2][i]);
        });
    }
    // src/System.cpp:79-82
    double temperature() const {
        const double dof = 3.0 * static_cast<double>(n) - 3.0;
        return 2.0 * kinetic() / dof;
    }
    // FNV-1a over (x, vx, y, vy, z, vz) per particle, src/System.cpp:85-105
    std::uint64_t hash() const {
        std::uint64_t h = 14695981039346656037ull;
        auto mix = [&h](double v) {
            std::uint64_t bits;
            std::memcpy(&bits, &v, 8);
            for (unsigned b = 0; b < 8; ++b) {
                h ^= (bits >> (8u * b)) & 0xffu;
                h *= 1099511628211ull;
            }
        };
        for (std::size_t i = 0; i < n; ++i) {
            for (int k = 0; k < 3; ++k) {
                mix(pos[4 * i + k]);
                mix(vel[k][i]);
            }
        }
        return h;
    }
};

struct Cells {
    double minSize = 0.0;
    int ncps = 0;
    std::vector<std::uint64_t> start;
    std::vector<std::uint64_t> particles;
    std::vector<int> cellOf;

    // Counting sort by cell, stable in particle index (src/CellList.cpp:9-52)
    void build(const Sys& s) {
        ncps = std::max(1, static_cast<int>(s.L / minSize));                       // :14
        const int nCells = ncps * ncps * ncps;
        const double inv = ncps / s.L;                                              // :18
        cellOf.assign(s.n, 0);
        start.assign(static_cast<std::size_t>(nCells) + 1, 0);
        particles.assign(s.n, 0);
        for (std::size_t i = 0; i < s.n; ++i) {
            int c[3];
            for (int k = 0; k < 3; ++k) {
                c[k] = std::min(static_cast<int>(s.pos[4 * i + k] * inv), ncps - 1);  // :34
            }
            cellOf[i] = (c[0] * ncps + c[1]) * ncps + c[2];                        // :38
            ++start[static_cast<std::size_t>(cellOf[i]) + 1];
        }
        for (int c = 0; c < nCells; ++c) {                                           // :43-45
            start[c + 1] += start[c];
        }
        std::vector<std::uint64_t> fill(start.begin(), start.end() - 1);           // :48-51
        for (std::size_t i = 0; i < s.n; ++i) {
            particles[fill[cellOf[i]]++] = i;
        }
    }
    // 27 wrapped cells, (dx, dy, dz) lexicographic from -1 to 1 (src/CellList.cpp:55-83)
    std::array<int, 27> neighbours(int cell) const {
        const int n = ncps;
        const int cx = cell / (n * n), cy = (cell / n) % n, cz = cell % n;
        std::array<int, 27> out {};
        int idx = 0;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz)
                    out[idx++] = (((cx + dx + n) % n) * n + (cy + dy + n) % n) * n + (cz + dz + n) % n;
        return out;
    }
};

struct NList {
    double rl = 0.0, rl2 = 0.0, maxDisp2 = 0.0;
    bool reverse = false;
    Cells cells;
    std::vector<std::uint64_t> offsets, neighbours, revOffsets, revPairs;
    std::vector<double> refPos;  // 3 per particle
    int rebuilds = 0;

    // src/NeighbourList.cpp:5-8
    NList(double rc, double skin, bool rev)
        : rl(rc + skin), rl2((rc + skin) * (rc + skin)), maxDisp2(0.25 * skin * skin), reverse(rev) {
        cells.minSize = rc + skin;
    }

    // src/NeighbourList.cpp:55-134 (serial: pass 1, CSR, concat, reverse index, reference positions)
    void build(Sys& s) {
        if (2.0 * rl > s.L) {
            throw std::runtime_error("Cutoff + skin must be less than half the box length");
        }
        const std::size_t n = s.n;
        cells.build(s);
        std::vector<std::size_t> order(cells.particles.begin(), cells.particles.end());
        s.reorder(order);
        cells.build(s);
        const bool useCells = cells.ncps >= 3;
        offsets.assign(n + 1, 0);
        neighbours.clear();
        for (std::size_t i = 0; i < n; ++i) {
            const std::size_t before = neighbours.size();
            auto visit = [&](std::size_t j) {
                if (j <= i) return;
                double dr[3];
                s.minimumImage(&s.pos[4 * i], &s.pos[4 * j], dr);
                if (dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2] < rl2) neighbours.push_back(j);
            };
            if (useCells) {  // forEachCandidate, src/NeighbourList.cpp:38-52
                for (int c : cells.neighbours(cells.cellOf[i]))
                    for (std::uint64_t k = cells.start[c]; k < cells.start[c + 1]; ++k) visit(cells.particles[k]);
            } else {
                for (std::size_t j = 0; j < n; ++j) visit(j);
            }
            offsets[i + 1] = offsets[i] + (neighbours.size() - before);
        }
        revOffsets.clear();
        revPairs.clear();
        if (reverse) {
            revOffsets.assign(n + 1, 0);
            for (std::uint64_t j : neighbours) ++revOffsets[j + 1];
            for (std::size_t i = 0; i < n; ++i) revOffsets[i + 1] += revOffsets[i];
            revPairs.resize(neighbours.size());
            std::vector<std::uint64_t> fill(revOffsets.begin(), revOffsets.end() - 1);
            for (std::size_t k = 0; k < neighbours.size(); ++k) revPairs[fill[neighbours[k]]++] = k;
        }
        refPos.resize(3 * n);
        for (std::size_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) refPos[3 * i + k] = s.pos[4 * i + k];
        ++rebuilds;
    }

    // src/NeighbourList.cpp:11-36
    bool update(Sys& s) {
        if (refPos.size() != 3 * s.n) {
            build(s);
            return true;
        }
        bool stale = false;
        for (std::size_t i = 0; i < s.n; ++i) {
            double d[3];
            s.minimumImage(&s.pos[4 * i], &refPos[3 * i], d);
            stale = stale || (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] > maxDisp2);
        }
        if (stale) build(s);
        return stale;
    }
};

struct FField {
    double eps, sigma, rc, rc2, shift;
    double virial = 0.0, inside = 0.0;

    // src/Forcefield.cpp:8-15
    FField(double e, double s, double c) : eps(e), sigma(s), rc(c), rc2(c * c) {
        double sr6 = std::pow(sigma / rc, 6);
        double sr12 = sr6 * sr6;
        shift = 4.0 * eps * (sr12 - sr6);
    }
    // src/Forcefield.cpp:18-22
    void check(const Sys& s) const {
        if (2.0 * rc > s.L) throw std::runtime_error("Cutoff must be less than half the box length");
    }
    // src/Forcefield.cpp:25-36
    void pairTerms(double r2, double& fr, double& e) const {
        double inv_r2 = 1.0 / r2;
        double sr2 = sigma * sigma * inv_r2;
        double sr6 = sr2 * sr2 * sr2;
        double sr12 = sr6 * sr6;
        fr = 24.0 * eps * (2.0 * sr12 - sr6) * inv_r2;
        e = 4.0 * eps * (sr12 - sr6) - shift;
    }

    // O(N^2) path, src/Forcefield.cpp:39-78
    double allPairs(Sys& s) {
        check(s);
        for (int k = 0; k < 3; ++k) std::fill(s.force[k].begin(), s.force[k].end(), 0.0);
        double pe = 0.0, w = 0.0, ins = 0.0;
        for (std::size_t i = 0; i < s.n; ++i) {
            for (std::size_t j = i + 1; j < s.n; ++j) {
                double dr[3];
                s.minimumImage(&s.pos[4 * i], &s.pos[4 * j], dr);
                double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
                if (r2 >= rc2) continue;
                double fr, e;
                pairTerms(r2, fr, e);
                for (int k = 0; k < 3; ++k) {
                    s.force[k][i] += fr * dr[k];
                    s.force[k][j] -= fr * dr[k];
                }
                pe += e;
                w += fr * r2;
                ins += 1.0;
            }
        }
        virial = w;
        inside = ins;
        return pe;
    }

    // Deterministic list path, src/Forcefield.cpp:214-326: per-pair slots, then each particle sums its own
    // pairs (+) followed by the pairs where it is second (-), then blocked sums for PE and virial
    double deterministic(Sys& s, const NList& nl) {
        check(s);
        if (!nl.reverse) throw std::runtime_error("Deterministic forces need a NeighbourList built with reverseIndex = true");
        const std::size_t P = nl.neighbours.size();
        std::vector<double> fx(P), fy(P), fz(P), pe(P), pw(P);
        double ins = 0.0;
        for (std::size_t i = 0; i < s.n; ++i) {
            double insI = 0.0;
            for (std::uint64_t k = nl.offsets[i]; k < nl.offsets[i + 1]; ++k) {
                const std::uint64_t j = nl.neighbours[k];
                double dx = s.pos[4 * i] - s.pos[4 * j];
                double dy = s.pos[4 * i + 1] - s.pos[4 * j + 1];
                double dz = s.pos[4 * i + 2] - s.pos[4 * j + 2];
                dx -= s.L * std::round(dx * s.invL);
                dy -= s.L * std::round(dy * s.invL);
                dz -= s.L * std::round(dz * s.invL);
                double r2 = dx * dx + dy * dy + dz * dz;
                double fr, e;
                pairTerms(r2, fr, e);
                const bool in = r2 < rc2;
                fr = in ? fr : 0.0;
                fx[k] = fr * dx;
                fy[k] = fr * dy;
                fz[k] = fr * dz;
                pe[k] = in ? e : 0.0;
                pw[k] = fr * r2;
                insI += in ? 1.0 : 0.0;
            }
            ins += insI;
        }
        for (std::size_t i = 0; i < s.n; ++i) {
            double f[3] = {0.0, 0.0, 0.0};
            for (std::uint64_t k = nl.offsets[i]; k < nl.offsets[i + 1]; ++k) {
                f[0] += fx[k];
                f[1] += fy[k];
                f[2] += fz[k];
            }
            for (std::uint64_t r = nl.revOffsets[i]; r < nl.revOffsets[i + 1]; ++r) {
                const std::uint64_t k = nl.revPairs[r];
                f[0] -= fx[k];
                f[1] -= fy[k];
                f[2] -= fz[k];
            }
            for (int c = 0; c < 3; ++c) s.force[c][i] = f[c];
        }
        virial = blockedSum(P, [&](std::size_t k) { return pw[k]; });
        inside = ins;
        return blockedSum(P, [&](std::size_t k) { return pe[k]; });
    }

    // Default list path run on one thread, src/Forcefield.cpp:81-211 (gather, masked SIMD maths, scatter)
    double listDefault(Sys& s, const NList& nl) {
        check(s);
        std::vector<double> acc(3 * s.n, 0.0);
        double pe = 0.0, w = 0.0, ins = 0.0;
        for (std::size_t i = 0; i < s.n; ++i) {
            double fi[3] = {0, 0, 0}, ei = 0.0, wi = 0.0, ii = 0.0;
            const double* ri = &s.pos[4 * i];
            for (std::uint64_t k = nl.offsets[i]; k < nl.offsets[i + 1]; ++k) {
                const std::uint64_t j = nl.neighbours[k];
                double dx = ri[0] - s.pos[4 * j], dy = ri[1] - s.pos[4 * j + 1], dz = ri[2] - s.pos[4 * j + 2];
                dx -= s.L * std::round(dx * s.invL);
                dy -= s.L * std::round(dy * s.invL);
                dz -= s.L * std::round(dz * s.invL);
                double r2 = dx * dx + dy * dy + dz * dz;
                double fr, e;
                pairTerms(r2, fr, e);
                const bool in = r2 < rc2;
                fr = in ? fr : 0.0;
                ei += in ? e : 0.0;
                wi += fr * r2;
                ii += in ? 1.0 : 0.0;
                fi[0] += fr * dx;
                fi[1] += fr * dy;
                fi[2] += fr * dz;
                acc[3 * j] -= fr * dx;
                acc[3 * j + 1] -= fr * dy;
                acc[3 * j + 2] -= fr * dz;
            }
            for (int c = 0; c < 3; ++c) acc[3 * i + c] += fi[c];
            pe += ei;
            w += wi;
            ins += ii;
        }
        for (std::size_t i = 0; i < s.n; ++i)
            for (int c = 0; c < 3; ++c) s.force[c][i] = 0.0 + acc[3 * i + c];
        virial = w;
        inside = ins;
        return pe;
    }

    // Mixed precision list path on one thread, src/Forcefield.cpp:333-450
    double listMixed(Sys& s, const NList& nl) {
        check(s);
        const float sig2 = static_cast<float>(sigma * sigma), e32 = static_cast<float>(eps);
        const float c2 = static_cast<float>(rc2), sh = static_cast<float>(shift);
        std::vector<double> acc(3 * s.n, 0.0);
        double pe = 0.0, w = 0.0, ins = 0.0;
        for (std::size_t i = 0; i < s.n; ++i) {
            float fx = 0, fy = 0, fz = 0, ei = 0, wi = 0, ii = 0;
            const double* ri = &s.pos[4 * i];
            for (std::uint64_t k = nl.offsets[i]; k < nl.offsets[i + 1]; ++k) {
                const std::uint64_t j = nl.neighbours[k];
                double dx = ri[0] - s.pos[4 * j], dy = ri[1] - s.pos[4 * j + 1], dz = ri[2] - s.pos[4 * j + 2];
                dx -= s.L * std::round(dx * s.invL);
                dy -= s.L * std::round(dy * s.invL);
                dz -= s.L * std::round(dz * s.invL);
                const float x = static_cast<float>(dx), y = static_cast<float>(dy), z = static_cast<float>(dz);
                const float r2 = x * x + y * y + z * z;
                const float inv = 1.0f / r2, sr2 = sig2 * inv, sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
                const bool in = r2 < c2;
                const float fr = in ? 24.0f * e32 * (2.0f * sr12 - sr6) * inv : 0.0f;
                ei += in ? 4.0f * e32 * (sr12 - sr6) - sh : 0.0f;
                wi += fr * r2;
                ii += in ? 1.0f : 0.0f;
                fx += fr * x;
                fy += fr * y;
                fz += fr * z;
                acc[3 * j] -= fr * x;
                acc[3 * j + 1] -= fr * y;
                acc[3 * j + 2] -= fr * z;
            }
            acc[3 * i] += fx;
            acc[3 * i + 1] += fy;
            acc[3 * i + 2] += fz;
            pe += ei;
            w += wi;
            ins += ii;
        }
        for (std::size_t i = 0; i < s.n; ++i)
            for (int c = 0; c < 3; ++c) s.force[c][i] = 0.0 + acc[3 * i + c];
        virial = w;
        inside = ins;
        return pe;
    }
};

// src/Integrator.cpp:32-53
void kickAndDrift(Sys& s, double dt) {
    const double h = 0.5 * dt;
    for (int k = 0; k < 3; ++k) {
        for (std::size_t i = 0; i < s.n; ++i) {
            s.vel[k][i] += h * s.force[k][i] / s.mass[i];
            s.pos[4 * i + k] = s.wrap(s.pos[4 * i + k] + dt * s.vel[k][i]);
        }
    }
}
// src/Integrator.cpp:55-71
void kick(Sys& s, double dt) {
    const double h = 0.5 * dt;
    for (int k = 0; k < 3; ++k)
        for (std::size_t i = 0; i < s.n; ++i) s.vel[k][i] += h * s.force[k][i] / s.mass[i];
}
// src/Thermostat.cpp:6-12
void scaleVelocities(Sys& s, double scale) {
    for (int k = 0; k < 3; ++k)
        for (double& v : s.vel[k]) v *= scale;
}
// src/Thermostat.cpp:17-30
void rescale(Sys& s, double target) {
    double current = s.temperature();
    if (current <= 0.0) return;
    scaleVelocities(s, std::sqrt(target / current));
}

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

}  // namespace

extern "C" {

const char* orc_last_error() { return g_error.c_str(); }

// Lattice constant a = cbrt(4 / density) and box n * a of md_sim's start (src/main.cpp:164-166)
void orc_fcc_box(int cells, double density, double* a, double* box) {
    *a = std::cbrt(4.0 / density);
    *box = cells * *a;
}

// FCC lattice offset by a quarter cell, src/Initialisation.cpp:7-44
void orc_fcc(int cells, double a, double* pos4) {
    static constexpr double basis[4][3] = {{0.0, 0.0, 0.0}, {0.5, 0.5, 0.0}, {0.5, 0.0, 0.5}, {0.0, 0.5, 0.5}};
    std::size_t p = 0;
    for (int ix = 0; ix < cells; ++ix)
        for (int iy = 0; iy < cells; ++iy)
            for (int iz = 0; iz < cells; ++iz)
                for (const auto& b : basis) {
                    pos4[4 * p + 0] = (ix + b[0] + 0.25) * a;
                    pos4[4 * p + 1] = (iy + b[1] + 0.25) * a;
                    pos4[4 * p + 2] = (iz + b[2] + 0.25) * a;
                    pos4[4 * p + 3] = 0.0;
                    ++p;
                }
}

Sys* orc_sys_create(std::int64_t n, double L, const double* pos4, const double* vel, const double* force,
                    const double* mass) {
    auto* s = new Sys;
    s->n = static_cast<std::size_t>(n);
    s->L = L;
    s->invL = 1.0 / L;  // src/System.cpp:9-10
    s->pos.assign(pos4, pos4 + 4 * n);
    for (int k = 0; k < 3; ++k) {
        s->vel[k].assign(n, 0.0);
        s->force[k].assign(n, 0.0);
        if (vel) std::copy(vel + k * n, vel + (k + 1) * n, s->vel[k].begin());
        if (force) std::copy(force + k * n, force + (k + 1) * n, s->force[k].begin());
    }
    s->mass.assign(n, 1.0);
    if (mass) std::copy(mass, mass + n, s->mass.begin());
    s->id.resize(n);
    for (std::int64_t i = 0; i < n; ++i) s->id[i] = static_cast<std::uint64_t>(i);
    return s;
}
void orc_sys_destroy(Sys* s) { delete s; }
void orc_sys_get(const Sys* s, double* pos4, double* vel, double* force, double* mass, std::uint64_t* ids) {
    const std::size_t n = s->n;
    if (pos4) std::copy(s->pos.begin(), s->pos.end(), pos4);
    for (int k = 0; k < 3; ++k) {
        if (vel) std::copy(s->vel[k].begin(), s->vel[k].end(), vel + k * n);
        if (force) std::copy(s->force[k].begin(), s->force[k].end(), force + k * n);
    }
    if (mass) std::copy(s->mass.begin(), s->mass.end(), mass);
    if (ids) std::copy(s->id.begin(), s->id.end(), ids);
}
void orc_sys_set(Sys* s, const double* pos4, const double* vel, const double* force) {
    const std::size_t n = s->n;
    if (pos4) std::copy(pos4, pos4 + 4 * n, s->pos.begin());
    for (int k = 0; k < 3; ++k) {
        if (vel) std::copy(vel + k * n, vel + (k + 1) * n, s->vel[k].begin());
        if (force) std::copy(force + k * n, force + (k + 1) * n, s->force[k].begin());
    }
}
int orc_sys_reorder(Sys* s, const std::uint64_t* order) {
    std::vector<std::size_t> o(order, order + s->n);
    s->reorder(o);
    return 0;
}
double orc_kinetic(const Sys* s) { return s->kinetic(); }
double orc_temperature(const Sys* s) { return s->temperature(); }
std::uint64_t orc_hash(const Sys* s) { return s->hash(); }
void orc_scale(Sys* s, double scale) { scaleVelocities(*s, scale); }
void orc_rescale(Sys* s, double target) { rescale(*s, target); }

// Maxwell-Boltzmann velocities, COM removal and exact rescale, src/Initialisation.cpp:47-76
void orc_init_velocities(Sys* s, double temperature, std::uint32_t seed) {
    std::mt19937 rng(seed);
    double mom[3] = {0, 0, 0}, total = 0.0;
    for (std::size_t i = 0; i < s->n; ++i) {
        std::normal_distribution<double> dist(0.0, std::sqrt(temperature / s->mass[i]));
        for (int k = 0; k < 3; ++k) {
            const double v = dist(rng);
            s->vel[k][i] = v;
            mom[k] += s->mass[i] * v;
        }
        total += s->mass[i];
    }
    for (int k = 0; k < 3; ++k)
        for (double& v : s->vel[k]) v -= mom[k] / total;
    rescale(*s, temperature);
}

// Bussi stochastic velocity rescaling, src/Thermostat.cpp:36-58. The random stream is the caller's:
// r1 and the chi-squared draw are passed in, so the same (r1, chi2) table can drive the CUDA path.
double orc_bussi_factor(double kinetic, std::int64_t n, double temperature, double c, double r1, double chi2) {
    if (kinetic <= 0.0) return 1.0;
    const double dof = 3.0 * static_cast<double>(n) - 3.0;
    const double target = 0.5 * dof * temperature;
    const double nk = kinetic + (1.0 - c) * (target * (chi2 + r1 * r1) / dof - kinetic) +
                      2.0 * r1 * std::sqrt(target / dof * kinetic * (1.0 - c) * c);
    return std::sqrt(nk / kinetic);
}
// The (r1, chi2) pairs that count successive BussiThermostat::apply calls draw from one
// std::mt19937_64(seed): a fresh normal_distribution(0, 1) and gamma_distribution(0.5 (dof - 1), 2) per call
// (src/Thermostat.cpp:48-51)
void orc_bussi_noise(std::uint64_t seed, std::int64_t n, std::int64_t count, double* r1, double* chi2) {
    std::mt19937_64 rng(seed);
    const double dof = 3.0 * static_cast<double>(n) - 3.0;
    for (std::int64_t k = 0; k < count; ++k) {
        std::normal_distribution<double> gaussian(0.0, 1.0);
        std::gamma_distribution<double> gamma(0.5 * (dof - 1.0), 2.0);
        r1[k] = gaussian(rng);
        chi2[k] = gamma(rng);
    }
}

void orc_bussi_apply(Sys* s, double temperature, double c, double r1, double chi2) {
    const double k = s->kinetic();
    if (k <= 0.0) return;
    scaleVelocities(*s, orc_bussi_factor(k, static_cast<std::int64_t>(s->n), temperature, c, r1, chi2));
}

// CellList (src/CellList.cpp:9-52). cell_start must hold ncps^3 + 1 entries: query ncps first.
int orc_cells_per_side(double L, double min_cell) { return std::max(1, static_cast<int>(L / min_cell)); }
int orc_cells_build(const Sys* s, double min_cell, int* particle_cell, std::uint64_t* cell_start,
                    std::uint64_t* cell_particles) {
    Cells c;
    c.minSize = min_cell;
    c.build(*s);
    std::copy(c.cellOf.begin(), c.cellOf.end(), particle_cell);
    std::copy(c.start.begin(), c.start.end(), cell_start);
    std::copy(c.particles.begin(), c.particles.end(), cell_particles);
    return c.ncps;
}
void orc_neighbour_cells(int ncps, int cell, int* out27) {
    Cells c;
    c.ncps = ncps;
    auto nb = c.neighbours(cell);
    std::copy(nb.begin(), nb.end(), out27);
}

NList* orc_nl_create(double rc, double skin, int reverse) { return new NList(rc, skin, reverse != 0); }
void orc_nl_destroy(NList* nl) { delete nl; }
int orc_nl_build(NList* nl, Sys* s) { return guarded([&] { nl->build(*s); }); }
int orc_nl_update(NList* nl, Sys* s, int* rebuilt) {
    return guarded([&] { *rebuilt = nl->update(*s) ? 1 : 0; });
}
std::uint64_t orc_nl_pairs(const NList* nl) { return nl->neighbours.size(); }
int orc_nl_rebuilds(const NList* nl) { return nl->rebuilds; }
int orc_nl_cells_per_side(const NList* nl) { return nl->cells.ncps; }
void orc_nl_get(const NList* nl, std::uint64_t* offsets, std::uint64_t* neighbours, std::uint64_t* rev_offsets,
                std::uint64_t* rev_pairs, int* particle_cell, std::uint64_t* cell_start) {
    if (offsets) std::copy(nl->offsets.begin(), nl->offsets.end(), offsets);
    if (neighbours) std::copy(nl->neighbours.begin(), nl->neighbours.end(), neighbours);
    if (rev_offsets) std::copy(nl->revOffsets.begin(), nl->revOffsets.end(), rev_offsets);
    if (rev_pairs) std::copy(nl->revPairs.begin(), nl->revPairs.end(), rev_pairs);
    if (particle_cell) std::copy(nl->cells.cellOf.begin(), nl->cells.cellOf.end(), particle_cell);
    if (cell_start) std::copy(nl->cells.start.begin(), nl->cells.start.end(), cell_start);
}

FField* orc_ff_create(double eps, double sigma, double rc) { return new FField(eps, sigma, rc); }
void orc_ff_destroy(FField* f) { delete f; }
double orc_ff_shift(const FField* f) { return f->shift; }
double orc_ff_virial(const FField* f) { return f->virial; }
double orc_ff_inside(const FField* f) { return f->inside; }
// mode 0 = default (one thread), 1 = deterministic, 2 = mixed precision (one thread), 3 = all pairs
int orc_ff_forces(FField* f, Sys* s, const NList* nl, int mode, double* pe) {
    return guarded([&] {
        switch (mode) {
            case 0: *pe = f->listDefault(*s, *nl); break;
            case 1: *pe = f->deterministic(*s, *nl); break;
            case 2: *pe = f->listMixed(*s, *nl); break;
            default: *pe = f->allPairs(*s); break;
        }
    });
}

// VelocityVerletIntegrator::step, src/Integrator.cpp:7-30. mode as orc_ff_forces; with mode 3 the list
// is not used (all-pairs step overload)
int orc_step(Sys* s, FField* f, NList* nl, double dt, int mode, double* pe) {
    return guarded([&] {
        kickAndDrift(*s, dt);
        if (mode != 3) nl->update(*s);
        switch (mode) {
            case 0: *pe = f->listDefault(*s, *nl); break;
            case 1: *pe = f->deterministic(*s, *nl); break;
            case 2: *pe = f->listMixed(*s, *nl); break;
            default: *pe = f->allPairs(*s); break;
        }
        kick(*s, dt);
    });
}

// RadialDistribution::sample over the half list, src/RadialDistribution.cpp:11-30. hist counts
// are accumulated in place (the reference keeps them as doubles; they are whole numbers).
void orc_rdf_sample(const Sys* s, const NList* nl, double rmax, int bins, double* hist) {
    const double bw = rmax / bins;
    const double rmax2 = rmax * rmax;
    for (std::size_t i = 0; i < s->n; ++i) {
        for (std::uint64_t k = nl->offsets[i]; k < nl->offsets[i + 1]; ++k) {
            double dr[3];
            s->minimumImage(&s->pos[4 * i], &s->pos[4 * nl->neighbours[k]], dr);
            double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
            if (r2 < rmax2) hist[static_cast<std::size_t>(std::sqrt(r2) / bw)] += 1.0;
        }
    }
}
// RadialDistribution::values, src/RadialDistribution.cpp:42-54
void orc_rdf_values(const double* hist, int bins, double rmax, int samples, double particles, double L, double* g) {
    const double bw = rmax / bins;
    const double density = particles / std::pow(L, 3);
    for (int b = 0; b < bins; ++b) {
        if (samples == 0) {
            g[b] = 0.0;
            continue;
        }
        const double lo = static_cast<double>(b) * bw;
        const double hi = lo + bw;
        const double shell = 4.0 / 3.0 * std::numbers::pi * (hi * hi * hi - lo * lo * lo);
        g[b] = hist[b] / (samples * 0.5 * particles * density * shell);
    }
}

}  // extern "C"
