// The reference's unit, integration and dynamics tests (tests/*.cpp of nhantran1711/molecular-dynamics),
// restated against the drop-in C++ classes of molecular-dynamics_b200/dropin, which run on the GPU.
// GoogleTest is not available offline, so a minimal harness stands in: every TEST runs, failures print
// file:line and the process exits non-zero. tests/test_gpu_dropin.py builds and runs this program.
#include "CellList.hpp"
#include "Forcefield.hpp"
#include "Initialisation.hpp"
#include "Integrator.hpp"
#include "NeighbourList.hpp"
#include "RadialDistribution.hpp"
#include "System.hpp"
#include "Thermostat.hpp"
#include "Trajectory.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <limits>
#include <memory>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

// ---- harness --------------------------------------------------------------------------------------------

namespace harness {
struct Case {
    const char* name;
    std::function<void()> body;
};
std::vector<Case>& cases() {
    static std::vector<Case> c;
    return c;
}
int failures = 0;
struct Register {
    Register(const char* n, std::function<void()> b) { cases().push_back({n, std::move(b)}); }
};
void fail(const char* file, int line, const std::string& what) {
    ++failures;
    std::printf("FAIL %s:%d %s\n", file, line, what.c_str());
}
}  // namespace harness

#define TEST(suite, name)                                                              \
    static void suite##_##name();                                                      \
    static harness::Register reg_##suite##_##name(#suite "." #name, suite##_##name);   \
    static void suite##_##name()
#define CHECK(cond) \
    do { if (!(cond)) harness::fail(__FILE__, __LINE__, #cond); } while (0)
#define CHECK_NEAR(a, b, tol)                                                                             \
    do {                                                                                                  \
        const double a_ = (a), b_ = (b);                                                                  \
        if (!(std::abs(a_ - b_) <= (tol)))                                                                \
            harness::fail(__FILE__, __LINE__, std::string(#a " vs " #b ": ") + std::to_string(a_) + " " + \
                                                  std::to_string(b_));                                    \
    } while (0)
#define CHECK_THROWS(stmt)                                \
    do {                                                  \
        bool thrown_ = false;                             \
        try {                                             \
            stmt;                                         \
        } catch (const std::runtime_error&) {             \
            thrown_ = true;                               \
        }                                                 \
        if (!thrown_) harness::fail(__FILE__, __LINE__, "no throw: " #stmt); \
    } while (0)

// ---- helpers (the reference's tests/TestHelpers.hpp state point) ------------------------------------------

namespace fixture {
constexpr double density = 0.8442, temperature = 0.728, cutOff = 2.5, skin = 0.2, dt = 0.005;
double latticeConstant() { return std::cbrt(4.0 / density); }
System makeLattice(int cells, unsigned seed = 42) {
    System s(createFCCLattice(cells, latticeConstant()), cells * latticeConstant());
    initializeVelocities(s, temperature, seed);
    return s;
}
System makeLiquid(int cells, int steps = 300) {
    System s = makeLattice(cells);
    LennardJonesForceField ff(1.0, 1.0, cutOff);
    VelocityVerletIntegrator integ(dt);
    NeighbourList list(cutOff, skin);
    list.build(s);
    ff.computeForces(s, list);
    for (int k = 1; k <= steps; ++k) {
        integ.step(s, ff, list);
        if (k % 10 == 0) rescaleVelocities(s, temperature);
    }
    return s;
}
std::array<double, 3> momentum(const System& s) {
    std::array<double, 3> p {0, 0, 0};
    for (int k = 0; k < 3; ++k)
        for (std::size_t i = 0; i < s.size(); ++i) p[k] += s.mass()[i] * s.velocity(k)[i];
    return p;
}
double ljForce(double r) { return 24.0 * (2.0 * std::pow(r, -13) - std::pow(r, -7)); }
double ljEnergy(double r, double rc) {
    auto v = [](double x) { return 4.0 * (std::pow(x, -12) - std::pow(x, -6)); };
    return v(r) - v(rc);
}
System pairAt(double x0, double x1, double box) {
    Particle a, b;
    a.position = {x0, 5.0, 5.0};
    b.position = {x1, 5.0, 5.0};
    return System({a, b}, box);
}
using PairSet = std::set<std::pair<std::size_t, std::size_t>>;
PairSet pairsInList(const NeighbourList& l, std::size_t n) {
    PairSet p;
    for (std::size_t i = 0; i < n; ++i)
        for (std::size_t j : l.neighboursOf(i)) {
            CHECK(j > i);
            p.insert({i, j});
        }
    return p;
}
PairSet pairsWithin(const System& s, double radius) {
    PairSet p;
    for (std::size_t i = 0; i < s.size(); ++i)
        for (std::size_t j = i + 1; j < s.size(); ++j) {
            auto d = s.minimumImageDistance(i, j);
            if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < radius * radius) p.insert({i, j});
        }
    return p;
}
}  // namespace fixture
using namespace fixture;

// ---- tests/test_system.cpp ------------------------------------------------------------------------------

TEST(System, MinimumImageAndWrap) {
    System s({}, 10.0);
    auto dr = s.minimumImageDistance({0.5, 0.5, 0.5}, {9.5, 9.5, 9.5});
    for (double d : dr) CHECK_NEAR(d, 1.0, 1e-12);
    std::array<double, 3> r {-0.5, 10.0, 23.0};
    s.wrapPosition(r);
    CHECK_NEAR(r[0], 9.5, 1e-12);
    CHECK_NEAR(r[1], 0.0, 1e-12);
    CHECK_NEAR(r[2], 3.0, 1e-12);
}

TEST(System, KineticEnergyTemperatureReorder) {
    Particle a, b;
    a.velocity = {1.0, 0.0, 0.0};
    b.velocity = {-1.0, 0.0, 0.0};
    b.mass = 2.0;
    System s({a, b}, 10.0);
    CHECK(s.kineticEnergy() == 1.5);
    CHECK(s.temperature() == 2.0 * 1.5 / 3.0);
    std::vector<Particle> ps(4);
    for (int i = 0; i < 4; ++i) ps[i].position = {static_cast<double>(i), 0.0, 0.0};
    System t(ps, 10.0);
    const std::vector<std::size_t> order {2, 0, 3, 1};
    t.reorder(order);
    for (std::size_t k = 0; k < order.size(); ++k) CHECK(t.positionOf(k)[0] == static_cast<double>(order[k]));
}

// ---- tests/test_forcefield.cpp ---------------------------------------------------------------------------

TEST(ForceField, TwoParticlesAnalytic) {
    LennardJonesForceField ff(1.0, 1.0, cutOff);
    for (double r : {0.95, 1.12, 1.5, 2.0, 2.45}) {
        System s = pairAt(5.0, 5.0 + r, 20.0);
        const double e = ff.computeForces(s);
        CHECK_NEAR(s.forceOf(0)[0], -ljForce(r), 1e-10);
        CHECK_NEAR(s.forceOf(1)[0], ljForce(r), 1e-10);
        CHECK_NEAR(s.forceOf(0)[1], 0.0, 1e-12);
        CHECK_NEAR(e, ljEnergy(r, cutOff), 1e-12);
    }
    System m = pairAt(5.0, 5.0 + std::pow(2.0, 1.0 / 6.0), 20.0);
    ff.computeForces(m);
    CHECK_NEAR(m.forceOf(0)[0], 0.0, 1e-12);
    System far = pairAt(5.0, 5.0 + cutOff + 1e-9, 20.0);
    CHECK(ff.computeForces(far) == 0.0 && far.forceOf(0)[0] == 0.0);
    System pbc = pairAt(0.5, 19.5, 20.0);
    const double e = ff.computeForces(pbc);
    CHECK_NEAR(pbc.forceOf(0)[0], ljForce(1.0), 1e-10);
    CHECK_NEAR(e, ljEnergy(1.0, cutOff), 1e-12);
    System small = pairAt(1.0, 2.0, 4.0);
    CHECK_THROWS(ff.computeForces(small));
}

TEST(ForceField, ListMatchesAllPairsAndSumsToZero) {
    System s = makeLiquid(8);
    LennardJonesForceField ff(1.0, 1.0, cutOff);
    NeighbourList list(cutOff, skin);
    list.build(s);
    const double le = ff.computeForces(s, list);
    std::vector<std::array<double, 3>> lf;
    for (std::size_t i = 0; i < s.size(); ++i) lf.push_back(s.forceOf(i));
    std::array<double, 3> total {0, 0, 0};
    for (int k = 0; k < 3; ++k)
        for (double f : s.force(k)) total[k] += f;
    for (double f : total) CHECK_NEAR(f, 0.0, 1e-10);
    const double re = ff.computeForces(s);
    CHECK_NEAR(le, re, 1e-9 * std::abs(re));
    double md = 0.0;
    for (std::size_t i = 0; i < lf.size(); ++i)
        for (int k = 0; k < 3; ++k) md = std::max(md, std::abs(lf[i][k] - s.forceOf(i)[k]));
    CHECK(md < 1e-11);
}

TEST(ForceField, MixedPrecisionMatchesDoubleAndConservesEnergy) {
    System s = makeLiquid(8);
    LennardJonesForceField ff(1.0, 1.0, cutOff);
    NeighbourList list(cutOff, skin);
    list.build(s);
    const double e = ff.computeForces(s, list);
    std::vector<std::array<double, 3>> ref;
    for (std::size_t i = 0; i < s.size(); ++i) ref.push_back(s.forceOf(i));
    ff.setMixedPrecision(true);
    const double me = ff.computeForces(s, list);
    CHECK_NEAR(me, e, 1e-5 * std::abs(e));
    double md = 0.0, mf = 0.0;
    for (std::size_t i = 0; i < ref.size(); ++i)
        for (int k = 0; k < 3; ++k) {
            md = std::max(md, std::abs(s.forceOf(i)[k] - ref[i][k]));
            mf = std::max(mf, std::abs(ref[i][k]));
        }
    CHECK(md < 1e-5 * mf);

    System l = makeLiquid(5, 500);
    LennardJonesForceField fm(1.0, 1.0, cutOff);
    fm.setMixedPrecision(true);
    VelocityVerletIntegrator integ(dt);
    NeighbourList nl(cutOff, skin);
    nl.build(l);
    double pe = fm.computeForces(l, nl);
    const double e0 = l.kineticEnergy() + pe;
    double drift = 0.0;
    for (int k = 0; k < 2000; ++k) {
        pe = integ.step(l, fm, nl);
        drift = std::max(drift, std::abs((l.kineticEnergy() + pe - e0) / e0));
    }
    CHECK(drift < 3e-4);
}

// Precision::FixedDouble (exact fixed-point separations, double pair terms): every particle's force within 1e-6
// of the rms force of the double path, the energy within 1e-9
TEST(ForceField, FixedDoublePrecisionMatchesDouble) {
    System s = makeLiquid(8);
    LennardJonesForceField ff(1.0, 1.0, cutOff);
    NeighbourList list(cutOff, skin);
    list.build(s);
    const double e = ff.computeForces(s, list);
    std::vector<std::array<double, 3>> ref;
    double rms = 0.0;
    for (std::size_t i = 0; i < s.size(); ++i) {
        ref.push_back(s.forceOf(i));
        for (double f : ref.back()) rms += f * f;
    }
    rms = std::sqrt(rms / static_cast<double>(s.size()));
    ff.setPrecision(LennardJonesForceField::Precision::FixedDouble);
    const double fe = ff.computeForces(s, list);
    CHECK_NEAR(fe, e, 1e-9 * std::abs(e));
    double worst = 0.0;
    for (std::size_t i = 0; i < ref.size(); ++i) {
        double d2 = 0.0;
        for (int k = 0; k < 3; ++k) d2 += (s.forceOf(i)[k] - ref[i][k]) * (s.forceOf(i)[k] - ref[i][k]);
        worst = std::max(worst, std::sqrt(d2));
    }
    CHECK(worst < 1e-6 * rms);
}

// ---- tests/test_neighbourlist.cpp --------------------------------------------------------------------------

TEST(NeighbourList, ContentsFallbackRebuildAndErrors) {
    System s = makeLiquid(8);
    NeighbourList list(cutOff, skin);
    list.build(s);
    const auto expected = pairsWithin(s, cutOff + skin);
    CHECK(pairsInList(list, s.size()) == expected);
    CHECK(list.getPairCount() == expected.size());

    System small = makeLiquid(4);
    NeighbourList sl(cutOff, skin);
    sl.build(small);
    CHECK(pairsInList(sl, small.size()) == pairsWithin(small, cutOff + skin));

    System m = makeLiquid(6);
    NeighbourList ml(cutOff, skin);
    ml.build(m);
    const int builds = ml.getRebuildCount();
    auto r = m.positionOf(0);
    r[0] += 0.4 * skin;
    m.wrapPosition(r);
    m.setPosition(0, r);
    CHECK(!ml.update(m));
    CHECK(ml.getRebuildCount() == builds);
    r[0] += 0.2 * skin;
    m.wrapPosition(r);
    m.setPosition(0, r);
    CHECK(ml.update(m));
    CHECK(ml.getRebuildCount() == builds + 1);

    System tiny = makeLattice(3);
    NeighbourList tl(cutOff, skin);
    CHECK_THROWS(tl.build(tiny));
}

TEST(CellList, MembershipAndNeighbourCells) {
    System s = makeLiquid(8);
    CellList cells(cutOff + skin);
    cells.build(s);
    const int n = cells.getCellsPerSide();
    CHECK(n >= 3);
    const double cs = s.getBoxLength() / n;
    std::vector<int> seen(s.size(), 0);
    for (int c = 0; c < n * n * n; ++c)
        for (std::size_t i : cells.particlesIn(c)) {
            ++seen[i];
            CHECK(cells.cellOf(i) == c);
            const auto r = s.positionOf(i);
            int want = 0;
            for (int k = 0; k < 3; ++k) want = want * n + std::min(static_cast<int>(r[k] / cs), n - 1);
            CHECK(want == c);
        }
    for (int c : seen) CHECK(c == 1);
    for (int c : {0, n * n * n - 1, n * n + n + 1}) {
        auto nb = cells.neighbourCells(c);
        std::set<int> u(nb.begin(), nb.end());
        CHECK(u.size() == 27u && u.count(c));
    }
}

// ---- tests/test_dynamics.cpp -------------------------------------------------------------------------------

TEST(Dynamics, LatticeVelocitiesRescale) {
    auto ps = createFCCLattice(3, 1.5);
    CHECK(ps.size() == 108u);
    System s(ps, 4.5);
    double md = std::numeric_limits<double>::max();
    for (std::size_t i = 0; i < ps.size(); ++i)
        for (std::size_t j = i + 1; j < ps.size(); ++j) {
            auto d = s.minimumImageDistance(ps[i].position, ps[j].position);
            md = std::min(md, std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
        }
    CHECK_NEAR(md, 1.5 / std::sqrt(2.0), 1e-12);
    System l = makeLattice(5);
    CHECK_NEAR(l.temperature(), temperature, 1e-12);
    for (double p : momentum(l)) CHECK_NEAR(p, 0.0, 1e-12);
    System t = makeLattice(4);
    rescaleVelocities(t, 1.7);
    CHECK_NEAR(t.temperature(), 1.7, 1e-12);
}

TEST(Dynamics, EnergyMomentumReversibility) {
    System s = makeLiquid(5, 500);
    LennardJonesForceField ff(1.0, 1.0, cutOff);
    VelocityVerletIntegrator integ(dt);
    NeighbourList list(cutOff, skin);
    list.build(s);
    double pe = ff.computeForces(s, list);
    const double e0 = s.kineticEnergy() + pe;
    double drift = 0.0;
    for (int k = 0; k < 2000; ++k) {
        pe = integ.step(s, ff, list);
        drift = std::max(drift, std::abs((s.kineticEnergy() + pe - e0) / e0));
    }
    CHECK(drift < 3e-4);
    CHECK(list.getRebuildCount() > 1);

    System m = makeLiquid(5, 0);
    NeighbourList ml(cutOff, skin);
    ml.build(m);
    ff.computeForces(m, ml);
    for (int k = 0; k < 1000; ++k) integ.step(m, ff, ml);
    for (double p : momentum(m)) CHECK_NEAR(p, 0.0, 1e-10);

    System r = makeLiquid(4, 200);
    ff.computeForces(r);
    std::vector<std::array<double, 3>> start;
    for (std::size_t i = 0; i < r.size(); ++i) start.push_back(r.positionOf(i));
    for (int k = 0; k < 100; ++k) integ.step(r, ff);
    for (int k = 0; k < 3; ++k)
        for (double& v : r.velocity(k)) v = -v;
    for (int k = 0; k < 100; ++k) integ.step(r, ff);
    double err = 0.0;
    for (std::size_t i = 0; i < r.size(); ++i) {
        auto d = r.minimumImageDistance(r.positionOf(i), start[i]);
        err = std::max({err, std::abs(d[0]), std::abs(d[1]), std::abs(d[2])});
    }
    CHECK(err < 1e-8);
}

// ---- tests/test_determinism.cpp ----------------------------------------------------------------------------

TEST(Determinism, ReverseIndexAndDeterministicForces) {
    System s = makeLiquid(8);
    LennardJonesForceField ff(1.0, 1.0, cutOff);
    NeighbourList list(cutOff, skin, true);
    list.build(s);
    ff.setDeterministic(true);
    const double e = ff.computeForces(s, list);
    std::vector<std::array<double, 3>> f;
    for (std::size_t i = 0; i < s.size(); ++i) f.push_back(s.forceOf(i));
    const double re = ff.computeForces(s);
    CHECK_NEAR(e, re, 1e-9 * std::abs(re));
    double md = 0.0;
    for (std::size_t i = 0; i < f.size(); ++i)
        for (int k = 0; k < 3; ++k) md = std::max(md, std::abs(f[i][k] - s.forceOf(i)[k]));
    CHECK(md < 1e-11);
    std::vector<int> seen(list.getPairCount(), 0);
    for (std::size_t j = 0; j < s.size(); ++j) {
        std::size_t prev = 0;
        bool first = true;
        for (std::size_t k : list.pairsAsSecond(j)) {
            ++seen[k];
            CHECK(first || k > prev);
            prev = k;
            first = false;
        }
    }
    for (int c : seen) CHECK(c == 1);
    System t = makeLattice(6);
    NeighbourList plain(cutOff, skin);
    plain.build(t);
    CHECK_THROWS(ff.computeForces(t, plain));
}

// md_sim 8 --deterministic --skin 0.3 --temperature 0.71 --equil 0 --steps N through the drop-in classes:
// the reference (compiled with -ffp-contract=off) prints state_hash 30089c6b979800c7 after one step and
// 9eb85613108f2388 after 1000
TEST(Determinism, MdSimConfig1Hashes) {
    const double a = std::cbrt(4.0 / 0.8442);
    System s(createFCCLattice(8, a), 8 * a);
    initializeVelocities(s, 0.71, 42);
    LennardJonesForceField ff(1.0, 1.0, 2.5);
    VelocityVerletIntegrator integ(0.005);
    NeighbourList list(2.5, 0.3, true);
    ff.setDeterministic(true);
    ff.computeForces(s);
    list.build(s);
    integ.step(s, ff, list);
    CHECK(s.stateHash() == 0x30089c6b979800c7ull);
    for (int k = 2; k <= 1000; ++k) integ.step(s, ff, list);
    CHECK(s.stateHash() == 0x9eb85613108f2388ull);
    CHECK(list.getRebuildCount() == 85);  // md_sim reports 85, the initial build included
}

// ---- tests/test_observables.cpp ------------------------------------------------------------------------------

TEST(Observables, VirialInsideBussiIdealGas) {
    LennardJonesForceField ff(1.0, 1.0, cutOff);
    System p = pairAt(5.0, 6.3, 20.0);
    ff.computeForces(p);
    CHECK_NEAR(ff.getVirial(), 1.3 * ljForce(1.3), 1e-12);
    CHECK(ff.getInsidePairs() == 1.0);

    System s = makeLiquid(8);
    NeighbourList list(cutOff, skin, true);
    list.build(s);
    ff.computeForces(s);
    const double w = ff.getVirial(), ins = ff.getInsidePairs();
    for (bool det : {false, true}) {
        ff.setDeterministic(det);
        ff.computeForces(s, list);
        CHECK_NEAR(ff.getVirial(), w, 1e-9 * std::abs(w));
        CHECK(ff.getInsidePairs() == ins);
    }

    System b = makeLattice(5);
    const double target = 0.85, dof = 3.0 * static_cast<double>(b.size()) - 3.0;
    BussiThermostat th(target, 0.05, 7);
    double sk = 0.0, sk2 = 0.0;
    int m = 0;
    for (int k = 0; k < 100000; ++k) {
        th.apply(b, 0.005);
        if (k >= 1000) {
            const double ke = b.kineticEnergy();
            sk += ke;
            sk2 += ke * ke;
            ++m;
        }
    }
    const double mk = sk / m, vk = sk2 / m - mk * mk;
    CHECK_NEAR(mk / (0.5 * dof), target, 0.005 * target);
    CHECK_NEAR(vk / (0.5 * dof * target * target), 1.0, 0.05);

    std::mt19937 rng(3);
    std::uniform_real_distribution<double> u(0.0, 12.0);
    RadialDistribution rdf(cutOff, 25);
    for (int k = 0; k < 40; ++k) {
        std::vector<Particle> ps(2000);
        for (auto& q : ps) q.position = {u(rng), u(rng), u(rng)};
        System g(ps, 12.0);
        NeighbourList gl(cutOff, skin);
        gl.build(g);
        rdf.sample(g, gl);
    }
    const auto r = rdf.radii();
    const auto gv = rdf.values();
    for (std::size_t k = 0; k < gv.size(); ++k)
        if (r[k] > 1.0) CHECK_NEAR(gv[k], 1.0, 0.06);
}

// ---- tests/test_trajectory.cpp --------------------------------------------------------------------------------

TEST(Trajectory, IdsAndFrames) {
    System s = makeLiquid(6, 0);
    std::vector<std::array<double, 3>> byId(s.size());
    for (std::size_t i = 0; i < s.size(); ++i) byId[s.ids()[i]] = s.positionOf(i);
    NeighbourList list(cutOff, skin);
    list.build(s);
    std::vector<std::size_t> ids(s.ids().begin(), s.ids().end());
    CHECK(!std::is_sorted(ids.begin(), ids.end()));
    for (std::size_t i = 0; i < s.size(); ++i) CHECK(s.positionOf(i) == byId[s.ids()[i]]);

    System t = makeLiquid(6);
    LennardJonesForceField ff(1.0, 1.0, cutOff);
    VelocityVerletIntegrator integ(dt);
    NeighbourList tl(cutOff, skin);
    tl.build(t);
    ff.computeForces(t, tl);
    std::unique_ptr<std::FILE, int (*)(std::FILE*)> owner(std::tmpfile(), &std::fclose);
    std::FILE* f = owner.get();
    writeXyzFrame(f, t, 0.0);
    integ.step(t, ff, tl);
    tl.build(t);
    writeXyzFrame(f, t, dt);
    std::fseek(f, 0, SEEK_SET);
    auto read = [&](std::vector<std::array<double, 3>>& pos) {
        char line[512];
        CHECK(std::fgets(line, sizeof line, f) != nullptr);
        const std::size_t n = std::stoul(line);
        CHECK(std::fgets(line, sizeof line, f) != nullptr);
        for (std::size_t k = 0; k < n; ++k) {
            CHECK(std::fgets(line, sizeof line, f) != nullptr);
            std::istringstream in(line);
            std::string sp;
            std::array<double, 3> r {}, v {};
            std::size_t id = 0;
            in >> sp >> r[0] >> r[1] >> r[2] >> v[0] >> v[1] >> v[2] >> id;
            CHECK(id == k);
            pos.push_back(r);
        }
    };
    std::vector<std::array<double, 3>> a, b;
    read(a);
    read(b);
    CHECK(a.size() == t.size() && b.size() == t.size());
    double mv = 0.0;
    for (std::size_t k = 0; k < a.size(); ++k) {
        auto d = t.minimumImageDistance(a[k], b[k]);
        mv = std::max(mv, std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
    }
    CHECK(mv < 0.1);
}

int main(int argc, char** argv) {
    const char* only = argc > 1 ? argv[1] : nullptr;
    for (auto& c : harness::cases()) {
        if (only && std::string(c.name).find(only) == std::string::npos) continue;
        const int before = harness::failures;
        try {
            c.body();
        } catch (const std::exception& e) {
            harness::fail(__FILE__, __LINE__, std::string(c.name) + " threw: " + e.what());
        }
        std::printf("%s %s\n", harness::failures == before ? "ok  " : "FAIL", c.name);
        std::fflush(stdout);
    }
    std::printf("%d failure(s)\n", harness::failures);
    return harness::failures == 0 ? 0 : 1;
}
