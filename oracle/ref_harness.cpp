// ORACLE HARNESS — test infrastructure only. A thin extern "C" shim over the reference's own classes
// (System, CellList, NeighbourList, LennardJonesForceField, VelocityVerletIntegrator, BussiThermostat,
// RadialDistribution, createFCCLattice, initializeVelocities), compiled together with the reference's
// unmodified sources by oracle/Makefile into oracle/_ref/libmdref.so. It lets tests/golden/make_golden.py
// record golden vectors from the reference itself and lets bench.py time the reference's OpenMP path.
// Nothing in the product links or loads it.
#include "CellList.hpp"
#include "Forcefield.hpp"
#include "Initialisation.hpp"
#include "Integrator.hpp"
#include "NeighbourList.hpp"
#include "RadialDistribution.hpp"
#include "System.hpp"
#include "Thermostat.hpp"

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
std::string g_error;

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

const char* ref_last_error() { return g_error.c_str(); }

void ref_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int ref_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// FCC lattice + seeded Maxwell-Boltzmann velocities, as md_sim and tests/TestHelpers.hpp set them up
System* ref_sys_create_fcc(int cells, double density, double temperature, unsigned seed) {
    const double a = std::cbrt(4.0 / density);
    auto* s = new System(createFCCLattice(cells, a), cells * a);
    initializeVelocities(*s, temperature, seed);
    return s;
}
System* ref_sys_create(std::int64_t n, double L, const double* pos4, const double* vel, const double* mass) {
    std::vector<Particle> p(static_cast<std::size_t>(n));
    for (std::int64_t i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) {
            p[i].position[k] = pos4[4 * i + k];
            if (vel) p[i].velocity[k] = vel[k * n + i];
        }
        if (mass) p[i].mass = mass[i];
    }
    return new System(p, L);
}
System* ref_sys_clone(const System* s) { return new System(*s); }
void ref_sys_destroy(System* s) { delete s; }
std::int64_t ref_sys_size(const System* s) { return static_cast<std::int64_t>(s->size()); }
double ref_sys_box(const System* s) { return s->getBoxLength(); }
void ref_sys_get(const System* s, double* pos4, double* vel, double* force, double* mass, std::uint64_t* ids) {
    const std::size_t n = s->size();
    if (pos4) std::memcpy(pos4, s->packedPositions(), sizeof(double) * 4 * n);
    for (int k = 0; k < 3; ++k) {
        if (vel) std::memcpy(vel + k * n, s->velocity(k).data(), sizeof(double) * n);
        if (force) std::memcpy(force + k * n, s->force(k).data(), sizeof(double) * n);
    }
    if (mass) std::memcpy(mass, s->mass().data(), sizeof(double) * n);
    if (ids)
        for (std::size_t i = 0; i < n; ++i) ids[i] = s->ids()[i];
}
void ref_sys_set_velocity(System* s, const double* vel) {
    const std::size_t n = s->size();
    for (int k = 0; k < 3; ++k) std::memcpy(s->velocity(k).data(), vel + k * n, sizeof(double) * n);
}
double ref_kinetic(const System* s) { return s->kineticEnergy(); }
double ref_temperature(const System* s) { return s->temperature(); }
std::uint64_t ref_hash(const System* s) { return s->stateHash(); }
void ref_rescale(System* s, double t) { rescaleVelocities(*s, t); }

int ref_cells_build(const System* s, double min_cell, int* particle_cell, std::uint64_t* cell_start,
                    std::uint64_t* cell_particles) {
    CellList c(min_cell);
    c.build(*s);
    const int n = c.getCellsPerSide();
    for (std::size_t i = 0; i < s->size(); ++i) particle_cell[i] = c.cellOf(i);
    std::uint64_t acc = 0;
    for (int cell = 0; cell < n * n * n; ++cell) {
        cell_start[cell] = acc;
        for (std::size_t p : c.particlesIn(cell)) cell_particles[acc++] = p;
    }
    cell_start[n * n * n] = acc;
    return n;
}

NeighbourList* ref_nl_create(double rc, double skin, int reverse) { return new NeighbourList(rc, skin, reverse != 0); }
void ref_nl_destroy(NeighbourList* nl) { delete nl; }
int ref_nl_build(NeighbourList* nl, System* s) { return guarded([&] { nl->build(*s); }); }
int ref_nl_update(NeighbourList* nl, System* s, int* rebuilt) {
    return guarded([&] { *rebuilt = nl->update(*s) ? 1 : 0; });
}
std::uint64_t ref_nl_pairs(const NeighbourList* nl) { return nl->getPairCount(); }
int ref_nl_rebuilds(const NeighbourList* nl) { return nl->getRebuildCount(); }
void ref_nl_get(const NeighbourList* nl, std::int64_t n, std::uint64_t* offsets, std::uint64_t* neighbours,
                std::uint64_t* rev_offsets, std::uint64_t* rev_pairs) {
    std::uint64_t k = 0, r = 0;
    for (std::int64_t i = 0; i < n; ++i) {
        if (offsets) offsets[i] = nl->firstPairOf(i);
        for (std::size_t j : nl->neighboursOf(i)) {
            if (neighbours) neighbours[k] = j;
            ++k;
        }
        if (nl->hasReverseIndex()) {
            if (rev_offsets) rev_offsets[i] = r;
            for (std::size_t p : nl->pairsAsSecond(i)) {
                if (rev_pairs) rev_pairs[r] = p;
                ++r;
            }
        }
    }
    if (offsets) offsets[n] = k;
    if (nl->hasReverseIndex() && rev_offsets) rev_offsets[n] = r;
}

LennardJonesForceField* ref_ff_create(double eps, double sigma, double rc) {
    return new LennardJonesForceField(eps, sigma, rc);
}
void ref_ff_destroy(LennardJonesForceField* f) { delete f; }
void ref_ff_set(LennardJonesForceField* f, int deterministic, int mixed) {
    f->setDeterministic(deterministic != 0);
    f->setMixedPrecision(mixed != 0);
}
double ref_ff_shift(const LennardJonesForceField* f) { return f->getEnergyShift(); }
double ref_ff_virial(const LennardJonesForceField* f) { return f->getVirial(); }
double ref_ff_inside(const LennardJonesForceField* f) { return f->getInsidePairs(); }
int ref_ff_forces_list(LennardJonesForceField* f, System* s, NeighbourList* nl, double* pe) {
    return guarded([&] { *pe = f->computeForces(*s, *nl); });
}
int ref_ff_forces_all(LennardJonesForceField* f, System* s, double* pe) {
    return guarded([&] { *pe = f->computeForces(*s); });
}

// n_steps of VelocityVerletIntegrator::step with the list (or all pairs when nl is null); pe[k] gets each
// step's potential energy and ke[k] the kinetic energy after it (either may be null). When rescale_every
// is positive the velocities are rescaled every that many steps, to rescale_t (md_sim's equilibration)
int ref_run(System* s, LennardJonesForceField* f, NeighbourList* nl, double dt, int n_steps, int rescale_every,
            double rescale_t, double* pe, double* ke) {
    return guarded([&] {
        VelocityVerletIntegrator integ(dt);
        for (int k = 1; k <= n_steps; ++k) {
            const double p = nl ? integ.step(*s, *f, *nl) : integ.step(*s, *f);
            if (rescale_every > 0 && k % rescale_every == 0) rescaleVelocities(*s, rescale_t);
            if (pe) pe[k - 1] = p;
            if (ke) ke[k - 1] = s->kineticEnergy();
        }
    });
}

// NVE steps recording the potential energy, the virial (getVirial) and the kinetic energy after each step
int ref_run_observables(System* s, LennardJonesForceField* f, NeighbourList* nl, double dt, int n_steps, double* pe,
                        double* w, double* ke) {
    return guarded([&] {
        VelocityVerletIntegrator integ(dt);
        for (int k = 0; k < n_steps; ++k) {
            pe[k] = integ.step(*s, *f, *nl);
            w[k] = f->getVirial();
            ke[k] = s->kineticEnergy();
        }
    });
}

BussiThermostat* ref_bussi_create(double t, double tau, std::uint64_t seed) { return new BussiThermostat(t, tau, seed); }
void ref_bussi_destroy(BussiThermostat* b) { delete b; }
void ref_bussi_apply(BussiThermostat* b, System* s, double dt) { b->apply(*s, dt); }

RadialDistribution* ref_rdf_create(double rmax, int bins) { return new RadialDistribution(rmax, bins); }
void ref_rdf_destroy(RadialDistribution* r) { delete r; }
void ref_rdf_sample(RadialDistribution* r, const System* s, const NeighbourList* nl) { r->sample(*s, *nl); }
void ref_rdf_values(const RadialDistribution* r, double* radii, double* g) {
    auto rr = r->radii();
    auto gg = r->values();
    for (std::size_t b = 0; b < gg.size(); ++b) {
        if (radii) radii[b] = rr[b];
        if (g) g[b] = gg[b];
    }
}

}  // extern "C"
