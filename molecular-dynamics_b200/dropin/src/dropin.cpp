// The reference's hot-path classes (System, CellList, NeighbourList, LennardJonesForceField,
// VelocityVerletIntegrator, thermostats, RadialDistribution, set-up and trajectory output) implemented over
// libmdgpu's C-ABI. Errors come back as the reference's std::runtime_error with the library's message.
#include "CellList.hpp"
#include "Forcefield.hpp"
#include "Initialisation.hpp"
#include "Integrator.hpp"
#include "NeighbourList.hpp"
#include "RadialDistribution.hpp"
#include "System.hpp"
#include "Thermostat.hpp"
#include "Trajectory.hpp"

#include "md_b200.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <numbers>
#include <stdexcept>
#include <string>

namespace {

void check(md_status s) {
    if (s != MD_OK) throw std::runtime_error(md_last_error());
}

}  // namespace

// ---- System -------------------------------------------------------------------------------------------------

System::System(const std::vector<Particle>& particles, double boxLength, int device)
    : n_(particles.size()), boxLength_(boxLength), inverseBoxLength_(1.0 / boxLength), device_(device) {
    positions_.assign(positionStride * n_, 0.0);
    for (int k = 0; k < 3; ++k) {
        velocity_[k].resize(n_);
        force_[k].resize(n_);
    }
    mass_.resize(n_);
    id_.resize(n_);
    for (std::size_t i = 0; i < n_; ++i) {
        for (int k = 0; k < 3; ++k) {
            positions_[positionStride * i + k] = particles[i].position[k];
            velocity_[k][i] = particles[i].velocity[k];
            force_[k][i] = particles[i].force[k];
        }
        mass_[i] = particles[i].mass;
        id_[i] = i;
    }
    check(md_system_create(static_cast<int64_t>(n_), boxLength, device, &h_));
    hostValid_ = kAll;
    hostDirty_ = kAll;  // the device starts empty: upload everything before the first device call
}

System::System(const System& other)
    : n_(other.n_), boxLength_(other.boxLength_), inverseBoxLength_(other.inverseBoxLength_), device_(other.device_) {
    for (unsigned g = 1; g <= kIds; g <<= 1) other.pull(g);
    positions_ = other.positions_;
    velocity_ = other.velocity_;
    force_ = other.force_;
    mass_ = other.mass_;
    id_ = other.id_;
    check(md_system_create(static_cast<int64_t>(n_), boxLength_, device_, &h_));
    hostValid_ = kAll;
    hostDirty_ = kAll;
}

System::System(System&& other) noexcept
    : n_(other.n_), boxLength_(other.boxLength_), inverseBoxLength_(other.inverseBoxLength_), device_(other.device_),
      h_(other.h_),
      positions_(std::move(other.positions_)), velocity_(std::move(other.velocity_)), force_(std::move(other.force_)),
      mass_(std::move(other.mass_)), id_(std::move(other.id_)), hostValid_(other.hostValid_),
      hostDirty_(other.hostDirty_) {
    other.h_ = nullptr;
}

System::~System() {
    if (h_) md_system_destroy(h_);
}

void System::pull(unsigned group) const {
    if (hostValid_ & group) return;
    const std::size_t n = n_;
    switch (group) {
        case kPositions:
            check(md_system_download(h_, positions_.data(), nullptr, nullptr, nullptr, nullptr));
            break;
        case kVelocities: {
            std::vector<double> v(3 * n);
            check(md_system_download(h_, nullptr, v.data(), nullptr, nullptr, nullptr));
            for (int k = 0; k < 3; ++k) std::memcpy(velocity_[k].data(), v.data() + k * n, sizeof(double) * n);
            break;
        }
        case kForces: {
            std::vector<double> f(3 * n);
            check(md_system_download(h_, nullptr, nullptr, f.data(), nullptr, nullptr));
            for (int k = 0; k < 3; ++k) std::memcpy(force_[k].data(), f.data() + k * n, sizeof(double) * n);
            break;
        }
        case kMasses:
            check(md_system_download(h_, nullptr, nullptr, nullptr, mass_.data(), nullptr));
            break;
        case kIds: {
            std::vector<uint64_t> ids(n);
            check(md_system_download(h_, nullptr, nullptr, nullptr, nullptr, ids.data()));
            for (std::size_t i = 0; i < n; ++i) id_[i] = static_cast<std::size_t>(ids[i]);
            break;
        }
        default:
            break;
    }
    hostValid_ |= group;
}

void System::touch(unsigned group) {
    pull(group);
    hostDirty_ |= group;
}

md_system* System::handle() const {
    if (hostDirty_) {
        const std::size_t n = n_;
        std::vector<double> v, f;
        std::vector<uint64_t> ids;
        if (hostDirty_ & kVelocities) {
            v.resize(3 * n);
            for (int k = 0; k < 3; ++k) std::memcpy(v.data() + k * n, velocity_[k].data(), sizeof(double) * n);
        }
        if (hostDirty_ & kForces) {
            f.resize(3 * n);
            for (int k = 0; k < 3; ++k) std::memcpy(f.data() + k * n, force_[k].data(), sizeof(double) * n);
        }
        if (hostDirty_ & kIds) ids.assign(id_.begin(), id_.end());
        check(md_system_upload(h_, (hostDirty_ & kPositions) ? positions_.data() : nullptr,
                               (hostDirty_ & kVelocities) ? v.data() : nullptr,
                               (hostDirty_ & kForces) ? f.data() : nullptr,
                               (hostDirty_ & kMasses) ? mass_.data() : nullptr,
                               (hostDirty_ & kIds) ? ids.data() : nullptr));
        hostDirty_ = 0;
    }
    return h_;
}

void System::deviceChanged(unsigned groups) const { hostValid_ &= ~groups; }

double* System::packedPositions() {
    touch(kPositions);
    return positions_.data();
}
const double* System::packedPositions() const {
    pull(kPositions);
    return positions_.data();
}
std::span<double> System::velocity(int k) {
    touch(kVelocities);
    return velocity_[k];
}
std::span<const double> System::velocity(int k) const {
    pull(kVelocities);
    return velocity_[k];
}
std::span<double> System::force(int k) {
    touch(kForces);
    return force_[k];
}
std::span<const double> System::force(int k) const {
    pull(kForces);
    return force_[k];
}
std::span<const double> System::mass() const {
    pull(kMasses);
    return mass_;
}
std::span<const std::size_t> System::ids() const {
    pull(kIds);
    return id_;
}
std::array<double, 3> System::positionOf(std::size_t i) const {
    pull(kPositions);
    const double* r = positions_.data() + positionStride * i;
    return {r[0], r[1], r[2]};
}
std::array<double, 3> System::velocityOf(std::size_t i) const {
    pull(kVelocities);
    return {velocity_[0][i], velocity_[1][i], velocity_[2][i]};
}
std::array<double, 3> System::forceOf(std::size_t i) const {
    pull(kForces);
    return {force_[0][i], force_[1][i], force_[2][i]};
}
void System::setPosition(std::size_t i, const std::array<double, 3>& r) {
    touch(kPositions);
    for (int k = 0; k < 3; ++k) positions_[positionStride * i + k] = r[k];
}
void System::setVelocity(std::size_t i, const std::array<double, 3>& v) {
    touch(kVelocities);
    for (int k = 0; k < 3; ++k) velocity_[k][i] = v[k];
}
Particle System::particle(std::size_t i) const {
    Particle p;
    p.position = positionOf(i);
    p.velocity = velocityOf(i);
    p.force = forceOf(i);
    p.mass = mass()[i];
    p.id = ids()[i];
    return p;
}

void System::reorder(std::span<const std::size_t> order) {
    std::vector<uint64_t> o(order.begin(), order.end());
    check(md_system_reorder(handle(), o.data()));
    deviceChanged(kAll);
}

double System::kineticEnergy() const {
    double k = 0.0;
    check(md_kinetic_energy(handle(), &k));
    return k;
}

double System::temperature() const {
    double t = 0.0;
    check(md_temperature(handle(), &t));
    return t;
}

std::uint64_t System::stateHash() const {
    uint64_t h = 0;
    check(md_state_hash(handle(), &h));
    return h;
}

// ---- CellList -----------------------------------------------------------------------------------------------

CellList::CellList(double minCellSize) { check(md_cells_create(minCellSize, &h_)); }
CellList::~CellList() { md_cells_destroy(h_); }

void CellList::build(const System& system) {
    check(md_cells_build(h_, system.handle(), &cellsPerSide_));
    const std::size_t n = system.size();
    const std::size_t ncells = static_cast<std::size_t>(cellsPerSide_) * cellsPerSide_ * cellsPerSide_;
    particleCell_.resize(n);
    std::vector<uint64_t> start(ncells + 1), parts(n);
    check(md_cells_download(h_, particleCell_.data(), start.data(), parts.data()));
    cellStart_.assign(start.begin(), start.end());
    cellParticles_.assign(parts.begin(), parts.end());
}

std::array<int, 27> CellList::neighbourCells(int cell) const {
    const int n = cellsPerSide_;
    const int c[3] = {cell / (n * n), (cell / n) % n, cell % n};
    std::array<int, 27> out {};
    for (int k = 0; k < 27; ++k) {
        // k enumerates (dx, dy, dz) in {-1, 0, 1}^3 with dz fastest
        const int x = (c[0] + k / 9 - 1 + n) % n;
        const int y = (c[1] + (k / 3) % 3 - 1 + n) % n;
        const int z = (c[2] + k % 3 - 1 + n) % n;
        out[k] = (x * n + y) * n + z;
    }
    return out;
}

// ---- NeighbourList ------------------------------------------------------------------------------------------

NeighbourList::NeighbourList(double cutOff, double skin, bool reverseIndex) : reverseIndex_(reverseIndex) {
    check(md_nlist_create(cutOff, skin, reverseIndex ? 1 : 0, &h_));
}
NeighbourList::~NeighbourList() { md_nlist_destroy(h_); }

bool NeighbourList::update(System& system) {
    int rebuilt = 0;
    check(md_nlist_update(h_, system.handle(), &rebuilt));
    if (rebuilt) {
        system.deviceChanged(System::kAll);
        n_ = system.size();
        fetched_ = false;
    }
    return rebuilt != 0;
}

void NeighbourList::build(System& system) {
    check(md_nlist_build(h_, system.handle()));
    system.deviceChanged(System::kAll);
    n_ = system.size();
    fetched_ = false;
}

int NeighbourList::getRebuildCount() const {
    int r = 0;
    check(md_nlist_info(h_, nullptr, &r, nullptr, nullptr));
    return r;
}

std::size_t NeighbourList::getPairCount() const {
    uint64_t p = 0;
    check(md_nlist_info(h_, &p, nullptr, nullptr, nullptr));
    return static_cast<std::size_t>(p);
}

void NeighbourList::fetch() const {
    if (fetched_) return;
    const std::size_t P = getPairCount();
    std::vector<uint64_t> off(n_ + 1), nb(P), roff, rp;
    if (reverseIndex_) {
        roff.resize(n_ + 1);
        rp.resize(P);
    }
    check(md_nlist_download(h_, off.data(), nb.data(), reverseIndex_ ? roff.data() : nullptr,
                            reverseIndex_ ? rp.data() : nullptr));
    offsets_.assign(off.begin(), off.end());
    neighbours_.assign(nb.begin(), nb.end());
    reverseOffsets_.assign(roff.begin(), roff.end());
    reversePairs_.assign(rp.begin(), rp.end());
    fetched_ = true;
}

// ---- LennardJonesForceField ---------------------------------------------------------------------------------

LennardJonesForceField::LennardJonesForceField(double epsilon, double sigma, double cut_off) : cut_off_(cut_off) {
    check(md_forcefield_create(epsilon, sigma, cut_off, &h_));
}
LennardJonesForceField::~LennardJonesForceField() { md_forcefield_destroy(h_); }

double LennardJonesForceField::getEnergyShift() const {
    double s = 0.0;
    check(md_forcefield_shift(h_, &s));
    return s;
}

void LennardJonesForceField::setDeterministic(bool deterministic) {
    check(md_forcefield_set_deterministic(h_, deterministic ? 1 : 0));
}

void LennardJonesForceField::setPrecision(Precision p) {
    check(md_forcefield_set_precision(h_, static_cast<int>(p)));
}

void LennardJonesForceField::fetchResults() const {
    double w = 0.0, ins = 0.0;
    check(md_forcefield_results(h_, &w, &ins));
    setResults(w, ins);
}

double LennardJonesForceField::computeForces(System& system) const {
    double pe = 0.0, w = 0.0, ins = 0.0;
    check(md_forces_all_pairs(h_, system.handle(), &pe, &w, &ins));
    system.deviceChanged(System::kForces);
    setResults(w, ins);
    return pe;
}

double LennardJonesForceField::computeForces(System& system, const NeighbourList& neighbourList) const {
    double pe = 0.0, w = 0.0, ins = 0.0;
    check(md_forces_list(h_, system.handle(), neighbourList.handle(), &pe, &w, &ins));
    system.deviceChanged(System::kForces);
    setResults(w, ins);
    return pe;
}

// ---- VelocityVerletIntegrator ---------------------------------------------------------------------------------

double VelocityVerletIntegrator::step(System& system, const LennardJonesForceField& forceField) const {
    double pe = 0.0;
    check(md_step_all_pairs(system.handle(), forceField.handle(), dt_, &pe));
    system.deviceChanged(System::kPositions | System::kVelocities | System::kForces);
    forceField.fetchResults();
    return pe;
}

double VelocityVerletIntegrator::step(System& system, const LennardJonesForceField& forceField,
                                      NeighbourList& neighbourList) const {
    double pe = 0.0;
    int rebuilt = 0;
    check(md_step_list(system.handle(), forceField.handle(), neighbourList.handle(), dt_, &pe, &rebuilt));
    system.deviceChanged(rebuilt ? System::kAll : (System::kPositions | System::kVelocities | System::kForces));
    if (rebuilt) neighbourList.listChanged();
    forceField.fetchResults();
    return pe;
}

// ---- thermostats ------------------------------------------------------------------------------------------------

void rescaleVelocities(System& system, double targetTemperature) {
    check(md_rescale_velocities(system.handle(), targetTemperature));
    system.deviceChanged(System::kVelocities);
}

BussiThermostat::BussiThermostat(double temperature, double tau, std::uint64_t seed)
    : temperature_(temperature), tau_(tau), rng_(seed) {}

void BussiThermostat::apply(System& system, double dt) {
    // The same two draws per call as the reference (src/Thermostat.cpp:48-51), from this object's stream
    const double dof = 3.0 * static_cast<double>(system.size()) - 3.0;
    std::normal_distribution<double> gaussian(0.0, 1.0);
    std::gamma_distribution<double> gamma(0.5 * (dof - 1.0), 2.0);
    const double r1 = gaussian(rng_);
    const double chi2 = gamma(rng_);
    check(md_bussi_apply(system.handle(), temperature_, tau_, dt, r1, chi2));
    system.deviceChanged(System::kVelocities);
}

// ---- RadialDistribution -------------------------------------------------------------------------------------

RadialDistribution::RadialDistribution(double rMax, int bins) : bins_(bins) { check(md_rdf_create(rMax, bins, &h_)); }
RadialDistribution::~RadialDistribution() { md_rdf_destroy(h_); }

void RadialDistribution::sample(const System& system, const NeighbourList& neighbourList) {
    check(md_rdf_sample(h_, system.handle(), neighbourList.handle()));
}

std::vector<double> RadialDistribution::radii() const {
    std::vector<double> r(bins_);
    check(md_rdf_values(h_, r.data(), nullptr, nullptr));
    return r;
}

std::vector<double> RadialDistribution::values() const {
    std::vector<double> g(bins_);
    check(md_rdf_values(h_, nullptr, g.data(), nullptr));
    return g;
}

bool RadialDistribution::write(const char* path) const {
    std::FILE* f = std::fopen(path, "w");
    if (!f) return false;
    const auto r = radii();
    const auto g = values();
    std::fprintf(f, "r,g\n");
    for (std::size_t b = 0; b < g.size(); ++b) std::fprintf(f, "%.6f,%.6f\n", r[b], g[b]);
    std::fclose(f);
    return true;
}

// ---- set-up and output ---------------------------------------------------------------------------------------

std::vector<Particle> createFCCLattice(int cellsPerSide, double latticeConstant) {
    const std::size_t n = 4 * static_cast<std::size_t>(cellsPerSide) * cellsPerSide * cellsPerSide;
    std::vector<double> pos(4 * n);
    check(md_fcc_lattice(cellsPerSide, latticeConstant, pos.data()));
    std::vector<Particle> out(n);
    for (std::size_t i = 0; i < n; ++i) out[i].position = {pos[4 * i], pos[4 * i + 1], pos[4 * i + 2]};
    return out;
}

void initializeVelocities(System& system, double temperature, std::uint32_t seed) {
    check(md_initialize_velocities(system.handle(), temperature, seed));
    system.deviceChanged(System::kVelocities);
}

void writeXyzFrame(std::FILE* file, const System& system, double time) {
    const std::size_t n = system.size();
    const double l = system.getBoxLength();
    // the frame in id order, gathered on the device (md_system_frame_by_id)
    std::vector<double> f(6 * n);
    check(md_system_frame_by_id(system.handle(), f.data(), 1));
    std::fprintf(file, "%zu\n", n);
    std::fprintf(file,
                 "Lattice=\"%.10g 0 0 0 %.10g 0 0 0 %.10g\" Properties=species:S:1:pos:R:3:velo:R:3:id:I:1 "
                 "Time=%.6f pbc=\"T T T\"\n",
                 l, l, l, time);
    for (std::size_t id = 0; id < n; ++id) {
        const double* r = f.data() + 6 * id;
        std::fprintf(file, "Ar %.8f %.8f %.8f %.8f %.8f %.8f %zu\n", r[0], r[1], r[2], r[3], r[4], r[5], id);
    }
}
