#pragma once
// Drop-in for the reference's include/System.hpp:12-136, backed by a GPU-resident md_system (md_b200.h).
//
// The particle arrays live on the device. Host copies are kept lazily per array group (positions,
// velocities, forces, masses, ids): a const accessor downloads a group the device has changed, a non-const
// accessor (packedPositions(), velocity(k), force(k), setPosition, setVelocity) marks the group as changed
// on the host, and the next operation that runs on the device uploads it first. Spans and pointers handed
// out stay valid, and writes through them are seen, until that next device operation.

#include "Particle.hpp"

#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <span>
#include <vector>

struct md_system;

class System {
public:
    // Ids are 0, 1, 2, ... in input order (src/System.cpp:9-29); ids in the records are ignored
    System(const std::vector<Particle>& particles, double boxLength, int device = 0);
    ~System();
    System(const System& other);  // a second device copy of the same state
    System(System&& other) noexcept;
    System& operator=(const System&) = delete;
    System& operator=(System&&) = delete;

    std::size_t size() const { return n_; }

    static constexpr std::size_t positionStride = 4;
    double* packedPositions();
    const double* packedPositions() const;

    std::span<double> velocity(int k);
    std::span<const double> velocity(int k) const;
    std::span<double> force(int k);
    std::span<const double> force(int k) const;
    std::span<const double> mass() const;
    std::span<const std::size_t> ids() const;

    std::array<double, 3> positionOf(std::size_t i) const;
    std::array<double, 3> velocityOf(std::size_t i) const;
    std::array<double, 3> forceOf(std::size_t i) const;
    void setPosition(std::size_t i, const std::array<double, 3>& r);
    void setVelocity(std::size_t i, const std::array<double, 3>& v);
    Particle particle(std::size_t i) const;

    double getBoxLength() const { return boxLength_; }
    double getInverseBoxLength() const { return inverseBoxLength_; }

    // Minimum image and wrap are host arithmetic with the reference's operation order
    // (include/System.hpp:86-112)
    std::array<double, 3> minimumImageDistance(const std::array<double, 3>& ri, const std::array<double, 3>& rj) const {
        std::array<double, 3> dr {};
        for (int k = 0; k < 3; ++k) {
            const double d = ri[k] - rj[k];
            dr[k] = d - boxLength_ * std::round(d * inverseBoxLength_);
        }
        return dr;
    }
    std::array<double, 3> minimumImageDistance(std::size_t i, std::size_t j) const {
        return minimumImageDistance(positionOf(i), positionOf(j));
    }
    void wrapPosition(std::array<double, 3>& r) const {
        for (double& x : r) x = wrapCoordinate(x);
    }
    double wrapCoordinate(double x) const { return x - boxLength_ * std::floor(x * inverseBoxLength_); }

    // New particle k is old particle order[k] (src/System.cpp:42-64)
    void reorder(std::span<const std::size_t> order);

    double kineticEnergy() const;      // blocked summation order of include/Parallel.hpp:32-57
    std::uint64_t stateHash() const;   // FNV-1a of positions and velocities (src/System.cpp:85-105)
    double temperature() const;

    // ---- GPU plumbing used by the other drop-in classes ----
    md_system* handle() const;          // uploads host-side changes first
    void deviceChanged(unsigned groups) const;  // the device rewrote these groups
    static constexpr unsigned kPositions = 1, kVelocities = 2, kForces = 4, kMasses = 8, kIds = 16, kAll = 31;

private:
    void pull(unsigned group) const;   // make the host copy of a group current
    void touch(unsigned group);        // the host copy of a group is now newer than the device's

    std::size_t n_;
    double boxLength_;
    double inverseBoxLength_;
    int device_;
    md_system* h_ = nullptr;
    mutable std::vector<double> positions_;
    mutable std::array<std::vector<double>, 3> velocity_;
    mutable std::array<std::vector<double>, 3> force_;
    mutable std::vector<double> mass_;
    mutable std::vector<std::size_t> id_;
    mutable unsigned hostValid_ = kAll;  // groups whose host copy matches the device
    mutable unsigned hostDirty_ = 0;     // groups changed on the host, not yet uploaded
};
