#pragma once
// Drop-in for the reference's include/Forcefield.hpp:6-78: truncated and shifted Lennard-Jones forces on the
// GPU (md_forcefield_*, md_forces_*). Every mode is deterministic on the device; setDeterministic(true) keeps
// the reference's requirement of a list with a reverse index. setMixedPrecision(true) selects float pair
// arithmetic with 64-bit fixed-point accumulation; setPrecision picks any of the modes of md_precision
// (include/md_b200.h): FixedDouble is exact fixed-point separations with double pair terms (MD_PREC_FX64),
// FixedMixed the same separations with float pair terms and double ones for the close pairs (MD_PREC_FX32).

#include "NeighbourList.hpp"
#include "System.hpp"

struct md_forcefield;

class LennardJonesForceField {
public:
    enum class Precision { Double = 0, FloatFixedPoint = 1, Float = 2, FixedDouble = 3, FixedMixed = 4 };

    LennardJonesForceField(double epsilon, double sigma, double cut_off);
    ~LennardJonesForceField();
    LennardJonesForceField(const LennardJonesForceField&) = delete;
    LennardJonesForceField& operator=(const LennardJonesForceField&) = delete;

    // O(N^2) forces (src/Forcefield.cpp:39-78); returns the potential energy
    double computeForces(System& system) const;
    // Neighbour-list forces (src/Forcefield.cpp:81-326); returns the potential energy
    double computeForces(System& system, const NeighbourList& neighbourList) const;

    double getCutOff() const { return cut_off_; }
    double getEnergyShift() const;
    double getVirial() const { return virial_; }
    double getInsidePairs() const { return insidePairs_; }

    void setMixedPrecision(bool mixed) { setPrecision(mixed ? Precision::FloatFixedPoint : Precision::Double); }
    void setDeterministic(bool deterministic);
    void setPrecision(Precision p);

    md_forcefield* handle() const { return h_; }
    // Refresh getVirial / getInsidePairs from the device's last evaluation (after an integrator step)
    void fetchResults() const;
    void setResults(double virial, double inside) const {
        virial_ = virial;
        insidePairs_ = inside;
    }

private:
    md_forcefield* h_ = nullptr;
    double cut_off_;
    mutable double virial_ = 0.0;
    mutable double insidePairs_ = 0.0;
};
