#pragma once
// Drop-in for the reference's include/Integrator.hpp:7-29: velocity Verlet on the GPU (md_step_*).

#include "Forcefield.hpp"
#include "NeighbourList.hpp"
#include "System.hpp"

class VelocityVerletIntegrator {
public:
    explicit VelocityVerletIntegrator(double dt) : dt_(dt) {}

    // One step with O(N^2) forces; returns the new potential energy
    double step(System& system, const LennardJonesForceField& forceField) const;
    // One step with the list: kick, drift and wrap, list update, forces, kick; returns the potential energy
    double step(System& system, const LennardJonesForceField& forceField, NeighbourList& neighbourList) const;

    double getTimestep() const { return dt_; }

private:
    double dt_;
};
