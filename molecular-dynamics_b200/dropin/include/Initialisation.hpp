#pragma once
// Drop-in for the reference's include/Initialisation.hpp:9-12.

#include "Particle.hpp"
#include "System.hpp"

#include <cstdint>
#include <vector>

// 4 cellsPerSide^3 particles on an FCC lattice offset by a quarter cell (src/Initialisation.cpp:7-44)
std::vector<Particle> createFCCLattice(int cellsPerSide, double latticeConstant);

// Maxwell-Boltzmann velocities from std::mt19937(seed), centre-of-mass removal, exact rescale
// (src/Initialisation.cpp:47-76)
void initializeVelocities(System& system, double temperature, std::uint32_t seed);
