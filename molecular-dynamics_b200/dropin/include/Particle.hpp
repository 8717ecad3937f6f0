#pragma once
// Drop-in for the reference's include/Particle.hpp:8-14: one particle as a plain record, used to build a
// System and to read single particles.

#include <array>
#include <cstddef>

struct Particle {
    std::array<double, 3> position {0.0, 0.0, 0.0};
    std::array<double, 3> velocity {0.0, 0.0, 0.0};
    std::array<double, 3> force {0.0, 0.0, 0.0};
    double mass {1.0};
    std::size_t id {0};  // stable identity: follows the particle through the re-sorting of list rebuilds
};
