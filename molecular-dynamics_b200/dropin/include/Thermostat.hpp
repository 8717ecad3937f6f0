#pragma once
// Drop-in for the reference's include/Thermostat.hpp:8-26. The scale factors are computed on the GPU from
// the device kinetic energy; the Bussi draws come from this object's own std::mt19937_64, with the
// reference's distributions, on the host.

#include "System.hpp"

#include <cstdint>
#include <random>

void rescaleVelocities(System& system, double targetTemperature);

class BussiThermostat {
public:
    BussiThermostat(double temperature, double tau, std::uint64_t seed);
    // Call once per timestep, after the integrator step
    void apply(System& system, double dt);
    void setTemperature(double temperature) { temperature_ = temperature; }

private:
    double temperature_;
    double tau_;
    std::mt19937_64 rng_;
};
