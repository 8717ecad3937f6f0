// md_sim for the GPU build: the reference's command-line driver (src/main.cpp of nhantran1711/molecular-dynamics)
// rebuilt over the drop-in classes, with the same flags, stdout tables, CSV columns and machine-readable
// RESULT line, so bench/benchmark.py and bench/validate.py can drive it unchanged. Two additions:
//   --precision fp64|fp32fx|fp32|fx64|fx32   force precision (--mixed is fp32fx)
//   --list-start                   initial forces from the neighbour list instead of the O(N^2) pass
//   --device N                     CUDA device
#include "Forcefield.hpp"
#include "Initialisation.hpp"
#include "Integrator.hpp"
#include "NeighbourList.hpp"
#include "RadialDistribution.hpp"
#include "System.hpp"
#include "Thermostat.hpp"
#include "Trajectory.hpp"

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <string_view>

namespace {

struct Options {
    int cells = 5;
    bool list = true;
    double dt = 0.005, skin = 0.2, cutoff = 2.5;
    int equil = 2000, steps = 5000;
    const char* csv = nullptr;
    bool quiet = false, deterministic = false, mixed = false;
    double density = 0.8442, temperature = 0.728;
    bool nvt = false;
    const char* rdf = nullptr;
    const char* xyz = nullptr;
    int xyzEvery = 100;
    unsigned seed = 42;
    bool melt = false;
    std::string precision;
    bool listStart = false;
    int device = 0;
};

void usage() {
    std::fprintf(stderr,
                 "Usage: md_sim [cellsPerSide] [--brute] [--dt X] [--skin X] [--cutoff X] [--equil N] [--steps N] "
                 "[--density X]\n              [--temperature X] [--nvt] [--seed N] [--melt] [--csv PATH] [--rdf PATH] "
                 "[--xyz PATH] [--xyz-every N]\n              [--deterministic] [--mixed] [--quiet] "
                 "[--precision fp64|fp32fx|fp32|fx64|fx32] [--list-start] [--device N]\n");
}

// Whole-string numeric parse with range checks (the reference's CommandLine.hpp contract)
template <typename T>
bool number(const char* s, T& out) {
    if (!s || !*s) return false;
    char* end = nullptr;
    errno = 0;
    if constexpr (std::is_floating_point_v<T>) {
        const double v = std::strtod(s, &end);
        if (errno || *end) return false;
        out = static_cast<T>(v);
    } else {
        const long long v = std::strtoll(s, &end, 10);
        if (errno || *end) return false;
        if (v < static_cast<long long>(std::numeric_limits<T>::min()) || v > static_cast<long long>(std::numeric_limits<T>::max()))
            return false;
        out = static_cast<T>(v);
    }
    return true;
}

bool parse(int argc, char** argv, Options& o) {
    for (int a = 1; a < argc; ++a) {
        const std::string_view arg = argv[a];
        const bool more = a + 1 < argc;
        auto next = [&]() { return argv[++a]; };
        if (arg == "--brute") o.list = false;
        else if (arg == "--quiet") o.quiet = true;
        else if (arg == "--deterministic") o.deterministic = true;
        else if (arg == "--mixed") o.mixed = true;
        else if (arg == "--nvt") o.nvt = true;
        else if (arg == "--melt") o.melt = true;
        else if (arg == "--list-start") o.listStart = true;
        else if (arg == "--seed" && more) { if (!number(next(), o.seed)) return false; }
        else if (arg == "--density" && more) { if (!number(next(), o.density)) return false; }
        else if (arg == "--temperature" && more) { if (!number(next(), o.temperature)) return false; }
        else if (arg == "--rdf" && more) o.rdf = next();
        else if (arg == "--xyz" && more) o.xyz = next();
        else if (arg == "--xyz-every" && more) { if (!number(next(), o.xyzEvery)) return false; }
        else if (arg == "--dt" && more) { if (!number(next(), o.dt)) return false; }
        else if (arg == "--skin" && more) { if (!number(next(), o.skin)) return false; }
        else if (arg == "--cutoff" && more) { if (!number(next(), o.cutoff)) return false; }
        else if (arg == "--equil" && more) { if (!number(next(), o.equil)) return false; }
        else if (arg == "--steps" && more) { if (!number(next(), o.steps)) return false; }
        else if (arg == "--csv" && more) o.csv = next();
        else if (arg == "--precision" && more) o.precision = next();
        else if (arg == "--device" && more) { if (!number(next(), o.device)) return false; }
        else if (!arg.empty() && arg[0] != '-') { if (!number(argv[a], o.cells)) return false; }
        else return false;
    }
    if (!o.precision.empty() && o.precision != "fp64" && o.precision != "fp32fx" && o.precision != "fp32" &&
        o.precision != "fx64" && o.precision != "fx32")
        return false;
    return o.cells > 0 && o.dt > 0.0 && o.skin > 0.0 && o.cutoff > 0.0 && o.density > 0.0 && o.temperature > 0.0 &&
           o.xyzEvery > 0 && o.steps > 0 && o.equil >= 0;
}

int run(const Options& o) {
    FILE* csv = nullptr;
    if (o.csv) {
        csv = std::fopen(o.csv, "w");
        if (!csv) {
            std::fprintf(stderr, "Could not open %s: %s\n", o.csv, std::strerror(errno));
            return 1;
        }
        std::fprintf(csv, "step,time,phase,ke_per_particle,pe_per_particle,e_per_particle,temperature,pressure,inside_pairs\n");
    }
    const double a = std::cbrt(4.0 / o.density);  // FCC: a^3 = 4 / density
    const double box = o.cells * a;
    System system(createFCCLattice(o.cells, a), box, o.device);
    initializeVelocities(system, o.temperature, o.seed);

    LennardJonesForceField ff(1.0, 1.0, o.cutoff);
    VelocityVerletIntegrator integ(o.dt);
    NeighbourList list(o.cutoff, o.skin, o.deterministic);
    ff.setDeterministic(o.deterministic);
    ff.setMixedPrecision(o.mixed);
    if (o.precision == "fp32fx") ff.setPrecision(LennardJonesForceField::Precision::FloatFixedPoint);
    if (o.precision == "fp32") ff.setPrecision(LennardJonesForceField::Precision::Float);
    if (o.precision == "fx64") ff.setPrecision(LennardJonesForceField::Precision::FixedDouble);
    if (o.precision == "fx32") ff.setPrecision(LennardJonesForceField::Precision::FixedMixed);
    if (o.mixed && (o.deterministic || !o.list)) {
        std::fprintf(stderr, "--mixed applies to the default neighbour list path only\n");
        return 1;
    }
    auto advance = [&]() { return o.list ? integ.step(system, ff, list) : integ.step(system, ff); };

    double potential = 0.0;
    if (o.listStart) {
        list.build(system);
        potential = ff.computeForces(system, list);
    } else {
        potential = ff.computeForces(system);  // the reference's O(N^2) start
        list.build(system);
    }
    const double n = static_cast<double>(system.size());
    if (!o.quiet) {
        std::printf("N = %zu, L = %.4f, rho = %.4f, dt = %.4f, forces = %s, threads = %d\n", system.size(), box,
                    o.density, o.dt, o.list ? "neighbour list" : "all pairs", 1);
        std::printf("\nEquilibration (%d steps, rescale every %d)\n", o.equil, 10);
        std::printf("%8s %12s %12s %12s %12s\n", "step", "KE/N", "PE/N", "E/N", "T");
    }
    const double volume = box * box * box;
    auto pressure = [&](double kinetic) { return (2.0 * kinetic + ff.getVirial()) / (3.0 * volume); };
    auto row = [&](int step, const char* phase, double kinetic, double pe, double t) {
        std::fprintf(csv, "%d,%.6f,%s,%.8f,%.8f,%.8f,%.8f,%.8f,%.0f\n", step, step * o.dt, phase, kinetic / n, pe / n,
                     (kinetic + pe) / n, t, pressure(kinetic), ff.getInsidePairs());
    };
    for (int step = 1; step <= o.equil; ++step) {
        potential = advance();
        if (step % 10 == 0) rescaleVelocities(system, o.melt && step <= o.equil / 3 ? 2.0 : o.temperature);
        if (csv) row(step, "equilibration", system.kineticEnergy(), potential, system.temperature());
        if (!o.quiet && step % 250 == 0) {
            const double k = system.kineticEnergy();
            std::printf("%8d %12.6f %12.6f %12.6f %12.6f\n", step, k / n, potential / n, (k + potential) / n,
                        system.temperature());
        }
    }

    BussiThermostat thermostat(o.temperature, 0.5, o.seed);
    RadialDistribution rdf(o.cutoff, 150);
    if (o.rdf && !o.list) {
        std::fprintf(stderr, "--rdf needs the neighbour list (drop --brute)\n");
        return 1;
    }
    const double e0 = system.kineticEnergy() + potential;
    double sumT = 0.0, sumT2 = 0.0, maxDrift = 0.0;
    if (!o.quiet) {
        std::printf("\nProduction (%d steps, %s)\n", o.steps, o.nvt ? "NVT, Bussi thermostat" : "NVE");
        std::printf("%8s %12s %12s %12s %12s %12s\n", "step", "KE/N", "PE/N", "E/N", "T", "dE/E0");
    }
    FILE* xyz = nullptr;
    if (o.xyz) {
        xyz = std::fopen(o.xyz, "w");
        if (!xyz) {
            std::fprintf(stderr, "Could not open %s: %s\n", o.xyz, std::strerror(errno));
            return 1;
        }
    }
    const auto start = std::chrono::steady_clock::now();
    for (int step = 1; step <= o.steps; ++step) {
        potential = advance();
        if (o.nvt) thermostat.apply(system, o.dt);
        if (o.rdf && step % 10 == 0) rdf.sample(system, list);
        if (xyz && step % o.xyzEvery == 0) writeXyzFrame(xyz, system, (o.equil + step) * o.dt);
        const double k = system.kineticEnergy();
        const double total = k + potential;
        const double t = system.temperature();
        const double drift = (total - e0) / std::abs(e0);
        sumT += t;
        sumT2 += t * t;
        maxDrift = std::max(maxDrift, std::abs(drift));
        if (csv) row(o.equil + step, "production", k, potential, t);
        if (!o.quiet && step % 250 == 0)
            std::printf("%8d %12.6f %12.6f %12.6f %12.6f %12.2e\n", step, k / n, potential / n, total / n, t, drift);
    }
    const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    if (csv) std::fclose(csv);
    if (xyz) std::fclose(xyz);
    if (o.rdf && !rdf.write(o.rdf)) {
        std::fprintf(stderr, "Could not write %s: %s\n", o.rdf, std::strerror(errno));
        return 1;
    }
    const double meanT = sumT / o.steps;
    const double stdT = std::sqrt(std::max(0.0, sumT2 / o.steps - meanT * meanT));
    if (!o.quiet) {
        if (o.nvt)
            std::printf("\n<T> = %.4f +/- %.4f (target %.4f), NVT: total energy not conserved by design\n", meanT, stdT,
                        o.temperature);
        else
            std::printf("\n<T> = %.4f +/- %.4f (target %.4f), max |dE/E0| = %.2e\n", meanT, stdT, o.temperature, maxDrift);
        if (o.list) {
            const int total = o.equil + o.steps;
            std::printf("Neighbour list: %d rebuilds in %d steps (every %.1f steps), %zu pairs\n", list.getRebuildCount(),
                        total, static_cast<double>(total) / list.getRebuildCount(), list.getPairCount());
        }
        std::printf("Production took %.3f s (%.4f ms per step)\n", seconds, 1000.0 * seconds / o.steps);
    }
    std::printf("RESULT n=%zu threads=%d forces=%s dt=%g steps=%d seconds=%.6f ms_per_step=%.6f mean_T=%.6f std_T=%.6f "
                "max_drift=%.6e skin=%g cutoff=%g rebuilds=%d deterministic=%d state_hash=%016llx\n",
                system.size(), 1, o.list ? "list" : "brute", o.dt, o.steps, seconds, 1000.0 * seconds / o.steps, meanT,
                stdT, maxDrift, o.skin, o.cutoff, list.getRebuildCount(), o.deterministic ? 1 : 0,
                static_cast<unsigned long long>(system.stateHash()));
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    Options o;
    if (!parse(argc, argv, o)) {
        usage();
        return 1;
    }
    try {
        return run(o);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "md_sim: %s\n", e.what());
        return 1;
    }
}
