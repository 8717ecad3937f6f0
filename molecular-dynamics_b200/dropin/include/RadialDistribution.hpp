#pragma once
// Drop-in for the reference's include/RadialDistribution.hpp:8-29: the pair histogram accumulates on the GPU
// (md_rdf_*); radii, values and write follow src/RadialDistribution.cpp:32-69.

#include "NeighbourList.hpp"
#include "System.hpp"

#include <vector>

struct md_rdf;

class RadialDistribution {
public:
    RadialDistribution(double rMax, int bins);
    ~RadialDistribution();
    RadialDistribution(const RadialDistribution&) = delete;
    RadialDistribution& operator=(const RadialDistribution&) = delete;

    void sample(const System& system, const NeighbourList& neighbourList);
    std::vector<double> radii() const;
    std::vector<double> values() const;
    bool write(const char* path) const;  // "r,g" CSV rows

private:
    md_rdf* h_ = nullptr;
    int bins_;
};
