#pragma once
// Drop-in for the reference's include/CellList.hpp:11-50: counting sort of particles into cubic cells, run on
// the GPU (md_cells_*); the result is copied to the host after each build.

#include "System.hpp"

#include <array>
#include <cstddef>
#include <span>
#include <vector>

struct md_cells;

class CellList {
public:
    explicit CellList(double minCellSize);
    ~CellList();
    CellList(const CellList&) = delete;
    CellList& operator=(const CellList&) = delete;

    void build(const System& system);
    int getCellsPerSide() const { return cellsPerSide_; }
    int cellOf(std::size_t particle) const { return particleCell_[particle]; }
    // The 27 cells around `cell`, wrapped, in (dx, dy, dz) order from -1 to 1 (src/CellList.cpp:55-83)
    std::array<int, 27> neighbourCells(int cell) const;
    std::span<const std::size_t> particlesIn(int cell) const {
        return {cellParticles_.data() + cellStart_[cell], cellStart_[cell + 1] - cellStart_[cell]};
    }
    std::span<const std::size_t> sortedOrder() const { return cellParticles_; }

private:
    md_cells* h_ = nullptr;
    int cellsPerSide_ = 0;
    std::vector<std::size_t> cellStart_;
    std::vector<std::size_t> cellParticles_;
    std::vector<int> particleCell_;
};
