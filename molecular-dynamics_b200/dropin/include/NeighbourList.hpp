#pragma once
// Drop-in for the reference's include/NeighbourList.hpp:10-76: the Verlet list lives on the GPU (md_nlist_*).
// The half list and the reverse index are copied to the host in the reference's CSR form the first time an
// accessor needs them after a build.

#include "System.hpp"

#include <cstddef>
#include <span>
#include <vector>

struct md_nlist;

class NeighbourList {
public:
    NeighbourList(double cutOff, double skin, bool reverseIndex = false);
    ~NeighbourList();
    NeighbourList(const NeighbourList&) = delete;
    NeighbourList& operator=(const NeighbourList&) = delete;

    // Rebuild only if a particle moved more than skin / 2 since the last build; true if rebuilt
    bool update(System& system);
    // Unconditional rebuild; sorts the system's particles by cell
    void build(System& system);

    std::span<const std::size_t> neighboursOf(std::size_t i) const {
        fetch();
        return {neighbours_.data() + offsets_[i], offsets_[i + 1] - offsets_[i]};
    }
    std::size_t firstPairOf(std::size_t i) const {
        fetch();
        return offsets_[i];
    }
    bool hasReverseIndex() const { return reverseIndex_; }
    std::span<const std::size_t> pairsAsSecond(std::size_t j) const {
        fetch();
        return {reversePairs_.data() + reverseOffsets_[j], reverseOffsets_[j + 1] - reverseOffsets_[j]};
    }
    int getRebuildCount() const;
    std::size_t getPairCount() const;

    md_nlist* handle() const { return h_; }
    void listChanged() { fetched_ = false; }  // the device list was rebuilt

private:
    void fetch() const;  // copy the current device list to the host CSR arrays if needed

    md_nlist* h_ = nullptr;
    bool reverseIndex_;
    std::size_t n_ = 0;
    mutable bool fetched_ = false;
    mutable std::vector<std::size_t> offsets_, neighbours_, reverseOffsets_, reversePairs_;
};
