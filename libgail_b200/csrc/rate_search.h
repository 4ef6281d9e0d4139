// The PCRD threshold search shared by the host rate control (allocateRate) and the
// device rate control (rate_gpu.h): the slope histogram size model and the search for
// one slope threshold per component under the DCI limits (Josephur/libgail
// src/core/rate_control.cpp:115-279). Both paths feed it the same bins and exact sizes,
// so both find the same thresholds.
#pragma once

#include <cstdint>
#include <functional>
#include <vector>

#include "codestream.h"

namespace gb {

// Per component, hull points binned by log2(slope) in 1/1024 octave from lo: the data
// bytes and the blocks included above each bin, so the size model costs O(1) per threshold.
class SlopeBins {
public:
    static constexpr double kPerOctave = 1024;
    SlopeBins(double lo, double hi);
    int size() const { return nb_; }
    double lo() const { return lo_; }
    int bin(double slope) const;  // the bin of a slope (+inf: the top bin)
    // adds a hull point's bytes (its rate step) and blocks (1 for a block's first point)
    void add(int comp, int b, double bytes, double blocks) {
        bytes_[comp][(size_t)b] += bytes;
        blocks_[comp][(size_t)b] += blocks;
    }
    void finish();  // totals over the bins at or above each; no add() after it
    void at(const double lam[3], double bytes[3], double blocks[3]) const;

private:
    double lo_;
    int nb_ = 0;
    std::vector<double> bytes_[3], blocks_[3];
};

// The search bounds from the range of the finite positive hull slopes (maxSlope 0 when
// there is none): log2 of each, widened by an octave.
void slopeBounds(double& minSlope, double& maxSlope, double& lo, double& hi);

// Thresholds lam[3] (in: all 0) for which the exact sizes fit lim, the largest set of
// passes the model's bisection and the exact measurements find; sz ends as the size at
// the final thresholds, measure() having been called last with them.
using MeasureFn = std::function<CodestreamSizes(const double lam[3])>;
void rateSearch(const RateLimits& lim, double minSlope, double maxSlope, double loBound, double hiBound,
                const SlopeBins& bins, const MeasureFn& measure, double lam[3], CodestreamSizes& sz);

}  // namespace gb
