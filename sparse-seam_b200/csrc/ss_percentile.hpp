// ss_percentile.hpp -- the harness's sample statistics.
//
// Percentiles interpolate linearly between the two order statistics around
// position q * (n - 1) of the sorted sample, the definition the reference's
// harness uses for its median and p95 columns
// (harness/primary/gpu_common_v0_6.cu:86-103), so the CSV columns of the two
// harnesses mean the same thing.  Header-only, so a CPU test can compile it
// on its own.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <vector>

namespace ss_harness {

inline double percentile(std::vector<double> v, double q) {
    if (v.empty()) {
        return 0.0;
    }
    std::sort(v.begin(), v.end());
    const double pos = q * static_cast<double>(v.size() - 1);
    const size_t lo = static_cast<size_t>(std::floor(pos));
    const size_t hi = std::min(v.size() - 1, lo + 1);
    const double frac = pos - static_cast<double>(lo);
    return v[lo] + (v[hi] - v[lo]) * frac;
}

}  // namespace ss_harness
