// Pins the harness's percentile definition: linear interpolation between
// the order statistics around q * (n - 1), as the reference's harness
// computes its median and p95 columns.
#include <cmath>
#include <cstdio>
#include <vector>

#include "ss_percentile.hpp"

static int fails = 0;

static void expect(double got, double want, const char* what) {
    if (std::fabs(got - want) > 1e-12) {
        std::printf("%s: got %.15g, want %.15g\n", what, got, want);
        ++fails;
    }
}

int main() {
    using ss_harness::percentile;
    // Even length: the median is the mean of the two middle values.
    expect(percentile({4.0, 1.0, 3.0, 2.0}, 0.5), 2.5, "median of 4");
    // p95 of 1..30 (the reference's 30 repetitions): position 27.55.
    std::vector<double> reps;
    for (int i = 30; i >= 1; --i) reps.push_back(i);
    expect(percentile(reps, 0.5), 15.5, "median of 30");
    expect(percentile(reps, 0.95), 28.55, "p95 of 30");
    expect(percentile({7.0}, 0.95), 7.0, "single value");
    expect(percentile({}, 0.5), 0.0, "empty sample");
    expect(percentile({1.0, 2.0, 10.0}, 1.0), 10.0, "maximum");
    expect(percentile({1.0, 2.0, 10.0}, 0.0), 1.0, "minimum");
    std::printf(fails ? "FAIL\n" : "OK\n");
    return fails ? 1 : 0;
}
