// Exercises the autotuner's search (albedo_b200/csrc/autotune.hpp) on synthetic
// cost functions and prints one line per check for tests/test_autotune_search.py.
#include "../../albedo_b200/csrc/autotune.hpp"

#include <cmath>
#include <cstdio>
#include <limits>

using namespace albedo_b200;

int main()
{
    // A separable bowl with its minimum at (16, 4, 64): coordinate descent finds it
    // in one sweep, exhaustive search visits every combination once.
    const std::vector<TuneKnob> knobs{{"a", {8, 16, 32}}, {"b", {2, 3, 4}}, {"c", {16, 32, 64, 128}}};
    int calls{0};
    const TuneMeasure bowl = [&](const std::vector<int>& v) {
        ++calls;
        return std::abs(v[0] - 16) + 10.0 * std::abs(v[1] - 4) + 0.1 * std::abs(v[2] - 64) + 1.0;
    };
    TuneOutcome e{tuneExhaustive(knobs, {8, 2, 16}, bowl)};
    std::printf("exhaustive %d %d %d evaluations=%d calls=%d best=%g start=%g\n", e.best[0], e.best[1], e.best[2],
                e.evaluations, calls, e.best_ms, e.start_ms);
    calls = 0;
    TuneOutcome c{tuneCoordinateDescent(knobs, {8, 2, 16}, bowl, 3)};
    std::printf("descent %d %d %d evaluations=%d calls=%d best=%g\n", c.best[0], c.best[1], c.best[2],
                c.evaluations, calls, c.best_ms);
    // A setting that cannot run (+inf) is never kept.
    const TuneMeasure broken = [&](const std::vector<int>& v) {
        return v[0] == 32 ? -std::numeric_limits<double>::infinity() * -1.0 : 5.0 - v[0] / 16.0;
    };
    TuneOutcome b{tuneCoordinateDescent(knobs, {8, 2, 16}, broken, 2)};
    std::printf("broken %d\n", b.best[0]);
    // A bad starting setting is refused.
    try {
        tuneExhaustive(knobs, {8, 2}, bowl);
        std::printf("mismatch accepted\n");
    } catch (const std::invalid_argument&) {
        std::printf("mismatch refused\n");
    }
    return 0;
}
