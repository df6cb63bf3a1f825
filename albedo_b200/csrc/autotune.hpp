// Launch-shape autotuner: searches a table of knobs, each with its candidate
// values, driven by a measurement callback that returns milliseconds (or
// +infinity for a setting that cannot run). A setting already measured is not
// timed again. Header-only and free of CUDA, so the search itself can be tested
// on a host without a GPU.
#pragma once

#include <cstddef>
#include <functional>
#include <limits>
#include <map>
#include <stdexcept>
#include <vector>

namespace albedo_b200 {

struct TuneKnob {
    const char* name;
    std::vector<int> values;
};

struct TuneOutcome {
    std::vector<int> best; // one value per knob
    double best_ms{std::numeric_limits<double>::infinity()};
    double start_ms{std::numeric_limits<double>::infinity()}; // the starting setting's time
    int evaluations{0};                                      // settings measured
};

using TuneMeasure = std::function<double(const std::vector<int>&)>;

namespace detail {

class MemoMeasure {
public:
    MemoMeasure(const TuneMeasure& measure, TuneOutcome& outcome) : measure_{measure}, outcome_{outcome} {}

    double operator()(const std::vector<int>& setting)
    {
        const auto found{seen_.find(setting)};
        if (found != seen_.end()) {
            return found->second;
        }
        const double ms{measure_(setting)};
        ++outcome_.evaluations;
        seen_.emplace(setting, ms);
        if (ms < outcome_.best_ms) {
            outcome_.best_ms = ms;
            outcome_.best = setting;
        }
        return ms;
    }

private:
    const TuneMeasure& measure_;
    TuneOutcome& outcome_;
    std::map<std::vector<int>, double> seen_;
};

inline void checkStart(const std::vector<TuneKnob>& knobs, const std::vector<int>& start)
{
    if (knobs.size() != start.size() || knobs.empty()) {
        throw std::invalid_argument{"the starting setting needs one value per knob"};
    }
    for (const TuneKnob& k : knobs) {
        if (k.values.empty()) {
            throw std::invalid_argument{"every knob needs at least one candidate value"};
        }
    }
}

} // namespace detail

// Measures every combination of the knobs' values; `start` is measured first.
inline TuneOutcome tuneExhaustive(const std::vector<TuneKnob>& knobs, const std::vector<int>& start,
                                  const TuneMeasure& measure)
{
    detail::checkStart(knobs, start);
    TuneOutcome outcome;
    outcome.best = start;
    detail::MemoMeasure memo{measure, outcome};
    outcome.start_ms = memo(start);
    std::vector<std::size_t> index(knobs.size(), 0);
    for (;;) {
        std::vector<int> setting(knobs.size());
        for (std::size_t k{0}; k < knobs.size(); ++k) {
            setting[k] = knobs[k].values[index[k]];
        }
        memo(setting);
        std::size_t k{0};
        while (k < knobs.size() && ++index[k] == knobs[k].values.size()) {
            index[k] = 0;
            ++k;
        }
        if (k == knobs.size()) {
            return outcome;
        }
    }
}

// Coordinate descent from `start`: each knob in turn takes the value that times
// fastest with the other knobs held at the best setting so far; repeats for
// `sweeps` passes or until a pass changes nothing.
inline TuneOutcome tuneCoordinateDescent(const std::vector<TuneKnob>& knobs, const std::vector<int>& start,
                                         const TuneMeasure& measure, int sweeps)
{
    detail::checkStart(knobs, start);
    TuneOutcome outcome;
    outcome.best = start;
    detail::MemoMeasure memo{measure, outcome};
    outcome.start_ms = memo(start);
    for (int sweep{0}; sweep < sweeps; ++sweep) {
        const std::vector<int> before{outcome.best};
        for (std::size_t k{0}; k < knobs.size(); ++k) {
            for (const int v : knobs[k].values) {
                std::vector<int> setting{outcome.best};
                setting[k] = v;
                memo(setting);
            }
        }
        if (outcome.best == before) {
            break;
        }
    }
    return outcome;
}

} // namespace albedo_b200
