// Minimal stand-in for boost accumulators (project-owned shim): only
// accumulator_set<float, stats<tag::mean>> with mean() = float sum / count.
#pragma once
#include <cstddef>
namespace boost { namespace accumulators {
namespace tag { struct mean {}; struct moment {}; }
template <typename... T> struct stats {};
template <typename Sample, typename Features>
class accumulator_set {
public:
    Sample sum = Sample(0);
    std::size_t count = 0;
    void operator()(Sample const &x) { sum += x; ++count; }
};
template <typename Sample, typename Features>
Sample mean(accumulator_set<Sample, Features> const &a) { return a.sum / a.count; }
}}
