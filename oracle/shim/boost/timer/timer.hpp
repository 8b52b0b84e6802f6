// Minimal stand-in for boost/timer/timer.hpp, written for this project so the
// reference sources compile without Boost.  Only what the reference's library
// code uses is provided: cpu_timer::elapsed().wall in nanoseconds.
#pragma once
#include <chrono>
#include <cstdint>
#include <iostream>
namespace boost { namespace timer {
struct cpu_times { int64_t wall, user, system; };
class cpu_timer {
    std::chrono::steady_clock::time_point t0;
public:
    cpu_timer() : t0(std::chrono::steady_clock::now()) {}
    void start() { t0 = std::chrono::steady_clock::now(); }
    cpu_times elapsed() const {
        auto d = std::chrono::steady_clock::now() - t0;
        int64_t ns = std::chrono::duration_cast<std::chrono::nanoseconds>(d).count();
        return cpu_times{ns, 0, 0};
    }
};
class auto_cpu_timer : public cpu_timer {
public:
    ~auto_cpu_timer() { std::cerr << elapsed().wall / 1e9 << "s wall" << std::endl; }
};
}}
