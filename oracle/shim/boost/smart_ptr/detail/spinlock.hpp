// Minimal stand-in for boost::detail::spinlock (project-owned shim).
#pragma once
#include <atomic>
namespace boost { namespace detail {
class spinlock {
    std::atomic<int> v{0};
public:
    spinlock() = default;
    spinlock(spinlock const &) : v(0) {}
    spinlock &operator=(spinlock const &) { return *this; }
    bool try_lock() { int e = 0; return v.compare_exchange_strong(e, 1, std::memory_order_acquire); }
    void lock() { while (!try_lock()) { } }
    void unlock() { v.store(0, std::memory_order_release); }
};
}}
