// Minimal stand-in for boost/dynamic_bitset.hpp (project-owned shim): an
// N-bit set with (n, value) construction and operator[] read/write.
#pragma once
#include <vector>
#include <cstddef>
#include <boost/assert.hpp>
namespace boost {
template <typename Block = unsigned long>
class dynamic_bitset {
    std::vector<Block> words;
    static constexpr size_t BITS = sizeof(Block) * 8;
public:
    class reference {
        Block &w; Block m;
    public:
        reference(Block &w_, Block m_) : w(w_), m(m_) {}
        operator bool() const { return (w & m) != 0; }
        reference &operator=(bool v) { if (v) w |= m; else w &= ~m; return *this; }
    };
    dynamic_bitset(size_t n, bool v = false) : words((n + BITS - 1) / BITS, v ? ~Block(0) : Block(0)) {}
    reference operator[](size_t i) { return reference(words[i / BITS], Block(1) << (i % BITS)); }
    bool operator[](size_t i) const { return (words[i / BITS] >> (i % BITS)) & 1; }
};
}
