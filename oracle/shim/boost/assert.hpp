// Minimal stand-in for boost/assert.hpp (project-owned shim).  BOOST_VERIFY
// must still evaluate its argument, as Boost's does in release builds.
#pragma once
#include <cassert>
#define BOOST_ASSERT(expr) assert(expr)
#define BOOST_VERIFY(expr) ((void)(expr))
