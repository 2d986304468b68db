// Minimal std-backed stand-in for the part of <boost/shared_ptr.hpp> the
// SZSNN host uses (Simulation.hpp:59, MemoryBuffer.hpp:27): a reference-
// counted owner with get().  Lets the reference host build with no Boost.
#pragma once
#include <memory>

namespace boost {
template <class T>
using shared_ptr = std::shared_ptr<T>;
}
