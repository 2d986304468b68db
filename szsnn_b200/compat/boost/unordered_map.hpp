// boost::unordered_map as std::unordered_map hashed by boost::hash (so the
// reference's hash_value overloads for its tuple keys are used,
// SynapseIndex.cpp:15-35).  Iteration order differs from Boost's; the
// reference's layout depends on it only through the order of groupMatrix
// rows (GroupData.cpp:70-228).
#pragma once
#include <unordered_map>

#include "functional/hash.hpp"

namespace boost {
template <class K, class V, class H = boost::hash<K>, class E = std::equal_to<K>>
using unordered_map = std::unordered_map<K, V, H, E>;
}
