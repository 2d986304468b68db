// std-backed stand-in for boost::enable_if_c / enable_if / disable_if as the
// SZSNN neuron models use them (models/NeuronModel.hpp:75-113).
#pragma once
#include <type_traits>

namespace boost {
template <bool B, class T = void>
struct enable_if_c : std::enable_if<B, T> {};
template <class Cond, class T = void>
struct enable_if : std::enable_if<Cond::value, T> {};
template <bool B, class T = void>
struct disable_if_c : std::enable_if<!B, T> {};
template <class Cond, class T = void>
struct disable_if : std::enable_if<!Cond::value, T> {};
}
