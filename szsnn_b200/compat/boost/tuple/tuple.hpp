// Stand-in for boost::tuple as the SZSNN host uses it (SynapseIndex.hpp:32-44,
// GroupData.cpp:75-125, SynapseData.ipp:73-79): a fixed-size tuple in
// namespace boost::tuples with member get<N>(), free get<N>(t) and
// make_tuple, compared element-wise (tuple_comparison.hpp).
#pragma once
#include <cstddef>
#include <tuple>
#include <utility>

namespace boost {
namespace tuples {
template <class... T>
struct tuple {
    std::tuple<T...> v;
    tuple() = default;
    tuple(const T&... a) : v(a...) {}
    template <int N>
    auto& get() { return std::get<N>(v); }
    template <int N>
    const auto& get() const { return std::get<N>(v); }
};

template <int N, class... T>
inline auto& get(tuple<T...>& t) { return std::get<N>(t.v); }
template <int N, class... T>
inline const auto& get(const tuple<T...>& t) { return std::get<N>(t.v); }

template <class... T>
inline tuple<T...> make_tuple(const T&... a) { return tuple<T...>(a...); }

template <class... T>
inline bool operator==(const tuple<T...>& a, const tuple<T...>& b) { return a.v == b.v; }
template <class... T>
inline bool operator!=(const tuple<T...>& a, const tuple<T...>& b) { return a.v != b.v; }
template <class... T>
inline bool operator<(const tuple<T...>& a, const tuple<T...>& b) { return a.v < b.v; }
}  // namespace tuples
using tuples::get;
using tuples::make_tuple;
using tuples::tuple;
}  // namespace boost
