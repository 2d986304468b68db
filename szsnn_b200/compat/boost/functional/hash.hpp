// Stand-in for the hashing part of Boost that the SZSNN host uses
// (SynapseIndex.cpp:15-35): boost::hash<T> finds hash_value(T) by argument-
// dependent lookup, and hash_combine folds a value into a seed.  The mixing
// is this library's own (a multiply-xorshift step); any good mix serves,
// since the reference only needs keys to spread over its hash tables.
#pragma once
#include <cstddef>
#include <cstdint>
#include <functional>
#include <type_traits>

namespace boost {
template <class T>
inline typename std::enable_if<std::is_arithmetic<T>::value || std::is_enum<T>::value, std::size_t>::type
hash_value(const T& v)
{
    return std::hash<T>()(v);
}

template <class T>
inline void hash_combine(std::size_t& seed, const T& v)
{
    using boost::hash_value;
    std::uint64_t x = (std::uint64_t)seed ^ ((std::uint64_t)hash_value(v) + 0x632BE59BD9B4E019ull);
    x *= 0xD6E8FEB86659FD93ull;
    x ^= x >> 32;
    seed = (std::size_t)x;
}

template <class T>
struct hash {
    std::size_t operator()(const T& v) const
    {
        using boost::hash_value;
        return hash_value(v);
    }
};
}
