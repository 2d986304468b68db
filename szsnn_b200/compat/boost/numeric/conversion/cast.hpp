// boost::numeric_cast as the SZSNN host uses it (SzsnnTimer.cpp:123,
// Connection.hpp:115-121): a conversion that throws bad_numeric_cast when the
// value does not fit the target type.
#pragma once
#include <limits>
#include <stdexcept>
#include <type_traits>

namespace boost {
struct bad_numeric_cast : std::bad_cast {
    const char* what() const noexcept override { return "bad numeric conversion: value out of range"; }
};

template <class To, class From>
inline To numeric_cast(From v)
{
    if constexpr (std::is_floating_point<From>::value && std::is_integral<To>::value) {
        if (!(v >= (From)std::numeric_limits<To>::min() && v <= (From)std::numeric_limits<To>::max()))
            throw bad_numeric_cast();
    } else if constexpr (std::is_integral<From>::value && std::is_integral<To>::value) {
        if (std::is_signed<From>::value && !std::is_signed<To>::value && v < 0) throw bad_numeric_cast();
        if ((unsigned long long)(v < 0 ? 0 : v) > (unsigned long long)std::numeric_limits<To>::max())
            throw bad_numeric_cast();
    }
    return static_cast<To>(v);
}
}
