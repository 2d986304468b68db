// boost::lexical_cast as the SZSNN host uses it (Connection.hpp:115-122,
// SynapseData.ipp:167): text <-> value through a string stream, throwing
// bad_lexical_cast when the whole text is not consumed.
#pragma once
#include <sstream>
#include <stdexcept>
#include <string>
#include <typeinfo>

namespace boost {
struct bad_lexical_cast : std::bad_cast {
    const char* what() const noexcept override { return "bad lexical cast"; }
};

template <class To, class From>
inline To lexical_cast(const From& v)
{
    std::stringstream ss;
    ss << v;
    if constexpr (std::is_same<To, std::string>::value) {
        return ss.str();
    } else {
        To out;
        if (!(ss >> out)) throw bad_lexical_cast();
        ss >> std::ws;
        if (!ss.eof()) throw bad_lexical_cast();
        return out;
    }
}
}
