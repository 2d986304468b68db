// The part of boost::posix_time the SZSNN timer uses (SzsnnTimer.cpp:7-123):
// ptime from microsec_clock::local_time(), a default ptime, differences as
// time_duration with total_milliseconds().  Backed by std::chrono.
#pragma once
#include <chrono>
#include <cstdint>

namespace boost {
namespace posix_time {
struct time_duration {
    typedef std::int64_t tick_type;
    std::int64_t us = 0;
    tick_type total_milliseconds() const { return us / 1000; }
    tick_type total_microseconds() const { return us; }
};

struct ptime {
    std::int64_t us = 0;  // microseconds since the steady clock's epoch
    ptime() = default;
    explicit ptime(std::int64_t t) : us(t) {}
    time_duration operator-(const ptime& o) const { return time_duration{us - o.us}; }
};

struct microsec_clock {
    static ptime local_time()
    {
        using namespace std::chrono;
        return ptime(duration_cast<microseconds>(steady_clock::now().time_since_epoch()).count());
    }
};
}  // namespace posix_time
}  // namespace boost
