// clemu_rt.hpp -- CPU work-group emulator for OpenCL C kernels.
// TEST INFRASTRUCTURE ONLY ("Oracle B"): lets the reference's own kernel
// sources (szsnn1.1/src/cl/*.cl) run on host cores, compiled as C++.
//
// Model: one OS thread runs the work-groups of a launch one after another;
// the work-items of a group are fibers that switch at barrier().  Fibers run
// in local-id order between barriers, so a launch is deterministic and the
// kernels' local and global atomics need no hardware atomicity.  __local
// variables become `static thread_local` (build_clemu.py rewrites them), which
// all fibers of the running group share.
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>

namespace clemu {
// run `groups` work-groups of `local_size` work-items executing `body`;
// returns 0, or 1 when a barrier was reached by only part of a group
int launch(size_t groups, int local_size, const std::function<void()>& body);
size_t local_id();
size_t group_id();
int local_size();
void barrier();
}  // namespace clemu

// ---- OpenCL C surface used by the reference kernels
typedef unsigned int uint;
typedef unsigned long ulong;
typedef unsigned short ushort;
typedef unsigned char uchar;
struct uint2 { uint x, y; };
struct short2 { short x, y; };
static inline short2 make_short2(int a, int b) { return short2{(short)a, (short)b}; }
static inline uint min(uint a, uint b) { return a < b ? a : b; }

#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
static inline void barrier(int) { clemu::barrier(); }
static inline size_t get_local_id(int) { return clemu::local_id(); }
static inline size_t get_group_id(int) { return clemu::group_id(); }
static inline size_t get_local_size(int) { return (size_t)clemu::local_size(); }
static inline size_t get_global_id(int) { return clemu::group_id() * (size_t)clemu::local_size() + clemu::local_id(); }

// work-items of one group never run concurrently, so read-modify-write is atomic
template <class T, class U> static inline T atomic_add(volatile T* p, U v) { T o = *p; *p = (T)(o + (T)v); return o; }
template <class T> static inline T atomic_inc(volatile T* p) { T o = *p; *p = (T)(o + 1); return o; }
template <class T, class U> static inline T atomic_xchg(volatile T* p, U v) { T o = *p; *p = (T)v; return o; }
template <class T, class U> static inline T atomic_or(volatile T* p, U v) { T o = *p; *p = (T)(o | (T)v); return o; }
template <class T, class U, class V> static inline T atomic_cmpxchg(volatile T* p, U cmp, V val)
{
    T o = *p;
    if (o == (T)cmp) *p = (T)val;
    return o;
}
