// cl.hpp -- the OpenCL C++ value types the SZSNN host names, backed by the
// szsnn C ABI (include/szsnn_cuda.h) instead of an OpenCL runtime.
//
// The reference host (Simulation.ipp, Context.hpp, DataBuffer.hpp,
// KernelWrapper.hpp, DeviceManager.cpp, types.h) uses a small part of the
// Khronos C++ bindings: scalar and vector types, a few status / flag /
// query constants, and the classes Buffer, Event, NDRange, Kernel (setArg),
// Device (getInfo), Platform, Context and CommandQueue (finish / flush).
// This header provides exactly that surface.  A Buffer owns a device
// allocation of the library (freed with the last copy); a Kernel records
// its arguments by index for szsnn::Context::enqueueKernel to pass to the
// matching szsnn_* launch; a CommandQueue carries the library context.
// Nothing here talks to OpenCL.
#pragma once

#include <cassert>  // the host uses assert without including it (pulled in by the Khronos header)
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "szsnn_cuda.h"

typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef int16_t cl_short;
typedef uint64_t cl_ulong;
typedef float cl_float;
typedef cl_uint cl_bool;
typedef cl_ulong cl_bitfield;
typedef cl_bitfield cl_mem_flags;
typedef cl_bitfield cl_map_flags;
typedef cl_uint cl_device_info;
typedef cl_uint cl_event_info;

typedef struct { cl_uint s[2]; } cl_uint2;
typedef struct { cl_short s[2]; } cl_short2;

#define CL_SUCCESS 0
#define CL_FALSE 0
#define CL_TRUE 1
#define CL_COMPLETE 0x0
#define CL_RUNNING 0x1
#define CL_SUBMITTED 0x2
#define CL_QUEUED 0x3
#define CL_MEM_READ_WRITE (1 << 0)
#define CL_MEM_WRITE_ONLY (1 << 1)
#define CL_MEM_READ_ONLY (1 << 2)
#define CL_INVALID_VALUE -30
#define CL_INVALID_KERNEL_ARGS -52
#define CL_OUT_OF_RESOURCES -5
#define CL_EVENT_COMMAND_EXECUTION_STATUS 0x11D3
#define CL_DEVICE_NAME 0x102B
#define CL_DEVICE_MIN_DATA_TYPE_ALIGN_SIZE 0x101A
#define CL_DEVICE_MAX_MEM_ALLOC_SIZE 0x1010
#define CL_DEVICE_GLOBAL_MEM_SIZE 0x101F
#define CL_DEVICE_MAX_CONSTANT_BUFFER_SIZE 0x1020
#define CL_DEVICE_LOCAL_MEM_SIZE 0x1023

namespace cl {

// the library context shared by the queue, events and buffers of one
// szsnn::Context (destroyed with its last holder)
struct CtxHandle {
    szsnn_ctx* h = nullptr;
    explicit CtxHandle(szsnn_ctx* c) : h(c) {}
    ~CtxHandle() { if (h) szsnn_ctx_destroy(h); }
    CtxHandle(const CtxHandle&) = delete;
    CtxHandle& operator=(const CtxHandle&) = delete;
};

class NDRange {
public:
    NDRange() : n_(0) { d_[0] = d_[1] = d_[2] = 0; }
    NDRange(size_t x) : n_(1) { d_[0] = x; d_[1] = d_[2] = 1; }
    NDRange(size_t x, size_t y) : n_(2) { d_[0] = x; d_[1] = y; d_[2] = 1; }
    NDRange(size_t x, size_t y, size_t z) : n_(3) { d_[0] = x; d_[1] = y; d_[2] = z; }
    size_t dimensions() const { return n_; }
    size_t operator[](int i) const { return d_[i]; }

private:
    size_t d_[3];
    size_t n_;
};

static const NDRange NullRange;

// a device allocation of the library; copies share it, the last frees it
class Buffer {
public:
    struct Alloc {
        std::shared_ptr<CtxHandle> ctx;
        void* dev = nullptr;
        size_t bytes = 0;
        ~Alloc() { if (dev && ctx && ctx->h) szsnn_free(ctx->h, dev); }
    };
    Buffer() = default;
    void* dev() const { return a_ ? a_->dev : nullptr; }
    size_t bytes() const { return a_ ? a_->bytes : 0; }
    void reset(std::shared_ptr<Alloc> a) { a_ = std::move(a); }

private:
    std::shared_ptr<Alloc> a_;
};

class Event {
public:
    Event() = default;
    void attach(std::shared_ptr<CtxHandle> c) { ctx_ = std::move(c); }
    // the launch has completed when wait returns (one in-order stream)
    cl_int wait() const { return ctx_ ? (szsnn_sync(ctx_->h) == SZSNN_OK ? CL_SUCCESS : CL_OUT_OF_RESOURCES) : CL_SUCCESS; }
    template <typename T>
    cl_int getInfo(cl_event_info name, T* out) const
    {
        if (name != CL_EVENT_COMMAND_EXECUTION_STATUS || !out) return CL_INVALID_VALUE;
        const cl_int rc = wait();
        *out = (T)CL_COMPLETE;
        return rc;
    }

private:
    std::shared_ptr<CtxHandle> ctx_;
};

// kernel arguments recorded by index: a buffer's device pointer or the bytes
// of a scalar
class Kernel {
public:
    struct Arg {
        bool set = false;
        bool is_buffer = false;
        void* dev = nullptr;
        unsigned char bytes[16] = {};
        size_t size = 0;
    };
    Kernel() = default;
    explicit Kernel(const std::string& name) : name_(name) {}
    const std::string& name() const { return name_; }
    cl_int setArg(cl_uint idx, const Buffer& b)
    {
        Arg& a = slot(idx);
        a.set = true;
        a.is_buffer = true;
        a.dev = b.dev();
        return CL_SUCCESS;
    }
    template <typename T>
    cl_int setArg(cl_uint idx, const T& v)
    {
        static_assert(sizeof(T) <= 16, "scalar kernel arguments of at most 16 bytes");
        Arg& a = slot(idx);
        a.set = true;
        a.is_buffer = false;
        std::memset(a.bytes, 0, sizeof(a.bytes));
        std::memcpy(a.bytes, &v, sizeof(T));
        a.size = sizeof(T);
        return CL_SUCCESS;
    }
    const std::vector<Arg>& args() const { return args_; }

private:
    Arg& slot(cl_uint idx)
    {
        if (args_.size() <= idx) args_.resize(idx + 1);
        return args_[idx];
    }
    std::string name_;
    std::vector<Arg> args_;
};

template <cl_device_info N>
struct device_info { typedef cl_ulong type; };
template <>
struct device_info<CL_DEVICE_NAME> { typedef std::string type; };
template <>
struct device_info<CL_DEVICE_MIN_DATA_TYPE_ALIGN_SIZE> { typedef cl_uint type; };

// the one CUDA device of the library context; sizes reported for the
// reference's memory bookkeeping (DeviceManager.cpp:36-50)
class Device {
public:
    template <cl_device_info N>
    typename device_info<N>::type getInfo() const
    {
        if constexpr (N == CL_DEVICE_NAME) {
            return std::string("szsnn sm_100a");
        } else if constexpr (N == CL_DEVICE_MIN_DATA_TYPE_ALIGN_SIZE) {
            return 128u;
        } else if constexpr (N == CL_DEVICE_MAX_MEM_ALLOC_SIZE || N == CL_DEVICE_GLOBAL_MEM_SIZE) {
            return (cl_ulong)180 << 30;
        } else if constexpr (N == CL_DEVICE_MAX_CONSTANT_BUFFER_SIZE) {
            return (cl_ulong)64 << 10;
        } else if constexpr (N == CL_DEVICE_LOCAL_MEM_SIZE) {
            return (cl_ulong)227 << 10;
        } else {
            return 0;
        }
    }
};

class Platform {};
class Program {};

class Context {
public:
    Context() = default;
};

class CommandQueue {
public:
    CommandQueue() = default;
    explicit CommandQueue(std::shared_ptr<CtxHandle> c) : ctx_(std::move(c)) {}
    szsnn_ctx* handle() const { return ctx_ ? ctx_->h : nullptr; }
    const std::shared_ptr<CtxHandle>& shared() const { return ctx_; }
    cl_int finish() const { return ctx_ ? (szsnn_sync(ctx_->h) == SZSNN_OK ? CL_SUCCESS : CL_OUT_OF_RESOURCES) : CL_SUCCESS; }
    cl_int flush() const { return CL_SUCCESS; }

private:
    std::shared_ptr<CtxHandle> ctx_;
};

}  // namespace cl
