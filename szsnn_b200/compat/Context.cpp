// Context.cpp -- szsnn::Context (declared by the reference's Context.hpp:77-303)
// implemented over the szsnn C ABI, so the reference's unchanged host
// (Simulation, NeuronData, SynapseData, GroupData, queues, SpikeBuffer,
// CurrentData, DeviceManager) runs its step on the sm_100a kernels of
// libszsnn_cuda.so.  It replaces the reference's own Context.cpp, the one
// place where that host talks to OpenCL:
//
//   setup()          szsnn_ctx_create with the build's layout constants
//                    (MAX_PARTITION_SIZE, THREADS_PER_GROUP, WARP_SIZE,
//                    MAX_SYNAPTIC_DELAY), in place of platform / device /
//                    context / queue discovery and the kernel-source build
//                    (Context.cpp:106-220, 243-355)
//   createKernel     names the kernel; its arguments are recorded by
//                    cl::Kernel::setArg as the host binds them
//   enqueueKernel    the szsnn_* launch of the kernel's name with the
//                    recorded arguments, in the reference's order
//                    (IF_curr_exp_update_kernel.cl:100-120,
//                    scatter_kernel.cl:68-83, gather_kernel.cl:67-77); the
//                    event returned completes on szsnn_sync
//   createBuffer /   szsnn_alloc, and blocking szsnn_h2d / szsnn_d2h with
//   write / read     the reference's offset and size (Context.cpp:398-505)
//
// Every failing status becomes the SzsnnException the reference throws
// (utils.h:144-155), carrying szsnn_last_error's message.
#include "Context.hpp"

#include <cstring>

namespace szsnn {

namespace {

uint64_t arg_u64(const cl::Kernel::Arg& a)
{
    uint64_t v = 0;
    std::memcpy(&v, a.bytes, a.size < 8 ? a.size : 8);
    return v;
}

uint32_t arg_u32(const cl::Kernel::Arg& a) { return (uint32_t)arg_u64(a); }

template <class T>
T* arg_ptr(const cl::Kernel::Arg& a)
{
    return static_cast<T*>(a.dev);
}

void check(szsnn_ctx* h, int rc, const std::string& what)
{
    if (rc != SZSNN_OK) {
        const char* m = szsnn_last_error(h);
        THROW_SZSNNEX("SZSNN::Context::" << what << " failed with status " << rc << ": " << (m ? m : ""));
    }
}

}  // namespace

void Context::setup()
{
    szsnn_layout_consts c;
    c.max_partition_size = MAX_PARTITION_SIZE;
    c.threads_per_group = THREADS_PER_GROUP;
    c.warp_size = WARP_SIZE;
    c.max_synaptic_delay = MAX_SYNAPTIC_DELAY;
    szsnn_ctx* h = nullptr;
    const int rc = szsnn_ctx_create(0, &c, &h);
    if (rc != SZSNN_OK) THROW_SZSNNEX("SZSNN::Context::setup: szsnn_ctx_create failed with status " << rc);
    commandQueue = cl::CommandQueue(std::make_shared<cl::CtxHandle>(h));
    device = cl::Device();
    deviceMgr.setup(device);
}

void Context::createKernel(cl::Kernel& kernel, std::string kernelFileName, std::string kernelName,
                           std::string flagsStr, size_t blockSizeX, size_t blockSizeY)
{
    (void)kernelFileName;
    (void)flagsStr;
    if (blockSizeX * blockSizeY > (size_t)THREADS_PER_GROUP)
        THROW_SZSNNEX("SZSNN::Context::createKernel: group of " << blockSizeX * blockSizeY << " work-items for "
                      << kernelName << " exceeds THREADS_PER_GROUP " << THREADS_PER_GROUP);
    kernel = cl::Kernel(kernelName);
    if (registerON) deviceMgr.registerKernel(kernelName);
}

void Context::createKernel(KernelWrapper& wrap)
{
    createKernel(wrap.kernel, wrap.kernelFileName, wrap.kernelName, wrap.flags, wrap.blockSizeX, wrap.blockSizeY);
}

void Context::enqueueKernel(const cl::Kernel& kernel, std::string kernelName, const cl::NDRange& global,
                            const cl::NDRange& local, const std::vector<cl::Event>* events, cl::Event* event)
{
    (void)global;
    (void)local;
    (void)events;  // one in-order stream: earlier launches complete first
    szsnn_ctx* h = commandQueue.handle();
    if (!h) THROW_SZSNNEX("SZSNN::Context::enqueueKernel: " << kernelName << " before setup()");
    const std::vector<cl::Kernel::Arg>& a = kernel.args();
    auto need = [&](size_t n) {
        if (a.size() < n) THROW_SZSNNEX("SZSNN::Context::enqueueKernel: " << kernelName << " has " << a.size()
                                        << " arguments bound, needs " << n);
        for (size_t i = 0; i < n; ++i)
            if (!a[i].set) THROW_SZSNNEX("SZSNN::Context::enqueueKernel: argument " << i << " of " << kernelName
                                         << " is not bound");
    };
    int rc = SZSNN_OK;
    if (kernelName == "IF_curr_exp_update" || kernelName == "Izhikevich_update" || kernelName == "Const_rate_update") {
        need(15);
        auto fn = kernelName == "IF_curr_exp_update" ? szsnn_update_if_curr_exp
                  : kernelName == "Izhikevich_update" ? szsnn_update_izhikevich
                                                      : szsnn_update_const_rate;
        rc = fn(h, arg_u64(a[0]), arg_u32(a[1]), arg_ptr<const uint32_t>(a[2]), arg_ptr<const float>(a[3]),
                arg_ptr<float>(a[4]), arg_u32(a[5]), arg_ptr<float>(a[6]), arg_ptr<float>(a[7]), arg_u32(a[8]),
                arg_ptr<uint32_t>(a[9]), arg_ptr<uint32_t>(a[10]), arg_ptr<uint32_t>(a[11]),
                arg_ptr<uint32_t>(a[12]), arg_u32(a[13]), arg_u32(a[14]));
    } else if (kernelName == "scatter") {
        need(14);
        rc = szsnn_scatter(h, arg_u64(a[0]), arg_u32(a[1]), arg_ptr<uint32_t>(a[2]), arg_ptr<uint32_t>(a[3]),
                           arg_u32(a[4]), arg_u32(a[5]), arg_ptr<const uint32_t>(a[6]),
                           arg_ptr<const uint32_t>(a[7]), arg_u64(a[8]), arg_ptr<uint32_t>(a[9]),
                           arg_ptr<uint32_t>(a[10]), arg_ptr<uint32_t>(a[11]), arg_ptr<int16_t>(a[12]),
                           arg_ptr<const uint64_t>(a[13]));
    } else if (kernelName == "gather") {
        need(9);
        rc = szsnn_gather(h, arg_u64(a[0]), arg_u32(a[1]), arg_ptr<const uint32_t>(a[2]), arg_ptr<float>(a[3]),
                          arg_u64(a[4]), arg_ptr<uint32_t>(a[5]), arg_ptr<uint32_t>(a[6]),
                          arg_ptr<const uint32_t>(a[7]), arg_ptr<const float>(a[8]));
    } else {
        THROW_SZSNNEX("SZSNN::Context::enqueueKernel: no sm_100a kernel for " << kernelName);
    }
    check(h, rc, "enqueueKernel(" + kernelName + ")");
    if (event) event->attach(commandQueue.shared());
}

void Context::enqueueKernel(const KernelWrapper& wrap, const std::vector<cl::Event>* events, cl::Event* event)
{
    enqueueKernel(wrap.kernel, wrap.kernelName, wrap.globalRange, wrap.localRange, events, event);
}

void Context::createBuffer(cl::Buffer& buffer, std::string bufferName, std::vector<std::string> kernelNames,
                           cl_mem_flags flags, size_t size)
{
    (void)flags;
    szsnn_ctx* h = commandQueue.handle();
    auto alloc = std::make_shared<cl::Buffer::Alloc>();
    alloc->ctx = commandQueue.shared();
    alloc->bytes = size;
    if (h) {
        void* p = nullptr;
        check(h, szsnn_alloc(h, size ? size : 1, &p), "createBuffer(" + bufferName + ")");
        alloc->dev = p;
    }  // before setup(): a host-only record (the layout builders run without a device)
    buffer.reset(alloc);
    if (registerON) deviceMgr.registerMemory(kernelNames, bufferName, DeviceManager::MEM_GLOBAL, size);
}

void Context::writeBuffer(const cl::Buffer& buffer, std::string bufferName, cl_bool block, cl_uint offset,
                          cl_uint size, const void* ptr)
{
    (void)block;  // copies are blocking, as the reference always asks (CL_TRUE)
    szsnn_ctx* h = commandQueue.handle();
    if (!h) THROW_SZSNNEX("SZSNN::Context::writeBuffer: " << bufferName << " before setup()");
    if ((size_t)offset + size > buffer.bytes())
        THROW_SZSNNEX("SZSNN::Context::writeBuffer: " << bufferName << " [" << offset << ", " << offset + size
                      << ") outside its " << buffer.bytes() << " bytes");
    if (size) check(h, szsnn_h2d(h, static_cast<char*>(buffer.dev()) + offset, ptr, size), "writeBuffer(" + bufferName + ")");
}

void Context::readBuffer(const cl::Buffer& buffer, std::string bufferName, cl_bool block, cl_uint offset,
                         cl_uint size, void* ptr)
{
    (void)block;
    szsnn_ctx* h = commandQueue.handle();
    if (!h) THROW_SZSNNEX("SZSNN::Context::readBuffer: " << bufferName << " before setup()");
    if ((size_t)offset + size > buffer.bytes())
        THROW_SZSNNEX("SZSNN::Context::readBuffer: " << bufferName << " [" << offset << ", " << offset + size
                      << ") outside its " << buffer.bytes() << " bytes");
    if (size) check(h, szsnn_d2h(h, ptr, static_cast<const char*>(buffer.dev()) + offset, size), "readBuffer(" + bufferName + ")");
}

}  // namespace szsnn
