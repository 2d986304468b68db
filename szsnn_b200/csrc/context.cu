// context.cu -- szsnn_ctx: device pick, stream, buffers, errors.
// Replaces szsnn::Context (Context.cpp:136-224 setup, :398-505 buffers): no
// OpenCL program build, the kernels are compiled ahead of time for sm_100a.
#include "common.cuh"

#include <cstring>

int szsnn_set_error(szsnn_ctx* ctx, int code, const std::string& msg)
{
    if (ctx) ctx->err = msg;
    return code;
}

extern "C" const char* szsnn_last_error(const szsnn_ctx* ctx)
{
    return ctx ? ctx->err.c_str() : "null context";
}

extern "C" int szsnn_ctx_create(int device, const szsnn_layout_consts* consts, szsnn_ctx** out)
{
    if (!out) return SZSNN_ERR_ARG;
    *out = nullptr;
    szsnn_ctx* ctx = new szsnn_ctx();
    if (consts) {
        ctx->c = *consts;
        const szsnn_layout_consts& c = ctx->c;
        if (c.max_partition_size == 0 || c.max_partition_size > 1024 || c.max_partition_size % 32 != 0 ||
            c.warp_size == 0 || c.warp_size > 32 || c.max_synaptic_delay == 0 || c.max_synaptic_delay > 64 ||
            c.threads_per_group == 0) {
            delete ctx;
            return SZSNN_ERR_ARG;
        }
    } else {
        // production constants of locales.h (commented values at :19,34,38,46)
        ctx->c.max_partition_size = 1024;
        ctx->c.threads_per_group = 256;
        ctx->c.warp_size = 32;
        ctx->c.max_synaptic_delay = 64;
    }
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        ctx->own_stream = true;
        e = cudaMalloc((void**)&ctx->d_err, 2 * sizeof(uint32_t));
    }
    if (e == cudaSuccess) e = cudaMemset(ctx->d_err, 0, 2 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return SZSNN_ERR_CUDA;
    }
    *out = ctx;
    return SZSNN_OK;
}

extern "C" int szsnn_ctx_destroy(szsnn_ctx* ctx)
{
    if (!ctx) return SZSNN_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (void* p : ctx->allocs) cudaFree(p);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SZSNN_OK;
}

extern "C" int szsnn_set_stream(szsnn_ctx* ctx, void* stream)
{
    if (!ctx) return SZSNN_ERR_ARG;
    if (ctx->own_stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
        ctx->own_stream = false;
    }
    ctx->stream = (cudaStream_t)stream;
    return SZSNN_OK;
}

extern "C" void* szsnn_get_stream(szsnn_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" int szsnn_alloc(szsnn_ctx* ctx, size_t bytes, void** dev_out)
{
    if (!ctx || !dev_out) return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_alloc: null argument");
    *dev_out = nullptr;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 1);
    if (e != cudaSuccess)
        return szsnn_set_error(ctx, SZSNN_ERR_NOMEM,
                               "szsnn_alloc(" + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    ctx->allocs.insert(p);
    *dev_out = p;
    return SZSNN_OK;
}

extern "C" int szsnn_free(szsnn_ctx* ctx, void* dev)
{
    if (!ctx) return SZSNN_ERR_ARG;
    auto it = ctx->allocs.find(dev);
    if (it == ctx->allocs.end()) return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_free: pointer not owned");
    cudaStreamSynchronize(ctx->stream);
    SZSNN_CUDA_TRY(ctx, cudaFree(dev));
    ctx->allocs.erase(it);
    return SZSNN_OK;
}

extern "C" int szsnn_h2d(szsnn_ctx* ctx, void* dev, const void* host, size_t bytes)
{
    if (!ctx || (!dev && bytes) || (!host && bytes)) return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_h2d: null");
    if (!bytes) return SZSNN_OK;
    SZSNN_CUDA_TRY(ctx, cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    SZSNN_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return SZSNN_OK;
}

extern "C" int szsnn_d2h(szsnn_ctx* ctx, void* host, const void* dev, size_t bytes)
{
    if (!ctx || (!dev && bytes) || (!host && bytes)) return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_d2h: null");
    if (!bytes) return SZSNN_OK;
    SZSNN_CUDA_TRY(ctx, cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    SZSNN_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return SZSNN_OK;
}

extern "C" int szsnn_memset(szsnn_ctx* ctx, void* dev, int value, size_t bytes)
{
    if (!ctx || (!dev && bytes)) return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_memset: null");
    if (!bytes) return SZSNN_OK;
    SZSNN_CUDA_TRY(ctx, cudaMemsetAsync(dev, value, bytes, ctx->stream));
    return SZSNN_OK;
}

extern "C" int szsnn_device_error(szsnn_ctx* ctx, uint32_t* code_out, uint32_t* info_out)
{
    if (!ctx) return SZSNN_ERR_ARG;
    uint32_t h[2] = {0, 0};
    SZSNN_CUDA_TRY(ctx, cudaMemcpyAsync(h, ctx->d_err, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    SZSNN_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (code_out) *code_out = h[0];
    if (info_out) *info_out = h[1];
    return SZSNN_OK;
}

extern "C" int szsnn_clear_device_error(szsnn_ctx* ctx)
{
    if (!ctx) return SZSNN_ERR_ARG;
    SZSNN_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_err, 0, 2 * sizeof(uint32_t), ctx->stream));
    return SZSNN_OK;
}

extern "C" int szsnn_sync(szsnn_ctx* ctx)
{
    if (!ctx) return SZSNN_ERR_ARG;
    SZSNN_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    uint32_t code = 0, info = 0;
    int rc = szsnn_device_error(ctx, &code, &info);
    if (rc) return rc;
    if (code) {
        static const char* const names[] = {"", "synapse target outside the network", "queue slot full",
                                            "spike ring slot full", "NaN or Inf in the state",
                                            "delay outside 1..max_delay",
                                            "launch parity disagrees with the step counter",
                                            "a bounded bulk-copy wait ran out"};
        const std::string what = code < sizeof(names) / sizeof(names[0]) ? names[code] : "unknown check";
        return szsnn_set_error(ctx, SZSNN_ERR_DEVICE,
                               "device check failed: code " + std::to_string(code) + " (" + what + ") info " +
                                   std::to_string(info));
    }
    return SZSNN_OK;
}

extern "C" int szsnn_set_option(szsnn_ctx* ctx, int option, int64_t value)
{
    if (!ctx) return SZSNN_ERR_ARG;
    switch (option) {
    case SZSNN_OPT_OUTPUT_SPARSE_INPUT: ctx->opt_sparse_input = value != 0; return SZSNN_OK;
    case SZSNN_OPT_FIRED_OUTPUT_PARTS: ctx->fired_output_parts = value; return SZSNN_OK;
    case SZSNN_OPT_IZH_HALF_STEPS: ctx->izh_half_steps = value != 0; return SZSNN_OK;
    default: return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_set_option: unknown option");
    }
}
