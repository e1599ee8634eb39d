// C-ABI plumbing of libsqs: contexts, device memory, copies, stream events
// and the L2 flush used by timed callers.
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>

#include "common.cuh"

namespace sqs {

static thread_local char g_err[1024] = {0};

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}
void clear_error() { g_err[0] = 0; }

int DevBuf::reserve(size_t want) {
    if (want <= bytes) return SQS_OK;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t sz = want + want / 4 + 256;
    SQS_CUDA(cudaMalloc(&p, sz));
    bytes = sz;
    return SQS_OK;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}
int HostBuf::reserve(size_t want) {
    if (want <= bytes) return SQS_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    size_t sz = want + want / 4 + 256;
    SQS_CUDA(cudaMallocHost(&p, sz));
    bytes = sz;
    return SQS_OK;
}
void HostBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
}

int enter(sqs_ctx* ctx) {
    SQS_REQUIRE(ctx != nullptr, "null context");
    SQS_CUDA(cudaSetDevice(ctx->device));
    return SQS_OK;
}

}  // namespace sqs

extern "C" {

const char* sqs_version(void) { return "sqs-b200 0.1 (sm_100a)"; }

const char* sqs_last_error(void) { return sqs::g_err; }

int sqs_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int sqs_ctx_create(int device, sqs_ctx** out) {
    sqs::clear_error();
    SQS_REQUIRE(out != nullptr, "null output pointer");
    *out = nullptr;
    int count = sqs_device_count();
    SQS_REQUIRE(device >= 0 && device < count, "device %d not present (%d visible)", device, count);
    SQS_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    SQS_CUDA(cudaGetDeviceProperties(&prop, device));
    SQS_REQUIRE(prop.major >= 10, "libsqs is built for sm_100a; device %d is sm_%d%d", device,
                prop.major, prop.minor);
    sqs_ctx* c = new sqs_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    std::strncpy(c->name, prop.name, sizeof(c->name) - 1);
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    for (int i = 0; e == cudaSuccess && i < 64; ++i) e = cudaEventCreate(&c->ev[i]);
    for (int i = 0; e == cudaSuccess && i < sqs_ctx::kAux; ++i) {
        e = cudaStreamCreateWithFlags(&c->aux[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->join[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        sqs::set_error("context set-up: %s", cudaGetErrorString(e));
        sqs_ctx_destroy(c);
        return SQS_ECUDA;
    }
    *out = c;
    return SQS_OK;
}

int sqs_ctx_destroy(sqs_ctx* ctx) {
    if (!ctx) return SQS_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (int i = 0; i < sqs_ctx::kAux; ++i) {
        if (ctx->aux[i]) cudaStreamSynchronize(ctx->aux[i]);
        if (ctx->aux[i]) cudaStreamDestroy(ctx->aux[i]);
        if (ctx->join[i]) cudaEventDestroy(ctx->join[i]);
    }
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    if (ctx->flush) cudaFree(ctx->flush);
    ctx->d_in.release();
    ctx->d_side.release();
    ctx->d_out.release();
    ctx->d_grad.release();
    ctx->d_cand.release();
    ctx->d_misc.release();
    ctx->d_anneal.release();
    ctx->d_cert.release();
    ctx->d_tune.release();
    ctx->d_polish.release();
    ctx->h_cert.release();
    ctx->h_text.release();
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SQS_OK;
}

int sqs_ctx_device_info(sqs_ctx* ctx, char* name, int name_cap, int* sm_count) {
    SQS_REQUIRE(ctx != nullptr, "null context");
    if (name && name_cap > 0) {
        std::strncpy(name, ctx->name, (size_t)name_cap - 1);
        name[name_cap - 1] = 0;
    }
    if (sm_count) *sm_count = ctx->sm_count;
    return SQS_OK;
}

int sqs_dev_alloc(sqs_ctx* ctx, size_t bytes, void** dptr) {
    if (int r = sqs::enter(ctx)) return r;
    SQS_REQUIRE(dptr != nullptr, "null output pointer");
    SQS_CUDA(cudaMalloc(dptr, bytes ? bytes : 1));
    return SQS_OK;
}

int sqs_dev_free(sqs_ctx* ctx, void* dptr) {
    if (int r = sqs::enter(ctx)) return r;
    SQS_CUDA(cudaFree(dptr));
    return SQS_OK;
}

int sqs_copy_h2d(sqs_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (int r = sqs::enter(ctx)) return r;
    SQS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return SQS_OK;
}

int sqs_copy_d2h(sqs_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (int r = sqs::enter(ctx)) return r;
    SQS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return SQS_OK;
}

int sqs_memset(sqs_ctx* ctx, void* dst, int value, size_t bytes) {
    if (int r = sqs::enter(ctx)) return r;
    SQS_CUDA(cudaMemsetAsync(dst, value, bytes, ctx->stream));
    return SQS_OK;
}

int sqs_host_alloc(size_t bytes, void** hptr) {
    SQS_REQUIRE(hptr != nullptr, "null output pointer");
    SQS_CUDA(cudaMallocHost(hptr, bytes ? bytes : 1));
    return SQS_OK;
}

int sqs_host_free(void* hptr) {
    SQS_CUDA(cudaFreeHost(hptr));
    return SQS_OK;
}

int sqs_sync(sqs_ctx* ctx) {
    if (int r = sqs::enter(ctx)) return r;
    SQS_CUDA(cudaStreamSynchronize(ctx->stream));
    return SQS_OK;
}

int sqs_event_record(sqs_ctx* ctx, int slot) {
    if (int r = sqs::enter(ctx)) return r;
    SQS_REQUIRE(slot >= 0 && slot < 64, "event slot %d out of 0..63", slot);
    SQS_CUDA(cudaEventRecord(ctx->ev[slot], ctx->stream));
    return SQS_OK;
}

int sqs_event_elapsed(sqs_ctx* ctx, int a, int b, float* ms) {
    if (int r = sqs::enter(ctx)) return r;
    SQS_REQUIRE(a >= 0 && a < 64 && b >= 0 && b < 64 && ms, "bad event slots");
    SQS_CUDA(cudaEventSynchronize(ctx->ev[b]));
    SQS_CUDA(cudaEventElapsedTime(ms, ctx->ev[a], ctx->ev[b]));
    return SQS_OK;
}

int sqs_flush_l2(sqs_ctx* ctx) {
    if (int r = sqs::enter(ctx)) return r;
    const size_t want = 256ull << 20;
    if (!ctx->flush) {
        SQS_CUDA(cudaMalloc(&ctx->flush, want));
        ctx->flush_bytes = want;
    }
    static int tick = 0;
    SQS_CUDA(cudaMemsetAsync(ctx->flush, (++tick) & 0xff, ctx->flush_bytes, ctx->stream));
    return SQS_OK;
}

int sqs_ctx_memory(sqs_ctx* ctx, size_t* device_free, size_t* device_total, size_t* staging_device,
                   size_t* staging_host) {
    if (int r = sqs::enter(ctx)) return r;
    size_t fr = 0, tot = 0;
    SQS_CUDA(cudaMemGetInfo(&fr, &tot));
    if (device_free) *device_free = fr;
    if (device_total) *device_total = tot;
    if (staging_device) {
        const sqs::DevBuf* bufs[] = {&ctx->d_in,    &ctx->d_side,  &ctx->d_out,  &ctx->d_grad,
                                     &ctx->d_cand,  &ctx->d_misc,  &ctx->d_anneal, &ctx->d_cert,
                                     &ctx->d_tune,  &ctx->d_polish};
        size_t b = ctx->flush_bytes;
        for (const sqs::DevBuf* d : bufs) b += d->bytes;
        *staging_device = b;
    }
    if (staging_host) *staging_host = ctx->h_cert.bytes + ctx->h_text.bytes;
    return SQS_OK;
}

int64_t sqs_launch_count(sqs_ctx* ctx) { return ctx ? ctx->launches : -1; }
int64_t sqs_graph_replay_count(sqs_ctx* ctx) { return ctx ? ctx->graph_replays : -1; }

}  // extern "C"
