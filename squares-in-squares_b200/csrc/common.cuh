// Shared host/device plumbing of libsqs: the context, error reporting and
// CUDA call checking.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/sqs.h"

namespace sqs {

// Per-thread message of the last failed C-ABI call.
void set_error(const char* fmt, ...);
void clear_error();

#define SQS_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t sqs_e_ = (call);                                                     \
        if (sqs_e_ != cudaSuccess) {                                                     \
            ::sqs::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,                  \
                             cudaGetErrorString(sqs_e_));                                \
            return sqs_e_ == cudaErrorMemoryAllocation ? SQS_ENOMEM : SQS_ECUDA;         \
        }                                                                                \
    } while (0)

#define SQS_REQUIRE(cond, ...)                                                           \
    do {                                                                                 \
        if (!(cond)) {                                                                   \
            ::sqs::set_error(__VA_ARGS__);                                               \
            return SQS_EINVAL;                                                           \
        }                                                                                \
    } while (0)

// Device buffer that only grows; used for staging host-pointer calls.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int reserve(size_t want);
    void release();
};

struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int reserve(size_t want);
    void release();
};

}  // namespace sqs

struct sqs_ctx {
    int device = 0;
    int sm_count = 0;
    char name[256] = {0};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[64] = {};
    // side streams that run independent launch groups concurrently, forked
    // from and joined back to `stream` with events (kAux of them)
    static constexpr int kAux = 4;
    cudaStream_t aux[kAux] = {};
    cudaEvent_t fork = nullptr, join[kAux] = {};
    void* flush = nullptr;
    size_t flush_bytes = 0;
    int64_t launches = 0;
    int64_t graph_replays = 0;  // CUDA-graph launches of captured slice loops
    // staging for the host-pointer entry points
    sqs::DevBuf d_in, d_side, d_out, d_grad, d_cand, d_misc, d_anneal;
    sqs::DevBuf d_cert;  // the certifier's per-square interval cache
    sqs::DevBuf d_tune;  // the annealer autotuner's trial state
    sqs::DevBuf d_polish;  // standalone polish batches
    sqs::HostBuf h_cert;   // the certifier's literal slice tables (pinned)
    sqs::HostBuf h_text;   // the certifier's literal text, when large (pinned)
};

namespace sqs {
// Make ctx's device current on the calling thread.
int enter(sqs_ctx* ctx);
}  // namespace sqs
