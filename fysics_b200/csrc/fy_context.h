// fy_context.h -- per-thread runtime state behind the C-ABI.
//
// The reference is reentrant through __thread scratch (fft.c:45, guided.c:49) and is
// called concurrently from OpenMP workers (pipeline.c:1008). The GPU library mirrors that:
// every host thread owns a CUDA stream, grow-only device workspaces and pinned staging,
// so concurrent callers never share mutable state. Twiddle tables are immutable and
// shared process-wide.
#pragma once
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stddef.h>
#include <stdint.h>
#include <string>
#include "fy_internal.h"

namespace fy {

// grow-only device buffer
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// grow-only pinned host buffer
struct HostBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
};

struct ThreadCtx {
    int dev = -1;
    int sms = 148;                     // SM count of the selected device
    cudaStream_t st = nullptr;
    cudaEvent_t ws_done = nullptr;     // last enqueue that used this thread's workspaces
    bool ws_pending = false;
    cudaStream_t side = nullptr;       // second stream for work that overlaps the chain
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    int status = 0;
    std::string err;
    unsigned long long launches = 0;
    DevBuf vin, vout, spec, spec2, aux, aux2, small;
    HostBuf pin, pin2;
    // deconvolution table cache (one live entry per thread)
    struct TabEntry { unsigned char key[160]; size_t keylen = 0; DevBuf buf; double us = 0; bool valid = false; };
    TabEntry tab;
    HostBuf tab_pin;                   // pinned staging of the table upload (asynchronous copy)
    cudaEvent_t tab_done = nullptr;    // the last upload from tab_pin has been read
    bool tab_pending = false;
    // batches of volumes (fy_batch.cu): the per-volume buffers, the uploaded plan (tables,
    // box-pass jobs, selection arguments) with its pinned staging and the event after its
    // copy, and kBatchStreams streams with a half-spectrum workspace each
    static constexpr int kBatchStreams = 8;
    DevBuf batch, batch_up;
    HostBuf batch_pin;
    cudaEvent_t batch_done = nullptr;
    bool batch_pending = false;
    cudaStream_t bst[kBatchStreams] = {};
    cudaEvent_t bev[kBatchStreams] = {};
    cudaEvent_t bfork = nullptr;
    DevBuf bspec[kBatchStreams];
};

ThreadCtx& ctx();
// Ensure a device is selected and the thread's stream exists. Returns FY_OK or an error
// code (FY_ENODEV when no CUDA device is usable) with the message recorded.
int ensure_ctx();
// Record a failure for fy_gpu_last_error(); returns code.
int fail(int code, const char* fmt, ...);
int fail_cuda(cudaError_t e, const char* what);
// The thread's side stream and its fork/join events, created on first use.
int ensure_side();
// The thread's batch streams and events, created on first use.
int ensure_batch_streams();
// Make `s` wait for the previous user of this thread's workspaces; call before reuse.
void ws_acquire(cudaStream_t s);
// Mark the workspaces as used by work enqueued on `s`.
void ws_release(cudaStream_t s);
// Immutable FP64-generated twiddle table exp(+2*pi*i*m/n), m < n, on the current device.
const float2* twiddles(int n);
inline void count_launch(int k = 1) { ctx().launches += k; }
// Start of every C entry point: the "last status" describes the latest call only.
inline void enter() { ThreadCtx& c = ctx(); c.status = 0; if (!c.err.empty()) c.err.clear(); }
// Is `p` host memory that the GPU can DMA directly (pinned / registered)?
bool is_pinned(const void* p);
// Is `p` device memory (or managed memory)?
bool is_device(const void* p);

}  // namespace fy
