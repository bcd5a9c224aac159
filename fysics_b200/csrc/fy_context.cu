// fy_context.cu -- per-thread CUDA state, error reporting and shared twiddle tables.
#include "fy_context.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace fy {

cudaError_t DevBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    if (p) { cudaFree(p); p = nullptr; cap = 0; }
    if (!bytes) return cudaSuccess;
    size_t want = bytes + (bytes >> 4);        // 6% slack for slowly growing sizes
    want = (want + 255) & ~(size_t)255;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) { p = nullptr; cap = 0; cudaGetLastError(); return e; }
    cap = want;
    return cudaSuccess;
}
void DevBuf::release() { if (p) cudaFree(p); p = nullptr; cap = 0; }

cudaError_t HostBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    if (p) { cudaFreeHost(p); p = nullptr; cap = 0; }
    if (!bytes) return cudaSuccess;
    cudaError_t e = cudaMallocHost(&p, bytes);
    if (e != cudaSuccess) { p = nullptr; cap = 0; cudaGetLastError(); return e; }
    cap = bytes;
    return cudaSuccess;
}
void HostBuf::release() { if (p) cudaFreeHost(p); p = nullptr; cap = 0; }

static thread_local ThreadCtx t_ctx;
ThreadCtx& ctx() { return t_ctx; }

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_ctx.status = code;
    t_ctx.err = buf;
    return code;
}

int fail_cuda(cudaError_t e, const char* what) {
    const int code = (e == cudaErrorMemoryAllocation) ? FY_ENOMEM : FY_ECUDA;
    return fail(code, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

static int init_device(int device) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return fail(FY_ENODEV, "no CUDA device available (%s); fysics_b200 has no CPU fallback",
                    e != cudaSuccess ? cudaGetErrorString(e) : "device count 0");
    }
    if (device < 0 || device >= n) return fail(FY_EINVAL, "device %d out of range [0,%d)", device, n);
    if ((e = cudaSetDevice(device)) != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
    ThreadCtx& c = t_ctx;
    if (c.st && c.dev != device) {          // switching devices: drop the old state
        cudaStreamDestroy(c.st); c.st = nullptr;
        if (c.ws_done) { cudaEventDestroy(c.ws_done); c.ws_done = nullptr; }
        if (c.side) { cudaStreamDestroy(c.side); c.side = nullptr; }
        if (c.fork_ev) { cudaEventDestroy(c.fork_ev); c.fork_ev = nullptr; }
        if (c.join_ev) { cudaEventDestroy(c.join_ev); c.join_ev = nullptr; }
        for (int i = 0; i < ThreadCtx::kBatchStreams; ++i) {
            if (c.bst[i]) { cudaStreamDestroy(c.bst[i]); c.bst[i] = nullptr; }
            if (c.bev[i]) { cudaEventDestroy(c.bev[i]); c.bev[i] = nullptr; }
        }
        if (c.bfork) { cudaEventDestroy(c.bfork); c.bfork = nullptr; }
        if (c.batch_done) { cudaEventDestroy(c.batch_done); c.batch_done = nullptr; }
        c.batch_pending = false;
    }
    c.dev = device;
    cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, device);
    if (!c.st && (e = cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking)) != cudaSuccess)
        return fail_cuda(e, "cudaStreamCreate");
    if (!c.ws_done && (e = cudaEventCreateWithFlags(&c.ws_done, cudaEventDisableTiming)) != cudaSuccess)
        return fail_cuda(e, "cudaEventCreate");
    return FY_OK;
}

int ensure_ctx() {
    ThreadCtx& c = t_ctx;
    if (c.dev >= 0 && c.st) {
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && cur == c.dev) return FY_OK;
        cudaError_t e = cudaSetDevice(c.dev);
        return e == cudaSuccess ? FY_OK : fail_cuda(e, "cudaSetDevice");
    }
    int dev = 0;
    if (const char* s = getenv("FY_DEVICE")) dev = atoi(s);
    return init_device(dev);
}

int ensure_side() {
    ThreadCtx& c = t_ctx;
    cudaError_t e = cudaSuccess;
    if (!c.side && (e = cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking)) != cudaSuccess)
        return fail_cuda(e, "cudaStreamCreate");
    if (!c.fork_ev && (e = cudaEventCreateWithFlags(&c.fork_ev, cudaEventDisableTiming)) != cudaSuccess)
        return fail_cuda(e, "cudaEventCreate");
    if (!c.join_ev && (e = cudaEventCreateWithFlags(&c.join_ev, cudaEventDisableTiming)) != cudaSuccess)
        return fail_cuda(e, "cudaEventCreate");
    return FY_OK;
}

int ensure_batch_streams() {
    ThreadCtx& c = t_ctx;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < ThreadCtx::kBatchStreams; ++i) {
        if (!c.bst[i] && (e = cudaStreamCreateWithFlags(&c.bst[i], cudaStreamNonBlocking)) != cudaSuccess)
            return fail_cuda(e, "cudaStreamCreate");
        if (!c.bev[i] && (e = cudaEventCreateWithFlags(&c.bev[i], cudaEventDisableTiming)) != cudaSuccess)
            return fail_cuda(e, "cudaEventCreate");
    }
    if (!c.bfork && (e = cudaEventCreateWithFlags(&c.bfork, cudaEventDisableTiming)) != cudaSuccess)
        return fail_cuda(e, "cudaEventCreate");
    if (!c.batch_done && (e = cudaEventCreateWithFlags(&c.batch_done, cudaEventDisableTiming)) != cudaSuccess)
        return fail_cuda(e, "cudaEventCreate");
    return FY_OK;
}

void ws_acquire(cudaStream_t s) {
    ThreadCtx& c = t_ctx;
    if (c.ws_pending) cudaStreamWaitEvent(s, c.ws_done, 0);
}
void ws_release(cudaStream_t s) {
    ThreadCtx& c = t_ctx;
    if (cudaEventRecord(c.ws_done, s) == cudaSuccess) c.ws_pending = true;
}

bool is_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return a.type == cudaMemoryTypeHost;
}
bool is_device(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Twiddles are generated in FP64 and rounded once (fft.c:47-61 does the same).
const float2* twiddles(int n) {
    static std::mutex mu;
    static std::map<std::pair<int, int>, float2*> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find({dev, n});
    if (it != cache.end()) return it->second;
    std::vector<float2> h((size_t)n);
    const double step = 2.0 * 3.14159265358979323846 / (double)n;
    for (int m = 0; m < n; ++m) h[(size_t)m] = make_float2((float)cos(step * m), (float)sin(step * m));
    float2* d = nullptr;
    if (cudaMalloc(&d, sizeof(float2) * (size_t)n) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    if (cudaMemcpy(d, h.data(), sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d); cudaGetLastError(); return nullptr;
    }
    cache[{dev, n}] = d;
    return d;
}

// ---------------------------------------------------------------- smem opt-in cache
}  // namespace fy

cudaError_t fy_smem_optin_raw(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    size_t& have = done[{kernel, dev}];
    if (have >= bytes) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) have = bytes;
    return e;
}

namespace fy {
// ---------------------------------------------------------------- profiling marks
struct Prof {
    bool on = false;
    int n = 0;
    std::vector<cudaEvent_t> ev;
    std::vector<const char*> names;
    std::vector<std::string> only;      // marks to record (empty: all)
};
static thread_local Prof t_prof;

}  // namespace fy

void fy_prof_mark(cudaStream_t st, const char* name) {
    fy::Prof& P = fy::t_prof;
    if (!P.on || P.n >= (int)P.ev.size()) return;
    if (P.n > 0 && !P.only.empty()) {              // mark 0 is the origin
        bool keep = false;
        for (const std::string& o : P.only) keep = keep || o == name;
        if (!keep) return;
    }
    if (cudaEventRecord(P.ev[(size_t)P.n], st) == cudaSuccess) P.names[(size_t)P.n++] = name;
}

extern "C" {
// Per-kernel timing with CUDA events recorded on the launching stream after every
// instrumented launch. start(capacity) arms it and records the origin mark; read(i)
// returns the name of mark i and the milliseconds since mark i-1 (after the stream has
// been synchronised).
int fy_gpu_profile_start(int capacity, void* stream) {
    fy::Prof& P = fy::t_prof;
    if (capacity < 2) capacity = 2;
    while ((int)P.ev.size() < capacity) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return fy::fail(FY_ECUDA, "fy_gpu_profile_start: event");
        P.ev.push_back(e);
        P.names.push_back(nullptr);
    }
    P.n = 0;
    P.on = true;
    fy_prof_mark((cudaStream_t)stream, "start");
    return FY_OK;
}
int fy_gpu_profile_select(const char* names) {
    fy::Prof& P = fy::t_prof;
    P.only.clear();
    if (!names) return FY_OK;
    std::string cur;
    for (const char* c = names;; ++c) {
        if (*c == ',' || *c == 0) {
            if (!cur.empty()) P.only.push_back(cur);
            cur.clear();
            if (*c == 0) break;
        } else if (*c != ' ') {
            cur.push_back(*c);
        }
    }
    return FY_OK;
}
int fy_gpu_profile_stop(void) {
    fy::t_prof.on = false;
    return fy::t_prof.n;
}
int fy_gpu_profile_read(int i, const char** name, float* ms) {
    fy::Prof& P = fy::t_prof;
    if (i <= 0 || i >= P.n) return FY_EINVAL;
    if (name) *name = P.names[(size_t)i];
    if (ms && cudaEventElapsedTime(ms, P.ev[(size_t)i - 1], P.ev[(size_t)i]) != cudaSuccess) return FY_ECUDA;
    return FY_OK;
}

int fy_gpu_init(int device) {
    fy::ThreadCtx& c = fy::ctx();
    c.status = 0; c.err.clear();
    return fy::init_device(device);
}
int fy_gpu_last_status(void) { return fy::ctx().status; }
const char* fy_gpu_last_error(void) { return fy::ctx().err.c_str(); }
unsigned long long fy_gpu_kernel_launches(void) { return fy::ctx().launches; }
int fy_gpu_kernel_timeouts(void) {
    const int a = fy_guided_wait_timeouts(), b = fy_noise_wait_timeouts(), d = fy_batch_wait_timeouts(),
              f = fy_deconv_wait_timeouts();
    return a < 0 || b < 0 || d < 0 || f < 0 ? -1 : a + b + d + f;
}
int fy_gpu_test_box_first_wait(int polls) {
    fy::enter();
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    cudaError_t e = fy_guided_set_first_wait_polls(polls);
    if (e == cudaSuccess) e = fy_noise_set_first_wait_polls(polls);
    if (e == cudaSuccess) e = fy_batch_set_first_wait_polls(polls);
    return e == cudaSuccess ? FY_OK : fy::fail_cuda(e, "fy_gpu_test_box_first_wait");
}
int fy_gpu_test_noise_paths(int force_radix, int* window_used) {
    fy::enter();
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = fy_noise_test_paths(force_radix, window_used);
    return e == cudaSuccess ? FY_OK : fy::fail_cuda(e, "fy_gpu_test_noise_paths");
}
void fy_gpu_release(void) {
    fy::ThreadCtx& c = fy::ctx();
    if (c.st) cudaStreamSynchronize(c.st);
    fy_tile_release();
    c.vin.release(); c.vout.release(); c.spec.release(); c.spec2.release();
    c.aux.release(); c.aux2.release(); c.small.release();
    c.pin.release(); c.pin2.release();
    c.tab.buf.release(); c.tab.valid = false;
    c.tab_pin.release();
    if (c.tab_done) { cudaEventDestroy(c.tab_done); c.tab_done = nullptr; }
    c.tab_pending = false;
    if (c.batch_pending && c.batch_done) cudaEventSynchronize(c.batch_done);
    c.batch_pending = false;
    c.batch.release(); c.batch_up.release(); c.batch_pin.release();
    for (int i = 0; i < fy::ThreadCtx::kBatchStreams; ++i) {
        if (c.bst[i]) cudaStreamSynchronize(c.bst[i]);
        c.bspec[i].release();
    }
}
}
