// fy_api_noise_noalloc.cu -- noise model whose scratch is a static device array.
//
// fy_gpu_estimate_noise_noalloc serves callers that may not allocate device memory while
// they run: a serving loop whose HBM is committed to its own pool (a cudaMalloc there can
// fail, or synchronise the device), or a caller that budgets every byte ahead of time. The
// scratch -- mean/variance fields, the bin labels, the selection control blocks, the sample
// and the candidate list -- lives in
// g_noise_scratch below, sized for FY_NOISE_NOALLOC_MAX_VOXELS voxels. It is part of the
// library's device image, so every GPU that loads the library holds it until exit. Nothing
// here calls cudaMalloc, cudaFree or any other allocating routine.
//
// All calls on a device share the array, and it keeps the previous call's contents. The
// control block is cleared on the stream at the start of every call. The fields are
// rewritten in full by the statistics and labelling kernels. Calls whose GPU work can
// overlap (unordered streams, several host threads) race on the array.
#include <mutex>

#include "fy_context.h"
#include "fysics_b200.h"

using fy::fail;
using fy::fail_cuda;

namespace {

constexpr size_t kMaxVoxels = FY_NOISE_NOALLOC_MAX_VOXELS;
constexpr size_t round64(size_t v) { return (v + 63) & ~(size_t)63; }
// control block first (it holds the 64 KB selection histograms), fields after it
constexpr size_t kCtlBytes = 128 << 10;
// mean, var, bin labels, the candidate selection's control block (<= 128 KB), the sample
// (16384 floats) and the candidate list (n/8 + 4096 values and labels); checked against
// fy_noise_scratch_floats at run time
constexpr size_t kCandMax = (kMaxVoxels + 7) / 8 + 4096;
constexpr size_t kFieldFloats = 2 * round64(kMaxVoxels) + round64((kMaxVoxels + 3) / 4) + (128 << 10) / 4 +
                                16384 + round64(kCandMax) + round64((kCandMax + 3) / 4);
constexpr size_t kScratchBytes = kCtlBytes + kFieldFloats * sizeof(float);
static_assert(kCtlBytes % 256 == 0, "fields must start 256-byte aligned");

static_assert(kScratchBytes == FY_NOISE_NOALLOC_SCRATCH_BYTES, "the header states the array's exact size");

static __device__ __align__(256) unsigned char g_noise_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices];   // last resolved device address of g_noise_scratch, per device

// The host-side name g_noise_scratch is only a handle, so the device address comes from
// cudaGetSymbolAddress, with the device current. It is resolved again on every call that is
// not being captured: a device reset or a new primary context reloads the module, and the
// array can then sit at another address. A call made while `st` is capturing cannot resolve
// (module loading is not a stream operation), so it uses the address of the latest
// uncaptured call on this device, and fails if there was none.
int scratch_on(int dev, cudaStream_t st, void** out, const char* what) {
    if (dev < 0 || dev >= kMaxDevices) return fail(FY_EUNSUPPORTED, "%s: device %d out of range", what, dev);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return fail_cuda(e, what);
    std::lock_guard<std::mutex> lk(g_mu);
    if (cap != cudaStreamCaptureStatusNone) {
        if (!g_addr[dev])
            return fail(FY_EINVAL, "%s: the first call on device %d must come before any stream capture", what, dev);
        *out = g_addr[dev];
        return FY_OK;
    }
    void* p = nullptr;
    if ((e = cudaGetSymbolAddress(&p, g_noise_scratch)) != cudaSuccess) return fail_cuda(e, what);
    if (!p || ((uintptr_t)p & 255)) return fail(FY_ECUDA, "%s: scratch address %p not 256-byte aligned", what, p);
    g_addr[dev] = p;
    *out = p;
    return FY_OK;
}

}  // namespace

extern "C" int fy_gpu_estimate_noise_noalloc(const float* d_in, int nz, int ny, int nx, int win, double flat_pct,
                                             double ref_intensity, fy_noise_model* d_model, float* d_eps,
                                             void* stream) {
    fy::enter();
    const char* what = "fy_gpu_estimate_noise_noalloc";
    if (!d_in || !d_model) return fail(FY_EINVAL, "%s: null pointer", what);
    // the model is written as doubles, eps as one float: misaligned pointers would fault
    if (((uintptr_t)d_model & 7) || ((uintptr_t)d_eps & 3))
        return fail(FY_EINVAL, "%s: d_model must be 8-byte and d_eps 4-byte aligned", what);
    if (nz < 1 || ny < 1 || nx < 1) return fail(FY_EINVAL, "%s: bad dims", what);
    if (win < 3) win = 5;                                         // noise.c:79-80
    if (flat_pct <= 0) flat_pct = 10.0;
    if (win / 2 > 4) return fail(FY_EUNSUPPORTED, "%s: win %d > 9 not supported", what, win);
    const long long n = (long long)nz * ny * nx;
    if (n > (long long)kMaxVoxels)
        return fail(FY_EUNSUPPORTED, "%s: %dx%dx%d = %lld voxels exceeds the static scratch limit of %lld voxels",
                    what, nz, ny, nx, n, (long long)kMaxVoxels);
    if (fy_noise_ctl_bytes() > kCtlBytes) return fail(FY_EUNSUPPORTED, "%s: control block too large", what);
    if (fy_noise_scratch_floats((size_t)n) > kFieldFloats) return fail(FY_EUNSUPPORTED, "%s: scratch layout too large", what);

    int dev = -1, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(FY_ENODEV, "%s: no CUDA device (%s)", what, cudaGetErrorString(e)); }
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return fail_cuda(e, what);
    cudaStream_t st = (cudaStream_t)stream;
    void* base = nullptr;
    int rc = scratch_on(dev, st, &base, what);
    if (rc) return rc;

    void* ctl = base;
    float* fields = (float*)((char*)base + kCtlBytes);
    if ((e = cudaMemsetAsync(ctl, 0, fy_noise_ctl_bytes(), st)) != cudaSuccess) return fail_cuda(e, what);
    int launches = 0;
    if ((e = fy_launch_estimate_noise(d_in, nz, ny, nx, win, flat_pct, ref_intensity, fields, ctl, sms, st,
                                      launches)) != cudaSuccess)
        return fail_cuda(e, what);
    if ((e = fy_noise_store(ctl, d_model, d_eps, st)) != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch(launches + 1);
    return FY_OK;
}
