// fy_autotune.cu -- measured launch shapes for the restoration chain, cached per GPU.
//
// Knobs (each changes how work is split over CTAs, never the arithmetic, so every choice
// gives bit-identical results):
//   x1.<n>, x5.<n>        lines per CTA (log2) of the deconvolution X passes (forward, inverse)
//                         of axis length n. Their tiles are line-major, so any power of two up
//                         to the default fits: fewer lines, more CTAs per SM.
// The z chunk count of the z-sliding box passes is not a knob: each chunk takes its variance
// shift from its own first plane, so the chunking changes the float rounding of the sums.
// fy_gpu_autotune measures candidates of each knob by timing the whole chain on a scratch
// cube of the given shape (coordinate descent, median of repeated CUDA-event timings) and
// writes the winners to a JSON cache, one entry per line:
//   {"device": "<name>|sm<count>|drv<version>|rt<version>", "knob": "...", "value": V, "ms": T}
// keyed by the GPU model, its SM count and the driver and runtime versions, so a cache made
// on another GPU or driver is ignored. The cache is $FY_TUNE_CACHE, else
// $XDG_CACHE_HOME/fysics_b200/tune.json, else ~/.cache/fysics_b200/tune.json; it is read on
// the first lookup. FY_TUNE=0 disables tuned values (the defaults run).
#include <ctype.h>
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

namespace {

std::mutex g_mu;
bool g_loaded = false;
bool g_disabled = false;
std::map<std::string, int> g_table;      // "<device>#<knob>" -> value
std::map<std::string, double> g_ms;      // chain time measured with the winning value
std::string g_path;

std::string cache_path() {
    if (const char* p = getenv("FY_TUNE_CACHE")) return p;
    std::string base;
    if (const char* x = getenv("XDG_CACHE_HOME")) base = x;
    else if (const char* h = getenv("HOME")) base = std::string(h) + "/.cache";
    else base = "/tmp";
    return base + "/fysics_b200/tune.json";
}

std::string device_key(int dev) {
    static std::mutex mu;
    static std::map<int, std::string> keys;
    std::lock_guard<std::mutex> lk(mu);
    auto it = keys.find(dev);
    if (it != keys.end()) return it->second;
    cudaDeviceProp pr;
    int drv = 0, rt = 0;
    if (cudaGetDeviceProperties(&pr, dev) != cudaSuccess) {
        cudaGetLastError();
        return "";
    }
    cudaDriverGetVersion(&drv);
    cudaRuntimeGetVersion(&rt);
    char buf[400];
    snprintf(buf, sizeof buf, "%s|sm%d|drv%d|rt%d", pr.name, pr.multiProcessorCount, drv, rt);
    for (char* c = buf; *c; ++c)
        if (*c == '"' || *c == '\\' || *c == '#') *c = '_';
    keys[dev] = buf;
    return buf;
}

int current_device() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return d;
}

// The value of "key": <digits or string> in one cache line.
bool field(const std::string& ln, const char* key, std::string& out) {
    const std::string k = std::string("\"") + key + "\"";
    size_t p = ln.find(k);
    if (p == std::string::npos) return false;
    p = ln.find(':', p + k.size());
    if (p == std::string::npos) return false;
    ++p;
    while (p < ln.size() && ln[p] == ' ') ++p;
    if (p < ln.size() && ln[p] == '"') {
        const size_t q = ln.find('"', p + 1);
        if (q == std::string::npos) return false;
        out = ln.substr(p + 1, q - p - 1);
        return true;
    }
    size_t q = p;
    while (q < ln.size() && (isdigit((unsigned char)ln[q]) || ln[q] == '-' || ln[q] == '.' || ln[q] == 'e')) ++q;
    out = ln.substr(p, q - p);
    return q > p;
}

// Read the cache (entries of every device; lookups match the current device). Called with g_mu held.
int load_locked(const std::string& path) {
    g_table.clear();
    g_ms.clear();
    g_path = path;
    g_loaded = true;
    FILE* f = fopen(path.c_str(), "r");
    if (!f) return 0;
    char line[2048];
    int n = 0;
    while (fgets(line, sizeof line, f)) {
        const std::string ln(line);
        std::string dev, knob, val, ms;
        if (!field(ln, "device", dev) || !field(ln, "knob", knob) || !field(ln, "value", val)) continue;
        const int v = atoi(val.c_str());
        if (v <= 0) continue;
        g_table[dev + "#" + knob] = v;
        if (field(ln, "ms", ms)) g_ms[dev + "#" + knob] = atof(ms.c_str());
        ++n;
    }
    fclose(f);
    return n;
}

void ensure_loaded() {
    if (g_loaded) return;
    const char* off = getenv("FY_TUNE");
    g_disabled = off && off[0] == '0';
    load_locked(cache_path());
}

int lookup(const std::string& knob) {
    const int dev = current_device();
    if (dev < 0) return 0;
    const std::string dk = device_key(dev);
    std::lock_guard<std::mutex> lk(g_mu);
    ensure_loaded();
    if (g_disabled) return 0;
    auto it = g_table.find(dk + "#" + knob);
    return it == g_table.end() ? 0 : it->second;
}

void mkdirs_for(const std::string& path) {
    for (size_t i = 0; i < path.size(); ++i) {
        if (path[i] == '/' && i > 0) mkdir(path.substr(0, i).c_str(), 0775);
    }
}

// Rewrite the cache with the in-memory table (all devices). Called with g_mu held.
int save_locked() {
    mkdirs_for(g_path);
    const std::string tmp = g_path + ".tmp";
    FILE* f = fopen(tmp.c_str(), "w");
    if (!f) return -1;
    for (const auto& kv : g_table) {
        const size_t h = kv.first.find('#');
        const std::string dev = kv.first.substr(0, h), knob = kv.first.substr(h + 1);
        auto m = g_ms.find(kv.first);
        fprintf(f, "{\"device\": \"%s\", \"knob\": \"%s\", \"value\": %d, \"ms\": %.5f}\n", dev.c_str(), knob.c_str(),
                kv.second, m == g_ms.end() ? 0.0 : m->second);
    }
    fclose(f);
    return rename(tmp.c_str(), g_path.c_str()) == 0 ? 0 : -1;
}

std::string x_knob(int pass, int n) { return "x" + std::to_string(pass) + "." + std::to_string(n); }

__global__ void k_tune_fill(unsigned char* p, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        unsigned h = (unsigned)i * 2654435761u;
        h ^= h >> 15;
        p[i] = (unsigned char)(96 + (h & 63));        // mid-grey texture: every stage does its full work
    }
}

}  // namespace

int fy_tuned_x_wlog(int pass, int n) { return lookup(x_knob(pass, n)); }

extern "C" int fy_gpu_tune_load(const char* path) {
    fy::enter();
    std::lock_guard<std::mutex> lk(g_mu);
    const char* off = getenv("FY_TUNE");
    g_disabled = off && off[0] == '0';
    return load_locked(path ? std::string(path) : cache_path());
}

extern "C" int fy_gpu_tune_value(const char* knob) {
    fy::enter();
    if (!knob) return 0;
    return lookup(knob);
}

extern "C" int fy_gpu_autotune(int nz, int ny, int nx, int flags) {
    fy::enter();
    const char* what = "fy_gpu_autotune";
    if (nz < 8 || ny < 8 || nx < 8) return fail(FY_EINVAL, "%s: dims %dx%dx%d too small to tune", what, nz, ny, nx);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    fy::ThreadCtx& c = ctx();
    const std::string dk = device_key(c.dev);
    if (dk.empty()) return fail(FY_ECUDA, "%s: device properties", what);
    const int px = fy_next_fft_size(nx);
    const std::vector<std::string> knobs = {x_knob(1, px), x_knob(5, px)};
    {
        std::lock_guard<std::mutex> lk(g_mu);
        ensure_loaded();
        bool all = true;
        for (const auto& k : knobs) all = all && g_table.count(dk + "#" + k);
        if (all && !(flags & 1)) return FY_OK;             // cached
    }
    // scratch cube, output and the chain's settings (matched anisotropic deconvolution, noise
    // window 5, exact guided filter r = 2)
    const size_t n = (size_t)nz * ny * nx;
    unsigned char* d_u8 = nullptr;
    float* d_out = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&d_u8, n)) != cudaSuccess) return fail_cuda(e, what);
    if ((e = cudaMalloc(&d_out, n * sizeof(float))) != cudaSuccess) {
        cudaFree(d_u8);
        return fail_cuda(e, what);
    }
    cudaStream_t st = c.st;
    k_tune_fill<<<c.sms * 4, 256, 0, st>>>(d_u8, n);
    fy_physics ph{500.0 * 0.35, 110.0, 1200.0, 2.4, 0.8, 0.5, 1.0, 1.17};
    fy_restore_cfg cfg;
    fy_restore_cfg_default(&cfg);
    cfg.deconv_kind = 1;
    cfg.deconv_param = 0.05;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto chain_ms = [&](double& ms) -> int {
        std::vector<float> t;
        for (int rep = 0; rep < 5; ++rep) {
            cudaEventRecord(e0, st);
            int q = fy_gpu_restore_u8(d_u8, d_out, nz, ny, nx, 0.0, 1.0, &ph, &cfg, st);
            if (q) return q;
            cudaEventRecord(e1, st);
            if ((e = cudaEventSynchronize(e1)) != cudaSuccess) return fail_cuda(e, what);
            float v = 0.f;
            cudaEventElapsedTime(&v, e0, e1);
            if (rep >= 2) t.push_back(v);                  // two warm-up chains
        }
        std::sort(t.begin(), t.end());
        ms = t[t.size() / 2];
        return FY_OK;
    };
    auto set = [&](const std::string& knob, int v) {
        std::lock_guard<std::mutex> lk(g_mu);
        if (v > 0) g_table[dk + "#" + knob] = v;
        else g_table.erase(dk + "#" + knob);
    };
    // candidates per knob (0 = the built-in default)
    const TileShape tx = fy_tile_shape(px);
    std::vector<int> xc = {0};
    for (int wl = tx.wlog - 1; wl >= 1 && wl >= tx.wlog - 2; --wl)
        if ((px << wl) / tx.E >= 32) xc.push_back(wl);
    for (const auto& k : knobs) set(k, 0);
    double best_ms = 0.0;
    rc = chain_ms(best_ms);
    for (size_t ki = 0; ki < knobs.size() && !rc; ++ki) {
        const std::vector<int>& cands = xc;
        int best = 0;
        for (size_t i = 1; i < cands.size() && !rc; ++i) {
            set(knobs[ki], cands[i]);
            double ms = 0.0;
            rc = chain_ms(ms);
            if (!rc && ms < best_ms * 0.995) {              // keep a change only for a clear gain
                best_ms = ms;
                best = cands[i];
            }
        }
        set(knobs[ki], best);
        if (!best) {                                       // the default won: record it explicitly
            std::lock_guard<std::mutex> lk(g_mu);
            g_table[dk + "#" + knobs[ki]] = tx.wlog;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_out);
    cudaFree(d_u8);
    if (rc) {
        for (const auto& k : knobs) set(k, 0);
        return rc;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    for (const auto& k : knobs) g_ms[dk + "#" + k] = best_ms;
    if (save_locked() != 0) return fail(FY_EIO, "%s: cannot write the tuning cache %s", what, g_path.c_str());
    return FY_OK;
}
