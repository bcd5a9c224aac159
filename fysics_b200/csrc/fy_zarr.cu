// fy_zarr.cu -- zarr v2 raw-u8 chunk staging into the GPU (zarr_io.c:133-331) and the
// zarr-fed per-tile chain fy_process_chunk (pipeline.c:512-537).
//
// Format (zarr_io.c:1-9, 237-331): <root>/0/.zarray is a flat JSON header (shape, chunks,
// fill_value); <root>/0/cz/cy/cx are raw C-order u8 chunk files holding the chunk's TRUE
// extent, so an edge chunk is smaller than chunk_z*chunk_y*chunk_x. A missing or empty file
// reads as fill, a short file's tail reads as fill, and region voxels outside the volume's
// shape are left untouched in the destination.
//
// Design. The reference maps each chunk file and copies row segments into the caller's
// buffer on the host. Here the host only reads whole chunk files -- one pread each, into
// pinned staging -- and copies them into a device chunk cache; a gather kernel assembles the
// region in device memory (1 B read + 1 B written per region voxel, out of L2 for a tile).
// Chunks stay resident in the cache (LRU within a byte limit, default 4 GiB of the 180 GB),
// so the halo slivers that neighbouring tiles share cross the host link once, and a cached
// chunk is revalidated by stat (inode, size, mtime) on every use. Local roots only: an
// "s3://" root returns 1, as the reference built without FYSICS_S3 does.
//
// Concurrency. Any number of host threads may read through the cache (the reference's pass 2
// calls fy_zarr_read from OpenMP workers). One thread loads a missing chunk while the others
// that need it wait for its copy; a chunk read by a gather stays pinned in the cache until
// that gather has completed on the GPU (per-call events, reaped before any eviction).
#include <errno.h>
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

namespace {

// ------------------------------------------------------------------ .zarray header
// The reference's header grammar (zarr_io.c:115-132): the FIRST occurrence of the quoted key,
// then the first integer after it ('-' or a digit starts it), parsed by strtol. Kept alike so
// that every header the reference accepts yields the same numbers here.
long header_int(const char* s, const char* key, int idx) {
    const char* q = strstr(s, key);
    if (!q) return -1;
    q += strlen(key);
    for (int i = 0;; ++i) {
        while (*q && !(*q >= '0' && *q <= '9') && *q != '-') ++q;
        if (i == idx) break;
        while (*q >= '0' && *q <= '9') ++q;
    }
    return strtol(q, nullptr, 10);
}

// ------------------------------------------------------------------ device chunk cache
struct FileId {
    bool exists = false;
    unsigned long long ino = 0, dev = 0;
    long long size = 0, mtime_ns = 0;
    bool operator==(const FileId& o) const {
        return exists == o.exists && ino == o.ino && dev == o.dev && size == o.size && mtime_ns == o.mtime_ns;
    }
};

FileId file_id(const char* path) {
    FileId f;
    struct stat st;
    if (stat(path, &st) != 0 || !S_ISREG(st.st_mode)) return f;
    f.exists = true;
    f.ino = st.st_ino;
    f.dev = st.st_dev;
    f.size = st.st_size;
    f.mtime_ns = (long long)st.st_mtim.tv_sec * 1000000000LL + st.st_mtim.tv_nsec;
    return f;
}

enum EntryState { kLoading, kReady, kFailed };

struct Entry {
    std::string key;                 // chunk file path
    FileId id;
    unsigned char* d = nullptr;      // device bytes
    size_t cap = 0;                  // device buffer capacity
    size_t len = 0;                  // valid bytes (min(file size, true chunk extent))
    EntryState state = kLoading;
    cudaEvent_t ready = nullptr;     // the H2D copy of the chunk has landed
    int pins = 0;                    // gathers enqueued or about to be enqueued that read it
    bool in_map = true;              // false once replaced by a newer version of the file
    std::list<Entry*>::iterator lru;
};

struct InFlight {                    // one call's gathers: their entries stay pinned until done
    cudaEvent_t done;
    std::vector<Entry*> entries;
};

struct DevCache {
    std::mutex mu;
    std::condition_variable cv;
    std::map<std::string, Entry*> map;
    std::list<Entry*> lru;           // front = most recently used
    std::multimap<size_t, unsigned char*> spare;   // device buffers free for reuse, by capacity
    std::deque<InFlight> inflight;
    std::vector<cudaEvent_t> spare_events;
    size_t bytes = 0;                // device bytes held (entries + spare)
};

constexpr int kMaxDevices = 64;
DevCache* g_cache[kMaxDevices];
std::mutex g_cache_mu;
size_t g_limit = (size_t)4 << 30;
std::atomic<unsigned long long> g_stats[3];   // chunk hits, chunk loads, bytes loaded (all devices)

DevCache& cache_for(int dev) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (!g_cache[dev]) g_cache[dev] = new DevCache();
    return *g_cache[dev];
}

void drop_entry(DevCache& c, Entry* e, bool to_spare) {
    if (e->d) {
        if (to_spare) {
            c.spare.emplace(e->cap, e->d);
        } else {
            cudaFree(e->d);
            c.bytes -= e->cap;
        }
    }
    if (e->ready) cudaEventDestroy(e->ready);
    delete e;
}

// Evict least recently used unpinned entries; stop once `enough()` holds. Called with c.mu held.
template <class F>
void evict_lru(DevCache& c, bool to_spare, F enough) {
    for (auto r = c.lru.rbegin(); r != c.lru.rend() && !enough();) {
        Entry* e = *r;
        if (e->pins == 0 && e->state != kLoading) {
            r = std::list<Entry*>::reverse_iterator(c.lru.erase(std::next(r).base()));
            c.map.erase(e->key);
            drop_entry(c, e, to_spare);
        } else {
            ++r;
        }
    }
}

// Unpin the entries of gathers that have completed; `block` waits for the oldest first. The
// limit is soft (reads in progress may pin more chunks than it holds), so afterwards the
// cache is trimmed back to it. Called with c.mu held.
void reap(DevCache& c, bool block) {
    while (!c.inflight.empty()) {
        InFlight& f = c.inflight.front();
        if (block) {
            cudaEventSynchronize(f.done);
            block = false;
        } else if (cudaEventQuery(f.done) != cudaSuccess) {
            cudaGetLastError();
            break;
        }
        for (Entry* e : f.entries)
            if (--e->pins == 0 && !e->in_map) drop_entry(c, e, true);   // a replaced version
        c.spare_events.push_back(f.done);
        c.inflight.pop_front();
    }
    while (c.bytes > g_limit && !c.spare.empty()) {
        auto s = c.spare.begin();
        cudaFree(s->second);
        c.bytes -= s->first;
        c.spare.erase(s);
    }
    if (c.bytes > g_limit) evict_lru(c, false, [&] { return c.bytes <= g_limit; });
}

// A device buffer of at least `need` bytes for a new entry: a spare one, a new allocation
// within the limit, the buffer of the least recently used unpinned entry, or -- when every
// cached chunk is pinned by reads in progress, even after waiting once for the oldest
// gather -- a new allocation past the limit (trimmed back by reap). Called with c.mu held.
unsigned char* take_buffer(DevCache& c, size_t need, size_t alloc, size_t& cap, cudaError_t& err) {
    err = cudaSuccess;
    auto fits = [&] { return c.spare.lower_bound(need) != c.spare.end(); };
    for (int round = 0;; ++round) {
        auto it = c.spare.lower_bound(need);
        if (it != c.spare.end()) {
            unsigned char* p = it->second;
            cap = it->first;
            c.spare.erase(it);
            return p;
        }
        if (c.bytes + alloc <= g_limit) break;
        evict_lru(c, true, fits);
        if (fits()) continue;
        while (!c.spare.empty() && c.bytes + alloc > g_limit) {      // spares too small for this size
            auto s = c.spare.begin();
            cudaFree(s->second);
            c.bytes -= s->first;
            c.spare.erase(s);
        }
        if (c.bytes + alloc <= g_limit) break;
        if (round > 0 || c.inflight.empty()) break;
        reap(c, true);                                              // wait for the oldest gather, once
    }
    void* p = nullptr;                                              // full chunk size: interchangeable
    if ((err = cudaMalloc(&p, alloc)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    c.bytes += alloc;
    cap = alloc;
    return (unsigned char*)p;
}

// ------------------------------------------------------------------ gather kernel
struct ChunkRef {
    const unsigned char* p;          // device bytes, or null: absent chunk (fill)
    unsigned long long len;          // valid bytes
    int ey, ex;                      // true extent (y, x) of the chunk
};
constexpr int kMaxRefs = 32;

struct GatherArgs {
    ChunkRef ref[kMaxRefs];          // chunks (cz, cy, cx) of the launch's box, z-major
    long long c0, c1, c2;            // chunk dims
    long long gz0, gy0, gx0;         // global origin of the destination region
    long long dy, dx;                // destination row / plane pitch (region dims)
    long long bz0, by0, bx0;         // this launch's box (global, inside the volume)
    int nbz, nby, nbx;               // box dims
    int kz0, ky0, kx0;               // chunk coordinates of ref[0]
    int nky, nkx;                    // chunk counts of the box in y and x
    unsigned char fill;
};

// One thread writes 16 consecutive destination bytes of one box row. Every written voxel
// takes byte (lz*ey + ly)*ex + lx of its chunk when that is below the chunk's valid length,
// else the fill value (zarr_io.c:311-320).
__global__ void k_zarr_gather(const GatherArgs a, unsigned char* __restrict__ out) {
    const long long segs = (a.nbx + 15) / 16;
    const long long total = (long long)a.nbz * a.nby * segs;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long seg = i % segs, row = i / segs;
        const long long gz = a.bz0 + row / a.nby, gy = a.by0 + row % a.nby;
        const long long cz = gz / a.c0, cy = gy / a.c1;
        const long long lz = gz - cz * a.c0, ly = gy - cy * a.c1;
        unsigned char* dst = out + ((gz - a.gz0) * a.dy + (gy - a.gy0)) * a.dx - a.gx0;
        const long long x0 = a.bx0 + seg * 16, x1 = min(x0 + 16, a.bx0 + a.nbx);
        long long cx = x0 / a.c2;
        long long lx = x0 - cx * a.c2;
        const ChunkRef* r = &a.ref[((cz - a.kz0) * a.nky + (cy - a.ky0)) * a.nkx + (cx - a.kx0)];
        long long off = (lz * r->ey + ly) * r->ex + lx;
        for (long long x = x0; x < x1; ++x) {
            if (lx == a.c2) {                                      // next chunk along x
                ++cx;
                lx = 0;
                ++r;
                off = (lz * r->ey + ly) * r->ex;
            }
            dst[x] = (r->p && (unsigned long long)off < r->len) ? r->p[off] : a.fill;
            ++lx;
            ++off;
        }
    }
}

// ------------------------------------------------------------------ per-thread staging
struct ZarrWs {
    fy::HostBuf stage[2];            // chunk file bytes, double-buffered against their H2D
    cudaEvent_t staged[2] = {nullptr, nullptr};
    bool staged_pending[2] = {false, false};
    fy::DevBuf region, tile_out;     // fy_zarr_read / fy_process_chunk device buffers
    fy::HostBuf hout;                // pageable destinations go through this
};
thread_local ZarrWs zws;

inline long long ceil_div(long long a, long long b) { return (a + b - 1) / b; }

// Read `len` bytes of a chunk file into pinned memory. Returns the bytes read (0 for a file
// that vanished), or -1 on an I/O error.
long long read_file(const char* path, void* dst, size_t len) {
    const int fd = open(path, O_RDONLY);
    if (fd < 0) return errno == ENOENT ? 0 : -1;
    size_t got = 0;
    while (got < len) {
        const ssize_t k = pread(fd, (char*)dst + got, len - got, (off_t)got);
        if (k < 0) {
            if (errno == EINTR) continue;
            close(fd);
            return -1;
        }
        if (k == 0) break;
        got += (size_t)k;
    }
    close(fd);
    return (long long)got;
}

struct Region {
    long long z0, y0, x0, dz, dy, dx;
};

// Stage the chunks of `reg` and gather it into d_out (region layout dz*dy*dx) on `st`.
int stage_and_gather(const fy_zarr* z, const Region& reg, unsigned char* d_out, cudaStream_t st, int dev,
                     const char* what) {
    const long long C0 = z->chunk[0], C1 = z->chunk[1], C2 = z->chunk[2];
    const long long S0 = z->shape[0], S1 = z->shape[1], S2 = z->shape[2];
    // the part of the region inside the volume; the rest is left untouched
    const long long bz0 = reg.z0, by0 = reg.y0, bx0 = reg.x0;
    const long long bz1 = std::min(reg.z0 + reg.dz, S0), by1 = std::min(reg.y0 + reg.dy, S1),
                    bx1 = std::min(reg.x0 + reg.dx, S2);
    if (bz1 <= bz0 || by1 <= by0 || bx1 <= bx0) return FY_OK;
    const long long kz0 = bz0 / C0, ky0 = by0 / C1, kx0 = bx0 / C2;
    const long long nkz = (bz1 - 1) / C0 - kz0 + 1, nky = (by1 - 1) / C1 - ky0 + 1, nkx = (bx1 - 1) / C2 - kx0 + 1;
    const long long nk = nkz * nky * nkx;
    if (nk > (1LL << 24)) return fail(FY_EUNSUPPORTED, "%s: region spans %lld chunks", what, nk);

    // 1. identify every chunk file (outside the lock)
    struct Want {
        std::string path;
        FileId id;
        long long extent;            // true extent of the chunk, bytes
        int ey, ex;
        Entry* e = nullptr;
        bool mine = false;
    };
    std::vector<Want> want((size_t)nk);
    char path[2200];
    for (long long i = 0; i < nk; ++i) {
        const long long cz = kz0 + i / (nky * nkx), cy = ky0 + (i / nkx) % nky, cx = kx0 + i % nkx;
        const long long ez = std::min(S0 - cz * C0, C0), ey = std::min(S1 - cy * C1, C1), ex = std::min(S2 - cx * C2, C2);
        snprintf(path, sizeof path, "%s/0/%lld/%lld/%lld", z->root, cz, cy, cx);
        Want& w = want[(size_t)i];
        w.path = path;
        w.id = file_id(path);
        w.extent = ez * ey * ex;
        w.ey = (int)ey;
        w.ex = (int)ex;
    }

    // 2. look the chunks up; claim the ones to load
    DevCache& c = cache_for(dev);
    cudaError_t err = cudaSuccess;
    {
        std::unique_lock<std::mutex> lk(c.mu);
        reap(c, false);
        for (Want& w : want) {
            if (!w.id.exists || w.id.size <= 0) continue;                 // absent: fill
            auto it = c.map.find(w.path);
            if (it != c.map.end() && it->second->id == w.id && it->second->state != kFailed) {
                Entry* e = it->second;
                ++e->pins;
                c.lru.splice(c.lru.begin(), c.lru, e->lru);
                w.e = e;
                ++g_stats[0];
                continue;
            }
            if (it != c.map.end()) {                                     // changed or failed: replace
                Entry* old = it->second;
                c.map.erase(it);
                c.lru.erase(old->lru);
                old->in_map = false;
                if (old->pins == 0 && old->state != kLoading) drop_entry(c, old, true);
            }
            const size_t need = (size_t)std::min<long long>(w.id.size, w.extent);
            size_t cap = 0;
            unsigned char* buf = take_buffer(c, std::max<size_t>(need, 1), (size_t)(C0 * C1 * C2), cap, err);
            if (!buf) break;
            Entry* e = new Entry();
            e->key = w.path;
            e->id = w.id;
            e->d = buf;
            e->cap = cap;
            e->len = need;
            e->pins = 1;
            if ((err = cudaEventCreateWithFlags(&e->ready, cudaEventDisableTiming)) != cudaSuccess) {
                c.spare.emplace(cap, buf);
                delete e;
                break;
            }
            c.lru.push_front(e);
            e->lru = c.lru.begin();
            c.map.emplace(w.path, e);
            w.e = e;
            w.mine = true;
        }
    }
    auto unpin_all = [&]() {
        std::lock_guard<std::mutex> lk(c.mu);
        for (Want& w : want)
            if (w.e) {
                Entry* e = w.e;
                if (w.mine && e->state == kLoading) e->state = kFailed;
                if (--e->pins == 0 && !e->in_map) drop_entry(c, e, true);
            }
        c.cv.notify_all();
    };
    if (err != cudaSuccess) {
        unpin_all();
        return err == cudaErrorMemoryAllocation
                   ? fail(FY_ENOMEM, "%s: no device memory for the region's chunks", what)
                   : fail_cuda(err, what);
    }

    // 3. load the claimed chunks: pread into pinned staging, H2D on `st`
    ZarrWs& ws = zws;
    int k = 0;
    int rc = FY_OK;
    for (Want& w : want) {
        if (!w.mine) continue;
        Entry* e = w.e;
        const int b = k++ & 1;
        if (!ws.staged[b] && (err = cudaEventCreateWithFlags(&ws.staged[b], cudaEventDisableTiming)) != cudaSuccess) {
            rc = fail_cuda(err, what);
            break;
        }
        if (ws.staged_pending[b]) cudaEventSynchronize(ws.staged[b]);   // its previous H2D has read it
        if ((err = ws.stage[b].ensure(std::max<size_t>(e->len, 1))) != cudaSuccess) { rc = fail_cuda(err, what); break; }
        const long long got = read_file(w.path.c_str(), ws.stage[b].p, e->len);
        if (got < 0) { rc = fail(FY_EIO, "%s: cannot read %s", what, w.path.c_str()); break; }
        e->len = (size_t)got;                                  // shorter than stat said: tail is fill
        if (got > 0 && (err = cudaMemcpyAsync(e->d, ws.stage[b].p, (size_t)got, cudaMemcpyHostToDevice, st)) !=
                           cudaSuccess) {
            rc = fail_cuda(err, what);
            break;
        }
        if ((err = cudaEventRecord(ws.staged[b], st)) != cudaSuccess || (err = cudaEventRecord(e->ready, st)) != cudaSuccess) {
            rc = fail_cuda(err, what);
            break;
        }
        ws.staged_pending[b] = true;
        g_stats[1]++;
        g_stats[2] += (unsigned long long)got;
        {
            std::lock_guard<std::mutex> lk(c.mu);
            e->state = kReady;
        }
        c.cv.notify_all();
    }
    if (rc) {
        unpin_all();
        return rc;
    }
    // 4. wait for chunks that other threads are loading; order this stream after every copy
    for (Want& w : want) {
        if (!w.e || w.mine) continue;
        {
            std::unique_lock<std::mutex> lk(c.mu);
            c.cv.wait(lk, [&] { return w.e->state != kLoading; });
            if (w.e->state == kFailed) rc = fail(FY_EIO, "%s: loading %s failed in another thread", what, w.path.c_str());
        }
        if (rc) break;
        if ((err = cudaStreamWaitEvent(st, w.e->ready, 0)) != cudaSuccess) { rc = fail_cuda(err, what); break; }
    }
    if (rc) {
        unpin_all();
        return rc;
    }

    // 5. gather: one launch per group of at most kMaxRefs chunks (z slabs, else rows, else runs)
    GatherArgs a{};
    a.c0 = C0; a.c1 = C1; a.c2 = C2;
    a.gz0 = reg.z0; a.gy0 = reg.y0; a.gx0 = reg.x0;
    a.dy = reg.dy; a.dx = reg.dx;
    a.fill = z->fill;
    auto launch = [&](long long qz0, long long qz1, long long qy0, long long qy1, long long qx0, long long qx1) -> int {
        // chunk sub-box [qz0,qz1) x [qy0,qy1) x [qx0,qx1) in chunk coordinates
        a.kz0 = (int)qz0; a.ky0 = (int)qy0; a.kx0 = (int)qx0;
        a.nky = (int)(qy1 - qy0); a.nkx = (int)(qx1 - qx0);
        int j = 0;
        for (long long cz = qz0; cz < qz1; ++cz)
            for (long long cy = qy0; cy < qy1; ++cy)
                for (long long cx = qx0; cx < qx1; ++cx) {
                    const Want& w = want[(size_t)(((cz - kz0) * nky + (cy - ky0)) * nkx + (cx - kx0))];
                    ChunkRef& r = a.ref[j++];
                    r.p = w.e ? w.e->d : nullptr;
                    r.len = w.e ? w.e->len : 0;
                    r.ey = w.ey;
                    r.ex = w.ex;
                }
        a.bz0 = std::max(bz0, qz0 * C0); a.by0 = std::max(by0, qy0 * C1); a.bx0 = std::max(bx0, qx0 * C2);
        a.nbz = (int)(std::min(bz1, qz1 * C0) - a.bz0);
        a.nby = (int)(std::min(by1, qy1 * C1) - a.by0);
        a.nbx = (int)(std::min(bx1, qx1 * C2) - a.bx0);
        const long long work = (long long)a.nbz * a.nby * ((a.nbx + 15) / 16);
        const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(ceil_div(work, 256), 148LL * 16));
        k_zarr_gather<<<grid, 256, 0, st>>>(a, d_out);
        cudaError_t e = cudaGetLastError();
        fy::count_launch();
        return e == cudaSuccess ? FY_OK : fail_cuda(e, what);
    };
    const long long kz1 = kz0 + nkz, ky1 = ky0 + nky, kx1 = kx0 + nkx;
    if (nk <= kMaxRefs) {
        rc = launch(kz0, kz1, ky0, ky1, kx0, kx1);
    } else if (nky * nkx <= kMaxRefs) {
        const long long per = kMaxRefs / (nky * nkx);
        for (long long q = kz0; q < kz1 && !rc; q += per) rc = launch(q, std::min(q + per, kz1), ky0, ky1, kx0, kx1);
    } else if (nkx <= kMaxRefs) {
        const long long per = kMaxRefs / nkx;
        for (long long qz = kz0; qz < kz1 && !rc; ++qz)
            for (long long q = ky0; q < ky1 && !rc; q += per) rc = launch(qz, qz + 1, q, std::min(q + per, ky1), kx0, kx1);
    } else {
        for (long long qz = kz0; qz < kz1 && !rc; ++qz)
            for (long long qy = ky0; qy < ky1 && !rc; ++qy)
                for (long long q = kx0; q < kx1 && !rc; q += kMaxRefs)
                    rc = launch(qz, qz + 1, qy, qy + 1, q, std::min<long long>(q + kMaxRefs, kx1));
    }

    // 6. keep the chunks pinned until the gathers are done
    std::lock_guard<std::mutex> lk(c.mu);
    cudaEvent_t done = nullptr;
    if (!c.spare_events.empty()) {
        done = c.spare_events.back();
        c.spare_events.pop_back();
    } else if ((err = cudaEventCreateWithFlags(&done, cudaEventDisableTiming)) != cudaSuccess) {
        cudaStreamSynchronize(st);               // no event: wait instead, then unpin
        for (Want& w : want)
            if (w.e) --w.e->pins;
        return rc ? rc : fail_cuda(err, what);
    }
    cudaEventRecord(done, st);
    InFlight f{done, {}};
    for (Want& w : want)
        if (w.e) f.entries.push_back(w.e);
    c.inflight.push_back(std::move(f));
    return rc;
}

int check_zarr(const fy_zarr* z, long z0, long y0, long x0, long dz, long dy, long dx, const void* out,
               const char* what) {
    if (!z || !out) return fail(FY_EINVAL, "%s: null pointer", what);
    if (strncmp(z->root, "s3://", 5) == 0)
        return fail(FY_EUNSUPPORTED, "%s: S3 roots are not supported (local zarr only)", what);
    if (z->chunk[0] <= 0 || z->chunk[1] <= 0 || z->chunk[2] <= 0 || z->shape[0] <= 0)
        return fail(FY_EINVAL, "%s: bad zarr header", what);
    if (z0 < 0 || y0 < 0 || x0 < 0 || dz < 0 || dy < 0 || dx < 0)
        return fail(FY_EINVAL, "%s: negative region origin or size", what);
    return FY_OK;
}

}  // namespace

extern "C" int fy_zarr_open(fy_zarr* z, const char* root) {
    fy::enter();
    if (!z || !root) return fail(1, "fy_zarr_open: null pointer");
    memset(z, 0, sizeof *z);
    snprintf(z->root, sizeof z->root, "%s", root);
    if (strncmp(root, "s3://", 5) == 0)
        return fail(1, "fy_zarr_open: %s: S3 roots are not supported (local zarr only)", root);
    char path[2048];
    snprintf(path, sizeof path, "%s/0/.zarray", root);
    FILE* f = fopen(path, "rb");
    if (!f) return fail(1, "fy_zarr_open: no %s", path);
    char buf[4096];
    const size_t n = fread(buf, 1, sizeof buf - 1, f);
    fclose(f);
    buf[n] = 0;
    for (int i = 0; i < 3; ++i) {
        z->shape[i] = header_int(buf, "\"shape\"", i);
        z->chunk[i] = header_int(buf, "\"chunks\"", i);
    }
    const long fv = header_int(buf, "\"fill_value\"", 0);
    z->fill = (unsigned char)(fv > 0 ? fv : 0);
    if (z->shape[0] <= 0 || z->chunk[0] <= 0) return fail(1, "fy_zarr_open: bad header in %s", path);
    return 0;
}

extern "C" int fy_gpu_zarr_read(const fy_zarr* z, long z0, long y0, long x0, long dz, long dy, long dx,
                                unsigned char* d_out, void* stream) {
    fy::enter();
    const char* what = "fy_gpu_zarr_read";
    int rc = check_zarr(z, z0, y0, x0, dz, dy, dx, d_out, what);
    if (rc) return rc;
    if ((rc = fy::ensure_ctx())) return rc;
    return stage_and_gather(z, Region{z0, y0, x0, dz, dy, dx}, d_out, (cudaStream_t)stream, ctx().dev, what);
}

extern "C" int fy_zarr_read(const fy_zarr* z, long z0, long y0, long x0, long dz, long dy, long dx,
                            unsigned char* out) {
    fy::enter();
    const char* what = "fy_zarr_read";
    int rc = check_zarr(z, z0, y0, x0, dz, dy, dx, out, what);
    if (rc) return rc;
    if ((rc = fy::ensure_ctx())) return rc;
    const long long vz = std::max<long long>(0, std::min<long long>(dz, z->shape[0] - z0));
    const long long vy = std::max<long long>(0, std::min<long long>(dy, z->shape[1] - y0));
    const long long vx = std::max<long long>(0, std::min<long long>(dx, z->shape[2] - x0));
    if (!vz || !vy || !vx) return FY_OK;                             // nothing inside the volume
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    ZarrWs& ws = zws;
    cudaError_t e;
    // gather the in-volume box densely, then place its rows into the caller's buffer
    const size_t vn = (size_t)(vz * vy * vx);
    if ((e = ws.region.ensure(vn)) != cudaSuccess) return fail_cuda(e, what);
    rc = stage_and_gather(z, Region{z0, y0, x0, vz, vy, vx}, ws.region.as<unsigned char>(), st, c.dev, what);
    if (rc) return rc;
    const bool dense = vz == dz && vy == dy && vx == dx;
    void* dst = out;
    if (!dense || !fy::is_pinned(out)) {
        if ((e = ws.hout.ensure(vn)) != cudaSuccess) return fail_cuda(e, what);
        dst = ws.hout.p;
    }
    if ((e = cudaMemcpyAsync(dst, ws.region.p, vn, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return fail_cuda(e, what);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
    if (dst != out) {
        if (dense) {
            memcpy(out, dst, vn);
        } else {
            for (long long zz = 0; zz < vz; ++zz)
                for (long long yy = 0; yy < vy; ++yy)
                    memcpy(out + ((size_t)zz * dy + yy) * dx, (const unsigned char*)dst + ((size_t)zz * vy + yy) * vx,
                           (size_t)vx);
        }
    }
    return FY_OK;
}

extern "C" int fy_process_chunk(const fy_zarr* zin, const fy_pipeline_cfg* cfg, long z0, long y0, long x0, int tile,
                                unsigned char* out, int* out_tz, int* out_ty, int* out_tx, int* all_air) {
    fy::enter();
    const char* what = "fy_process_chunk";
    if (!zin || !cfg || !out) return fail(FY_EINVAL, "%s: null pointer", what);
    // the reference's tile and halo geometry (pipeline.c:521-527)
    const long Z = zin->shape[0], Y = zin->shape[1], X = zin->shape[2];
    const long halo = cfg->halo > 0 ? cfg->halo : 8;
    const long tz = std::min<long>(tile, Z - z0), ty = std::min<long>(tile, Y - y0), tx = std::min<long>(tile, X - x0);
    if (out_tz) *out_tz = (int)tz;
    if (out_ty) *out_ty = (int)ty;
    if (out_tx) *out_tx = (int)tx;
    const long rz0 = std::max(0L, z0 - halo), ry0 = std::max(0L, y0 - halo), rx0 = std::max(0L, x0 - halo);
    const long rz1 = std::min(Z, z0 + tz + halo), ry1 = std::min(Y, y0 + ty + halo), rx1 = std::min(X, x0 + tx + halo);
    const long hz = rz1 - rz0, hy = ry1 - ry0, hx = rx1 - rx0;
    if (hz < 1 || hy < 1 || hx < 1 || tz < 1 || ty < 1 || tx < 1)
        return fail(FY_EINVAL, "%s: tile (%ld,%ld,%ld) of %d outside the volume", what, z0, y0, x0, tile);
    int rc = check_zarr(zin, rz0, ry0, rx0, hz, hy, hx, out, what);
    if (rc) return rc;
    if ((rc = fy::ensure_ctx())) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    ZarrWs& ws = zws;
    const size_t hn = (size_t)hz * hy * hx, tn = (size_t)tz * ty * tx;
    cudaError_t e;
    if ((e = ws.region.ensure(hn)) != cudaSuccess || (e = ws.tile_out.ensure(tn)) != cudaSuccess)
        return fail_cuda(e, what);
    if ((rc = stage_and_gather(zin, Region{rz0, ry0, rx0, hz, hy, hx}, ws.region.as<unsigned char>(), st, c.dev, what)))
        return rc;
    int air = 1;
    if ((rc = fy_gpu_process_buffer(cfg, ws.region.as<unsigned char>(), rz0, ry0, rx0, hz, hy, hx, z0, y0, x0, tz, ty,
                                    tx, Y, X, ws.tile_out.as<unsigned char>(), &air, st)))
        return rc;
    const bool pin_out = fy::is_pinned(out);
    void* dst = out;
    if (!pin_out) {
        if ((e = ws.hout.ensure(tn)) != cudaSuccess) return fail_cuda(e, what);
        dst = ws.hout.p;
    }
    if ((e = cudaMemcpyAsync(dst, ws.tile_out.p, tn, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return fail_cuda(e, what);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
    if (!pin_out) memcpy(out, dst, tn);
    if (all_air) *all_air = air;
    return FY_OK;
}

extern "C" int fy_gpu_zarr_cache_limit(size_t bytes) {
    fy::enter();
    if (bytes < ((size_t)16 << 20)) return fail(FY_EINVAL, "fy_gpu_zarr_cache_limit: below 16 MiB");
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_limit = bytes;
    return FY_OK;
}

extern "C" void fy_gpu_zarr_cache_stats(unsigned long long* hits, unsigned long long* loads,
                                        unsigned long long* bytes_loaded) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (hits) *hits = g_stats[0];
    if (loads) *loads = g_stats[1];
    if (bytes_loaded) *bytes_loaded = g_stats[2];
}
