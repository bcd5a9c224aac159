// fy_server.cu -- the request loop: continuous batching of restoration requests on one GPU.
//
// A viewer or exporter issues cubes as they are needed, from many threads, with sizes and
// per-volume metadata that vary request by request. The server keeps a FIFO of submitted
// requests and a pool of worker threads. Each worker owns CUDA streams and its own
// device workspaces (the per-thread context of the C-ABI), so the chains of different
// requests run concurrently on the GPU, and one request's host<->device copies overlap
// other requests' kernels. A request is admitted when a worker is free and the estimated
// device footprint of everything in flight stays within the HBM budget. General workers take
// the head of the queue, which is never overtaken by them, so no request starves; a few
// reserved workers take the first small request instead, so small cubes do not wait for a
// worker behind large ones. All host<->device copies go through one scheduler per link
// direction that serves the request with the fewest bytes left first (Link below), so a small
// result never queues behind a large one on the copy engine. Each request's result is
// the same as the single-cube fy_gpu_restore_u8 call on its own: the kernels are
// deterministic and a worker's workspaces are private to the request it runs.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

extern "C" int fy_gpu_restore_u8(const unsigned char* d_u8, float* d_out, int nz, int ny, int nx, double f32_min,
                                 double f32_max, const fy_physics* p, const fy_restore_cfg* cfg, void* stream);

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Ticket {
    fy_request req;
    long long id = 0;
    size_t footprint = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    float h2d_ms = 0, chain_ms = 0, d2h_ms = 0;   // copies: host clock incl. link wait; chain: CUDA events
    int status = -1;          // -1 pending, else the chain's status
    bool done = false;
};

// Worker-owned device and pinned buffers (grow-only) and two streams: requests up to
// priority_voxels run on the high-priority one, so the GPU's block scheduler serves their
// kernels ahead of a large request's.
struct WorkerBufs {
    fy::DevBuf d_in, d_out;
    fy::HostBuf h_in, h_out;
    cudaStream_t hi = nullptr, lo = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};   // chain start, chain end
};

// One direction of the host<->device link, shared by all workers. A copy engine runs one
// direction's copies in the order they were issued, so a small request's result would wait
// behind every queued chunk of a large one. Instead one scheduler thread per direction
// issues the copies chunk by chunk on its own stream, keeps at most kInflight chunks queued
// on the engine (enough to keep the link busy), and always issues next from the job with
// the fewest bytes left (ties: the earlier job). A small request then waits for at most the
// chunks already queued.
constexpr size_t kLinkChunk = (size_t)8 << 20;
constexpr int kInflight = 2;

struct LinkJob {
    char* dst;
    const char* src;
    size_t bytes, issued = 0, done = 0;
    long long seq = 0;
    cudaError_t err = cudaSuccess;
    bool finished = false;
};

class Link {
  public:
    // Starts the scheduler thread on `device`; returns once its stream and events exist.
    cudaError_t start(int device, cudaMemcpyKind kind) {
        device_ = device;
        kind_ = kind;
        th_ = std::thread([this] { run(); });
        std::unique_lock<std::mutex> lk(mu_);
        cv_done_.wait(lk, [&] { return ready_; });
        if (init_err_ != cudaSuccess) {
            lk.unlock();
            th_.join();
        }
        return init_err_;
    }
    // Copies bytes and returns when they have landed (or with the first error).
    cudaError_t copy(void* dst, const void* src, size_t bytes) {
        if (!bytes) return cudaSuccess;
        LinkJob job;
        job.dst = (char*)dst;
        job.src = (const char*)src;
        job.bytes = bytes;
        std::unique_lock<std::mutex> lk(mu_);
        job.seq = seq_++;
        pending_.push_back(&job);
        cv_.notify_one();
        cv_done_.wait(lk, [&] { return job.finished; });
        return job.err;
    }
    void stop() {
        if (th_.joinable()) {
            {
                std::lock_guard<std::mutex> lk(mu_);
                stopping_ = true;
            }
            cv_.notify_one();
            th_.join();
        }
        release();
    }

  private:
    struct Slot {
        LinkJob* job;
        size_t len;
    };
    void release() {
        for (cudaEvent_t& ev : ev_)
            if (ev) { cudaEventDestroy(ev); ev = nullptr; }
        if (st_) { cudaStreamDestroy(st_); st_ = nullptr; }
    }
    // Caller holds mu_. Completed bytes of a job; the last ones finish it.
    void complete(LinkJob* j, size_t len, cudaError_t e) {
        if (e != cudaSuccess && j->err == cudaSuccess) j->err = e;
        j->done += len;
        if (j->done == j->bytes) {
            j->finished = true;
            cv_done_.notify_all();
        }
    }
    void run() {
        cudaError_t e0 = cudaSetDevice(device_);
        if (e0 == cudaSuccess) e0 = cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking);
        for (int i = 0; i < kInflight && e0 == cudaSuccess; ++i)
            e0 = cudaEventCreateWithFlags(&ev_[i], cudaEventDisableTiming);
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (e0 != cudaSuccess) { cudaGetLastError(); release(); }
            init_err_ = e0;
            ready_ = true;
            cv_done_.notify_all();
        }
        if (e0 != cudaSuccess) return;
        Slot slot[kInflight];
        int head = 0, n = 0;
        for (;;) {
            LinkJob* pick = nullptr;
            size_t off = 0, len = 0;
            {
                std::unique_lock<std::mutex> lk(mu_);
                if (n == 0) cv_.wait(lk, [&] { return stopping_ || !pending_.empty(); });
                if (n == 0 && pending_.empty()) break;           // stopping, nothing left
                if (n < kInflight && !pending_.empty()) {
                    auto best = pending_.begin();
                    for (auto it = pending_.begin(); it != pending_.end(); ++it) {
                        const size_t left = (*it)->bytes - (*it)->issued, bl = (*best)->bytes - (*best)->issued;
                        if (left < bl || (left == bl && (*it)->seq < (*best)->seq)) best = it;
                    }
                    pick = *best;
                    off = pick->issued;
                    len = pick->bytes - off < kLinkChunk ? pick->bytes - off : kLinkChunk;
                    pick->issued += len;
                    if (pick->issued == pick->bytes) pending_.erase(best);
                }
            }
            if (pick) {
                const int k = (head + n) % kInflight;
                cudaError_t e = cudaMemcpyAsync(pick->dst + off, pick->src + off, len, kind_, st_);
                if (e == cudaSuccess) e = cudaEventRecord(ev_[k], st_);
                if (e != cudaSuccess) {                            // drop the job's unissued rest
                    cudaGetLastError();
                    std::lock_guard<std::mutex> lk(mu_);
                    const size_t rest = pick->bytes - pick->issued;
                    if (rest) {
                        pick->issued = pick->bytes;
                        pending_.erase(std::find(pending_.begin(), pending_.end(), pick));
                    }
                    complete(pick, len + rest, e);
                    continue;
                }
                slot[k] = Slot{pick, len};
                ++n;
                continue;                                          // fill the next slot first
            }
            const cudaError_t e = cudaEventSynchronize(ev_[head]);   // oldest chunk in flight
            if (e != cudaSuccess) cudaGetLastError();
            const Slot sl = slot[head];
            head = (head + 1) % kInflight;
            --n;
            std::lock_guard<std::mutex> lk(mu_);
            complete(sl.job, sl.len, e);
        }
    }

    int device_ = 0;
    cudaMemcpyKind kind_ = cudaMemcpyHostToDevice;
    cudaStream_t st_ = nullptr;
    cudaEvent_t ev_[kInflight] = {};
    std::mutex mu_;
    std::condition_variable cv_, cv_done_;
    std::vector<LinkJob*> pending_;
    long long seq_ = 0;
    bool stopping_ = false, ready_ = false;
    cudaError_t init_err_ = cudaSuccess;
    std::thread th_;
};

}  // namespace

struct fy_server {
    fy_server_cfg cfg{};
    Link h2d, d2h;                 // the two directions of the host<->device link
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Ticket*> queue;
    std::unordered_map<long long, Ticket*> tickets;
    std::vector<std::thread> workers;
    size_t inflight_bytes = 0;
    int inflight = 0;
    bool stop = false;
    long long next_id = 1;
    // completed-request statistics
    std::vector<double> lat_ms;
    double voxels = 0;
    double first_start = 0, last_done = 0;
    int init_status = 0;
};

namespace {

// Device bytes a request holds while it runs: u8 in, f32 out, the deconvolved volume, the
// half spectrum (<= 8 B per padded complex over half the x axis), the noise statistics
// (9 B per voxel) and the guided filter's (mean, var) pairs (8 B per voxel); tables are small.
size_t footprint_of(const fy_request& r) {
    const size_t n = (size_t)r.nz * r.ny * r.nx;
    const size_t pz = (size_t)fy_next_fft_size(r.nz), py = (size_t)fy_next_fft_size(r.ny);
    const size_t px = (size_t)fy_next_fft_size(r.nx);
    const size_t spec = r.nz * py * ((px / 2 + 1 + 15) & ~(size_t)15) * 8;
    (void)pz;
    return n + 4 * n + 4 * n + spec + 9 * n + 8 * n + (8u << 20);
}

void run_one(fy_server* s, Ticket* t, WorkerBufs& wb) {
    const fy_request& r = t->req;
    const size_t n = (size_t)r.nz * r.ny * r.nx;
    cudaStream_t st = n <= s->cfg.priority_voxels ? wb.hi : wb.lo;
    cudaError_t e;
    int rc = FY_OK;
    const bool in_pinned = fy::is_pinned(r.u8), out_pinned = fy::is_pinned(r.out);
    const bool timed = wb.ev[1] != nullptr;
    if (fy::is_device(r.u8) && fy::is_device(r.out)) {   // device-resident request: no link copies
        if (timed) cudaEventRecord(wb.ev[0], st);
        rc = fy_gpu_restore_u8(r.u8, r.out, r.nz, r.ny, r.nx, r.f32_min, r.f32_max, &r.phys, &r.cfg, st);
        if (!rc && timed) cudaEventRecord(wb.ev[1], st);
        if (!rc && (e = cudaStreamSynchronize(st)) != cudaSuccess) rc = fail_cuda(e, "fy_server");
        if (!rc && timed && cudaEventElapsedTime(&t->chain_ms, wb.ev[0], wb.ev[1]) != cudaSuccess) cudaGetLastError();
    } else do {
        if ((e = wb.d_in.ensure(n)) != cudaSuccess || (e = wb.d_out.ensure(4 * n)) != cudaSuccess) {
            rc = fail_cuda(e, "fy_server");
            break;
        }
        const unsigned char* src = r.u8;
        if (!in_pinned) {                        // stage pageable input through pinned memory
            if ((e = wb.h_in.ensure(n)) != cudaSuccess) { rc = fail_cuda(e, "fy_server"); break; }
            memcpy(wb.h_in.p, r.u8, n);
            src = (const unsigned char*)wb.h_in.p;
        }
        double t0 = now_ms();
        if ((e = s->h2d.copy(wb.d_in.p, src, n)) != cudaSuccess) {
            rc = fail_cuda(e, "fy_server");
            break;
        }
        t->h2d_ms = (float)(now_ms() - t0);
        if (timed) cudaEventRecord(wb.ev[0], st);
        rc = fy_gpu_restore_u8(wb.d_in.as<unsigned char>(), wb.d_out.as<float>(), r.nz, r.ny, r.nx, r.f32_min,
                               r.f32_max, &r.phys, &r.cfg, st);
        if (rc) break;
        if (timed) cudaEventRecord(wb.ev[1], st);
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) {
            rc = fail_cuda(e, "fy_server");
            break;
        }
        if (timed && cudaEventElapsedTime(&t->chain_ms, wb.ev[0], wb.ev[1]) != cudaSuccess) cudaGetLastError();
        float* dst = r.out;
        if (!out_pinned) {
            if ((e = wb.h_out.ensure(4 * n)) != cudaSuccess) { rc = fail_cuda(e, "fy_server"); break; }
            dst = (float*)wb.h_out.p;
        }
        t0 = now_ms();
        if ((e = s->d2h.copy(dst, wb.d_out.p, 4 * n)) != cudaSuccess) {
            rc = fail_cuda(e, "fy_server");
            break;
        }
        t->d2h_ms = (float)(now_ms() - t0);
        if (!out_pinned) memcpy(r.out, wb.h_out.p, 4 * n);
    } while (false);
    std::lock_guard<std::mutex> lk(s->mu);
    t->status = rc;
    t->t_done = now_ms();
    t->done = true;
    s->inflight_bytes -= t->footprint;
    s->inflight -= 1;
    if (rc == FY_OK) {
        s->lat_ms.push_back(t->t_done - t->t_submit);
        s->voxels += (double)n;
        s->last_done = t->t_done;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
}

void worker_main(fy_server* s, int idx) {
    const int rc0 = fy_gpu_init(s->cfg.device);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (rc0 && !s->init_status) s->init_status = rc0;
    }
    WorkerBufs wb;
    (void)idx;
    int prio_lo = 0, prio_hi = 0;
    if (!rc0 && s->cfg.reserve_nz > 0 && s->cfg.reserve_ny > 0 && s->cfg.reserve_nx > 0) {
        // resident workspaces for the largest expected cube: no allocation while serving
        const size_t rn = (size_t)s->cfg.reserve_nz * s->cfg.reserve_ny * s->cfg.reserve_nx;
        if (fy_restore_reserve(s->cfg.reserve_nz, s->cfg.reserve_ny, s->cfg.reserve_nx) != FY_OK ||
            wb.d_in.ensure(rn) != cudaSuccess || wb.d_out.ensure(4 * rn) != cudaSuccess)
            cudaGetLastError();                    // serving still works; buffers grow on demand
    }
    if (!rc0) {
        cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);      // (least, greatest)
        if (cudaStreamCreateWithPriority(&wb.hi, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
            cudaStreamCreateWithPriority(&wb.lo, cudaStreamNonBlocking, prio_lo) != cudaSuccess) {
            cudaGetLastError();
            wb.hi = wb.lo = ctx().st;
        }
        for (cudaEvent_t& ev : wb.ev)
            if (cudaEventCreate(&ev) != cudaSuccess) { cudaGetLastError(); ev = nullptr; }
        if (!wb.ev[0] || !wb.ev[1])                                      // untimed unless both exist
            for (cudaEvent_t& ev : wb.ev)
                if (ev) { cudaEventDestroy(ev); ev = nullptr; }
    }
    for (;;) {
        Ticket* t = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            // Workers [0, small_workers) take only requests up to priority_voxels: the first
            // such request in the queue, so small cubes never wait behind large ones for a
            // worker. The others take the head of the queue.
            const bool small_only = idx < s->cfg.small_workers;
            auto fits = [&](const Ticket* q) {
                return s->inflight == 0 || s->inflight_bytes + q->footprint <= s->cfg.hbm_budget_bytes;
            };
            auto pick = [&]() -> std::deque<Ticket*>::iterator {
                if (!small_only) {
                    auto it = s->queue.begin();
                    return it != s->queue.end() && fits(*it) ? it : s->queue.end();
                }
                for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
                    const fy_request& r = (*it)->req;
                    if ((size_t)r.nz * r.ny * r.nx <= s->cfg.priority_voxels) return fits(*it) ? it : s->queue.end();
                }
                return s->queue.end();
            };
            std::deque<Ticket*>::iterator chosen = s->queue.end();
            s->cv_work.wait(lk, [&] {
                if (s->stop) return true;
                chosen = pick();
                return chosen != s->queue.end();
            });
            if (s->stop && s->queue.empty()) break;
            if (s->stop) {                       // drain: cancel what never started
                while (!s->queue.empty()) {
                    Ticket* q = s->queue.front();
                    s->queue.pop_front();
                    q->status = FY_EBUSY;
                    q->done = true;
                }
                s->cv_done.notify_all();
                break;
            }
            t = *chosen;
            s->queue.erase(chosen);
            s->inflight_bytes += t->footprint;
            s->inflight += 1;
            t->t_start = now_ms();
            if (s->first_start == 0) s->first_start = t->t_start;
        }
        if (rc0) {
            std::lock_guard<std::mutex> lk(s->mu);
            t->status = rc0;
            t->done = true;
            t->t_done = now_ms();
            s->inflight_bytes -= t->footprint;
            s->inflight -= 1;
            s->cv_done.notify_all();
            s->cv_work.notify_all();
            continue;
        }
        run_one(s, t, wb);
    }
    if (wb.hi && wb.hi != ctx().st) cudaStreamDestroy(wb.hi);
    if (wb.lo && wb.lo != ctx().st) cudaStreamDestroy(wb.lo);
    for (cudaEvent_t ev : wb.ev)
        if (ev) cudaEventDestroy(ev);
    wb.d_in.release();
    wb.d_out.release();
    wb.h_in.release();
    wb.h_out.release();
    fy_gpu_release();
}

}  // namespace

extern "C" void fy_server_cfg_default(fy_server_cfg* c) {
    c->hbm_budget_bytes = (size_t)150 << 30;    // 150 GB
    c->workers = 8;
    c->device = 0;
    c->priority_voxels = (size_t)256 * 256 * 256;
    c->small_workers = 2;
    c->reserve_nz = c->reserve_ny = c->reserve_nx = 0;
}

extern "C" int fy_server_create(fy_server** out, const fy_server_cfg* cfg) {
    fy::enter();
    if (!out) return fail(FY_EINVAL, "fy_server_create: null handle");
    *out = nullptr;
    int rc = fy::ensure_ctx();                  // fails with FY_ENODEV without a GPU
    if (rc) return rc;
    fy_server* s = new fy_server();
    if (cfg) s->cfg = *cfg;
    else fy_server_cfg_default(&s->cfg);
    if (s->cfg.workers < 1) s->cfg.workers = 1;
    if (s->cfg.small_workers < 0) s->cfg.small_workers = 0;
    if (s->cfg.small_workers >= s->cfg.workers) s->cfg.small_workers = s->cfg.workers - 1;
    if (s->cfg.workers > 64) s->cfg.workers = 64;
    if (s->cfg.hbm_budget_bytes == 0) s->cfg.hbm_budget_bytes = (size_t)150 << 30;
    cudaError_t e = s->h2d.start(s->cfg.device, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && (e = s->d2h.start(s->cfg.device, cudaMemcpyDeviceToHost)) != cudaSuccess) s->h2d.stop();
    if (e != cudaSuccess) {
        delete s;
        return fail_cuda(e, "fy_server_create: link scheduler");
    }
    for (int i = 0; i < s->cfg.workers; ++i) s->workers.emplace_back(worker_main, s, i);
    *out = s;
    return FY_OK;
}

extern "C" int fy_server_submit(fy_server* s, const fy_request* r, long long* ticket) {
    fy::enter();
    if (!s || !r || !ticket) return fail(FY_EINVAL, "fy_server_submit: null pointer");
    if (!r->u8 || !r->out) return fail(FY_EINVAL, "fy_server_submit: null buffer");
    if (r->nz < 1 || r->ny < 1 || r->nx < 1) return fail(FY_EINVAL, "fy_server_submit: bad dims");
    if (r->cfg.dering && r->cfg.dering_accumulate)
        return fail(FY_EINVAL, "fy_server_submit: ring accumulation into a shared handle is not allowed here");
    Ticket* t = new Ticket();
    t->req = *r;
    t->footprint = footprint_of(*r);
    if (t->footprint > s->cfg.hbm_budget_bytes) {
        const size_t fp = t->footprint;
        delete t;
        return fail(FY_EUNSUPPORTED, "fy_server_submit: request needs ~%zu MB, above the HBM budget of %zu MB",
                    fp >> 20, s->cfg.hbm_budget_bytes >> 20);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) { delete t; return fail(FY_EBUSY, "fy_server_submit: server is stopping"); }
    t->id = s->next_id++;
    t->t_submit = now_ms();
    s->tickets[t->id] = t;
    s->queue.push_back(t);
    *ticket = t->id;
    s->cv_work.notify_one();
    return FY_OK;
}

extern "C" int fy_server_wait(fy_server* s, long long ticket, double timeout_ms, fy_request_result* res) {
    fy::enter();
    if (!s) return fail(FY_EINVAL, "fy_server_wait: null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return fail(FY_EINVAL, "fy_server_wait: unknown ticket %lld", ticket);
    Ticket* t = it->second;
    auto ready = [&] { return t->done; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready)) {
        return fail(FY_ETIMEDOUT, "fy_server_wait: ticket %lld not done after %.1f ms", ticket, timeout_ms);
    }
    if (res) {
        res->status = t->status;
        res->queue_ms = t->t_start > 0 ? t->t_start - t->t_submit : 0.0;
        res->run_ms = t->t_start > 0 ? t->t_done - t->t_start : 0.0;
        res->latency_ms = t->t_done - t->t_submit;
        res->h2d_ms = t->h2d_ms;
        res->chain_ms = t->chain_ms;
        res->d2h_ms = t->d2h_ms;
    }
    const int st = t->status;
    s->tickets.erase(it);
    delete t;
    if (st) return fail(st, "fy_server_wait: request failed with status %d", st);
    return FY_OK;
}

extern "C" int fy_server_get_stats(fy_server* s, fy_server_stats* out) {
    fy::enter();
    if (!s || !out) return fail(FY_EINVAL, "fy_server_get_stats: null pointer");
    std::lock_guard<std::mutex> lk(s->mu);
    out->completed = (long long)s->lat_ms.size();
    out->voxels = s->voxels;
    const double span = s->last_done - s->first_start;
    out->mvox_per_s = span > 0 ? s->voxels / (span * 1e-3) / 1e6 : 0.0;
    std::vector<double> v = s->lat_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) {            // nearest-rank percentile
        if (v.empty()) return 0.0;
        size_t k = (size_t)std::ceil(q / 100.0 * (double)v.size());
        if (k < 1) k = 1;
        return v[k - 1];
    };
    out->p50_ms = pct(50.0);
    out->p99_ms = pct(99.0);
    out->inflight = s->inflight;
    out->queued = (int)s->queue.size();
    return FY_OK;
}

extern "C" void fy_server_reset_stats(fy_server* s) {
    if (!s) return;
    std::lock_guard<std::mutex> lk(s->mu);
    s->lat_ms.clear();
    s->voxels = 0;
    s->first_start = 0;
    s->last_done = 0;
}

extern "C" void fy_server_destroy(fy_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& w : s->workers) w.join();
    s->h2d.stop();
    s->d2h.stop();
    for (auto& kv : s->tickets) delete kv.second;
    delete s;
}
