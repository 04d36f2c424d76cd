// serve.cu -- continuous-batching commit server (include/zeknox_b200.h).
//
// Host side: any thread submits requests into a FIFO; one server thread per
// server admits the head of the queue whenever a slot stream is idle and the
// job's device memory fits, enqueues the whole commit (LDE, Merkle, caps
// copy-out) on that slot's stream, and polls the slot events to retire
// finished jobs.  While the head waits for memory (not for a slot), small
// requests behind it (at most 1/8 of the budget each) that fit now may start
// ahead of it, at most `slots` of them per waiting head: a large request then
// holds up no small one, and waits for at most `slots` small ones itself.
//
// Memory: the budget is one device allocation made when the server is
// created (an arena), and every job takes one contiguous range of it
// (first fit, freed ranges merged with their neighbours).  Jobs therefore
// never call the driver's allocator, and a job the budget admits always has
// the memory: per-job stream-ordered allocations of multi-GB buffers measured
// out-of-memory failures and long allocation stalls at this size mix.
//
// Device side: jobs on different slots overlap; twiddle, coset and
// round-constant tables stay resident in the device context across requests
// (zeknox_server_prepare builds them ahead of the stream).
#include <cuda_runtime.h>
#include <string.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/zeknox_b200.h"
#include "batch.cuh"
#include "runtime.cuh"

namespace zk {
namespace {

using Clock = std::chrono::steady_clock;

constexpr uint64_t ARENA_ALIGN = 256;
constexpr uint64_t NO_RANGE = ~0ULL;

uint64_t align_up(uint64_t x) { return (x + ARENA_ALIGN - 1) / ARENA_ALIGN * ARENA_ALIGN; }

// First-fit allocator over the byte offsets of the arena.
struct RangeAlloc {
    std::map<uint64_t, uint64_t> free_;  // offset -> size
    void init(uint64_t size)
    {
        free_.clear();
        if (size) free_[0] = size;
    }
    uint64_t take(uint64_t size)
    {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < size) continue;
            const uint64_t off = it->first, rest = it->second - size;
            free_.erase(it);
            if (rest) free_[off + size] = rest;
            return off;
        }
        return NO_RANGE;
    }
    bool fits(uint64_t size) const
    {
        for (const auto &kv : free_)
            if (kv.second >= size) return true;
        return false;
    }
    void give(uint64_t off, uint64_t size)
    {
        auto it = free_.emplace(off, size).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Ticket {
    zk_serve_request req;
    Clock::time_point t_submit, t_admit, t_done;
    int status = 0;  // 0 queued, 1 running, 2 done, < 0 failed or cancelled
    int slot = -1;
    uint64_t bytes = 0;        // arena bytes of the job (aligned pieces)
    uint64_t off = NO_RANGE;   // its range in the arena while admitted
    uint64_t *leaves = nullptr, *digests = nullptr, *caps = nullptr, *scratch = nullptr;
    cudaEvent_t done_ev = nullptr;
};

struct Server {
    DeviceCtx *ctx = nullptr;
    uint64_t budget = 0, in_use = 0, peak = 0, completed = 0;
    uint8_t *arena = nullptr;
    RangeAlloc ranges;
    std::vector<cudaStream_t> slot_stream;
    std::vector<uint64_t> slot_ticket;  // 0 = idle
    cudaEvent_t tables_ready = nullptr; // recorded on the context stream after a start's table builds
    std::mutex mu;
    std::condition_variable cv;  // signalled on submit, completion, release, stop
    std::deque<uint64_t> queue;
    std::map<uint64_t, Ticket> tickets;
    uint64_t next_id = 1;
    uint64_t blocked_head = 0;  // head of the queue that waits for memory
    uint32_t bypassed = 0;      // small requests started ahead of it
    int inject_next = 0;        // test hook: the next start fails at this stage (ZK_SERVE_FAIL_*)
    bool stop = false;
    std::thread worker;

    // Arena bytes of a job: leaves, digests, caps and LDE scratch, each
    // starting on an ARENA_ALIGN boundary.
    static uint64_t job_bytes(const zk_serve_request &r)
    {
        const uint64_t N = 1ULL << (r.lg_n + r.rate_bits);
        const uint64_t caps = 1ULL << r.cap_height;
        return align_up(8 * N * r.cols) + align_up(64 * (N - caps)) + align_up(32 * caps) +
               align_up(8 * commit_scratch_words(r.lg_n, r.rate_bits, r.cols, r.input_is_values != 0));
    }

    void place(Ticket &t)
    {
        const zk_serve_request &r = t.req;
        const uint64_t N = 1ULL << (r.lg_n + r.rate_bits);
        const uint64_t n_caps = 1ULL << r.cap_height;
        const uint64_t sw = commit_scratch_words(r.lg_n, r.rate_bits, r.cols, r.input_is_values != 0);
        uint8_t *p = arena + t.off;
        t.leaves = (uint64_t *)p;
        p += align_up(8 * N * r.cols);
        t.digests = N > n_caps ? (uint64_t *)p : nullptr;
        p += align_up(64 * (N - n_caps));
        t.caps = (uint64_t *)p;
        p += align_up(32 * n_caps);
        t.scratch = sw ? (uint64_t *)p : nullptr;
    }

    // Give an admitted job's range back (caller holds mu; nothing on the GPU
    // may still use it).
    void unadmit(Ticket &t)
    {
        if (t.off != NO_RANGE) {
            ranges.give(t.off, t.bytes);
            in_use -= t.bytes;
            t.off = NO_RANGE;
        }
        t.leaves = t.digests = t.caps = t.scratch = nullptr;
    }

    // Queue an admitted job's whole commit on its slot stream.  Runs on the
    // server thread without `mu` (client threads keep submitting, waiting and
    // releasing meanwhile): a starting ticket can be neither released nor
    // cancelled, and only this thread starts jobs.  Returns 1 when the work is
    // queued, else a negative status (the slot stream has then finished
    // whatever this start queued, so the range may be reused at once).
    int start(Ticket &t, int slot, int inject)
    {
        const zk_serve_request &r = t.req;
        cudaStream_t s = slot_stream[slot];
        const uint64_t n_caps = 1ULL << r.cap_height;
        NvtxRange range("zeknox serve start");
        std::lock_guard<std::recursive_mutex> lk(ctx->mu);
        try {
            zk_commit_job j{};
            j.lg_n = r.lg_n;
            j.rate_bits = r.rate_bits;
            j.cols = r.cols;
            j.cap_height = r.cap_height;
            j.hash_type = r.hash_type;
            j.input_is_values = r.input_is_values;
            j.coset_gen = r.coset_gen;
            j.input = r.input;
            j.leaves = t.leaves;
            j.digests = t.digests;
            j.caps = t.caps;
            if (inject == ZK_SERVE_FAIL_SHAPE) j.cap_height = j.lg_n + j.rate_bits + 1;  // a shape that cannot commit
            if (inject == ZK_SERVE_FAIL_ALLOC)
                throw cuda_failure(-(int)cudaErrorMemoryAllocation, "device allocation refused (injected)");
            check_job(j);
            // tables this shape reads that are not resident yet are built on
            // the context stream; the slot stream waits for them on the
            // device, not the server thread on the host
            prepare_job(*ctx, j);
            ZK_CUDA(cudaEventRecord(tables_ready, ctx->stream));
            ZK_CUDA(cudaStreamWaitEvent(s, tables_ready, 0));
            if (inject == ZK_SERVE_FAIL_LAUNCH)
                throw cuda_failure(-(int)cudaErrorLaunchFailure, "kernel launch refused (injected)");
            commit_enqueue(*ctx, j, s, t.scratch);
            if (r.caps_host) ZK_CUDA(cudaMemcpyAsync(r.caps_host, t.caps, n_caps * 32, cudaMemcpyDeviceToHost, s));
            ZK_CUDA(cudaEventCreateWithFlags(&t.done_ev, cudaEventDisableTiming));
            ZK_CUDA(cudaEventRecord(t.done_ev, s));
            return 1;
        } catch (const std::exception &e) {
            const cuda_failure *cf = dynamic_cast<const cuda_failure *>(&e);
            const arg_failure *af = dynamic_cast<const arg_failure *>(&e);
            (void)cudaStreamSynchronize(s);  // whatever was queued finishes before the range is reused
            (void)cudaGetLastError();
            if (t.done_ev) {
                cudaEventDestroy(t.done_ev);
                t.done_ev = nullptr;
            }
            return cf ? (cf->code < 0 ? cf->code : -1) : af ? -af->code : -1;
        }
    }

    void loop()
    {
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            // retire finished jobs
            bool progressed = false;
            for (size_t k = 0; k < slot_ticket.size(); k++) {
                uint64_t id = slot_ticket[k];
                if (!id) continue;
                Ticket &t = tickets[id];
                cudaError_t q = cudaEventQuery(t.done_ev);
                if (q == cudaErrorNotReady) continue;
                t.t_done = Clock::now();
                t.status = q == cudaSuccess ? 2 : -(int)q;
                if (q != cudaSuccess) (void)cudaGetLastError();
                cudaEventDestroy(t.done_ev);
                t.done_ev = nullptr;
                slot_ticket[k] = 0;
                completed++;
                progressed = true;
            }
            if (progressed) cv.notify_all();
            // admit in arrival order, small requests past a head that waits for memory
            while (!queue.empty()) {
                int slot = -1;
                for (size_t k = 0; k < slot_ticket.size(); k++)
                    if (!slot_ticket[k]) {
                        slot = (int)k;
                        break;
                    }
                if (slot < 0) break;
                auto pick = queue.begin();
                if (!ranges.fits(tickets[*pick].bytes)) {
                    if (blocked_head != *pick) {
                        blocked_head = *pick;
                        bypassed = 0;
                    }
                    if (bypassed >= slot_ticket.size()) break;
                    for (++pick; pick != queue.end(); ++pick) {
                        const uint64_t b = tickets[*pick].bytes;
                        if (b <= budget / 8 && ranges.fits(b)) break;
                    }
                    if (pick == queue.end()) break;
                    bypassed++;
                }
                const uint64_t id = *pick;
                Ticket &t = tickets[id];
                queue.erase(pick);
                t.off = ranges.take(t.bytes);
                in_use += t.bytes;
                peak = in_use > peak ? in_use : peak;
                place(t);
                t.slot = slot;
                t.t_admit = Clock::now();
                t.status = 1;
                slot_ticket[slot] = id;
                const int inject = inject_next;
                inject_next = 0;
                lk.unlock();
                const int st = start(t, slot, inject);
                lk.lock();
                if (st < 0) {
                    // could not start: the slot and the range are free again
                    t.status = st;
                    t.t_done = Clock::now();
                    unadmit(t);
                    slot_ticket[slot] = 0;
                }
                cv.notify_all();
            }
            bool busy = false;
            for (uint64_t id : slot_ticket) busy |= id != 0;
            if (stop && !busy && queue.empty()) break;
            if (busy) {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(50));
                lk.lock();
            } else {
                cv.wait_for(lk, std::chrono::milliseconds(5));
            }
        }
    }
};

Server *as_server(void *p)
{
    if (!p) throw arg_failure("null server");
    return (Server *)p;
}

RustError to_error(int code, const std::string &msg)
{
    RustError e;
    e.code = code;
    e.message = msg.empty() ? nullptr : strdup(msg.c_str());
    return e;
}

template <class F>
RustError guard(F &&f)
{
    try {
        f();
        return RustError{0, nullptr};
    } catch (const arg_failure &e) {
        return to_error(e.code, e.what());
    } catch (const cuda_failure &e) {
        return to_error(e.code, e.what());
    } catch (const std::exception &e) {
        return to_error(-(int)cudaErrorUnknown, e.what());
    }
}

}  // namespace
}  // namespace zk

using zk::Server;

extern "C" RustError zeknox_server_create(size_t device_id, uint64_t budget_bytes, uint32_t slots, void **server)
{
    return zk::guard([&] {
        if (!server) throw zk::arg_failure("null out pointer");
        if (slots == 0 || slots > 64) throw zk::arg_failure("slots must be 1..64");
        if (budget_bytes < zk::ARENA_ALIGN) throw zk::arg_failure("budget below one allocation unit");
        zk::DeviceCtx &c = zk::device(device_id);
        Server *s = new Server();
        try {
            s->ctx = &c;
            s->budget = budget_bytes / zk::ARENA_ALIGN * zk::ARENA_ALIGN;
            {
                std::lock_guard<std::recursive_mutex> dl(c.mu);
                // the pool's cached temporaries go back to the driver first, so
                // the reservation sees the device's free memory
                cudaMemPool_t pool;
                if (cudaDeviceGetDefaultMemPool(&pool, c.id) == cudaSuccess) (void)cudaMemPoolTrimTo(pool, 0);
                ZK_CUDA(cudaMalloc((void **)&s->arena, s->budget));
            }
            s->ranges.init(s->budget);
            s->slot_stream.assign(slots, nullptr);
            s->slot_ticket.assign(slots, 0);
            for (auto &st : s->slot_stream) ZK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            ZK_CUDA(cudaEventCreateWithFlags(&s->tables_ready, cudaEventDisableTiming));
        } catch (...) {
            for (auto &st : s->slot_stream)
                if (st) cudaStreamDestroy(st);
            if (s->tables_ready) cudaEventDestroy(s->tables_ready);
            if (s->arena) cudaFree(s->arena);
            delete s;
            throw;
        }
        s->worker = std::thread([s] {
            cudaSetDevice(s->ctx->id);
            s->loop();
        });
        *server = s;
    });
}

extern "C" RustError zeknox_server_submit(void *server, const zk_serve_request *req, uint64_t *ticket)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        if (!req || !ticket) throw zk::arg_failure("null pointer");
        zk_commit_job j{};
        j.lg_n = req->lg_n;
        j.rate_bits = req->rate_bits;
        j.cols = req->cols;
        j.cap_height = req->cap_height;
        j.hash_type = req->hash_type;
        j.input = req->input;
        j.leaves = (uint64_t *)1;  // buffers are the server's: check shape only
        j.digests = (uint64_t *)1;
        j.caps = (uint64_t *)1;
        zk::check_job(j);
        const uint64_t bytes = Server::job_bytes(*req);
        std::lock_guard<std::mutex> lk(s->mu);
        if (bytes > s->budget) throw zk::arg_failure("request needs more device memory than the server's budget");
        const uint64_t id = s->next_id++;
        zk::Ticket &t = s->tickets[id];
        t.req = *req;
        t.bytes = bytes;
        t.t_submit = zk::Clock::now();
        s->queue.push_back(id);
        *ticket = id;
        s->cv.notify_all();
    });
}

extern "C" RustError zeknox_server_wait(void *server, uint64_t ticket, double timeout_ms, zk_serve_result *result)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) throw zk::arg_failure("unknown ticket");
        auto done = [&] { return it->second.status == 2 || it->second.status < 0; };
        if (timeout_ms < 0) s->cv.wait(lk, done);
        else s->cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), done);
        const zk::Ticket &t = it->second;
        if (result) {
            result->status = t.status;
            result->latency_ms = t.status == 2 ? std::chrono::duration<double, std::milli>(t.t_done - t.t_submit).count() : 0;
            result->queue_ms = t.status >= 1 || t.status < 0
                                   ? std::chrono::duration<double, std::milli>(t.t_admit - t.t_submit).count()
                                   : 0;
            result->leaves = t.status == 2 ? t.leaves : nullptr;
            result->digests = t.status == 2 ? t.digests : nullptr;
            result->caps = t.status == 2 ? t.caps : nullptr;
        }
    });
}

extern "C" RustError zeknox_server_release(void *server, uint64_t ticket)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) throw zk::arg_failure("unknown ticket");
        zk::Ticket &t = it->second;
        if (t.status == 0 || t.status == 1) throw zk::arg_failure("ticket still queued or running");
        s->unadmit(t);  // its work has finished: the range is free at once
        s->tickets.erase(it);
        s->cv.notify_all();
    });
}

extern "C" RustError zeknox_server_stats(void *server, uint64_t *in_use_bytes, uint64_t *peak_bytes,
                                         uint64_t *completed)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        std::lock_guard<std::mutex> lk(s->mu);
        if (in_use_bytes) *in_use_bytes = s->in_use;
        if (peak_bytes) *peak_bytes = s->peak;
        if (completed) *completed = s->completed;
    });
}

extern "C" RustError zeknox_server_prepare(void *server, uint32_t lg_n_min, uint32_t lg_n_max, uint32_t rate_bits,
                                           uint64_t coset_gen)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        if (lg_n_min == 0 || lg_n_min > lg_n_max || rate_bits == 0 || rate_bits > 32 || lg_n_max > 32 - rate_bits)
            throw zk::arg_failure("need 1 <= lg_n_min <= lg_n_max and lg_n_max + rate_bits <= 32");
        std::lock_guard<std::recursive_mutex> dl(s->ctx->mu);
        ZK_CUDA(cudaSetDevice(s->ctx->id));
        for (uint32_t lg = lg_n_min; lg <= lg_n_max; lg++) {
            zk_commit_job j{};
            j.lg_n = lg;
            j.rate_bits = rate_bits;
            j.coset_gen = coset_gen;
            j.input_is_values = 1;  // the inverse tables too
            zk::prepare_job(*s->ctx, j);
        }
        s->ctx->sync();
    });
}

extern "C" RustError zeknox_server_cancel(void *server, uint64_t ticket)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) throw zk::arg_failure("unknown ticket");
        zk::Ticket &t = it->second;
        if (t.status != 0) throw zk::arg_failure("only a queued request can be cancelled");
        for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
            if (*q == ticket) {
                s->queue.erase(q);
                break;
            }
        if (s->blocked_head == ticket) s->blocked_head = 0;
        t.status = ZK_SERVE_CANCELLED;  // never admitted: it holds no range
        t.t_done = t.t_admit = zk::Clock::now();
        s->cv.notify_all();
    });
}

extern "C" RustError zeknox_server_inject_failure(void *server, int stage)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        if (stage < 0 || stage > ZK_SERVE_FAIL_LAUNCH) throw zk::arg_failure("unknown failure stage");
        std::lock_guard<std::mutex> lk(s->mu);
        s->inject_next = stage;
    });
}

extern "C" RustError zeknox_server_destroy(void *server)
{
    return zk::guard([&] {
        Server *s = zk::as_server(server);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = true;
            s->cv.notify_all();
        }
        s->worker.join();
        std::lock_guard<std::recursive_mutex> dl(s->ctx->mu);
        ZK_CUDA(cudaSetDevice(s->ctx->id));
        for (auto &st : s->slot_stream) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        cudaEventDestroy(s->tables_ready);
        cudaFree(s->arena);
        delete s;
    });
}
