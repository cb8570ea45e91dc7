// server.cu -- continuous-batching matmul server (fg_server_*).
//
// Host threads submit requests whose operands already live on the device.
// A dispatcher thread admits queued requests in arrival order while their
// HBM need fits the budget and a stream slot is free, and launches them:
//   * "small" requests (max(m, n, k) <= kGroupMaxDim) of dtype f32 (plain or
//     split) or i8 / u8i8 are folded, per (dtype, mode) class, into ONE
//     grouped launch of up to max_group problems (grouped.cu);
//   * everything else (f64 / complex, large shapes) runs as its own launch.
// Each launch goes to the next free slot (own stream, own workspace), so a
// batch admitted while earlier ones are still on the GPU overlaps with them.
// A completion thread waits on the slots' events, completes their tickets,
// records submit-to-completion latency and returns the HBM to the budget.
// A request's route depends only on its class, so a result is the same
// whether the request ran alone or folded into a mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "runtime.h"

namespace {

constexpr long long kGroupMaxDim = 1024;

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

bool groupable(const fg_request& r) {
    const bool dt = r.dtype == FG_F32 || r.dtype == FG_I8 || r.dtype == FG_U8I8;
    return dt && std::max(r.m, std::max(r.n, r.k)) <= kGroupMaxDim;
}

// Device bytes a request holds while in flight: operands, output, scratch.
size_t request_bytes(const fg_request& r) {
    const size_t in = fgrt::in_size(r.dtype), out = fgrt::out_size(r.dtype);
    const size_t a = in * r.m * r.k, b = in * r.k * r.n, c = out * r.m * r.n;
    size_t scratch = r.scratch_bytes;
    if (!scratch) {
        if (r.mode != FG_MODE_PLAIN && (r.dtype == FG_F32 || r.dtype == FG_C32))
            scratch = (r.dtype == FG_C32 ? 4 : 1) * 2 * 2 * (r.m * r.k + r.k * r.n) * 2;
        else if (r.mode != FG_MODE_PLAIN && (r.dtype == FG_F64 || r.dtype == FG_C64))
            // default split: Ozaki scheme II with 16 moduli -> 16 int8 residue
            // planes of A, B and of the result bytes (x4 for the complex
            // embedding), plus scales
            scratch = (r.dtype == FG_C64 ? 4 : 1) * 16 * (r.m * r.k + r.k * r.n + r.m * r.n) +
                      32 * (r.m + r.n + r.k);
        else if (r.dtype == FG_I16)
            scratch = 2 * (r.m * r.k + r.k * r.n) + 64 * (r.m + r.n);
        else if (r.dtype == FG_I8 || r.dtype == FG_U8I8)
            scratch = (r.m * r.k + r.k * r.n) + 64 * (r.m + r.n);
    }
    return a + b + c + scratch;
}

double request_flops(const fg_request& r) {
    const double f = 2.0 * r.m * r.n * r.k;
    return (r.dtype == FG_C64 || r.dtype == FG_C32) ? 4.0 * f : f;
}

}  // namespace

struct fg_server {
    struct Req {
        fg_request r;
        double t_submit = 0, t_done = 0;
        size_t bytes = 0;
        int state = 0;  // 0 queued, 1 in flight, 2 done
        fg_status status = FG_OK;
    };
    struct Slot {
        cudaStream_t st = nullptr;
        cudaEvent_t done = nullptr;
        void* ws = nullptr;
        size_t ws_bytes = 0;
        void* host = nullptr;
        size_t host_bytes = 0;
        fgrt::GroupedJob* job = nullptr;
        std::vector<uint64_t> tickets;
        bool busy = false;
        bool grouped = false;
        bool recorded = false;  // the completion event of this batch is recorded
    };
    fg_ctx* ctx = nullptr;
    size_t budget = 0;
    int max_group = 256;
    std::mutex mu;
    std::condition_variable cv;       // queue / slot / completion changes
    std::condition_variable cv_done;  // ticket completions
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, Req> reqs;
    uint64_t next_ticket = 1;
    size_t in_use = 0, peak = 0;
    bool stop = false;
    std::vector<Slot> slots;
    std::thread dispatcher, completer;
    // stats
    std::vector<double> lat;
    uint64_t completed = 0, launches = 0, grouped_launches = 0;
    double flops = 0, t_first = 0, t_last = 0;
};

namespace {

void dispatch_loop(fg_server* s) {
    cudaSetDevice(s->ctx->device);
    std::vector<fg_problem> table;
    while (true) {
        std::vector<uint64_t> batch;
        int slot_id = -1;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait(lk, [&] {
                if (s->stop) return true;
                if (s->queue.empty()) return false;
                for (auto& sl : s->slots)
                    if (!sl.busy) return true;
                return false;
            });
            if (s->stop) return;
            for (size_t i = 0; i < s->slots.size(); ++i)
                if (!s->slots[i].busy) {
                    slot_id = static_cast<int>(i);
                    break;
                }
            // admit in arrival order; the head defines the class of the batch
            const uint64_t head = s->queue.front();
            auto& hr = s->reqs[head];
            if (s->in_use + hr.bytes > s->budget && s->in_use > 0) {
                // wait for memory to come back before admitting the head
                s->cv.wait(lk, [&] { return s->stop || s->in_use + hr.bytes <= s->budget || s->in_use == 0; });
                if (s->stop) return;
            }
            const bool grp = groupable(hr.r);
            for (auto it = s->queue.begin(); it != s->queue.end() && (int)batch.size() < (grp ? s->max_group : 1);) {
                auto& rq = s->reqs[*it];
                const bool same = grp ? (groupable(rq.r) && rq.r.dtype == hr.r.dtype && rq.r.mode == hr.r.mode)
                                      : (*it == head);
                if (same && (s->in_use + rq.bytes <= s->budget || batch.empty())) {
                    batch.push_back(*it);
                    s->in_use += rq.bytes;
                    rq.state = 1;
                    it = s->queue.erase(it);
                } else {
                    ++it;
                }
            }
            s->peak = std::max(s->peak, s->in_use);
            if (s->t_first == 0) s->t_first = now_s();
            auto& sl = s->slots[slot_id];
            sl.busy = true;
            sl.recorded = false;
            sl.grouped = grp;
            sl.tickets = batch;
        }
        auto& sl = s->slots[slot_id];
        fg_status st = FG_OK;
        if (sl.grouped) {
            table.clear();
            fg_dtype dt = FG_F32;
            fg_mode md = FG_MODE_PLAIN;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                for (uint64_t t : batch) {
                    const fg_request& r = s->reqs[t].r;
                    dt = r.dtype;
                    md = r.mode;
                    table.push_back(fg_problem{r.m, r.n, r.k, r.a, r.b, r.c, r.k, r.n, r.n});
                }
            }
            st = fgrt::grouped_job_build(s->ctx, dt, md, table.data(), table.size(), sl.job);
            if (st == FG_OK) {
                const size_t need = fgrt::grouped_job_dev_bytes(sl.job), hneed = fgrt::grouped_job_host_bytes(sl.job);
                if (need > sl.ws_bytes) {
                    // stream-ordered, so growing one slot never stalls the others
                    if (sl.ws) cudaFreeAsync(sl.ws, sl.st);
                    sl.ws_bytes = std::max(need, sl.ws_bytes * 2);
                    if (cudaMallocAsync(&sl.ws, sl.ws_bytes, sl.st) != cudaSuccess) {
                        cudaGetLastError();
                        sl.ws = nullptr;
                        sl.ws_bytes = 0;
                        st = fgrt::set_error(FG_ERR_OOM, "server workspace");
                    }
                }
                if (st == FG_OK && hneed > sl.host_bytes) {
                    if (sl.host) cudaFreeHost(sl.host);
                    sl.host_bytes = std::max(hneed, sl.host_bytes * 2);
                    if (cudaMallocHost(&sl.host, sl.host_bytes) != cudaSuccess) {
                        cudaGetLastError();
                        sl.host = nullptr;
                        sl.host_bytes = 0;
                        st = fgrt::set_error(FG_ERR_OOM, "server staging");
                    }
                }
                if (st == FG_OK) st = fgrt::grouped_job_bind(sl.job, sl.ws, sl.host);
                if (st == FG_OK) st = fgrt::grouped_job_launch(sl.job, sl.st);
            }
        } else {
            fg_request r;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                r = s->reqs[batch[0]].r;
            }
            double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
            float onef[2] = {1.f, 0.f}, zerof[2] = {0.f, 0.f};
            const bool f32ish = r.dtype == FG_F32 || r.dtype == FG_C32;
            st = fg_gemm(s->ctx, r.dtype, r.mode, 0, r.m, r.n, r.k, f32ish ? (void*)onef : (void*)one, r.a,
                         r.k, r.b, r.n, f32ish ? (void*)zerof : (void*)zero, r.c, r.n, 0, sl.st);
        }
        if (cudaEventRecord(sl.done, sl.st) != cudaSuccess && st == FG_OK)
            st = fgrt::set_error(FG_ERR_DEVICE, "server event");
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->launches++;
            if (sl.grouped) s->grouped_launches++;
            for (uint64_t t : batch) s->reqs[t].status = st;
            sl.recorded = true;
        }
        s->cv.notify_all();
    }
}

void complete_loop(fg_server* s) {
    cudaSetDevice(s->ctx->device);
    while (true) {
        std::vector<int> busy;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait_for(lk, std::chrono::milliseconds(2), [&] {
                if (s->stop) return true;
                for (auto& sl : s->slots)
                    if (sl.busy && sl.recorded) return true;
                return false;
            });
            if (s->stop) return;
            for (size_t i = 0; i < s->slots.size(); ++i)
                if (s->slots[i].busy && s->slots[i].recorded) busy.push_back(static_cast<int>(i));
        }
        bool any = false;
        for (int i : busy) {
            auto& sl = s->slots[i];
            cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaErrorNotReady) continue;
            const double t = now_s();
            std::lock_guard<std::mutex> lk(s->mu);
            if (!sl.busy) continue;
            for (uint64_t tk : sl.tickets) {
                auto& rq = s->reqs[tk];
                if (rq.state != 1) continue;
                rq.state = 2;
                rq.t_done = t;
                if (q != cudaSuccess && rq.status == FG_OK) rq.status = FG_ERR_DEVICE;
                s->in_use -= rq.bytes;
                s->lat.push_back((t - rq.t_submit) * 1e3);
                s->completed++;
                s->flops += request_flops(rq.r);
            }
            s->t_last = t;
            sl.tickets.clear();
            sl.busy = false;
            any = true;
        }
        if (any) {
            s->cv.notify_all();
            s->cv_done.notify_all();
        } else {
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
}

}  // namespace

using namespace fgrt;

extern "C" {

fg_status fg_server_start(fg_ctx* ctx, size_t hbm_budget_bytes, int streams, int max_group,
                          fg_server** out) {
    if (!ctx || !out) return set_error(FG_ERR_INVALID, "null argument");
    if (streams <= 0) streams = 4;
    if (max_group <= 0) max_group = 256;
    if (hbm_budget_bytes == 0) return set_error(FG_ERR_INVALID, "zero HBM budget");
    FG_CUDA(cudaSetDevice(ctx->device));
    auto* s = new fg_server();
    s->ctx = ctx;
    s->budget = hbm_budget_bytes;
    s->max_group = max_group;
    s->slots.resize(streams);
    for (auto& sl : s->slots) {
        cudaError_t e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            fg_server_stop(s);
            return cuda_error(e, "fg_server_start");
        }
        sl.job = grouped_job_new();
    }
    s->dispatcher = std::thread(dispatch_loop, s);
    s->completer = std::thread(complete_loop, s);
    *out = s;
    return FG_OK;
}

fg_status fg_server_submit(fg_server* s, const fg_request* req, uint64_t* ticket) {
    if (!s || !req || !ticket) return set_error(FG_ERR_INVALID, "null argument");
    if (req->dtype < FG_F64 || req->dtype > FG_I16) return set_error(FG_ERR_DTYPE, "bad dtype");
    if (req->m < 0 || req->n < 0 || req->k < 0) return set_error(FG_ERR_SHAPE, "negative dimension");
    if (!req->c || (req->k > 0 && (!req->a || !req->b))) return set_error(FG_ERR_INVALID, "null operand");
    fg_server::Req r;
    r.r = *req;
    r.bytes = request_bytes(*req);
    if (r.bytes > s->budget)
        return set_error(FG_ERR_BUDGET, "request needs " + std::to_string(r.bytes) + " bytes, budget is " +
                                            std::to_string(s->budget));
    r.t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return set_error(FG_ERR_INVALID, "server stopped");
        *ticket = s->next_ticket++;
        s->reqs.emplace(*ticket, r);
        s->queue.push_back(*ticket);
    }
    s->cv.notify_all();
    return FG_OK;
}

fg_status fg_server_wait(fg_server* s, uint64_t ticket, int64_t timeout_ms) {
    return fg_server_wait_times(s, ticket, timeout_ms, nullptr, nullptr);
}

double fg_server_clock(void) { return now_s(); }

fg_status fg_server_wait_times(fg_server* s, uint64_t ticket, int64_t timeout_ms, double* submit_s,
                               double* done_s) {
    if (!s) return set_error(FG_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return set_error(FG_ERR_INVALID, "unknown ticket");
    auto done = [&] { return s->reqs[ticket].state == 2; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, done);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
        return set_error(FG_ERR_TIMEOUT, "ticket not complete");
    }
    const fg_status st = s->reqs[ticket].status;
    if (submit_s) *submit_s = s->reqs[ticket].t_submit;
    if (done_s) *done_s = s->reqs[ticket].t_done;
    s->reqs.erase(ticket);
    if (st != FG_OK) return set_error(st, "request failed");
    return FG_OK;
}

fg_status fg_server_stats_get(fg_server* s, fg_server_stats* out) {
    if (!s || !out) return set_error(FG_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = fg_server_stats{};
    out->completed = s->completed;
    out->launches = s->launches;
    out->grouped_launches = s->grouped_launches;
    if (!s->lat.empty()) {
        std::vector<double> v = s->lat;
        std::sort(v.begin(), v.end());
        auto q = [&](double p) { return v[std::min(v.size() - 1, static_cast<size_t>(p * (v.size() - 1) + 0.5))]; };
        out->p50_ms = q(0.50);
        out->p99_ms = q(0.99);
        double sum = 0;
        for (double x : v) sum += x;
        out->mean_ms = sum / v.size();
    }
    out->useful_flops = s->flops;
    out->busy_seconds = s->t_last > s->t_first ? s->t_last - s->t_first : 0;
    out->hbm_in_use = s->in_use;
    out->hbm_peak = s->peak;
    return FG_OK;
}

fg_status fg_server_stop(fg_server* s) {
    if (!s) return FG_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    s->cv_done.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    if (s->completer.joinable()) s->completer.join();
    cudaSetDevice(s->ctx->device);
    for (auto& sl : s->slots) {
        // free the workspace on its own stream while the stream still exists
        if (sl.ws && sl.st) cudaFreeAsync(sl.ws, sl.st);
        if (sl.st) cudaStreamSynchronize(sl.st);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.st) cudaStreamDestroy(sl.st);
        if (sl.host) cudaFreeHost(sl.host);
        if (sl.job) grouped_job_free(sl.job);
    }
    delete s;
    return FG_OK;
}

}  // extern "C"
