// svdag_server.cu - the serving form: a request loop on its own host thread with continuous batching
// of edits into persistent launches, a frame after every launch (edit-to-visible), admission by
// reserved item-region memory, and a timed replay driver. SVDAG_SERVE_PLAIN turns the same loop into
// the per-edit baseline (one request at a time, synchronously).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "svdag_edit.cuh"
#include "svdag_host.hpp"

using namespace svdag;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket;
    uint32_t kind; // 0 edit, 1 frame
    svdag_edit edit;
    svdag_trace_params frame;
    double submit;
    unsigned long long reserve; // admission estimate (edits)
};

struct Flight {
    std::vector<Request> reqs;
    std::vector<uint32_t> lastRecord; // per request: index of its last record (edits), or ~0u
    uint32_t slot = 0;
    uint32_t launch = 0;
    unsigned long long reserved = 0;
    cudaEvent_t done = nullptr;
};

constexpr uint32_t kNoRecord = 0xFFFFFFFFu;

// Upper estimate of the item-region bytes an edit can add: its intermediate SVO bounds the new items.
// Leaves: the footprint's bounding volume in 4^3 bricks, or for spheres and boxes whose volume is
// large, a shell of three bricks' thickness around the surface (interior nodes are filled or emptied
// whole). Nodes above the leaves add at most a seventh; each item takes at most 48 bytes with its
// share of the slab header.
unsigned long long edit_reserve_bytes(const svdag_edit& e, uint32_t levels)
{
    const double r = std::max(1.0, (double)e.radius);
    const double side = 2.0 * r / 4.0 + 2.0; // bricks per axis
    const double volume = side * side * side;
    double leaves = volume;
    switch (e.tool) {
    case SVDAG_TOOL_SPHERE_ADD:
    case SVDAG_TOOL_SPHERE_REMOVE:
    case SVDAG_TOOL_SPHERE_PAINT:
        leaves = std::min(volume, 3.0 * 4.0 * M_PI * (r / 4.0 + 1.0) * (r / 4.0 + 1.0));
        break;
    case SVDAG_TOOL_BOX_ADD:
    case SVDAG_TOOL_BOX_REMOVE:
        leaves = std::min(volume, 3.0 * 6.0 * side * side);
        break;
    case SVDAG_TOOL_MOVE:
        leaves = 2.0 * volume;
        break;
    default:
        break;
    }
    const double items = leaves * 8.0 / 7.0 + 8.0 * levels;
    return (unsigned long long)(items * 48.0);
}

double now_since(Clock::time_point t0) { return std::chrono::duration<double>(Clock::now() - t0).count(); }

} // namespace

struct svdag_server {
    svdag_ctx* ctx = nullptr;
    svdag_server_config cfg {};
    Clock::time_point t0;
    cudaStream_t stream = nullptr;
    svdag_hit* hits = nullptr; // device frame
    svdag_hit* hostHits = nullptr; // pinned copy (SVDAG_SERVE_COPY_FRAMES)
    size_t frameHits = 0;
    uint32_t nslots = 0;
    size_t slotBytes = 0;
    std::vector<EditRecord*> hostRecords; // pinned, one array per slot
    std::vector<unsigned long long*> hostTop; // pinned item-region top after each launch
    std::vector<cudaEvent_t> events;
    unsigned long long capBytes = 0;
    unsigned long long usedBytes = 0; // item region in use after the last completed launch

    std::mutex m;
    std::condition_variable cv, doneCv;
    std::deque<Request> queue;
    std::unordered_map<uint64_t, svdag_request_result> done;
    uint64_t nextTicket = 1;
    bool stop = false;
    svdag_status fatal = SVDAG_OK;
    std::deque<Flight> inflight; // touched by the worker thread only
    uint32_t launches = 0;
    std::thread worker;

    bool plain() const { return cfg.flags & SVDAG_SERVE_PLAIN; }

    svdag_status launch(std::vector<Request>& reqs, unsigned long long reserved)
    {
        Flight f;
        f.slot = launches % nslots;
        f.launch = launches++;
        f.reserved = reserved;
        f.done = events[f.slot];
        std::vector<DevEditor> eds;
        svdag_trace_params frame = cfg.frame;
        for (auto& r : reqs) {
            if (r.kind == 0) {
                DevEditor tmp[2];
                const int n = expand_edit(ctx, r.edit, tmp);
                eds.insert(eds.end(), tmp, tmp + n);
                f.lastRecord.push_back((uint32_t)eds.size() - 1);
            } else {
                frame = r.frame;
                f.lastRecord.push_back(kNoRecord);
            }
        }
        char* region = ctx->batch + (size_t)f.slot * slotBytes;
        if (!eds.empty()) {
            SVDAG_TRY(launch_edits_at(ctx, eds.data(), (uint32_t)eds.size(), region, slotBytes, stream));
            const size_t edBytes = align256(eds.size() * sizeof(DevEditor));
            SVDAG_CUDA(cudaMemcpyAsync(hostRecords[f.slot], region + edBytes, eds.size() * sizeof(EditRecord), cudaMemcpyDeviceToHost,
                stream));
            SVDAG_CUDA(cudaMemcpyAsync(hostTop[f.slot], &ctx->ctl->itemTop, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
        }
        // The frame of the new state: edit-to-visible ends when it completes.
        if ((size_t)frame.width * frame.height > frameHits)
            frame = cfg.frame;
        SVDAG_TRY((svdag_status)svdag_trace_primary(ctx, &frame, hits, stream));
        if (cfg.flags & SVDAG_SERVE_COPY_FRAMES)
            SVDAG_CUDA(cudaMemcpyAsync(hostHits, hits, (size_t)frame.width * frame.height * sizeof(svdag_hit), cudaMemcpyDeviceToHost,
                stream));
        SVDAG_CUDA(cudaEventRecord(f.done, stream));
        f.reqs = std::move(reqs);
        inflight.push_back(std::move(f));
        return SVDAG_OK;
    }

    // Waits for the oldest launch and hands out its results.
    svdag_status complete_oldest()
    {
        SVDAG_CUDA(cudaEventSynchronize(inflight.front().done));
        const double t = now_since(t0);
        Flight f = std::move(inflight.front());
        inflight.pop_front();
        const EditRecord* rec = hostRecords[f.slot];
        std::lock_guard<std::mutex> lk(m);
        bool anyEdit = false;
        for (size_t i = 0; i < f.reqs.size(); ++i) {
            const Request& r = f.reqs[i];
            svdag_request_result out {};
            out.ticket = r.ticket;
            out.kind = r.kind;
            out.launch = f.launch;
            out.submit_s = r.submit;
            out.visible_s = t;
            if (f.lastRecord[i] != kNoRecord) {
                anyEdit = true;
                const EditRecord& e = rec[f.lastRecord[i]];
                out.status = e.status;
                if (r.edit.tool == SVDAG_TOOL_MOVE && f.lastRecord[i] > 0 && rec[f.lastRecord[i] - 1].status)
                    out.status = rec[f.lastRecord[i] - 1].status;
                out.root_after = e.rootAfter;
                out.edited_voxels = e.edited;
            }
            done[r.ticket] = out;
        }
        if (anyEdit)
            usedBytes = *hostTop[f.slot] * 4ull;
        doneCv.notify_all();
        return SVDAG_OK;
    }

    unsigned long long reserved_in_flight()
    {
        unsigned long long s = 0;
        for (auto& f : inflight)
            s += f.reserved;
        return s;
    }

    // Hands out failed results for requests that will never become visible.
    void fail_requests(const std::vector<Request>& reqs, svdag_status st)
    {
        const double t = now_since(t0);
        for (auto& r : reqs) {
            svdag_request_result out {};
            out.ticket = r.ticket;
            out.kind = r.kind;
            out.status = st;
            out.submit_s = r.submit;
            out.visible_s = t;
            done[r.ticket] = out;
        }
        doneCv.notify_all();
    }

    void run()
    {
        const uint32_t maxBatch = plain() ? 1u : (cfg.max_batch ? cfg.max_batch : 256u);
        const uint32_t maxInflight = plain() ? 1u : std::min<uint32_t>(cfg.max_inflight ? cfg.max_inflight : 2u, nslots - 1);
        for (;;) {
            // Results of finished launches.
            while (!inflight.empty() && cudaEventQuery(inflight.front().done) == cudaSuccess)
                if (complete_oldest() != SVDAG_OK)
                    break;
            std::vector<Request> take;
            unsigned long long reserve = 0;
            {
                std::unique_lock<std::mutex> lk(m);
                if (stop && queue.empty() && inflight.empty())
                    break;
                if (inflight.size() < maxInflight && !queue.empty()) {
                    const unsigned long long inUse = usedBytes + reserved_in_flight();
                    uint32_t edits = 0;
                    while (!queue.empty()) {
                        Request& r = queue.front();
                        if (r.kind == 0) {
                            if (edits == maxBatch)
                                break;
                            const bool first = inflight.empty() && edits == 0; // always make progress
                            if (!first && inUse + reserve + r.reserve > capBytes)
                                break;
                            reserve += r.reserve;
                            ++edits;
                        }
                        take.push_back(r);
                        queue.pop_front();
                        if (plain())
                            break;
                    }
                }
            }
            if (!take.empty()) {
                const svdag_status st = launch(take, reserve);
                if (st != SVDAG_OK) {
                    std::lock_guard<std::mutex> lk(m);
                    fatal = st;
                    fail_requests(take, st);
                }
                continue;
            }
            if (!inflight.empty() && inflight.size() >= maxInflight) {
                // Full: wait for the oldest launch.
                if (complete_oldest() != SVDAG_OK) {
                    std::lock_guard<std::mutex> lk(m);
                    fatal = SVDAG_ERR_CUDA;
                    for (auto& f : inflight)
                        fail_requests(f.reqs, SVDAG_ERR_CUDA);
                    inflight.clear();
                }
                continue;
            }
            std::unique_lock<std::mutex> lk(m);
            if (inflight.empty())
                cv.wait(lk, [&] { return stop || !queue.empty(); });
            else // a launch is on the GPU: wake for new requests or to look at it again
                cv.wait_for(lk, std::chrono::microseconds(20), [&] { return stop || !queue.empty(); });
        }
    }
};

extern "C" {

svdag_status svdag_server_create(svdag_ctx* ctx, const svdag_server_config* config, svdag_server** out)
{
    if (!ctx || !config || !out || config->frame.width == 0 || config->frame.height == 0)
        return SVDAG_ERR_INVALID;
    SVDAG_CUDA(cudaSetDevice(ctx->device));
    SVDAG_TRY(ensure_level_tables(ctx, nullptr));
    SVDAG_CUDA(cudaStreamSynchronize(nullptr));
    auto* s = new svdag_server();
    s->ctx = ctx;
    s->cfg = *config;
    s->t0 = Clock::now();
    s->nslots = 4;
    s->slotBytes = (ctx->batchBytes / s->nslots) & ~(size_t)255;
    s->capBytes = ctx->itemWords * 4ull;
    if (config->memory_cap_bytes)
        s->capBytes = std::min<unsigned long long>(s->capBytes, config->memory_cap_bytes);
    s->frameHits = (size_t)config->frame.width * config->frame.height;
    svdag_status st = SVDAG_OK;
    auto fail = [&](cudaError_t e) {
        if (e != cudaSuccess && st == SVDAG_OK)
            st = cuda_status(e);
    };
    fail(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    fail(cudaMalloc(&s->hits, s->frameHits * sizeof(svdag_hit)));
    if (config->flags & SVDAG_SERVE_COPY_FRAMES)
        fail(cudaMallocHost(&s->hostHits, s->frameHits * sizeof(svdag_hit)));
    const size_t maxRecords = s->slotBytes / (sizeof(DevEditor) + sizeof(EditRecord));
    for (uint32_t i = 0; i < s->nslots; ++i) {
        EditRecord* r = nullptr;
        unsigned long long* t = nullptr;
        cudaEvent_t ev = nullptr;
        fail(cudaMallocHost(&r, maxRecords * sizeof(EditRecord)));
        fail(cudaMallocHost(&t, sizeof(unsigned long long)));
        fail(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        s->hostRecords.push_back(r);
        s->hostTop.push_back(t);
        s->events.push_back(ev);
    }
    {
        unsigned long long top = 0;
        fail(cudaMemcpy(&top, &ctx->ctl->itemTop, sizeof(top), cudaMemcpyDeviceToHost));
        s->usedBytes = top * 4ull;
    }
    if (st != SVDAG_OK) {
        s->stop = true;
        svdag_server_destroy(s);
        return st;
    }
    if (s->cfg.max_batch > maxRecords / 2)
        s->cfg.max_batch = (uint32_t)(maxRecords / 2);
    s->worker = std::thread([s] {
        cudaSetDevice(s->ctx->device);
        s->run();
    });
    *out = s;
    return SVDAG_OK;
}

svdag_status svdag_server_destroy(svdag_server* s)
{
    if (!s)
        return SVDAG_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable())
        s->worker.join();
    if (s->stream)
        cudaStreamSynchronize(s->stream);
    for (auto* r : s->hostRecords)
        cudaFreeHost(r);
    for (auto* t : s->hostTop)
        cudaFreeHost(t);
    for (auto ev : s->events)
        cudaEventDestroy(ev);
    if (s->hostHits)
        cudaFreeHost(s->hostHits);
    if (s->hits)
        cudaFree(s->hits);
    if (s->stream)
        cudaStreamDestroy(s->stream);
    const svdag_status st = s->fatal;
    delete s;
    return st;
}

svdag_status svdag_submit_edit(svdag_server* s, const svdag_edit* e, uint64_t* ticket)
{
    if (!s || !ticket || !valid_edit(e))
        return SVDAG_ERR_INVALID;
    Request r {};
    r.kind = 0;
    r.edit = *e;
    r.reserve = edit_reserve_bytes(*e, s->ctx->cfg.levels);
    {
        std::lock_guard<std::mutex> lk(s->m);
        if (s->stop)
            return SVDAG_ERR_INVALID;
        r.ticket = s->nextTicket++;
        r.submit = now_since(s->t0);
        s->queue.push_back(r);
    }
    s->cv.notify_one();
    *ticket = r.ticket;
    return SVDAG_OK;
}

svdag_status svdag_submit_frame(svdag_server* s, const svdag_trace_params* p, uint64_t* ticket)
{
    if (!s || !ticket)
        return SVDAG_ERR_INVALID;
    Request r {};
    r.kind = 1;
    r.frame = p ? *p : s->cfg.frame;
    if ((size_t)r.frame.width * r.frame.height > s->frameHits || r.frame.width == 0 || r.frame.height == 0)
        return SVDAG_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->m);
        if (s->stop)
            return SVDAG_ERR_INVALID;
        r.ticket = s->nextTicket++;
        r.submit = now_since(s->t0);
        s->queue.push_back(r);
    }
    s->cv.notify_one();
    *ticket = r.ticket;
    return SVDAG_OK;
}

svdag_status svdag_poll(svdag_server* s, uint64_t ticket, int wait, svdag_request_result* out)
{
    if (!s || !out)
        return SVDAG_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->m);
    if (ticket == 0 || ticket >= s->nextTicket)
        return SVDAG_ERR_INVALID;
    auto it = s->done.find(ticket);
    if (it == s->done.end()) {
        if (!wait)
            return SVDAG_ERR_BUSY;
        s->doneCv.wait(lk, [&] { return s->done.count(ticket) != 0; });
        it = s->done.find(ticket);
    }
    *out = it->second;
    s->done.erase(it);
    return SVDAG_OK;
}

svdag_status svdag_server_frame(svdag_server* s, svdag_hit* out, uint64_t capacity)
{
    if (!s || !out || !s->hostHits || capacity < s->frameHits)
        return SVDAG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->m);
    std::memcpy(out, s->hostHits, s->frameHits * sizeof(svdag_hit));
    return SVDAG_OK;
}

svdag_status svdag_server_replay(svdag_server* s, const svdag_edit* edits, const double* editTimes, uint32_t nEdits,
    const double* frameTimes, uint32_t nFrames, svdag_request_result* results)
{
    if (!s || !results || (nEdits && (!edits || !editTimes)) || (nFrames && !frameTimes))
        return SVDAG_ERR_INVALID;
    for (uint32_t i = 0; i < nEdits; ++i)
        if (!valid_edit(&edits[i]))
            return SVDAG_ERR_INVALID;
    std::vector<uint64_t> tickets(nEdits + nFrames, 0);
    const Clock::time_point start = Clock::now();
    uint32_t ie = 0, jf = 0;
    while (ie < nEdits || jf < nFrames) {
        const bool edit = jf >= nFrames || (ie < nEdits && editTimes[ie] <= frameTimes[jf]);
        const double at = edit ? editTimes[ie] : frameTimes[jf];
        std::this_thread::sleep_until(start + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(at)));
        if (edit) {
            SVDAG_TRY(svdag_submit_edit(s, &edits[ie], &tickets[ie]));
            ++ie;
        } else {
            SVDAG_TRY(svdag_submit_frame(s, nullptr, &tickets[nEdits + jf]));
            ++jf;
        }
    }
    for (uint32_t i = 0; i < nEdits + nFrames; ++i)
        SVDAG_TRY(svdag_poll(s, tickets[i], 1, &results[i]));
    return SVDAG_OK;
}

} // extern "C"
