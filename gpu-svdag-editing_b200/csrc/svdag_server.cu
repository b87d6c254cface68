// svdag_server.cu - the serving form: a request loop on its own host thread with continuous batching
// of edits into batched launches on one stream, frames on a second stream (one in flight at a time,
// each behind every batch launched before it, so the GPU renders while the next batch edits),
// admission by reserved item-region memory, garbage collection in the loop when that memory fills,
// and a timed replay driver. SVDAG_SERVE_PLAIN turns the loop into the per-edit baseline (one
// request at a time: an edit, then its frame, synchronously).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
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
#include "svdag_serve_geometry.h"
#include "svdag_host.hpp"

using namespace svdag;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket;
    uint32_t kind; // 0 edit, 1 frame, 2 undo, 3 redo
    svdag_edit edit;
    svdag_trace_params frame;
    double submit;
    unsigned long long reserve; // admission estimate (edits)
};

// An edit launch: its requests, where its records are, and what they said once it finished.
struct Batch {
    std::vector<Request> reqs;
    std::vector<uint32_t> lastRecord; // per request: index of its last record
    std::vector<EditRecord> records; // copied from the slot's pinned buffer when the launch finished
    uint32_t slot = 0;
    uint32_t launch = 0;
    uint32_t root = 0; // undo/redo launches: the root they left
    unsigned long long reserved = 0;
    cudaEvent_t done = nullptr;
    bool finished = false;
};

double now_since(Clock::time_point t0) { return std::chrono::duration<double>(Clock::now() - t0).count(); }

constexpr uint32_t kMaxFrameBoxes = 512; // changed regions one incremental frame tests; more: a whole frame
constexpr uint32_t kMaxCopyRuns = 16; // row runs copied to the host after an incremental frame; more: the whole frame

using serve::box_rows;
using serve::edit_boxes;
using serve::edit_reserve_bytes;

} // namespace

struct svdag_server {
    svdag_ctx* ctx = nullptr;
    svdag_server_config cfg {};
    Clock::time_point t0;
    cudaStream_t stream = nullptr; // edit launches
    cudaStream_t frameStream = nullptr; // frames
    svdag_hit* hits = nullptr; // device frame
    svdag_hit* hostHits = nullptr; // pinned copy (SVDAG_SERVE_COPY_FRAMES)
    size_t frameHits = 0;
    uint32_t nslots = 0;
    size_t slotBytes = 0;
    std::vector<EditRecord*> hostRecords; // pinned, one array per slot
    std::vector<MemSnapshot*> hostMem; // pinned head of the control block after each launch
    std::vector<uint32_t*> hostRoot; // pinned root after each undo/redo launch
    std::vector<cudaEvent_t> events; // one per slot
    cudaEvent_t frameDone = nullptr;
    uint32_t* frameRoot = nullptr; // root the frame in flight shows (batches may commit meanwhile)
    float* boxesDev = nullptr; // changed regions of an incremental frame
    float* boxesHost = nullptr; // pinned staging (one frame in flight: reused only after it finished)
    bool haveFrame = false; // `hits` holds a frame of lastFrame's camera
    std::atomic<unsigned long long> framesWhole { 0 }, framesIncremental { 0 }, frameBytesToHost { 0 };
    unsigned long long capBytes = 0;
    std::atomic<unsigned long long> usedBytes { 0 }; // item and header region in use after the last finished launch
    unsigned long long gcThreshold = 0; // configured threshold
    unsigned long long gcTrigger = 0; // bytes in use that start the next collection
    // Slots a collection frees stay in their slabs (only overflow slabs left empty go back), so the
    // bump-pointer bytes in use stay high after it while inserts fill those slots. The credit is
    // the slot bytes the last collection freed (16 per item, the smallest slot) less 50 per item
    // inserted since (the largest); memory pressure is the bytes in use less the credit.
    std::atomic<unsigned long long> reuseCredit { 0 };
    bool dirtySinceGc = true; // a launch finished since the last collection (one could free something)
    bool gcWanted = false; // admit nothing until the GPU is idle, then collect
    // Memory counters: written by the worker thread, read by svdag_server_memory_stats.
    std::atomic<unsigned long long> gcRuns { 0 }, gcFreedBytes { 0 }, rejectedEdits { 0 }, failedEdits { 0 };
    std::atomic<double> gcSeconds { 0.0 };

    std::mutex m;
    std::condition_variable cv, doneCv;
    std::deque<Request> queue;
    std::unordered_map<uint64_t, svdag_request_result> done;
    uint64_t nextTicket = 1;
    bool stop = false;
    svdag_status fatal = SVDAG_OK;
    // Worker-thread state: launched batches not yet shown by a finished frame, the frame in flight
    // (it shows every batch launched before it) and the frame requests it will answer.
    std::deque<Batch> batches;
    bool frameActive = false;
    uint32_t frameCovers = 0; // batches with launch < frameCovers are shown by the frame in flight
    uint32_t covered = 0; // batches with launch < covered have a frame launched behind them
    std::vector<Request> frameReqs, pendingFrames;
    svdag_trace_params lastFrame {}; // camera of the last frame launched
    uint32_t launches = 0;
    std::thread worker;

    bool plain() const { return cfg.flags & SVDAG_SERVE_PLAIN; }
    unsigned long long pressure() const
    {
        const unsigned long long u = usedBytes.load(), c = reuseCredit.load();
        return u > c ? u - c : 0ull;
    }
    bool gcAllowed() const { return !(cfg.flags & SVDAG_SERVE_NO_GC); }

    // A collection that keeps every undo/redo root (nothing of the context may be on the GPU), then
    // the bytes in use it left. Runs on the worker thread; the loop admits nothing meanwhile.
    svdag_status collect_garbage()
    {
        const Clock::time_point a = Clock::now();
        const svdag_status st = svdag_gc_keep_history(ctx, stream);
        MemSnapshot ms {};
        unsigned long long freedItems = 0;
        SVDAG_CUDA(cudaMemcpyAsync(&ms, &ctx->ctl->itemTop, sizeof(ms), cudaMemcpyDeviceToHost, stream));
        SVDAG_CUDA(cudaMemcpyAsync(&freedItems, &ctx->ctl->gcFreedItems, sizeof(freedItems), cudaMemcpyDeviceToHost, stream));
        SVDAG_CUDA(cudaStreamSynchronize(stream));
        if (st == SVDAG_OK)
            reuseCredit = freedItems * 16ull;
        const unsigned long long before = usedBytes;
        usedBytes = used_region_bytes(ctx, ms.itemTop, ms.headerTop, ms.freeBytes);
        gcSeconds.store(gcSeconds.load() + std::chrono::duration<double>(Clock::now() - a).count());
        ++gcRuns;
        gcFreedBytes += before > usedBytes ? before - usedBytes : 0ull;
        // The next collection waits until a quarter of the room left above what this one kept has
        // filled, so that live data near the threshold does not start a collection per launch.
        const unsigned long long kept = pressure();
        gcTrigger = std::max(gcThreshold, kept < capBytes ? kept + (capBytes - kept) / 4 : capBytes);
        dirtySinceGc = false;
        gcWanted = false;
        return st;
    }

    svdag_status launch_batch(std::vector<Request>& reqs, unsigned long long reserved)
    {
        Batch b;
        b.slot = launches % nslots;
        b.launch = launches++;
        b.reserved = reserved;
        b.done = events[b.slot];
        if (reqs.size() == 1 && reqs[0].kind >= 2) { // an undo or redo is a launch of its own
            SVDAG_TRY(reqs[0].kind == 2 ? svdag_undo(ctx, stream) : svdag_redo(ctx, stream));
            SVDAG_CUDA(cudaMemcpyAsync(hostRoot[b.slot], &ctx->ctl->root, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            SVDAG_CUDA(cudaMemcpyAsync(hostMem[b.slot], &ctx->ctl->itemTop, sizeof(MemSnapshot), cudaMemcpyDeviceToHost, stream));
            SVDAG_CUDA(cudaEventRecord(b.done, stream));
            b.reqs = std::move(reqs);
            batches.push_back(std::move(b));
            return SVDAG_OK;
        }
        std::vector<DevEditor> eds;
        for (auto& r : reqs) {
            DevEditor tmp[2];
            const int n = expand_edit(ctx, r.edit, tmp);
            eds.insert(eds.end(), tmp, tmp + n);
            b.lastRecord.push_back((uint32_t)eds.size() - 1);
        }
        char* region = ctx->batch + (size_t)b.slot * slotBytes;
        SVDAG_TRY(launch_edits_at(ctx, eds.data(), (uint32_t)eds.size(), region, slotBytes, stream));
        const size_t edBytes = align256(eds.size() * sizeof(DevEditor));
        b.records.resize(eds.size());
        SVDAG_CUDA(cudaMemcpyAsync(hostRecords[b.slot], region + edBytes, eds.size() * sizeof(EditRecord), cudaMemcpyDeviceToHost, stream));
        SVDAG_CUDA(cudaMemcpyAsync(hostMem[b.slot], &ctx->ctl->itemTop, sizeof(MemSnapshot), cudaMemcpyDeviceToHost, stream));
        SVDAG_CUDA(cudaEventRecord(b.done, stream));
        b.reqs = std::move(reqs);
        batches.push_back(std::move(b));
        return SVDAG_OK;
    }

    // A frame of the newest state, behind every batch launched so far.
    svdag_status launch_frame()
    {
        if (!batches.empty() && batches.back().launch >= covered)
            SVDAG_CUDA(cudaStreamWaitEvent(frameStream, batches.back().done, 0));
        svdag_trace_params frame = cfg.frame;
        for (auto& r : pendingFrames)
            frame = r.frame;
        if ((size_t)frame.width * frame.height > frameHits || frame.width == 0 || frame.height == 0)
            frame = cfg.frame;
        SVDAG_CUDA(cudaMemcpyAsync(frameRoot, &ctx->ctl->root, sizeof(uint32_t), cudaMemcpyDeviceToDevice, frameStream));
        // Incremental when the camera is the last frame's and only edits ran since (the batches from
        // `covered` on are the ones launched after that frame).
        bool whole = plain() || (cfg.flags & SVDAG_SERVE_FULL_FRAMES) || !haveFrame
            || std::memcmp(&frame, &lastFrame, sizeof(frame)) != 0;
        uint32_t nBoxes = 0;
        for (auto it = batches.begin(); !whole && it != batches.end(); ++it) {
            if (it->launch < covered)
                continue;
            for (auto& r : it->reqs) {
                if (r.kind != 0 || nBoxes + 2 > kMaxFrameBoxes) {
                    whole = true;
                    break;
                }
                nBoxes += edit_boxes(r.edit, boxesHost + 6 * nBoxes);
            }
        }
        if (whole) {
            SVDAG_TRY(trace_frame(ctx, &frame, hits, frameRoot, frameStream));
        } else {
            if (nBoxes)
                SVDAG_CUDA(cudaMemcpyAsync(boxesDev, boxesHost, nBoxes * 6 * sizeof(float), cudaMemcpyHostToDevice, frameStream));
            SVDAG_TRY(trace_frame_incremental(ctx, &frame, hits, frameRoot, boxesDev, nBoxes, frameStream));
        }
        haveFrame = true;
        lastFrame = frame;
        (whole ? framesWhole : framesIncremental).fetch_add(1);
        if (cfg.flags & SVDAG_SERVE_COPY_FRAMES) {
            // After an incremental frame only the pixels its boxes project to can differ from the host
            // copy of the previous frame: runs of rows, each with the union of its boxes' columns,
            // copied as one rectangle each.
            struct Run {
                int64_t r0, r1, c0, c1;
            };
            std::vector<Run> runs;
            bool all = whole;
            for (uint32_t b = 0; b < nBoxes && !all; ++b) {
                Run r {};
                if (!box_rows(frame, boxesHost + 6 * b, r.r0, r.r1, r.c0, r.c1))
                    all = true;
                else if (r.r0 <= r.r1 && r.c0 <= r.c1)
                    runs.push_back(r);
            }
            std::sort(runs.begin(), runs.end(), [](const Run& a, const Run& b) { return a.r0 < b.r0; });
            std::vector<Run> merged;
            for (auto& r : runs) {
                if (!merged.empty() && r.r0 <= merged.back().r1 + 1) {
                    Run& m = merged.back();
                    m.r1 = std::max(m.r1, r.r1);
                    m.c0 = std::min(m.c0, r.c0);
                    m.c1 = std::max(m.c1, r.c1);
                } else {
                    merged.push_back(r);
                }
            }
            if (merged.size() > kMaxCopyRuns)
                all = true;
            const size_t rowBytes = (size_t)frame.width * sizeof(svdag_hit);
            if (all) {
                SVDAG_CUDA(cudaMemcpyAsync(hostHits, hits, rowBytes * frame.height, cudaMemcpyDeviceToHost, frameStream));
                frameBytesToHost.fetch_add(rowBytes * frame.height);
            } else {
                for (auto& r : merged) {
                    frameBytesToHost.fetch_add(sizeof(svdag_hit) * (size_t)(r.c1 - r.c0 + 1) * (size_t)(r.r1 - r.r0 + 1));
                    const size_t off = rowBytes * (size_t)r.r0 + sizeof(svdag_hit) * (size_t)r.c0;
                    SVDAG_CUDA(cudaMemcpy2DAsync(reinterpret_cast<char*>(hostHits) + off, rowBytes, reinterpret_cast<const char*>(hits) + off,
                        rowBytes, sizeof(svdag_hit) * (size_t)(r.c1 - r.c0 + 1), (size_t)(r.r1 - r.r0 + 1), cudaMemcpyDeviceToHost,
                        frameStream));
                }
            }
        }
        SVDAG_CUDA(cudaEventRecord(frameDone, frameStream));
        frameActive = true;
        frameCovers = covered = launches;
        frameReqs = std::move(pendingFrames);
        pendingFrames.clear();
        return SVDAG_OK;
    }

    void finish_batch(Batch& b)
    {
        if (b.finished)
            return;
        std::memcpy(b.records.data(), hostRecords[b.slot], b.records.size() * sizeof(EditRecord));
        if (b.records.empty())
            b.root = *hostRoot[b.slot];
        const MemSnapshot& ms = *hostMem[b.slot];
        usedBytes = used_region_bytes(ctx, ms.itemTop, ms.headerTop, ms.freeBytes);
        for (size_t i = 0; i < b.lastRecord.size(); ++i)
            failedEdits += b.records[b.lastRecord[i]].status != 0 ? 1u : 0u;
        unsigned long long added = 0;
        for (const EditRecord& r : b.records)
            added += r.added;
        const unsigned long long c = reuseCredit.load();
        reuseCredit = c > 50ull * added ? c - 50ull * added : 0ull;
        dirtySinceGc = true;
        b.finished = true;
    }

    // Results of the batches the finished frame shows and of the frame requests it answers.
    void complete_frame()
    {
        const double t = now_since(t0);
        std::lock_guard<std::mutex> lk(m);
        while (!batches.empty() && batches.front().launch < frameCovers) {
            Batch& b = batches.front();
            finish_batch(b); // its event completed before the frame ran
            for (size_t i = 0; i < b.reqs.size(); ++i) {
                const Request& r = b.reqs[i];
                svdag_request_result out {};
                out.ticket = r.ticket;
                out.kind = r.kind;
                out.launch = b.launch;
                out.submit_s = r.submit;
                out.visible_s = t;
                if (r.kind >= 2) {
                    out.root_after = b.root;
                    done[r.ticket] = out;
                    continue;
                }
                const EditRecord& e = b.records[b.lastRecord[i]];
                out.status = e.status;
                if (r.edit.tool == SVDAG_TOOL_MOVE && b.lastRecord[i] > 0 && b.records[b.lastRecord[i] - 1].status)
                    out.status = b.records[b.lastRecord[i] - 1].status;
                out.root_after = e.rootAfter;
                out.edited_voxels = e.edited;
                done[r.ticket] = out;
            }
            batches.pop_front();
        }
        for (auto& r : frameReqs) {
            svdag_request_result out {};
            out.ticket = r.ticket;
            out.kind = 1;
            out.launch = frameCovers;
            out.submit_s = r.submit;
            out.visible_s = t;
            done[r.ticket] = out;
        }
        frameReqs.clear();
        frameActive = false;
        doneCv.notify_all();
    }

    unsigned long long reserved_in_flight() const
    {
        unsigned long long s = 0;
        for (auto& b : batches)
            if (!b.finished)
                s += b.reserved;
        return s;
    }
    uint32_t unfinished() const
    {
        uint32_t n = 0;
        for (auto& b : batches)
            n += b.finished ? 0u : 1u;
        return n;
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
    void fail_everything(svdag_status st)
    {
        std::lock_guard<std::mutex> lk(m);
        fatal = st;
        for (auto& b : batches)
            fail_requests(b.reqs, st);
        batches.clear();
        fail_requests(frameReqs, st);
        fail_requests(pendingFrames, st);
        frameReqs.clear();
        pendingFrames.clear();
        frameActive = false;
    }

    // The per-edit baseline: one request, then its frame, synchronously.
    void run_plain()
    {
        for (;;) {
            Request r;
            {
                std::unique_lock<std::mutex> lk(m);
                cv.wait(lk, [&] { return stop || !queue.empty(); });
                if (queue.empty())
                    break;
                r = queue.front();
                queue.pop_front();
            }
            std::vector<Request> one { r };
            svdag_status st = SVDAG_OK;
            if (r.kind == 0 && gcAllowed() && dirtySinceGc && (pressure() > gcTrigger || pressure() + r.reserve > capBytes))
                collect_garbage(); // a failed collection frees nothing; the edit is then admitted or refused as it is
            if (r.kind == 0 && pressure() + r.reserve > capBytes) {
                std::lock_guard<std::mutex> lk(m);
                ++rejectedEdits;
                fail_requests(one, SVDAG_ERR_OOM);
                continue;
            }
            if (r.kind != 1) // an edit, undo or redo
                st = launch_batch(one, r.reserve);
            else
                pendingFrames.push_back(r);
            if (st == SVDAG_OK)
                st = launch_frame();
            if (st == SVDAG_OK && cudaEventSynchronize(frameDone) != cudaSuccess)
                st = SVDAG_ERR_CUDA;
            if (st != SVDAG_OK) {
                if (r.kind != 1 && batches.empty()) {
                    std::lock_guard<std::mutex> lk(m);
                    fail_requests(one, st);
                }
                fail_everything(st);
                continue;
            }
            complete_frame();
        }
    }

    void run()
    {
        if (plain()) {
            run_plain();
            return;
        }
        const uint32_t maxBatch = cfg.max_batch ? cfg.max_batch : 256u;
        const uint32_t maxInflight = std::min<uint32_t>(cfg.max_inflight ? cfg.max_inflight : 2u, nslots - 1);
        for (;;) {
            // Finished launches (records, memory in use), then a finished frame.
            for (auto& b : batches)
                if (!b.finished && cudaEventQuery(b.done) == cudaSuccess)
                    finish_batch(b);
            if (frameActive && cudaEventQuery(frameDone) == cudaSuccess)
                complete_frame();
            // Memory: past the threshold, admit nothing until the launches and the frame in flight
            // are done, then collect (every undo/redo root kept).
            if (gcAllowed() && dirtySinceGc && pressure() > gcTrigger)
                gcWanted = true;
            if (gcWanted && unfinished() == 0 && !frameActive) {
                collect_garbage(); // a failed collection frees nothing; admission then weighs edits as they are
                continue;
            }
            std::vector<Request> take;
            unsigned long long reserve = 0;
            {
                std::unique_lock<std::mutex> lk(m);
                if (stop && queue.empty() && batches.empty() && !frameActive && pendingFrames.empty())
                    break;
                const bool canLaunch = unfinished() < maxInflight && !gcWanted;
                const unsigned long long inUse = pressure() + reserved_in_flight();
                uint32_t edits = 0;
                for (auto it = queue.begin(); it != queue.end();) {
                    if (it->kind == 1) { // answered by the next frame
                        pendingFrames.push_back(*it);
                        it = queue.erase(it);
                        continue;
                    }
                    if (it->kind >= 2) { // undo/redo: a launch of its own, after the edits before it
                        if (canLaunch && edits == 0) {
                            take.push_back(*it);
                            queue.erase(it);
                        }
                        break;
                    }
                    if (!canLaunch || edits == maxBatch)
                        break;
                    if (inUse + reserve + it->reserve > capBytes) {
                        // Does not fit. With launches in flight, wait for them; with nothing in flight
                        // only a collection can make room, and after one the edit fails up front.
                        if (edits == 0 && unfinished() == 0) {
                            if (gcAllowed() && dirtySinceGc) {
                                gcWanted = true;
                            } else {
                                ++rejectedEdits;
                                fail_requests({ *it }, SVDAG_ERR_OOM);
                                it = queue.erase(it);
                                continue;
                            }
                        }
                        break;
                    }
                    reserve += it->reserve;
                    ++edits;
                    take.push_back(*it);
                    it = queue.erase(it);
                }
            }
            bool launched = false;
            if (!take.empty()) {
                if (launch_batch(take, reserve) != SVDAG_OK) {
                    std::lock_guard<std::mutex> lk(m);
                    fail_requests(take, SVDAG_ERR_CUDA);
                    continue;
                }
                launched = true;
            }
            // One frame in flight at a time, behind everything launched so far.
            // (While a collection waits, frames run only to show launched edits.)
            const bool uncovered = !batches.empty() && batches.back().launch >= covered;
            if (!frameActive && (uncovered || (!pendingFrames.empty() && !gcWanted))) {
                if (launch_frame() != SVDAG_OK) {
                    fail_everything(SVDAG_ERR_CUDA);
                    continue;
                }
                launched = true;
            }
            if (launched)
                continue;
            std::unique_lock<std::mutex> lk(m);
            if (batches.empty() && !frameActive && pendingFrames.empty())
                cv.wait(lk, [&] { return stop || !queue.empty(); });
            else // work on the GPU: wake for new requests or to look at it again
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
    fail(cudaStreamCreateWithFlags(&s->frameStream, cudaStreamNonBlocking));
    fail(cudaEventCreateWithFlags(&s->frameDone, cudaEventDisableTiming));
    fail(cudaMalloc(&s->frameRoot, 256));
    fail(cudaMalloc(&s->boxesDev, kMaxFrameBoxes * 6 * sizeof(float)));
    fail(cudaMallocHost(&s->boxesHost, kMaxFrameBoxes * 6 * sizeof(float)));
    fail(cudaMalloc(&s->hits, s->frameHits * sizeof(svdag_hit)));
    if (config->flags & SVDAG_SERVE_COPY_FRAMES)
        fail(cudaMallocHost(&s->hostHits, s->frameHits * sizeof(svdag_hit)));
    const size_t maxRecords = s->slotBytes / (sizeof(DevEditor) + sizeof(EditRecord));
    for (uint32_t i = 0; i < s->nslots; ++i) {
        EditRecord* r = nullptr;
        MemSnapshot* t = nullptr;
        uint32_t* root = nullptr;
        cudaEvent_t ev = nullptr;
        fail(cudaMallocHost(&r, maxRecords * sizeof(EditRecord)));
        fail(cudaMallocHost(&t, sizeof(MemSnapshot)));
        fail(cudaMallocHost(&root, sizeof(uint32_t)));
        fail(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        s->hostRecords.push_back(r);
        s->hostMem.push_back(t);
        s->hostRoot.push_back(root);
        s->events.push_back(ev);
    }
    {
        MemSnapshot ms {};
        fail(cudaMemcpy(&ms, &ctx->ctl->itemTop, sizeof(ms), cudaMemcpyDeviceToHost));
        s->usedBytes = used_region_bytes(ctx, ms.itemTop, ms.headerTop, ms.freeBytes);
    }
    // Default: collect when less than 1/32 of the cap (at least 1 GiB, at most an eighth) is left.
    const unsigned long long room = std::min(s->capBytes / 8, std::max(s->capBytes / 32, 1ull << 30));
    s->gcThreshold = config->gc_threshold_bytes ? config->gc_threshold_bytes : s->capBytes - room;
    s->gcTrigger = s->gcThreshold;
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
    if (s->frameStream)
        cudaStreamSynchronize(s->frameStream);
    for (auto* r : s->hostRecords)
        cudaFreeHost(r);
    for (auto* t : s->hostMem)
        cudaFreeHost(t);
    for (auto* r : s->hostRoot)
        cudaFreeHost(r);
    for (auto ev : s->events)
        cudaEventDestroy(ev);
    if (s->hostHits)
        cudaFreeHost(s->hostHits);
    if (s->hits)
        cudaFree(s->hits);
    if (s->frameRoot)
        cudaFree(s->frameRoot);
    if (s->boxesDev)
        cudaFree(s->boxesDev);
    if (s->boxesHost)
        cudaFreeHost(s->boxesHost);
    if (s->frameDone)
        cudaEventDestroy(s->frameDone);
    if (s->stream)
        cudaStreamDestroy(s->stream);
    if (s->frameStream)
        cudaStreamDestroy(s->frameStream);
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

svdag_status svdag_server_counters(svdag_server* s, uint64_t* whole, uint64_t* incremental, uint64_t* bytesToHost)
{
    if (!s)
        return SVDAG_ERR_INVALID;
    if (whole)
        *whole = s->framesWhole.load();
    if (incremental)
        *incremental = s->framesIncremental.load();
    if (bytesToHost)
        *bytesToHost = s->frameBytesToHost.load();
    return SVDAG_OK;
}

svdag_status svdag_server_memory_stats(svdag_server* s, svdag_server_memory* out)
{
    if (!s || !out)
        return SVDAG_ERR_INVALID;
    svdag_server_memory r {};
    r.used_bytes = s->usedBytes.load();
    r.cap_bytes = s->capBytes;
    r.gc_threshold_bytes = s->gcThreshold;
    r.gc_runs = s->gcRuns.load();
    r.gc_freed_bytes = s->gcFreedBytes.load();
    r.gc_seconds = s->gcSeconds.load();
    r.rejected_edits = s->rejectedEdits.load();
    r.failed_edits = s->failedEdits.load();
    r.reuse_credit_bytes = s->reuseCredit.load();
    *out = r;
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

svdag_status svdag_submit_undo(svdag_server* s, int redo, uint64_t* ticket)
{
    if (!s || !ticket)
        return SVDAG_ERR_INVALID;
    Request r {};
    r.kind = redo ? 3u : 2u;
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

svdag_status svdag_server_replay_actions(svdag_server* s, const svdag_replay_action* actions, uint64_t n, double period,
    const svdag_trace_params* frames, svdag_request_result* results)
{
    if (!s || !results || (n && !actions) || !(period >= 0.0))
        return SVDAG_ERR_INVALID;
    for (uint64_t i = 0; i < n; ++i)
        if (actions[i].kind == SVDAG_REPLAY_EDIT && !valid_edit(&actions[i].edit))
            return SVDAG_ERR_INVALID;
    std::vector<uint64_t> tickets(n, 0);
    const Clock::time_point start = Clock::now();
    uint64_t frame = 0;
    for (uint64_t i = 0; i < n; ++i) {
        switch (actions[i].kind) {
        case SVDAG_REPLAY_EDIT:
            SVDAG_TRY(svdag_submit_edit(s, &actions[i].edit, &tickets[i]));
            break;
        case SVDAG_REPLAY_UNDO:
        case SVDAG_REPLAY_REDO:
            SVDAG_TRY(svdag_submit_undo(s, actions[i].kind == SVDAG_REPLAY_REDO, &tickets[i]));
            break;
        case SVDAG_REPLAY_END_FRAME:
            SVDAG_TRY(svdag_submit_frame(s, frames ? &frames[frame] : nullptr, &tickets[i]));
            ++frame;
            std::this_thread::sleep_until(
                start + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(period * (double)frame)));
            break;
        default:
            break;
        }
    }
    for (uint64_t i = 0; i < n; ++i) {
        if (tickets[i])
            SVDAG_TRY(svdag_poll(s, tickets[i], 1, &results[i]));
        else
            results[i] = svdag_request_result {};
    }
    return SVDAG_OK;
}

} // extern "C"
