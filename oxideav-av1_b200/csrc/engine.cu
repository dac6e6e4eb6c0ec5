// engine.cu — the serving engine: streams with device-resident reference
// slots, tickets, and a step loop that batches one frame of every ready
// stream into shared launches.
//
// The reference decodes one stream on one thread: per frame the tile walk
// reconstructs (prediction + residual), then decode_frame_spec_tiles runs the
// §7.4 chain, stores the pre-grain frame in the refreshed §7.20 slots
// (reference_frame_update, src/decoder/frame_driver.rs:1409) and returns the
// output frame (frame_driver.rs:1101-1116, output_existing_frame at 1495).
//
// Worker threads ("lanes", each with its own CUDA stream; a stream of frames
// belongs to one lane) form steps: a lane takes the oldest pending frame of
// each of its streams that has one (up to max_batch frames, round robin, and
// while their luma samples stay within max_step_samples), and
// enqueues for the whole step one inter launch, one residual launch, the
// intra wavefront and the post-filter chain (one launch per stage), then the
// slot refreshes and the output copies, on its CUDA stream; lanes overlap
// their host preparation and their device work.  A stream's next frame can
// join the very next step: its references are the slot buffers the previous
// step writes, and stream order on the device keeps the two in sequence.  A
// completion thread retires steps in order through their events and wakes
// pollers.  Frames that arrive while steps run join the next step (continuous
// batching); streams are admitted while their eight reference slots fit the
// HBM budget, and a frame waits for work memory to free up.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace av1g {
av1g_status recon_run(const av1g_recon_job* jobs, int n, cudaStream_t s, std::string& err);
av1g_status intra_run(const av1g_intra_job* jobs, int n, cudaStream_t s, std::string& err);
av1g_status intra_run_status(const av1g_intra_job* jobs, int n, cudaStream_t s, std::string& err,
                             int32_t* frame_status);
av1g_status inter_run(const av1g_inter_job* jobs, int n, cudaStream_t s, std::string& err);
av1g_status postfilter_run(const av1g_frame_job* jobs, int n, cudaStream_t s, std::string& err);
av1g_status postfilter_result_planes(const av1g_frame_job& j, PlaneDev pre[3], PlaneDev out[3], std::string& err);
void set_last_error_text(const std::string& s);  // the C ABI's thread-local error text (api.cu)
}  // namespace av1g

using namespace av1g;
using Clock = std::chrono::steady_clock;

namespace {

// Makes a device current for a scope and restores the caller's afterwards.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

size_t pitch_of(int w, int bps) { return ((size_t)w * bps + 63) & ~(size_t)63; }
size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
int r2u(int v, int s) { return (v + s) >> s; }

// One §7.20 slot payload on the device: the cropped pre-grain planes plus what
// output_existing_frame needs (grain parameters, format).
struct SlotBuf {
    av1g_engine* eng = nullptr;
    cudaStream_t cs = nullptr;  // the lane stream every use of the slot is ordered on
    uint8_t* dev = nullptr;
    size_t bytes = 0;
    av1g_plane planes[3] = {};
    int32_t upscaled_width = 0, frame_height = 0;
    av1g_film_grain grain = {};
    uint8_t bit_depth = 8, ssx = 1, ssy = 1, num_planes = 3, matrix_coefficients = 0;
    ~SlotBuf();
};

struct Ticket {
    uint64_t id = 0;
    av1g_stream* st = nullptr;
    bool reset_marker = false;     // av1g_stream_reset_refs in submission order
    bool done = false;
    av1g_status status = AV1G_OK;
    std::string err;
    // host copy of the descriptor
    av1g_frame_header hdr = {};
    av1g_quant_params quant = {};
    // the device-bound arrays (grids 0-8, CDEF indices 9, LR units 10-12,
    // coefficients 13), laid out at submit in one pinned block that the
    // frame's step copies to its allocation with one cudaMemcpyAsync; the
    // block goes back to the pool when that step has finished
    uint8_t* blob = nullptr;
    size_t blob_bytes = 0;
    size_t blob_off[14] = {}, blob_len[14] = {};
    std::vector<av1g_inter_pred> preds;
    std::vector<av1g_obmc_neighbour> nbs;
    std::vector<av1g_warp_ctx> warps;
    std::vector<av1g_tu> inter_tus;
    std::vector<av1g_intra_tu> intra_tus;
    std::vector<uint8_t> maps;
    std::vector<int32_t> coeffs;
    uint8_t ref_frame_idx[7] = {};
    uint8_t refresh = 0, show = 0, show_existing = 0, show_idx = 0;
    bool has_interintra = false;  // inter halves wait in side planes for the intra pass
    // output
    uint8_t* host_out = nullptr;
    size_t host_bytes = 0;
    av1g_plane out_planes[3] = {};
    int shown = 0;
    Clock::time_point t_submit, t_done;
    size_t work_bytes = 0;
};

struct Step {
    cudaEvent_t ev = nullptr, ev0 = nullptr;
    std::vector<std::shared_ptr<Ticket>> tickets;
    // the intra launch's per-frame wait status (pinned, filled in stream
    // order) and the ticket of each of its jobs
    int32_t* intra_status = nullptr;
    std::vector<std::shared_ptr<Ticket>> intra_tickets;
    std::vector<uint8_t*> blobs;  // the frames' pinned descriptor blocks
    size_t work_bytes = 0;
    Clock::time_point t_enqueued;
};

// A worker thread with its own CUDA stream.  Each stream of frames belongs to
// one lane, so its frames and slot updates stay ordered on that CUDA stream
// while lanes prepare and run steps concurrently.
struct Lane {
    int idx = 0;
    cudaStream_t cs = nullptr;
    std::deque<Step> steps;
    std::thread thread;
};

}  // namespace

struct av1g_stream {
    av1g_engine* eng = nullptr;
    int lane = 0;
    av1g_seq_info seq = {};
    std::shared_ptr<SlotBuf> slots[8];
    std::deque<std::shared_ptr<Ticket>> pending;
    int inflight = 0;
    size_t reserved = 0;
    bool closing = false;
};

struct av1g_engine {
    int device = 0;
    size_t budget = 0, reserved = 0, inflight_bytes = 0;
    int max_batch = 64, max_steps = 3;
    int64_t max_step_samples = 4194304;  // < 0: no limit
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::vector<av1g_stream*> streams;
    size_t rr = 0, next_lane = 0;
    std::unordered_map<uint64_t, std::shared_ptr<Ticket>> tickets;
    std::vector<std::unique_ptr<Lane>> lanes;
    std::thread completer;
    bool stop = false, worker_done = false;
    uint64_t next_id = 1;
    int64_t frames_done = 0, steps_done = 0;
    double host_ms = 0, device_ms = 0, host_stage_ms[6] = {};
    // pinned host blocks (descriptor blobs, outputs, status words) by
    // capacity.  Blocks come from slabs of up to eight blocks of one capacity
    // class (cudaHostAlloc pins pages and is slow and serialising, so it runs
    // once per slab, not per block); a block returns to the free list and the
    // slabs are freed with the engine.
    static constexpr size_t kPinHeader = 256;  // keeps blocks 256-byte aligned
    std::mutex pin_mu;
    std::multimap<size_t, uint8_t*> pinned_free;
    std::vector<uint8_t*> pinned_slabs;

    uint8_t* pinned_get(size_t n) {
        // power-of-two capacities (from 256 KiB), so buffers recycle across
        // frames of similar size
        size_t cap = (size_t)256 << 10;
        while (cap < n) cap <<= 1;
        std::lock_guard<std::mutex> lk(pin_mu);
        auto it = pinned_free.lower_bound(cap);
        if (it != pinned_free.end() && it->first <= 2 * cap) {
            uint8_t* p = it->second;
            pinned_free.erase(it);
            return p;
        }
        const size_t blk = cap + kPinHeader;
        size_t k = ((size_t)64 << 20) / cap;
        k = k < 1 ? 1 : (k > 8 ? 8 : k);
        uint8_t* slab = nullptr;
        if (cudaHostAlloc((void**)&slab, k * blk, cudaHostAllocPortable) != cudaSuccess) {
            k = 1;  // retry with one block
            if (cudaHostAlloc((void**)&slab, blk, cudaHostAllocPortable) != cudaSuccess) return nullptr;
        }
        pinned_slabs.push_back(slab);
        for (size_t j = 0; j < k; j++) *(size_t*)(slab + j * blk) = cap;
        for (size_t j = 1; j < k; j++) pinned_free.emplace(cap, slab + j * blk + kPinHeader);
        return slab + kPinHeader;
    }
    void pinned_put(uint8_t* p) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(pin_mu);
        pinned_free.emplace(*(size_t*)(p - kPinHeader), p);
    }
};

SlotBuf::~SlotBuf() {
    if (dev && eng) {
        DeviceGuard g(eng->device);
        cudaFreeAsync(dev, cs);
    }
}

namespace {

size_t slot_bytes(int uw, int fh, int bd, int ssx, int ssy, int np) {
    int bps = bd > 8 ? 2 : 1;
    size_t t = 0;
    for (int p = 0; p < np; p++) {
        int sx = p ? ssx : 0, sy = p ? ssy : 0;
        t += align256(pitch_of(r2u(uw, sx), bps) * r2u(fh, sy));
    }
    return t;
}

// Device planes of one decoded frame (all in one allocation).
struct FrameBufs {
    uint8_t* dev = nullptr;
    size_t bytes = 0;
    av1g_plane recon[3] = {}, deb[3] = {}, cdef[3] = {}, upcdef[3] = {}, updeb[3] = {}, lr[3] = {}, out[3] = {};
    av1g_plane side[3] = {};  // inter halves of inter-intra blocks (only when the frame has some)
    uint8_t* grid[9] = {};
    int8_t* cdef_idx = nullptr;
    av1g_lr_unit* lr_units[3] = {};
    int32_t* coeffs = nullptr;
    size_t host_bytes = 0;  // prefix of the allocation uploaded from the blob
};

int lr_unit_count(const av1g_frame_header& h, int p) {
    int sx = p ? h.subsampling_x : 0, sy = p ? h.subsampling_y : 0;
    int us = h.lr_unit_size[p];
    auto cu = [](int us_, int sz) {
        if (us_ <= 0) return 1;
        int n = (sz + (us_ >> 1)) / us_;
        return n > 1 ? n : 1;
    };
    return cu(us, r2u(h.frame_height, sy)) * cu(us, r2u(h.upscaled_width, sx));
}

// Layout: [uploaded blob: grids | cdef_idx | lr units | coeffs] [planes]
size_t plan_frame(const Ticket& t, FrameBufs& B) {
    const av1g_frame_header& h = t.hdr;
    const int bps = h.bit_depth > 8 ? 2 : 1, np = h.num_planes;
    size_t off = t.blob_bytes;
    B.host_bytes = off;
    bool sr = h.use_superres && h.upscaled_width > h.frame_width;
    auto plane = [&](av1g_plane& pl, int w, int hh) {
        pl.stride = (int32_t)pitch_of(w, bps);
        pl.width = w;
        pl.height = hh;
        pl.data = (void*)off;  // offset until the allocation exists
        off = align256(off + (size_t)pl.stride * hh);
    };
    for (int p = 0; p < np; p++) {
        int sx = p ? h.subsampling_x : 0, sy = p ? h.subsampling_y : 0;
        int pw = (h.mi_cols * 4) >> sx, ph = (h.mi_rows * 4) >> sy;
        int uw = r2u(h.upscaled_width, sx), fh = r2u(h.frame_height, sy);
        plane(B.recon[p], pw, ph);
        plane(B.deb[p], pw, ph);
        plane(B.cdef[p], pw, ph);
        if (sr) {
            plane(B.upcdef[p], uw, fh);
            plane(B.updeb[p], uw, fh);
            plane(B.lr[p], uw, fh);
        } else {
            plane(B.lr[p], pw, ph);
        }
        plane(B.out[p], uw, fh);
        if (t.has_interintra) plane(B.side[p], pw, ph);
    }
    B.bytes = off;
    return off;
}

void rebase(FrameBufs& B, const Ticket& t) {
    auto fix = [&](av1g_plane* a) {
        for (int p = 0; p < 3; p++)
            if (a[p].width) a[p].data = B.dev + (size_t)a[p].data;
    };
    fix(B.recon);
    fix(B.deb);
    fix(B.cdef);
    fix(B.upcdef);
    fix(B.updeb);
    fix(B.lr);
    fix(B.out);
    fix(B.side);
    for (int g = 0; g < 9; g++) B.grid[g] = t.blob_len[g] ? B.dev + t.blob_off[g] : nullptr;
    B.cdef_idx = t.blob_len[9] ? (int8_t*)(B.dev + t.blob_off[9]) : nullptr;
    for (int p = 0; p < 3; p++)
        B.lr_units[p] = t.blob_len[10 + p] ? (av1g_lr_unit*)(B.dev + t.blob_off[10 + p]) : nullptr;
    B.coeffs = t.blob_len[13] ? (int32_t*)(B.dev + t.blob_off[13]) : nullptr;
}

// What a step does for one ticket.
struct Work {
    std::shared_ptr<Ticket> t;
    FrameBufs B;
    std::shared_ptr<SlotBuf> shown_slot;  // show_existing source
    av1g_ref_frame refs[7] = {};
    av1g_frame_header pf_hdr = {};        // header the post-filter chain sees
    bool decode = false, run_chain = false, failed = false;
};

void fail_work(Work& w, av1g_status st, const std::string& m) {
    w.failed = true;
    w.t->status = st;
    w.t->err = m;
}

// Runs a stage for all live works: batched, and per frame when the batch is
// rejected so that only the offending frames fail.
template <class Job, class Fn>
void run_stage(std::vector<Work*>& ws, std::vector<Job>& jobs, Fn fn, cudaStream_t cs) {
    if (jobs.empty()) return;
    std::string err;
    av1g_status st = fn(jobs.data(), (int)jobs.size(), cs, err);
    if (st == AV1G_OK) return;
    for (size_t i = 0; i < jobs.size(); i++) {
        std::string e1;
        av1g_status s1 = fn(&jobs[i], 1, cs, e1);
        if (s1 != AV1G_OK) fail_work(*ws[i], s1, e1);
    }
}

void enqueue_step(av1g_engine* E, cudaStream_t cs, std::vector<std::shared_ptr<Ticket>>& batch, Step& step,
                  double part_ms[6]) {
    NvtxRange range("av1g engine step");
    auto tp = Clock::now();
    auto lap = [&](int k) {
        auto now = Clock::now();
        part_ms[k] += std::chrono::duration<double, std::milli>(now - tp).count();
        tp = now;
    };
    std::vector<Work> works(batch.size());
    for (size_t i = 0; i < batch.size(); i++) {
        Work& w = works[i];
        w.t = batch[i];
        Ticket& t = *w.t;
        av1g_stream* S = t.st;
        if (t.show_existing) {
            if (t.show_idx >= 8 || !S->slots[t.show_idx]) {
                fail_work(w, AV1G_EINVAL, "show_existing_frame of an empty slot");
                continue;
            }
            w.shown_slot = S->slots[t.show_idx];
            const SlotBuf& sl = *w.shown_slot;
            if (sl.grain.apply_grain) {
                // grain on a copy of the slot frame: the chain with every
                // filter off and film grain on
                av1g_frame_header& h = t.hdr;
                memset(&h, 0, sizeof h);
                h.frame_width = h.upscaled_width = sl.upscaled_width;
                h.frame_height = sl.frame_height;
                h.mi_cols = 2 * ((sl.upscaled_width + 7) >> 3);
                h.mi_rows = 2 * ((sl.frame_height + 7) >> 3);
                h.bit_depth = sl.bit_depth;
                h.subsampling_x = sl.ssx;
                h.subsampling_y = sl.ssy;
                h.num_planes = sl.num_planes;
                h.matrix_coefficients = sl.matrix_coefficients;
                h.cdef_damping = 3;
                h.film_grain = sl.grain;
                w.run_chain = true;
            }
        } else {
            w.decode = true;
            w.run_chain = true;
            for (int r = 0; r < 7; r++) {
                const std::shared_ptr<SlotBuf>& sl = S->slots[t.ref_frame_idx[r] & 7];
                if (sl) {
                    for (int p = 0; p < 3; p++) w.refs[r].planes[p] = sl->planes[p];
                    w.refs[r].upscaled_width = sl->upscaled_width;
                    w.refs[r].frame_height = sl->frame_height;
                }
            }
        }
        if (w.run_chain) {
            plan_frame(t, w.B);
            cudaError_t e = cudaMallocAsync((void**)&w.B.dev, w.B.bytes, cs);
            if (e != cudaSuccess) {
                w.B.dev = nullptr;
                fail_work(w, AV1G_EDEVICE, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
                continue;
            }
            step.work_bytes += w.B.bytes;
            rebase(w.B, t);
            // the frame's grids, CDEF indices, LR units and coefficients: the
            // pinned block submit filled, in one copy (the block is returned
            // to the pool once the step has finished)
            if (t.blob_bytes) e = cudaMemcpyAsync(w.B.dev, t.blob, t.blob_bytes, cudaMemcpyHostToDevice, cs);
            // CurrFrame starts at zero, like the walker's fresh planes
            for (int p = 0; e == cudaSuccess && p < t.hdr.num_planes; p++)
                e = cudaMemsetAsync(w.B.recon[p].data, 0, (size_t)w.B.recon[p].stride * w.B.recon[p].height, cs);
            if (e == cudaSuccess && t.show_existing) {
                const SlotBuf& sl = *w.shown_slot;
                int bps = sl.bit_depth > 8 ? 2 : 1;
                for (int p = 0; e == cudaSuccess && p < sl.num_planes; p++)
                    e = cudaMemcpy2DAsync(w.B.recon[p].data, w.B.recon[p].stride, sl.planes[p].data, sl.planes[p].stride,
                                          (size_t)sl.planes[p].width * bps, sl.planes[p].height,
                                          cudaMemcpyDeviceToDevice, cs);
            }
            if (e != cudaSuccess) fail_work(w, AV1G_EDEVICE, std::string("upload: ") + cudaGetErrorString(e));
        }
    }
    lap(0);
    // prediction and residual stages, batched across the step's frames
    {
        std::vector<Work*> ws;
        std::vector<av1g_inter_job> jobs;
        for (Work& w : works) {
            if (w.failed || !w.decode || w.t->preds.empty()) continue;
            av1g_inter_job j = {};
            j.hdr = &w.t->hdr;
            j.refs = w.refs;
            j.preds = w.t->preds.data();
            j.num_preds = (int32_t)w.t->preds.size();
            j.neighbours = w.t->nbs.empty() ? nullptr : w.t->nbs.data();
            j.num_neighbours = (int32_t)w.t->nbs.size();
            j.warps = w.t->warps.empty() ? nullptr : w.t->warps.data();
            j.num_warps = (int32_t)w.t->warps.size();
            for (int p = 0; p < 3; p++) {
                j.planes[p] = w.B.recon[p];
                j.interintra_out[p] = w.B.side[p];
            }
            jobs.push_back(j);
            ws.push_back(&w);
        }
        run_stage(ws, jobs, inter_run, cs);
    }
    lap(1);
    {
        std::vector<Work*> ws;
        std::vector<av1g_recon_job> jobs;
        for (Work& w : works) {
            if (w.failed || !w.decode || w.t->inter_tus.empty()) continue;
            av1g_recon_job j = {};
            j.hdr = &w.t->hdr;
            j.quant = &w.t->quant;
            j.tus = w.t->inter_tus.data();
            j.num_tus = (int32_t)w.t->inter_tus.size();
            j.coeffs = w.B.coeffs;
            for (int p = 0; p < 3; p++) j.planes[p] = w.B.recon[p];
            jobs.push_back(j);
            ws.push_back(&w);
        }
        run_stage(ws, jobs, recon_run, cs);
    }
    lap(2);
    {
        std::vector<Work*> ws;
        std::vector<av1g_intra_job> jobs;
        for (Work& w : works) {
            if (w.failed || !w.decode || w.t->intra_tus.empty()) continue;
            av1g_intra_job j = {};
            j.hdr = &w.t->hdr;
            j.quant = &w.t->quant;
            j.tus = w.t->intra_tus.data();
            j.num_tus = (int32_t)w.t->intra_tus.size();
            j.sb_size = w.t->st->seq.sb_size;
            j.coeffs = w.B.coeffs;
            for (int p = 0; p < 3; p++) j.planes[p] = w.B.recon[p];
            j.palette_maps = w.t->maps.empty() ? nullptr : w.t->maps.data();
            j.palette_map_bytes = (int64_t)w.t->maps.size();
            for (int p = 0; p < 3; p++) j.interintra_in[p] = w.B.side[p];
            jobs.push_back(j);
            ws.push_back(&w);
        }
        if (!jobs.empty()) {
            // every job's wait status is read back after the step (the
            // completer fails that frame's ticket if its wait ran out)
            step.intra_status = (int32_t*)E->pinned_get(sizeof(int32_t) * jobs.size());
            if (!step.intra_status) {
                run_stage(ws, jobs, intra_run, cs);  // no pinned memory: no status readback
                goto intra_done;
            }
            {
            std::string err;
            av1g_status st = intra_run_status(jobs.data(), (int)jobs.size(), cs, err, step.intra_status);
            if (st == AV1G_OK) {
                for (Work* w : ws) step.intra_tickets.push_back(w->t);
            } else {
                // the batch was rejected: per frame, so that only the offending frames fail
                for (size_t i = 0; i < jobs.size(); i++) {
                    std::string e1;
                    av1g_status s1 = intra_run_status(&jobs[i], 1, cs, e1, step.intra_status + i);
                    if (s1 != AV1G_OK) fail_work(*ws[i], s1, e1);
                    else step.intra_tickets.push_back(ws[i]->t);
                    if (s1 != AV1G_OK) step.intra_status[i] = 0;
                }
                // keep the job-to-ticket order: rejected jobs map to no ticket
                std::vector<std::shared_ptr<Ticket>> tk;
                for (size_t i = 0; i < jobs.size(); i++) tk.push_back(ws[i]->failed ? nullptr : ws[i]->t);
                step.intra_tickets.swap(tk);
            }
            }
        }
    intra_done:;
    }
    lap(3);
    // the §7.4 chain
    std::vector<av1g_frame_job> fjobs(works.size());
    {
        std::vector<Work*> ws;
        std::vector<av1g_frame_job> jobs;
        for (size_t i = 0; i < works.size(); i++) {
            Work& w = works[i];
            if (w.failed || !w.run_chain) continue;
            av1g_frame_job j = {};
            j.hdr = &w.t->hdr;
            j.grid.mi_size = w.B.grid[0];
            j.grid.skip = w.B.grid[1];
            j.grid.is_inter = w.B.grid[2];
            j.grid.ref_frame0 = (const int8_t*)w.B.grid[3];
            j.grid.y_mode = w.B.grid[4];
            j.grid.segment_id = (const int8_t*)w.B.grid[5];
            j.grid.delta_lf = (const int8_t*)w.B.grid[6];
            j.grid.tx_size = w.B.grid[7];
            j.grid.inter_tx_size = w.B.grid[8];
            j.cdef_idx = w.B.cdef_idx;
            for (int p = 0; p < 3; p++) {
                j.lr_units[p] = w.B.lr_units[p];
                j.recon[p] = w.B.recon[p];
                j.deblocked[p] = w.B.deb[p];
                j.cdef[p] = w.B.cdef[p];
                j.up_cdef[p] = w.B.upcdef[p];
                j.up_deblocked[p] = w.B.updeb[p];
                j.lr[p] = w.B.lr[p];
                j.out[p] = w.B.out[p];
            }
            fjobs[i] = j;
            jobs.push_back(j);
            ws.push_back(&w);
        }
        run_stage(ws, jobs, postfilter_run, cs);
    }
    lap(4);
    // slot refreshes and outputs
    for (size_t i = 0; i < works.size(); i++) {
        Work& w = works[i];
        Ticket& t = *w.t;
        av1g_stream* S = t.st;
        cudaError_t e = cudaSuccess;
        if (!w.failed) {
            std::shared_ptr<SlotBuf> payload;
            PlaneDev pre[3] = {}, out[3] = {};
            int np = t.hdr.num_planes, bd = t.hdr.bit_depth;
            if (w.run_chain) {
                std::string err;
                av1g_status st = postfilter_result_planes(fjobs[i], pre, out, err);
                if (st != AV1G_OK) fail_work(w, st, err);
            }
            if (!w.failed && w.decode && t.refresh) {
                payload = std::make_shared<SlotBuf>();
                SlotBuf& sl = *payload;
                sl.eng = E;
                sl.cs = cs;
                sl.upscaled_width = t.hdr.upscaled_width;
                sl.frame_height = t.hdr.frame_height;
                sl.grain = t.hdr.film_grain;
                sl.bit_depth = (uint8_t)bd;
                sl.ssx = t.hdr.subsampling_x;
                sl.ssy = t.hdr.subsampling_y;
                sl.num_planes = (uint8_t)np;
                sl.matrix_coefficients = t.hdr.matrix_coefficients;
                sl.bytes = slot_bytes(sl.upscaled_width, sl.frame_height, bd, sl.ssx, sl.ssy, np);
                e = cudaMallocAsync((void**)&sl.dev, sl.bytes, cs);
                if (e != cudaSuccess) sl.dev = nullptr;
                size_t off = 0;
                int bps = bd > 8 ? 2 : 1;
                for (int p = 0; e == cudaSuccess && p < np; p++) {
                    int w_ = pre[p].w, h_ = pre[p].h;
                    sl.planes[p].data = sl.dev + off;
                    sl.planes[p].stride = (int32_t)pitch_of(w_, bps);
                    sl.planes[p].width = w_;
                    sl.planes[p].height = h_;
                    off += align256((size_t)sl.planes[p].stride * h_);
                    e = cudaMemcpy2DAsync(sl.planes[p].data, sl.planes[p].stride, pre[p].p, pre[p].stride,
                                          (size_t)w_ * bps, h_, cudaMemcpyDeviceToDevice, cs);
                }
                if (e != cudaSuccess) fail_work(w, AV1G_EDEVICE, std::string("slot copy: ") + cudaGetErrorString(e));
            } else if (!w.failed && t.show_existing) {
                payload = w.shown_slot;
            }
            if (!w.failed && payload) {
                for (int k = 0; k < 8; k++)
                    if ((t.refresh >> k) & 1) S->slots[k] = payload;
            }
            bool shown = !w.failed && (t.show || t.show_existing);
            if (shown) {
                av1g_plane src[3] = {};
                int bps = 1;
                if (t.show_existing && !w.run_chain) {
                    const SlotBuf& sl = *w.shown_slot;
                    np = sl.num_planes;
                    bps = sl.bit_depth > 8 ? 2 : 1;
                    for (int p = 0; p < np; p++) src[p] = sl.planes[p];
                } else {
                    bps = t.hdr.bit_depth > 8 ? 2 : 1;
                    for (int p = 0; p < np; p++)
                        src[p] = av1g_plane{out[p].p, out[p].stride, out[p].w, out[p].h};
                }
                size_t need = 0;
                for (int p = 0; p < np; p++) need += (size_t)src[p].width * bps * src[p].height;
                t.host_out = E->pinned_get(need);
                t.host_bytes = need;
                if (!t.host_out) {
                    fail_work(w, AV1G_EDEVICE, "pinned output allocation failed");
                } else {
                    size_t off = 0;
                    for (int p = 0; e == cudaSuccess && p < np; p++) {
                        size_t row = (size_t)src[p].width * bps;
                        t.out_planes[p] = av1g_plane{t.host_out + off, (int32_t)row, src[p].width, src[p].height};
                        e = cudaMemcpy2DAsync(t.host_out + off, row, src[p].data, src[p].stride, row, src[p].height,
                                              cudaMemcpyDeviceToHost, cs);
                        off += row * src[p].height;
                    }
                    t.shown = 1;
                    if (e != cudaSuccess) fail_work(w, AV1G_EDEVICE, std::string("output copy: ") + cudaGetErrorString(e));
                }
            }
        }
        if (w.B.dev) cudaFreeAsync(w.B.dev, cs);
    }
    lap(5);
}

void worker_loop(av1g_engine* E, Lane* L) {
    cudaSetDevice(E->device);
    std::unique_lock<std::mutex> lk(E->mu);
    size_t rr = 0;
    while (!E->stop) {
        std::vector<std::shared_ptr<Ticket>> batch;
        size_t extra = 0;
        int64_t samples = 0;  // luma samples of the frames taken
        if ((int)L->steps.size() < E->max_steps) {
            size_t n = E->streams.size();
            for (size_t k = 0; k < n && (int)batch.size() < E->max_batch; k++) {
                av1g_stream* S = E->streams[(rr + k) % n];
                if (S->lane != L->idx) continue;
                // reset markers are applied in order, between frames
                while (!S->pending.empty() && S->pending.front()->reset_marker) {
                    std::shared_ptr<Ticket> r = S->pending.front();
                    S->pending.pop_front();
                    for (auto& sl : S->slots) sl.reset();
                    r->done = true;
                    E->tickets.erase(r->id);
                }
                if (S->pending.empty()) continue;
                std::shared_ptr<Ticket> t = S->pending.front();
                // a step's host preparation is serial: bound its size so that
                // large frames pipeline instead of waiting for each other
                const int64_t tpx = (int64_t)t->hdr.upscaled_width * t->hdr.frame_height;
                if (!batch.empty() && E->max_step_samples > 0 && samples + tpx > E->max_step_samples) break;
                if (E->reserved + E->inflight_bytes + extra + t->work_bytes > E->budget) {
                    if (E->inflight_bytes + extra == 0 && batch.empty()) {
                        // can never fit: fail it
                        S->pending.pop_front();
                        E->pinned_put(t->blob);
                        t->blob = nullptr;
                        t->status = AV1G_ENOMEM_BUDGET;
                        t->err = "frame work memory exceeds the engine budget";
                        t->done = true;
                        t->t_done = Clock::now();
                        E->cv_done.notify_all();
                    }
                    continue;
                }
                S->pending.pop_front();
                S->inflight++;
                extra += t->work_bytes;
                samples += tpx;
                batch.push_back(t);
            }
            if (n) rr = (rr + 1) % n;
        }
        if (batch.empty()) {
            E->cv_work.wait_for(lk, std::chrono::milliseconds(20));
            continue;
        }
        E->inflight_bytes += extra;
        lk.unlock();
        auto h0 = Clock::now();
        Step step;
        cudaEventCreate(&step.ev0);
        cudaEventRecord(step.ev0, L->cs);
        double part[6] = {};
        enqueue_step(E, L->cs, batch, step, part);
        // the descriptor copies have been staged; keep only the outputs (the
        // pinned blocks of the device-bound arrays go with the step)
        for (auto& t : batch) {
            if (t->blob) step.blobs.push_back(t->blob);
            t->blob = nullptr;
            std::vector<av1g_inter_pred>().swap(t->preds);
            std::vector<av1g_obmc_neighbour>().swap(t->nbs);
            std::vector<av1g_warp_ctx>().swap(t->warps);
            std::vector<av1g_tu>().swap(t->inter_tus);
            std::vector<av1g_intra_tu>().swap(t->intra_tus);
            std::vector<uint8_t>().swap(t->maps);
        }
        step.tickets = batch;
        step.work_bytes = extra;
        cudaEventCreate(&step.ev);
        cudaEventRecord(step.ev, L->cs);
        step.t_enqueued = Clock::now();
        double hms = std::chrono::duration<double, std::milli>(Clock::now() - h0).count();
        lk.lock();
        E->host_ms += hms;
        for (int k = 0; k < 6; k++) E->host_stage_ms[k] += part[k];
        L->steps.push_back(std::move(step));
        E->cv_done.notify_all();
    }
}

void completer_loop(av1g_engine* E) {
    cudaSetDevice(E->device);
    std::unique_lock<std::mutex> lk(E->mu);
    for (;;) {
        bool any = false;
        for (auto& L : E->lanes) any = any || !L->steps.empty();
        if (!any) {
            if (E->worker_done) break;
            E->cv_done.wait_for(lk, std::chrono::milliseconds(20));
            continue;
        }
        // retire, per lane and in order, every step whose event has completed;
        // a step still running a minute after it was enqueued is failed
        bool progressed = false;
        for (auto& L : E->lanes) {
            while (!L->steps.empty()) {
                Step& front = L->steps.front();
                cudaError_t q = cudaEventQuery(front.ev);
                bool expired = q == cudaErrorNotReady && Clock::now() - front.t_enqueued > std::chrono::seconds(60);
                if (q == cudaErrorNotReady && !expired) break;
                Step step = std::move(front);
                L->steps.pop_front();
                auto now = Clock::now();
                if (q == cudaSuccess && step.intra_status) {
                    for (size_t i = 0; i < step.intra_tickets.size(); i++) {
                        auto& t = step.intra_tickets[i];
                        if (t && step.intra_status[i] && t->status == AV1G_OK) {
                            t->status = AV1G_EDEVICE;
                            t->err = "intra: a superblock dependency wait ran out of time";
                        }
                    }
                }
                if (step.intra_status && !expired) E->pinned_put((uint8_t*)step.intra_status);
                if (!expired)
                    for (uint8_t* b : step.blobs) E->pinned_put(b);
                for (auto& t : step.tickets) {
                    if (q != cudaSuccess && t->status == AV1G_OK) {
                        t->status = expired ? AV1G_TIMEOUT : AV1G_EDEVICE;
                        t->err = expired ? "step did not finish within 60 s" : cudaGetErrorString(q);
                    }
                    t->done = true;
                    t->t_done = now;
                    t->st->inflight--;
                    E->frames_done++;
                }
                E->steps_done++;
                E->inflight_bytes -= step.work_bytes;
                float dms = 0.f;
                if (q == cudaSuccess && cudaEventElapsedTime(&dms, step.ev0, step.ev) == cudaSuccess)
                    E->device_ms += dms;
                if (!expired) {
                    cudaEventDestroy(step.ev);
                    cudaEventDestroy(step.ev0);
                }
                progressed = true;
            }
        }
        if (progressed) {
            E->cv_done.notify_all();
            E->cv_work.notify_all();
        } else {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(50));
            lk.lock();
        }
    }
}

// Upper bound of a frame's work allocation (planes + blob) for admission.
size_t work_estimate(const av1g_frame_header& h, size_t blob) {
    const int bps = h.bit_depth > 8 ? 2 : 1;
    size_t t = blob;
    for (int p = 0; p < h.num_planes; p++) {
        int sx = p ? h.subsampling_x : 0, sy = p ? h.subsampling_y : 0;
        size_t padded = pitch_of((h.mi_cols * 4) >> sx, bps) * ((h.mi_rows * 4) >> sy);
        size_t up = pitch_of(r2u(h.upscaled_width, sx), bps) * r2u(h.frame_height, sy);
        t += 4 * padded + 4 * up + 8 * 256;
    }
    return t;
}

template <class T>
void copy_in(std::vector<T>& v, const T* p, int64_t n) {
    if (p && n > 0) v.assign(p, p + n);
}

}  // namespace

extern "C" {

av1g_status av1g_engine_create(const av1g_config* cfg, av1g_engine** out) {
    if (!cfg || !out) return AV1G_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) return AV1G_EDEVICE;
    DeviceGuard g(cfg->device);
    auto* E = new av1g_engine();
    E->device = cfg->device;
    E->max_batch = cfg->max_batch > 0 ? cfg->max_batch : 64;
    E->max_step_samples = cfg->max_step_samples != 0 ? cfg->max_step_samples : 4194304;
    E->max_steps = cfg->max_inflight_steps > 0 ? cfg->max_inflight_steps : 3;
    int nl = cfg->lanes > 0 ? cfg->lanes : 4;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    E->budget = cfg->hbm_budget_bytes > 0 ? (size_t)cfg->hbm_budget_bytes : free_b / 10 * 8;
    if (cfg->autotune_cache) {
        std::string err;
        if (load_shapes(cfg->autotune_cache, err) != AV1G_OK) {
            delete E;
            return AV1G_EINVAL;
        }
    }
    for (int i = 0; i < nl; i++) {
        auto L = std::make_unique<Lane>();
        L->idx = i;
        if (cudaStreamCreateWithFlags(&L->cs, cudaStreamNonBlocking) != cudaSuccess) {
            for (auto& l : E->lanes) cudaStreamDestroy(l->cs);
            delete E;
            return AV1G_EDEVICE;
        }
        E->lanes.push_back(std::move(L));
    }
    // keep freed stream-ordered memory in the pool between steps
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, E->device) == cudaSuccess) {
        uint64_t thr = E->budget;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    for (auto& L : E->lanes) L->thread = std::thread(worker_loop, E, L.get());
    E->completer = std::thread(completer_loop, E);
    *out = E;
    return AV1G_OK;
}

void av1g_engine_destroy(av1g_engine* E) {
    if (!E) return;
    {
        std::unique_lock<std::mutex> lk(E->mu);
        // let queued frames drain (bounded)
        auto t0 = Clock::now();
        while (Clock::now() - t0 < std::chrono::seconds(120)) {
            bool busy = false;
            for (auto& L : E->lanes) busy = busy || !L->steps.empty();
            for (auto* S : E->streams) busy = busy || !S->pending.empty();
            if (!busy) break;
            E->cv_done.wait_for(lk, std::chrono::milliseconds(20));
        }
        E->stop = true;
    }
    E->cv_work.notify_all();
    for (auto& L : E->lanes) L->thread.join();
    {
        std::lock_guard<std::mutex> lk(E->mu);
        E->worker_done = true;
    }
    E->cv_done.notify_all();
    E->completer.join();
    DeviceGuard g(E->device);
    for (auto* S : E->streams) {
        for (auto& sl : S->slots) sl.reset();
        delete S;
    }
    for (auto& kv : E->tickets) {
        E->pinned_put(kv.second->host_out);
        E->pinned_put(kv.second->blob);  // never enqueued
    }
    E->tickets.clear();
    for (auto& L : E->lanes) cudaStreamSynchronize(L->cs);
    for (uint8_t* slab : E->pinned_slabs) cudaFreeHost(slab);
    for (auto& L : E->lanes) cudaStreamDestroy(L->cs);
    delete E;
}

av1g_status av1g_engine_get_stats(av1g_engine* E, av1g_engine_stats* o) {
    if (!E || !o) return AV1G_EINVAL;
    std::lock_guard<std::mutex> lk(E->mu);
    o->frames_done = E->frames_done;
    o->steps_done = E->steps_done;
    o->bytes_reserved = (int64_t)E->reserved;
    o->bytes_in_flight = (int64_t)E->inflight_bytes;
    o->budget = (int64_t)E->budget;
    o->streams_open = (int32_t)E->streams.size();
    o->pad = 0;
    o->host_ms = E->host_ms;
    o->device_ms = E->device_ms;
    for (int k = 0; k < 6; k++) o->host_stage_ms[k] = E->host_stage_ms[k];
    return AV1G_OK;
}

av1g_status av1g_stream_open(av1g_engine* E, const av1g_seq_info* q, av1g_stream** out) {
    if (!E || !q || !out) return AV1G_EINVAL;
    *out = nullptr;
    if (q->max_width <= 0 || q->max_height <= 0 || q->max_width > 65535 || q->max_height > 65535 ||
        (q->bit_depth != 8 && q->bit_depth != 10 && q->bit_depth != 12) || q->subsampling_x > 1 ||
        q->subsampling_y > 1 || (q->num_planes != 1 && q->num_planes != 3) || (q->sb_size != 64 && q->sb_size != 128))
        return AV1G_EINVAL;
    size_t need = 9 * slot_bytes(q->max_width, q->max_height, q->bit_depth, q->subsampling_x, q->subsampling_y,
                                 q->num_planes);
    std::lock_guard<std::mutex> lk(E->mu);
    if (E->reserved + need > E->budget) return AV1G_ENOMEM_BUDGET;
    auto* S = new av1g_stream();
    S->eng = E;
    S->lane = (int)(E->next_lane++ % E->lanes.size());
    S->seq = *q;
    S->reserved = need;
    E->reserved += need;
    E->streams.push_back(S);
    *out = S;
    return AV1G_OK;
}

av1g_status av1g_stream_close(av1g_stream* S) {
    if (!S) return AV1G_EINVAL;
    av1g_engine* E = S->eng;
    std::unique_lock<std::mutex> lk(E->mu);
    S->closing = true;
    auto t0 = Clock::now();
    while ((!S->pending.empty() || S->inflight > 0) && Clock::now() - t0 < std::chrono::seconds(120))
        E->cv_done.wait_for(lk, std::chrono::milliseconds(20));
    if (!S->pending.empty() || S->inflight > 0) return AV1G_TIMEOUT;
    E->streams.erase(std::find(E->streams.begin(), E->streams.end(), S));
    E->reserved -= S->reserved;
    for (auto it = E->tickets.begin(); it != E->tickets.end();) {
        if (it->second->st == S) {
            E->pinned_put(it->second->host_out);
            it = E->tickets.erase(it);
        } else {
            ++it;
        }
    }
    lk.unlock();
    for (auto& sl : S->slots) sl.reset();
    delete S;
    E->cv_work.notify_all();
    return AV1G_OK;
}

av1g_status av1g_stream_reset_refs(av1g_stream* S) {
    if (!S) return AV1G_EINVAL;
    av1g_engine* E = S->eng;
    auto t = std::make_shared<Ticket>();
    t->st = S;
    t->reset_marker = true;
    std::lock_guard<std::mutex> lk(E->mu);
    t->id = E->next_id++;
    E->tickets[t->id] = t;
    S->pending.push_back(t);
    E->cv_work.notify_all();
    return AV1G_OK;
}

av1g_status av1g_submit_frame(av1g_stream* S, const av1g_frame_desc* d, uint64_t* ticket) {
    if (!S || !d || !ticket || !d->hdr || (!d->show_existing_frame && !d->quant)) return AV1G_EINVAL;
    const av1g_frame_header& h = *d->hdr;
    const av1g_seq_info& q = S->seq;
    if (!d->show_existing_frame &&
        (h.bit_depth != q.bit_depth || h.subsampling_x != q.subsampling_x || h.subsampling_y != q.subsampling_y ||
         h.num_planes != q.num_planes || h.upscaled_width > q.max_width || h.frame_height > q.max_height ||
         h.frame_width <= 0 || h.frame_height <= 0 || h.mi_rows <= 0 || h.mi_cols <= 0))
        return AV1G_EINVAL;
    if (d->num_inter_preds < 0 || d->num_neighbours < 0 || d->num_warps < 0 || d->num_inter_tus < 0 ||
        d->num_intra_tus < 0 || d->palette_map_bytes < 0 || d->num_coeffs < 0)
        return AV1G_EINVAL;
    auto t = std::make_shared<Ticket>();
    t->st = S;
    t->hdr = h;
    if (d->quant) t->quant = *d->quant;
    t->show_existing = d->show_existing_frame;
    t->show_idx = d->frame_to_show_map_idx;
    t->show = d->show_frame;
    t->refresh = d->refresh_frame_flags;
    memcpy(t->ref_frame_idx, d->ref_frame_idx, 7);
    size_t blob = 0;
    if (!d->show_existing_frame) {
        size_t M = (size_t)h.mi_rows * h.mi_cols;
        const void* src[14] = {d->grid.mi_size, d->grid.skip, d->grid.is_inter, d->grid.ref_frame0, d->grid.y_mode,
                               d->grid.segment_id, d->grid.delta_lf, d->grid.tx_size, d->grid.inter_tx_size,
                               d->cdef_idx, d->lr_units[0], d->lr_units[1], d->lr_units[2], d->coeffs};
        size_t len[14] = {};
        for (int k = 0; k < 9; k++) len[k] = src[k] ? (k == 6 ? 4 * M : M) : 0;
        len[9] = d->cdef_idx ? (size_t)((h.mi_rows + 15) >> 4) * ((h.mi_cols + 15) >> 4) : 0;
        for (int p = 0; p < 3; p++)
            if (h.uses_lr && p < h.num_planes && h.lr_type[p] && d->lr_units[p])
                len[10 + p] = (size_t)lr_unit_count(h, p) * sizeof(av1g_lr_unit);
        len[13] = d->coeffs && d->num_coeffs > 0 ? (size_t)d->num_coeffs * sizeof(int32_t) : 0;
        size_t off = 0;
        for (int k = 0; k < 14; k++) {
            t->blob_off[k] = off;
            t->blob_len[k] = len[k];
            off = align256(off + len[k]);
        }
        t->blob_bytes = off;
        if (off) {
            {
                DeviceGuard g(S->eng->device);
                t->blob = S->eng->pinned_get(off);
            }
            if (!t->blob) return AV1G_EDEVICE;
            // the arrays cover the block but for alignment gaps, which nothing reads
            for (int k = 0; k < 14; k++)
                if (len[k]) memcpy(t->blob + t->blob_off[k], src[k], len[k]);
        }
        copy_in(t->preds, d->inter_preds, d->num_inter_preds);
        for (const av1g_inter_pred& pr : t->preds) t->has_interintra |= pr.kind == AV1G_INTER_INTRA;
        copy_in(t->nbs, d->neighbours, d->num_neighbours);
        copy_in(t->warps, d->warps, d->num_warps);
        copy_in(t->inter_tus, d->inter_tus, d->num_inter_tus);
        copy_in(t->intra_tus, d->intra_tus, d->num_intra_tus);
        copy_in(t->maps, d->palette_maps, d->palette_map_bytes);
        blob = off + 9 * 256 + 4096;
        t->work_bytes = work_estimate(h, blob);
    } else {
        av1g_frame_header hh = {};
        hh.bit_depth = q.bit_depth;
        hh.num_planes = q.num_planes;
        hh.subsampling_x = q.subsampling_x;
        hh.subsampling_y = q.subsampling_y;
        hh.frame_width = hh.upscaled_width = q.max_width;
        hh.frame_height = q.max_height;
        hh.mi_cols = 2 * ((q.max_width + 7) >> 3);
        hh.mi_rows = 2 * ((q.max_height + 7) >> 3);
        t->work_bytes = work_estimate(hh, 4096);
    }
    av1g_engine* E = S->eng;
    std::lock_guard<std::mutex> lk(E->mu);
    if (S->closing) {
        E->pinned_put(t->blob);
        return AV1G_EINVAL;
    }
    t->id = E->next_id++;
    t->t_submit = Clock::now();
    E->tickets[t->id] = t;
    S->pending.push_back(t);
    *ticket = t->id;
    E->cv_work.notify_all();
    return AV1G_OK;
}

av1g_status av1g_poll(av1g_engine* E, uint64_t id, int64_t timeout_ns, av1g_status* result) {
    if (!E) return AV1G_EINVAL;
    std::unique_lock<std::mutex> lk(E->mu);
    auto it = E->tickets.find(id);
    if (it == E->tickets.end()) return AV1G_EINVAL;
    std::shared_ptr<Ticket> t = it->second;
    if (!t->done && timeout_ns > 0)
        E->cv_done.wait_for(lk, std::chrono::nanoseconds(timeout_ns), [&] { return t->done; });
    if (!t->done) return timeout_ns > 0 ? AV1G_TIMEOUT : AV1G_ENOTREADY;
    if (result) *result = t->status;
    if (t->status != AV1G_OK) set_last_error_text(t->err);  // why the frame failed
    return AV1G_OK;
}

av1g_status av1g_fetch_output(av1g_stream* S, uint64_t id, av1g_frame_out* o) {
    if (!S || !o) return AV1G_EINVAL;
    av1g_engine* E = S->eng;
    std::lock_guard<std::mutex> lk(E->mu);
    auto it = E->tickets.find(id);
    if (it == E->tickets.end() || it->second->st != S) return AV1G_EINVAL;
    const Ticket& t = *it->second;
    if (!t.done) return AV1G_ENOTREADY;
    memset(o, 0, sizeof *o);
    o->shown = t.shown;
    o->num_planes = t.shown ? (t.show_existing ? t.st->seq.num_planes : t.hdr.num_planes) : 0;
    o->bit_depth = t.show_existing ? t.st->seq.bit_depth : t.hdr.bit_depth;
    for (int p = 0; p < 3; p++) o->planes[p] = t.out_planes[p];
    o->latency_ms = std::chrono::duration<double, std::milli>(t.t_done - t.t_submit).count();
    if (t.status != AV1G_OK) set_last_error_text(t.err);
    return t.status;
}

av1g_status av1g_release_output(av1g_stream* S, uint64_t id) {
    if (!S) return AV1G_EINVAL;
    av1g_engine* E = S->eng;
    std::lock_guard<std::mutex> lk(E->mu);
    auto it = E->tickets.find(id);
    if (it == E->tickets.end() || it->second->st != S) return AV1G_EINVAL;
    if (!it->second->done) return AV1G_ENOTREADY;
    E->pinned_put(it->second->host_out);
    E->tickets.erase(it);
    return AV1G_OK;
}

}  // extern "C"
