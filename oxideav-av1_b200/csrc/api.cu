// api.cu — the av1g_* C ABI: descriptor validation, stage gating and the
// batched / per-frame launch of the §7.4 post-filter chain.
//
// Gating and buffer flow follow decode_frame_spec_tiles
// (src/decoder/frame_driver.rs:790-1116):
//   deblock  iff (lf_level[0] || lf_level[1]) && !CodedLossless && !allow_intrabc   (832-836)
//   CDEF     iff !CodedLossless && !allow_intrabc && enable_cdef && cdef coded      (870)
//   superres iff use_superres && UpscaledWidth > FrameWidth                          (906)
//   LR       iff UsesLr                                                             (971)
//   grain    iff apply_grain                                                        (1060)
// A stage that is off forwards its input plane to the next stage (pointer
// aliasing, no copy), and so does a chroma plane whose deblock level
// (loop_filter.rs:274-278) or restoration type is zero.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace av1g {
size_t lr_smem_bytes();
av1g_status recon_run(const av1g_recon_job* jobs, int n, cudaStream_t s, std::string& err);
av1g_status intra_run(const av1g_intra_job* jobs, int n, cudaStream_t s, std::string& err);
av1g_status intra_run_status(const av1g_intra_job* jobs, int n, cudaStream_t s, std::string& err,
                             int32_t* frame_status);
av1g_status inter_run(const av1g_inter_job* jobs, int n, cudaStream_t s, std::string& err);
av1g_status mf_store_run(const av1g_mf_store_job* jobs, int n, cudaStream_t s, std::string& err);
av1g_status mf_project_run(const av1g_mf_project_job* jobs, int n, cudaStream_t s, std::string& err);
av1g_status tile_list_run(const av1g_tile_list_job* jobs, int n, cudaStream_t s, std::string& err);
}

using namespace av1g;

namespace {

thread_local std::string g_err;

av1g_status fail(av1g_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

av1g_status cuda_fail(cudaError_t e, const char* what) {
    return fail(AV1G_EDEVICE, "%s: %s", what, cudaGetErrorString(e));
}

int r2u(int x, int n) { return n ? (x + (1 << (n - 1))) >> n : x; }

// The kernels see a plane at exactly the extent the reference's buffer has
// (the padded mi extent, or UpscaledWidth x FrameHeight after superres): the
// CDEF availability test and every clamp are relative to that extent, so a
// caller's larger allocation must not widen it.
PlaneDev to_dev(const av1g_plane& p, int w, int h) { return PlaneDev{(uint8_t*)p.data, p.stride, w, h}; }

// Planes must start on a 16-byte boundary with a stride that is a multiple
// of 16 bytes: the kernels move samples with 4- and 8-byte vector accesses.
bool plane_ok(const av1g_plane& p, int w, int h, int bps) {
    return p.data && ((uintptr_t)p.data & 15) == 0 && (p.stride & 15) == 0 && p.width >= w && p.height >= h &&
           p.stride >= w * bps;
}

int count_units(int us, int sz) {
    if (us <= 0) return 1;
    int n = (sz + (us >> 1)) / us;
    return n > 1 ? n : 1;
}

// Builds the FrameDev record of one job and validates it.
av1g_status prepare_frame(const av1g_frame_job& j, FrameDev& F) {
    if (!j.hdr) return fail(AV1G_EINVAL, "job without header");
    const av1g_frame_header& h = *j.hdr;
    memset(&F, 0, sizeof F);
    F.h = h;
    if (h.bit_depth != 8 && h.bit_depth != 10 && h.bit_depth != 12)
        return fail(AV1G_EINVAL, "bit_depth %d", h.bit_depth);
    if (h.num_planes != 1 && h.num_planes != 3) return fail(AV1G_EINVAL, "num_planes %d", h.num_planes);
    if (h.subsampling_x > 1 || h.subsampling_y > 1 || (h.subsampling_y && !h.subsampling_x))
        return fail(AV1G_EINVAL, "subsampling %d,%d", h.subsampling_x, h.subsampling_y);
    if (h.frame_width <= 0 || h.frame_height <= 0 || h.upscaled_width < h.frame_width)
        return fail(AV1G_EINVAL, "frame size %dx%d upscaled %d", h.frame_width, h.frame_height, h.upscaled_width);
    if (h.mi_cols != 2 * ((h.frame_width + 7) >> 3) || h.mi_rows != 2 * ((h.frame_height + 7) >> 3))
        return fail(AV1G_EINVAL, "MiRows/MiCols %d/%d do not match %dx%d", h.mi_rows, h.mi_cols, h.frame_width,
                    h.frame_height);
    if (h.cdef_bits > 3 || h.cdef_damping < 3 || h.cdef_damping > 6)
        return fail(AV1G_EINVAL, "cdef_bits %d damping %d", h.cdef_bits, h.cdef_damping);
    const int hbd = h.bit_depth > 8, bps = hbd ? 2 : 1;
    F.hbd = hbd;
    F.g = j.grid;
    F.cdef_idx = j.cdef_idx;
    const int np = h.num_planes, ssx = h.subsampling_x, ssy = h.subsampling_y;
    int pw[3], ph[3], uw[3], fh[3];
    for (int p = 0; p < np; p++) {
        int sx = p ? ssx : 0, sy = p ? ssy : 0;
        pw[p] = (h.mi_cols * 4) >> sx;
        ph[p] = (h.mi_rows * 4) >> sy;
        uw[p] = r2u(h.upscaled_width, sx);
        fh[p] = r2u(h.frame_height, sy);
        if (!plane_ok(j.recon[p], pw[p], ph[p], bps)) return fail(AV1G_EINVAL, "recon plane %d too small", p);
    }
    F.do_stage[ST_DEBLOCK] = (h.lf_level[0] || h.lf_level[1]) && !h.coded_lossless && !h.allow_intrabc;
    F.do_stage[ST_CDEF] = !h.coded_lossless && !h.allow_intrabc && h.enable_cdef && !h.cdef_short_circuited;
    F.do_stage[ST_SUPERRES] = h.use_superres && h.upscaled_width > h.frame_width;
    F.do_stage[ST_LR] = h.uses_lr != 0;
    F.do_stage[ST_GRAIN] = h.film_grain.apply_grain != 0;
    bool grid_needed = F.do_stage[ST_DEBLOCK] || F.do_stage[ST_CDEF];
    if (grid_needed && (!j.grid.skip || !j.grid.mi_size))
        return fail(AV1G_EINVAL, "mi grid missing");
    if (F.do_stage[ST_DEBLOCK] && (!j.grid.is_inter || !j.grid.ref_frame0 || !j.grid.y_mode || !j.grid.segment_id ||
                                   !j.grid.delta_lf || !j.grid.tx_size || !j.grid.inter_tx_size))
        return fail(AV1G_EINVAL, "mi grid incomplete for deblock");
    if (F.do_stage[ST_CDEF] && !j.cdef_idx) return fail(AV1G_EINVAL, "cdef_idx missing");
    for (int p = 0; p < np; p++) {
        F.recon[p] = to_dev(j.recon[p], pw[p], ph[p]);
        bool deb = F.do_stage[ST_DEBLOCK] && (p == 0 || h.lf_level[1 + p] != 0);
        if (deb && !plane_ok(j.deblocked[p], pw[p], ph[p], bps)) return fail(AV1G_EINVAL, "deblocked plane %d", p);
        F.deb[p] = deb ? to_dev(j.deblocked[p], pw[p], ph[p]) : F.recon[p];
        if (F.do_stage[ST_CDEF] && !plane_ok(j.cdef[p], pw[p], ph[p], bps)) return fail(AV1G_EINVAL, "cdef plane %d", p);
        F.cdef[p] = F.do_stage[ST_CDEF] ? to_dev(j.cdef[p], pw[p], ph[p]) : F.deb[p];
        if (F.do_stage[ST_SUPERRES]) {
            if (!plane_ok(j.up_cdef[p], uw[p], fh[p], bps)) return fail(AV1G_EINVAL, "up_cdef plane %d", p);
            F.upcdef[p] = to_dev(j.up_cdef[p], uw[p], fh[p]);
            if (F.do_stage[ST_LR]) {
                if (!plane_ok(j.up_deblocked[p], uw[p], fh[p], bps)) return fail(AV1G_EINVAL, "up_deblocked plane %d", p);
                F.updeb[p] = to_dev(j.up_deblocked[p], uw[p], fh[p]);
            } else {
                F.updeb[p] = F.deb[p];
            }
        } else {
            F.upcdef[p] = F.cdef[p];
            F.updeb[p] = F.deb[p];
        }
        bool lr = F.do_stage[ST_LR] && h.lr_type[p] != 0;
        if (lr) {
            if (!plane_ok(j.lr[p], uw[p], fh[p], bps)) return fail(AV1G_EINVAL, "lr plane %d", p);
            // LoopRestorationSize: 64..256 for luma, halved for 4:2:0 chroma (§5.9.20)
            int umin = 64 >> (p ? ssy : 0);
            if (h.lr_unit_size[p] < umin || h.lr_unit_size[p] > 256 || (h.lr_unit_size[p] & (h.lr_unit_size[p] - 1)))
                return fail(AV1G_EINVAL, "lr unit size %d for plane %d", h.lr_unit_size[p], p);
            F.lr[p] = to_dev(j.lr[p], uw[p], fh[p]);
            F.lr_units[p] = j.lr_units[p];
            F.lr_unit_rows[p] = count_units(h.lr_unit_size[p], fh[p]);
            F.lr_unit_cols[p] = count_units(h.lr_unit_size[p], uw[p]);
        } else {
            F.lr[p] = F.upcdef[p];
        }
        F.lr[p].w = uw[p];  // the cropped view the reference stores (frame_driver.rs:1018-1052)
        F.lr[p].h = fh[p];
        if (F.do_stage[ST_GRAIN]) {
            if (!plane_ok(j.out[p], uw[p], fh[p], bps)) return fail(AV1G_EINVAL, "out plane %d", p);
            F.out[p] = to_dev(j.out[p], uw[p], fh[p]);
            F.out[p].w = uw[p];
            F.out[p].h = fh[p];
        } else {
            F.out[p] = F.lr[p];
        }
    }
    if (F.do_stage[ST_GRAIN]) {
        const av1g_film_grain& g = h.film_grain;
        if (g.num_y_points > 14 || g.num_cb_points > 10 || g.num_cr_points > 10 || g.ar_coeff_lag > 3 ||
            g.grain_scaling < 8 || g.grain_scaling > 11 || g.ar_coeff_shift < 6 || g.ar_coeff_shift > 9 ||
            g.grain_scale_shift > 3)
            return fail(AV1G_EINVAL, "film grain parameters out of range");
        F.grain_nblocks = ((h.upscaled_width + 1) / 2 + 15) / 16;
    }
    return AV1G_OK;
}

int grain_scratch_bytes(const FrameDev& F) {
    int nstripes = ((F.h.frame_height + 1) / 2 + 15) / 16;
    return (3 * 73 * 82 * 2 + 768 + nstripes * F.grain_nblocks + 255) & ~255;
}

struct Batch {
    std::vector<FrameDev> frames;
    // per stage (and the grain template pass, index ST_COUNT) tile counts per frame
    std::vector<int32_t> tiles[ST_COUNT + 1];
};

int stage_tiles(const FrameDev& F, int st, int sr_tile) {
    if (st < ST_COUNT && !F.do_stage[st]) return 0;
    switch (st) {
        case ST_DEBLOCK: return tiles_deblock(F);
        case ST_CDEF: return tiles_cdef(F);
        case ST_SUPERRES: return tiles_superres(F, sr_tile);
        case ST_LR: return tiles_lr(F);
        case ST_GRAIN: return tiles_grain_blend(F);
        default: return F.do_stage[ST_GRAIN] ? 1 : 0;  // template pass
    }
}

// Runs `stages` (bit mask over ST_*) for the jobs.
// A batch's frame records, tile prefixes and scratch layout, built on the
// host; bind() points the records at a device allocation of total_bytes.
struct Prepared {
    static constexpr int NS = ST_COUNT + 1;
    Batch b;
    int n = 0, stage_mask = 0, mode = 0, max_cells = 0;
    size_t off_starts = 0, off_pf = 0, off_scratch = 0, total_bytes = 0;
    std::vector<size_t> lf_off, grain_off;
    std::vector<uint8_t> host;  // the uploaded prefix [0, off_scratch)
    int32_t totals[NS] = {};
    StageShape shape[ST_COUNT] = {};  // launch shapes (by the first frame's sample width)
};

av1g_status prepare(const av1g_frame_job* jobs, int n, int stage_mask, int mode, Prepared& P) {
    if (n < 0 || (n > 0 && !jobs)) return fail(AV1G_EINVAL, "bad job array");
    if (mode != AV1G_MODE_BATCHED && mode != AV1G_MODE_PER_FRAME) return fail(AV1G_EINVAL, "mode %d", mode);
    P.n = n;
    P.stage_mask = stage_mask;
    P.mode = mode;
    P.b.frames.resize(n);
    for (int i = 0; i < n; i++) {
        av1g_status st = prepare_frame(jobs[i], P.b.frames[i]);
        if (st != AV1G_OK) {
            std::string m = g_err;
            return fail(st, "job %d: %s", i, m.c_str());
        }
    }
    for (int st = 0; st < ST_COUNT; st++) P.shape[st] = stage_shape(st, P.b.frames[0].hbd);
    // layout: frames | starts (batched: NS x (n+1)) | per-frame starts (n x NS x 2) | scratch
    const int NS = Prepared::NS;
    P.off_starts = ((sizeof(FrameDev) * n) + 255) & ~(size_t)255;
    P.off_pf = P.off_starts + sizeof(int32_t) * NS * (n + 1);
    P.off_scratch = (P.off_pf + sizeof(int32_t) * n * NS * 2 + 255) & ~(size_t)255;
    // per-frame scratch: deblock cell codes, film grain templates / LUTs / offsets
    size_t scratch = 0;
    P.lf_off.assign(n, 0);
    P.grain_off.assign(n, 0);
    for (int i = 0; i < n; i++) {
        const FrameDev& F = P.b.frames[i];
        if ((stage_mask & (1 << ST_DEBLOCK)) && F.do_stage[ST_DEBLOCK]) {
            int cells = cells_deblock(F);
            P.max_cells = cells > P.max_cells ? cells : P.max_cells;
            P.lf_off[i] = P.off_scratch + scratch;
            scratch += ((size_t)cells * 2 + 255) & ~(size_t)255;
        }
        if ((stage_mask & (1 << ST_GRAIN)) && F.do_stage[ST_GRAIN]) {
            P.grain_off[i] = P.off_scratch + scratch;
            scratch += grain_scratch_bytes(F);
        }
    }
    P.total_bytes = P.off_scratch + scratch;
    return AV1G_OK;
}

// Points the records at dev and builds the uploaded prefix.
void bind(Prepared& P, uint8_t* dev) {
    const int n = P.n, NS = Prepared::NS;
    for (int i = 0; i < n; i++) {
        FrameDev& F = P.b.frames[i];
        if (P.lf_off[i]) {
            uint16_t* c = (uint16_t*)(dev + P.lf_off[i]);
            for (int p = 0; p < F.h.num_planes; p++) {
                F.lf_codes[p] = c;
                c += (F.recon[p].w >> 2) * (F.recon[p].h >> 2);
            }
        }
        if (P.grain_off[i]) {
            F.grain_tmpl = (int16_t*)(dev + P.grain_off[i]);
            F.grain_lut = (uint8_t*)(dev + P.grain_off[i] + 3 * 73 * 82 * 2);
            F.grain_offs = F.grain_lut + 768;
        }
    }
    P.host.assign(P.off_scratch, 0);
    memcpy(P.host.data(), P.b.frames.data(), sizeof(FrameDev) * n);
    int32_t* hs = (int32_t*)(P.host.data() + P.off_starts);
    int32_t* hpf = (int32_t*)(P.host.data() + P.off_pf);
    for (int st = 0; st < NS; st++) {
        int32_t acc = 0;
        for (int i = 0; i < n; i++) {
            int c = (P.stage_mask & (1 << (st < ST_COUNT ? st : ST_GRAIN)))
                        ? stage_tiles(P.b.frames[i], st, P.shape[ST_SUPERRES].tile) : 0;
            hs[st * (n + 1) + i] = acc;
            hpf[(i * NS + st) * 2 + 0] = 0;
            hpf[(i * NS + st) * 2 + 1] = c;
            acc += c;
        }
        hs[st * (n + 1) + n] = acc;
        P.totals[st] = acc;
    }
}

// The stage launches of a bound batch (records at dev); returns how many.
int launch_all(const Prepared& P, const uint8_t* dev, cudaStream_t s) {
    const int n = P.n, NS = Prepared::NS;
    const FrameDev* dframes = (const FrameDev*)dev;
    const int32_t* ds = (const int32_t*)(dev + P.off_starts);
    const int32_t* dpf = (const int32_t*)(dev + P.off_pf);
    const int32_t* hpf = (const int32_t*)(P.host.data() + P.off_pf);
    int nl = 0;
    auto launch_stage = [&](int st, const FrameDev* fr, const int32_t* starts, const int32_t* starts_tmpl, int nn,
                            int total, int total_tmpl, int cells) {
        static const char* const names[ST_COUNT] = {"av1g deblock", "av1g cdef", "av1g superres",
                                                     "av1g loop restoration", "av1g film grain"};
        NvtxRange range(names[st]);
        switch (st) {
            case ST_DEBLOCK: if (total) { launch_deblock(fr, starts, nn, total, cells, P.shape[st], s); nl += 2; } break;
            case ST_CDEF: if (total) { launch_cdef(fr, starts, nn, total, P.shape[st], s); nl++; } break;
            case ST_SUPERRES: if (total) { launch_superres(fr, starts, nn, total, P.shape[st], s); nl++; } break;
            case ST_LR: if (total) { launch_lr(fr, starts, nn, total, P.shape[st], s); nl++; } break;
            case ST_GRAIN:
                launch_grain(fr, starts_tmpl, starts, nn, total_tmpl, total, P.shape[st], s);
                nl += (total_tmpl > 0) + (total > 0);
                break;
        }
    };
    for (int st = 0; st < ST_COUNT; st++) {
        if (!(P.stage_mask & (1 << st))) continue;
        if (P.mode == AV1G_MODE_BATCHED) {
            launch_stage(st, dframes, ds + st * (n + 1), ds + ST_COUNT * (n + 1), n, P.totals[st], P.totals[ST_COUNT],
                         P.max_cells);
        } else {
            for (int i = 0; i < n; i++)
                launch_stage(st, dframes + i, dpf + (i * NS + st) * 2, dpf + (i * NS + ST_COUNT) * 2, 1,
                             hpf[(i * NS + st) * 2 + 1], hpf[(i * NS + ST_COUNT) * 2 + 1], cells_deblock(P.b.frames[i]));
        }
    }
    return nl;
}

av1g_status run(const av1g_frame_job* jobs, int n, int stage_mask, int mode, void* stream, int* launches) {
    g_err.clear();
    if (launches) *launches = 0;
    if (n < 0 || (n > 0 && !jobs)) return fail(AV1G_EINVAL, "bad job array");
    if (n == 0) return AV1G_OK;
    Prepared P;
    av1g_status st = prepare(jobs, n, stage_mask, mode, P);
    if (st != AV1G_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    uint8_t* dev = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dev, P.total_bytes, s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    bind(P, dev);
    // the prefix is 256-byte aligned; one or two launches carry a small one
    e = P.off_scratch <= 2 * kUploadChunk ? upload_by_launch(dev, P.host.data(), P.off_scratch, s)
                                          : upload(dev, P.host.data(), P.off_scratch, s);
    if (e != cudaSuccess) {
        cudaFreeAsync(dev, s);
        return cuda_fail(e, "cudaMemcpyAsync");
    }
    int nl = launch_all(P, dev, s);
    e = cudaGetLastError();
    cudaFreeAsync(dev, s);
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    if (launches) *launches = nl;
    return AV1G_OK;
}

}  // namespace

namespace av1g {

// The whole chain for a batch (the serving engine's post-filter step).
av1g_status postfilter_run(const av1g_frame_job* jobs, int n, cudaStream_t s, std::string& err) {
    av1g_status st = run(jobs, n, (1 << ST_COUNT) - 1, AV1G_MODE_BATCHED, s, nullptr);
    if (st != AV1G_OK) err = g_err;
    return st;
}

// The planes holding a job's cropped pre-grain result (the reference-slot
// payload) and its output, after the stage gating.
av1g_status postfilter_result_planes(const av1g_frame_job& j, PlaneDev pre[3], PlaneDev out[3], std::string& err) {
    FrameDev F;
    av1g_status st = prepare_frame(j, F);
    if (st != AV1G_OK) {
        err = g_err;
        return st;
    }
    for (int p = 0; p < 3; p++) {
        pre[p] = F.lr[p];
        out[p] = F.out[p];
    }
    return AV1G_OK;
}

}  // namespace av1g

namespace av1g {
// The framing functions (framing.cpp) report through the same error text.
void set_last_error_text(const std::string& s) { g_err = s; }
}  // namespace av1g

extern "C" {

int32_t av1g_abi_version(void) { return AV1G_ABI_VERSION; }

int32_t av1g_struct_size(const char* name) {
    if (!name) return -1;
    if (!strcmp(name, "av1g_film_grain")) return (int32_t)sizeof(av1g_film_grain);
    if (!strcmp(name, "av1g_frame_header")) return (int32_t)sizeof(av1g_frame_header);
    if (!strcmp(name, "av1g_lr_unit")) return (int32_t)sizeof(av1g_lr_unit);
    if (!strcmp(name, "av1g_mi_grid")) return (int32_t)sizeof(av1g_mi_grid);
    if (!strcmp(name, "av1g_plane")) return (int32_t)sizeof(av1g_plane);
    if (!strcmp(name, "av1g_frame_job")) return (int32_t)sizeof(av1g_frame_job);
    if (!strcmp(name, "av1g_quant_params")) return (int32_t)sizeof(av1g_quant_params);
    if (!strcmp(name, "av1g_tu")) return (int32_t)sizeof(av1g_tu);
    if (!strcmp(name, "av1g_recon_job")) return (int32_t)sizeof(av1g_recon_job);
    if (!strcmp(name, "av1g_intra_tu")) return (int32_t)sizeof(av1g_intra_tu);
    if (!strcmp(name, "av1g_intra_plan_stats")) return (int32_t)sizeof(av1g_intra_plan_stats);
    if (!strcmp(name, "av1g_intra_job")) return (int32_t)sizeof(av1g_intra_job);
    if (!strcmp(name, "av1g_ref_frame")) return (int32_t)sizeof(av1g_ref_frame);
    if (!strcmp(name, "av1g_warp_ctx")) return (int32_t)sizeof(av1g_warp_ctx);
    if (!strcmp(name, "av1g_obmc_neighbour")) return (int32_t)sizeof(av1g_obmc_neighbour);
    if (!strcmp(name, "av1g_inter_pred")) return (int32_t)sizeof(av1g_inter_pred);
    if (!strcmp(name, "av1g_inter_job")) return (int32_t)sizeof(av1g_inter_job);
    if (!strcmp(name, "av1g_warp_sample")) return (int32_t)sizeof(av1g_warp_sample);
    if (!strcmp(name, "av1g_config")) return (int32_t)sizeof(av1g_config);
    if (!strcmp(name, "av1g_seq_info")) return (int32_t)sizeof(av1g_seq_info);
    if (!strcmp(name, "av1g_frame_desc")) return (int32_t)sizeof(av1g_frame_desc);
    if (!strcmp(name, "av1g_frame_out")) return (int32_t)sizeof(av1g_frame_out);
    if (!strcmp(name, "av1g_engine_stats")) return (int32_t)sizeof(av1g_engine_stats);
    if (!strcmp(name, "av1g_mf_store_job")) return (int32_t)sizeof(av1g_mf_store_job);
    if (!strcmp(name, "av1g_mf_slot")) return (int32_t)sizeof(av1g_mf_slot);
    if (!strcmp(name, "av1g_mf_project_job")) return (int32_t)sizeof(av1g_mf_project_job);
    if (!strcmp(name, "av1g_obu")) return (int32_t)sizeof(av1g_obu);
    if (!strcmp(name, "av1g_ivf_header")) return (int32_t)sizeof(av1g_ivf_header);
    if (!strcmp(name, "av1g_ivf_frame")) return (int32_t)sizeof(av1g_ivf_frame);
    if (!strcmp(name, "av1g_operating_point")) return (int32_t)sizeof(av1g_operating_point);
    if (!strcmp(name, "av1g_sequence_header")) return (int32_t)sizeof(av1g_sequence_header);
    if (!strcmp(name, "av1g_frame_prefix")) return (int32_t)sizeof(av1g_frame_prefix);
    if (!strcmp(name, "av1g_tile_list_entry")) return (int32_t)sizeof(av1g_tile_list_entry);
    if (!strcmp(name, "av1g_tile_list_job")) return (int32_t)sizeof(av1g_tile_list_job);
    if (!strcmp(name, "av1g_tile_list_header")) return (int32_t)sizeof(av1g_tile_list_header);
    if (!strcmp(name, "av1g_tile_list_obu_entry")) return (int32_t)sizeof(av1g_tile_list_obu_entry);
    if (!strcmp(name, "av1g_symbol_decoder")) return (int32_t)sizeof(av1g_symbol_decoder);
    if (!strcmp(name, "av1g_ref_state")) return (int32_t)sizeof(av1g_ref_state);
    if (!strcmp(name, "av1g_parsed_frame_header")) return (int32_t)sizeof(av1g_parsed_frame_header);
    if (!strcmp(name, "av1g_tile_span")) return (int32_t)sizeof(av1g_tile_span);
    return -1;
}

const char* av1g_last_error(void) { return g_err.c_str(); }

int32_t av1g_lr_units_in_frame(int32_t unit_size, int32_t plane_size) { return count_units(unit_size, plane_size); }

av1g_status av1g_run_deblock(const av1g_frame_job* jobs, int32_t n, void* stream) {
    return run(jobs, n, 1 << ST_DEBLOCK, AV1G_MODE_BATCHED, stream, nullptr);
}
av1g_status av1g_run_cdef(const av1g_frame_job* jobs, int32_t n, void* stream) {
    return run(jobs, n, 1 << ST_CDEF, AV1G_MODE_BATCHED, stream, nullptr);
}
av1g_status av1g_run_superres(const av1g_frame_job* jobs, int32_t n, void* stream) {
    return run(jobs, n, 1 << ST_SUPERRES, AV1G_MODE_BATCHED, stream, nullptr);
}
av1g_status av1g_run_lr(const av1g_frame_job* jobs, int32_t n, void* stream) {
    return run(jobs, n, 1 << ST_LR, AV1G_MODE_BATCHED, stream, nullptr);
}
av1g_status av1g_run_film_grain(const av1g_frame_job* jobs, int32_t n, void* stream) {
    return run(jobs, n, 1 << ST_GRAIN, AV1G_MODE_BATCHED, stream, nullptr);
}
av1g_status av1g_run_recon(const av1g_recon_job* jobs, int32_t n, void* stream) {
    NvtxRange range("av1g recon");
    g_err.clear();
    if (n < 0 || (n > 0 && !jobs)) return fail(AV1G_EINVAL, "bad job array");
    if (n == 0) return AV1G_OK;
    std::string err;
    av1g_status st = recon_run(jobs, n, (cudaStream_t)stream, err);
    if (st != AV1G_OK) g_err = err;
    return st;
}
av1g_status av1g_run_intra(const av1g_intra_job* jobs, int32_t n, void* stream) {
    NvtxRange range("av1g intra");
    g_err.clear();
    if (n < 0 || (n > 0 && !jobs)) return fail(AV1G_EINVAL, "bad job array");
    if (n == 0) return AV1G_OK;
    // each job's wait status lands in pinned memory after the launch; the
    // call returns once the launch has finished so that it reports it
    thread_local int32_t* t_status = nullptr;
    thread_local int32_t t_cap = 0;
    if (t_cap < n) {
        if (t_status) cudaFreeHost(t_status);
        t_status = nullptr;
        t_cap = 0;
        cudaError_t e = cudaHostAlloc((void**)&t_status, sizeof(int32_t) * (size_t)n, cudaHostAllocDefault);
        if (e != cudaSuccess) return cuda_fail(e, "cudaHostAlloc");
        t_cap = n;
    }
    std::string err;
    av1g_status st = intra_run_status(jobs, n, (cudaStream_t)stream, err, t_status);
    if (st != AV1G_OK) {
        g_err = err;
        return st;
    }
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    for (int i = 0; i < n; i++)
        if (t_status[i])
            return fail(AV1G_EDEVICE, "intra job %d: a superblock dependency wait ran out of time", i);
    return AV1G_OK;
}
av1g_status av1g_run_inter(const av1g_inter_job* jobs, int32_t n, void* stream) {
    NvtxRange range("av1g inter");
    g_err.clear();
    if (n < 0 || (n > 0 && !jobs)) return fail(AV1G_EINVAL, "bad job array");
    if (n == 0) return AV1G_OK;
    std::string err;
    av1g_status st = inter_run(jobs, n, (cudaStream_t)stream, err);
    if (st != AV1G_OK) g_err = err;
    return st;
}
av1g_status av1g_run_mf_store(const av1g_mf_store_job* jobs, int32_t n, void* stream) {
    NvtxRange range("av1g motion field store");
    g_err.clear();
    if (n < 0 || (n > 0 && !jobs)) return fail(AV1G_EINVAL, "bad job array");
    if (n == 0) return AV1G_OK;
    std::string err;
    av1g_status st = mf_store_run(jobs, n, (cudaStream_t)stream, err);
    if (st != AV1G_OK) g_err = err;
    return st;
}
av1g_status av1g_run_mf_project(const av1g_mf_project_job* jobs, int32_t n, void* stream) {
    NvtxRange range("av1g motion field projection");
    g_err.clear();
    if (n < 0 || (n > 0 && !jobs)) return fail(AV1G_EINVAL, "bad job array");
    if (n == 0) return AV1G_OK;
    std::string err;
    av1g_status st = mf_project_run(jobs, n, (cudaStream_t)stream, err);
    if (st != AV1G_OK) g_err = err;
    return st;
}
av1g_status av1g_run_tile_list_output(const av1g_tile_list_job* jobs, int32_t n, void* stream) {
    NvtxRange range("av1g tile list output");
    g_err.clear();
    if (n < 0 || (n > 0 && !jobs)) return fail(AV1G_EINVAL, "bad job array");
    if (n == 0) return AV1G_OK;
    std::string err;
    av1g_status st = tile_list_run(jobs, n, (cudaStream_t)stream, err);
    if (st != AV1G_OK) g_err = err;
    return st;
}
av1g_status av1g_run_postfilter(const av1g_frame_job* jobs, int32_t n, int32_t mode, void* stream,
                                int32_t* launches) {
    return run(jobs, n, (1 << ST_COUNT) - 1, mode, stream, launches);
}

av1g_status av1g_autotune_postfilter(const av1g_frame_job* jobs, int32_t n, void* stream, const char* cache_path) {
    g_err.clear();
    if (n <= 0 || !jobs) return fail(AV1G_EINVAL, "bad job array");
    Prepared P;
    av1g_status st = prepare(jobs, n, (1 << ST_COUNT) - 1, AV1G_MODE_BATCHED, P);
    if (st != AV1G_OK) return st;
    const int hbd = P.b.frames[0].hbd;
    cudaStream_t s = (cudaStream_t)stream;
    uint8_t* dev = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dev, P.total_bytes, s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    bind(P, dev);
    e = cudaMemcpyAsync(dev, P.host.data(), P.off_scratch, cudaMemcpyHostToDevice, s);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    const FrameDev* fr = (const FrameDev*)dev;
    int32_t* hs = (int32_t*)(P.host.data() + P.off_starts);
    const int32_t* ds = (const int32_t*)(dev + P.off_starts);
    auto starts = [&](int stage) { return ds + stage * (n + 1); };
    auto launch = [&](int stage, const StageShape& sh, int total) {
        switch (stage) {
            case ST_DEBLOCK: launch_deblock(fr, starts(stage), n, total, P.max_cells, sh, s); break;
            case ST_CDEF: launch_cdef(fr, starts(stage), n, total, sh, s); break;
            case ST_SUPERRES: launch_superres(fr, starts(stage), n, total, sh, s); break;
            case ST_LR: launch_lr(fr, starts(stage), n, total, sh, s); break;
            default:
                launch_grain(fr, starts(ST_COUNT), starts(ST_GRAIN), n, P.totals[ST_COUNT], total, sh, s);
                break;
        }
    };
    // superres tile counts depend on the tile width
    auto sr_total = [&](int tile) {
        int32_t acc = 0;
        for (int i = 0; i < n; i++) {
            hs[ST_SUPERRES * (n + 1) + i] = acc;
            acc += stage_tiles(P.b.frames[i], ST_SUPERRES, tile);
        }
        hs[ST_SUPERRES * (n + 1) + n] = acc;
        return acc;
    };
    // in chain order, so every stage's input is the previous stage's output
    for (int stage = 0; e == cudaSuccess && stage < ST_COUNT; stage++) {
        if (P.totals[stage] == 0) continue;
        std::vector<StageShape> cands;
        static const int kCtas[ST_COUNT][6] = {{2, 4, 6, 8, 12, 16}, {2, 4, 6, 8, 12, 16}, {4, 8, 16, 32, 0, 0},
                                               {2, 3, 4, 6, 8, 0}, {4, 8, 16, 32, 0, 0}};
        for (int c : kCtas[stage]) {
            if (!c) continue;
            if (stage == ST_SUPERRES)
                for (int t : {256, 512, 1024}) cands.push_back(StageShape{c, t});
            else
                cands.push_back(StageShape{c, 0});
        }
        StageShape best = P.shape[stage];
        float best_ms = 1e30f;
        for (const StageShape& sh : cands) {
            int total = P.totals[stage];
            if (stage == ST_SUPERRES) {
                total = sr_total(sh.tile);
                e = cudaMemcpyAsync(dev + P.off_starts + sizeof(int32_t) * ST_SUPERRES * (n + 1),
                                    hs + ST_SUPERRES * (n + 1), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, s);
                if (e != cudaSuccess) break;
            }
            launch(stage, sh, total);  // warm
            e = cudaEventRecord(e0, s);
            for (int r = 0; r < 3; r++) launch(stage, sh, total);
            if (e == cudaSuccess) e = cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = sh;
            }
        }
        if (e == cudaSuccess) set_stage_shape(stage, hbd, best);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFreeAsync(dev, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "autotune");
    if (cache_path) {
        std::string err;
        av1g_status sv = save_shapes(cache_path, err);
        if (sv != AV1G_OK) return fail(sv, "%s", err.c_str());
    }
    return AV1G_OK;
}

av1g_status av1g_autotune_load(const char* cache_path) {
    g_err.clear();
    if (!cache_path) return fail(AV1G_EINVAL, "no cache path");
    std::string err;
    av1g_status st = load_shapes(cache_path, err);
    return st == AV1G_OK ? st : fail(st, "%s", err.c_str());
}

av1g_status av1g_autotune_get(int32_t stage, int32_t hbd, int32_t* ctas_per_sm, int32_t* tile) {
    g_err.clear();
    if (stage < 0 || stage >= ST_COUNT || !ctas_per_sm || !tile) return fail(AV1G_EINVAL, "stage %d", stage);
    const StageShape sh = stage_shape(stage, hbd);
    *ctas_per_sm = sh.ctas_per_sm;
    *tile = sh.tile;
    return AV1G_OK;
}

struct av1g_chain_graph {
    uint8_t* dev = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int32_t launches = 0;
};

av1g_status av1g_chain_graph_create(const av1g_frame_job* jobs, int32_t n, int32_t stage_mask, int32_t mode,
                                    void* stream, av1g_chain_graph** out) {
    g_err.clear();
    if (!out) return fail(AV1G_EINVAL, "no output pointer");
    *out = nullptr;
    if (n <= 0 || !jobs) return fail(AV1G_EINVAL, "bad job array");
    if (stage_mask <= 0 || (stage_mask & ~((1 << ST_COUNT) - 1))) return fail(AV1G_EINVAL, "stage mask %d", stage_mask);
    Prepared P;
    av1g_status st = prepare(jobs, n, stage_mask, mode, P);
    if (st != AV1G_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    auto* G = new av1g_chain_graph;
    auto bail = [&](cudaError_t e, const char* what) {
        if (G->exec) cudaGraphExecDestroy(G->exec);
        if (G->graph) cudaGraphDestroy(G->graph);
        if (G->dev) cudaFree(G->dev);
        delete G;
        return cuda_fail(e, what);
    };
    cudaError_t e = cudaMalloc((void**)&G->dev, P.total_bytes);
    if (e != cudaSuccess) {
        G->dev = nullptr;
        return bail(e, "cudaMalloc");
    }
    bind(P, G->dev);
    e = cudaMemcpyAsync(G->dev, P.host.data(), P.off_scratch, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        launch_all(P, G->dev, s);  // once uncaptured: validates the launches
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bail(e, "chain run");
    cudaStream_t cs = nullptr;
    e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(e, "cudaStreamCreate");
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        G->launches = launch_all(P, G->dev, cs);
        cudaError_t e2 = cudaStreamEndCapture(cs, &G->graph);
        e = e2 != cudaSuccess ? e2 : cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&G->exec, G->graph, 0);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) return bail(e, "graph capture");
    *out = G;
    return AV1G_OK;
}

av1g_status av1g_chain_graph_launch(av1g_chain_graph* g, void* stream) {
    g_err.clear();
    if (!g || !g->exec) return fail(AV1G_EINVAL, "no graph");
    cudaError_t e = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
    return e == cudaSuccess ? AV1G_OK : cuda_fail(e, "cudaGraphLaunch");
}

int32_t av1g_chain_graph_launches(const av1g_chain_graph* g) { return g ? g->launches : 0; }

av1g_status av1g_chain_graph_destroy(av1g_chain_graph* g) {
    g_err.clear();
    if (!g) return AV1G_OK;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    cudaError_t e = g->dev ? cudaFree(g->dev) : cudaSuccess;
    delete g;
    return e == cudaSuccess ? AV1G_OK : cuda_fail(e, "cudaFree");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Film grain without device allocation.
//
// For callers that may not allocate device memory on the per-frame path: a
// host application that reserves the whole device-memory budget up front
// (broadcast and other real-time pipelines) and forbids its plug-ins from
// allocating while frames flow, because an allocation there can stall on the
// allocator or fail once the pool is full.  av1g_run_film_grain takes its
// frame records and grain scratch from the stream-ordered allocator; this
// variant keeps them in one fixed array in device memory instead.
//
// The array is a file-scope static __device__ object of
// AV1G_NOALLOC_SCRATCH_BYTES, so every GPU that loads this library holds it
// until the process exits.  Host code may not use the symbol as a device
// address: on first use on a device (with that device current) the entry
// point asks the runtime for the array's address with cudaGetSymbolAddress,
// checks the result, caches it per device, and passes that address to the
// kernels.  Every call on a device shares the one array and the array keeps
// the previous call's contents: the kernels write every template, table and
// offset before reading it, so nothing needs clearing, and calls that overlap
// on the GPU (two streams, or a second call before the first has finished on
// another stream) race on the array.
// ---------------------------------------------------------------------------

static __device__ __align__(256) uint8_t g_noalloc_scratch[AV1G_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mu;
void* g_noalloc_addr[256];  // per device ordinal; null until set up on that device

// Device address of the static scratch on the current device (set up once per device).
av1g_status noalloc_address(uint8_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= 256) return fail(AV1G_EDEVICE, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
        g_noalloc_addr[dev] = p;
    }
    *out = (uint8_t*)g_noalloc_addr[dev];
    return AV1G_OK;
}

// Host staging of the frame records and tile starts (no heap allocation).
thread_local FrameDev t_noalloc_frames[AV1G_NOALLOC_MAX_FRAMES];
thread_local int32_t t_noalloc_starts[2 * (AV1G_NOALLOC_MAX_FRAMES + 1)];

}  // namespace

extern "C" av1g_status av1g_run_film_grain_noalloc(const av1g_frame_job* jobs, int32_t n, void* stream) {
    g_err.clear();
    if (n < 0 || (n > 0 && !jobs)) return fail(AV1G_EINVAL, "bad job array");
    if (n > AV1G_NOALLOC_MAX_FRAMES)
        return fail(AV1G_EINVAL, "%d frames exceed the %d-frame limit of the allocation-free entry point", n,
                    AV1G_NOALLOC_MAX_FRAMES);
    if (n == 0) return AV1G_OK;
    cudaStream_t s = (cudaStream_t)stream;
    FrameDev* fr = t_noalloc_frames;
    for (int i = 0; i < n; i++) {
        av1g_status st = prepare_frame(jobs[i], fr[i]);
        if (st != AV1G_OK) {
            std::string m = g_err;
            return fail(st, "job %d: %s", i, m.c_str());
        }
    }
    // layout: frames | template starts (n+1) | blend starts (n+1) | per-frame grain scratch
    size_t off_starts = (sizeof(FrameDev) * n + 255) & ~(size_t)255;
    size_t off_scratch = (off_starts + sizeof(int32_t) * 2 * (n + 1) + 255) & ~(size_t)255;
    size_t total = off_scratch;
    for (int i = 0; i < n; i++)
        if (fr[i].do_stage[ST_GRAIN]) total += grain_scratch_bytes(fr[i]);
    if (total > AV1G_NOALLOC_SCRATCH_BYTES)
        return fail(AV1G_EINVAL, "batch needs %zu bytes of scratch, above the %d-byte static array", total,
                    AV1G_NOALLOC_SCRATCH_BYTES);
    uint8_t* base = nullptr;
    av1g_status st = noalloc_address(&base);
    if (st != AV1G_OK) return st;
    int32_t* hs = t_noalloc_starts;
    size_t off = off_scratch;
    int tmpl = 0, blend = 0;
    for (int i = 0; i < n; i++) {
        FrameDev& F = fr[i];
        hs[i] = tmpl;
        hs[n + 1 + i] = blend;
        if (F.do_stage[ST_GRAIN]) {
            F.grain_tmpl = (int16_t*)(base + off);
            F.grain_lut = (uint8_t*)(base + off + 3 * 73 * 82 * 2);
            F.grain_offs = F.grain_lut + 768;
            off += grain_scratch_bytes(F);
            tmpl += 1;
            blend += tiles_grain_blend(F);
        }
    }
    hs[n] = tmpl;
    hs[2 * n + 1] = blend;
    cudaError_t e = cudaMemcpyAsync(base, fr, sizeof(FrameDev) * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(base + off_starts, hs, sizeof(int32_t) * 2 * (n + 1), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
    const int32_t* ds = (const int32_t*)(base + off_starts);
    launch_grain((const FrameDev*)base, ds, ds + n + 1, n, tmpl, blend, stage_shape(ST_GRAIN, fr[0].hbd), s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return AV1G_OK;
}
