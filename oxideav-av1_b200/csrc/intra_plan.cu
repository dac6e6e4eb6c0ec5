// intra_plan.cu — host side of the intra wavefront: validation of the jobs
// and the dependency analysis behind one persistent launch (intra.cu).
//
// Walks each frame's TUs in decode order (transform_block_emit,
// src/cdf.rs:32540-32910) and records the areas every TU reads: the row above
// and the column to its left that intra_predict_block_samples gathers
// (cdf.rs:17030-17075, availability from the TU's flags), the co-located luma
// of chroma from luma (cdf.rs:17256-17340) and the window of an intra block
// copy (cdf.rs:19235).  Inside a superblock each TU gets a level one above
// the last writer of every 4x4 cell it reads or writes and the last reader of
// every cell it writes; across superblocks a read of another superblock's
// area orders the two in decode order.  Replaying the levels and the waits
// therefore reproduces the reference's sequential decode sample for sample.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "av1_spec_tables.h"
#include "intra_plan.h"
#include "wedge.cuh"

namespace av1g {

namespace {

constexpr int kW[19] = AV1T_TX_WIDTH_INIT;
constexpr int kH[19] = AV1T_TX_HEIGHT_INIT;

// An area of one plane, inclusive, in that plane's sample coordinates.
struct Rect {
    int p, x0, y0, x1, y1;
};

// A rect's 4x4 cells inside the current superblock (empty when cx1 < cx0 or cy1 < cy0).
struct Cells {
    int base, stride, cx0, cx1, cy0, cy1;
};

}  // namespace

av1g_status intra_plan(const av1g_intra_job* jobs, int n, IntraPlan& plan, std::string& err) {
    plan = IntraPlan{};
    plan.frames.resize(n);
    plan.map_base.assign(n, 0);
    struct SbHost {
        int frame, seq, depth;
        SbItem item;
        std::vector<int3> waits;  // {level, global superblock index, progress}
    };
    std::vector<SbHost> sbs_all;
    size_t total_tus = 0;
    for (int i = 0; i < n; i++) total_tus += jobs[i].num_tus > 0 ? (size_t)jobs[i].num_tus : 0;
    plan.tus.reserve(total_tus);
    plan.lvtab.reserve(total_tus + 1024);
    std::vector<int> lvl, order, bucket, sb_index, hw, hr, fwl, pend_head;
    struct Pend {
        int sb, level, next;
    };
    std::vector<Pend> pend;
    std::vector<uint32_t> wedge;
    for (int i = 0; i < n; i++) {
        const av1g_intra_job& j = jobs[i];
        if (!j.hdr || !j.quant || j.num_tus < 0 || (j.num_tus > 0 && !j.tus) || (j.sb_size != 64 && j.sb_size != 128) ||
            j.palette_map_bytes < 0 || (j.palette_map_bytes > 0 && !j.palette_maps)) {
            err = "intra job " + std::to_string(i) + ": missing header/quantizer/TUs/maps or superblock size not 64/128";
            return AV1G_EINVAL;
        }
        const av1g_frame_header& h = *j.hdr;
        if (h.bit_depth != 8 && h.bit_depth != 10 && h.bit_depth != 12) {
            err = "intra job " + std::to_string(i) + ": bit depth";
            return AV1G_EINVAL;
        }
        if (h.num_planes != 1 && h.num_planes != 3) {
            err = "intra job " + std::to_string(i) + ": plane count";
            return AV1G_EINVAL;
        }
        IntraFrame& F = plan.frames[i];
        memset(&F, 0, sizeof F);
        F.bd = h.bit_depth;
        F.hbd = h.bit_depth > 8;
        F.q = *j.quant;
        F.coeffs = j.coeffs;
        F.ssx = h.subsampling_x;
        F.ssy = h.subsampling_y;
        F.np = h.num_planes;
        int pw[3] = {}, ph[3] = {};
        for (int p = 0; p < h.num_planes; p++) {
            int sx = p ? h.subsampling_x : 0, sy = p ? h.subsampling_y : 0;
            pw[p] = (h.mi_cols * 4) >> sx;
            ph[p] = (h.mi_rows * 4) >> sy;
            const av1g_plane& pl = j.planes[p];
            if (!pl.data || pl.width < pw[p] || pl.height < ph[p] || pl.stride < pw[p] * (F.hbd ? 2 : 1) ||
                (pl.stride & 15) || ((uintptr_t)pl.data & 15)) {
                err = "intra job " + std::to_string(i) + ": plane " + std::to_string(p);
                return AV1G_EINVAL;
            }
            F.planes[p] = PlaneDev{(uint8_t*)pl.data, pl.stride, pw[p], ph[p]};
        }
        const int sb = j.sb_size, log2sb = sb == 128 ? 7 : 6;
        const int ssx = h.subsampling_x, ssy = h.subsampling_y;
        {
            size_t cb = (size_t)sb * sb;
            if (h.num_planes > 1) cb += 2 * (size_t)(sb >> ssx) * (sb >> ssy);
            plan.cache_bytes = std::max(plan.cache_bytes, cb * sizeof(uint16_t));
        }
        plan.map_base[i] = plan.maps.size();
        if (j.palette_map_bytes > 0) plan.maps.insert(plan.maps.end(), j.palette_maps, j.palette_maps + j.palette_map_bytes);

        // --- validation, and the superblocks in decode order ---
        struct Sb {
            int sbx, sby, first, count;
        };
        std::vector<Sb> sbs;
        const int sb_cols = (h.mi_cols * 4 + sb - 1) >> log2sb, sb_rows = (h.mi_rows * 4 + sb - 1) >> log2sb;
        sb_index.assign((size_t)sb_cols * sb_rows, -1);  // superblock grid -> decode-order index
        wedge.assign(j.num_tus, 0);
        long long prev = -1;
        for (int k = 0; k < j.num_tus; k++) {
            const av1g_intra_tu& t = j.tus[k];
            bool res = t.flags & AV1G_INTRA_RESIDUAL;
            bool fi_ok = !(t.plane == 0 && t.filter_intra_mode < 5) || (t.tx_size != 4 && t.tx_size != 11 &&
                                                                        t.tx_size != 12 && t.tx_size != 17 &&
                                                                        t.tx_size != 18);
            if (t.tx_size >= 19 || t.plane >= h.num_planes || !fi_ok ||
                (res && (t.res.tx_size != t.tx_size || t.res.plane != t.plane || t.res.x != t.x || t.res.y != t.y ||
                         t.res.tx_type >= 16 || !j.coeffs))) {
                err = "intra job " + std::to_string(i) + ": TU " + std::to_string(k) + " is malformed";
                return AV1G_EINVAL;
            }
            const int tw = kW[t.tx_size], th = kH[t.tx_size];
            const int pss_x = t.plane ? ssx : 0, pss_y = t.plane ? ssy : 0;
            const int sbx = (t.x << pss_x) >> log2sb, sby = (t.y << pss_y) >> log2sb;
            // a TU lies inside its superblock (the superblock's copy holds all it writes)
            if (t.x + tw > ((sbx + 1) << log2sb) >> pss_x || t.y + th > ((sby + 1) << log2sb) >> pss_y ||
                t.x >= pw[t.plane] || t.y >= ph[t.plane]) {
                err = "intra job " + std::to_string(i) + ": TU " + std::to_string(k) +
                      " leaves its superblock or the plane";
                return AV1G_EINVAL;
            }
            if (t.interintra) {
                // the intra half of an inter-intra block: an II mode's intra
                // mode (DC, V, H, SMOOTH) over the whole block, then the blend
                static const uint8_t ii_to_intra[4] = {0, 1, 2, 9};
                const av1g_plane& sp = j.interintra_in[t.plane];
                wedge::Orient o{};
                bool ok = t.interintra <= 2 && t.interintra_mode <= 3 && t.mode == ii_to_intra[t.interintra_mode] &&
                          t.filter_intra_mode >= 5 && !(t.flags & AV1G_INTRA_CFL) && sp.data &&
                          sp.width >= pw[t.plane] && sp.height >= ph[t.plane] &&
                          sp.stride >= pw[t.plane] * (F.hbd ? 2 : 1) && !(sp.stride & 15);
                if (ok && t.interintra == 2) ok = wedge::orient(t.mi_size, t.wedge_index, 0, tw, th, pss_x, pss_y, o);
                if (!ok) {
                    err = "intra job " + std::to_string(i) + ": inter-intra TU " + std::to_string(k) + " is malformed";
                    return AV1G_EINVAL;
                }
                F.side[t.plane] = PlaneDev{(uint8_t*)sp.data, sp.stride, pw[t.plane], ph[t.plane]};
                // the device copy of the TU carries the wedge window in
                // palette_map (an inter-intra TU has no palette)
                wedge[k] = (uint32_t)o.dir | ((uint32_t)o.xoff << 8) | ((uint32_t)o.yoff << 16) |
                           ((uint32_t)o.invert << 24);
            }
            if (t.mode == AV1G_INTRA_MODE_PALETTE) {
                // predict_palette's checks (cdf.rs:11907-11960)
                long long last = (long long)t.palette_map + (long long)(th - 1) * t.palette_stride + (tw - 1);
                bool ok = t.palette_size >= 1 && t.palette_size <= 8 && t.palette_stride >= tw &&
                          last < j.palette_map_bytes;
                for (int r = 0; ok && r < th; r++)
                    for (int c = 0; ok && c < tw; c++)
                        ok = j.palette_maps[t.palette_map + (long long)r * t.palette_stride + c] < t.palette_size;
                if (!ok) {
                    err = "intra job " + std::to_string(i) + ": palette TU " + std::to_string(k) + " is malformed";
                    return AV1G_EINVAL;
                }
            }
            if (t.mode == AV1G_INTRA_MODE_INTRABC &&
                (std::abs((int)t.mv[0]) >= (1 << 14) || std::abs((int)t.mv[1]) >= (1 << 14))) {
                err = "intra job " + std::to_string(i) + ": intra block copy TU " + std::to_string(k) +
                      " has a motion vector out of range";
                return AV1G_EINVAL;
            }
            const long long key = (long long)sby * sb_cols + sbx;
            if (key != prev) {
                if (sb_index[key] >= 0) {
                    err = "intra job " + std::to_string(i) + ": TUs of a superblock are not contiguous in decode order";
                    return AV1G_EINVAL;
                }
                sb_index[key] = (int)sbs.size();
                sbs.push_back(Sb{sbx, sby, k, 0});
                prev = key;
            }
            sbs.back().count++;
        }

        // --- the areas a TU reads, inside the plane (the kernel clamps every
        // coordinate the same way); returns how many ---
        auto reads = [&](const av1g_intra_tu& t, Rect* out) {
            int m = 0;
            const int p = t.plane, W = kW[t.tx_size], H = kH[t.tx_size];
            const int sx = t.x, sy = t.y, mx = pw[p] - 1, my = ph[p] - 1;
            if (t.mode < 13) {
                const bool ha = (t.flags & AV1G_INTRA_HAVE_ABOVE) && sy > 0;
                const bool hl = (t.flags & AV1G_INTRA_HAVE_LEFT) && sx > 0;
                const bool har = t.flags & AV1G_INTRA_HAVE_ABOVE_RIGHT, hbl = t.flags & AV1G_INTRA_HAVE_BELOW_LEFT;
                if (ha)
                    out[m++] = Rect{p, std::min(hl ? sx - 1 : sx, mx), std::min(sy - 1, my),
                                    std::min(mx, sx + (har ? 2 * W : W) - 1), std::min(sy - 1, my)};
                if (hl)
                    out[m++] = Rect{p, std::min(sx - 1, mx), std::min(ha ? sy - 1 : sy, my), std::min(sx - 1, mx),
                                    std::min(my, sy + (hbl ? 2 * H : H) - 1)};
            }
            if (t.mode == AV1G_INTRA_MODE_INTRABC) {
                const int pss_x = p ? ssx : 0, pss_y = p ? ssy : 0;
                const int stx = (sx << 10) + ((2 * t.mv[1]) >> pss_x) * 64 + 32;
                const int sty = (sy << 10) + ((2 * t.mv[0]) >> pss_y) * 64 + 32;
                out[m++] = Rect{p, std::min(std::max((stx >> 10) - 3, 0), mx), std::min(std::max((sty >> 10) - 3, 0), my),
                                std::min(std::max((stx >> 10) + W - 1 + 4, 0), mx),
                                std::min(std::max((sty >> 10) + H - 1 + 4, 0), my)};
            }
            if ((t.flags & AV1G_INTRA_CFL) && p > 0) {
                const int cx = std::max((int)t.max_luma_w - (1 << ssx), 0), cy = std::max((int)t.max_luma_h - (1 << ssy), 0);
                const int y0 = std::min(sy << ssy, cy), y1 = std::min(std::min((sy + H - 1) << ssy, cy) + ssy, ph[0] - 1);
                const int x0 = std::min(sx << ssx, cx), x1 = std::min(std::min((sx + W - 1) << ssx, cx) + ssx, pw[0] - 1);
                if (y0 <= y1 && x0 <= x1) out[m++] = Rect{0, x0, y0, x1, y1};
            }
            return m;
        };

        // --- levels inside each superblock and waits between superblocks ---
        const int gbase = (int)sbs_all.size();
        for (size_t q = 0; q < sbs.size(); q++) {
            SbHost sh;
            sh.frame = i;
            sh.seq = (int)q;
            sh.depth = 0;
            sh.item = SbItem{i, 0, 0, 0, 0, sbs[q].sbx << log2sb, sbs[q].sby << log2sb, log2sb, 0, 0};
            sbs_all.push_back(std::move(sh));
        }
        // 4x4-cell hazard maps of the current superblock: the last writer's
        // and the last reader's level plus `epoch`; entries of earlier
        // superblocks lie below epoch and so count as no constraint
        int gw[3], gh[3], cbase[3], ncell = 0;
        for (int p = 0; p < 3; p++) {
            gw[p] = (sb >> (p ? ssx : 0)) >> 2;
            gh[p] = (sb >> (p ? ssy : 0)) >> 2;
            cbase[p] = ncell;
            if (p < h.num_planes) ncell += gw[p] * gh[p];
        }
        hw.assign(ncell, -1);
        hr.assign(ncell, -1);
        // frame-wide, per 4x4 cell inside the plane: the level of its last
        // writer (within that writer's superblock), and the reads made of it
        // by superblocks decoded before the one it belongs to
        int fgw[3] = {}, fgh[3] = {}, fbase[3] = {}, nf = 0;
        for (int p = 0; p < h.num_planes; p++) {
            fgw[p] = (pw[p] + 3) >> 2;
            fgh[p] = (ph[p] + 3) >> 2;
            fbase[p] = nf;
            nf += fgw[p] * fgh[p];
        }
        fwl.assign(nf, -1);
        pend_head.assign(nf, -1);
        pend.clear();
        int epoch = 0;
        for (size_t q = 0; q < sbs.size(); q++) {
            const Sb& b = sbs[q];
            std::vector<int3>& waits = sbs_all[gbase + q].waits;  // {level, superblock, progress}
            lvl.resize(b.count);
            int nlv = 0;
            int ox[3], oy[3];
            for (int p = 0; p < 3; p++) {
                ox[p] = (b.sbx << log2sb) >> (p ? ssx : 0);
                oy[p] = (b.sby << log2sb) >> (p ? ssy : 0);
            }
            auto cells_of = [&](const Rect& r) {
                const int p = r.p;
                const int x0 = std::max(r.x0 - ox[p], 0), x1 = std::min(r.x1 - ox[p], 4 * gw[p] - 1);
                const int y0 = std::max(r.y0 - oy[p], 0), y1 = std::min(r.y1 - oy[p], 4 * gh[p] - 1);
                return Cells{cbase[p], gw[p], x0 >> 2, x1 < x0 ? -1 : x1 >> 2, y0 >> 2, y1 < y0 ? -1 : y1 >> 2};
            };
            for (int k = 0; k < b.count; k++) {
                const av1g_intra_tu& t = j.tus[b.first + k];
                Rect rr[4];
                const int nr = reads(t, rr);
                Cells rc[4];
                int L = 0;
                for (int u = 0; u < nr; u++) {
                    rc[u] = cells_of(rr[u]);
                    const Cells& c = rc[u];
                    for (int cy = c.cy0; cy <= c.cy1; cy++)
                        for (int cx = c.cx0; cx <= c.cx1; cx++) L = std::max(L, hw[c.base + cy * c.stride + cx] - epoch + 1);
                }
                const Cells wc = cells_of(Rect{t.plane, t.x, t.y, t.x + kW[t.tx_size] - 1, t.y + kH[t.tx_size] - 1});
                for (int cy = wc.cy0; cy <= wc.cy1; cy++)
                    for (int cx = wc.cx0; cx <= wc.cx1; cx++) {
                        const int c = wc.base + cy * wc.stride + cx;
                        L = std::max(L, std::max(hw[c], hr[c]) - epoch + 1);
                    }
                for (int u = 0; u < nr; u++) {
                    const Cells& c = rc[u];
                    for (int cy = c.cy0; cy <= c.cy1; cy++)
                        for (int cx = c.cx0; cx <= c.cx1; cx++) {
                            int& v = hr[c.base + cy * c.stride + cx];
                            v = std::max(v, epoch + L);
                        }
                }
                for (int cy = wc.cy0; cy <= wc.cy1; cy++)
                    for (int cx = wc.cx0; cx <= wc.cx1; cx++) hw[wc.base + cy * wc.stride + cx] = epoch + L;
                lvl[k] = L;
                nlv = std::max(nlv, L + 1);
                // reads of other superblocks' areas: wait for the level that
                // wrote the cell (an earlier superblock), or make the later
                // superblock's writer wait for this reader
                int3 tw[8];  // this TU's waits, one per superblock
                int ntw = 0;
                for (int u = 0; u < nr; u++) {
                    const Rect& r = rr[u];
                    const int p = r.p, sw = sb >> (p ? ssx : 0), shh = sb >> (p ? ssy : 0);
                    if (r.x0 >= ox[p] && r.x1 < ox[p] + sw && r.y0 >= oy[p] && r.y1 < oy[p] + shh) continue;
                    for (int cy = r.y0 >> 2; cy <= r.y1 >> 2; cy++) {
                        const int py = cy << 2;
                        const bool row_in = py >= oy[p] && py < oy[p] + shh;
                        const int by = (py << (p ? ssy : 0)) >> log2sb;
                        for (int cx = r.x0 >> 2; cx <= r.x1 >> 2; cx++) {
                            const int px = cx << 2;
                            if (row_in && px >= ox[p] && px < ox[p] + sw) continue;
                            const int o = sb_index[(size_t)by * sb_cols + ((px << (p ? ssx : 0)) >> log2sb)];
                            if (o < 0) continue;
                            const int fc = fbase[p] + cy * fgw[p] + cx;
                            if (o < (int)q) {
                                const int need = fwl[fc] + 1;
                                if (need <= 0) continue;
                                int a = 0;
                                while (a < ntw && tw[a].y != gbase + o) a++;
                                if (a == ntw) {
                                    if (ntw == 8) {
                                        waits.push_back(int3{L, gbase + o, need});
                                        continue;
                                    }
                                    tw[ntw++] = int3{L, gbase + o, need};
                                } else {
                                    tw[a].z = std::max(tw[a].z, need);
                                }
                            } else {
                                pend.push_back(Pend{gbase + (int)q, L, pend_head[fc]});
                                pend_head[fc] = (int)pend.size() - 1;
                            }
                        }
                    }
                }
                waits.insert(waits.end(), tw, tw + ntw);
                // this TU's cells (inside the plane): their writer, and the
                // reads earlier superblocks made of them before this write
                {
                    const int p = t.plane;
                    const int cx0 = t.x >> 2, cy0 = t.y >> 2;
                    const int cx1 = std::min((t.x + kW[t.tx_size] - 1) >> 2, fgw[p] - 1);
                    const int cy1 = std::min((t.y + kH[t.tx_size] - 1) >> 2, fgh[p] - 1);
                    for (int cy = cy0; cy <= cy1; cy++)
                        for (int cx = cx0; cx <= cx1; cx++) {
                            const int fc = fbase[p] + cy * fgw[p] + cx;
                            fwl[fc] = L;
                            for (int e = pend_head[fc]; e >= 0; e = pend[e].next)
                                waits.push_back(int3{L, pend[e].sb, pend[e].level + 1});
                            pend_head[fc] = -1;
                        }
                }
            }
            epoch += b.count + 1;
            // the waits: the strongest per (level, superblock), and only those
            // a smaller level does not already imply
            std::sort(waits.begin(), waits.end(), [](const int3& a, const int3& c) {
                return a.y != c.y ? a.y < c.y : (a.x != c.x ? a.x < c.x : a.z > c.z);
            });
            {
                size_t o = 0;
                int cur = -1, best = 0;
                for (size_t u = 0; u < waits.size(); u++) {
                    const int3 w = waits[u];
                    if (w.y != cur) {
                        cur = w.y;
                        best = 0;
                    }
                    if (w.z > best) {
                        best = w.z;
                        waits[o++] = w;
                    }
                }
                waits.resize(o);
                std::sort(waits.begin(), waits.end(), [](const int3& a, const int3& c) { return a.x < c.x; });
            }
            // the TUs by level, a level's small TUs before its large ones (a
            // counting sort on 2 * level + large, stable in decode order)
            auto large = [&](int k) {
                const int tx = j.tus[b.first + k].tx_size;
                return kW[tx] * kH[tx] > kIntraSmallPx ? 1 : 0;
            };
            bucket.assign(2 * nlv + 1, 0);
            for (int k = 0; k < b.count; k++) bucket[2 * lvl[k] + large(k) + 1]++;
            for (int u = 1; u <= 2 * nlv; u++) bucket[u] += bucket[u - 1];
            order.resize(b.count);
            for (int k = 0; k < b.count; k++) order[bucket[2 * lvl[k] + large(k)]++] = k;
            SbItem& it = sbs_all[gbase + q].item;
            it.lv_first = (int)plan.lvtab.size();
            it.nlv = nlv;
            it.tu_first = (int)plan.tus.size();
            it.tu_end = it.tu_first + b.count;
            int cur = -1;
            for (int u = 0; u < b.count; u++) {
                const int k = order[u];
                const int at = (int)plan.tus.size();
                if (lvl[k] != cur) {
                    cur = lvl[k];
                    plan.lvtab.push_back(int2{at, at});
                }
                if (!large(k)) plan.lvtab.back().y = at + 1;
                plan.tus.push_back(j.tus[b.first + k]);
                if (plan.tus.back().interintra) plan.tus.back().palette_map = wedge[b.first + k];
            }
            const int end = (int)plan.tus.size();
            plan.lvtab.push_back(int2{end, end});
            // dependency depth (every wait points to a superblock earlier in decode order)
            SbHost& sh = sbs_all[gbase + q];
            for (const int3& w : sh.waits) sh.depth = std::max(sh.depth, sbs_all[w.y].depth + 1);
        }
    }
    // claim order: depth, then frame, then decode order — a topological order
    // of the waits, so a CTA only ever waits for superblocks claimed earlier
    std::vector<int> claim(sbs_all.size());
    for (size_t q = 0; q < claim.size(); q++) claim[q] = (int)q;
    std::stable_sort(claim.begin(), claim.end(), [&](int a, int b) {
        const SbHost& x = sbs_all[a];
        const SbHost& y = sbs_all[b];
        if (x.depth != y.depth) return x.depth < y.depth;
        if (x.frame != y.frame) return x.frame < y.frame;
        return x.seq < y.seq;
    });
    std::vector<int> pos(sbs_all.size());
    for (size_t q = 0; q < claim.size(); q++) pos[claim[q]] = (int)q;
    for (size_t q = 0, run = 0; q < claim.size(); q++) {
        run = (q > 0 && sbs_all[claim[q]].depth == sbs_all[claim[q - 1]].depth) ? run + 1 : 1;
        plan.width = std::max(plan.width, (int)run);
        plan.depth = std::max(plan.depth, sbs_all[claim[q]].depth + 1);
    }
    // the levels some superblock waits for are published (progress z means
    // z levels done: published after level z - 1)
    for (const SbHost& sh : sbs_all)
        for (const int3& w : sh.waits) plan.lvtab[sbs_all[w.y].item.lv_first + w.z - 1].y |= kLevelPublished;
    plan.items.resize(claim.size());
    for (size_t q = 0; q < claim.size(); q++) {
        const SbHost& sh = sbs_all[claim[q]];
        SbItem it = sh.item;
        it.wait_first = (int)plan.waits.size();
        it.nwait = (int)sh.waits.size();
        for (const int3& w : sh.waits) plan.waits.push_back(int4{w.x, pos[w.y], w.z, 0});
        plan.items[q] = it;
    }
    return AV1G_OK;
}

}  // namespace av1g
