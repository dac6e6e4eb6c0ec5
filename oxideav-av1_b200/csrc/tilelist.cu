// tilelist.cu — §7.3.1 output assembly of a large-scale-tile decode.
//
// Replaces the placement loop of decode_tile_list (src/tile_list.rs:693-716):
// decoded camera tile `k` (extracted from its camera frame at the tile's
// origin, decode_camera_tile tile_list.rs:600-646) is written into the output
// frame at (TileWidth * (k % widthInTiles), TileHeight * (k / widthInTiles)),
// chroma at those positions shifted by the subsampling; output tiles no entry
// covers keep the output buffer's initial zeros.  One CTA per (tile list,
// output tile, plane); rows are moved in 16-byte pieces when source, target
// and row length allow it.
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace av1g {

namespace {

constexpr int kThreads = 128;

struct JobDev {
    int32_t tile_w, tile_h, wt, ht;
    int32_t np, ssx, ssy, hbd;
    int32_t nent, ent_first;
    uint8_t* out[3];
    int32_t out_stride[3];
};

struct EntryDev {
    const uint8_t* src[3];
    int32_t stride[3];
    int32_t x0, y0;
};

__global__ void __launch_bounds__(kThreads) tile_list_kernel(const JobDev* __restrict__ jobs,
                                                             const EntryDev* __restrict__ ents,
                                                             const int32_t* __restrict__ starts, int n, int total) {
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int j = find_frame(starts, n, t);
        const JobDev& J = jobs[j];
        const int local = t - starts[j];
        const int k = local / J.np, p = local - k * J.np;
        const int sx = p ? J.ssx : 0, sy = p ? J.ssy : 0;
        const int tw = (J.tile_w + sx) >> sx, th = (J.tile_h + sy) >> sy;
        const int dx = (J.tile_w * (k % J.wt)) >> sx, dy = (J.tile_h * (k / J.wt)) >> sy;
        const int bps = J.hbd ? 2 : 1;
        const int row_bytes = tw * bps;
        uint8_t* dst = J.out[p] + (size_t)dy * J.out_stride[p] + (size_t)dx * bps;
        const int ds = J.out_stride[p];
        if (k >= J.nent) {  // not covered: zeros
            const bool vec = !((reinterpret_cast<uintptr_t>(dst) | (uintptr_t)ds | (uintptr_t)row_bytes) & 15);
            if (vec) {
                const int per = row_bytes >> 4;
                for (int q = threadIdx.x; q < th * per; q += kThreads)
                    reinterpret_cast<uint4*>(dst + (size_t)(q / per) * ds)[q % per] = make_uint4(0, 0, 0, 0);
            } else {
                for (int q = threadIdx.x; q < th * row_bytes; q += kThreads)
                    dst[(size_t)(q / row_bytes) * ds + q % row_bytes] = 0;
            }
            continue;
        }
        const EntryDev& E = ents[J.ent_first + k];
        const int ss = E.stride[p];
        const uint8_t* src = E.src[p] + (size_t)(E.y0 >> sy) * ss + (size_t)(E.x0 >> sx) * bps;
        const bool vec = !((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src) | (uintptr_t)ds |
                            (uintptr_t)ss | (uintptr_t)row_bytes) & 15);
        if (vec) {
            const int per = row_bytes >> 4;
            for (int q = threadIdx.x; q < th * per; q += kThreads) {
                const int r = q / per, c = q - r * per;
                reinterpret_cast<uint4*>(dst + (size_t)r * ds)[c] =
                    __ldg(reinterpret_cast<const uint4*>(src + (size_t)r * ss) + c);
            }
        } else {
            for (int q = threadIdx.x; q < th * row_bytes; q += kThreads) {
                const int r = q / row_bytes, c = q - r * row_bytes;
                dst[(size_t)r * ds + c] = src[(size_t)r * ss + c];
            }
        }
    }
}

}  // namespace

av1g_status tile_list_run(const av1g_tile_list_job* jobs, int n, cudaStream_t s, std::string& err) {
    std::vector<JobDev> jd(n);
    std::vector<EntryDev> ed;
    std::vector<int32_t> starts(n + 1, 0);
    long long total = 0;
    for (int i = 0; i < n; i++) {
        const av1g_tile_list_job& J = jobs[i];
        const std::string who = "tile list job " + std::to_string(i);
        if (J.tile_width <= 0 || J.tile_height <= 0 || J.width_in_tiles < 1 || J.width_in_tiles > 256 ||
            J.height_in_tiles < 1 || J.height_in_tiles > 256 || (J.num_planes != 1 && J.num_planes != 3) ||
            J.subsampling_x < 0 || J.subsampling_x > 1 || J.subsampling_y < 0 || J.subsampling_y > 1 ||
            (J.bit_depth != 8 && J.bit_depth != 10 && J.bit_depth != 12) || J.num_entries < 1 ||
            J.num_entries > J.width_in_tiles * J.height_in_tiles || !J.entries) {
            err = who + ": tile size, output size in tiles, format or entry count out of range "
                        "(1 <= entries <= width_in_tiles * height_in_tiles)";
            return AV1G_EINVAL;
        }
        const int bps = J.bit_depth > 8 ? 2 : 1;
        JobDev& d = jd[i];
        memset(&d, 0, sizeof d);
        d.tile_w = J.tile_width;
        d.tile_h = J.tile_height;
        d.wt = J.width_in_tiles;
        d.ht = J.height_in_tiles;
        d.np = J.num_planes;
        d.ssx = J.subsampling_x;
        d.ssy = J.subsampling_y;
        d.hbd = bps == 2;
        d.nent = J.num_entries;
        d.ent_first = (int32_t)ed.size();
        for (int p = 0; p < J.num_planes; p++) {
            const int sx = p ? J.subsampling_x : 0, sy = p ? J.subsampling_y : 0;
            const long long ow = ((long long)J.width_in_tiles * J.tile_width) >> sx;
            const long long oh = ((long long)J.height_in_tiles * J.tile_height) >> sy;
            const av1g_plane& o = J.out[p];
            if (!o.data || o.width < ow || o.height < oh || o.stride < ow * bps) {
                err = who + ": output plane " + std::to_string(p) + " is missing or smaller than the output frame";
                return AV1G_EINVAL;
            }
            d.out[p] = (uint8_t*)o.data;
            d.out_stride[p] = o.stride;
        }
        for (int k = 0; k < J.num_entries; k++) {
            const av1g_tile_list_entry& e = J.entries[k];
            EntryDev x;
            memset(&x, 0, sizeof x);
            x.x0 = e.x0;
            x.y0 = e.y0;
            for (int p = 0; p < J.num_planes; p++) {
                const int sx = p ? J.subsampling_x : 0, sy = p ? J.subsampling_y : 0;
                const int tw = (J.tile_width + sx) >> sx, th = (J.tile_height + sy) >> sy;
                const av1g_plane& sp = e.src[p];
                if (e.x0 < 0 || e.y0 < 0 || !sp.data || (e.x0 >> sx) + tw > sp.width ||
                    (e.y0 >> sy) + th > sp.height || sp.stride < sp.width * bps) {
                    err = who + ": entry " + std::to_string(k) + " plane " + std::to_string(p) +
                          ": the tile lies outside its camera frame";
                    return AV1G_EINVAL;
                }
                x.src[p] = (const uint8_t*)sp.data;
                x.stride[p] = sp.stride;
            }
            ed.push_back(x);
        }
        starts[i] = (int32_t)total;
        total += (long long)J.width_in_tiles * J.height_in_tiles * J.num_planes;
    }
    starts[n] = (int32_t)total;
    const size_t off_ent = (sizeof(JobDev) * n + 255) & ~(size_t)255;
    const size_t off_st = (off_ent + sizeof(EntryDev) * ed.size() + 255) & ~(size_t)255;
    const size_t bytes = off_st + sizeof(int32_t) * (n + 1);
    uint8_t* buf = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&buf, bytes, s);
    if (e != cudaSuccess) {
        err = std::string("cudaMallocAsync: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    e = upload_with(buf, bytes, s, [&](uint8_t* h) {
        memcpy(h, jd.data(), sizeof(JobDev) * n);
        memcpy(h + off_ent, ed.data(), sizeof(EntryDev) * ed.size());
        memcpy(h + off_st, starts.data(), sizeof(int32_t) * (n + 1));
    });
    if (e == cudaSuccess) {
        const int grid = (int)(total < kSMs * 8 ? total : kSMs * 8);
        tile_list_kernel<<<grid, kThreads, 0, s>>>((const JobDev*)buf, (const EntryDev*)(buf + off_ent),
                                                   (const int32_t*)(buf + off_st), n, (int)total);
        e = cudaGetLastError();
    }
    cudaFreeAsync(buf, s);
    if (e != cudaSuccess) {
        err = std::string("tile list launch: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    return AV1G_OK;
}

}  // namespace av1g
