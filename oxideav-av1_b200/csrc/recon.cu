// recon.cu — §7.12.3 dequantization, §7.13.3 inverse transform and the
// §7.12.3 step-3 reconstruction merge.
//
// Replaces the reconstruct tail of transform_block_emit (src/cdf.rs:32874-
// 32910): dequantize_step1 (cdf.rs:13655-13703), inverse_transform_2d and its
// 1-D kernels (src/transform.rs:96-847), curr_frame_step3_merge
// (cdf.rs:17398-17470).  The reference runs these per TU, interleaved with
// parsing, on i64 vectors.  Here the TUs of a batch are bucketed on the host
// by (size, type); one CTA of 128 threads reconstructs 128 / max(w, h) TUs of
// one size: dequantized coefficients go to shared memory, one thread per row
// runs the row transform in registers (the butterfly network fully unrolled
// at compile time for the TU's length), one thread per column runs the column
// transform and adds the residual to the prediction already in CurrFrame.
//
// Arithmetic: values are held in int32 and every product is formed in 64 bits.
// This is exact: the reference's intermediates after each rounding or clamp
// fit 32 bits for 8-, 10- and 12-bit content (butterfly outputs are bounded by
// sqrt(2) times their clamped inputs; dequantized inputs by 2^(7+BitDepth)).
#include <algorithm>
#include <string>
#include <type_traits>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "itx.cuh"

namespace av1g {

namespace {

using namespace itx;

struct TuDev {
    av1g_tu tu;
    int32_t frame;
};

struct Task {
    int32_t first, count, tx_size, pad;
};

constexpr int kThreads = 128;

// Reconstructs `count` TUs of size TX (one slot of L = max(w, h) threads each).
template <int TX>
__device__ void recon_tus(const ReconFrame* frames, const TuDev* tus, const Task& task, int* smem) {
    constexpr int W = kTxW[TX], H = kTxH[TX], L = W > H ? W : H;
    const int slot = threadIdx.x / L, lane = threadIdx.x % L;
    const bool live = slot < task.count;
    const TuDev* td = tus + task.first + slot;
    const av1g_tu tu = live ? td->tu : av1g_tu{};
    recon_core<TX>(frames[live ? td->frame : 0], tu, live, lane, smem + slot * W * H);
}

__global__ void __launch_bounds__(kThreads) recon_kernel(const ReconFrame* __restrict__ frames,
                                                         const TuDev* __restrict__ tus,
                                                         const Task* __restrict__ tasks, int ntasks) {
    __shared__ int smem[8192];
    for (int b = blockIdx.x; b < ntasks; b += gridDim.x) {
        const Task task = tasks[b];
        __syncthreads();
        switch (task.tx_size) {
            case 0: recon_tus<0>(frames, tus, task, smem); break;
            case 1: recon_tus<1>(frames, tus, task, smem); break;
            case 2: recon_tus<2>(frames, tus, task, smem); break;
            case 3: recon_tus<3>(frames, tus, task, smem); break;
            case 4: recon_tus<4>(frames, tus, task, smem); break;
            case 5: recon_tus<5>(frames, tus, task, smem); break;
            case 6: recon_tus<6>(frames, tus, task, smem); break;
            case 7: recon_tus<7>(frames, tus, task, smem); break;
            case 8: recon_tus<8>(frames, tus, task, smem); break;
            case 9: recon_tus<9>(frames, tus, task, smem); break;
            case 10: recon_tus<10>(frames, tus, task, smem); break;
            case 11: recon_tus<11>(frames, tus, task, smem); break;
            case 12: recon_tus<12>(frames, tus, task, smem); break;
            case 13: recon_tus<13>(frames, tus, task, smem); break;
            case 14: recon_tus<14>(frames, tus, task, smem); break;
            case 15: recon_tus<15>(frames, tus, task, smem); break;
            case 16: recon_tus<16>(frames, tus, task, smem); break;
            case 17: recon_tus<17>(frames, tus, task, smem); break;
            default: recon_tus<18>(frames, tus, task, smem); break;
        }
    }
}

int slots_for(int tx) {
    int l = kTxW[tx] > kTxH[tx] ? kTxW[tx] : kTxH[tx];
    return kThreads / l;
}

}  // namespace

// Host side of av1g_run_recon: validation, bucketing, upload, launch.
av1g_status recon_run(const av1g_recon_job* jobs, int n, cudaStream_t s, std::string& err) {
    std::vector<ReconFrame> frames(n);
    size_t total = 0;
    for (int i = 0; i < n; i++) total += jobs[i].num_tus > 0 ? jobs[i].num_tus : 0;
    // TUs bucketed by (size, type) so the threads of a warp run one butterfly
    // network: a counting sort, stable in (job, decode order)
    constexpr int kKeys = 19 * 16;
    std::vector<uint32_t> count(kKeys + 1, 0);
    for (int i = 0; i < n; i++) {
        const av1g_recon_job& j = jobs[i];
        if (!j.hdr || !j.quant || (j.num_tus > 0 && (!j.tus || !j.coeffs)) || j.num_tus < 0) {
            err = "recon job " + std::to_string(i) + ": missing header, quantizer state, TU list or coefficients";
            return AV1G_EINVAL;
        }
        const av1g_frame_header& h = *j.hdr;
        if (h.bit_depth != 8 && h.bit_depth != 10 && h.bit_depth != 12) {
            err = "recon job " + std::to_string(i) + ": bit depth";
            return AV1G_EINVAL;
        }
        ReconFrame& F = frames[i];
        memset(&F, 0, sizeof F);
        F.bd = h.bit_depth;
        F.hbd = h.bit_depth > 8;
        F.q = *j.quant;
        F.coeffs = j.coeffs;
        for (int p = 0; p < h.num_planes; p++) {
            int sx = p ? h.subsampling_x : 0, sy = p ? h.subsampling_y : 0;
            int pw = (h.mi_cols * 4) >> sx, ph = (h.mi_rows * 4) >> sy;
            const av1g_plane& pl = j.planes[p];
            if (!pl.data || pl.width < pw || pl.height < ph || pl.stride < pw * (F.hbd ? 2 : 1) || (pl.stride & 15)) {
                err = "recon job " + std::to_string(i) + ": plane " + std::to_string(p);
                return AV1G_EINVAL;
            }
            F.planes[p] = PlaneDev{(uint8_t*)pl.data, pl.stride, pw, ph};
        }
        for (int k = 0; k < j.num_tus; k++) {
            const av1g_tu& t = j.tus[k];
            if (t.tx_size >= 19 || t.tx_type >= 16 || t.plane >= h.num_planes) {
                err = "recon job " + std::to_string(i) + ": TU " + std::to_string(k) + " has an invalid size/type/plane";
                return AV1G_EINVAL;
            }
            count[t.tx_size * 16 + t.tx_type + 1]++;
        }
    }
    if (total == 0) return AV1G_OK;
    for (int k = 1; k <= kKeys; k++) count[k] += count[k - 1];  // count[key]: TUs with a smaller key
    // tasks: runs of at most slots_for(tx) TUs of one size; keys are
    // size-major, so the TUs of size tx are [count[16 tx], count[16 tx + 16])
    std::vector<Task> tasks;
    for (int tx = 0; tx < 19; tx++) {
        const int first = (int)count[tx * 16], len = (int)(count[tx * 16 + 16] - count[tx * 16]);
        const int cap = slots_for(tx);
        for (int k = 0; k < len; k += cap) tasks.push_back(Task{first + k, len - k < cap ? len - k : cap, tx, 0});
    }
    size_t off_tus = (sizeof(ReconFrame) * n + 255) & ~(size_t)255;
    size_t off_tasks = (off_tus + sizeof(TuDev) * total + 255) & ~(size_t)255;
    size_t bytes = off_tasks + sizeof(Task) * tasks.size();
    uint8_t* dev = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dev, bytes, s);
    if (e != cudaSuccess) {
        err = std::string("cudaMallocAsync: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    // the TU records bucketed straight into the pinned staging block (a
    // counting sort, stable in (job, decode order))
    e = upload_with(dev, bytes, s, [&](uint8_t* host) {
        memcpy(host, frames.data(), sizeof(ReconFrame) * n);
        TuDev* dst = reinterpret_cast<TuDev*>(host + off_tus);
        for (int i = 0; i < n; i++)
            for (int k = 0; k < jobs[i].num_tus; k++) {
                const av1g_tu& t = jobs[i].tus[k];
                dst[count[t.tx_size * 16 + t.tx_type]++] = TuDev{t, i};
            }
        memcpy(host + off_tasks, tasks.data(), sizeof(Task) * tasks.size());
    });
    if (e == cudaSuccess) {
        int nt = (int)tasks.size();
        int grid = nt < kSMs * 16 ? nt : kSMs * 16;
        recon_kernel<<<grid, kThreads, 0, s>>>((const ReconFrame*)dev, (const TuDev*)(dev + off_tus),
                                               (const Task*)(dev + off_tasks), nt);
        e = cudaGetLastError();
    }
    cudaFreeAsync(dev, s);
    if (e != cudaSuccess) {
        err = std::string("recon launch: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    return AV1G_OK;
}

}  // namespace av1g
