// streams.cu -- kernels of the stand-alone stream APIs: byte histograms,
// flat packing, and histogram + normalise + V-ANS over many independent
// device streams.
#include "common.cuh"

namespace pz {

struct STask {
    uint64_t src;    // device address of the symbols
    uint64_t dst;    // device address of the output container
    uint64_t scr;    // device address of the lane scratch (ans_task_bytes(cap))
    uint32_t n;      // symbols
    uint32_t cap;    // lane layout capacity (>= n)
    uint32_t norm;   // 0 NormalizeFreq (Go), 1 NormalizeFrequencies, 2 table given by the caller
    uint32_t flags;  // container flag byte
};

// Byte histogram of a task, 64 KiB per block (blockIdx.x: the chunk), privatised per warp
// and merged with one global atomic per (block, symbol) -- the reference's
// przm_byte_histogram_kernel (przm_ans.cu:73-192) with warp-aggregated
// shared-memory increments (__match_any_sync groups equal bytes of a warp).
constexpr uint32_t kHistChunk = 65536;

__device__ __forceinline__ void stream_hist_task(const STask t, uint32_t ti, uint32_t (&s_h)[8][256],
                                                 uint32_t* __restrict__ counts) {
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (uint32_t i = tid; i < 8 * 256; i += 256) (&s_h[0][0])[i] = 0;
    __syncthreads();
    const uint64_t lo = (uint64_t)blockIdx.x * kHistChunk;
    if (lo < t.n) {
        const uint32_t len = (uint32_t)(t.n - lo < kHistChunk ? t.n - lo : kHistChunk);
        const uint8_t* p = reinterpret_cast<const uint8_t*>(t.src) + lo;
        const uintptr_t a = reinterpret_cast<uintptr_t>(p);
        const uint32_t head = min((uint32_t)((16 - (a & 15)) & 15), len);
        for (uint32_t i = tid; i < head; i += 256) atomicAdd(&s_h[warp][p[i]], 1u);
        const uint32_t nv = (len - head) / 16;
        const uint4* v4 = reinterpret_cast<const uint4*>(p + head);
        for (uint32_t v = tid; v < nv; v += 256) {
            const uint4 x = __ldg(v4 + v);
            const uint32_t w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const uint32_t b = (w[k >> 2] >> (8 * (k & 3))) & 0xFFu;
                const uint32_t peers = __match_any_sync(__activemask(), b);
                if ((__ffs(peers) - 1) == (int)lane) atomicAdd(&s_h[warp][b], (uint32_t)__popc(peers));
            }
        }
        for (uint32_t i = head + nv * 16 + tid; i < len; i += 256) atomicAdd(&s_h[warp][p[i]], 1u);
    }
    __syncthreads();
    uint32_t sum = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) sum += s_h[w][tid];
    if (sum) atomicAdd(&counts[(uint64_t)ti * 256 + tid], sum);
    __syncthreads();  // s_h is cleared for the next task
}

// Tasks blockIdx.y, blockIdx.y + gridDim.y, ... (grid y is at most 65535).
__global__ void __launch_bounds__(256) k_stream_hist(const STask* __restrict__ tasks, uint32_t ntasks,
                                                     uint32_t* __restrict__ counts) {
    __shared__ uint32_t s_h[8][256];
    for (uint32_t ti = blockIdx.y; ti < ntasks; ti += gridDim.y) stream_hist_task(tasks[ti], ti, s_h, counts);
}

// One warp per task: normalise and build the encoding table + matrix.
__global__ void k_stream_norm(const STask* __restrict__ tasks, uint32_t ntasks, const uint32_t* __restrict__ counts,
                              EncSym* __restrict__ tabs, TableInfo* __restrict__ infos) {
    __shared__ uint32_t s_cnt[256];
    __shared__ uint16_t s_freq[256];
    __shared__ GoRem s_rem[256];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t ti = blockIdx.x;
    if (ti >= ntasks) return;
    const STask t = tasks[ti];
    if (t.norm == 2 || t.n == 0) return;
    for (uint32_t s = lane; s < 256; s += 32) s_cnt[s] = counts[(uint64_t)ti * 256 + s];
    __syncwarp();
    if (t.norm == 0) warp_normalize_freq_go(s_cnt, s_freq, s_rem, lane);
    else warp_normalize_frequencies(s_cnt, s_freq, lane);
    warp_build_table(s_freq, tabs + (uint64_t)ti * 256, infos + ti, lane);
}

// One warp per 8 tasks (4 lanes each), tables and rings in shared memory.
__global__ void __launch_bounds__(kRansWarps * 32) k_stream_rans(const STask* __restrict__ tasks, uint32_t ntasks,
                                                                 const EncSym* __restrict__ tabs,
                                                                 TaskOut* __restrict__ outs) {
    extern __shared__ __align__(16) uint8_t smem_s[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t wg = blockIdx.x * kRansWarps + warp;
    EncSym* wtab = reinterpret_cast<EncSym*>(smem_s + warp * kRansTabBytes);
    uint4* wring = reinterpret_cast<uint4*>(smem_s + kRansWarps * kRansTabBytes + warp * kRingBytesPerWarp);
    for (uint32_t k = 0; k < 8; k++) {
        const uint32_t tk = wg * 8 + k;
        if (tk >= ntasks) break;
        for (uint32_t i = lane; i < 256; i += 32) wtab[k * 256 + i] = tabs[(uint64_t)tk * 256 + i];
    }
    __syncwarp();
    const uint32_t ti = wg * 8 + (lane >> 2), l = lane & 3;
    if (ti >= ntasks) return;
    const STask t = tasks[ti];
    if (t.n == 0) return;
    LaneIO io = lane_io(reinterpret_cast<uint8_t*>(t.scr), t.cap, l);
    rans_lane<false>(reinterpret_cast<const uint8_t*>(t.src), t.n, l, wtab + (lane >> 2) * 256, nullptr, wring, io,
                     &outs[ti].state[l], &outs[ti].count[l]);
}

constexpr int kStitchThreads = 256;

__global__ void __launch_bounds__(kStitchThreads) k_stream_stitch(const STask* __restrict__ tasks, uint32_t ntasks,
                                                                  const TableInfo* __restrict__ infos,
                                                                  const TaskOut* __restrict__ outs,
                                                                  uint32_t* __restrict__ out_lens) {
    const uint32_t ti = blockIdx.x;
    if (ti >= ntasks) return;
    const STask t = tasks[ti];
    if (t.n == 0) { if (threadIdx.x == 0) out_lens[ti] = 0; return; }
    uint8_t* dst = reinterpret_cast<uint8_t*>(t.dst);
    const TableInfo* info = infos + ti;
    const TaskOut o = outs[ti];
    const uint32_t h = 8 + info->mat_len;
    if (threadIdx.x == 0) {
        dst[0] = 'V'; dst[1] = 'A'; dst[2] = 0x01; dst[3] = (uint8_t)t.flags;
        for (int k = 0; k < 4; k++) dst[4 + k] = (uint8_t)(t.n >> (8 * k));
        for (int l = 0; l < 4; l++)
            for (int k = 0; k < 4; k++) dst[h + 4 * l + k] = (uint8_t)(o.state[l] >> (8 * k));
        out_lens[ti] = h + 16 + o.count[0] + o.count[1] + o.count[2] + o.count[3];
    }
    for (uint32_t i = threadIdx.x; i < info->mat_len; i += kStitchThreads) dst[8 + i] = info->mat[i];
    block_stitch<kStitchThreads>(reinterpret_cast<const uint8_t*>(t.scr), t.cap, t.n, dst + h + 16);
}

// PackStreamFlat (przm_ans.cu:202-234): 0x00 | LE32 n | payload.
__global__ void k_pack_flat(const uint8_t* __restrict__ in, uint32_t n, uint8_t* __restrict__ out) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, st = (uint64_t)gridDim.x * blockDim.x;
    if (g == 0) { out[0] = 0; out[1] = (uint8_t)n; out[2] = (uint8_t)(n >> 8); out[3] = (uint8_t)(n >> 16); out[4] = (uint8_t)(n >> 24); }
    for (uint64_t i = g; i < n; i += st) out[5 + i] = in[i];
}

// Copy kernel for the HBM bandwidth probe (16-byte vectors, grid-stride).
__global__ void k_copy_bw(const uint4* __restrict__ in, uint4* __restrict__ out, uint64_t n) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, st = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = g; i < n; i += st) out[i] = __ldg(in + i);
}

}  // namespace pz
