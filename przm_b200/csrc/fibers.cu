// fibers.cu -- Section 4 of the P3 frame inside the batch pipeline: the
// frame's literals split into the four fibers of each étale-sheaf foliation
// (DecomposeFibers, core/literals/sheaf.go:110-137, with the classifiers
// ContextClassify :39-88 and ContextClassifyOrder2 :91-107), for
// PackageLiteralsSection (core/literals/literals.go:664-693) as the
// reference's CPU compressor writes Section 4 (compress.go:957).
//
// k_frame_fibers: one block per (frame, foliation): a counting pass gives the
// four fiber lengths, a stable scatter (block scans of the class flags) writes
// each literal to its fiber and counts the fibers' histograms.  Every
// non-empty fiber is then one more adaptive task of the frame's rANS launch
// (its model normalised with the others), and k_plan compares the sizes of
// the raw literals, their adaptive container and the four foliations as the
// reference does.
#include "common.cuh"

namespace pz {

__device__ __forceinline__ bool lit_ws(uint32_t b) { return b == ' ' || b == '\t' || b == '\r' || b == '\n'; }
__device__ __forceinline__ bool lit_ident(uint32_t b) { return (b >= 'a' && b <= 'z') || b == '_'; }
__device__ __forceinline__ bool lit_digit(uint32_t b) { return b >= '0' && b <= '9'; }
__device__ __forceinline__ bool lit_syntax(uint32_t b) {
    switch (b) {
        case '{': case '}': case '[': case ']': case '(': case ')': case '<': case '>': case ':': case ';':
        case ',': case '.': case '"': case '\'': case '`': case '=': case '+': case '-': case '*': case '/':
        case '%': case '&': case '|': case '^': case '!': case '~': case '?': case '\\': case '#':
            return true;
        default:
            return false;
    }
}

// Fiber class of a literal after p2, p1 (sheaf.go:39-107).
__device__ __forceinline__ uint32_t lit_class(uint32_t p2, uint32_t p1, uint32_t mode) {
    switch (mode) {
        case 0: return lit_ws(p1) ? 0u : lit_syntax(p1) ? 1u : lit_ident(p1) ? 2u : 3u;
        case 1: return (p1 == '"' || p1 == ':') ? 0u : lit_ident(p1) ? 1u : lit_digit(p1) ? 2u : 3u;
        case 2: return (lit_ws(p1) || lit_syntax(p1)) ? 0u : 1u;
        default:
            if (lit_digit(p1)) return (lit_digit(p2) || p2 == '.' || p2 == '-') ? 0u : 1u;
            if (lit_ident(p1)) return lit_ident(p2) ? 2u : 3u;
            return lit_ws(p1) ? 0u : 1u;
    }
}

// DecomposeFibers of frame j0 + blockIdx.x in foliation blockIdx.y: fiber
// lengths, histograms and bytes into the frame's fiber region.  Frames whose
// literals are empty or above 8 MiB get empty fibers (no foliation is tried).
__global__ void __launch_bounds__(1024) k_frame_fibers(const Job* __restrict__ jobs, uint32_t j0,
                                                       const uint32_t* __restrict__ job_lens,
                                                       const uint8_t* __restrict__ streams, uint8_t* __restrict__ fibbase) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_cnt[4];
    __shared__ uint32_t s_hist[4][256];
    const uint32_t j = j0 + blockIdx.x, mode = blockIdx.y, tid = threadIdx.x;
    const Job job = jobs[j];
    if (job.profile < 3) return;
    const uint32_t n = job_lens[(uint64_t)j * S_COUNT + S_LIT];
    uint8_t* fr = fibbase + job.fib_off;
    uint32_t* fl = reinterpret_cast<uint32_t*>(fr);
    if (n == 0 || n > kFibMax) {
        if (tid < 4) fl[4 * mode + tid] = 0;
        return;
    }
    const uint8_t* src = streams + job.str_off + stream_base(job, S_LIT);
    if (tid < 4) s_cnt[tid] = 0;
    for (uint32_t i = tid; i < 4 * 256; i += blockDim.x) (&s_hist[0][0])[i] = 0;
    __syncthreads();
    uint32_t c4[4] = {0, 0, 0, 0};
    for (uint32_t i = tid; i < n; i += blockDim.x) {
        const uint32_t p1 = i ? src[i - 1] : 0u, p2 = i > 1 ? src[i - 2] : 0u;
        c4[lit_class(p2, p1, mode)]++;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) atomicAdd(&s_cnt[k], c4[k]);
    __syncthreads();
    const uint32_t l0 = s_cnt[0], l1 = s_cnt[1], l2 = s_cnt[2], l3 = s_cnt[3];
    uint8_t* f = fr + kFibAreaOff + mode * fib_mode_bytes(job);
    const uint32_t a0 = (l0 + 15) & ~15u, a1 = (l1 + 15) & ~15u, a2 = (l2 + 15) & ~15u;
    uint8_t* fb[4] = {f, f + a0, f + a0 + a1, f + a0 + a1 + a2};
    uint32_t carry[4] = {0, 0, 0, 0};
    for (uint32_t b0 = 0; b0 < n; b0 += 1024) {  // uniform trip count: every thread scans
        const uint32_t i = b0 + tid;
        uint32_t k = 4, v = 0;
        if (i < n) {
            v = src[i];
            k = lit_class(i > 1 ? src[i - 2] : 0u, i ? src[i - 1] : 0u, mode);
        }
        // places among this pass's literals of the same class: two scans of
        // two 16-bit counters each (at most 1024 per pass)
        const uint32_t a = (k == 0 ? 1u : 0u) | (k == 1 ? 1u << 16 : 0u);
        const uint32_t c = (k == 2 ? 1u : 0u) | (k == 3 ? 1u << 16 : 0u);
        uint32_t ta, tc;
        const uint32_t ea = block_exclusive_scan<1024>(a, s_warp, ta);
        const uint32_t ec = block_exclusive_scan<1024>(c, s_warp, tc);
        if (k < 4) {
            const uint32_t r = k == 0 ? (ea & 0xFFFFu) : k == 1 ? (ea >> 16) : k == 2 ? (ec & 0xFFFFu) : (ec >> 16);
            fb[k][carry[k] + r] = (uint8_t)v;
            atomicAdd(&s_hist[k][v], 1u);
        }
        carry[0] += ta & 0xFFFFu;
        carry[1] += ta >> 16;
        carry[2] += tc & 0xFFFFu;
        carry[3] += tc >> 16;
    }
    __syncthreads();
    uint32_t* gh = reinterpret_cast<uint32_t*>(fr + kFibHistOff) + (uint64_t)(4 * mode) * 256;
    for (uint32_t i = tid; i < 4 * 256; i += blockDim.x) gh[i] = (&s_hist[0][0])[i];
    if (tid < 4) fl[4 * mode + tid] = tid == 0 ? l0 : tid == 1 ? l1 : tid == 2 ? l2 : l3;
}

}  // namespace pz
