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
// reference does.  The split itself (fib_split) is also the standalone
// Section 4 entry point's, there reading the caller's literals exactly.

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

// The classifier as a table in shared memory: for modes 0-2 the class of
// every previous byte p1; for mode 3 four flags per byte (digit, identifier,
// whitespace, digit or '.' or '-') from which ContextClassifyOrder2 picks.
// Built by the block (lit_class itself is a chain of character tests).
struct ClassLut {
    uint8_t c[256];
};
__device__ __forceinline__ void class_lut_build(ClassLut& L, uint32_t mode, uint32_t tid, uint32_t nthr) {
    for (uint32_t b = tid; b < 256; b += nthr) {
        if (mode < 3) {
            L.c[b] = (uint8_t)lit_class(0, b, mode);
        } else {
            const uint32_t f = (lit_digit(b) ? 1u : 0u) | (lit_ident(b) ? 2u : 0u) | (lit_ws(b) ? 4u : 0u) |
                               ((lit_digit(b) || b == '.' || b == '-') ? 8u : 0u);
            L.c[b] = (uint8_t)f;
        }
    }
}
__device__ __forceinline__ uint32_t class_lut(const ClassLut& L, uint32_t p2, uint32_t p1, uint32_t mode) {
    if (mode < 3) return L.c[p1];
    const uint32_t f1 = L.c[p1], f2 = L.c[p2];
    if (f1 & 1u) return (f2 & 8u) ? 0u : 1u;
    if (f1 & 2u) return (f2 & 2u) ? 2u : 3u;
    return (f1 & 4u) ? 0u : 1u;
}

constexpr uint32_t kFibThreads = 512, kFibPer = 16, kFibTile = kFibThreads * kFibPer;

// Classes of the 16 literals [16 tid, 16 tid + 16) of the staged tile, 2
// bits each: one 16-byte shared load (conflict-free across the warp) and
// the word before it (the two previous literals in its top bytes).
__device__ __forceinline__ uint32_t fib_classes16(const uint8_t* s_tile, const ClassLut& L, uint32_t mode,
                                                  uint32_t tid, uint4& v) {
    v = reinterpret_cast<const uint4*>(s_tile + 16)[tid];
    const uint32_t prev = reinterpret_cast<const uint32_t*>(s_tile + 16)[4 * tid - 1];  // tid 0: s_tile[12..15]
    const uint32_t w[5] = {prev, v.x, v.y, v.z, v.w};
    uint32_t cls = 0;
    uint32_t p2 = (prev >> 16) & 0xFFu, p1 = prev >> 24;
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const uint32_t b = (w[1 + (q >> 2)] >> (8 * (q & 3))) & 0xFFu;
        cls |= class_lut(L, p2, p1, mode) << (2 * q);
        p2 = p1;
        p1 = b;
    }
    return cls;
}

// Tile [t0, t0 + tn) of the literals into s_tile[16 ..], one 16-byte load per
// thread, and the two literals before it into s_tile[14], s_tile[15] (0
// before the stream).  kExact: src is caller memory of any alignment, read
// without passing its end (byte loads where a 16-byte load would not be
// aligned or would pass tn); otherwise src is 16-byte aligned and padded, and
// bytes past tn are loaded but never classified.
template <bool kExact>
__device__ __forceinline__ void fib_load_tile(uint8_t* s_tile, const uint8_t* src, uint32_t t0, uint32_t tn,
                                              uint32_t tid) {
    const uint8_t* p = src + t0;
    if (tid * 16 < tn) {
        if (!kExact || (((reinterpret_cast<uintptr_t>(p) & 15u) == 0) && tid * 16 + 16 <= tn)) {
            reinterpret_cast<uint4*>(s_tile + 16)[tid] = reinterpret_cast<const uint4*>(p)[tid];
        } else {
            const uint32_t e = min(tid * 16 + 16, tn);
            for (uint32_t q = tid * 16; q < e; q++) s_tile[16 + q] = p[q];
        }
    }
    if (tid < 2) s_tile[14 + tid] = t0 + tid >= 2 ? src[t0 + tid - 2] : 0u;
}

struct FibShared {
    uint32_t warp[32];
    uint32_t cnt[4];
    uint32_t hist[4][256];
    __align__(16) uint8_t tile[kFibTile + 16];  // [14], [15]: the two literals before the tile
    __align__(16) uint8_t stage[kFibTile];
    ClassLut lut;
};

// DecomposeFibers (sheaf.go:110-137) of the n literals at src in foliation
// `mode`, by the whole block: fiber k goes to f + fo_k (fo_0 = 0, each start
// 16-byte aligned, fo_k + l_k <= n + 48), fl[0..3] receive the lengths and,
// with kHist, hist[256 k + b] the count of byte b in fiber k.  A counting
// pass gives the fiber lengths (hence where each fiber starts); then tiles of
// kFibTile literals: each thread classifies kFibPer consecutive literals, one
// block scan of the four packed counts gives every literal its place among
// the tile's literals of its fiber, the tile is partitioned in shared memory
// and copied out fiber by fiber (contiguous runs), so a tile costs one scan
// instead of one per thread-sized pass.
template <bool kExact, bool kHist>
__device__ void fib_split(const uint8_t* src, uint32_t n, uint32_t mode, uint8_t* f, uint32_t* fl, uint32_t* hist,
                          FibShared& sh) {
    const uint32_t tid = threadIdx.x;
    if (tid < 4) sh.cnt[tid] = 0;
    if (kHist)
        for (uint32_t i = tid; i < 4 * 256; i += kFibThreads) (&sh.hist[0][0])[i] = 0;
    class_lut_build(sh.lut, mode, tid, kFibThreads);
    uint32_t c4 = 0, c4hi = 0;  // counts of classes 0, 1 (16 bits each) and 2, 3, per thread
    for (uint32_t t0 = 0; t0 < n; t0 += kFibTile) {
        const uint32_t tn = min(kFibTile, n - t0);
        fib_load_tile<kExact>(sh.tile, src, t0, tn, tid);
        __syncthreads();
        const uint32_t q0 = min(tid * kFibPer, tn), q1 = min(q0 + kFibPer, tn);
        if (q0 < q1) {
            uint4 v;
            const uint32_t cls = fib_classes16(sh.tile, sh.lut, mode, tid, v);
            for (uint32_t q = q0; q < q1; q++) {
                const uint32_t k = (cls >> (2 * (q - q0))) & 3u;
                const uint32_t inc = 1u << (16 * (k & 1));
                c4 += k < 2 ? inc : 0u;
                c4hi += k < 2 ? 0u : inc;
            }
        }
        __syncthreads();
        if (((t0 / kFibTile) & 2047) == 2047) {  // flush before a 16-bit count can wrap (<= 16 per tile)
            atomicAdd(&sh.cnt[0], c4 & 0xFFFFu); atomicAdd(&sh.cnt[1], c4 >> 16);
            atomicAdd(&sh.cnt[2], c4hi & 0xFFFFu); atomicAdd(&sh.cnt[3], c4hi >> 16);
            c4 = c4hi = 0;
        }
    }
    atomicAdd(&sh.cnt[0], c4 & 0xFFFFu); atomicAdd(&sh.cnt[1], c4 >> 16);
    atomicAdd(&sh.cnt[2], c4hi & 0xFFFFu); atomicAdd(&sh.cnt[3], c4hi >> 16);
    __syncthreads();
    const uint32_t l0 = sh.cnt[0], l1 = sh.cnt[1], l2 = sh.cnt[2], l3 = sh.cnt[3];
    // fiber k starts at f + fo_k; c_k: its bytes written so far.  Per-fiber
    // values are selected, not indexed, so they stay in registers.
    const uint32_t fo1 = (l0 + 15) & ~15u, fo2 = fo1 + ((l1 + 15) & ~15u), fo3 = fo2 + ((l2 + 15) & ~15u);
    uint32_t c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    for (uint32_t t0 = 0; t0 < n; t0 += kFibTile) {
        const uint32_t tn = min(kFibTile, n - t0);
        fib_load_tile<kExact>(sh.tile, src, t0, tn, tid);
        __syncthreads();
        // this thread's literals [q0, q1) of the tile: classes and packed counts
        const uint32_t q0 = min(tid * kFibPer, tn), q1 = min(q0 + kFibPer, tn);
        uint32_t cls = 0, lo = 0, hi = 0;  // cls: 2 bits per literal; lo = n0 | n1 << 16, hi = n2 | n3 << 16
        uint4 v = make_uint4(0, 0, 0, 0);
        if (q0 < q1) cls = fib_classes16(sh.tile, sh.lut, mode, tid, v);
        for (uint32_t q = q0; q < q1; q++) {
            const uint32_t k = (cls >> (2 * (q - q0))) & 3u;
            const uint32_t inc = 1u << (16 * (k & 1));
            lo += k < 2 ? inc : 0u;
            hi += k < 2 ? 0u : inc;
        }
        uint32_t tlo, thi;
        const uint32_t elo = block_exclusive_scan<kFibThreads>(lo, sh.warp, tlo);
        const uint32_t ehi = block_exclusive_scan<kFibThreads>(hi, sh.warp, thi);
        const uint32_t n0 = tlo & 0xFFFFu, n1 = tlo >> 16, n2 = thi & 0xFFFFu, n3 = thi >> 16;
        const uint32_t b1 = n0, b2 = n0 + n1, b3 = n0 + n1 + n2;  // each fiber's run in the staged tile
        uint32_t p0 = elo & 0xFFFFu, p1 = b1 + (elo >> 16), p2 = b2 + (ehi & 0xFFFFu), p3 = b3 + (ehi >> 16);
        const uint32_t vw[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (uint32_t r = 0; r < 16; r++) {
            if (q0 + r >= q1) break;
            const uint32_t k = (cls >> (2 * r)) & 3u;
            const uint32_t v = (vw[r >> 2] >> (8 * (r & 3))) & 0xFFu;
            const uint32_t at = k == 0 ? p0 : k == 1 ? p1 : k == 2 ? p2 : p3;
            p0 += k == 0;
            p1 += k == 1;
            p2 += k == 2;
            p3 += k == 3;
            sh.stage[at] = (uint8_t)v;
            if (kHist) atomicAdd(&sh.hist[k][v], 1u);
        }
        __syncthreads();
        for (uint32_t i = tid; i < tn; i += kFibThreads) {
            // fiber of staged byte i, and where it goes
            const uint32_t o = i >= b3 ? fo3 + c3 + (i - b3)
                             : i >= b2 ? fo2 + c2 + (i - b2)
                             : i >= b1 ? fo1 + c1 + (i - b1)
                                       : c0 + i;
            f[o] = sh.stage[i];
        }
        c0 += n0;
        c1 += n1;
        c2 += n2;
        c3 += n3;
        __syncthreads();
    }
    if (kHist)
        for (uint32_t i = tid; i < 4 * 256; i += kFibThreads) hist[i] = (&sh.hist[0][0])[i];
    if (tid < 4) fl[tid] = tid == 0 ? l0 : tid == 1 ? l1 : tid == 2 ? l2 : l3;
}

// The foliations of frame j0 + blockIdx.x in mode blockIdx.y: fiber lengths,
// histograms and bytes into the frame's fiber region.  Frames whose literals
// are empty or above 8 MiB get empty fibers (no foliation is tried).
__global__ void __launch_bounds__(kFibThreads) k_frame_fibers(const Job* __restrict__ jobs, uint32_t j0,
                                                              const uint32_t* __restrict__ job_lens,
                                                              const uint8_t* __restrict__ streams,
                                                              uint8_t* __restrict__ fibbase) {
    __shared__ FibShared sh;
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
    // the literal stream is 16-byte aligned and padded past n (the stream
    // region is lit_cap >= n bytes, the streams buffer 64 more)
    const uint8_t* src = streams + job.str_off + stream_base(job, S_LIT);
    fib_split<false, true>(src, n, mode, fr + kFibAreaOff + mode * fib_mode_bytes(job), fl + 4 * mode,
                           reinterpret_cast<uint32_t*>(fr + kFibHistOff) + (uint64_t)(4 * mode) * 256, sh);
}

}  // namespace pz
