// tokenize.cu -- greedy LZ parse of the match table into PRZM opcodes, and
// per-frame gathering of the per-tile streams.
//
// Semantics of przm_fused_tokenizer_kernel (gpu/kernel/przm_tokenizer.cuh:
// 115-466): each 32 KiB tile is parsed independently; tile 0 starts with the
// repeat distances {1, 4, 8}, later tiles with none.  The parse is a serial
// walk (each decision fixes where the next one starts); one warp walks one
// tile, all 32 lanes holding the same walk state, and the long inner loops
// (run-length scan, forward match extension, literal copies) are spread over
// the lanes.  Besides the linear command stream the walk also writes its
// Mode 8 split (op / meta / var substreams, core/commands/commands.go:18-202),
// because every opcode it emits is complete within its tile.
#include "common.cuh"

namespace pz {

constexpr uint32_t kSlotStride = 4 * kSlotCmd + kSlotOff + kSlotLit;
__host__ __device__ inline uint32_t slot_base(int s) {
    switch (s) {
        case S_CMD: return 0;
        case S_OP: return kSlotCmd;
        case S_META: return 2 * kSlotCmd;
        case S_VAR: return 3 * kSlotCmd;
        case S_OFF: return 4 * kSlotCmd;
        default: return 4 * kSlotCmd + kSlotOff;
    }
}
__host__ __device__ inline uint32_t slot_cap(int s) { return s == S_OFF ? kSlotOff : (s == S_LIT ? kSlotLit : kSlotCmd); }

struct TokTile { uint32_t job; uint32_t tile; };

// Warp-uniform emitter for one tile: all lanes keep the same lengths, lane 0
// stores the bytes.
struct Emit {
    uint8_t* base;  // this tile's slot block
    uint32_t len[S_COUNT];
    bool ok;
    uint32_t lane;
    __device__ void put(int s, uint8_t b) {
        if (len[s] >= slot_cap(s)) { ok = false; return; }
        if (lane == 0) base[slot_base(s) + len[s]] = b;
        len[s]++;
    }
    __device__ void cmd_op(uint8_t b) { put(S_CMD, b); put(S_OP, b); }   // opcode byte
    __device__ void cmd_meta(uint8_t b) { put(S_CMD, b); put(S_META, b); }
    __device__ void cmd_varint(uint32_t v) {                              // przm_tokenizer.cuh:33-55
        while (v >= 0x80) { put(S_CMD, (uint8_t)(v | 0x80)); put(S_VAR, (uint8_t)(v | 0x80)); v >>= 7; }
        put(S_CMD, (uint8_t)v);
        put(S_VAR, (uint8_t)v);
    }
    __device__ void off_varint(uint32_t v) {
        while (v >= 0x80) { put(S_OFF, (uint8_t)(v | 0x80)); v >>= 7; }
        put(S_OFF, (uint8_t)v);
    }
    __device__ void lit_op(uint32_t count) {                              // przm_tokenizer.cuh:57-76
        if (count == 0) return;
        if (count <= 8) { cmd_op((uint8_t)(0xF2 + count)); return; }
        cmd_op(0xF0);
        cmd_varint(count);
    }
    // Literal bytes go to the literal slot in walk order.  Runs of up to 256
    // bytes are copied one token late: each lane loads its 8 bytes now (two
    // aligned words) and stores them at the next copy or at flush(), so the
    // loads overlap the next token's descriptor search.  Longer runs are
    // copied at once by the whole warp.  Source buffers are padded by 64
    // bytes, so the aligned word loads never leave the input buffer.
    uint32_t p_w0, p_w1, p_w2, p_sh, p_n;  // this lane's pending bytes: aligned words, byte shift, count
    uint8_t* p_dst;
    __device__ void flush() {
        if (p_n) {
            const uint32_t lo = p_sh ? __funnelshift_r(p_w0, p_w1, p_sh) : p_w0;
            const uint32_t hi = p_sh ? __funnelshift_r(p_w1, p_w2, p_sh) : p_w1;
            const uint64_t x = ((uint64_t)hi << 32) | lo;
            for (uint32_t i = 0; i < p_n; i++) p_dst[i] = (uint8_t)(x >> (8 * i));
        }
        p_n = 0;
    }
    __device__ void lits(const uint8_t* src, uint32_t count) {
        if (count == 0) return;
        if (len[S_LIT] + count > kSlotLit) { ok = false; return; }
        uint8_t* d = base + slot_base(S_LIT) + len[S_LIT];
        flush();
        if (count <= 256) {
            const uint32_t o = 8 * lane;
            if (o < count) {
                const uintptr_t a = reinterpret_cast<uintptr_t>(src + o);
                const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
                const uint32_t sh = (uint32_t)(a & 3) * 8;
                // the 8 bytes at src + o; nothing here waits for the loads
                p_w0 = __ldg(w);
                p_w1 = __ldg(w + 1);
                p_w2 = __ldg(w + 2);
                p_sh = sh;
                p_n = count - o < 8 ? count - o : 8;
                p_dst = d + o;
            }
        } else {
            for (uint32_t i = lane; i < count; i += 32) d[i] = src[i];
        }
        len[S_LIT] += count;
    }
};

// First index i in [from, lim) with src[i] != b (or lim), lanes in parallel.
__device__ uint32_t warp_run_end(const uint8_t* src, uint32_t from, uint32_t lim, uint8_t b, uint32_t lane) {
    const uint64_t rep = 0x0101010101010101ull * b;
    for (uint32_t base = from; base < lim; base += 256) {
        const uint32_t i = base + lane * 8;
        uint32_t first = 0xFFFFFFFFu;
        if (i < lim) {
            uint64_t x = ld64_global_u(src + i) ^ rep;
            if (x) first = i + ((uint32_t)(__ffsll((long long)x) - 1) >> 3);
        }
        uint32_t m = __ballot_sync(0xFFFFFFFFu, first != 0xFFFFFFFFu);
        if (m) {
            uint32_t f = __shfl_sync(0xFFFFFFFFu, first, __ffs(m) - 1);
            return f < lim ? f : lim;
        }
    }
    return lim;
}

// First k in [from, lim) with src[a+k] != src[b+k] (or lim), lanes in parallel.
__device__ uint32_t warp_match_end(const uint8_t* src, uint32_t a, uint32_t b, uint32_t from, uint32_t lim,
                                   uint32_t lane) {
    for (uint32_t base = from; base < lim; base += 256) {
        const uint32_t k = base + lane * 8;
        uint32_t first = 0xFFFFFFFFu;
        if (k < lim) {
            uint64_t x = ld64_global_u(src + a + k) ^ ld64_global_u(src + b + k);
            if (x) first = k + ((uint32_t)(__ffsll((long long)x) - 1) >> 3);
        }
        uint32_t m = __ballot_sync(0xFFFFFFFFu, first != 0xFFFFFFFFu);
        if (m) {
            uint32_t f = __shfl_sync(0xFFFFFFFFu, first, __ffs(m) - 1);
            return f < lim ? f : lim;
        }
    }
    return lim;
}

__global__ void __launch_bounds__(256) k_tokenize(const uint8_t* __restrict__ in, const Job* __restrict__ jobs,
                                                  const TokTile* __restrict__ tiles, uint32_t ntiles,
                                                  const uint32_t* __restrict__ desc, uint8_t* __restrict__ slots,
                                                  uint32_t* __restrict__ tile_lens, uint32_t* __restrict__ err) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t T = wid; T < ntiles; T += nw) {
        const TokTile tt = tiles[T];
        const Job job = jobs[tt.job];
        const uint8_t* src = in + job.in_off;
        const uint32_t* dj = desc + job.desc_off;
        const uint32_t start = tt.tile * kTile;
        const uint32_t end = min(start + kTile, job.n);
        const bool radix = job.kind != 0;
        const uint32_t ncand = job.n >= 8 ? (job.n - 8) / 8 + 1 : 0;
        const uint64_t S = (uint64_t)job.tile0 + tt.tile;  // slot of this tile
        Emit e;
        e.base = slots + S * kSlotStride;
        for (int s = 0; s < S_COUNT; s++) e.len[s] = 0;
        e.ok = true;
        e.lane = lane;
        e.p_n = 0;
        int rep0 = tt.tile == 0 ? 1 : -1, rep1 = tt.tile == 0 ? 4 : -1, rep2 = tt.tile == 0 ? 8 : -1;
        uint32_t pos = start, litStart = start;
        auto dsc = [&](uint32_t q) -> uint32_t {
            if (q >= end) return 0u;
            if (!radix) return dj[q];
            return ((q & 7) == 0 && (q >> 3) < ncand) ? dj[q >> 3] : 0u;
        };
        while (pos < end && e.ok) {
            // next position q >= pos holding a match descriptor (przm_tokenizer.cuh:170-194)
            // Each lane that sees a descriptor also loads the 4 source bytes
            // at its position, so the run-length test below needs no second
            // round trip to memory.
            uint32_t q = 0xFFFFFFFFu, qd = 0, qw = 0, nd = 0;
            if (!radix) {
                for (uint32_t w = pos; w < end; w += 32) {
                    uint32_t i = w + lane;
                    uint32_t v = i < end ? dj[i] : 0u;
                    const uint32_t sw = v ? ld32_global_u(src + i) : 0u;
                    uint32_t m = __ballot_sync(0xFFFFFFFFu, v != 0);
                    if (m) {
                        int l = __ffs(m) - 1;
                        q = w + l;
                        qd = __shfl_sync(0xFFFFFFFFu, v, l);
                        qw = __shfl_sync(0xFFFFFFFFu, sw, l);
                        nd = __shfl_sync(0xFFFFFFFFu, v, (l + 1) & 31);  // descriptor at q + 1
                        if (l == 31) nd = dsc(q + 1);
                        break;
                    }
                }
            } else {
                const uint32_t cend = min(ncand, (end + 7) >> 3);
                for (uint32_t c = (pos + 7) >> 3; c < cend; c += 32) {
                    uint32_t i = c + lane;
                    uint32_t v = i < cend ? dj[i] : 0u;
                    const uint32_t sw = v ? __ldg(reinterpret_cast<const uint32_t*>(src) + 2 * i) : 0u;
                    uint32_t m = __ballot_sync(0xFFFFFFFFu, v != 0);
                    if (m) {
                        int l = __ffs(m) - 1;
                        q = (c + l) * 8;
                        qd = __shfl_sync(0xFFFFFFFFu, v, l);
                        qw = __shfl_sync(0xFFFFFFFFu, sw, l);
                        break;
                    }
                }
                // nd stays 0: q + 1 is never 8-aligned, so it has no descriptor
            }
            if (q >= end) break;
            uint32_t mLen = qd >> 20;
            const uint32_t d = qd & 0xFFFFFu;
            // lookahead (:196-216)
            if (q + 1 < end && nd != 0 && (nd >> 20) > mLen + 1) { pos = q + 1; continue; }
            // run-length token (:218-286)
            if (q + 12 <= end) {
                const uint8_t b0 = (uint8_t)qw;
                if (qw == 0x01010101u * b0) {
                    const uint32_t lim = q + min(end - q, 65535u);
                    const uint32_t r = warp_run_end(src, q + 4, lim, b0, lane) - q;
                    if (r >= 12 && r >= mLen) {
                        if (q > litStart) e.lit_op(q - litStart);
                        e.cmd_op(0xF1);
                        e.cmd_varint(r);
                        e.lits(src + litStart, q + 1 - litStart);  // pending literals, then the run byte
                        pos = q + r;
                        litStart = pos;
                        continue;
                    }
                }
            }
            // match (:289-320).  The reference re-checks d <= q, mLen >= 4 and
            // the first 4 bytes here; every non-zero descriptor of both finders
            // (k_tile_find, k_rx_resolve) already satisfies them.  Both finders
            // also stop a match at its first mismatch unless it reached 4095
            // bytes or the end of the data, so the forward extension can only
            // continue a 4095-byte descriptor.
            if (q + mLen > end) mLen = end - q;
            if (mLen >= kMaxLen32) {
                const uint32_t lim = min(end - q, 65530u);
                if (mLen < lim && src[q + mLen] == src[q - d + mLen])
                    mLen = warp_match_end(src, q, q - d, mLen, lim, lane);
            }
            // encode (:328-427)
            int k = -1;
            if ((int)d == rep0 && rep0 > 0) k = 0;
            else if ((int)d == rep1 && rep1 > 0) k = 1;
            else if ((int)d == rep2 && rep2 > 0) k = 2;
            uint32_t litLen = q - litStart;
            const uint32_t litAll = litLen;
            const uint32_t keep = k >= 0 ? (mLen <= 7 ? 7u : 15u) : 3u;
            if (litLen > keep) {
                e.lit_op(litLen - keep);  // flushed literal op; its bytes go out with the rest below
                litLen = keep;
            }
            const uint32_t base = mLen - 4 > 14 ? 15u : mLen - 4;
            if (k >= 0 && mLen <= 7) {
                e.cmd_op((uint8_t)((litLen << 4) | ((mLen - 4) << 2) | (uint32_t)k));
            } else if (k >= 0) {
                e.cmd_op((uint8_t)(0xC0 | k));
                e.cmd_meta((uint8_t)((litLen << 4) | base));
                if (base == 15) e.cmd_varint(mLen - 19);
            } else {
                e.cmd_op((uint8_t)(0x80 | (litLen << 4) | base));
                if (base == 15) e.cmd_varint(mLen - 19);
            }
            e.lits(src + litStart, litAll);
            if (k < 0) {
                e.off_varint(d);
                rep2 = rep1; rep1 = rep0; rep0 = (int)d;
            } else if (k == 1) {
                rep1 = rep0; rep0 = (int)d;
            } else if (k == 2) {
                rep2 = rep1; rep1 = rep0; rep0 = (int)d;
            }
            pos = q + mLen;
            litStart = pos;
        }
        if (e.ok && litStart < end) {  // trailing literals (:440-464)
            e.lit_op(end - litStart);
            e.lits(src + litStart, end - litStart);
        }
        e.flush();
        if (lane == 0) {
            for (int s = 0; s < S_COUNT; s++) tile_lens[S * S_COUNT + s] = e.len[s];
            if (!e.ok) atomicOr(err, (uint32_t)E_SLOT_OVERFLOW);
        }
    }
}

// ---------------------------------------------------------------------------
// Gather: one CTA per frame concatenates its tiles' slots into the frame's
// contiguous streams (przm_tokenizer.cuh:474-609) and counts the byte
// histograms of the literal stream and of the three command substreams,
// privatised per warp in shared memory.
// ---------------------------------------------------------------------------
constexpr uint32_t kGatherThreads = 512;

__global__ void __launch_bounds__(kGatherThreads) k_gather(const Job* __restrict__ jobs, uint32_t njobs,
                                                          const uint8_t* __restrict__ slots,
                                                          const uint32_t* __restrict__ tile_lens,
                                                          uint8_t* __restrict__ streams, uint32_t* __restrict__ job_lens,
                                                          uint32_t* __restrict__ hist /* njobs x 4 x 256 */,
                                                          uint32_t* __restrict__ err) {
    extern __shared__ uint32_t smem_g[];
    uint32_t* s_off = smem_g;                      // (maxtiles + 1) per stream, filled per stream
    __shared__ uint32_t s_hist[4][4][256];         // [stream][warp group][symbol]
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t j = blockIdx.x; j < njobs; j += gridDim.x) {
        const Job job = jobs[j];
        uint8_t* sreg = streams + job.str_off;
        for (uint32_t i = tid; i < 4 * 4 * 256; i += kGatherThreads) (&s_hist[0][0][0])[i] = 0;
        for (int s = 0; s < S_COUNT; s++) {
            __syncthreads();
            // exclusive scan of this stream's tile lengths (<= 512 tiles)
            if (warp == 0) {
                uint32_t carry = 0;
                for (uint32_t b = 0; b < job.ntiles; b += 32) {
                    uint32_t i = b + lane;
                    uint32_t v = i < job.ntiles ? tile_lens[(uint64_t)(job.tile0 + i) * S_COUNT + s] : 0;
                    uint32_t x = v;
                    for (uint32_t o = 1; o < 32; o <<= 1) {
                        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                        if (lane >= o) x += y;
                    }
                    if (i < job.ntiles) s_off[i] = carry + x - v;
                    carry += __shfl_sync(0xFFFFFFFFu, x, 31);
                }
                if (lane == 0) s_off[job.ntiles] = carry;
            }
            __syncthreads();
            const uint32_t total = s_off[job.ntiles];
            const uint32_t cap = s == S_OFF ? job.off_cap : (s == S_LIT ? job.lit_cap : job.cmd_cap);
            if (total > cap) {
                if (tid == 0) atomicOr(err, (uint32_t)E_STREAM_OVERFLOW);
                continue;
            }
            uint8_t* dst = sreg + stream_base(job, s);
            const int hs = s == S_LIT ? 0 : (s == S_OP ? 1 : (s == S_META ? 2 : (s == S_VAR ? 3 : -1)));
            // one warp per tile, bytes in order
            for (uint32_t t = warp; t < job.ntiles; t += kGatherThreads / 32) {
                const uint32_t o = s_off[t], l = s_off[t + 1] - o;
                const uint8_t* sp = slots + (uint64_t)(job.tile0 + t) * kSlotStride + slot_base(s);
                for (uint32_t i = lane; i < l; i += 32) {
                    uint8_t b = sp[i];
                    dst[o + i] = b;
                    if (hs >= 0) atomicAdd(&s_hist[hs][warp & 3][b], 1u);
                }
            }
            if (tid == 0) job_lens[(uint64_t)j * S_COUNT + s] = total;
        }
        __syncthreads();
        for (uint32_t i = tid; i < 4 * 256; i += kGatherThreads) {
            uint32_t hs = i >> 8, sym = i & 255;
            hist[(uint64_t)j * 1024 + i] = s_hist[hs][0][sym] + s_hist[hs][1][sym] + s_hist[hs][2][sym] + s_hist[hs][3][sym];
        }
        __syncthreads();
    }
}

}  // namespace pz
