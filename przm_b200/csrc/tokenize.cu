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

// 16 unaligned bytes at p as two little-endian u64 (three aligned 8-byte
// loads; inputs are padded by 64 bytes, so reading up to 24 bytes past p is
// safe).
__device__ __forceinline__ void ld128_global_u(const uint8_t* p, uint64_t& lo, uint64_t& hi) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint64_t* w = reinterpret_cast<const uint64_t*>(a & ~uintptr_t(7));
    const uint32_t sh = (uint32_t)(a & 7) * 8;
    const uint64_t w0 = __ldg(w), w1 = __ldg(w + 1);
    if (!sh) { lo = w0; hi = w1; return; }
    const uint64_t w2 = __ldg(w + 2);
    lo = (w0 >> sh) | (w1 << (64 - sh));
    hi = (w1 >> sh) | (w2 << (64 - sh));
}

// Position of the first set byte of a 16-byte difference (lo, hi) from k,
// or 0xFFFFFFFF.
__device__ __forceinline__ uint32_t first_diff16(uint32_t k, uint64_t lo, uint64_t hi) {
    if (lo) return k + ((uint32_t)(__ffsll((long long)lo) - 1) >> 3);
    if (hi) return k + 8 + ((uint32_t)(__ffsll((long long)hi) - 1) >> 3);
    return 0xFFFFFFFFu;
}

// First index i in [from, lim) with src[i] != b (or lim), the warp comparing
// 16 bytes per lane, 512 per step.
__device__ uint32_t warp_run_end(const uint8_t* src, uint32_t from, uint32_t lim, uint8_t b, uint32_t lane) {
    const uint64_t rep = 0x0101010101010101ull * b;
    for (uint32_t base = from; base < lim; base += 512) {
        const uint32_t i = base + lane * 16;
        uint32_t first = 0xFFFFFFFFu;
        if (i < lim) {
            uint64_t lo, hi;
            ld128_global_u(src + i, lo, hi);
            first = first_diff16(i, lo ^ rep, hi ^ rep);
        }
        uint32_t m = __ballot_sync(0xFFFFFFFFu, first != 0xFFFFFFFFu);
        if (m) {
            uint32_t f = __shfl_sync(0xFFFFFFFFu, first, __ffs(m) - 1);
            return f < lim ? f : lim;
        }
    }
    return lim;
}

// First k in [from, lim) with src[a+k] != src[b+k] (or lim), the warp
// comparing 16 bytes per lane, 512 per step.
__device__ uint32_t warp_match_end(const uint8_t* src, uint32_t a, uint32_t b, uint32_t from, uint32_t lim,
                                   uint32_t lane) {
    for (uint32_t base = from; base < lim; base += 512) {
        const uint32_t k = base + lane * 16;
        uint32_t first = 0xFFFFFFFFu;
        if (k < lim) {
            uint64_t alo, ahi, blo, bhi;
            ld128_global_u(src + a + k, alo, ahi);
            ld128_global_u(src + b + k, blo, bhi);
            first = first_diff16(k, alo ^ blo, ahi ^ bhi);
        }
        uint32_t m = __ballot_sync(0xFFFFFFFFu, first != 0xFFFFFFFFu);
        if (m) {
            uint32_t f = __shfl_sync(0xFFFFFFFFu, first, __ffs(m) - 1);
            return f < lim ? f : lim;
        }
    }
    return lim;
}

// ---------------------------------------------------------------------------
// Tokenizer, in two phases per tile (one warp per 32 KiB tile).
//
// Walk.  The greedy parse is serial: each decision fixes where the next one
// starts.  It runs over a shared window of kTokWin match descriptors
// (radix frames: 8-aligned candidates; small frames: every position), with
// two shared bitmaps of the window -- non-zero descriptors, and positions
// whose 4 bytes are equal (the run-length test) -- and a register summary of
// the non-empty bitmap words.  Finding the next descriptor is a warp-uniform
// lookup in those; only run-length scans and the extension of 4095-byte
// matches read global memory.  Every decision
// becomes a record in shared memory (16 bytes, the fourth word unused):
//   r0 = q - tile start | literals before q << 16
//   r1 = match or run length | kind << 16 | repeat slot << 18
//   r2 = offset
// kinds: 0 explicit match, 1 repeat match, 2 run-length, 3 trailing literals.
// Emit.  Every kTokRec records (and at the end of the tile) the warp writes
// them out, 32 at a time: each lane turns one record into its bytes for the
// command, op, meta, var and offset streams (encodings of
// przm_tokenizer.cuh:57-76,329-426; Mode 8 split of commands.go:18-202),
// warp prefix sums give every lane its offsets, and the records' literal
// runs are copied by all lanes together.
// ---------------------------------------------------------------------------
constexpr uint32_t kTokWin = 1024;   // descriptor window entries
constexpr uint32_t kTokRec = 256;    // records buffered before emission
constexpr uint32_t kTokWarps = 4;    // warps (tiles) per block
constexpr uint32_t kLongLit = 128;   // literal runs copied 16 bytes per lane

struct TokSmem {
    uint32_t desc[kTokWin];
    uint32_t nz[kTokWin / 32];  // non-zero descriptors of the window, word per 32 entries
    uint32_t eq[kTokWin / 32];  // ... whose 4 bytes are equal
    uint4 rec[kTokRec];         // records (x, y, z; w unused): one 16-byte store each
};

__device__ __forceinline__ uint32_t vlen(uint32_t v) { return v < 0x80u ? 1u : v < 0x4000u ? 2u : v < 0x200000u ? 3u : v < 0x10000000u ? 4u : 5u; }

__device__ __forceinline__ uint32_t put_varint(uint8_t* d, uint32_t v) {  // przm_tokenizer.cuh:33-55
    uint32_t k = 0;
    while (v >= 0x80u) { d[k++] = (uint8_t)(v | 0x80u); v >>= 7; }
    d[k++] = (uint8_t)v;
    return k;
}

// Inclusive warp prefix sum.
__device__ __forceinline__ uint32_t warp_incl(uint32_t v, uint32_t lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= (uint32_t)o) v += y;
    }
    return v;
}

struct TokTileOut {
    uint8_t* base;          // the tile's slot block
    uint32_t len[S_COUNT];  // bytes written per stream (warp-uniform)
    bool ok;
};

__device__ __forceinline__ void hist4(uint32_t* h, uint32_t w) {
    atomicAdd(&h[w & 0xFFu], 1u);
    atomicAdd(&h[(w >> 8) & 0xFFu], 1u);
    atomicAdd(&h[(w >> 16) & 0xFFu], 1u);
    atomicAdd(&h[w >> 24], 1u);
}

// 16 source bytes at sw + 4v, shifted right by sh bits (sh = 8 x the
// source's offset from its 4-byte boundary); ld_stage<kC> loads (see there).
template <bool kC>
__device__ __forceinline__ uint4 ld16_shifted(const uint32_t* sw, uint32_t v, uint32_t sh) {
    const uint32_t* q = sw + 4 * v;
    const uint32_t w0 = ld_stage<kC>(q), w1 = ld_stage<kC>(q + 1), w2 = ld_stage<kC>(q + 2), w3 = ld_stage<kC>(q + 3);
    if (sh == 0) return make_uint4(w0, w1, w2, w3);
    const uint32_t w4 = ld_stage<kC>(q + 4);
    return make_uint4(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh), __funnelshift_r(w2, w3, sh),
                      __funnelshift_r(w3, w4, sh));
}

// Copies n bytes s -> d with the warp and counts them into h (shared, may be
// null): bytes up to d's first 16-byte boundary, then aligned 16-byte stores,
// four per lane in flight (source words loaded aligned and funnel-shifted, so
// reading up to 3 bytes past s + n: slot blocks and inputs have room), then
// the tail bytes.
template <bool kC>
__device__ void warp_copy_hist(uint8_t* __restrict__ d, const uint8_t* s, uint32_t n, uint32_t* __restrict__ h,
                               uint32_t lane) {
    const uint32_t head = min(n, (uint32_t)((16 - (reinterpret_cast<uintptr_t>(d) & 15)) & 15));
    if (lane < head) {
        const uint8_t b = ld_stage<kC>(s + lane);
        d[lane] = b;
        if (h) atomicAdd(&h[b], 1u);
    }
    d += head;
    s += head;
    n -= head;
    const uint32_t nv = n / 16;
    const uint32_t sh = 8 * (uint32_t)(reinterpret_cast<uintptr_t>(s) & 3);
    const uint32_t* sw = reinterpret_cast<const uint32_t*>(reinterpret_cast<uintptr_t>(s) & ~uintptr_t(3));
    uint4* d4 = reinterpret_cast<uint4*>(d);
    uint32_t v = lane;
    for (; v + 96 < nv; v += 128) {
        uint4 o[4];
#pragma unroll
        for (int u = 0; u < 4; u++) o[u] = ld16_shifted<kC>(sw, v + 32 * u, sh);
#pragma unroll
        for (int u = 0; u < 4; u++) {
            d4[v + 32 * u] = o[u];
            if (h) { hist4(h, o[u].x); hist4(h, o[u].y); hist4(h, o[u].z); hist4(h, o[u].w); }
        }
    }
    for (; v < nv; v += 32) {
        const uint4 o = ld16_shifted<kC>(sw, v, sh);
        d4[v] = o;
        if (h) { hist4(h, o.x); hist4(h, o.y); hist4(h, o.z); hist4(h, o.w); }
    }
    for (uint32_t i = 16 * nv + lane; i < n; i += 32) {
        const uint8_t b = ld_stage<kC>(s + i);
        d[i] = b;
        if (h) atomicAdd(&h[b], 1u);
    }
}

// Writes records [0, nrec) of the warp's buffer.
__device__ void tok_emit(const uint4* rec, uint32_t nrec, const uint8_t* tile_src, TokTileOut& o, uint32_t lane) {
    for (uint32_t g = 0; g < nrec; g += 32) {
        const uint32_t i = g + lane;
        const bool v = i < nrec;
        uint32_t r0 = 0, r1 = 0, r2 = 0;
        if (v) { const uint4 x = rec[i]; r0 = x.x; r1 = x.y; r2 = x.z; }
        const uint32_t q = r0 & 0xFFFFu, lit = r0 >> 16, len = r1 & 0xFFFFu, kind = (r1 >> 16) & 3u, k = r1 >> 18;
        // literal-op count, op byte and the rest, per record kind
        uint32_t flush = 0, litLen = 0, base = 0;
        if (kind <= 1) {
            const uint32_t keep = kind == 1 ? (len <= 7 ? 7u : 15u) : 3u;
            flush = lit > keep ? lit - keep : 0u;
            litLen = lit - flush;
            base = len - 4 > 14 ? 15u : len - 4;
        } else {
            flush = lit;
        }
        const uint32_t lop = flush == 0 ? 0u : (flush <= 8 ? 1u : 1u + vlen(flush));  // literal-op bytes
        const uint32_t lvar = flush > 8 ? vlen(flush) : 0u;
        const bool rep_long = kind == 1 && len > 7;
        const bool tail_var = (kind == 0 || rep_long) && base == 15;
        uint32_t c[S_COUNT] = {0, 0, 0, 0, 0, 0};
        if (v) {
            c[S_OP] = (flush ? 1u : 0u) + (kind <= 2 ? 1u : 0u);
            c[S_META] = rep_long ? 1u : 0u;
            c[S_VAR] = lvar + (tail_var ? vlen(len - 19) : 0u) + (kind == 2 ? vlen(len) : 0u);
            c[S_CMD] = lop + (kind <= 2 ? 1u : 0u) + c[S_META] + (c[S_VAR] - lvar);
            c[S_OFF] = kind == 0 ? vlen(r2) : 0u;
            c[S_LIT] = lit + (kind == 2 ? 1u : 0u);
        }
        uint32_t off[S_COUNT], tot[S_COUNT];
#pragma unroll
        for (int s = 0; s < S_COUNT; s++) {
            const uint32_t inc = warp_incl(c[s], lane);
            tot[s] = __shfl_sync(0xFFFFFFFFu, inc, 31);
            off[s] = o.len[s] + inc - c[s];
        }
        bool fits = o.ok;
#pragma unroll
        for (int s = 0; s < S_COUNT; s++) fits = fits && o.len[s] + tot[s] <= slot_cap(s);
        if (!fits) {
            o.ok = false;
            return;
        }
        if (v) {
            uint8_t* cmd = o.base + slot_base(S_CMD) + off[S_CMD];
            uint8_t* op = o.base + slot_base(S_OP) + off[S_OP];
            uint8_t* var = o.base + slot_base(S_VAR) + off[S_VAR];
            if (flush) {
                const uint8_t b = flush <= 8 ? (uint8_t)(0xF2u + flush) : (uint8_t)0xF0u;
                *cmd++ = b;
                *op++ = b;
                if (flush > 8) {
                    const uint32_t n = put_varint(cmd, flush);
                    put_varint(var, flush);
                    cmd += n;
                    var += n;
                }
            }
            if (kind == 2) {
                *cmd++ = 0xF1u;
                *op = 0xF1u;
                put_varint(cmd, len);
                put_varint(var, len);
            } else if (kind == 1 && len <= 7) {
                const uint8_t b = (uint8_t)((litLen << 4) | ((len - 4) << 2) | k);
                *cmd = b;
                *op = b;
            } else if (kind <= 1) {
                const uint8_t b = kind == 1 ? (uint8_t)(0xC0u | k) : (uint8_t)(0x80u | (litLen << 4) | base);
                *cmd++ = b;
                *op = b;
                if (kind == 1) {
                    const uint8_t t = (uint8_t)((litLen << 4) | base);
                    *cmd++ = t;
                    o.base[slot_base(S_META) + off[S_META]] = t;
                }
                if (base == 15) {
                    put_varint(cmd, len - 19);
                    put_varint(var, len - 19);
                }
                if (kind == 0) put_varint(o.base + slot_base(S_OFF) + off[S_OFF], r2);
            }
        }
        // literal runs of these records: runs of kLongLit bytes or more one at a
        // time with the warp's 16-byte copy, the shorter ones all lanes over
        // their concatenated bytes, four bytes per lane in flight
        {
            const uint32_t cl = c[S_LIT];
            const bool lng = cl >= kLongLit;
            const uint32_t cs = lng ? 0u : cl;
            const uint32_t incl = warp_incl(cs, lane), ts = __shfl_sync(0xFFFFFFFFu, incl, 31);
            const uint32_t from = q - lit;                     // first literal of this record, tile-relative
            const uint32_t dx = off[S_LIT] - o.len[S_LIT];     // its place in this group's literal bytes
            uint8_t* dl = o.base + slot_base(S_LIT) + o.len[S_LIT];
            for (uint32_t b0 = 0; b0 < ts; b0 += 128) {  // warp-uniform trip count: every lane shuffles
                uint32_t si[4], di[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const uint32_t b = b0 + 32 * u + lane;
                    // record j with incl[j-1] <= b < incl[j]
                    uint32_t j = 0;
#pragma unroll
                    for (int st = 16; st >= 1; st >>= 1) {
                        const uint32_t x = __shfl_sync(0xFFFFFFFFu, incl, j + st - 1);
                        if (x <= b) j += st;
                    }
                    const uint32_t ex = __shfl_sync(0xFFFFFFFFu, incl, j ? j - 1 : 0);
                    const uint32_t f = __shfl_sync(0xFFFFFFFFu, from, j & 31);
                    const uint32_t dj = __shfl_sync(0xFFFFFFFFu, dx, j & 31);
                    const uint32_t k = b - (j ? ex : 0u);
                    si[u] = f + k;
                    di[u] = dj + k;
                }
                uint8_t vb[4];
#pragma unroll
                for (int u = 0; u < 4; u++) vb[u] = b0 + 32 * u + lane < ts ? tile_src[si[u]] : 0;
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (b0 + 32 * u + lane < ts) dl[di[u]] = vb[u];
            }
            uint32_t lm = __ballot_sync(0xFFFFFFFFu, lng);
            while (lm) {
                const uint32_t j = __ffs(lm) - 1;
                lm &= lm - 1;
                warp_copy_hist<false>(dl + __shfl_sync(0xFFFFFFFFu, dx, j), tile_src + __shfl_sync(0xFFFFFFFFu, from, j),
                               __shfl_sync(0xFFFFFFFFu, cl, j), nullptr, lane);
            }
        }
#pragma unroll
        for (int s = 0; s < S_COUNT; s++) o.len[s] += tot[s];
    }
}

// One 32 KiB tile, by one warp with its TokSmem.
template <bool kC>
__device__ void tokenize_tile(const uint8_t* __restrict__ in, const Job* __restrict__ jobs, const TokTile tt,
                              const uint32_t* desc, uint8_t* __restrict__ slots,
                              uint32_t* __restrict__ tile_lens, uint32_t* __restrict__ err, TokSmem& sm) {
    const uint32_t lane = threadIdx.x & 31;
    {
        const Job job = jobs[tt.job];
        const uint8_t* src = in + job.in_off;
        const uint32_t* dj = desc + job.desc_off;
        const uint32_t start = tt.tile * kTile;
        const uint32_t end = min(start + kTile, job.n);
        const bool radix = job.kind != 0;
        const uint32_t ncand = job.n >= 8 ? (job.n - 8) / 8 + 1 : 0;
        // descriptor index space of this tile ends at e_hi
        const uint32_t e_hi = radix ? min(ncand, (end + 7) >> 3) : end;
        const uint64_t S = (uint64_t)job.tile0 + tt.tile;
        TokTileOut o;
        o.base = slots + S * kSlotStride;
        for (int s = 0; s < S_COUNT; s++) o.len[s] = 0;
        o.ok = true;
        int rep0 = tt.tile == 0 ? 1 : -1, rep1 = tt.tile == 0 ? 4 : -1, rep2 = tt.tile == 0 ? 8 : -1;
        uint32_t pos = start, litStart = start, nrec = 0;
        uint32_t wb = 0xFFFFFFFFu, wsum = 0;  // window base entry; bit k: word k of the window has a descriptor
        auto refill = [&](uint32_t base) {
            // entries [base, base + kTokWin): descriptors to shared memory, one
            // bitmap word per lane.  Every load instruction of the warp reads
            // 512 contiguous bytes; the bitmaps are put together from ballots.
            __syncwarp();
            wb = base;
            // descriptors: round i, lane t holds entries 128 i + 4 t .. + 3, so
            // bit 4u + b of word k is component b of lane 8 (k & 3) + u in
            // round k >> 2
            uint32_t cap0 = 0, cap1 = 0, cap2 = 0, cap3 = 0;
#pragma unroll
            for (uint32_t h = 0; h < 8; h += 4) {
                uint4 v[4];
#pragma unroll
                for (uint32_t u = 0; u < 4; u++) {
                    const uint32_t e = base + 128 * (h + u) + 4 * lane;
                    v[u] = make_uint4(0u, 0u, 0u, 0u);
                    if (e < e_hi) {  // dj + e is 16-byte aligned; the array holds whole uint4s below e_hi
                        v[u] = ld_stage<kC>(reinterpret_cast<const uint4*>(dj + e));
                        if (e + 1 >= e_hi) v[u].y = 0;
                        if (e + 2 >= e_hi) v[u].z = 0;
                        if (e + 3 >= e_hi) v[u].w = 0;
                    }
                }
#pragma unroll
                for (uint32_t u = 0; u < 4; u++) {
                    *reinterpret_cast<uint4*>(&sm.desc[128 * (h + u) + 4 * lane]) = v[u];
                    const uint32_t b0 = __ballot_sync(0xFFFFFFFFu, v[u].x != 0), b1 = __ballot_sync(0xFFFFFFFFu, v[u].y != 0);
                    const uint32_t b2 = __ballot_sync(0xFFFFFFFFu, v[u].z != 0), b3 = __ballot_sync(0xFFFFFFFFu, v[u].w != 0);
                    if ((lane >> 2) == h + u) { cap0 = b0; cap1 = b1; cap2 = b2; cap3 = b3; }
                }
            }
            const uint32_t s8 = 8 * (lane & 3);
            const uint32_t nz = spread8_4(cap0 >> s8) | (spread8_4(cap1 >> s8) << 1) | (spread8_4(cap2 >> s8) << 2) |
                                (spread8_4(cap3 >> s8) << 3);
            wsum = __ballot_sync(0xFFFFFFFFu, nz != 0);
            uint32_t eq = 0;
            if (radix) {
                // candidate base + r starts at byte 8 (base + r); uint4 u = 32 i + t
                // covers candidates 2u and 2u + 1, so bits 2v and 2v + 1 of word k
                // are lane 16 (k & 1) + v of round k >> 1 (rounds whose two words
                // hold no descriptor are skipped)
                const uint4* s4 = reinterpret_cast<const uint4*>(src + 8ull * base);
                uint32_t capa = 0, capb = 0;
#pragma unroll 4
                for (uint32_t i = 0; i < 16; i++) {
                    if (((wsum >> (2 * i)) & 3u) == 0) continue;
                    const uint32_t u = 32 * i + lane;
                    bool ea = false, eb = false;
                    if (base + 2 * u < e_hi) {  // bytes below 8 e_hi + 8 <= n + 8
                        const uint4 v = __ldg(s4 + u);
                        ea = v.x == 0x01010101u * (v.x & 0xFFu);
                        eb = v.z == 0x01010101u * (v.z & 0xFFu);
                    }
                    const uint32_t ba = __ballot_sync(0xFFFFFFFFu, ea), bb = __ballot_sync(0xFFFFFFFFu, eb);
                    if ((lane >> 1) == i) { capa = ba; capb = bb; }
                }
                const uint32_t s16 = 16 * (lane & 1);
                eq = spread16((capa >> s16) & 0xFFFFu) | (spread16((capb >> s16) & 0xFFFFu) << 1);
            } else if (nz) {
                // positions base + 32 lane .. + 31 (32-aligned, inputs are 16-aligned
                // and padded by 64 bytes past n)
                const uint4* s4 = reinterpret_cast<const uint4*>(src + base + 32 * lane);
                const uint4 a = __ldg(s4), b = __ldg(s4 + 1), c = __ldg(s4 + 2);
                const uint32_t w[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
#pragma unroll
                for (uint32_t k = 0; k < 32; k++) {
                    const uint32_t x = (k & 3) ? __funnelshift_r(w[k >> 2], w[(k >> 2) + 1], 8 * (k & 3)) : w[k >> 2];
                    eq |= (x == 0x01010101u * (x & 0xFFu) ? 1u : 0u) << k;
                }
            }
            sm.nz[lane] = nz;
            sm.eq[lane] = eq & nz;
            __syncwarp();
        };
        while (pos < end && o.ok) {
            const uint32_t e0 = radix ? (pos + 7) >> 3 : pos;
            if (e0 >= e_hi) break;
            if (wb == 0xFFFFFFFFu || e0 >= wb + kTokWin || e0 < wb) refill(e0 & ~31u);
            // next descriptor at or after e0: the rest of e0's word, else the
            // first non-empty word after it (warp-uniform, no shuffles)
            const uint32_t rel = e0 - wb;
            uint32_t l = rel >> 5;
            uint32_t wl = sm.nz[l] & (0xFFFFFFFFu << (rel & 31));
            if (!wl) {
                const uint32_t rest = l < 31 ? wsum & (0xFFFFFFFEu << l) : 0u;
                if (!rest) {  // nothing more in this window: continue after it
                    const uint32_t nb = wb + kTokWin;
                    if (nb >= e_hi) break;
                    pos = radix ? max(pos, 8 * nb) : max(pos, nb);
                    continue;
                }
                l = __ffs(rest) - 1;
                wl = sm.nz[l];
            }
            const uint32_t eql = sm.eq[l];
            const uint32_t bit = __ffs(wl) - 1;
            const uint32_t ent = wb + 32 * l + bit;
            const uint32_t q = radix ? 8 * ent : ent;
            if (q >= end) break;
            const uint32_t qd = sm.desc[ent - wb];
            uint32_t mLen = qd >> 20;
            const uint32_t d = qd & 0xFFFFFu;
            // lookahead (przm_tokenizer.cuh:196-216): radix frames have no
            // descriptor at q + 1
            if (!radix && q + 1 < end) {
                const uint32_t nd = ent + 1 - wb < kTokWin ? sm.desc[ent + 1 - wb] : ld_stage<kC>(dj + ent + 1);
                if (nd != 0 && (nd >> 20) > mLen + 1) { pos = q + 1; continue; }
            }
            // run-length token (:218-286)
            if (q + 12 <= end && ((eql >> bit) & 1u)) {
                const uint8_t b0 = src[q];
                const uint32_t lim = q + min(end - q, 65535u);
                const uint32_t r = warp_run_end(src, q + 4, lim, b0, lane) - q;
                if (r >= 12 && r >= mLen) {
                    if (lane == 0) sm.rec[nrec] = make_uint4((q - start) | ((q - litStart) << 16), r | (2u << 16), 0u, 0u);
                    nrec++;
                    pos = q + r;
                    litStart = pos;
                    if (nrec == kTokRec) { __syncwarp(); tok_emit(sm.rec, nrec, src + start, o, lane); nrec = 0; __syncwarp(); }
                    continue;
                }
            }
            // match (:289-320).  The reference re-checks d <= q, mLen >= 4 and
            // the first 4 bytes here; every non-zero descriptor of both finders
            // (k_tile_find, k_rx_verify) already satisfies them.  Both finders
            // also stop a match at its first mismatch unless it reached 4095
            // bytes or the end of the data, so the forward extension can only
            // continue a 4095-byte descriptor.
            if (q + mLen > end) mLen = end - q;
            if (mLen >= kMaxLen32) {
                const uint32_t lim = min(end - q, 65530u);
                if (mLen < lim && src[q + mLen] == src[q - d + mLen])
                    mLen = warp_match_end(src, q, q - d, mLen, lim, lane);
            }
            int k = -1;
            if ((int)d == rep0 && rep0 > 0) k = 0;
            else if ((int)d == rep1 && rep1 > 0) k = 1;
            else if ((int)d == rep2 && rep2 > 0) k = 2;
            if (lane == 0)
                sm.rec[nrec] = make_uint4((q - start) | ((q - litStart) << 16),
                                          mLen | ((k >= 0 ? 1u : 0u) << 16) | ((uint32_t)(k >= 0 ? k : 0) << 18), d, 0u);
            nrec++;
            if (k < 0) {
                rep2 = rep1; rep1 = rep0; rep0 = (int)d;
            } else if (k == 1) {
                rep1 = rep0; rep0 = (int)d;
            } else if (k == 2) {
                rep2 = rep1; rep1 = rep0; rep0 = (int)d;
            }
            pos = q + mLen;
            litStart = pos;
            if (nrec == kTokRec) { __syncwarp(); tok_emit(sm.rec, nrec, src + start, o, lane); nrec = 0; __syncwarp(); }
        }
        if (o.ok && litStart < end) {  // trailing literals (:440-464)
            if (lane == 0) sm.rec[nrec] = make_uint4((end - start) | ((end - litStart) << 16), 3u << 16, 0u, 0u);
            nrec++;
        }
        __syncwarp();
        if (o.ok && nrec) tok_emit(sm.rec, nrec, src + start, o, lane);
        __syncwarp();
        if (lane == 0) {
            for (int s = 0; s < S_COUNT; s++) tile_lens[S * S_COUNT + s] = o.len[s];
            if (!o.ok) atomicOr(err, (uint32_t)E_SLOT_OVERFLOW);
        }
    }
}

__global__ void __launch_bounds__(kTokWarps * 32) k_tokenize(const uint8_t* __restrict__ in, const Job* __restrict__ jobs,
                                                            const TokTile* __restrict__ tiles, uint32_t ntiles,
                                                            const uint32_t* __restrict__ order,
                                                            const uint32_t* __restrict__ desc, uint8_t* __restrict__ slots,
                                                            uint32_t* __restrict__ tile_lens, uint32_t* __restrict__ err) {
    __shared__ TokSmem s_tok[kTokWarps];
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t wid = blockIdx.x * kTokWarps + warp;
    const uint32_t nw = gridDim.x * kTokWarps;
    for (uint32_t T = wid; T < ntiles; T += nw) tokenize_tile<false>(in, jobs, tiles[order[T]], desc, slots, tile_lens, err, s_tok[warp]);
}

// ---------------------------------------------------------------------------
// Tokenizer schedule.  A tile's walk costs about one step per match it takes,
// and tiles of one batch differ by 10x or more (a tile of short repeats
// against one of long copies or of no matches at all); walked in list order,
// heavy tiles that start late would set the kernel's length.  So the tiles
// are walked heaviest first: the weight of a tile is its number of non-zero
// match descriptors, and the order buckets tiles by the bit length of that
// weight.  The order changes no output byte (every tile is parsed alone).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_tile_weight(const Job* __restrict__ jobs, const TokTile* __restrict__ tiles,
                                                     uint32_t ntiles, const uint32_t* __restrict__ desc,
                                                     uint32_t* __restrict__ weight) {
    __shared__ uint32_t s_w[8];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t T = blockIdx.x; T < ntiles; T += gridDim.x) {
        const TokTile tt = tiles[T];
        const Job job = jobs[tt.job];
        const uint32_t start = tt.tile * kTile, end = min(start + kTile, job.n);
        const uint32_t ncand = job.n >= 8 ? (job.n - 8) / 8 + 1 : 0;
        // the tile's descriptor entries [e_lo, e_hi), as the walk indexes them;
        // e_lo is a multiple of 4, so the uint4 loads are aligned, and whole
        // uint4s below e_hi lie inside the frame's descriptor array
        const uint32_t e_lo = job.kind != 0 ? min(ncand, start >> 3) : start;
        const uint32_t e_hi = job.kind != 0 ? min(ncand, (end + 7) >> 3) : end;
        const uint32_t* dj = desc + job.desc_off;
        uint32_t c = 0;
        for (uint32_t e = e_lo + 4 * threadIdx.x; e < e_hi; e += 1024) {
            const uint4 v = __ldg(reinterpret_cast<const uint4*>(dj + e));
            c += (v.x != 0 ? 1u : 0u) + (e + 1 < e_hi && v.y != 0 ? 1u : 0u) + (e + 2 < e_hi && v.z != 0 ? 1u : 0u) +
                 (e + 3 < e_hi && v.w != 0 ? 1u : 0u);
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
        if (lane == 0) s_w[warp] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (int w = 0; w < 8; w++) t += s_w[w];
            weight[T] = t;
        }
        __syncthreads();
    }
}

// order[0, ntiles): tile list indices, heaviest bit-length bucket first.  One
// block; the warps rank equal buckets together (one shared atomic per bucket
// and warp).
__global__ void __launch_bounds__(1024) k_tile_order(const uint32_t* __restrict__ weight, uint32_t ntiles,
                                                     uint32_t* __restrict__ order) {
    __shared__ uint32_t s_cnt[33], s_pos[33];
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    const uint32_t lt = (1u << lane) - 1u;
    if (tid < 33) s_cnt[tid] = 0;
    __syncthreads();
    for (uint32_t b0 = 0; b0 < ntiles; b0 += 1024) {  // uniform trip count: every lane takes part in the match
        const uint32_t T = b0 + tid;
        const uint32_t k = T < ntiles ? 32u - __clz(weight[T]) : 33u;
        const uint32_t peers = warp_match<6>(k);  // buckets 0..33
        if (k < 33 && (peers & lt) == 0) atomicAdd(&s_cnt[k], __popc(peers));
    }
    __syncthreads();
    if (tid == 0) {
        uint32_t a = 0;
        for (int k = 32; k >= 0; k--) { s_pos[k] = a; a += s_cnt[k]; }
    }
    __syncthreads();
    for (uint32_t b0 = 0; b0 < ntiles; b0 += 1024) {
        const uint32_t T = b0 + tid;
        const uint32_t k = T < ntiles ? 32u - __clz(weight[T]) : 33u;
        const uint32_t peers = warp_match<6>(k);  // buckets 0..33
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (k < 33 && lane == leader) base = atomicAdd(&s_pos[k], __popc(peers));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        if (k < 33) order[base + __popc(peers & lt)] = T;
    }
}

// ---------------------------------------------------------------------------
// Gather: one CTA per frame concatenates its tiles' slots into the frame's
// contiguous streams (przm_tokenizer.cuh:474-609) and counts the byte
// histograms of the literal stream and of the three command substreams,
// privatised per warp in shared memory.
// ---------------------------------------------------------------------------
constexpr uint32_t kGatherThreads = 512;

// Frame j by the whole block (any multiple of 128 threads); s_off =
// ntiles + 1 words, s_hist = [stream][warp group][symbol] counts.
template <bool kC>
__device__ void gather_item(const Job* __restrict__ jobs, uint32_t j, const uint8_t* slots,
                            const uint32_t* tile_lens, uint8_t* __restrict__ streams,
                            uint32_t* __restrict__ job_lens, uint32_t* __restrict__ hist, uint32_t* __restrict__ err,
                            uint32_t* s_off, uint32_t (*s_hist)[4][256]) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nthr = blockDim.x;
    {
        const Job job = jobs[j];
        uint8_t* sreg = streams + job.str_off;
        __syncthreads();
        for (uint32_t i = tid; i < 4 * 4 * 256; i += nthr) (&s_hist[0][0][0])[i] = 0;
        for (int s = 0; s < S_COUNT; s++) {
            __syncthreads();
            // exclusive scan of this stream's tile lengths (<= 512 tiles)
            if (warp == 0) {
                uint32_t carry = 0;
                for (uint32_t b = 0; b < job.ntiles; b += 32) {
                    uint32_t i = b + lane;
                    // an empty input has no tokenizer tile: its one tile
                    // slot is never written, so its streams are empty
                    uint32_t v = (i < job.ntiles && job.n > 0) ? ld_stage<kC>(tile_lens + (uint64_t)(job.tile0 + i) * S_COUNT + s) : 0;
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
            // one warp per tile
            for (uint32_t t = warp; t < job.ntiles; t += nthr / 32) {
                const uint32_t o = s_off[t], l = s_off[t + 1] - o;
                const uint8_t* sp = slots + (uint64_t)(job.tile0 + t) * kSlotStride + slot_base(s);
                warp_copy_hist<kC>(dst + o, sp, l, hs >= 0 ? s_hist[hs][warp & 3] : nullptr, lane);
            }
            if (tid == 0) job_lens[(uint64_t)j * S_COUNT + s] = total;
        }
        __syncthreads();
        for (uint32_t i = tid; i < 4 * 256; i += nthr) {
            uint32_t hs = i >> 8, sym = i & 255;
            hist[(uint64_t)j * 1024 + i] = s_hist[hs][0][sym] + s_hist[hs][1][sym] + s_hist[hs][2][sym] + s_hist[hs][3][sym];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kGatherThreads) k_gather(const Job* __restrict__ jobs, uint32_t j0, uint32_t njobs,
                                                          const uint8_t* __restrict__ slots,
                                                          const uint32_t* __restrict__ tile_lens,
                                                          uint8_t* __restrict__ streams, uint32_t* __restrict__ job_lens,
                                                          uint32_t* __restrict__ hist /* njobs x 4 x 256 */,
                                                          uint32_t* __restrict__ err) {
    extern __shared__ uint32_t smem_g[];
    __shared__ uint32_t s_hist[4][4][256];
    for (uint32_t jl = blockIdx.x; jl < njobs; jl += gridDim.x)
        gather_item<false>(jobs, j0 + jl, slots, tile_lens, streams, job_lens, hist, err, smem_g, s_hist);
}

}  // namespace pz
