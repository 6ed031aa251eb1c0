// match.cu -- LZ77 match finders (per-position 32-bit descriptors).
//
// Two finders, selected per frame exactly as the reference host does
// (gpu/bridge.go:924-950): frames of <= 64 KiB use the shared-memory tile
// finder, larger frames the radix-strike k-mer finder.
#include "common.cuh"

namespace pz {

__device__ __forceinline__ uint32_t hash4(uint32_t w) { return ((w * kHashPrime) >> 21) & (kBuckets - 1); }

// Exact common-prefix length of two shared-memory byte runs that are known to
// agree on their first 4 bytes, capped at limit (przm_lz77.cu:63-85).
// 16 bytes of a 4-byte aligned shared buffer from byte i, as four words
// (five aligned loads, funnel-shifted; the buffer is padded by 32 bytes).
__device__ __forceinline__ void ld128_smem_u(const uint8_t* base, uint32_t i, uint32_t* o) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(base) + (i >> 2);
    const uint32_t sh = (i & 3) * 8;
    const uint32_t w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3], w4 = w[4];
    o[0] = __funnelshift_r(w0, w1, sh);
    o[1] = __funnelshift_r(w1, w2, sh);
    o[2] = __funnelshift_r(w2, w3, sh);
    o[3] = __funnelshift_r(w3, w4, sh);
}

// Exact common-prefix length of two shared-memory byte runs that are known to
// agree on their first 4 bytes, capped at limit (przm_lz77.cu:63-85), 16
// bytes per step.  Reads stay below a + limit + 20 (inside the tile's pad).
__device__ __forceinline__ uint32_t lcp_smem(const uint8_t* t, uint32_t a, uint32_t b, uint32_t limit) {
    for (uint32_t len = 4; len < limit; len += 16) {
        uint32_t x[4], y[4];
        ld128_smem_u(t, a + len, x);
        ld128_smem_u(t, b + len, y);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint32_t d = x[k] ^ y[k];
            if (d) return min(limit, len + 4 * k + ((uint32_t)(__ffs(d) - 1) >> 3));
        }
    }
    return limit;
}

// ---------------------------------------------------------------------------
// Tile finder: one CTA of 256 threads per 32 KiB tile of a small frame.
// Semantics of przm_lz77_search_matches_kernel (przm_lz77.cu:221-360) with
// the race-free bucket update: per 256-position step the bucket takes the
// largest p+1 of the step (high half) and the step's second-largest p+1, or
// its previous head when one position hit it (low half).
// ---------------------------------------------------------------------------
struct TileRef { uint32_t job; uint32_t tile; };
// shared layout: tile + 32 bytes of pad, the copy's mbarrier (16), then the
// three bucket arrays
constexpr uint32_t kTilePad = 32;
constexpr uint32_t kTileFindSmem = kTile + kTilePad + 16 + 3 * kBuckets * 4;

// One tile, by a block of 256 threads; smem = kTileFindSmem bytes.
__device__ void tile_find_item(const uint8_t* __restrict__ in, const Job* __restrict__ jobs, const TileRef ref,
                               uint32_t* __restrict__ desc, uint8_t* smem_tf, uint32_t* err) {
    uint8_t* s_tile = smem_tf;                                                      // kTile + kTilePad
    uint64_t* s_bar = reinterpret_cast<uint64_t*>(smem_tf + kTile + kTilePad);     // copy completion
    uint32_t* s_head = reinterpret_cast<uint32_t*>(smem_tf + kTile + kTilePad + 16);  // kBuckets each
    uint32_t* s_top = s_head + kBuckets;
    uint32_t* s_sec = s_top + kBuckets;
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    {
        const Job job = jobs[ref.job];
        const uint32_t ts = ref.tile * kTile;
        const uint32_t tl = min(kTile, job.n - ts);
        const uint8_t* src = in + job.in_off + ts;
        uint32_t* out = desc + job.desc_off + ts;
        __syncthreads();
        // stage the tile with one bulk copy (src: in_off is 16-byte aligned,
        // tiles are 32 KiB apart; the input region is padded past n, so the
        // copy may round up to 16 bytes) while the buckets are cleared
        const uint32_t nv = (tl + 15) / 16;
        if (tid == 0) mbar_init(s_bar, 1);
        __syncthreads();
        if (tid == 0) bulk_load(s_tile, src, nv * 16, s_bar);
        if (tid < kTilePad / 4) reinterpret_cast<uint32_t*>(s_tile)[(nv * 16) / 4 + tid] = 0;
        for (uint32_t h = tid; h < kBuckets; h += 256) { s_head[h] = 0; s_top[h] = 0; s_sec[h] = 0; }
        mbar_wait_bounded(s_bar, 0, err);
        __syncthreads();
        if (tid == 0) mbar_inval(s_bar);
        const uint32_t steps = (tl + 255) / 256;
        for (uint32_t st = 0; st < steps; st++) {
            const uint32_t p = st * 256 + tid;
            const bool valid = p + 4 <= tl;
            const uint32_t w4 = valid ? ld32_smem_u(s_tile, p) : 0;
            const uint32_t h = valid ? hash4(w4) : 0;
            uint32_t best_len = 0, best_off = 0, d = 0;
            const uint32_t lim = valid ? min(tl - p, kMaxLen32) : 0;
#pragma unroll
            for (uint32_t delta = 1; delta <= 4; delta++) {
                uint32_t pw = __shfl_up_sync(0xFFFFFFFFu, w4, delta);
                if (valid && lane >= delta && pw == w4) {
                    uint32_t l = lcp_smem(s_tile, p, p - delta, lim);
                    if (l > best_len) { best_len = l; best_off = delta; }
                }
            }
            if (valid) {
                const uint32_t bv = s_head[h];
                const uint32_t c0 = bv >> 16, c1 = bv & 0xFFFFu;
                if (c0) {
                    uint32_t c = c0 - 1;
                    if (c < p && p - c <= kWindow && ld32_smem_u(s_tile, c) == w4) {
                        uint32_t l = lcp_smem(s_tile, p, c, lim);
                        if (l > best_len) { best_len = l; best_off = p - c; }
                    }
                }
                if (c1 && best_len < 258) {
                    uint32_t c = c1 - 1;
                    if (c < p && p - c <= kWindow && ld32_smem_u(s_tile, c) == w4) {
                        uint32_t l = lcp_smem(s_tile, p, c, lim);
                        if (l > best_len) { best_len = l; best_off = p - c; }
                    }
                }
                if (best_len >= 4 && best_off <= kMaxOff32) d = pack_match32(best_len, best_off);
            }
            if (p < tl) out[p] = d;
            __syncthreads();
            if (valid) atomicMax(&s_top[h], p + 1);
            __syncthreads();
            if (valid && s_top[h] != p + 1) atomicMax(&s_sec[h], p + 1);
            __syncthreads();
            if (valid && s_top[h] == p + 1) {
                const uint32_t sec = s_sec[h];
                s_head[h] = ((p + 1) << 16) | (sec ? sec : (s_head[h] >> 16));
                s_top[h] = 0;
                s_sec[h] = 0;
            }
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(256) k_tile_find(const uint8_t* __restrict__ in, const Job* __restrict__ jobs,
                                                   const TileRef* __restrict__ refs, uint32_t nrefs,
                                                   uint32_t* __restrict__ desc, uint32_t* __restrict__ err) {
    extern __shared__ __align__(16) uint8_t smem_tf[];
    for (uint32_t r = blockIdx.x; r < nrefs; r += gridDim.x) tile_find_item(in, jobs, refs[r], desc, smem_tf, err);
}

// ---------------------------------------------------------------------------
// Radix-strike finder, semantics of przm_lz77_radix_strike_kernel
// (przm_lz77.cu:156-213) in sequential insertion order: candidate c (the
// k-mer at byte 8c) takes as predecessor the latest candidate q < c with the
// same 19-bit hash; the match is verified and extended against it.
//
// Candidates with equal hashes share the hash's top 8 bits, so each frame is
// split into 256 partitions that never interact:
//   k_rx_sort    per 32 KiB tile (4096 candidates): hashes, then a stable
//                sort of the tile's candidates by partition in shared memory,
//                written out as the tile's slice of the candidate list (one
//                word per candidate: its low 11 hash bits and its index in
//                the tile) with the start of every partition's run;
//   k_rx_resolve one warp per (frame, partition): walks the partition's runs
//                tile by tile (so in position order) 32 candidates at a time
//                with a 2048-entry shared table of the latest candidate per
//                low-11-bit key (ties inside the 32 resolved with
//                warp_match) and stores each candidate's predecessor in its
//                slot of the list;
//   k_rx_verify  one thread per slot: verifies and extends the match against
//                the predecessor and writes the descriptor.
// Output: one descriptor per 8-aligned position (d8[c]), every candidate
// written exactly once.
// ---------------------------------------------------------------------------
constexpr uint32_t kRxKeyBits = 11;
constexpr uint32_t kRxParts = 256;       // partitions: hash >> 11
constexpr uint32_t kRxKeys = 2048;       // keys inside a partition: hash & 2047
constexpr uint32_t kRxResolveWarps = 8;  // warps per k_rx_resolve block
constexpr uint32_t kRxResolveSmem = kRxResolveWarps * kRxKeys * 4;
static_assert(kCandPerTile == 4096, "a list word holds a 12-bit index in the tile");

struct RxTile { uint32_t job; uint32_t tile; };

__device__ __forceinline__ uint32_t kmer_hash(uint64_t k) {
    return (uint32_t)((k * kRadixPrime) >> 43) & (kRadixBuckets - 1);
}
__host__ __device__ inline uint32_t rx_ncand(uint32_t n) { return n >= 8 ? (n - 8) / 8 + 1 : 0; }

struct RxSortSmem {
    uint32_t w[8][kRxParts];         // per warp and partition: count, then next slot
    uint32_t list[kCandPerTile];     // the tile's list, partition-sorted
    uint32_t warp[32];
};

// One radix tile by a block of 256 threads: warp w takes candidates
// [c0 + 512 w, c0 + 512 w + 512) in 16 rounds of 32.  Slots follow
// (partition, warp, round, lane), i.e. position order inside a partition.
// toff[(tile0 + t) * 256 + b]: where partition b's run starts in the tile's
// slice; the slice of tile t is list[c0, c1) of the frame.
__device__ void rx_sort_item(const uint8_t* __restrict__ in, const Job* __restrict__ jobs, const RxTile tt,
                             uint32_t* __restrict__ toff, uint32_t* __restrict__ list, RxSortSmem& sm) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const Job job = jobs[tt.job];
    const uint64_t* src = reinterpret_cast<const uint64_t*>(in + job.in_off);
    const uint32_t C = rx_ncand(job.n), c0 = tt.tile * kCandPerTile, c1 = min(C, c0 + kCandPerTile);
    __syncthreads();  // the previous item no longer reads sm
    for (uint32_t i = tid; i < 8 * kRxParts; i += 256) (&sm.w[0][0])[i] = 0;
    __syncthreads();
    uint32_t h[16], peers[16];  // hash and same-partition lanes of each round
#pragma unroll
    for (int r = 0; r < 16; r++) {
        const uint32_t c = c0 + 512 * warp + 32 * r + lane;
        h[r] = c < c1 ? kmer_hash(__ldg(src + c)) : 0xFFFFFFFFu;
    }
#pragma unroll
    for (int r = 0; r < 16; r++) {
        peers[r] = warp_match<9>(h[r] != 0xFFFFFFFFu ? h[r] >> kRxKeyBits : kRxParts);  // 256: no candidate
        if (h[r] != 0xFFFFFFFFu && (peers[r] & lt) == 0) sm.w[warp][h[r] >> kRxKeyBits] += __popc(peers[r]);
        __syncwarp();
    }
    __syncthreads();
    {  // thread b: partition b's start in the slice, then each warp's first slot in it
        const uint32_t b = tid;
        uint32_t tot = 0;
#pragma unroll
        for (int w = 0; w < 8; w++) tot += sm.w[w][b];
        uint32_t all;
        uint32_t run = block_exclusive_scan<256>(tot, sm.warp, all);
        toff[(uint64_t)(job.tile0 + tt.tile) * kRxParts + b] = run;
#pragma unroll
        for (int w = 0; w < 8; w++) {
            const uint32_t k = sm.w[w][b];
            sm.w[w][b] = run;
            run += k;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 16; r++) {
        const uint32_t c = c0 + 512 * warp + 32 * r + lane;
        uint32_t slot = 0;
        if (h[r] != 0xFFFFFFFFu) slot = sm.w[warp][h[r] >> kRxKeyBits] + __popc(peers[r] & lt);
        __syncwarp();
        if (h[r] != 0xFFFFFFFFu) {
            if ((peers[r] & lt) == 0) sm.w[warp][h[r] >> kRxKeyBits] += __popc(peers[r]);
            sm.list[slot] = (h[r] & (kRxKeys - 1)) << 12 | (c - c0);
        }
        __syncwarp();
    }
    __syncthreads();
    uint32_t* lj = list + job.desc_off + c0;
    const uint32_t m = c1 - c0;
    if ((reinterpret_cast<uintptr_t>(lj) & 15) == 0) {
        for (uint32_t i = tid; i < m / 4; i += 256) reinterpret_cast<uint4*>(lj)[i] = reinterpret_cast<const uint4*>(sm.list)[i];
        for (uint32_t i = (m & ~3u) + tid; i < m; i += 256) lj[i] = sm.list[i];
    } else {
        for (uint32_t i = tid; i < m; i += 256) lj[i] = sm.list[i];
    }
}

__global__ void __launch_bounds__(256) k_rx_sort(const uint8_t* __restrict__ in, const Job* __restrict__ jobs,
                                                 const RxTile* __restrict__ rt, uint32_t nrt,
                                                 uint32_t* __restrict__ toff, uint32_t* __restrict__ list) {
    __shared__ RxSortSmem sm;
    for (uint32_t T = blockIdx.x; T < nrt; T += gridDim.x) rx_sort_item(in, jobs, rt[T], toff, list, sm);
}

// Verification and extension of candidate c against its predecessor q
// (przm_lz77.cu:180-209): the match grows in 8-byte steps while
// p + L + 8 <= n and L + 8 <= 4095, then byte by byte below 4095.  Four steps
// are loaded per round trip (all loads 8-aligned; the input is padded by 64
// bytes, so words past n are readable and only used where a step allows).
// rx_first is the first round trip: the XOR of the 32 bytes at the candidate
// and at its predecessor (loaded whatever the distance; both lie in the
// frame's padded input).
__device__ __forceinline__ void rx_first(const uint8_t* src, uint32_t c, uint32_t q, uint64_t* x) {
    const uint64_t* a = reinterpret_cast<const uint64_t*>(src + 8 * c);
    const uint64_t* b = reinterpret_cast<const uint64_t*>(src + 8 * q);
#pragma unroll
    for (int k = 0; k < 4; k++) x[k] = __ldg(a + k) ^ __ldg(b + k);
}

// The descriptor of candidate c against predecessor q, given rx_first's words.
__device__ __forceinline__ uint32_t rx_finish(const uint8_t* src, uint32_t n, uint32_t c, uint32_t q, uint64_t* x) {
    const uint32_t p = c * 8, pq = q * 8;
    const uint32_t dist = p - pq;
    if (dist > kWindow || dist > kMaxOff32) return 0;
    if (x[0]) return 0;
    const uint64_t* a = reinterpret_cast<const uint64_t*>(src + p);
    const uint64_t* b = reinterpret_cast<const uint64_t*>(src + pq);
    uint32_t L = 8;
    int k0 = 1;
    for (;;) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (k < k0) continue;
            if (!((uint64_t)p + L + 8 <= n && L + 8 <= kMaxLen32)) goto bytes;
            if (x[k]) return pack_match32(L + ((uint32_t)(__ffsll((long long)x[k]) - 1) >> 3), dist);
            L += 8;
        }
#pragma unroll
        for (int k = 0; k < 4; k++) x[k] = __ldg(a + L / 8 + k) ^ __ldg(b + L / 8 + k);
        k0 = 0;
    }
bytes:
    while (p + L < n && src[p + L] == src[pq + L] && L < kMaxLen32) L++;
    return pack_match32(L, dist);
}

// Partition b of large frame j, by one warp; table = kRxKeys words of
// shared memory (latest candidate + 1 per key, 0 = none).  The partition is
// the concatenation of its runs in tiles 0, 1, ...: 32 tiles at a time, lane
// l holds tile t0 + l's run, and the slot of the warp's i-th entry is found
// by a binary search over the runs' prefix sums.  pred[slot] = predecessor
// + 1 (0: none).
template <bool kC>
__device__ void rx_resolve_warp(const Job* __restrict__ jobs, uint32_t j, uint32_t b, const uint32_t* toff,
                                const uint32_t* list, uint32_t* __restrict__ pred, uint32_t* table) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const Job job = jobs[j];
    const uint32_t C = rx_ncand(job.n), nt = (C + kCandPerTile - 1) / kCandPerTile;
    const uint32_t* lj = list + job.desc_off;
    uint32_t* pj = pred + job.desc_off;
    for (uint32_t i = lane; i < kRxKeys / 4; i += 32) reinterpret_cast<uint4*>(table)[i] = make_uint4(0, 0, 0, 0);
    __syncwarp();
    for (uint32_t t0 = 0; t0 < nt; t0 += 32) {
        // lane l: the run of tile t0 + l, as slots [st, st + len) of the frame's list
        const uint32_t t = t0 + lane;
        uint32_t st = 0, len = 0;
        if (t < nt) {
            const uint32_t* to = toff + (uint64_t)(job.tile0 + t) * kRxParts;
            const uint32_t tc = min(C - t * kCandPerTile, kCandPerTile);
            const uint32_t a = ld_stage<kC>(to + b);
            const uint32_t e = b + 1 < kRxParts ? ld_stage<kC>(to + b + 1) : tc;
            st = t * kCandPerTile + a;
            len = e - a;
        }
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= (uint32_t)o) incl += y;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        const uint32_t excl = incl - len;
        // 256 entries per round trip: each lane loads 8 (one per chunk of 32)
        // together, then the 8 chunks resolve in order from registers
        for (uint32_t b0 = 0; b0 < total; b0 += 256) {
            uint32_t ee[8], sl[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const uint32_t i = b0 + 32 * u + lane;
                // the run holding entry i: the first lane whose inclusive sum exceeds i
                uint32_t k = 0;
#pragma unroll
                for (uint32_t w = 16; w >= 1; w >>= 1) {
                    const uint32_t probe = __shfl_sync(0xFFFFFFFFu, incl, k + w - 1);
                    if (probe <= i) k += w;
                }
                const uint32_t sk = __shfl_sync(0xFFFFFFFFu, st, k & 31), xk = __shfl_sync(0xFFFFFFFFu, excl, k & 31);
                sl[u] = i < total ? sk + (i - xk) : 0u;
                ee[u] = i < total ? ld_stage<kC>(lj + sl[u]) : 0xFFFFFFFFu;
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const uint32_t i = b0 + 32 * u + lane;
                const bool v = i < total;
                const uint32_t k = ee[u] >> 12;
                const uint32_t c = (sl[u] & ~(kCandPerTile - 1)) | (ee[u] & (kCandPerTile - 1));
                const uint32_t peers = warp_match<12>(v ? k : kRxKeys);  // 2048: no entry
                const uint32_t lower = peers & lt;
                const uint32_t from = lower ? 31u - __clz(lower) : lane;
                const uint32_t cl = __shfl_sync(0xFFFFFFFFu, c, from);
                uint32_t pv = 0;  // predecessor + 1
                if (v) pv = lower ? cl + 1 : table[k];
                __syncwarp();
                if (v && (peers >> lane) == 1u) table[k] = c + 1;
                __syncwarp();
                if (v) pj[sl[u]] = pv;
            }
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kRxResolveWarps * 32) k_rx_resolve(const Job* __restrict__ jobs,
                                                                     const uint32_t* __restrict__ big, uint32_t nbig,
                                                                     const uint32_t* __restrict__ toff,
                                                                     const uint32_t* __restrict__ list,
                                                                     uint32_t* __restrict__ pred) {
    extern __shared__ __align__(16) uint32_t smem_rx[];
    const uint32_t warp = threadIdx.x >> 5;
    uint32_t* table = smem_rx + warp * kRxKeys;
    const uint32_t nw = gridDim.x * kRxResolveWarps;
    for (uint32_t x = blockIdx.x * kRxResolveWarps + warp; x < nbig * kRxParts; x += nw)
        rx_resolve_warp<false>(jobs, big[x / kRxParts], x % kRxParts, toff, list, pred, table);
}

// Slots [lo, hi) of large frame `job`'s list, thread t of nthr: verify and
// extend each slot's candidate against its predecessor and write the
// descriptor; two slots per thread per step, their first loads in flight
// together.  Slot i lies in tile i / 4096's slice, so its candidate is that
// tile's base plus the index in the list word.
template <bool kC>
__device__ __forceinline__ void rx_verify_range(const uint8_t* __restrict__ in, const Job& job,
                                                const uint32_t* list, const uint32_t* pred,
                                                uint32_t* __restrict__ desc, uint32_t lo, uint32_t hi, uint32_t t,
                                                uint32_t nthr) {
    const uint8_t* src = in + job.in_off;
    const uint32_t* lj = list + job.desc_off;
    const uint32_t* pj = pred + job.desc_off;
    uint32_t* d8 = desc + job.desc_off;
    const uint32_t stride = nthr;
    constexpr uint32_t kHi = ~(kCandPerTile - 1), kLo = kCandPerTile - 1;
    for (uint32_t i = lo + t; i < hi; i += 2 * stride) {
        const uint32_t i2 = i + stride;
        const bool two = i2 < hi;
        const uint32_t c1 = (i & kHi) | (ld_stage<kC>(lj + i) & kLo), p1 = ld_stage<kC>(pj + i);
        const uint32_t c2 = two ? (i2 & kHi) | (ld_stage<kC>(lj + i2) & kLo) : 0u, p2 = two ? ld_stage<kC>(pj + i2) : 0u;
        uint64_t x1[4], x2[4];
        if (p1) rx_first(src, c1, p1 - 1, x1);
        if (p2) rx_first(src, c2, p2 - 1, x2);
        d8[c1] = p1 ? rx_finish(src, job.n, c1, p1 - 1, x1) : 0u;
        if (two) d8[c2] = p2 ? rx_finish(src, job.n, c2, p2 - 1, x2) : 0u;
    }
}

__global__ void __launch_bounds__(256) k_rx_verify(const uint8_t* __restrict__ in, const Job* __restrict__ jobs,
                                                   const uint32_t* __restrict__ big, const uint32_t* __restrict__ list,
                                                   const uint32_t* __restrict__ pred, uint32_t nbig,
                                                   uint32_t* __restrict__ desc) {
    for (uint32_t y = blockIdx.y; y < nbig; y += gridDim.y) {
        const Job job = jobs[big[y]];
        rx_verify_range<false>(in, job, list, pred, desc, 0, rx_ncand(job.n), blockIdx.x * 256 + threadIdx.x, gridDim.x * 256);
    }
}

// ---------------------------------------------------------------------------
// Compaction for the MatchLZ77 API (przm_lz77.cu:510-664): ascending
// (position, descriptor) pairs of the non-zero 8-aligned descriptors.
// Single-pass: per-block counts, then a decoupled look-back-free two-kernel
// scan is unnecessary here -- the block count is small, so one block scans.
// ---------------------------------------------------------------------------
__global__ void k_compact_count(const uint32_t* __restrict__ d8, uint32_t nd, uint32_t* __restrict__ counts) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t v = (i < nd && d8[i] != 0) ? 1u : 0u;
    uint32_t b = __syncthreads_count(v);
    if (threadIdx.x == 0) counts[blockIdx.x] = b;
}

__global__ void k_compact_scan(uint32_t* __restrict__ counts, uint32_t nblocks, uint32_t* __restrict__ total) {
    __shared__ uint32_t s[1024];
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nblocks; base += 1024) {
        uint32_t i = base + threadIdx.x;
        uint32_t v = i < nblocks ? counts[i] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (uint32_t o = 1; o < 1024; o <<= 1) {
            uint32_t t = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < nblocks) counts[i] = carry + s[threadIdx.x] - v;
        uint32_t tot = s[1023];
        __syncthreads();
        carry += tot;
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_compact_scatter(const uint32_t* __restrict__ d8, uint32_t nd, const uint32_t* __restrict__ offs,
                                  uint32_t pos_base, uint32_t* __restrict__ out_pos, uint32_t* __restrict__ out_desc) {
    __shared__ uint32_t s_w[32];
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    bool v = i < nd && d8[i] != 0;
    uint32_t m = __ballot_sync(0xFFFFFFFFu, v);
    if (lane == 0) s_w[warp] = __popc(m);
    __syncthreads();
    if (warp == 0) {
        uint32_t x = lane < (blockDim.x >> 5) ? s_w[lane] : 0;
        for (uint32_t o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        s_w[lane] = x;
    }
    __syncthreads();
    if (v) {
        uint32_t r = offs[blockIdx.x] + (warp ? s_w[warp - 1] : 0) + __popc(m & ((1u << lane) - 1u));
        out_pos[r] = pos_base + i * 8;
        out_desc[r] = d8[i];
    }
}

}  // namespace pz
