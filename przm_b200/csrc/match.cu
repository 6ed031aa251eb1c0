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
__device__ __forceinline__ uint32_t lcp_smem(const uint8_t* t, uint32_t a, uint32_t b, uint32_t limit) {
    uint32_t len = 4;
    while (len < limit) {
        uint32_t d = ld32_smem_u(t, a + len) ^ ld32_smem_u(t, b + len);
        if (d) { len += (uint32_t)(__ffs(d) - 1) >> 3; break; }
        len += 4;
    }
    return len < limit ? len : limit;
}

// ---------------------------------------------------------------------------
// Tile finder: one CTA of 256 threads per 32 KiB tile of a small frame.
// Semantics of przm_lz77_search_matches_kernel (przm_lz77.cu:221-360) with
// the race-free bucket update: per 256-position step the bucket takes the
// largest p+1 of the step (high half) and the step's second-largest p+1, or
// its previous head when one position hit it (low half).
// ---------------------------------------------------------------------------
struct TileRef { uint32_t job; uint32_t tile; };
constexpr uint32_t kTileFindSmem = kTile + 16 + 3 * kBuckets * 4;

__global__ void __launch_bounds__(256) k_tile_find(const uint8_t* __restrict__ in, const Job* __restrict__ jobs,
                                                   const TileRef* __restrict__ refs, uint32_t nrefs,
                                                   uint32_t* __restrict__ desc) {
    extern __shared__ __align__(16) uint8_t smem_tf[];
    uint8_t* s_tile = smem_tf;                                          // kTile + 16
    uint32_t* s_head = reinterpret_cast<uint32_t*>(smem_tf + kTile + 16); // kBuckets each
    uint32_t* s_top = s_head + kBuckets;
    uint32_t* s_sec = s_top + kBuckets;
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    for (uint32_t r = blockIdx.x; r < nrefs; r += gridDim.x) {
        const Job job = jobs[refs[r].job];
        const uint32_t ts = refs[r].tile * kTile;
        const uint32_t tl = min(kTile, job.n - ts);
        const uint8_t* src = in + job.in_off + ts;
        uint32_t* out = desc + job.desc_off + ts;
        __syncthreads();
        // stage the tile (16-byte vectors; the input region is padded)
        const uint32_t nv = (tl + 15) / 16;
        for (uint32_t v = tid; v < nv; v += 256)
            reinterpret_cast<uint4*>(s_tile)[v] = __ldg(reinterpret_cast<const uint4*>(src) + v);
        if (tid < 4) reinterpret_cast<uint32_t*>(s_tile)[(nv * 16) / 4 + tid] = 0;
        for (uint32_t h = tid; h < kBuckets; h += 256) { s_head[h] = 0; s_top[h] = 0; s_sec[h] = 0; }
        __syncthreads();
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

// ---------------------------------------------------------------------------
// Radix-strike finder: one CTA per large frame (pulled from a work counter),
// walking the frame's 8-aligned k-mer candidates 4096 at a time (one 32 KiB
// tile).  Semantics of przm_lz77_radix_strike_kernel (przm_lz77.cu:156-213)
// in sequential insertion order: the predecessor of candidate p is the latest
// candidate q < p with the same 19-bit hash.  Inside a tile the predecessor
// is resolved in shared memory (slot ids from a small hash, then one ordered
// warp pass); across tiles it comes from the frame's 2^19-entry table in
// global memory, whose entries carry a per-frame tag so it never needs
// clearing.  Output: one descriptor per 8-aligned position (d8[p/8]).
// ---------------------------------------------------------------------------
constexpr uint32_t kRadixThreads = 512;
constexpr uint32_t kSlotHash = 8192;
constexpr uint32_t kRadixSmem = kSlotHash * 4 + kCandPerTile * 4 + 2 * kCandPerTile * 2 + kSlotHash * 2;

__device__ __forceinline__ uint32_t kmer_hash(uint64_t k) {
    return (uint32_t)((k * kRadixPrime) >> 43) & (kRadixBuckets - 1);
}

__global__ void __launch_bounds__(kRadixThreads) k_radix_find(const uint8_t* __restrict__ in,
                                                              const Job* __restrict__ jobs,
                                                              const uint32_t* __restrict__ big, uint32_t nbig,
                                                              uint32_t* __restrict__ work, uint64_t* __restrict__ tables,
                                                              uint64_t* __restrict__ tags, uint32_t* __restrict__ desc) {
    extern __shared__ __align__(16) uint8_t smem_rf[];
    uint32_t* s_key = reinterpret_cast<uint32_t*>(smem_rf);             // kSlotHash
    uint32_t* s_h = s_key + kSlotHash;                                   // kCandPerTile
    uint16_t* s_slot = reinterpret_cast<uint16_t*>(s_h + kCandPerTile);  // kCandPerTile
    uint16_t* s_pred = s_slot + kCandPerTile;                            // kCandPerTile
    uint16_t* s_last = s_pred + kCandPerTile;                            // kSlotHash
    __shared__ uint32_t s_job;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint64_t* table = tables + (uint64_t)blockIdx.x * kRadixBuckets;
    uint64_t tag = tags[blockIdx.x];
    for (;;) {
        __syncthreads();
        if (tid == 0) s_job = atomicAdd(work, 1u);
        __syncthreads();
        const uint32_t jx = s_job;
        if (jx >= nbig) break;
        tag++;
        const Job job = jobs[big[jx]];
        const uint8_t* src = in + job.in_off;
        uint32_t* d8 = desc + job.desc_off;
        const uint32_t n = job.n;
        const uint32_t ncand_total = n >= 8 ? (n - 8) / 8 + 1 : 0;
        for (uint32_t t0 = 0; t0 < ncand_total; t0 += kCandPerTile) {
            const uint32_t nc = min(kCandPerTile, ncand_total - t0);
            __syncthreads();
            for (uint32_t i = tid; i < kSlotHash; i += kRadixThreads) { s_key[i] = 0; s_last[i] = 0xFFFFu; }
            for (uint32_t c = tid; c < nc; c += kRadixThreads) {
                uint64_t k = __ldg(reinterpret_cast<const uint64_t*>(src) + t0 + c);
                s_h[c] = kmer_hash(k);
            }
            __syncthreads();
            for (uint32_t c = tid; c < nc; c += kRadixThreads) {
                const uint32_t key = s_h[c] + 1;
                uint32_t sl = (key * 2654435761u) >> 19;  // 13-bit start slot
                for (;;) {
                    uint32_t prev = atomicCAS(&s_key[sl], 0u, key);
                    if (prev == 0 || prev == key) break;
                    sl = (sl + 1) & (kSlotHash - 1);
                }
                s_slot[c] = (uint16_t)sl;
            }
            __syncthreads();
            if (warp == 0) {
                for (uint32_t g = 0; g < nc; g += 32) {
                    const uint32_t c = g + lane;
                    const bool v = c < nc;
                    const uint32_t act = __ballot_sync(0xFFFFFFFFu, v);
                    const uint32_t sl = v ? s_slot[c] : 0xFFFFFFFFu;
                    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, sl) & act;
                    const uint32_t lower = peers & ((1u << lane) - 1u);
                    uint32_t pred = 0xFFFFu;
                    if (v) pred = lower ? g + (31 - __clz(lower)) : s_last[sl];
                    __syncwarp();
                    if (v) {
                        s_pred[c] = (uint16_t)pred;
                        if ((peers >> lane) == 1u) s_last[sl] = (uint16_t)c;
                    }
                    __syncwarp();
                }
            }
            __syncthreads();
            // resolve predecessors (table reads strictly before this tile's writes)
            uint32_t prevs[kCandPerTile / kRadixThreads];
#pragma unroll
            for (uint32_t k = 0; k < kCandPerTile / kRadixThreads; k++) {
                const uint32_t c = tid + k * kRadixThreads;
                uint32_t pv = 0;  // candidate index + 1 of the predecessor, 0 = none
                if (c < nc) {
                    const uint32_t pr = s_pred[c];
                    if (pr != 0xFFFFu) pv = t0 + pr + 1;
                    else {
                        const uint64_t e = table[s_h[c]];
                        if ((e >> 32) == tag) pv = (uint32_t)e;
                    }
                }
                prevs[k] = pv;
            }
            __syncthreads();
            for (uint32_t c = tid; c < nc; c += kRadixThreads)
                if (s_last[s_slot[c]] == c) table[s_h[c]] = (tag << 32) | (uint64_t)(t0 + c + 1);
            // verify and extend (przm_lz77.cu:180-209); all loads are 8-aligned
#pragma unroll
            for (uint32_t k = 0; k < kCandPerTile / kRadixThreads; k++) {
                const uint32_t c = tid + k * kRadixThreads;
                if (c >= nc) continue;
                uint32_t dsc = 0;
                if (prevs[k]) {
                    const uint32_t p = (t0 + c) * 8, q = (prevs[k] - 1) * 8;
                    const uint32_t dist = p - q;
                    if (dist <= kWindow && dist <= kMaxOff32) {
                        const uint64_t* a = reinterpret_cast<const uint64_t*>(src + p);
                        const uint64_t* b = reinterpret_cast<const uint64_t*>(src + q);
                        if (__ldg(a) == __ldg(b)) {
                            uint32_t L = 8;
                            bool done = false;
                            while ((uint64_t)p + L + 8 <= n && L + 8 <= kMaxLen32) {
                                uint64_t x = __ldg(a + L / 8) ^ __ldg(b + L / 8);
                                if (x) { L += (uint32_t)(__ffsll((long long)x) - 1) >> 3; done = true; break; }
                                L += 8;
                            }
                            if (!done)
                                while (p + L < n && src[p + L] == src[q + L] && L < kMaxLen32) L++;
                            dsc = pack_match32(L, dist);
                        }
                    }
                }
                d8[t0 + c] = dsc;
            }
        }
    }
    __syncthreads();
    if (tid == 0) tags[blockIdx.x] = tag;
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
