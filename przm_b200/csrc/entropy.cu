// entropy.cu -- frequency normalisation, 4-lane interleaved rANS (V-ANS and
// Meta8) and stitching of the lane outputs into the reference byte order.
#include "common.cuh"
#include "meta8_tables.h"

namespace pz {

// ---------------------------------------------------------------------------
// Encoding tables.  The step x' = x + bias + floor(x / f) * (M - f) with the
// quotient from a multiply-high by a per-symbol reciprocal, and the f = 1
// case done as a one-short reciprocal with the deficit moved into the bias,
// is the reciprocal-encoder form of rANS that F. Giesen published with
// ryg_rans (rans_byte.h, RansEncSymbolInit / RansEncPutSymbol, 2014); the
// reciprocal itself is Granlund-Montgomery's (PLDI 1994).
// ---------------------------------------------------------------------------
__host__ __device__ inline EncSym make_encsym(uint32_t f, uint32_t c) {
    EncSym e;
    if (f == 0) { e.m = 0; e.t1 = 0xFFFFFFFFu; e.t2 = 0xFFFFFFFFu; e.w = 0; return e; }
    uint32_t s = 0;
    while ((2u << s) <= f) s++;  // floor(log2 f)
    uint32_t cb = c;
    if (f == 1) { e.m = 0xFFFFFFFFu; s = 0; cb = c + 4095; }
    else if ((f & (f - 1)) == 0) { e.m = 1u << (32 - s); s = 0; }
    else e.m = (uint32_t)(((1ull << (32 + s)) + f - 1) / f);
    e.t1 = 4096u * f;
    const uint64_t t2 = 256ull * e.t1;
    e.t2 = t2 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)t2;
    e.w = cb | ((4096u - f) << 13) | (s << 25);
    return e;
}

// SerializeMatrix (gpu/bridge.go:2844-2886) == EncodeJointNibbleFreq
// (core/literals/literals.go:143-184).
__host__ __device__ inline uint32_t serialize_matrix(const uint16_t* freq, uint8_t* out) {
    uint32_t n = 0;
    uint32_t rowMask = 0;
    for (int h = 0; h < 16; h++)
        for (int l = 0; l < 16; l++)
            if (freq[(h << 4) | l]) { rowMask |= 1u << h; break; }
    out[n++] = (uint8_t)rowMask;
    out[n++] = (uint8_t)(rowMask >> 8);
    for (int h = 0; h < 16; h++) {
        if (!(rowMask & (1u << h))) continue;
        uint32_t colMask = 0;
        for (int l = 0; l < 16; l++)
            if (freq[(h << 4) | l]) colMask |= 1u << l;
        out[n++] = (uint8_t)colMask;
        out[n++] = (uint8_t)(colMask >> 8);
        for (int l = 0; l < 16; l++) {
            if (!(colMask & (1u << l))) continue;
            uint32_t w = freq[(h << 4) | l];
            if (w < 128) out[n++] = (uint8_t)w;
            else { out[n++] = (uint8_t)(0x80 | (w >> 8)); out[n++] = (uint8_t)(w & 0xFF); }
        }
    }
    return n;
}

// ---------------------------------------------------------------------------
// Go sort.Slice (pdqsort, Go standard library sort/zsortfunc.go, Go >= 1.19)
// restated for the descending-remainder sort of NormalizeFreq
// (gpu/bridge.go:2818-2824); it fixes where equal remainders land.
// ---------------------------------------------------------------------------
struct GoRem { uint32_t sym; uint64_t rem; };
struct GoSort {
    GoRem* v;
    __host__ __device__ bool less(int i, int j) const { return v[i].rem > v[j].rem; }
    __host__ __device__ void swap(int i, int j) { GoRem t = v[i]; v[i] = v[j]; v[j] = t; }
    __host__ __device__ void insertion(int a, int b) {
        for (int i = a + 1; i < b; i++)
            for (int j = i; j > a && less(j, j - 1); j--) swap(j, j - 1);
    }
    __host__ __device__ void sift(int lo, int hi, int first) {
        int root = lo;
        for (;;) {
            int child = 2 * root + 1;
            if (child >= hi) return;
            if (child + 1 < hi && less(first + child, first + child + 1)) child++;
            if (!less(first + root, first + child)) return;
            swap(first + root, first + child);
            root = child;
        }
    }
    __host__ __device__ void heap(int a, int b) {
        int first = a, hi = b - a;
        for (int i = (hi - 1) / 2; i >= 0; i--) sift(i, hi, first);
        for (int i = hi - 1; i >= 0; i--) { swap(first, first + i); sift(0, i, first); }
    }
    __host__ __device__ static int bits_len(unsigned x) { int n = 0; while (x) { n++; x >>= 1; } return n; }
    __host__ __device__ void break_patterns(int a, int b) {
        int length = b - a;
        if (length < 8) return;
        uint64_t r = (uint64_t)length;
        unsigned modulus = 1u << bits_len((unsigned)length);
        int idx = a + (length / 4) * 2 - 1;
        for (int i = 0; i < 3; i++) {
            r ^= r << 13; r ^= r >> 7; r ^= r << 17;
            int other = (int)((unsigned)r & (modulus - 1));
            if (other >= length) other -= length;
            swap(idx - 1 + i, a + other);
        }
    }
    __host__ __device__ void order2(int& a, int& b, int& swaps) {
        if (less(b, a)) { int t = a; a = b; b = t; swaps++; }
    }
    __host__ __device__ int median(int a, int b, int c, int& swaps) {
        order2(a, b, swaps); order2(b, c, swaps); order2(a, b, swaps);
        return b;
    }
    __host__ __device__ int choose_pivot(int a, int b, int& hint) {
        int l = b - a, swaps = 0;
        int i = a + l / 4 * 1, j = a + l / 4 * 2, k = a + l / 4 * 3;
        if (l >= 8) {
            if (l >= 50) {
                i = median(i - 1, i, i + 1, swaps);
                j = median(j - 1, j, j + 1, swaps);
                k = median(k - 1, k, k + 1, swaps);
            }
            j = median(i, j, k, swaps);
        }
        hint = swaps == 0 ? 1 : (swaps == 12 ? 2 : 0);
        return j;
    }
    __host__ __device__ void reverse(int a, int b) { for (int i = a, j = b - 1; i < j; i++, j--) swap(i, j); }
    __host__ __device__ bool partial_insertion(int a, int b) {
        int i = a + 1;
        for (int step = 0; step < 5; step++) {
            while (i < b && !less(i, i - 1)) i++;
            if (i == b) return true;
            if (b - a < 50) return false;
            swap(i, i - 1);
            if (i - a >= 2)
                for (int j = i - 1; j >= 1; j--) { if (!less(j, j - 1)) break; swap(j, j - 1); }
            if (b - i >= 2)
                for (int j = i + 1; j < b; j++) { if (!less(j, j - 1)) break; swap(j, j - 1); }
        }
        return false;
    }
    __host__ __device__ int partition_equal(int a, int b, int pivot) {
        swap(a, pivot);
        int i = a + 1, j = b - 1;
        for (;;) {
            while (i <= j && !less(a, i)) i++;
            while (i <= j && less(a, j)) j--;
            if (i > j) break;
            swap(i, j); i++; j--;
        }
        return i;
    }
    __host__ __device__ int partition(int a, int b, int pivot, bool& already) {
        swap(a, pivot);
        int i = a + 1, j = b - 1;
        while (i <= j && less(i, a)) i++;
        while (i <= j && !less(j, a)) j--;
        if (i > j) { swap(j, a); already = true; return j; }
        swap(i, j); i++; j--;
        for (;;) {
            while (i <= j && less(i, a)) i++;
            while (i <= j && !less(j, a)) j--;
            if (i > j) break;
            swap(i, j); i++; j--;
        }
        swap(j, a);
        already = false;
        return j;
    }
    // pdqsort_func: the recursion goes to the smaller side, so its depth is
    // at most log2(n) + 1 (<= 9 for the 256-entry remainder list)
    __host__ __device__ void pdq(int a, int b, int limit) {
        bool was_balanced = true, was_partitioned = true;
        for (;;) {
            int length = b - a;
            if (length <= 12) { insertion(a, b); return; }
            if (limit == 0) { heap(a, b); return; }
            if (!was_balanced) { break_patterns(a, b); limit--; }
            int hint;
            int pivot = choose_pivot(a, b, hint);
            if (hint == 2) { reverse(a, b); pivot = (b - 1) - (pivot - a); hint = 1; }
            if (was_balanced && was_partitioned && hint == 1)
                if (partial_insertion(a, b)) return;
            if (a > 0 && !less(a - 1, pivot)) { a = partition_equal(a, b, pivot); continue; }
            bool already;
            int mid = partition(a, b, pivot, already);
            was_partitioned = already;
            int left = mid - a, right = b - mid, thr = length / 8;
            if (left < right) {
                was_balanced = left >= thr;
                pdq(a, mid, limit);
                a = mid + 1;
            } else {
                was_balanced = right >= thr;
                pdq(mid + 1, b, limit);
                b = mid;
            }
        }
    }
    __host__ __device__ void sort(int n) { pdq(0, n, bits_len((unsigned)n)); }
};


// ---------------------------------------------------------------------------
// Normalisers (one warp per histogram).  All lanes return the same table.
// ---------------------------------------------------------------------------

// literals.NormalizeFrequencies + adjustFrequencySum
// (core/literals/literals.go:78-140): f = 1 + c*(4096-unique)/total, then the
// shortfall goes +1 each to the symbols with the largest counts (lowest
// symbol first among equal counts).
__device__ void warp_normalize_frequencies(const uint32_t* __restrict__ cnt /* smem */, uint16_t* __restrict__ freq /* smem */,
                                           uint32_t lane) {
    uint64_t total = 0;
    uint32_t unique = 0;
    for (uint32_t s = lane; s < 256; s += 32) { total += cnt[s]; unique += cnt[s] ? 1 : 0; }
    for (int o = 16; o; o >>= 1) {
        total += __shfl_xor_sync(0xFFFFFFFFu, total, o);
        unique += __shfl_xor_sync(0xFFFFFFFFu, unique, o);
    }
    uint32_t sum = 0;
    for (uint32_t s = lane; s < 256; s += 32) {
        uint32_t f = 0;
        if (cnt[s]) f = 1 + (uint32_t)(((uint64_t)cnt[s] * (4096 - unique)) / total);
        freq[s] = (uint16_t)f;
        sum += f;
    }
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
    __syncwarp();
    if (unique == 0) return;
    const int diff = 4096 - (int)(sum & 0xFFFF);
    if (diff > 0) {
        // rank among active symbols by (count desc, symbol asc)
        for (uint32_t s = lane; s < 256; s += 32) {
            const uint32_t c = cnt[s];
            if (!c) continue;
            uint32_t rank = 0;
            for (uint32_t t = 0; t < 256; t++) {
                const uint32_t ct = cnt[t];
                rank += (ct > c || (ct == c && ct != 0 && t < s)) ? 1 : 0;
            }
            if (rank < (uint32_t)diff) freq[s] = (uint16_t)(freq[s] + 1);
        }
    } else if (diff < 0 && lane == 0) {
        for (int it = 0; it < -diff; it++)
            for (int s = 255; s >= 0; s--)
                if (freq[s] > 1) { freq[s]--; break; }
    }
    __syncwarp();
}

// gpu.NormalizeFreq (gpu/bridge.go:2777-2829): f = 1 + c*(M-active)/total,
// then +1 to the symbols with the largest remainders in Go sort.Slice order.
__device__ void warp_normalize_freq_go(const uint32_t* __restrict__ cnt, uint16_t* __restrict__ freq, GoRem* __restrict__ rems,
                                       uint32_t lane) {
    if (lane == 0) {
        uint64_t total = 0;
        int active = 0;
        for (int s = 0; s < 256; s++) { freq[s] = 0; total += cnt[s]; active += cnt[s] ? 1 : 0; }
        if (total != 0 && active != 0) {
            const uint32_t rt = 4096 - (uint32_t)active;
            uint32_t alloc = 0;
            int nr = 0;
            for (int s = 0; s < 256; s++) {
                if (!cnt[s]) continue;
                const uint64_t prod = (uint64_t)cnt[s] * rt;
                const uint32_t add = (uint32_t)(prod / total);
                freq[s] = (uint16_t)(1 + add);
                alloc += 1 + add;
                rems[nr].sym = (uint32_t)s;
                rems[nr].rem = prod % total;
                nr++;
            }
            if (alloc < 4096) {
                const int diff = (int)(4096 - alloc);
                GoSort g{rems};
                g.sort(nr);
                for (int i = 0; i < diff && i < nr; i++) freq[rems[i].sym]++;
            }
        }
    }
    __syncwarp();
}

// CDF + encoding table + serialized matrix of one normalised model.
__device__ void warp_build_table(const uint16_t* __restrict__ freq /* smem */, EncSym* __restrict__ tab, TableInfo* __restrict__ info,
                                 uint32_t lane) {
    // exclusive prefix sum over 256 frequencies, 8 per lane in symbol order
    uint32_t f[8], loc = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) { f[k] = freq[lane * 8 + k]; loc += f[k]; }
    uint32_t x = loc;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    uint32_t c = x - loc;
#pragma unroll
    for (int k = 0; k < 8; k++) { tab[lane * 8 + k] = make_encsym(f[k], c); c += f[k]; }
    if (lane == 0) {
        uint32_t act = 0;
        for (int s = 0; s < 256; s++) act += freq[s] ? 1 : 0;
        info->active = act;
        info->mat_len = serialize_matrix(freq, info->mat);
    }
}

// One block per frame of [j0, j0 + gridDim.x), one warp per adaptive model:
// lit, op, meta, var; for P2 frames and up with a codes task the distance
// codes (their histogram in the frame's Section 3 region); for P3 frames
// every non-empty fiber (histograms in the frame's fiber region).
__global__ void __launch_bounds__(32 * kModels) k_normalize(const Job* __restrict__ jobs, uint32_t j0,
                                                            const uint32_t* __restrict__ hist,
                                                            const uint8_t* __restrict__ s3base,
                                                            const S3Frame* __restrict__ s3f,
                                                            const uint8_t* __restrict__ fibbase, EncSym* __restrict__ tabs,
                                                            TableInfo* __restrict__ infos) {
    __shared__ uint32_t s_cnt[kModels][256];
    __shared__ uint16_t s_freq[kModels][256];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t j = j0 + blockIdx.x, gw = kModels * j + w;
    const uint32_t* src;
    if (w < 4) {
        src = hist + (uint64_t)j * 1024 + w * 256;
    } else {
        const Job job = jobs[j];
        if (w == 4) {
            if (job.profile < 2 || s3_task_nd(s3f[j]) < 64) return;
            src = reinterpret_cast<const uint32_t*>(s3base + job.s3_off + s3_hist_off(job));
        } else {
            if (job.profile < 3) return;
            const uint8_t* fr = fibbase + job.fib_off;
            const uint32_t f = w - kFibModel;
            if (reinterpret_cast<const uint32_t*>(fr)[f] == 0) return;
            src = reinterpret_cast<const uint32_t*>(fr + kFibHistOff) + f * 256;
        }
    }
    for (uint32_t s = lane; s < 256; s += 32) s_cnt[w][s] = src[s];
    __syncwarp();
    warp_normalize_frequencies(s_cnt[w], s_freq[w], lane);
    warp_build_table(s_freq[w], tabs + (uint64_t)gw * 256, infos + gw, lane);
}

// ---------------------------------------------------------------------------
// 4-lane interleaved rANS: one thread per lane.
//
// Encoder of core/literals/literals.go:289-341 / przm_ans.cu:270-313 and of
// core/commands/vans_meta.go:104-138: lane = i & 3 of symbol i, symbols
// consumed from the end, x starts at 65536, bytes leave from the low end
// while x >= 4096*f, then x = (x/f)*4096 + c + x%f.  The reference writes all
// lanes' bytes into one stream in processing order and reverses it; here each
// lane writes its own bytes in order together with 2-bit counts per round,
// and the stitch below interleaves them into exactly that reversed stream.
// The division is a multiply-high by a per-symbol reciprocal (exact for
// x < 2^24, see EncSym).
// ---------------------------------------------------------------------------
struct LaneIO {
    uint8_t* bytes;     // lane byte stream
    uint32_t* nbw;      // 2-bit emitted-byte counts, 16 rounds per word (round j -> word j/16)
    uint32_t* cum;      // cum[k]: bytes of rounds >= kStitchRounds k (written where the lane has round kStitchRounds k)
};

__device__ __forceinline__ LaneIO lane_io(uint8_t* task_base, uint32_t cap, uint32_t l) {
    LaneIO io;
    io.bytes = task_base + (uint64_t)l * ans_lane_cap(cap);
    io.nbw = reinterpret_cast<uint32_t*>(task_base + 4 * ans_lane_cap(cap)) + (uint64_t)l * ans_nbw_cap(cap);
    io.cum = io.nbw + ans_nbw_words(cap);
    return io;
}

// One rANS step (table entry e of the symbol already in registers): returns
// the number k of low bytes of x the reference would emit (x >= 4096 f, and
// again when x >= 2^20 f), and advances x.  The caller keeps the low 16 bits
// of x from before the step; its first k bytes (low byte first) are what the
// reference writes.  x < 2^24 throughout, so x >= t2 can only hold for f < 16.
// The renormalised state is selected first and divided once: computing the
// three candidates (0, 1 or 2 bytes shifted out) side by side and selecting
// last keeps the compares off the multiply's chain, but its extra
// instructions made the kernel slower (7.68 vs 7.45 ms on the 256 x 1 MiB
// mixed batch).
__device__ __forceinline__ uint32_t rans_next(uint32_t x, const EncSym& e) {
    const uint32_t s = e.w >> 25, cf = (e.w >> 13) & 0xFFFu, cb = e.w & 0x1FFFu;
    const uint32_t xs = x >= e.t2 ? (x >> 16) : (x >= e.t1 ? (x >> 8) : x);
    return xs + cb + (__umulhi(xs, e.m) >> s) * cf;
}
__device__ __forceinline__ uint32_t rans_step(uint32_t& x, const EncSym& e) {
    const uint32_t k = (uint32_t)(x >= e.t1) + (uint32_t)(x >= e.t2);
    x = rans_next(x, e);
    return k;
}

// Table index of round r of a 16-round group (words w, group g, lane l).
template <bool kMeta8>
__device__ __forceinline__ uint32_t group_index(const uint32_t* w, uint32_t below, int r, int32_t g, uint32_t l,
                                                uint32_t sel, uint32_t selp, const uint8_t* ctxlut) {
    uint32_t ti = __byte_perm(w[r], 0, sel);
    if (kMeta8) {
        uint32_t prev;
        if (l > 0) prev = __byte_perm(w[r], 0, selp);
        else prev = r > 0 ? (w[r - 1] >> 24) : (below >> 24);
        const bool first = (g == 0 && r == 0 && l == 0);
        ti |= (first ? 0u : (uint32_t)ctxlut[prev]) << 8;
    }
    return ti;
}

__device__ __forceinline__ void words16(const uint4* c, uint32_t* w) {
#pragma unroll
    for (int v = 0; v < 4; v++) { w[4 * v] = c[v].x; w[4 * v + 1] = c[v].y; w[4 * v + 2] = c[v].z; w[4 * v + 3] = c[v].w; }
}

// The 16 chain steps of one full group with the entries already in
// registers; writes the group's records and its 2-bit count word.
__device__ __forceinline__ void encode_group(uint32_t& x, uint32_t& cnt, const EncSym* e, int32_t g, uint4* r4,
                                             uint32_t* nbw) {
    uint32_t rec[16], m1 = 0, m2 = 0;
#pragma unroll
    for (int r = 15; r >= 0; r--) {
        rec[r] = x & 0xFFFFu;
        m1 |= x >= e[r].t1 ? (1u << r) : 0u;
        m2 |= x >= e[r].t2 ? (1u << r) : 0u;
        x = rans_next(x, e[r]);
    }
    // k = p1 + p2 with p2 => p1: bit 0 = p1 ^ p2, bit 1 = p2
    nbw[g] = spread16(m1 ^ m2) | (spread16(m2) << 1);
    cnt += __popc(m1) + __popc(m2);
    r4[2 * g] = make_uint4(rec[0] | (rec[1] << 16), rec[2] | (rec[3] << 16), rec[4] | (rec[5] << 16),
                           rec[6] | (rec[7] << 16));
    r4[2 * g + 1] = make_uint4(rec[8] | (rec[9] << 16), rec[10] | (rec[11] << 16), rec[12] | (rec[13] << 16),
                               rec[14] | (rec[15] << 16));
}

// ---- per-lane symbol ring: cp.async copies of the 64-byte groups ---------
// Each thread owns kRing slots of 64 bytes in its warp's ring; chunk v of
// slot q of lane t sits at uint4 index (q * 4 + v) * 32 + t, so the 32 lanes
// of one access touch 32 consecutive 16-byte words (no bank conflicts).
constexpr int kRing = 4;                                              // groups in flight per lane
constexpr uint32_t kRingBytesPerWarp = kRing * 4 * 32 * sizeof(uint4);  // 8 KiB

__device__ __forceinline__ void ring_fetch(uint4* ring, uint32_t t, int32_t slot, const uint4* s4, int32_t g) {
#pragma unroll
    for (int v = 0; v < 4; v++) {
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(ring + (((slot & (kRing - 1)) * 4 + v) << 5) + t);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(s4 + 4 * g + v) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void ring_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void ring_read(const uint4* ring, uint32_t t, int32_t slot, uint4* w) {
#pragma unroll
    for (int v = 0; v < 4; v++) w[v] = ring[(((slot & (kRing - 1)) * 4 + v) << 5) + t];
}

// Encodes lane l of one task.  Symbols of lane l are i = 4j + l, rounds j
// from the top down.  Per round the lane stores the 16 low bits of x before
// the step at raw[j] and the byte count k in 2 bits of nbw[j / 16]; the
// stitch turns (raw, k) back into the reference byte order.  Rounds come in
// groups of 16 (the 64 source bytes 64g .. 64g + 63 hold the four lanes'
// symbols); the rounds above the G = n / 64 full groups take the byte path.
// Full groups stream through the thread's ring: the 64 bytes of group g - 4
// are requested (cp.async, no register waits on them) while group g is
// encoded, the words of group g - 1 are read from the ring one group ahead,
// and the 16 table entries of group g are fetched before its chain runs.
template <bool kMeta8>
__device__ __forceinline__ void rans_lane(const uint8_t* __restrict__ src, uint32_t n, uint32_t l,
                                          const EncSym* __restrict__ tab, const uint8_t* __restrict__ ctxlut,
                                          uint4* ring, LaneIO io, uint32_t* out_state, uint32_t* out_count) {
    uint32_t x = 65536, cnt = 0;
    uint16_t* raw = reinterpret_cast<uint16_t*>(io.bytes);
    const uint32_t t = threadIdx.x & 31;
    if (n > l) {
        const uint32_t J = (n - 1 - l) >> 2;
        const bool vec = (reinterpret_cast<uintptr_t>(src) & 15) == 0;
        const int32_t G = vec ? (int32_t)(n >> 6) : 0;
        {
            uint32_t acc = 0;
            for (int32_t j = (int32_t)J; j >= 16 * G; j--) {
                const uint32_t i = 4u * (uint32_t)j + l;
                uint32_t ti = src[i];
                if (kMeta8) ti |= (i ? (uint32_t)ctxlut[src[i - 1]] : 0u) << 8;
                raw[j] = (uint16_t)x;
                const uint32_t k = rans_step(x, tab[ti]);
                cnt += k;
                acc |= k << (2 * (j & 15));
                if ((j & 15) == 0) {
                    io.nbw[j >> 4] = acc;
                    acc = 0;
                }
                if ((j & (kStitchRounds - 1)) == 0) io.cum[j / kStitchRounds] = cnt;
            }
        }
        if (G > 0) {
            const uint4* s4 = reinterpret_cast<const uint4*>(src);
            uint4* r4 = reinterpret_cast<uint4*>(raw);
            const uint32_t sel = 0x4440u | l;               // __byte_perm selector of byte l
            const uint32_t selp = 0x4440u | ((l + 3) & 3);  // byte l-1 (used for l >= 1)
            // prologue: groups G-1 .. G-kRing (clamped at 0), one commit group each
#pragma unroll
            for (int d = 0; d < kRing; d++) ring_fetch(ring, t, G - 1 - d, s4, max(G - 1 - d, 0));
            ring_wait<kRing - 1>();
            uint4 cur[4];
            ring_read(ring, t, G - 1, cur);
            for (int32_t g = G - 1; g >= 0; g--) {
                ring_wait<kRing - 2>();  // group g - 1 has landed
                uint4 nxt[4];
                ring_read(ring, t, g - 1, nxt);
                EncSym e[16];
                {
                    uint32_t w[16];
                    words16(cur, w);
                    const uint32_t below = g > 0 ? nxt[3].w : 0u;
#pragma unroll
                    for (int r = 15; r >= 0; r--) e[r] = tab[group_index<kMeta8>(w, below, r, g, l, sel, selp, ctxlut)];
                }
                // the slot of group g is free once its words are in registers
                ring_fetch(ring, t, g, s4, max(g - kRing, 0));
                encode_group(x, cnt, e, g, r4, io.nbw);
                if ((g & (kStitchRounds / 16 - 1)) == 0) io.cum[g / (kStitchRounds / 16)] = cnt;
#pragma unroll
                for (int v = 0; v < 4; v++) cur[v] = nxt[v];
            }
            ring_wait<0>();
        }
    }
    *out_state = x;
    *out_count = cnt;
}

// Meta8 static model (core/commands/vans_meta_tables.go) in EncSym form,
// 8 x 256 entries, and the context classifier ContextMeta
// (core/commands/vans_meta.go:46-69) as a 256-entry table; built on the host.
inline void build_meta8_tables(EncSym* tab, uint8_t* ctxlut) {
    for (int c = 0; c < 8; c++) {
        uint32_t cum = 0;
        for (int s = 0; s < 256; s++) {
            tab[c * 256 + s] = make_encsym(przm_meta8_freq[c][s], cum);
            cum += przm_meta8_freq[c][s];
        }
    }
    for (int p = 0; p < 256; p++)
        ctxlut[p] = p == 0 ? 0 : p < 4 ? 1 : p < 16 ? 2 : p < 32 ? 3 : p < 64 ? 4 : p < 128 ? 5 : p < 192 ? 6 : 7;
}

// Task eligibility for the entropy-coded frame (packSubstream,
// core/commands/commands.go:371-406; PackageLiteralsSection selection; the
// adaptive container of the distance codes for 64 codes or more,
// PackDistancePrefix, core/distance/distance.go:692-748; every non-empty
// sheaf fiber, tryEncodeFiber, core/literals/literals.go:633-643).  nd: the
// frame's distances for the codes' task (s3_task_nd); fl: its 16 fiber
// lengths (P3), else null.
__host__ __device__ inline bool task_is_m8(int t) { return t == T_OP_M8 || t == T_META_M8 || t == T_VAR_M8; }
__host__ __device__ inline uint32_t task_len(const uint32_t* lens, int t, uint32_t nd = 0, const uint32_t* fl = nullptr) {
    if (t >= T_FIB) return fl ? fl[t - T_FIB] : 0u;
    return t == T_LIT ? lens[S_LIT] : t == T_S3 ? nd : lens[S_OP + (t - 1) / 2];
}
__host__ __device__ inline bool task_active(const Job& job, const uint32_t* lens, int t, uint32_t nd = 0,
                                            const uint32_t* fl = nullptr) {
    if (job.profile == 0) return false;
    const uint32_t n = task_len(lens, t, nd, fl);
    if (t >= T_FIB) return job.profile >= 3 && n >= 1;
    if (t == T_S3) return job.profile >= 2 && n >= 64 && n <= kS3Scratch;
    if (t == T_LIT) return n >= 1 && n <= (8u << 20);
    if (lens[S_CMD] > (2u << 20)) return false;
    return n <= (2u << 20) && n >= (task_is_m8(t) ? 24u : 16u);
}
// The per-frame facts a task needs, from device memory.
__device__ __forceinline__ uint32_t task_nd(const Job& job, const S3Frame* s3f, uint32_t j, int t) {
    return t == T_S3 && job.profile >= 2 ? s3_task_nd(s3f[j]) : 0u;
}
__device__ __forceinline__ const uint32_t* task_fl(const Job& job, const uint8_t* fibbase) {
    return job.profile >= 3 ? reinterpret_cast<const uint32_t*>(fibbase + job.fib_off) : nullptr;
}

// Where a task's symbols are, how many, its scratch layout's capacity and
// its scratch offset in the job's ANS region.
struct TaskView {
    const uint8_t* src;
    uint64_t ans_off;
    uint32_t n, cap;
};
__device__ __forceinline__ TaskView task_view(const Job& job, const uint32_t* lens, const uint8_t* streams,
                                              const uint8_t* s3base, const uint8_t* fibbase, uint32_t nd,
                                              const uint32_t* fl, int t) {
    TaskView v;
    v.n = task_len(lens, t, nd, fl);
    if (t >= T_FIB) {
        const FibGeom g = fib_geom(job, fl, (uint32_t)(t - T_FIB) >> 2, (uint32_t)(t - T_FIB) & 3u);
        v.src = fibbase + job.fib_off + g.byte_off;
        v.ans_off = g.ans_off;
        v.cap = g.n;
    } else {
        v.src = t == T_S3 ? s3base + job.s3_off
                          : streams + job.str_off + stream_base(job, t == T_LIT ? S_LIT : S_OP + (t - 1) / 2);
        v.ans_off = ans_task_off(job, t);
        v.cap = task_cap(job, t);
    }
    return v;
}
__device__ __forceinline__ uint32_t task_model(int t) {
    return t == T_LIT ? 0u : t == T_S3 ? 4u : t >= T_FIB ? (uint32_t)(kFibModel + t - T_FIB) : 1u + (uint32_t)(t - 1) / 2;
}

// One rANS task as the rANS kernel takes it, resolved by the task list.
struct __align__(16) TaskDesc {
    const uint8_t* src;  // the symbols
    uint8_t* base;       // the task's rANS scratch
    uint32_t n, cap;     // symbols; the scratch layout's capacity
    uint32_t out;        // TaskOut index: frame * T_COUNT + task
    uint32_t tab;        // adaptive model row: frame * kModels + model
};

// Task list: every active (frame, task) pair, split by model kind and
// ordered longest-first (by the bit length of the symbol count) so that the
// 8 tasks sharing a warp have similar lengths and the long chains start
// first; each entry is the task's resolved descriptor.  One block.
__global__ void __launch_bounds__(1024) k_task_list(const Job* __restrict__ jobs, uint32_t j0, uint32_t njobs,
                                                    const uint32_t* __restrict__ job_lens,
                                                    const S3Frame* __restrict__ s3f, const uint8_t* __restrict__ streams,
                                                    const uint8_t* __restrict__ s3base, const uint8_t* __restrict__ fibbase,
                                                    uint8_t* __restrict__ ans, TaskDesc* __restrict__ lists,
                                                    uint32_t list_cap, uint32_t* __restrict__ counts) {
    __shared__ uint32_t s_cnt[2][33];
    __shared__ uint32_t s_pos[2][33];
    const uint32_t tid = threadIdx.x;
    if (tid < 66) (&s_cnt[0][0])[tid] = 0;
    __syncthreads();
    const uint32_t total = njobs * T_COUNT;
    for (uint32_t e = tid; e < total; e += blockDim.x) {
        const uint32_t j = j0 + e / T_COUNT;
        const int t = (int)(e % T_COUNT);
        const uint32_t* lens = job_lens + (uint64_t)j * S_COUNT;
        const Job job = jobs[j];
        const uint32_t nd = task_nd(job, s3f, j, t);
        const uint32_t* fl = task_fl(job, fibbase);
        if (!task_active(job, lens, t, nd, fl)) continue;
        const uint32_t kind = task_is_m8(t) ? 1u : 0u;
        atomicAdd(&s_cnt[kind][32 - __clz(task_len(lens, t, nd, fl))], 1u);
    }
    __syncthreads();
    if (tid < 2) {
        uint32_t a = 0;
        for (int b = 32; b >= 0; b--) { s_pos[tid][b] = a; a += s_cnt[tid][b]; }
        counts[tid] = a;
    }
    __syncthreads();
    for (uint32_t e = tid; e < total; e += blockDim.x) {
        const uint32_t j = j0 + e / T_COUNT;
        const int t = (int)(e % T_COUNT);
        const uint32_t* lens = job_lens + (uint64_t)j * S_COUNT;
        const Job job = jobs[j];
        const uint32_t nd = task_nd(job, s3f, j, t);
        const uint32_t* fl = task_fl(job, fibbase);
        if (!task_active(job, lens, t, nd, fl)) continue;
        const uint32_t kind = task_is_m8(t) ? 1u : 0u;
        const uint32_t p = atomicAdd(&s_pos[kind][32 - __clz(task_len(lens, t, nd, fl))], 1u);
        const TaskView v = task_view(job, lens, streams, s3base, fibbase, nd, fl, t);
        TaskDesc d;
        d.src = v.src;
        d.base = ans + job.ans_off + v.ans_off;
        d.n = v.n;
        d.cap = v.cap;
        d.out = j * T_COUNT + (uint32_t)t;
        d.tab = j * kModels + task_model(t);
        lists[kind * list_cap + p] = d;
    }
}

// One warp per block: the chains are latency-bound and every lane's 16
// table loads per group go through the SM's shared-memory pipe, so warps
// that share an SM slow each other down; with one warp per block the block
// scheduler spreads the (longest-first) warps over distinct SMs.
constexpr int kRansWarps = 1;
constexpr uint32_t kRansTabBytes = 8 * 256 * sizeof(EncSym);          // 8 models per warp (32 KiB)
constexpr uint32_t kRansSmem = kRansWarps * (kRansTabBytes + kRingBytesPerWarp);  // tables, rings

// Blocks [0, nb_ad) run adaptive-model tasks, the rest Meta8 tasks; each
// warp takes 8 consecutive tasks of its list (4 lanes per task).
__global__ void __launch_bounds__(kRansWarps * 32) k_rans(const TaskDesc* __restrict__ lists, uint32_t list_cap,
                                                          const uint32_t* __restrict__ counts, uint32_t nb_ad,
                                                          const EncSym* __restrict__ tabs,
                                                          const EncSym* __restrict__ meta8,
                                                          const uint8_t* __restrict__ ctxlut, TaskOut* __restrict__ outs) {
    extern __shared__ __align__(16) uint8_t smem_r[];
    __shared__ uint8_t s_lut[256];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool m8 = blockIdx.x >= nb_ad;
    const uint32_t nlist = counts[m8 ? 1 : 0];
    const TaskDesc* dl = lists + (m8 ? list_cap : 0);
    const uint32_t wg = (m8 ? blockIdx.x - nb_ad : blockIdx.x) * kRansWarps + warp;  // warp index in its list
    EncSym* wtab = reinterpret_cast<EncSym*>(smem_r + warp * kRansTabBytes);
    uint4* wring = reinterpret_cast<uint4*>(smem_r + kRansWarps * kRansTabBytes + warp * kRingBytesPerWarp);
    if (m8) {
        // the block shares the 8 static models; every warp holds a copy
        for (uint32_t i = lane; i < 8 * 256; i += 32) wtab[i] = meta8[i];
        if (warp == 0) for (uint32_t i = lane; i < 256; i += 32) s_lut[i] = ctxlut[i];
    } else {
        // this warp's 8 adaptive tables
        for (uint32_t k = 0; k < 8; k++) {
            const uint32_t tk = wg * 8 + k;
            if (tk >= nlist) break;
            const EncSym* src = tabs + (uint64_t)dl[tk].tab * 256;
            for (uint32_t i = lane; i < 256; i += 32) wtab[k * 256 + i] = src[i];
        }
    }
    const uint32_t slot = lane >> 2, l = lane & 3;
    const uint32_t ti = wg * 8 + slot;
    __syncthreads();
    if (ti >= nlist) return;
    const TaskDesc d = dl[ti];
    LaneIO io = lane_io(d.base, d.cap, l);
    TaskOut* o = outs + d.out;
    if (m8) rans_lane<true>(d.src, d.n, l, wtab, s_lut, wring, io, &o->state[l], &o->count[l]);
    else rans_lane<false>(d.src, d.n, l, wtab + slot * 256, nullptr, wring, io, &o->state[l], &o->count[l]);
}

// ---------------------------------------------------------------------------
// Stitch: write the reference byte order of a 4-lane rANS stream, i.e. the
// reversal of the interleaved emission sequence (the reference emits round
// j's bytes lane 3 first, rounds from the top down, then reverses).  For
// rounds j = 0, 1, ... and lanes l = 0..3 it places the k(l, j) bytes of
// raw[l][j], second-emitted byte first.  Rounds are taken 16 per thread per
// pass; one block-wide exclusive scan of the per-thread byte counts gives
// every thread its output position.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t sum2(uint32_t w) {  // sum of the 16 2-bit fields
    w = (w & 0x33333333u) + ((w >> 2) & 0x33333333u);
    w = (w + (w >> 4)) & 0x0F0F0F0Fu;
    return (w * 0x01010101u) >> 24;
}

template <int NT>
__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_warp, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t t = lane < NT / 32 ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= (uint32_t)o) t += y;
        }
        s_warp[lane] = t;  // inclusive warp prefix
    }
    __syncthreads();
    total = s_warp[NT / 32 - 1];
    const uint32_t base = warp ? s_warp[warp - 1] : 0;
    __syncthreads();
    return base + x - v;
}

// Byte r (0..15) of the 16 u16 records held in two uint4.
__device__ __forceinline__ uint32_t rec16(const uint4* v, int r) {
    const uint4 q = v[r >> 3];
    const uint32_t w = ((r >> 1) & 3) == 0 ? q.x : ((r >> 1) & 3) == 1 ? q.y : ((r >> 1) & 3) == 2 ? q.z : q.w;
    return (r & 1) ? (w >> 16) : (w & 0xFFFFu);
}

// Bytes a stitch pass of NT threads x 16 rounds can produce (8 per round).
template <int NT>
struct StitchStage {
    static constexpr uint32_t kBytes = NT * 16 * 8 + 16;
};

// One stitch pass: thread t takes rounds [r0 + 16t, r0 + 16t + 16) of the
// four lanes (two 16-byte loads of records and one count word per lane), one
// block scan gives its byte offset, it writes its bytes into a shared staging
// buffer placed at the output's 16-byte phase, and the block then stores the
// staged run at dst with aligned 16-byte stores (byte stores only for the
// partial first and last 16 bytes of the run).  Returns the run's length.
template <int NT>
__device__ uint32_t stitch_pass(const uint8_t* task_base, uint32_t cap, uint32_t n, uint32_t r0, uint8_t* __restrict__ dst) {
    __shared__ uint32_t s_warp[32];
    __shared__ __align__(16) uint8_t s_stage[StitchStage<NT>::kBytes];
    const uint32_t tid = threadIdx.x;
    const uint32_t rounds = (n + 3) / 4;
    const uint32_t rb = r0 + 16 * tid;  // first round of this thread (multiple of 16)
    uint32_t w[4] = {0, 0, 0, 0}, c = 0;
    uint4 rv[4][2];
#pragma unroll
    for (uint32_t l = 0; l < 4; l++) {
        rv[l][0] = rv[l][1] = make_uint4(0, 0, 0, 0);
        if (rb >= rounds || n <= l) continue;
        const uint32_t jmax = (n - 1 - l) / 4;
        if (rb > jmax) continue;
        const uint16_t* raw = reinterpret_cast<const uint16_t*>(task_base + (uint64_t)l * ans_lane_cap(cap));
        const uint32_t* nw = reinterpret_cast<const uint32_t*>(task_base + 4 * ans_lane_cap(cap)) + (uint64_t)l * ans_nbw_cap(cap);
        uint32_t v = nw[rb >> 4];
        const uint32_t top = jmax - rb;  // rounds of this word the lane has
        if (top < 15) v &= (1u << (2 * (top + 1))) - 1u;
        w[l] = v;
        c += sum2(v);
        // rounds past jmax are in the lane region (it holds ceil(cap/4) + 64 records) and masked by w
        const uint4* rp = reinterpret_cast<const uint4*>(raw + rb);
        rv[l][0] = rp[0];
        rv[l][1] = rp[1];
    }
    uint32_t total;
    const uint32_t excl = block_exclusive_scan<NT>(c, s_warp, total);
    const uint32_t a = (uint32_t)(reinterpret_cast<uintptr_t>(dst) & 15);
    uint32_t q = a + excl;
#pragma unroll
    for (int r = 0; r < 16; r++) {
#pragma unroll
        for (int l = 0; l < 4; l++) {
            const uint32_t k = (w[l] >> (2 * r)) & 3u;
            if (!k) continue;
            const uint32_t v = rec16(rv[l], r);
            if (k == 2) {
                s_stage[q] = (uint8_t)(v >> 8);
                s_stage[q + 1] = (uint8_t)v;
                q += 2;
            } else {
                s_stage[q] = (uint8_t)v;
                q += 1;
            }
        }
    }
    __syncthreads();
    uint8_t* g0 = dst - a;  // 16-byte aligned; only bytes [a, a + total) are written
    const uint32_t end = a + total, nch = (end + 15) / 16;
    for (uint32_t ch = tid; ch < nch; ch += NT) {
        const uint32_t lo = ch * 16, hi = lo + 16;
        if (lo >= a && hi <= end) {
            *reinterpret_cast<uint4*>(g0 + lo) = *reinterpret_cast<const uint4*>(s_stage + lo);
        } else {
            for (uint32_t b = lo > a ? lo : a; b < (hi < end ? hi : end); b++) g0[b] = s_stage[b];
        }
    }
    __syncthreads();  // the staging buffer is reused by the next pass
    return total;
}

// The whole stream, pass after pass, by one block.
template <int NT>
__device__ void block_stitch(const uint8_t* task_base, uint32_t cap, uint32_t n, uint8_t* __restrict__ out) {
    const uint32_t rounds = (n + 3) / 4;
    uint32_t carry = 0;
    for (uint32_t r0 = 0; r0 < rounds; r0 += 16 * NT) carry += stitch_pass<NT>(task_base, cap, n, r0, out + carry);
}

// Output offset of the stitch pass starting at round r0 (a multiple of
// kStitchRounds): the bytes of all rounds below r0, from each lane's total
// and its recorded count of the rounds from r0 up.
__device__ __forceinline__ uint32_t stitch_offset(const uint8_t* task_base, uint32_t cap, uint32_t n, const TaskOut& o,
                                                  uint32_t r0) {
    uint32_t off = 0;
#pragma unroll
    for (uint32_t l = 0; l < 4; l++) {
        if (n <= l) continue;
        const uint32_t jmax = (n - 1 - l) / 4;
        const uint32_t* cum = reinterpret_cast<const uint32_t*>(task_base + 4 * ans_lane_cap(cap)) +
                              (uint64_t)l * ans_nbw_cap(cap) + ans_nbw_words(cap);
        off += o.count[l] - (r0 <= jmax ? cum[r0 / kStitchRounds] : 0u);
    }
    return off;
}

}  // namespace pz
