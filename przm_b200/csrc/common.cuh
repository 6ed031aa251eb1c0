// common.cuh -- shared constants, job descriptors and device helpers of the
// PRZM B200 compression path.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pz {

// ---- format constants (reference: gpu/kernel/przm_lz77.h:21-38,
//      przm_lz77.cu:24-33, przm_ans.h:22-36, gpu/bridge.go:148-153) ----------
constexpr uint32_t kTile = 32768;            // finder and tokenizer tile
constexpr uint32_t kBuckets = 2048;          // tile-finder hash buckets
constexpr uint32_t kHashPrime = 0x1E35A7BDu; // przm_gpu_hash4
constexpr uint32_t kRadixBuckets = 524288;   // radix-strike table (2^19)
constexpr uint64_t kRadixPrime = 0x9E3779B97F4A7C15ull;
constexpr uint32_t kWindow = 1u << 20;       // Window1M passed by the bridge
constexpr uint32_t kMaxLen32 = 4095;
constexpr uint32_t kMaxOff32 = 1048575;
constexpr uint32_t kSmallMax = 65536;        // n <= 64 KiB -> tile finder
constexpr uint32_t kCandPerTile = kTile / 8; // radix candidates per tile

// Per-tile output slots of the tokenizer.  Bounds: every command token covers
// >= 4 input bytes per command byte (literal flush + token included), so a
// tile emits <= 8192 + 4 command bytes; offsets are <= 3 bytes per >= 4-byte
// explicit match; literals never exceed the tile.  Writes are checked against
// these sizes on the device.
constexpr uint32_t kSlotCmd = 8704;
constexpr uint32_t kSlotOff = 24832;
constexpr uint32_t kSlotLit = 33024;

enum Stream : int { S_CMD = 0, S_OP = 1, S_META = 2, S_VAR = 3, S_OFF = 4, S_LIT = 5, S_COUNT = 6 };

// ANS task slots per job: literal stream (adaptive), the three command
// substreams, each with the Meta8 and the adaptive model, (P2 frames and
// up) the adaptive container of the Section 3 distance codes, and (P3) the
// sixteen sheaf fibers, T_FIB + 4 mode + fiber.
enum Task : int {
    T_LIT = 0, T_OP_M8 = 1, T_OP_AD = 2, T_META_M8 = 3, T_META_AD = 4, T_VAR_M8 = 5, T_VAR_AD = 6, T_S3 = 7,
    T_FIB = 8, T_COUNT = 24
};
// adaptive models per job (tables and serialized matrices): literals, op,
// meta, var, distance codes, then the fibers (model 5 + 4 mode + fiber)
constexpr int kModels = 21;
constexpr int kFibModel = 5;

// error bits reported through the per-batch status word
enum Err : uint32_t { E_SLOT_OVERFLOW = 1, E_STREAM_OVERFLOW = 2, E_BAD_TOKEN = 4, E_TABLE = 8, E_COPY_TIMEOUT = 32 };

// ---- bulk copies (the TMA engine's one-dimensional form) into this CTA's
// shared memory, completed on an mbarrier.  Source and destination 16-byte
// aligned, size a multiple of 16.  No multicast.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(m)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* m) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(m)) : "memory");
}
// expect `bytes` and start one bulk copy global -> shared that completes them
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* m) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for phase `parity`: false (and E_COPY_TIMEOUT in *err) when
// the copy has not completed after 2^22 polls, far beyond a tile's copy time.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* m, uint32_t parity, uint32_t* err) {
    for (uint32_t it = 0; it < (1u << 22); it++)
        if (mbar_try_wait(m, parity)) return true;
    atomicOr(err, (uint32_t)E_COPY_TIMEOUT);
    return false;
}

// Load of data an earlier stage wrote.  When that stage ran in an earlier
// launch the data is read-only for this one and goes through the read-only
// path (kCoherent = false); inside the persistent front end the producing
// stage may have run in the same launch, on another SM, so the load goes to
// L2 (ld.global.cg), where the producer's writes are.
template <bool kCoherent, class T>
__device__ __forceinline__ T ld_stage(const T* p) {
    if constexpr (kCoherent) return __ldcg(p);
    else return __ldg(p);
}

struct Job {
    uint64_t in_off;    // input byte offset (16-byte aligned)
    uint64_t desc_off;  // u32 index of this job's descriptor table
    uint64_t str_off;   // byte offset of this job's stream region
    uint64_t ans_off;   // byte offset of this job's ANS scratch region
    uint64_t out_off;   // byte offset of this job's frame
    uint32_t n;         // input bytes
    uint32_t tile0;     // first global tile index
    uint32_t ntiles;
    uint32_t kind;      // 0: tile finder (n <= 64 KiB), 1: radix strike
    uint32_t cmd_cap;   // capacity of cmd/op/meta/var streams
    uint32_t off_cap;   // capacity of the offset stream
    uint32_t lit_cap;   // capacity of the literal stream
    uint32_t profile;   // 0: CompressD2D frame (P0), 1: entropy-coded frame (P1), 2: P1 with coded Section 3 (P2)
    uint32_t out_cap;
    uint32_t dist_cap;  // distances a P2 frame can hold (n / 4 + 64: every match covers >= 4 bytes); 0 below P2
    uint64_t s3_off;    // byte offset of this job's Section 3 region (P2 and up)
    uint64_t fib_off;   // byte offset of this job's fiber region (P3)
};

// A P2 job's Section 3 region: the distance codes (dist_cap + 16 bytes),
// the MSB-first extra-bit stream (3 bytes per distance + 16: at most 18
// extra bits for distances below 2^20, so at most four bytes are touched
// per distance), the Mode 12 bytes in emission order (2 per code at most,
// capped at the reference's 2 MiB scratch, + 16), and the codes' histogram
// (256 u32).
constexpr uint32_t kS3Scratch = 2u * 1024 * 1024;  // the reference's 2 MiB distance scratch buffers
__host__ __device__ inline uint64_t s3_extra_off(const Job& j) { return (j.dist_cap + 16ull + 15) & ~15ull; }
__host__ __device__ inline uint64_t s3_em_off(const Job& j) { return s3_extra_off(j) + ((3ull * j.dist_cap + 16 + 15) & ~15ull); }
__host__ __device__ inline uint64_t s3_em_cap(const Job& j) {
    return 2ull * j.dist_cap < kS3Scratch ? 2ull * j.dist_cap : (uint64_t)kS3Scratch;
}
__host__ __device__ inline uint64_t s3_hist_off(const Job& j) { return s3_em_off(j) + ((s3_em_cap(j) + 16 + 15) & ~15ull); }
__host__ __device__ inline uint64_t s3_region_bytes(const Job& j) { return s3_hist_off(j) + 256 * 4; }

// Per-frame Section 3 facts from k_s3_frame and k_s3_chain.
struct S3Frame {
    uint32_t nd;     // distances
    uint32_t bits;   // their extra bits
    uint32_t bad;    // a distance of 0 or above 2^24 (the reference's ErrOffsetOOB)
    uint32_t orig;   // bytes of their LEB128 varints
    uint32_t m12e;   // Mode 12 bytes emitted; 0xFFFFFFFF past the 2 MiB scratch
    uint32_t m12x;   // Mode 12 final state
    uint32_t pad[2];
};
// distances the codes' adaptive task codes (0: no task)
__host__ __device__ inline uint32_t s3_task_nd(const S3Frame& f) { return f.bad ? 0u : f.nd; }

// byte offsets of the six streams inside a job's stream region
__host__ __device__ inline uint64_t stream_base(const Job& j, int s) {
    const uint64_t c = j.cmd_cap, o = j.off_cap;
    switch (s) {
        case S_CMD: return 0;
        case S_OP: return c;
        case S_META: return 2 * c;
        case S_VAR: return 3 * c;
        case S_OFF: return 4 * c;
        default: return 4 * c + o;
    }
}
__host__ __device__ inline uint64_t stream_region_bytes(const Job& j) {
    return 4ull * j.cmd_cap + j.off_cap + j.lit_cap;
}

// ANS scratch of one task: four lane byte streams, then per lane its count
// words (2 bits per round) followed by its running byte count at every
// kStitchRounds-th round (the bytes of rounds >= 4096 k, k = 0, 1, ...), from
// which a stitch pass finds its output offset without the passes before it.
// L = symbol capacity of the task's stream.  Lane streams are written in
// 64-byte chunks (64-byte aligned), so every lane region is a multiple of 64
// with room for the last partial chunk.
constexpr uint32_t kStitchRounds = 4096;  // rounds of one stitch pass (256 threads x 16)
// (constexpr, so that fixed-size scratch can be checked against them at
// compile time)
__host__ __device__ constexpr uint64_t ans_lane_cap(uint32_t L) { return ((2ull * ((L + 3) / 4) + 128) + 63) & ~63ull; }
__host__ __device__ constexpr uint64_t ans_nbw_words(uint32_t L) { return (((L + 3) / 4) + 15) / 16 + 1; }
__host__ __device__ constexpr uint64_t ans_cum_words(uint32_t L) { return ((L + 3) / 4 + kStitchRounds - 1) / kStitchRounds + 1; }
__host__ __device__ constexpr uint64_t ans_nbw_cap(uint32_t L) { return ans_nbw_words(L) + ans_cum_words(L); }  // u32 words
__host__ __device__ constexpr uint64_t ans_task_bytes(uint32_t L) {
    uint64_t b = 4 * ans_lane_cap(L) + 4 * 4 * ans_nbw_cap(L);
    return (b + 63) & ~63ull;
}
__host__ __device__ inline uint32_t task_cap(const Job& j, int t) {
    return t == T_LIT ? j.lit_cap : t == T_S3 ? j.dist_cap : j.cmd_cap;
}
__host__ __device__ inline uint64_t ans_task_off(const Job& j, int t) {
    uint64_t o = 0;
    for (int k = 0; k < t; k++) o += ans_task_bytes(task_cap(j, k));
    return o;
}
// A P3 job's fiber region: the 16 fiber lengths (u32, [mode][fiber]), their
// 16 histograms (256 u32 each), then per mode its four fibers one after
// another, each starting on a 16-byte boundary.  The fiber tasks' rANS
// scratch follows the fixed tasks' in the job's ANS region, one budget per
// mode: the four fibers' task scratch exceeds one task of their total length
// by less than 3 KiB (per-lane rounding), so one literal task's bytes plus
// 8 KiB always hold them.
constexpr uint32_t kFibHistOff = 64;
constexpr uint32_t kFibAreaOff = 64 + 16 * 256 * 4;
constexpr uint32_t kFibMax = 8u * 1024 * 1024;  // literals split into fibers: the reference's 8 MiB literal buffers
__host__ __device__ inline uint64_t fib_mode_bytes(const Job& j) { return (j.lit_cap + 64ull + 15) & ~15ull; }
__host__ __device__ inline uint64_t fib_region_bytes(const Job& j) { return kFibAreaOff + 4 * fib_mode_bytes(j); }
__host__ __device__ inline uint64_t fib_mode_ans(const Job& j) { return ans_task_bytes(j.lit_cap) + 8192; }
__host__ __device__ inline uint64_t ans_region_bytes(const Job& j) {
    return ans_task_off(j, T_FIB) + (j.profile >= 3 ? 4 * fib_mode_ans(j) : 0);
}
// Fiber k of mode m: its length (fl: the 16 lengths), its byte offset in the
// fiber region and its rANS scratch offset in the job's ANS region.
struct FibGeom {
    uint32_t n;
    uint64_t byte_off, ans_off;
};
__host__ __device__ inline FibGeom fib_geom(const Job& j, const uint32_t* fl, uint32_t m, uint32_t k) {
    FibGeom g;
    g.byte_off = kFibAreaOff + m * fib_mode_bytes(j);
    g.ans_off = ans_task_off(j, T_FIB) + m * fib_mode_ans(j);
    for (uint32_t q = 0; q < k; q++) {
        g.byte_off += (fl[4 * m + q] + 15ull) & ~15ull;
        g.ans_off += ans_task_bytes(fl[4 * m + q]);
    }
    g.n = fl[4 * m + k];
    return g;
}

// Encoding table entry for one symbol of one model:
//   m   : 32-bit reciprocal so that floor(x_r / f) == umulhi(x_r, m) >> s for
//         every x_r < 2^24 (Granlund-Montgomery 1994, round-up variant);
//         f = 2^t uses m = 2^(32-t), s = 0; f = 1 uses m = 2^32-1 (one short)
//         with the deficit folded into cb.
//   t1  : 4096 * f, the renormalisation bound (x >= t1 -> emit a byte)
//   t2  : 256 * t1 saturated to 2^32-1 (x >= t2 -> emit a second byte)
//   w   : cb | (4096 - f) << 13 | s << 25, cb = cumulative frequency c
//         (+4095 when f == 1)
struct __align__(16) EncSym {
    uint32_t m, t1, t2, w;
};

// Per-task results of the rANS kernel.
struct TaskOut {
    uint32_t state[4];
    uint32_t count[4];  // bytes emitted by each lane
};

// Per-job section plan computed by the selection kernel.
struct Plan {
    uint32_t frame_size;
    uint32_t flags;
    uint32_t l2, l3, l4;      // section sizes
    uint32_t sub_len[3];      // packed op/meta/var substream sizes (Mode 8)
    uint32_t sub_mode[3];     // 0 flat 0x09, 1 Meta8, 2 adaptive
    uint32_t s2_mode;         // 0 flat 0x00 (P0), 1 Mode 8, 2 flat 0x09
    uint32_t s4_mode;         // 0 raw, 1 V-ANS
    uint32_t uncompressed;
    uint32_t wlog;
    // Section 3 of a P2 frame: form 0 flat 0x00 (P0/P1), 1 distance-prefix
    // container, 2 flat 0x09 varints, 3 empty (no distance); code stream 0
    // Mode 12, 1 the adaptive container; header, code stream and extra-bit
    // bytes of the container
    uint32_t s3_form, s3_code, s3_hlen, s3_cl, s3_xl;
    // Section 4 of a P3 frame in sheaf form (s4_mode 2): the foliation and
    // each fiber's bytes in the container (0: empty; == its length: raw)
    uint32_t s4_sheaf, fe[4];
};

struct TableInfo {            // adaptive model of one (job, stream)
    uint32_t mat_len;
    uint32_t active;
    uint8_t mat[600];         // serialized 16x16 joint-nibble matrix (<= 2 + 32 + 512)
};

// ---- device helpers --------------------------------------------------------
__device__ __forceinline__ uint32_t ld32_smem_u(const uint8_t* base, uint32_t i) {
    // unaligned little-endian u32 from a 4-byte aligned shared buffer padded by 8 bytes
    const uint32_t* w = reinterpret_cast<const uint32_t*>(base) + (i >> 2);
    return __funnelshift_r(w[0], w[1], (i & 3) * 8);
}

__device__ __forceinline__ uint64_t ld64_global_u(const uint8_t* p) {
    // unaligned u64 through two aligned loads; buffers are padded by 16 bytes
    uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint64_t* w = reinterpret_cast<const uint64_t*>(a & ~uintptr_t(7));
    uint32_t sh = (uint32_t)(a & 7) * 8;
    uint64_t lo = __ldg(w), hi = __ldg(w + 1);
    return sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
}

__device__ __forceinline__ uint32_t ld32_global_u(const uint8_t* p) { return (uint32_t)ld64_global_u(p); }

__device__ __forceinline__ uint32_t pack_match32(uint32_t len, uint32_t off) {
    if (len < 4 || off == 0) return 0;
    return ((len > kMaxLen32 ? kMaxLen32 : len) << 20) | (off & 0xFFFFFu);
}

// Spreads the 16 bits of v to the even bit positions of a 32-bit word.
__device__ __forceinline__ uint32_t spread16(uint32_t v) {
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

// Spreads the low 8 bits of v to bit positions 0, 4, 8, ..., 28.
__device__ __forceinline__ uint32_t spread8_4(uint32_t v) {
    v &= 0xFFu;
    v = (v | (v << 12)) & 0x000F000Fu;
    v = (v | (v << 6)) & 0x03030303u;
    v = (v | (v << 3)) & 0x11111111u;
    return v;
}

// Lanes of the warp whose key equals this lane's, for keys below 2^kBits
// (all 32 lanes take part): the AND over the key's bits of the ballot of that
// bit, or of its complement where the bit is clear.  __match_any_sync gives
// the same mask in one instruction, but on sm_100 that instruction costs
// about 380 cycles of latency and one issue per ~63 SM cycles, while these
// kBits ballots are independent and cheap.
template <int kBits>
__device__ __forceinline__ uint32_t warp_match(uint32_t key) {
    uint32_t m = 0xFFFFFFFFu;
#pragma unroll
    for (int b = 0; b < kBits; b++) {
        const bool x = ((key >> b) & 1u) != 0;
        const uint32_t bb = __ballot_sync(0xFFFFFFFFu, x);
        m &= x ? bb : ~bb;
    }
    return m;
}

}  // namespace pz
