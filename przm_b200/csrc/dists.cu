// dists.cu -- Section 3 of the P2 frame inside the batch pipeline: the
// frame's distances coded as PackageOffsetsSection
// (core/distance/distance.go:692-849, as the reference's CPU compressor
// writes Section 3, compress.go:956).
//
// The tokenizer already wrote the frame's distances as LEB128 varints (its
// offset stream).  Per frame, on the device:
//   k_s3_frame  one block: decodes the varints (a varint ends at a byte below
//               0x80, so the distance index of a terminator is a block scan
//               of the terminator flags), writes the 49-bracket codes
//               (DistanceToCode :165-180), ORs the extra bits into a zeroed
//               MSB-first stream (BitWriter :204-247) at offsets from a
//               second scan, and counts the codes' histogram;
//   k_s3_chain  one thread per frame: the Mode 12 chain
//               (EncodeDistClusteredVans :323-377), one rANS state over the
//               codes from the last to the first, each coded with the static
//               weights of its predecessor's class; the emitted bytes are
//               kept in emission order and reversed by the assembler;
//   the codes' adaptive V-ANS container (EncodeAdaptiveVANS4x, for 64 codes
//   or more) is one more task of the frame's rANS launch (model 4, task
//   T_S3), and k_plan picks the form from the sizes as PackDistancePrefix /
//   PackageOffsetsSection do, with the reference's 2 MiB scratch limits.
#include "common.cuh"
#include "dist_tables.h"

namespace pz {

constexpr uint32_t kS3Threads = 1024;

// DistanceToCode for 1 <= d <= 2^24 (distance.go:165-180): code, extra bits
// and their count.
__device__ __forceinline__ uint32_t s3_code(uint32_t d, uint32_t& extra, uint32_t& nb) {
    if (d <= 4) {
        extra = 0;
        nb = 0;
        return d - 1;
    }
    const uint32_t u = d - 1;
    const uint32_t b = 32u - __clz(u) - 2u;  // bits.Len32(u) - 2
    const uint32_t half = (u >> b) & 1u;
    nb = b;
    extra = d - (((2u + half) << b) + 1u);
    return 2 * b + 2 + half;
}

__device__ __forceinline__ uint32_t leb_len(uint32_t d) {
    return d <= 0x7Fu ? 1u : d <= 0x3FFFu ? 2u : d <= 0x1FFFFFu ? 3u : d <= 0x0FFFFFFFu ? 4u : 5u;
}

// ContextDist (distance.go:190-202): the class of the previous code.
__host__ __device__ __forceinline__ uint32_t s3_ctx(uint32_t prev) { return prev < 6 ? 0u : prev < 14 ? 1u : prev < 26 ? 2u : 3u; }

// One block per frame of [j0, j0 + gridDim.x): decode the offset stream's
// varints into codes, extra bits and the codes' histogram.  Every thread
// looks at one byte per pass; the thread on a terminator byte (< 0x80)
// decodes the varint that ends there (at most five bytes back).
__global__ void __launch_bounds__(kS3Threads) k_s3_frame(const Job* __restrict__ jobs, uint32_t j0,
                                                         const uint32_t* __restrict__ job_lens,
                                                         const uint8_t* __restrict__ streams, uint8_t* __restrict__ s3base,
                                                         S3Frame* __restrict__ s3f, uint32_t* __restrict__ err) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_hist[256];
    const uint32_t j = j0 + blockIdx.x, tid = threadIdx.x;
    const Job job = jobs[j];
    if (job.profile < 2) return;
    const uint32_t L = job_lens[(uint64_t)j * S_COUNT + S_OFF];
    const uint8_t* off = streams + job.str_off + stream_base(job, S_OFF);
    uint8_t* base = s3base + job.s3_off;
    uint32_t* extra = reinterpret_cast<uint32_t*>(base + s3_extra_off(job));
    const uint32_t dcap = job.dist_cap;
    const uint32_t lim = min(L, dcap);
    for (uint32_t w = tid; w < (3 * lim + 16) / 4; w += kS3Threads) extra[w] = 0;
    if (tid < 256) s_hist[tid] = 0;
    __syncthreads();
    uint32_t nd = 0, bits = 0, flags = 0;  // flags: 1 a bad distance, 2 a malformed varint
    for (uint32_t b0 = 0; b0 < L; b0 += kS3Threads) {  // uniform trip count: every thread scans
        const uint32_t i = b0 + tid;
        const bool term = i < L && off[i] < 0x80u;
        uint32_t code = 0, ex = 0, nb = 0, f = 0;
        if (term) {
            uint32_t st = i;
            while (st > 0 && i - st < 4 && off[st - 1] >= 0x80u) st--;
            if (st > 0 && off[st - 1] >= 0x80u) f |= 2;  // longer than five bytes
            uint32_t d = 0;
            for (uint32_t k = st; k <= i; k++) d |= (uint32_t)(off[k] & 0x7Fu) << (7 * (k - st));
            if (i - st + 1 != leb_len(d)) f |= 2;  // not the minimal encoding
            if (d >= 1 && d <= 16777216u) code = s3_code(d, ex, nb);
            else f |= 1;
        }
        if (i + 1 == L && !term) f |= 2;  // a varint runs past the stream's end
        uint32_t tn, tb;
        const uint32_t di = nd + block_exclusive_scan<kS3Threads>(term ? 1u : 0u, s_warp, tn);
        const uint32_t ob = bits + block_exclusive_scan<kS3Threads>(nb, s_warp, tb);
        if (term) {
            if (di < dcap) {
                base[di] = (uint8_t)code;
                atomicAdd(&s_hist[code], 1u);
                if (nb) {
                    // the nb bits go to stream bits [ob, ob + nb), MSB first: as a
                    // big-endian word starting at byte ob / 8 they span at most
                    // four bytes (nb <= 22, ob % 8 <= 7)
                    const uint32_t W = ex << (32u - nb - (ob & 7u));
#pragma unroll
                    for (uint32_t t = 0; t < 4; t++) {
                        const uint32_t bv = (W >> (24 - 8 * t)) & 0xFFu;
                        if (bv) {
                            const uint32_t k = (ob >> 3) + t;
                            atomicOr(&extra[k >> 2], bv << (8 * (k & 3)));
                        }
                    }
                }
            } else {
                atomicOr(err, (uint32_t)E_STREAM_OVERFLOW);
            }
        }
        nd += tn;
        bits += tb;
        flags |= (uint32_t)__syncthreads_or(f & 1) | ((uint32_t)__syncthreads_or(f & 2) << 1);
    }
    uint32_t* hist = reinterpret_cast<uint32_t*>(base + s3_hist_off(job));
    for (uint32_t s = tid; s < 256; s += kS3Threads) hist[s] = s_hist[s];
    if (tid == 0) {
        if (flags & 2) atomicOr(err, (uint32_t)E_BAD_TOKEN);
        S3Frame fr{};
        fr.nd = nd;
        fr.bits = bits;
        fr.bad = flags & 1;
        fr.orig = L;  // minimal varints: the stream's bytes are their LEB128 bytes
        fr.m12e = 0;
        fr.m12x = 65536;
        s3f[j] = fr;
    }
}

// One Mode 12 step: the code's entry in registers; emits the bytes the
// reference would write (low byte first) into em[e..] and advances x.
// False when they would pass the reference's 2 MiB emission scratch.
__device__ __forceinline__ bool m12_step(uint32_t& x, uint32_t& e, const EncSym& es, uint8_t* __restrict__ em) {
    const uint32_t k = (uint32_t)(x >= es.t1) + (uint32_t)(x >= es.t2);
    if (k) {
        if (e + k > kS3Scratch) return false;
        em[e] = (uint8_t)x;
        if (k == 2) em[e + 1] = (uint8_t)(x >> 8);
        e += k;
    }
    x = rans_next(x, es);
    return true;
}

// The Mode 12 chain over codes[0, nd) (one thread): codes from the last to
// the first, each with the model of its predecessor's class (s_tab: the
// 4 x 64 static weights in EncSym form); the emitted bytes go to em in
// emission order.  Codes are taken eight at a time from aligned words (codes
// 16-byte aligned), so the table entries of a group load before its
// dependent steps run.  False where the reference's 2 MiB emission scratch
// would overflow.
__device__ bool m12_chain(const uint8_t* __restrict__ codes, uint32_t nd, uint8_t* __restrict__ em,
                          const EncSym* s_tab, uint32_t& x, uint32_t& e) {
    x = 65536;
    e = 0;
    bool ok = true;
    const uint32_t full = nd & ~7u;  // codes [0, full) in aligned groups of eight
    for (uint32_t i = nd; i > full && ok;) {
        i--;
        const uint32_t prev = i ? codes[i - 1] : 0u;
        ok = m12_step(x, e, s_tab[s3_ctx(prev) * 64 + codes[i]], em);
    }
    for (int32_t g = (int32_t)(full / 8) - 1; g >= 0 && ok; g--) {
        const uint2 w = *reinterpret_cast<const uint2*>(codes + 8 * g);
        const uint32_t below = g ? codes[8 * g - 1] : 0u;
        uint32_t c[8];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            c[r] = (w.x >> (8 * r)) & 0xFFu;
            c[r + 4] = (w.y >> (8 * r)) & 0xFFu;
        }
        EncSym es[8];
#pragma unroll
        for (int r = 0; r < 8; r++) es[r] = s_tab[s3_ctx(r ? c[r - 1] : below) * 64 + c[r]];
#pragma unroll
        for (int r = 7; r >= 0; r--)
            if (ok) ok = m12_step(x, e, es[r], em);
    }
    return ok;
}

// The Mode 12 chains of frames [j0, j0 + njobs), one thread each.  tab12:
// the 4 x 64 static weights in EncSym form.
__global__ void __launch_bounds__(32) k_s3_chain(const Job* __restrict__ jobs, uint32_t j0, uint32_t njobs,
                                                 uint8_t* __restrict__ s3base, S3Frame* __restrict__ s3f,
                                                 const EncSym* __restrict__ tab12) {
    __shared__ EncSym s_tab[4 * 64];
    for (uint32_t i = threadIdx.x; i < 4 * 64; i += 32) s_tab[i] = tab12[i];
    __syncwarp();
    const uint32_t jl = blockIdx.x * 32 + threadIdx.x;
    if (jl >= njobs) return;
    const uint32_t j = j0 + jl;
    const Job job = jobs[j];
    if (job.profile < 2) return;
    const uint32_t nd = s3f[j].nd;
    if (nd == 0 || s3f[j].bad || nd > job.dist_cap) return;
    uint32_t x, e;
    const bool ok = m12_chain(s3base + job.s3_off, nd, s3base + job.s3_off + s3_em_off(job), s_tab, x, e);
    s3f[j].m12e = ok ? e : 0xFFFFFFFFu;
    s3f[j].m12x = x;
}

}  // namespace pz
