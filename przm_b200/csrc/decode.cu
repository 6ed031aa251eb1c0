// decode.cu -- the GPU decoder: PRZM frames back to their bytes, many frames
// per launch sequence, with the semantics of the reference's decoder
// (decompress.go:380-700 stageExecuteCommands and the section stages before
// it; src/przm_dec.c:741-1529 is the same decoder in C).
//
// Per frame, on the device:
//   k_dec_parse    one thread per frame: header, directory and sections
//                  (stage_parse_header / stage_resolve_sections); the form
//                  of each section; one entropy task per coded stream.
//   k_dec_static   one warp per Meta8 container (8 static context models)
//                  or Mode 12 code stream (4 static context models), the
//                  chain on lane 0, one symbol at a time (each symbol's
//                  context is the symbol before it);
//   k_dec_lists    the adaptive V-ANS bodies, longest first;
//   k_dec_adaptive eight bodies per warp: a group of four lanes per body,
//                  lane l holding interleaved state l; the four states share
//                  one stream pointer, so each round of four symbols waits
//                  for the one before it (matrix -> frequencies -> model,
//                  built by the warp).
//   k_dec_prefix   one block per frame with a distance-prefix Section 3:
//                  extra-bit offsets and varint lengths by block scans, the
//                  distances rebuilt and written as LEB128 varints.
//   k_dec_sheaf    one thread per sheaf frame: the literals re-interleaved
//                  from their four fibers by the class of the bytes before
//                  each (serial by the format).
//   k_dec_exec     one warp per frame: the command walk, every lane running
//                  the same scalar parse, literal and match copies split over
//                  the lanes (a match closer than its length repeats with
//                  period d, so byte i comes from source byte i mod d).
//
// Frames this decoder does not take (an external dictionary, the base64
// normalisation flag, delta-masked matches, the nibble-plane literal form,
// the dictionary-word opcodes) come back as PRZMG_ERR_UNSUPPORTED; they
// decode on the host.  Every read of a frame is bounds-checked against its
// length, every write against the capacities the host gave.
#include "common.cuh"

namespace pz {

enum DecErr : uint32_t { D_OK = 0, D_CORRUPT = 1, D_UNSUPPORTED = 2, D_CAP = 3, D_MAGIC = 4, D_BLOCK = 5 };

constexpr uint32_t kDecMaxBlock = 16777216u;  // PRZM_MAX_BLOCK_SIZE

// Host-filled, one per frame.  cap: the frame's output capacity and the
// capacity of each of its scratch buffers.
struct DecJob {
    uint64_t src_off;  // frame bytes in the source buffer
    uint64_t out_off;  // decoded bytes in the output buffer
    uint64_t scr_off;  // scratch region (kDecBufs buffers of dec_buf_bytes(cap))
    uint32_t src_len;
    uint32_t cap;
};

// scratch buffers of one frame
enum DecBuf : int { DB_OP = 0, DB_META = 1, DB_VAR = 2, DB_LIT = 3, DB_FIB = 4, DB_CODES = 5, DB_OFFS = 6, kDecBufs = 7 };
__host__ __device__ inline uint64_t dec_buf_bytes(uint32_t cap) { return (cap + 64ull + 15) & ~15ull; }

enum DecTaskKind : uint32_t { DT_NONE = 0, DT_ADAPTIVE = 1, DT_META8 = 2, DT_MODE12 = 3 };

// One coded stream: payload (for DT_ADAPTIVE the V-ANS body: matrix, four
// states, stream; for DT_META8 the whole container; for DT_MODE12 the code
// stream from its 0x0C byte), n symbols into dst.
struct DecTask {
    uint64_t src, dst;
    uint32_t kind, n, slen, frame;
};
constexpr int kDecTasks = 8;  // per frame: op, meta, var, codes, literals or four fibers

// Per-frame results of the parse.  Streams are device addresses.
struct DecInfo {
    uint32_t err;        // DecErr
    uint32_t u_size;
    uint32_t flags;
    uint32_t stored;     // uncompressed frame: bytes at src + 8
    uint32_t bmin, stride;
    uint32_t cmd_mode;   // 0: one command stream (cmd); 1: Mode 8 op / meta / var
    uint32_t cmd_len, meta_len, var_len, cmd_orig;
    uint32_t off_len, lit_len;
    uint32_t s3_prefix;  // 1: distance-prefix container, varints rebuilt into DB_OFFS
    uint32_t nd, extra_len, s3_orig;
    uint32_t sheaf, sheaf_mode;
    uint32_t fl[4];
    uint64_t cmd, meta, var, off, lit, codes, extra;
    uint64_t fib[4];
};

__device__ __forceinline__ uint32_t drd16(const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8); }
__device__ __forceinline__ uint32_t drd24(const uint8_t* p) { return drd16(p) | ((uint32_t)p[2] << 16); }
__device__ __forceinline__ uint32_t drd32(const uint8_t* p) { return drd24(p) | ((uint32_t)p[3] << 24); }

// A stream of an unpack_substream form (przm_dec.c:503-541): empty, a Meta8
// container, an adaptive container (flags byte 0), 0x09 + raw bytes or
// 0x00 + LE32 length + raw bytes.  Raw streams point into the frame; coded
// ones become a task decoding into dst (cap bytes).  Returns the DecErr.
__device__ uint32_t dec_substream(const uint8_t* s, uint32_t slen, uint8_t* dst, uint32_t cap, uint32_t frame,
                                  DecTask* task, uint64_t* out, uint32_t* out_len) {
    *out = 0;
    *out_len = 0;
    if (slen == 0) return D_OK;
    if (slen >= 8 && s[0] == 'V' && s[1] == 'A' && s[2] == 0x01) {
        const uint32_t n = drd32(s + 4);
        if (s[3] & 0x40) {
            if (slen < 24) return D_CORRUPT;
            if (n > cap) return D_CAP;
            *task = DecTask{(uint64_t)(uintptr_t)s, (uint64_t)(uintptr_t)dst, DT_META8, n, slen, frame};
            *out = (uint64_t)(uintptr_t)dst;
            *out_len = n;
            return D_OK;
        }
        if (s[3] == 0) {
            if (n > cap) return D_CAP;
            *task = DecTask{(uint64_t)(uintptr_t)(s + 8), (uint64_t)(uintptr_t)dst, DT_ADAPTIVE, n, slen - 8, frame};
            *out = (uint64_t)(uintptr_t)dst;
            *out_len = n;
            return D_OK;
        }
    }
    if (s[0] == 0x09) {
        *out = (uint64_t)(uintptr_t)(s + 1);
        *out_len = slen - 1;
        return D_OK;
    }
    if (s[0] == 0x00) {
        if (slen < 5) return D_CORRUPT;
        const uint32_t n = drd32(s + 1);
        if (5ull + n > slen) return D_CORRUPT;
        *out = (uint64_t)(uintptr_t)(s + 5);
        *out_len = n;
        return D_OK;
    }
    return D_UNSUPPORTED;
}

// Header, sections and entropy tasks of frame f (one thread).
__device__ uint32_t dec_parse_frame(const uint8_t* __restrict__ src, const DecJob& jb, uint8_t* scr, uint32_t f,
                                    DecInfo& I, DecTask* T) {
    const uint8_t* s = src + jb.src_off;
    const uint32_t len = jb.src_len, cap = jb.cap;
    const uint64_t bb = dec_buf_bytes(cap);
    if (len == 0) return D_OK;  // an empty frame is an empty input
    if (len < 8) return D_CORRUPT;
    if (drd32(s) != 0x4D5A5250u) return D_MAGIC;
    I.flags = s[4];
    I.u_size = drd24(s + 5);
    if (I.u_size > kDecMaxBlock) return D_BLOCK;
    if (I.u_size == 0) return D_OK;
    if (I.u_size > cap) return D_CAP;
    if (I.flags & 0x04) {  // uncompressed
        if (len < 8ull + I.u_size) return D_CORRUPT;
        I.stored = 1;
        return D_OK;
    }
    if (I.flags & (0x02 | 0x10 | 0x20)) return D_UNSUPPORTED;  // delta mask, dictionary, base64 normalisation
    I.bmin = (I.flags & 0x40) ? 3 : 4;
    uint32_t off = 8;
    I.stride = 1;
    if (I.flags & 0x01) {
        if (off >= len) return D_CORRUPT;
        I.stride = (uint32_t)s[off++] + 1;
    }
    uint32_t l_cmd, l_off;
    if (!(I.flags & 0x08)) {
        if (off + 4 > len) return D_CORRUPT;
        l_cmd = drd16(s + off);
        l_off = drd16(s + off + 2);
        off += 4;
    } else {
        if (off + 6 > len) return D_CORRUPT;
        l_cmd = drd24(s + off);
        l_off = drd24(s + off + 3);
        off += 6;
    }
    const uint32_t l1 = (off + 8 <= len) ? 8 + 2 * (uint32_t)s[off + 5] : 0;
    const uint64_t o2 = (uint64_t)off + l1, o3 = o2 + l_cmd, o4 = o3 + l_off;
    if (o4 > len) return D_CORRUPT;
    const uint32_t l4 = len - (uint32_t)o4;
    uint32_t r;
    // Section 4 (stage_unpack_literals, przm_dec.c:851-879)
    if (l4 > 0) {
        const uint8_t* s4 = s + o4;
        if (l4 >= 8 && s4[0] == 'V' && s4[1] == 'A' && s4[2] == 0x01) {
            const uint32_t fl = s4[3], ul = drd32(s4 + 4);
            if (ul > cap) return D_CAP;
            if (fl & 0x04) {  // sheaf (stage_unpack_sheaf :805-849)
                if (l4 < 40) return D_CORRUPT;
                const uint32_t mode = (fl >> 4) & 0x0F;
                if (mode > 3) return D_CORRUPT;
                uint32_t e[4];
                uint64_t sum = 0;
                for (int k = 0; k < 4; k++) {
                    I.fl[k] = drd32(s4 + 8 + 4 * k);
                    e[k] = drd32(s4 + 24 + 4 * k);
                    sum += I.fl[k];
                }
                if (sum != ul) return D_CORRUPT;
                if (mode == 2 && (I.fl[2] || I.fl[3])) return D_CORRUPT;
                uint64_t cur = 40;
                for (int k = 0; k < 4; k++) {
                    if (I.fl[k] == 0 && e[k] != 0) return D_CORRUPT;
                    if (e[k] > I.fl[k] || cur + e[k] > l4) return D_CORRUPT;
                    cur += e[k];
                }
                cur = 40;
                uint64_t fd = 0;
                uint8_t* fb = scr + DB_FIB * bb;
                for (int k = 0; k < 4; k++) {
                    I.fib[k] = 0;
                    if (I.fl[k]) {
                        if (e[k] == I.fl[k]) {
                            I.fib[k] = (uint64_t)(uintptr_t)(s4 + cur);
                        } else {
                            I.fib[k] = (uint64_t)(uintptr_t)(fb + fd);
                            T[4 + k] = DecTask{(uint64_t)(uintptr_t)(s4 + cur), I.fib[k], DT_ADAPTIVE, I.fl[k], e[k], f};
                        }
                    }
                    cur += e[k];
                    fd += I.fl[k];
                }
                I.sheaf = 1;
                I.sheaf_mode = mode;
                I.lit = (uint64_t)(uintptr_t)(scr + DB_LIT * bb);
                I.lit_len = ul;
            } else {
                T[4] = DecTask{(uint64_t)(uintptr_t)(s4 + 8), (uint64_t)(uintptr_t)(scr + DB_LIT * bb), DT_ADAPTIVE, ul,
                               l4 - 8, f};
                I.lit = (uint64_t)(uintptr_t)(scr + DB_LIT * bb);
                I.lit_len = ul;
            }
        } else if (l4 >= 8 && drd32(s4 + 4) == (uint32_t)(((uint64_t)drd32(s4) + 1) / 2)) {
            return D_UNSUPPORTED;  // nibble planes
        } else {
            I.lit = (uint64_t)(uintptr_t)s4;
            I.lit_len = l4;
        }
    }
    // Section 2 (stage_unpack_commands :881-923)
    if (l_cmd > 0) {
        const uint8_t* s2 = s + o2;
        if (s2[0] == 0x08) {
            if (l_cmd < 13) return D_CORRUPT;
            I.cmd_orig = drd32(s2 + 1);
            const uint32_t lo = drd32(s2 + 5), lm = drd32(s2 + 9);
            if (13ull + lo + lm > l_cmd) return D_CORRUPT;
            const uint32_t lv = l_cmd - 13 - lo - lm;
            I.cmd_mode = 1;
            if ((r = dec_substream(s2 + 13, lo, scr + DB_OP * bb, cap, f, &T[0], &I.cmd, &I.cmd_len))) return r;
            if ((r = dec_substream(s2 + 13 + lo, lm, scr + DB_META * bb, cap, f, &T[1], &I.meta, &I.meta_len))) return r;
            if ((r = dec_substream(s2 + 13 + lo + lm, lv, scr + DB_VAR * bb, cap, f, &T[2], &I.var, &I.var_len))) return r;
        } else if (s2[0] == 0x09) {
            I.cmd = (uint64_t)(uintptr_t)(s2 + 1);
            I.cmd_len = l_cmd - 1;
        } else if (s2[0] == 0x00) {
            if (l_cmd < 5) return D_CORRUPT;
            I.cmd_len = drd32(s2 + 1);
            if (5ull + I.cmd_len > l_cmd) return D_CORRUPT;  // (a length past the section)
            I.cmd = (uint64_t)(uintptr_t)(s2 + 5);
        } else {
            I.cmd = (uint64_t)(uintptr_t)s2;
            I.cmd_len = l_cmd;
        }
    }
    // Section 3 (stage_unpack_offsets :1132-1158)
    if (l_off > 0) {
        const uint8_t* s3 = s + o3;
        if (s3[0] == 0x09) {
            I.off = (uint64_t)(uintptr_t)(s3 + 1);
            I.off_len = l_off - 1;
        } else if (s3[0] == 0x00) {
            if (l_off < 5) return D_CORRUPT;
            I.off_len = drd32(s3 + 1);
            if (5ull + I.off_len > l_off) return D_CORRUPT;  // (a length past the section)
            I.off = (uint64_t)(uintptr_t)(s3 + 5);
        } else if (s3[0] == 0x06 || s3[0] == 0x0A || s3[0] == 0x0B) {
            // przm_distance_prefix_decode (:1057-1129)
            uint32_t orig, cnt, cl, h;
            if (l_off < 4) return D_CORRUPT;
            if (s3[0] == 0x06) {
                if (l_off < 13) return D_CORRUPT;
                orig = drd32(s3 + 1); cnt = drd32(s3 + 5); cl = drd32(s3 + 9); h = 13;
            } else if (s3[0] == 0x0A) {
                if (l_off < 7) return D_CORRUPT;
                orig = drd16(s3 + 1); cnt = drd16(s3 + 3); cl = drd16(s3 + 5); h = 7;
            } else {
                orig = s3[1]; cnt = s3[2]; cl = s3[3]; h = 4;
            }
            if ((uint64_t)h + cl > l_off) return D_CORRUPT;
            if (orig > kDecMaxBlock || cnt > orig) return D_CORRUPT;
            if (orig > cap) return D_CAP;
            I.s3_prefix = 1;
            I.s3_orig = orig;
            I.nd = cnt;
            I.off = (uint64_t)(uintptr_t)(scr + DB_OFFS * bb);
            I.off_len = cnt ? orig : 0;  // no distance: an empty offset stream whatever the header's length
            I.extra = (uint64_t)(uintptr_t)(s3 + h + cl);
            I.extra_len = l_off - h - cl;
            if (cnt > 0) {
                const uint8_t* cs = s3 + h;
                uint8_t* codes = scr + DB_CODES * bb;
                if (cl == cnt) {
                    I.codes = (uint64_t)(uintptr_t)cs;
                } else if (cl > 0 && cs[0] == 0x0C) {
                    if (cl < 5) return D_CORRUPT;
                    T[3] = DecTask{(uint64_t)(uintptr_t)cs, (uint64_t)(uintptr_t)codes, DT_MODE12, cnt, cl, f};
                    I.codes = (uint64_t)(uintptr_t)codes;
                } else {
                    uint64_t p;
                    uint32_t n;
                    if ((r = dec_substream(cs, cl, codes, cap, f, &T[3], &p, &n))) return r;
                    if (n < cnt) return D_CORRUPT;
                    I.codes = p;
                }
            }
        } else {
            I.off = (uint64_t)(uintptr_t)s3;
            I.off_len = l_off;
        }
    }
    return D_OK;
}

__global__ void k_dec_parse(const uint8_t* __restrict__ src, const DecJob* __restrict__ jobs, uint32_t nf,
                            uint8_t* __restrict__ scr, DecInfo* __restrict__ infos, DecTask* __restrict__ tasks) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const DecJob jb = jobs[f];
    DecInfo I = {};
    DecTask T[kDecTasks];
    for (int k = 0; k < kDecTasks; k++) T[k] = DecTask{0, 0, DT_NONE, 0, 0, f};
    I.err = dec_parse_frame(src, jb, scr + jb.scr_off, f, I, T);
    if (I.err) {
        for (int k = 0; k < kDecTasks; k++) T[k].kind = DT_NONE;
    }
    infos[f] = I;
    for (int k = 0; k < kDecTasks; k++) tasks[(uint64_t)f * kDecTasks + k] = T[k];
}

// Static decode models: the 8 Meta8 models (core/commands/vans_meta_tables.go)
// and the 4 Mode 12 distance-code models (core/distance/distance.go:67-93),
// built on the host.  Per context: the symbol of every slot, and per symbol
// (f - 1) << 20 | its cumulative frequency (the adaptive models' form too).
// Compact (41 KiB for Meta8), so a decoding warp keeps its model in shared
// memory: the serial chain's lookups then never wait on L2.
struct DecStatic {
    uint8_t m8sym[8][4096];
    uint32_t m8fc[8][256];
    uint8_t d12sym[4][4096];
    uint32_t d12fc[4][64];
};

__device__ __forceinline__ uint32_t ctx_meta8(uint32_t p) {  // ContextMeta, core/commands/vans_meta.go:46-69
    return p == 0 ? 0u : p < 4 ? 1u : p < 16 ? 2u : p < 32 ? 3u : p < 64 ? 4u : p < 128 ? 5u : p < 192 ? 6u : 7u;
}

__device__ __forceinline__ void dec_fail(DecInfo* infos, uint32_t f, uint32_t code) { atomicCAS(&infos[f].err, 0u, code); }

// The adaptive body's matrix (vans_read_joint_nibbles, przm_dec.c:155-185):
// LE16 row mask, per row an LE16 column mask and per column a weight of one
// byte (< 128) or two (15 bits, high byte first); the weights sum to 4096.
// Lane 0; freq zeroed by the caller.  Returns the bytes read, 0 if corrupt.
__device__ uint32_t dec_matrix(const uint8_t* s, uint32_t slen, uint16_t* freq) {
    uint32_t p = 0, sum = 0;
    if (p + 2 > slen) return 0;
    const uint32_t rows = drd16(s);
    p += 2;
    for (int h = 0; h < 16; h++) {
        if (!(rows & (1u << h))) continue;
        if (p + 2 > slen) return 0;
        const uint32_t cols = drd16(s + p);
        p += 2;
        for (int l = 0; l < 16; l++) {
            if (!(cols & (1u << l))) continue;
            if (p >= slen) return 0;
            uint32_t w = s[p++];
            if (w >= 128) {
                if (p >= slen) return 0;
                w = ((w & 0x7Fu) << 8) | s[p++];
            }
            if (w == 0 || w > 4096) return 0;
            freq[(h << 4) | l] = (uint16_t)w;
            sum += w;
        }
    }
    return sum == 4096 ? p : 0;
}

// The stream as the chain reads it: the next `av` bytes in w (first byte
// lowest) and the four after them prefetched in nx, loaded a round ahead so
// their latency stays off the chain.  renorm shifts bytes into x while x <
// 2^16 (the reference's renormalisation) and fails where the stream ends.
struct ByteWin {
    const uint8_t* s;
    uint32_t slen, q;  // q: next byte not yet loaded
    uint64_t w;
    uint32_t av, nx, nn;
    __device__ __forceinline__ void init(const uint8_t* src, uint32_t len, uint32_t p) {
        s = src;
        slen = len;
        q = p;
        w = 0;
        av = 0;
        nx = 0;
        nn = 0;
    }
    __device__ __forceinline__ void prefetch() {
        if (nn == 0 && q < slen) {
            const uint32_t m = min(4u, slen - q);
            uint32_t v = 0;
#pragma unroll
            for (uint32_t i = 0; i < 4; i++) v |= (i < m ? (uint32_t)s[q + i] : 0u) << (8 * i);
            nx = v;
            nn = m;
            q += m;
        }
    }
    __device__ __forceinline__ void merge() {
        if (nn && av <= 4) {
            w |= (uint64_t)nx << (8 * av);
            av += nn;
            nn = 0;
        }
    }
    // once per round: the prefetched bytes in, the next ones requested
    __device__ __forceinline__ void step() {
        merge();
        prefetch();
    }
    __device__ __forceinline__ bool renorm(uint32_t& x) {
        while (x < 65536u) {
            if (av == 0) {
                merge();
                if (av == 0) {
                    prefetch();
                    merge();
                    if (av == 0) return false;
                }
            }
            x = (x << 8) | (uint32_t)(w & 0xFFu);
            w >>= 8;
            av--;
        }
        return true;
    }
    __device__ __forceinline__ uint32_t pos() const { return q - nn - av; }  // bytes consumed
};

// Shared memory of a static-model task (the Meta8 models, the larger of the
// two kinds).  Static-model and adaptive tasks run as separate launches so the
// long adaptive chains are not held to the occupancy of this allotment.
constexpr uint32_t kDecStaticSmem = 8 * 4096 + 8 * 256 * 4;
static_assert(kDecStaticSmem >= 4 * 4096 + 4 * 64 * 4, "Mode 12 models");

// After a decode step x' = f (x >> 12) + j >= 16 when x >= 2^16, so a state
// takes 0, 1 or 2 bytes (the reference's loop runs while x < 2^16).

// Static-model tasks (Meta8 containers, Mode 12 code streams), one warp per
// task slot (tasks[blockIdx.x]; other kinds return at once): the warp copies
// the models into shared memory, lane 0 runs the chain (one symbol at a
// time: each symbol's context is the symbol before it).
__global__ void __launch_bounds__(32) k_dec_static(const DecTask* __restrict__ tasks, const DecStatic* __restrict__ st,
                                                   DecInfo* __restrict__ infos) {
    extern __shared__ __align__(16) uint8_t smem_d[];
    const DecTask t = tasks[blockIdx.x];
    const uint32_t lane = threadIdx.x;
    if ((t.kind != DT_META8 && t.kind != DT_MODE12) || t.n == 0) return;
    const uint8_t* s = reinterpret_cast<const uint8_t*>(t.src);
    uint8_t* dst = reinterpret_cast<uint8_t*>(t.dst);
    const uint32_t n = t.n, slen = t.slen;
    // the static models into shared memory (the warp), then the chain (lane 0)
    const bool m8 = t.kind == DT_META8;
    const uint32_t nsym = m8 ? 8 * 4096 : 4 * 4096, nfc = m8 ? 8 * 256 : 4 * 64;
    const uint4* gs = reinterpret_cast<const uint4*>(m8 ? &st->m8sym[0][0] : &st->d12sym[0][0]);
    const uint4* gf = reinterpret_cast<const uint4*>(m8 ? &st->m8fc[0][0] : &st->d12fc[0][0]);
    uint8_t* ssym = smem_d;
    uint32_t* sfc = reinterpret_cast<uint32_t*>(smem_d + nsym);
    for (uint32_t i = lane; i < nsym / 16; i += 32) reinterpret_cast<uint4*>(ssym)[i] = gs[i];
    for (uint32_t i = lane; i < nfc / 4; i += 32) reinterpret_cast<uint4*>(sfc)[i] = gf[i];
    __syncwarp();
    if (lane != 0) return;
    if (m8) {  // przm_vans_decode_meta8, przm_dec.c:459-500
        uint32_t xs[4] = {drd32(s + 8), drd32(s + 12), drd32(s + 16), drd32(s + 20)};
        uint32_t prev = 0;
        ByteWin bw;
        bw.init(s, slen, 24);
        bw.prefetch();
        bool ok = true;
        for (uint32_t i = 0; i < n && ok; i++) {
            const uint32_t l = i & 3;
            if (l == 0) bw.step();
            const uint32_t c = ctx_meta8(prev), slot = xs[l] & 4095;
            const uint32_t sym = ssym[c * 4096 + slot], fc = sfc[c * 256 + sym];
            dst[i] = (uint8_t)sym;
            prev = sym;
            xs[l] = ((fc >> 20) + 1) * (xs[l] >> 12) + slot - (fc & 0xFFFFFu);
            ok = bw.renorm(xs[l]);
        }
        if (!ok || bw.pos() != slen) dec_fail(infos, t.frame, D_CORRUPT);
        return;
    }
    // DT_MODE12: przm_vans_decode_dist4, przm_dec.c:958-990
    uint32_t x = drd32(s + 1), prev = 0;
    ByteWin bw;
    bw.init(s, slen, 5);
    bw.prefetch();
    bool ok = true;
    for (uint32_t i = 0; i < n && ok; i++) {
        if ((i & 1) == 0) bw.step();
        const uint32_t c = s3_ctx(prev), slot = x & 4095;
        const uint32_t sym = ssym[c * 4096 + slot], fc = sfc[c * 64 + sym];
        dst[i] = (uint8_t)sym;
        prev = sym;
        x = ((fc >> 20) + 1) * (x >> 12) + slot - (fc & 0xFFFFFu);
        ok = bw.renorm(x);
    }
    if (!ok) dec_fail(infos, t.frame, D_CORRUPT);
}

// Decode-table entry of slot j of symbol s (frequency f): s | j << 8 |
// (f - 1) << 20, so x' = f (x >> 12) + j is ((e >> 20) + 1) (x >> 12) +
// ((e >> 8) & 0xFFF) (the rANS decode step, przm_dec.c:187-199).
__host__ __device__ inline uint32_t dec_entry(uint32_t f, uint32_t j, uint32_t s) { return ((f - 1) << 20) | (j << 8) | s; }
__device__ __forceinline__ uint32_t dec_next(uint32_t x, uint32_t e) {
    return ((e >> 20) + 1) * (x >> 12) + ((e >> 8) & 0xFFFu);
}

// One round of an adaptive body on lanes 0-3 (lane l: state l, stream
// pointer p in every lane): the lane's symbol (returned with its table
// entry) and its state renormalised.  The round's eight stream bytes come
// from three aligned words (below p + 12; the caller keeps p + 16 <= the
// stream's length).  A state needs 0, 1 or 2 bytes (x < 2^16, x < 2^8
// after the step, the reference's loop); two ballots of those tests give
// every lane all four counts, hence its offset o (the bytes of the lanes
// before it) and the pointer's advance.  One byte permute puts bytes o,
// o + 1 in the low half of y, a second shifts them into x.
__device__ __forceinline__ uint32_t dec_round(const uint32_t* tab, uintptr_t sa, uint32_t lt, uint32_t& x,
                                              uint32_t& p) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>((sa + p) & ~uintptr_t(3));
    const uint32_t sh = 8u * (uint32_t)((sa + p) & 3u);
    const uint32_t w0 = w[0], w1 = w[1], w2 = w[2];
    const uint32_t lo = __funnelshift_r(w0, w1, sh), hi = __funnelshift_r(w1, w2, sh);
    const uint32_t e = tab[x & 4095];
    x = dec_next(x, e);
    const bool r1 = x < 65536u, r2 = x < 256u;
    const uint32_t b1 = __ballot_sync(0xFu, r1), b2 = __ballot_sync(0xFu, r2);
    const uint32_t o = __popc(b1 & lt) + __popc(b2 & lt);
    const uint32_t y = __byte_perm(lo, hi, 17u * o + 16u);  // byte 0: stream byte o, byte 1: byte o + 1
    x = __byte_perm(x, y, r2 ? 0x1045u : (r1 ? 0x2104u : 0x3210u));  // (x << 16 | o, o + 1), (x << 8 | o), x
    p += __popc(b1) + __popc(b2);
    return e;
}

// One adaptive body per warp (task slot blockIdx.x; other kinds return at
// once), for batches whose bodies all fit on the SMs at once: the warp builds
// a 4096-entry table (s | j << 8 | (f - 1) << 20 per slot, one shared load
// per step), lanes 0-3 run the body's four states.  Its rounds are the
// shortest of the two adaptive kernels; k_dec_adaptive trades them for eight
// bodies per warp when there are many.
constexpr uint32_t kDecAdaptive1Smem = 4096 * 4 + 256 * 2;
__global__ void __launch_bounds__(32) k_dec_adaptive1(const DecTask* __restrict__ tasks, DecInfo* __restrict__ infos) {
    extern __shared__ __align__(16) uint8_t smem_d[];
    uint32_t* tab = reinterpret_cast<uint32_t*>(smem_d);
    uint16_t* freq = reinterpret_cast<uint16_t*>(smem_d + 4096 * 4);
    const DecTask t = tasks[blockIdx.x];
    const uint32_t lane = threadIdx.x;
    if (t.kind != DT_ADAPTIVE || t.n == 0) return;
    const uint8_t* s = reinterpret_cast<const uint8_t*>(t.src);
    uint8_t* dst = reinterpret_cast<uint8_t*>(t.dst);
    const uint32_t n = t.n, slen = t.slen;
    for (uint32_t i = lane; i < 256; i += 32) freq[i] = 0;
    __syncwarp();
    uint32_t p = 0;
    if (lane == 0) p = dec_matrix(s, slen, freq);
    p = __shfl_sync(0xFFFFFFFFu, p, 0);
    if (p == 0 || p + 16 > slen) {
        if (lane == 0) dec_fail(infos, t.frame, D_CORRUPT);
        return;
    }
    __syncwarp();
    // decode table: lane l takes symbols 8l .. 8l + 7
    uint32_t f8[8], loc = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) { f8[k] = freq[lane * 8 + k]; loc += f8[k]; }
    uint32_t x = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    uint32_t c = x - loc;
    for (int k = 0; k < 8; k++) {
        for (uint32_t j = 0; j < f8[k]; j++) tab[c + j] = dec_entry(f8[k], j, lane * 8 + k);
        c += f8[k];
    }
    __syncwarp();
    if (lane >= 4) return;
    // lane l holds state l (the state of symbols l, l + 4, ...)
    uint32_t xl = drd32(s + p + 4 * lane);
    p += 16;
    uint32_t i = 0;
    bool ok = true;
    if (__all_sync(0xFu, xl >= 65536u)) {
        // Rounds of four symbols, one per lane: each lane's byte count
        // comes from its own state; two ballots give every lane all four,
        // hence its offset in the round's 8 bytes and the stream's
        // advance, so only the stream position links one round to the
        // next.
        const uintptr_t sa = reinterpret_cast<uintptr_t>(s);
        const uint32_t lt = (1u << lane) - 1u;
        uint8_t* dl = dst + lane;
        for (; i + 8 <= n && p + 24 <= slen; i += 8) {  // two rounds per trip
            dl[i] = (uint8_t)dec_round(tab, sa, lt, xl, p);
            dl[i + 4] = (uint8_t)dec_round(tab, sa, lt, xl, p);
        }
        for (; i + 4 <= n && p + 16 <= slen; i += 4) dl[i] = (uint8_t)dec_round(tab, sa, lt, xl, p);
    }
    uint32_t x0 = __shfl_sync(0xFu, xl, 0), x1 = __shfl_sync(0xFu, xl, 1), x2 = __shfl_sync(0xFu, xl, 2),
             x3 = __shfl_sync(0xFu, xl, 3);
    if (lane != 0) return;
    // the rest (the stream's last 16 bytes, or initial states below 2^16)
    // byte by byte
    ByteWin bw;
    bw.init(s, slen, p);
    bw.prefetch();
    for (; i + 4 <= n && ok; i += 4) {  // vans_run_4x_loop, przm_dec.c:201-255
        bw.step();
        const uint32_t e0 = tab[x0 & 4095], e1 = tab[x1 & 4095], e2 = tab[x2 & 4095], e3 = tab[x3 & 4095];
        x0 = dec_next(x0, e0);
        x1 = dec_next(x1, e1);
        x2 = dec_next(x2, e2);
        x3 = dec_next(x3, e3);
        ok = bw.renorm(x0) && bw.renorm(x1) && bw.renorm(x2) && bw.renorm(x3);
        dst[i] = (uint8_t)e0;
        dst[i + 1] = (uint8_t)e1;
        dst[i + 2] = (uint8_t)e2;
        dst[i + 3] = (uint8_t)e3;
    }
    uint32_t xs[4] = {x0, x1, x2, x3};
    for (; i < n && ok; i++) {
        bw.step();
        const uint32_t e = tab[xs[i & 3] & 4095];
        dst[i] = (uint8_t)e;
        xs[i & 3] = dec_next(xs[i & 3], e);
        ok = bw.renorm(xs[i & 3]);
    }
    if (!ok) dec_fail(infos, t.frame, D_CORRUPT);
}

// Adaptive bodies, eight per warp: lane group g (lanes 4g .. 4g + 3) of
// block b decodes task list[8 b + g], lane 4g + l holding state l.  The warp
// builds the eight models one after another (per model the symbol of every
// slot and (f - 1) << 20 | cumulative frequency per symbol, 5 KiB), then all
// groups run their rounds together, so one warp instruction advances eight
// chains; the list is sorted by length (k_dec_lists), so a warp's chains
// end close together.
constexpr uint32_t kDecGroups = 8;
// Batches of up to this many frames decode their adaptive bodies one per
// warp (k_dec_adaptive1): at 13 such warps per SM their bodies all run at
// once.  Measured on 1 MiB frames: 128 frames 29.4 ms one per warp against
// 67 ms eight per warp; 2560 frames 89 ms (whole decode) eight per warp
// against 97 ms.
constexpr uint32_t kDecOneWarpFrames = 512;
constexpr uint32_t kDecModel = 4096 + 256 * 4;
constexpr uint32_t kDecAdaptiveSmem = kDecGroups * kDecModel + 256 * 2 + kDecGroups * 4;

// The decoded state after symbol slot x & 4095 with model word g = (f - 1)
// << 20 | cumulative frequency: f (x >> 12) + (x & 4095) - cum (the rANS
// decode step, przm_dec.c:187-199).
__device__ __forceinline__ uint32_t dec_step(uint32_t x, uint32_t g) {
    return ((g >> 20) + 1) * (x >> 12) + (x & 4095u) - (g & 0xFFFFFu);
}

// The adaptive tasks of the slots, longest first by bit length of their
// symbol count: list[0] = their number, list[4 ..] their slot indices.  One
// block of 1024 threads (counts per bit length, their offsets, then places).
__global__ void __launch_bounds__(1024) k_dec_lists(const DecTask* __restrict__ tasks, uint32_t nslots,
                                                    uint32_t* __restrict__ list) {
    __shared__ uint32_t s_cnt[32], s_off[32];
    if (threadIdx.x < 32) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nslots; i += 1024) {
        const DecTask t = tasks[i];
        if (t.kind == DT_ADAPTIVE && t.n) atomicAdd(&s_cnt[31 - __clz(t.n)], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t o = 0;
        for (int b = 31; b >= 0; b--) {
            s_off[b] = o;
            o += s_cnt[b];
        }
        list[0] = o;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nslots; i += 1024) {
        const DecTask t = tasks[i];
        if (t.kind == DT_ADAPTIVE && t.n) list[4 + atomicAdd(&s_off[31 - __clz(t.n)], 1u)] = i;
    }
}

__global__ void __launch_bounds__(32) k_dec_adaptive(const DecTask* __restrict__ tasks, const uint32_t* __restrict__ list,
                                                     DecInfo* __restrict__ infos) {
    extern __shared__ __align__(16) uint8_t smem_d[];
    uint16_t* freq = reinterpret_cast<uint16_t*>(smem_d + kDecGroups * kDecModel);
    uint32_t* gp = reinterpret_cast<uint32_t*>(smem_d + kDecGroups * kDecModel + 512);
    const uint32_t lane = threadIdx.x, g = lane >> 2, l = lane & 3;
    const uint32_t base = blockIdx.x * kDecGroups, cnt = list[0];
    if (base >= cnt) return;
    // the models, one after another by the whole warp; gp[k]: group k's
    // stream offset after its matrix (0: no task, or a corrupt matrix)
    for (uint32_t k = 0; k < kDecGroups; k++) {
        uint32_t p = 0;
        if (base + k < cnt) {
            const DecTask t = tasks[list[4 + base + k]];
            const uint8_t* s = reinterpret_cast<const uint8_t*>(t.src);
            for (uint32_t i = lane; i < 256; i += 32) freq[i] = 0;
            __syncwarp();
            if (lane == 0) p = dec_matrix(s, t.slen, freq);
            p = __shfl_sync(0xFFFFFFFFu, p, 0);
            if (p == 0 || p + 16 > t.slen) {
                if (lane == 0) dec_fail(infos, t.frame, D_CORRUPT);
                p = 0;
            } else {
                // lane l takes symbols 8l .. 8l + 7 (the frequencies sum to
                // 4096, so every slot is written)
                uint8_t* sym = smem_d + k * kDecModel;
                uint32_t* fct = reinterpret_cast<uint32_t*>(sym + 4096);
                uint32_t f8[8], loc = 0;
#pragma unroll
                for (int q = 0; q < 8; q++) { f8[q] = freq[lane * 8 + q]; loc += f8[q]; }
                uint32_t x = loc;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                    if (lane >= (uint32_t)o) x += y;
                }
                uint32_t c = x - loc;
                for (int q = 0; q < 8; q++) {
                    fct[lane * 8 + q] = f8[q] ? ((f8[q] - 1) << 20) | c : 0u;
                    for (uint32_t j = 0; j < f8[q]; j++) sym[c + j] = (uint8_t)(lane * 8 + q);
                    c += f8[q];
                }
            }
        }
        if (lane == 0) gp[k] = p;
        __syncwarp();
    }
    // this lane's group and state
    const bool has = base + g < cnt;
    DecTask t = {};
    if (has) t = tasks[list[4 + base + g]];
    uint32_t p = gp[g];
    const bool valid = has && p != 0;
    const uint8_t* s = reinterpret_cast<const uint8_t*>(t.src);
    uint8_t* dst = reinterpret_cast<uint8_t*>(t.dst);
    const uint32_t n = t.n, slen = t.slen;
    const uint8_t* sym = smem_d + g * kDecModel;
    const uint32_t* fct = reinterpret_cast<const uint32_t*>(sym + 4096);
    uint32_t x = valid ? drd32(s + p + 4 * l) : 0u;
    p += 16;
    const uint32_t gm = 0xFu << (4 * g), lt = (1u << lane) - 1u;
    // every lane takes part in each warp vote below, whether its group has a
    // task or not (a lane that skipped one would leave the others waiting)
    const uint32_t vb = __ballot_sync(0xFFFFFFFFu, valid && x >= 65536u);
    const bool fast = valid && (vb & gm) == gm;
    uint32_t i = 0;
    const uintptr_t sa = reinterpret_cast<uintptr_t>(s);
    // Rounds of four symbols per group.  The round's eight stream bytes come
    // from three aligned words (below p + 12; the loop keeps p + 16 <= the
    // stream's length).  A state needs 0, 1 or 2 bytes (x < 2^16, x < 2^8
    // after the step); two ballots of those tests, each group reading its
    // own four bits, give every lane its offset o (the bytes of the group's
    // lanes before it) and the pointer's advance.  One byte permute puts
    // bytes o, o + 1 in the low half of y, a second shifts them into x.
    for (;;) {
        const bool act = fast && i + 4 <= n && p + 16 <= slen;
        if (!__any_sync(0xFFFFFFFFu, act)) break;
        uint32_t lo = 0, hi = 0, sv = 0;
        if (act) {
            const uint32_t* w = reinterpret_cast<const uint32_t*>((sa + p) & ~uintptr_t(3));
            const uint32_t sh = 8u * (uint32_t)((sa + p) & 3u);
            const uint32_t w0 = w[0], w1 = w[1], w2 = w[2];
            lo = __funnelshift_r(w0, w1, sh);
            hi = __funnelshift_r(w1, w2, sh);
            sv = sym[x & 4095];
            x = dec_step(x, fct[sv]);
        }
        const bool r1 = act && x < 65536u, r2 = act && x < 256u;
        const uint32_t b1 = __ballot_sync(0xFFFFFFFFu, r1) & gm, b2 = __ballot_sync(0xFFFFFFFFu, r2) & gm;
        if (act) {
            const uint32_t o = __popc(b1 & lt) + __popc(b2 & lt);
            const uint32_t y = __byte_perm(lo, hi, 17u * o + 16u);
            x = __byte_perm(x, y, r2 ? 0x1045u : (r1 ? 0x2104u : 0x3210u));
            p += __popc(b1) + __popc(b2);
            dst[i + l] = (uint8_t)sv;
            i += 4;
        }
    }
    uint32_t x0 = __shfl_sync(0xFFFFFFFFu, x, 4 * g), x1 = __shfl_sync(0xFFFFFFFFu, x, 4 * g + 1),
             x2 = __shfl_sync(0xFFFFFFFFu, x, 4 * g + 2), x3 = __shfl_sync(0xFFFFFFFFu, x, 4 * g + 3);
    if (l != 0 || !valid) return;
    // the rest (the stream's last 16 bytes, or initial states below 2^16)
    // byte by byte, on the group's first lane
    bool ok = true;
    ByteWin bw;
    bw.init(s, slen, p);
    bw.prefetch();
    for (; i + 4 <= n && ok; i += 4) {  // vans_run_4x_loop, przm_dec.c:201-255
        bw.step();
        const uint32_t s0 = sym[x0 & 4095], s1 = sym[x1 & 4095], s2 = sym[x2 & 4095], s3 = sym[x3 & 4095];
        x0 = dec_step(x0, fct[s0]);
        x1 = dec_step(x1, fct[s1]);
        x2 = dec_step(x2, fct[s2]);
        x3 = dec_step(x3, fct[s3]);
        ok = bw.renorm(x0) && bw.renorm(x1) && bw.renorm(x2) && bw.renorm(x3);
        dst[i] = (uint8_t)s0;
        dst[i + 1] = (uint8_t)s1;
        dst[i + 2] = (uint8_t)s2;
        dst[i + 3] = (uint8_t)s3;
    }
    uint32_t xs[4] = {x0, x1, x2, x3};
    for (; i < n && ok; i++) {
        bw.step();
        const uint32_t v = sym[xs[i & 3] & 4095];
        dst[i] = (uint8_t)v;
        xs[i & 3] = dec_step(xs[i & 3], fct[v]);
        ok = bw.renorm(xs[i & 3]);
    }
    if (!ok) dec_fail(infos, t.frame, D_CORRUPT);
}

// Distance-prefix Section 3 of frame blockIdx.x (przm_distance_prefix_decode,
// przm_dec.c:1057-1129): code c gives base(c) + the next nb(c) bits of the
// MSB-first extra-bit stream; the distances are written back as LEB128
// varints, which must fill exactly the header's varint length.
__device__ __forceinline__ uint32_t code_bits(uint32_t c) { return c < 4 ? 0u : c == 48 ? 24u : (c - 2) >> 1; }
__device__ __forceinline__ uint32_t code_base(uint32_t c) {
    if (c < 4) return c + 1;
    if (c == 48) return 16777217u;
    const uint32_t b = (c - 2) >> 1;
    return ((2u + ((c - 2) & 1u)) << b) + 1u;
}

__global__ void __launch_bounds__(1024) k_dec_prefix(DecInfo* __restrict__ infos) {
    __shared__ uint32_t s_warp[32];
    const uint32_t f = blockIdx.x, tid = threadIdx.x;
    const DecInfo I = infos[f];
    if (I.err || !I.s3_prefix || I.nd == 0) return;
    const uint8_t* codes = reinterpret_cast<const uint8_t*>(I.codes);
    const uint8_t* ex = reinterpret_cast<const uint8_t*>(I.extra);
    uint8_t* out = reinterpret_cast<uint8_t*>(I.off);
    const uint32_t nd = I.nd, xl = I.extra_len, orig = I.s3_orig;
    uint64_t bits = 0;
    uint32_t vpos = 0, bad = 0;
    for (uint32_t b0 = 0; b0 < nd; b0 += 1024) {  // uniform trip count: every thread scans
        const uint32_t i = b0 + tid;
        const uint32_t c = i < nd ? codes[i] : 0u;
        uint32_t nb = 0, bf = 0;
        if (i < nd) {
            if (c > 48) bf = 1;
            else nb = code_bits(c);
        }
        uint32_t tb, tv;
        const uint64_t ob = bits + block_exclusive_scan<1024>(nb, s_warp, tb);
        uint32_t d = 0, vl = 0;
        if (i < nd && !bf) {
            uint32_t v = 0;
            if (nb) {
                if (((ob + nb + 7) >> 3) > xl) {
                    bf = 1;  // the bit reader runs past the stream
                } else {
                    const uint64_t q = ob >> 3;
                    uint32_t w = 0;
#pragma unroll
                    for (int k = 0; k < 4; k++) w = (w << 8) | (q + k < xl ? (uint32_t)ex[q + k] : 0u);
                    v = (w << (ob & 7)) >> (32 - nb);
                }
            }
            d = code_base(c) + v;
            vl = d <= 0x7Fu ? 1u : d <= 0x3FFFu ? 2u : d <= 0x1FFFFFu ? 3u : 4u;
        }
        const uint32_t ov = vpos + block_exclusive_scan<1024>(vl, s_warp, tv);
        if (vl) {
            if ((uint64_t)ov + vl > orig) {
                bf = 1;
            } else {
                uint32_t x = d, q = ov;
                while (x >= 0x80u) {
                    out[q++] = (uint8_t)(x | 0x80u);
                    x >>= 7;
                }
                out[q] = (uint8_t)x;
            }
        }
        bits += tb;
        vpos += tv;
        bad |= (uint32_t)__syncthreads_or(bf);
    }
    if (tid == 0 && (bad || vpos != orig)) dec_fail(infos, f, D_CORRUPT);
}

// Literals of a sheaf frame from their fibers (przm_reconstitute_fibers,
// przm_dec.c:354-394); one thread per frame.
__global__ void k_dec_sheaf(DecInfo* __restrict__ infos, uint32_t nf) {
    __shared__ ClassLut s_lut[4];
    for (uint32_t m = 0; m < 4; m++) class_lut_build(s_lut[m], m, threadIdx.x, blockDim.x);
    __syncthreads();
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const DecInfo I = infos[f];
    if (I.err || !I.sheaf) return;
    const ClassLut& L = s_lut[I.sheaf_mode];
    const uint32_t mode = I.sheaf_mode, n = I.lit_len;
    const uint32_t l0 = I.fl[0], l1 = I.fl[1], l2 = I.fl[2], l3 = I.fl[3];
    const uint8_t *f0 = reinterpret_cast<const uint8_t*>(I.fib[0]), *f1 = reinterpret_cast<const uint8_t*>(I.fib[1]),
                  *f2 = reinterpret_cast<const uint8_t*>(I.fib[2]), *f3 = reinterpret_cast<const uint8_t*>(I.fib[3]);
    uint8_t* lit = reinterpret_cast<uint8_t*>(I.lit);
    uint32_t q0 = 0, q1 = 0, q2 = 0, q3 = 0, p1 = 0, p2 = 0;  // per-fiber positions in registers (selected, not indexed)
    for (uint32_t j = 0; j < n; j++) {
        const uint32_t c = class_lut(L, p2, p1, mode);
        const bool ok = c == 0 ? q0 < l0 : c == 1 ? q1 < l1 : c == 2 ? q2 < l2 : q3 < l3;
        if (!ok) {
            dec_fail(infos, f, D_CORRUPT);
            return;
        }
        const uint32_t b = c == 0 ? f0[q0] : c == 1 ? f1[q1] : c == 2 ? f2[q2] : f3[q3];
        q0 += c == 0;
        q1 += c == 1;
        q2 += c == 2;
        q3 += c == 3;
        lit[j] = (uint8_t)b;
        p2 = p1;
        p1 = b;
    }
}

// The frame's command streams: one stream (Section 2 flat), or the Mode 8
// op / meta / var substreams read in the order of their joined stream
// (demux_step, przm_dec.c:544-603), j counting the joined bytes.
struct CmdReader {
    const uint8_t *c, *m, *v;
    uint32_t cl, ml, vl, cp, mp, vp, j, jlim;
    bool split;
    __device__ bool more() const { return split ? j < jlim && cp < cl : cp < cl; }
    __device__ bool op(uint32_t& b) {
        if (!more()) return false;
        b = c[cp++];
        j++;
        return true;
    }
    __device__ bool meta(uint32_t& b) {
        if (split) {
            if (mp >= ml || j >= jlim) return false;
            b = m[mp++];
        } else {
            if (cp >= cl) return false;
            b = c[cp++];
        }
        j++;
        return true;
    }
    // read_leb128 (przm_dec.c:98-115): at most four bytes, at most 2^24
    __device__ bool leb(uint32_t& val) {
        uint32_t r = 0;
        for (int i = 0; i < 4; i++) {
            uint32_t b;
            if (split) {
                if (vp >= vl || j >= jlim) return false;
                b = v[vp++];
            } else {
                if (cp >= cl) return false;
                b = c[cp++];
            }
            j++;
            r |= (b & 0x7Fu) << (7 * i);
            if (!(b & 0x80u)) {
                if (r > kDecMaxBlock) return false;
                val = r;
                return true;
            }
        }
        return false;
    }
    // a varint of the joined stream copied without its value (copy_leb128_raw)
    __device__ bool skip_leb() {
        for (int i = 0; i < 4; i++) {
            if (vp >= vl) return false;
            j++;
            if (!(v[vp++] & 0x80u)) return true;
        }
        return false;
    }
};

__device__ __forceinline__ bool off_leb(const uint8_t* o, uint32_t ol, uint32_t& op, uint32_t& val) {
    uint32_t r = 0;
    for (int i = 0; i < 4; i++) {
        if (op >= ol) return false;
        const uint32_t b = o[op++];
        r |= (b & 0x7Fu) << (7 * i);
        if (!(b & 0x80u)) {
            if (r > kDecMaxBlock) return false;
            val = r;
            return true;
        }
    }
    return false;
}

// The four repeat distances in registers (selected, not indexed).
struct Reps {
    uint32_t r0, r1, r2, r3;
    __device__ __forceinline__ uint32_t get(uint32_t k) const { return k == 0 ? r0 : k == 1 ? r1 : k == 2 ? r2 : r3; }
    // update_lru_repeat, przm_dec.c:1161-1166: entry k moves to the front
    __device__ __forceinline__ void repeat(uint32_t k) {
        const uint32_t t = get(k);
        if (k >= 3) r3 = r2;
        if (k >= 2) r2 = r1;
        if (k >= 1) { r1 = r0; r0 = t; }
    }
    // update_lru_explicit (:1168-1170)
    __device__ __forceinline__ void explicit_(uint32_t d) { r3 = r2; r2 = r1; r1 = r0; r0 = d; }
};

// Warp copies into dst (the output at position pos) and into the ring, the
// last kExecRing output bytes in shared memory.  Literals: n bytes from src.
// Match: n bytes from d back, byte i from byte (i mod d) of the source run
// (the byte-wise forward copy of an overlapping match repeats with period
// d); read from the ring when d + n <= kExecRing (every source byte is then
// in it and no byte the match writes lands on one it still reads), else from
// the output in global memory.
constexpr uint32_t kExecRing = 8192;
__device__ __forceinline__ void warp_copy_lits(uint8_t* dst, uint8_t* ring, uint32_t pos, const uint8_t* src,
                                               uint32_t n) {
    for (uint32_t i = threadIdx.x & 31; i < n; i += 32) {
        const uint8_t b = src[i];
        dst[i] = b;
        ring[(pos + i) & (kExecRing - 1)] = b;
    }
    __syncwarp();
}
__device__ __forceinline__ void warp_copy_match(uint8_t* dst, uint8_t* ring, uint32_t pos, uint32_t d, uint32_t n) {
    const uint32_t lane = threadIdx.x & 31;
    if (d + n <= kExecRing) {
        const uint32_t base = pos - d;
        for (uint32_t i = lane; i < n; i += 32) {
            const uint8_t b = ring[(base + (d >= n ? i : i % d)) & (kExecRing - 1)];
            dst[i] = b;
            ring[(pos + i) & (kExecRing - 1)] = b;
        }
    } else {
        const uint8_t* s = dst - d;
        for (uint32_t i = lane; i < n; i += 32) {
            const uint8_t b = s[d >= n ? i : i % d];
            dst[i] = b;
            ring[(pos + i) & (kExecRing - 1)] = b;
        }
    }
    __syncwarp();
}

// The command walk of frame blockIdx.x (stage_execute_commands,
// przm_dec.c:1285-1525; decompress.go:380-672): one warp, every lane
// parsing the same commands; the opcodes of the tokenizer (fused repeat
// < 0x80, fused explicit 0x80-0xBF, long repeat 0xC0-0xC3, literal runs
// 0xF0 / 0xF3-0xFA, byte runs 0xF1) and the plain-distance matches
// (brackets 0xC4-0xCD, the difference lattice 0xCE, strides 0xD0-0xD7).
__global__ void __launch_bounds__(32) k_dec_exec(const uint8_t* __restrict__ src, const DecJob* __restrict__ jobs,
                                                 DecInfo* __restrict__ infos, uint8_t* __restrict__ out) {
    const uint32_t f = blockIdx.x, lane = threadIdx.x;
    const DecInfo I = infos[f];
    if (I.err || I.u_size == 0) return;
    const DecJob jb = jobs[f];
    uint8_t* dst = out + jb.out_off;
    const uint32_t u = I.u_size;
    __shared__ __align__(16) uint8_t ring[kExecRing];
    if (I.stored) {
        warp_copy_lits(dst, ring, 0, src + jb.src_off + 8, u);
        return;
    }
    CmdReader R;
    R.c = reinterpret_cast<const uint8_t*>(I.cmd);
    R.m = reinterpret_cast<const uint8_t*>(I.meta);
    R.v = reinterpret_cast<const uint8_t*>(I.var);
    R.cl = I.cmd_len;
    R.ml = I.meta_len;
    R.vl = I.var_len;
    R.cp = R.mp = R.vp = R.j = 0;
    R.split = I.cmd_mode == 1;
    R.jlim = R.split ? I.cmd_orig : I.cmd_len;
    const uint8_t* lit = reinterpret_cast<const uint8_t*>(I.lit);
    const uint8_t* offs = reinterpret_cast<const uint8_t*>(I.off);
    const uint32_t ll = I.lit_len, ol = I.off_len, bmin = I.bmin, stride = I.stride;
    Reps r;
    if ((I.flags & 0x01) && stride > 1) { r.r0 = 1; r.r1 = stride; r.r2 = 2 * stride; r.r3 = 3 * stride; }
    else { r.r0 = 1; r.r1 = 4; r.r2 = 8; r.r3 = 16; }
    uint32_t dp = 0, lp = 0, opos = 0, err = D_OK;
    while (dp < u && R.more()) {
        uint32_t op;
        R.op(op);
        uint32_t llit = 0, lmatch = 0, d = 0, kind = 0;  // kind 0: literals only, 1 repeat k, 2 explicit d, 3 offset stream, 4 byte run
        uint32_t k = 0;
        if (op < 0x80) {
            llit = (op >> 4) & 7; lmatch = ((op >> 2) & 3) + bmin; k = op & 3; kind = 1;
        } else if (op < 0xC0) {
            llit = (op >> 4) & 3; lmatch = (op & 15) + bmin; kind = 3;
            if ((op & 15) == 15) { uint32_t x; if (!R.leb(x)) { err = D_CORRUPT; break; } lmatch += x; }
        } else if (op <= 0xC3) {
            uint32_t tok;
            if (!R.meta(tok)) { err = D_CORRUPT; break; }
            llit = tok >> 4; lmatch = (tok & 15) + bmin; k = op & 3; kind = 1;
            if ((tok & 15) == 15) { uint32_t x; if (!R.leb(x)) { err = D_CORRUPT; break; } lmatch += x; }
        } else if (op <= 0xCD) {
            uint32_t tok;
            if (!R.meta(tok)) { err = D_CORRUPT; break; }
            const uint32_t b = op - 0xC4;
            d = b <= 7 ? b + 1 : b == 8 ? 16u : 32u;
            llit = tok >> 4; lmatch = (tok & 15) + bmin; kind = 2;
        } else if (op == 0xCE) {
            uint32_t desc, dl;
            if (!R.meta(desc) || !R.meta(dl)) { err = D_CORRUPT; break; }
            const int32_t delta = (int32_t)(int8_t)dl;
            const uint32_t mode = (desc >> 6) & 3;
            int64_t dd;
            if (mode < 3) dd = (int64_t)r.get(mode) + delta;
            else dd = stride > 1 ? (int64_t)r.r0 + (int64_t)delta * stride : (int64_t)(uint8_t)dl + 1;
            if (dd <= 0 || dd > 0xFFFFFFFFll) { err = D_CORRUPT; break; }
            d = (uint32_t)dd;
            llit = (desc >> 3) & 7; lmatch = (desc & 7) + bmin; kind = 2;
            if (llit == 7) { uint32_t x; if (!R.leb(x)) { err = D_CORRUPT; break; } llit += x; }
            if ((desc & 7) == 7) { uint32_t x; if (!R.leb(x)) { err = D_CORRUPT; break; } lmatch += x; }
        } else if (op >= 0xD0 && op <= 0xD7) {
            uint32_t tok;
            if (!R.meta(tok)) { err = D_CORRUPT; break; }
            d = ((op & 7) + 1) * stride;
            llit = tok >> 4; lmatch = (tok & 15) + bmin; kind = 2;
        } else if (op == 0xF0) {
            if (!R.leb(llit)) { err = D_CORRUPT; break; }
        } else if (op == 0xF1) {
            if (!R.leb(lmatch)) { err = D_CORRUPT; break; }
            kind = 4;
        } else if (op >= 0xF3 && op <= 0xFA) {
            llit = op - 0xF2;
        } else if (op == 0xF2 || op >= 0xFB) {
            err = D_CORRUPT;
            break;
        } else {
            err = D_UNSUPPORTED;  // dictionary words, dictionary matches, delta-masked repeats
            break;
        }
        if (kind == 4) {  // byte run
            if (lp >= ll || dp + lmatch > u) { err = D_CORRUPT; break; }
            const uint8_t b = lit[lp++];
            for (uint32_t i = lane; i < lmatch; i += 32) {
                dst[dp + i] = b;
                ring[(dp + i) & (kExecRing - 1)] = b;
            }
            __syncwarp();
            dp += lmatch;
            continue;
        }
        if (lp + llit > ll || dp + llit > u) { err = D_CORRUPT; break; }
        warp_copy_lits(dst + dp, ring, dp, lit + lp, llit);
        lp += llit;
        dp += llit;
        if (kind == 0) continue;
        if (dp == u) break;
        if (kind == 1) {
            d = r.get(k);
            r.repeat(k);
        } else {
            if (kind == 3 && !off_leb(offs, ol, opos, d)) { err = D_CORRUPT; break; }
            r.explicit_(d);
        }
        if (d == 0 || d > dp || dp + lmatch > u) { err = D_CORRUPT; break; }  // no dictionary: d <= dp
        warp_copy_match(dst + dp, ring, dp, d, lmatch);
        dp += lmatch;
    }
    if (!err && dp != u) err = D_CORRUPT;
    if (!err && R.split) {
        // the rest of the joined stream, demultiplexed without executing
        // (demux_commands, przm_dec.c:605-623): it must fill the joined
        // length and use up the three substreams
        while (!err && R.cp < R.cl && R.j < R.jlim) {
            uint32_t op = R.c[R.cp++];
            R.j++;
            uint32_t t;
            bool ok = true;
            if (op < 0x80 || (op >= 0xF3 && op <= 0xFA)) {
            } else if (op < 0xC0) {
                if ((op & 15) == 15) ok = R.skip_leb();
            } else if (op <= 0xC3 || op == 0xE9) {
                ok = R.meta(t) && ((t & 15) != 15 || R.skip_leb());
            } else if (op <= 0xCD || (op >= 0xD0 && op <= 0xD7)) {
                ok = R.meta(t);
            } else if (op == 0xCE) {
                uint32_t t2;
                ok = R.meta(t) && R.meta(t2) && (((t >> 3) & 7) != 7 || R.skip_leb()) && ((t & 7) != 7 || R.skip_leb());
            } else if (op == 0xCF || (op >= 0xEA && op <= 0xEF)) {
                ok = R.meta(t) && R.skip_leb();
            } else if (op <= 0xE8) {
                ok = R.meta(t) && (t != 255 || R.skip_leb());
            } else if (op == 0xF0 || op == 0xF1) {
                ok = R.skip_leb();
            } else {
                ok = false;
            }
            if (!ok) err = D_CORRUPT;
        }
        if (!err && (R.j != R.jlim || R.cp != R.cl || R.mp != R.ml || R.vp != R.vl)) err = D_CORRUPT;
    }
    if (err && lane == 0) dec_fail(infos, f, err);
}

}  // namespace pz
