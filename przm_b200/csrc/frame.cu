// frame.cu -- section selection and PRZM frame assembly.
//
// Profile 0 is the CompressD2D frame (gpu/bridge.go:2287-2458 with
// przm_write_frame_header_kernel, przm_ans.cu:497-539): flat 0x00 command and
// offset sections, raw literals.
// Profile 1 is the entropy-coded frame: Section 2 as PackageCommandsSection
// (core/commands/commands.go:371-444, 537-568) when the command stream is at
// most 2 MiB, Section 3 flat, Section 4 the adaptive V-ANS container
// (core/literals/literals.go:368-384) when it beats the raw literals (or the
// raw literals would be misread as a container), FlagNibble with a V-ANS
// Section 4 (compress.go:990), and the uncompressed-frame fallback of
// assembleContainer (compress.go:962-985).
// Profile 2 is profile 1 with Section 3 as PackageOffsetsSection of the
// frame's distances (distance.go:825-849, compress.go:956), empty when the
// frame has no distance.  Profile 3 is profile 2 with Section 4 as
// PackageLiteralsSection (literals.go:664-693, compress.go:957): the
// smallest of the raw literals, their adaptive container and the four
// étale-sheaf foliations (PackEtaleSheaf :600-631, assembleSheafContainer
// :645-662), under profile 1's decodability rule when raw wins.
#include "common.cuh"

namespace pz {

__host__ __device__ inline uint32_t d2d_wlog(uint32_t n) { return n <= 65536 ? 16 : (n > 1048576 ? 23 : 20); }

__device__ inline uint32_t tsum(const TaskOut& o) { return o.count[0] + o.count[1] + o.count[2] + o.count[3]; }

__device__ inline uint32_t rd32b(const uint8_t* p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

// Section 3 of a P2 frame (PackageOffsetsSection, distance.go:825-849 with
// PackDistancePrefix :692-748 and SelectPrefixMode :750-758): empty without
// distances; else the distance-prefix container (Mode 12 code stream, or the
// codes' adaptive container for 64 codes or more when that fits 2 MiB and is
// smaller; header 0x0B / 0x0A / 0x06 by size) when it fits the reference's
// 2 MiB scratch and is smaller than the varints, else 0x09 + the varints.
// The reference's errors (a distance of 0 or above 2^24, more than 2^21
// codes, extra bits or Mode 12 bytes past 2 MiB) give the varint form.
__device__ inline void plan_s3(Plan& p, const Job& job, const uint32_t* lens, const S3Frame& f,
                               const TableInfo* infos, const TaskOut* outs, uint32_t j) {
    p.l3 = 0;
    if (f.nd == 0) {
        p.s3_form = 3;
        return;
    }
    const uint32_t nd = f.nd, xl = (f.bits + 7) / 8;
    if (!(f.bad || nd > kS3Scratch || xl > kS3Scratch || f.m12e == 0xFFFFFFFFu)) {
        uint32_t cl = 5 + f.m12e, code = 0;
        if (task_active(job, lens, T_S3, nd)) {
            const uint32_t al = 8 + infos[(uint64_t)j * kModels + 4].mat_len + 16 + tsum(outs[(uint64_t)j * T_COUNT + T_S3]);
            if (al <= kS3Scratch && al < cl) {
                cl = al;
                code = 1;
            }
        }
        const uint32_t orig = f.orig;
        const uint32_t h = (orig <= 255 && nd <= 255 && cl <= 255) ? 4u : (orig <= 65535 && nd <= 65535 && cl <= 65535) ? 7u : 13u;
        const uint64_t total = (uint64_t)h + cl + xl;
        if (total <= kS3Scratch && total < orig) {
            p.s3_form = 1;
            p.s3_code = code;
            p.s3_hlen = h;
            p.s3_cl = cl;
            p.s3_xl = xl;
            p.l3 = (uint32_t)total;
            return;
        }
    }
    p.s3_form = 2;
    p.l3 = 1 + f.orig;
}

__global__ void k_plan(const Job* __restrict__ jobs, uint32_t j0, uint32_t njobs, const uint32_t* __restrict__ job_lens,
                       const TableInfo* __restrict__ infos, const TaskOut* __restrict__ outs,
                       const uint8_t* __restrict__ streams, const S3Frame* __restrict__ s3f,
                       const uint8_t* __restrict__ fibbase, Plan* __restrict__ plans, uint32_t* __restrict__ sizes) {
    const uint32_t jl = blockIdx.x * blockDim.x + threadIdx.x;
    if (jl >= njobs) return;
    const uint32_t j = j0 + jl;
    const Job job = jobs[j];
    const uint32_t* lens = job_lens + (uint64_t)j * S_COUNT;
    Plan p = {};
    const uint32_t n = job.n;
    p.wlog = d2d_wlog(n);
    if (n == 0) {  // empty input gives an empty result (gpu/bridge.go:2491-2493)
        plans[j] = p;
        sizes[j] = 0;
        return;
    }
    if (job.profile == 0) {
        p.l2 = lens[S_CMD] + 5;
        p.l3 = lens[S_OFF] + 5;
        p.l4 = lens[S_LIT];
        const bool ext = n > 65535 || p.l2 > 65535 || p.l3 > 65535 || p.wlog > 16;
        p.flags = ext ? 0x08 : 0;
        p.frame_size = 8 + (ext ? 6 : 4) + 8 + p.l2 + p.l3 + p.l4;
    } else {
        const uint32_t cmd = lens[S_CMD];
        p.s2_mode = 2;
        p.l2 = 1 + cmd;
        if (cmd <= (2u << 20)) {
            uint32_t m8 = 13;
            for (int sub = 0; sub < 3; sub++) {
                const uint32_t len = lens[S_OP + sub];
                uint32_t best = 1 + len, mode = 0;
                const int tm = T_OP_M8 + 2 * sub, ta = tm + 1;
                if (task_active(job, lens, tm)) {
                    uint32_t sz = 24 + tsum(outs[(uint64_t)j * T_COUNT + tm]);
                    if (sz < best) { best = sz; mode = 1; }
                }
                if (task_active(job, lens, ta)) {
                    uint32_t sz = 8 + infos[(uint64_t)j * kModels + 1 + sub].mat_len + 16 + tsum(outs[(uint64_t)j * T_COUNT + ta]);
                    if (sz < best) { best = sz; mode = 2; }
                }
                p.sub_len[sub] = best;
                p.sub_mode[sub] = mode;
                m8 += best;
            }
            if (m8 < cmd) { p.s2_mode = 1; p.l2 = m8; }
        }
        if (job.profile >= 2) plan_s3(p, job, lens, s3f[j], infos, outs, j);
        else p.l3 = lens[S_OFF] + 5;
        const uint32_t lit = lens[S_LIT];
        p.l4 = lit;
        bool fallback = false;
        if (lit > 0) {
            const uint8_t* lp = streams + job.str_off + stream_base(job, S_LIT);
            bool raw_ok = true;
            if (lit >= 8) {
                if (lp[0] == 'V' && lp[1] == 'A' && lp[2] == 0x01) raw_ok = false;
                else if (rd32b(lp + 4) == (uint32_t)(((uint64_t)rd32b(lp) + 1) / 2)) raw_ok = false;
            }
            bool vans = false;
            uint32_t vsz = 0;
            if (task_active(job, lens, T_LIT)) {
                const uint32_t e = tsum(outs[(uint64_t)j * T_COUNT + T_LIT]);
                if (e <= (8u << 20)) { vans = true; vsz = 8 + infos[(uint64_t)j * kModels].mat_len + 16 + e; }
            }
            uint32_t choice = 0;  // 0 raw, 1 adaptive container, 2 a foliation
            uint32_t best = lit;
            if (job.profile >= 3 && lit <= kFibMax) {
                // PackageLiteralsSection: strictly smaller wins, adaptive first, then modes 0-3
                if (vans && vsz < best) { best = vsz; choice = 1; }
                const uint32_t* fl = reinterpret_cast<const uint32_t*>(fibbase + job.fib_off);
                for (uint32_t m = 0; m < 4; m++) {
                    uint32_t fe[4], sl = 40;
                    for (uint32_t k = 0; k < 4; k++) {
                        const uint32_t l = fl[4 * m + k];
                        fe[k] = 0;
                        if (l == 0) continue;
                        const uint32_t e = tsum(outs[(uint64_t)j * T_COUNT + T_FIB + 4 * m + k]);
                        const uint32_t el = e <= (8u << 20)
                                                ? infos[(uint64_t)j * kModels + kFibModel + 4 * m + k].mat_len + 16 + e
                                                : 0xFFFFFFFFu;
                        fe[k] = el < l ? el : l;
                        sl += fe[k];
                    }
                    if (sl < best) {
                        best = sl;
                        choice = 2;
                        p.s4_sheaf = m;
                        for (uint32_t k = 0; k < 4; k++) p.fe[k] = fe[k];
                    }
                }
            } else if (vans && (vsz < lit || !raw_ok)) {
                choice = 1;
            }
            if (choice == 0 && !raw_ok && vans) choice = 1;  // the raw bytes would be misread as a container
            if (choice == 1) { p.s4_mode = 1; p.l4 = vsz; }
            else if (choice == 2) { p.s4_mode = 2; p.l4 = best; }
            else if (!raw_ok) fallback = true;
        }
        const bool ext = n > 65535 || p.l2 > 65535 || p.l3 > 65535 || p.wlog > 16;
        p.flags = (p.s4_mode ? 0x80u : 0u) | (ext ? 0x08u : 0u);
        const uint64_t comp = 8ull + (ext ? 6 : 4) + 8 + p.l2 + p.l3 + p.l4;
        if (fallback || comp >= n) { p.uncompressed = 1; p.flags = 0x04; p.frame_size = 8 + n; }
        else p.frame_size = (uint32_t)comp;
    }
    plans[j] = p;
    sizes[j] = p.frame_size;
}

constexpr int kAsmThreads = 256;

// Block-wide copy: byte stores up to the first 16-byte boundary of d, then
// one aligned 16-byte store per thread per step (the source words are
// loaded aligned and funnel-shifted into place), then the tail bytes.
// Source buffers are padded, so reading up to 3 bytes past s + n is safe.
__device__ void block_copy(uint8_t* __restrict__ d, const uint8_t* __restrict__ s, uint32_t n) {
    const uint32_t head = min(n, (uint32_t)((16 - (reinterpret_cast<uintptr_t>(d) & 15)) & 15));
    for (uint32_t i = threadIdx.x; i < head; i += blockDim.x) d[i] = s[i];
    d += head;
    s += head;
    n -= head;
    const uint32_t nv = n / 16;
    const uint32_t so = (uint32_t)(reinterpret_cast<uintptr_t>(s) & 3);
    const uint32_t* s4 = reinterpret_cast<const uint32_t*>(reinterpret_cast<uintptr_t>(s) & ~uintptr_t(3));
    uint4* d4 = reinterpret_cast<uint4*>(d);
    for (uint32_t v = threadIdx.x; v < nv; v += blockDim.x) {
        const uint32_t* p = s4 + 4 * v;
        uint4 o;
        if (so == 0) {
            o = make_uint4(p[0], p[1], p[2], p[3]);
        } else {
            const uint32_t sh = 8 * so, w4 = p[4];
            o = make_uint4(__funnelshift_r(p[0], p[1], sh), __funnelshift_r(p[1], p[2], sh),
                           __funnelshift_r(p[2], p[3], sh), __funnelshift_r(p[3], w4, sh));
        }
        d4[v] = o;
    }
    for (uint32_t i = 16 * nv + threadIdx.x; i < n; i += blockDim.x) d[i] = s[i];
}
__device__ inline void put32(uint8_t* p, uint32_t v) {
    p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
}

// container: 'V','A',01,flags | LE32 n | [matrix] | 4 x LE32 state | stream.
// Writes everything but the stream; returns the stream's offset.
__device__ uint32_t container_head(uint8_t* dst, uint8_t flags, uint32_t n, const TableInfo* info, const TaskOut& o) {
    const uint32_t h = 8 + (info ? info->mat_len : 0);
    if (threadIdx.x == 0) {
        dst[0] = 'V'; dst[1] = 'A'; dst[2] = 0x01; dst[3] = flags;
        put32(dst + 4, n);
        for (int k = 0; k < 4; k++) put32(dst + h + 4 * k, o.state[k]);
    }
    if (info) block_copy(dst + 8, info->mat, info->mat_len);
    return h + 16;
}

__device__ void write_container(uint8_t* dst, uint8_t flags, uint32_t n, const TableInfo* info, const TaskOut& o,
                                const uint8_t* task_base, uint32_t cap) {
    block_stitch<kAsmThreads>(task_base, cap, n, dst + container_head(dst, flags, n, info, o));
}

// Frame assembly as independent parts, one block each: part 0 of a frame
// writes its header and Sections 2 and 3 and the head of Section 4; part
// k + 1 writes bytes [k kAsmChunk, (k + 1) kAsmChunk) of the Section 4
// literals (raw) or the k-th stitch pass of their V-ANS stream, at the
// offset recorded by the rANS lanes, or that slice of an uncompressed frame.
// So a frame's literals are written by many blocks at once, and every part
// writes bytes no other part writes.
constexpr uint32_t kAsmChunk = 4 * kStitchRounds;  // literal bytes (symbols) per part
static_assert(16 * kAsmThreads == kStitchRounds, "a literal part is one stitch pass");

// Parts after part 0: the literal chunks, and for P3 four more (the four
// fibers of a foliation take at most floor(n / kAsmChunk) + 4 chunks).
__host__ __device__ inline uint32_t asm_lit_parts(const Job& j) {
    return j.n == 0 ? 0u : (j.lit_cap + kAsmChunk - 1) / kAsmChunk + (j.profile >= 3 ? 4u : 0u);
}

// Sheaf container (assembleSheafContainer, literals.go:645-662): 'V','A',01,
// 0x01 | 0x04 | mode << 4, LE32 n, LE32 fiber lengths x 4, LE32 fiber bytes
// x 4, then the fibers; a coded fiber is its V-ANS body (matrix, four
// states, stream).  The head: the 40 bytes and every coded fiber's matrix
// and states.
__device__ void sheaf_head(const Job& job, const Plan& p, uint32_t j, uint32_t n, const uint8_t* fibbase,
                           const TableInfo* infos, const TaskOut* outs, uint8_t* s4) {
    const uint32_t m = p.s4_sheaf;
    const uint32_t* fl = reinterpret_cast<const uint32_t*>(fibbase + job.fib_off) + 4 * m;
    if (threadIdx.x == 0) {
        s4[0] = 'V'; s4[1] = 'A'; s4[2] = 0x01; s4[3] = (uint8_t)(0x01 | 0x04 | (m << 4));
        put32(s4 + 4, n);
        for (int k = 0; k < 4; k++) { put32(s4 + 8 + 4 * k, fl[k]); put32(s4 + 24 + 4 * k, p.fe[k]); }
    }
    uint32_t o = 40;
    for (uint32_t k = 0; k < 4; k++) {
        if (fl[k] && p.fe[k] < fl[k]) {
            const TableInfo* inf = infos + (uint64_t)j * kModels + kFibModel + 4 * m + k;
            const TaskOut& to = outs[(uint64_t)j * T_COUNT + T_FIB + 4 * m + k];
            const uint32_t ml = inf->mat_len;
            block_copy(s4 + o, inf->mat, ml);
            if (threadIdx.x < 4) put32(s4 + o + ml + 4 * threadIdx.x, to.state[threadIdx.x]);
        }
        o += p.fe[k];
    }
}

// Chunk q of the chosen foliation's fibers (fiber after fiber, kAsmChunk
// symbols each): a stitch pass of a coded fiber or a slice of a raw one.
__device__ void sheaf_part(const Job& job, const Plan& p, uint32_t j, uint32_t q, const uint8_t* fibbase,
                           const TableInfo* infos, const TaskOut* outs, const uint8_t* abase, uint8_t* s4) {
    const uint32_t m = p.s4_sheaf;
    const uint32_t* fl = reinterpret_cast<const uint32_t*>(fibbase + job.fib_off);
    uint32_t o = 40;
    for (uint32_t k = 0; k < 4; k++) {
        const uint32_t l = fl[4 * m + k], passes = (l + kAsmChunk - 1) / kAsmChunk;
        if (q < passes) {
            const FibGeom g = fib_geom(job, fl, m, k);
            if (p.fe[k] < l) {
                const uint8_t* tb = abase + g.ans_off;
                const TaskOut to = outs[(uint64_t)j * T_COUNT + T_FIB + 4 * m + k];
                const uint32_t h = infos[(uint64_t)j * kModels + kFibModel + 4 * m + k].mat_len + 16;
                const uint32_t r0 = q * kStitchRounds;
                stitch_pass<kAsmThreads>(tb, l, l, r0, s4 + o + h + stitch_offset(tb, l, l, to, r0));
            } else {
                const uint32_t lo = q * kAsmChunk;
                block_copy(s4 + o + lo, fibbase + job.fib_off + g.byte_off + lo, min(kAsmChunk, l - lo));
            }
            return;
        }
        q -= passes;
        o += p.fe[k];
    }
}

// Four blocks per SM (64 registers): the parts are short and latency-bound.
__global__ void __launch_bounds__(kAsmThreads, 4) k_assemble(const uint8_t* __restrict__ in, const Job* __restrict__ jobs,
                                                          const uint2* __restrict__ items, uint32_t nitems,
                                                          const uint32_t* __restrict__ job_lens,
                                                          const Plan* __restrict__ plans, const TableInfo* __restrict__ infos,
                                                          const TaskOut* __restrict__ outs,
                                                          const uint8_t* __restrict__ streams,
                                                          const uint8_t* __restrict__ ans,
                                                          const uint8_t* __restrict__ s3base,
                                                          const S3Frame* __restrict__ s3f,
                                                          const uint8_t* __restrict__ fibbase, uint8_t* __restrict__ out) {
    for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        const uint32_t j = items[it].x, part = items[it].y;
        const Job job = jobs[j];
        const Plan p = plans[j];
        const uint32_t* lens = job_lens + (uint64_t)j * S_COUNT;
        uint8_t* f = out + job.out_off;
        const uint32_t n = job.n;
        __syncthreads();
        if (n == 0) continue;
        if (p.uncompressed) {
            if (part == 0) {
                if (threadIdx.x == 0) {
                    f[0] = 'P'; f[1] = 'R'; f[2] = 'Z'; f[3] = 'M'; f[4] = 0x04;
                    f[5] = (uint8_t)n; f[6] = (uint8_t)(n >> 8); f[7] = (uint8_t)(n >> 16);
                }
            } else {
                const uint32_t lo = (part - 1) * kAsmChunk;
                if (lo < n) block_copy(f + 8 + lo, in + job.in_off + lo, min(kAsmChunk, n - lo));
            }
            continue;
        }
        const bool ext = (p.flags & 0x08) != 0;
        uint32_t w = 8 + (ext ? 6 : 4);
        const uint8_t* sreg = streams + job.str_off;
        const uint8_t* abase = ans + job.ans_off;
        uint8_t* s4 = f + w + 8 + p.l2 + p.l3;
        if (part > 0) {  // Section 4 literals, part - 1
            const uint32_t k = part - 1, len = lens[S_LIT];
            if (p.s4_mode == 2) {
                sheaf_part(job, p, j, k, fibbase, infos, outs, abase, s4);
            } else if (p.s4_mode == 1) {
                const uint32_t r0 = k * kStitchRounds;
                if (r0 < (len + 3) / 4) {
                    const TaskOut to = outs[(uint64_t)j * T_COUNT + T_LIT];
                    const uint8_t* tb = abase + ans_task_off(job, T_LIT);
                    const uint32_t cap = task_cap(job, T_LIT);
                    const uint32_t h = 8 + infos[(uint64_t)j * kModels].mat_len + 16;
                    stitch_pass<kAsmThreads>(tb, cap, len, r0, s4 + h + stitch_offset(tb, cap, len, to, r0));
                }
            } else {
                const uint32_t lo = k * kAsmChunk;
                if (lo < len) block_copy(s4 + lo, sreg + stream_base(job, S_LIT) + lo, min(kAsmChunk, len - lo));
            }
            continue;
        }
        if (threadIdx.x == 0) {
            f[0] = 'P'; f[1] = 'R'; f[2] = 'Z'; f[3] = 'M'; f[4] = (uint8_t)p.flags;
            f[5] = (uint8_t)n; f[6] = (uint8_t)(n >> 8); f[7] = (uint8_t)(n >> 16);
            if (!ext) {
                f[8] = (uint8_t)p.l2; f[9] = (uint8_t)(p.l2 >> 8);
                f[10] = (uint8_t)p.l3; f[11] = (uint8_t)(p.l3 >> 8);
            } else {
                f[8] = (uint8_t)p.l2; f[9] = (uint8_t)(p.l2 >> 8); f[10] = (uint8_t)(p.l2 >> 16);
                f[11] = (uint8_t)p.l3; f[12] = (uint8_t)(p.l3 >> 8); f[13] = (uint8_t)(p.l3 >> 16);
            }
            for (int k = 0; k < 8; k++) f[w + k] = 0;
            f[w + 1] = (uint8_t)p.wlog;
        }
        w += 8;
        // Section 2
        uint8_t* s2 = f + w;
        if (job.profile == 0) {
            if (threadIdx.x == 0) { s2[0] = 0x00; put32(s2 + 1, lens[S_CMD]); }
            block_copy(s2 + 5, sreg + stream_base(job, S_CMD), lens[S_CMD]);
        } else if (p.s2_mode == 2) {
            if (threadIdx.x == 0) s2[0] = 0x09;
            block_copy(s2 + 1, sreg + stream_base(job, S_CMD), lens[S_CMD]);
        } else {
            if (threadIdx.x == 0) {
                s2[0] = 0x08;
                put32(s2 + 1, lens[S_CMD]);
                put32(s2 + 5, p.sub_len[0]);
                put32(s2 + 9, p.sub_len[1]);
            }
            uint32_t o = 13;
            for (int sub = 0; sub < 3; sub++) {
                const uint32_t len = lens[S_OP + sub];
                uint8_t* d = s2 + o;
                if (p.sub_mode[sub] == 0) {
                    if (threadIdx.x == 0) d[0] = 0x09;
                    block_copy(d + 1, sreg + stream_base(job, S_OP + sub), len);
                } else {
                    const int t = T_OP_M8 + 2 * sub + (p.sub_mode[sub] == 2 ? 1 : 0);
                    const TaskOut to = outs[(uint64_t)j * T_COUNT + t];
                    if (p.sub_mode[sub] == 1)
                        write_container(d, 0x41, len, nullptr, to, abase + ans_task_off(job, t), task_cap(job, t));
                    else
                        write_container(d, 0x00, len, infos + (uint64_t)j * kModels + 1 + sub, to, abase + ans_task_off(job, t),
                                        task_cap(job, t));
                }
                o += p.sub_len[sub];
            }
        }
        w += p.l2;
        // Section 3
        uint8_t* s3 = f + w;
        if (job.profile < 2) {  // flat
            if (threadIdx.x == 0) { s3[0] = 0x00; put32(s3 + 1, lens[S_OFF]); }
            block_copy(s3 + 5, sreg + stream_base(job, S_OFF), lens[S_OFF]);
        } else if (p.s3_form == 2) {  // 0x09 + the varints
            if (threadIdx.x == 0) s3[0] = 0x09;
            block_copy(s3 + 1, sreg + stream_base(job, S_OFF), lens[S_OFF]);
        } else if (p.s3_form == 1) {  // distance-prefix container
            const S3Frame fr = s3f[j];
            const uint32_t h = p.s3_hlen, orig = fr.orig, nd = fr.nd, cl = p.s3_cl;
            if (threadIdx.x == 0) {
                if (h == 4) {
                    s3[0] = 0x0B; s3[1] = (uint8_t)orig; s3[2] = (uint8_t)nd; s3[3] = (uint8_t)cl;
                } else if (h == 7) {
                    s3[0] = 0x0A;
                    s3[1] = (uint8_t)orig; s3[2] = (uint8_t)(orig >> 8);
                    s3[3] = (uint8_t)nd; s3[4] = (uint8_t)(nd >> 8);
                    s3[5] = (uint8_t)cl; s3[6] = (uint8_t)(cl >> 8);
                } else {
                    s3[0] = 0x06; put32(s3 + 1, orig); put32(s3 + 5, nd); put32(s3 + 9, cl);
                }
            }
            uint8_t* cs = s3 + h;
            const uint8_t* rb = s3base + job.s3_off;
            if (p.s3_code == 0) {  // Mode 12: 0x0C | LE32 state | the emitted bytes reversed
                if (threadIdx.x == 0) { cs[0] = 0x0C; put32(cs + 1, fr.m12x); }
                const uint8_t* em = rb + s3_em_off(job);
                const uint32_t e = fr.m12e;
                for (uint32_t k = threadIdx.x; k < e; k += blockDim.x) cs[5 + k] = em[e - 1 - k];
            } else {
                write_container(cs, 0x00, nd, infos + (uint64_t)j * kModels + 4, outs[(uint64_t)j * T_COUNT + T_S3],
                                abase + ans_task_off(job, T_S3), task_cap(job, T_S3));
            }
            block_copy(cs + cl, rb + s3_extra_off(job), p.s3_xl);
        }
        // Section 4: the container head here, the literals in parts 1, 2, ...
        if (p.s4_mode == 1)
            container_head(s4, 0x00, lens[S_LIT], infos + (uint64_t)j * kModels, outs[(uint64_t)j * T_COUNT + T_LIT]);
        else if (p.s4_mode == 2)
            sheaf_head(job, p, j, lens[S_LIT], fibbase, infos, outs, s4);
    }
}

}  // namespace pz
