/*
 * przm_oracle.c -- CPU restatement of the PRZM GPU compression path, and of
 * the two section encoders it widens into (Section 3 distance coding,
 * Section 4 selection with the sheaf foliations).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product is
 * compared against; it is never linked into, called by, or used as a fallback
 * for the product library.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py load it.
 *
 * Every function restates one piece of the reference (Lemon4ksan/przm) and
 * cites the file:line it follows.  Two reference kernels are racy on a GPU
 * (gpu/kernel/przm_lz77.cu:177-178 and :350-355); for those the restatement
 * fixes the sequential ("canonical") semantics that the kernels intend:
 *   - radix strike: the predecessor of an 8-aligned position p is the latest
 *     8-aligned q < p with the same 19-bit k-mer hash (table insert order);
 *   - tile finder: within each 256-position step, bucket updates happen in
 *     ascending position order, so a bucket ends the step holding the largest
 *     p+1 (high half) and the next-largest p+1 of that step, or the bucket's
 *     previous head when only one position of the step hit it (low half).
 *
 * Parity pin: the reference's Go code cannot be built here (no Go toolchain),
 * and the reference GPU path ships no golden vectors.  The restatement is
 * pinned by (1) the known-answer properties the reference's own tests state
 * (tests/test_oracle.py), (2) byte-exact round trips of every stream and frame
 * through the reference's own C99 decoder (src/przm_dec.c, built from its
 * sources by oracle/Makefile into oracle/_ref/), and (3) on a GPU, comparison
 * with the reference's own deterministic CUDA kernels (tokenizer, histogram,
 * V-ANS) built from gpu/kernel/przm_lz77.cu into oracle/_ref/.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../przm_b200/csrc/meta8_tables.h"
#include "../przm_b200/csrc/dist_tables.h"

#define OR_TILE 32768u
#define OR_BUCKETS 2048u
#define OR_HASH_PRIME 0x1E35A7BDu
#define OR_RADIX_BUCKETS 524288u
#define OR_RADIX_PRIME 0x9E3779B97F4A7C15ull
#define OR_WINDOW (1024u * 1024u)
#define OR_MAX_LEN32 4095u
#define OR_MAX_OFF32 1048575u

static inline uint32_t rd32(const uint8_t *p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static inline uint64_t rd64(const uint8_t *p) { return (uint64_t)rd32(p) | ((uint64_t)rd32(p + 4) << 32); }
static inline void wr32(uint8_t *p, uint32_t v) {
    p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
}

/* przm_lz77.h:53-60 / gpu/types.go:27-33 */
uint32_t or_pack_match32(uint32_t length, uint32_t offset) {
    if (length < 4 || offset == 0) return 0;
    uint32_t l = length > OR_MAX_LEN32 ? OR_MAX_LEN32 : length;
    return (l << 20) | (offset & 0xFFFFFu);
}

/* przm_lz77.cu:63-85 (first 4 bytes already equal) */
static uint32_t lcp_tile(const uint8_t *a, const uint8_t *b, uint32_t limit) {
    uint32_t len = 4;
    while (len + 4 <= limit) {
        uint32_t d = rd32(a + len) ^ rd32(b + len);
        if (d) return len + (uint32_t)__builtin_ctz(d) / 8;
        len += 4;
    }
    while (len < limit && a[len] == b[len]) len++;
    return len;
}

static inline uint32_t hash4(uint32_t w) { return ((w * OR_HASH_PRIME) >> 21) & (OR_BUCKETS - 1); }

/* Shared-memory tile finder, przm_lz77.cu:221-360, with the canonical bucket
 * update described in the header.  Writes desc[] for every position of every
 * tile (positions with p + 4 > tile_len get 0).  window is the byte window
 * passed by the host (gpu/bridge.go:931: 1 MiB). */
void or_tile_find(const uint8_t *in, uint64_t n, uint32_t window, uint32_t *desc) {
    uint32_t head[OR_BUCKETS];
    uint32_t w4s[256], hs[256];
    int valids[256];
    for (uint64_t ts = 0; ts < n; ts += OR_TILE) {
        uint32_t tl = (uint32_t)((n - ts) < OR_TILE ? (n - ts) : OR_TILE);
        const uint8_t *t = in + ts;
        memset(head, 0, sizeof head);
        uint32_t steps = (tl + 255) / 256;
        for (uint32_t st = 0; st < steps; st++) {
            for (uint32_t tid = 0; tid < 256; tid++) {
                uint32_t p = st * 256 + tid;
                valids[tid] = (p + 4 <= tl);
                w4s[tid] = valids[tid] ? rd32(t + p) : 0;
                hs[tid] = valids[tid] ? hash4(w4s[tid]) : 0;
            }
            for (uint32_t tid = 0; tid < 256; tid++) {
                uint32_t p = st * 256 + tid, lane = tid & 31, d = 0;
                if (valids[tid]) {
                    uint32_t best_len = 0, best_off = 0;
                    uint32_t lim = tl - p;
                    if (lim > OR_MAX_LEN32) lim = OR_MAX_LEN32;
                    for (uint32_t delta = 1; delta <= 4; delta++) {
                        if (lane >= delta && w4s[tid - delta] == w4s[tid]) {
                            uint32_t l = lcp_tile(t + p, t + p - delta, lim);
                            if (l > best_len) { best_len = l; best_off = delta; }
                        }
                    }
                    uint32_t bv = head[hs[tid]];
                    uint32_t c16[2] = {bv >> 16, bv & 0xFFFFu};
                    for (int k = 0; k < 2; k++) {
                        if (c16[k] == 0) continue;
                        if (k == 1 && best_len >= 258) continue;
                        uint32_t c = c16[k] - 1;
                        if (c >= p) continue;
                        uint32_t dist = p - c;
                        if (dist > window || dist == 0) continue;
                        if (rd32(t + c) != w4s[tid]) continue;
                        uint32_t l = lcp_tile(t + p, t + c, lim);
                        if (l > best_len) { best_len = l; best_off = dist; }
                    }
                    if (best_len >= 4 && best_off <= OR_MAX_OFF32) d = or_pack_match32(best_len, best_off);
                }
                if (p < tl) desc[ts + p] = d;
            }
            /* canonical update: ascending p (przm_lz77.cu:350-355 intent) */
            for (uint32_t tid = 0; tid < 256; tid++) {
                if (!valids[tid]) continue;
                uint32_t p = st * 256 + tid;
                uint32_t old = head[hs[tid]];
                head[hs[tid]] = ((p + 1) << 16) | (old >> 16);
            }
        }
    }
}

/* Radix-strike finder, przm_lz77.cu:156-213 with the table cleared first
 * (gpu/bridge.go:955-975), run sequentially (canonical predecessor).  desc[]
 * must hold n zeroed entries; only 8-aligned positions are written. */
void or_radix_find(const uint8_t *in, uint64_t n, uint32_t window, uint32_t *desc) {
    uint32_t *table = (uint32_t *)calloc(OR_RADIX_BUCKETS, sizeof(uint32_t));
    for (uint64_t p64 = 0; p64 + 8 <= n; p64 += 8) {
        uint32_t p = (uint32_t)p64;
        uint64_t k = rd64(in + p);
        uint32_t h = (uint32_t)((k * OR_RADIX_PRIME) >> 43) & (OR_RADIX_BUCKETS - 1);
        uint32_t prev = table[h];
        table[h] = p + 1;
        if (prev == 0 || prev > p) continue;
        uint32_t c = prev - 1, dist = p - c;
        if (!(dist <= window && dist > 0 && dist <= OR_MAX_OFF32)) continue;
        if (rd64(in + c) != k) continue;
        uint32_t L = 8;
        int done = 0;
        while ((uint64_t)p + L + 8 <= n && (uint64_t)c + L + 8 <= n && L + 8 <= OR_MAX_LEN32) {
            uint64_t d = rd64(in + p + L) ^ rd64(in + c + L);
            if (d) { L += (uint32_t)__builtin_ctzll(d) / 8; done = 1; break; }
            L += 8;
        }
        if (!done)
            while ((uint64_t)p + L < n && in[p + L] == in[c + L] && L < OR_MAX_LEN32) L++;
        desc[p] = or_pack_match32(L, dist);
    }
    free(table);
}

/* launchMatchSearch dispatch used by Tokenize/CompressD2D, gpu/bridge.go:924-950:
 * n <= 65536 -> tile finder, else cleared table + radix strike. */
void or_match_table(const uint8_t *in, uint64_t n, uint32_t *desc) {
    memset(desc, 0, n * sizeof(uint32_t));
    if (n <= 65536) or_tile_find(in, n, OR_WINDOW, desc);
    else or_radix_find(in, n, OR_WINDOW, desc);
}

/* MatchLZ77, gpu/bridge.go:1480-1499: radix strike for every size
 * (launchSlotKernel, :952-1068) followed by ascending compaction
 * (przm_lz77.cu:510-664); n > 16 MiB streams in chunk_size pieces that are
 * searched independently (matchLZ77StreamingLocked, :1216-1458).  Returns the
 * number of matches written to pos/desc (both capacity n). */
uint64_t or_match_lz77_chunked(const uint8_t *in, uint64_t n, uint64_t chunk, uint32_t *pos, uint32_t *dsc) {
    uint64_t cnt = 0;
    if (n == 0) return 0;
    if (chunk == 0 || chunk >= n) chunk = n;
    uint32_t *tab = (uint32_t *)malloc((chunk ? chunk : 1) * sizeof(uint32_t));
    for (uint64_t base = 0; base < n; base += chunk) {
        uint64_t len = (n - base) < chunk ? (n - base) : chunk;
        memset(tab, 0, len * sizeof(uint32_t));
        or_radix_find(in + base, len, OR_WINDOW, tab);
        for (uint64_t i = 0; i < len; i++)
            if (tab[i]) { pos[cnt] = (uint32_t)(base + i); dsc[cnt] = tab[i]; cnt++; }
    }
    free(tab);
    return cnt;
}

uint64_t or_match_lz77(const uint8_t *in, uint64_t n, uint32_t *pos, uint32_t *dsc) {
    return or_match_lz77_chunked(in, n, n > 16u * 1024 * 1024 ? 8u * 1024 * 1024 : 0, pos, dsc);
}

/* matchLZ77StreamingLocked chunk-size rule, gpu/bridge.go:1222-1233 */
uint64_t or_streaming_chunk(uint64_t n, int64_t chunk) {
    uint64_t c;
    if (chunk <= 0) c = (n / 2 > 16u * 1024 * 1024) ? n / 2 : 16u * 1024 * 1024;
    else c = (uint64_t)chunk;
    if (c > 64u * 1024 * 1024) c = 64u * 1024 * 1024;
    return c;
}

/* ---------------------------------------------------------------------------
 * Tokenizer, przm_tokenizer.cuh:33-466, one tile at a time (the kernel's parse
 * decisions are taken serially by lane 0, so a serial walk is exact).
 * ------------------------------------------------------------------------- */
typedef struct { uint8_t *b; uint32_t n; } obuf;

static void put_varint(obuf *o, uint32_t v) { /* przm_tokenizer.cuh:33-55 */
    if (v < 0x80) { o->b[o->n++] = (uint8_t)v; }
    else if (v < 0x4000) { o->b[o->n++] = (uint8_t)(v | 0x80); o->b[o->n++] = (uint8_t)(v >> 7); }
    else if (v < 0x200000) {
        o->b[o->n++] = (uint8_t)(v | 0x80); o->b[o->n++] = (uint8_t)((v >> 7) | 0x80); o->b[o->n++] = (uint8_t)(v >> 14);
    } else if (v < 0x10000000) {
        o->b[o->n++] = (uint8_t)(v | 0x80); o->b[o->n++] = (uint8_t)((v >> 7) | 0x80);
        o->b[o->n++] = (uint8_t)((v >> 14) | 0x80); o->b[o->n++] = (uint8_t)(v >> 21);
    } else {
        o->b[o->n++] = (uint8_t)(v | 0x80); o->b[o->n++] = (uint8_t)((v >> 7) | 0x80);
        o->b[o->n++] = (uint8_t)((v >> 14) | 0x80); o->b[o->n++] = (uint8_t)((v >> 21) | 0x80);
        o->b[o->n++] = (uint8_t)(v >> 28);
    }
}

static void put_litop(obuf *c, uint32_t count) { /* przm_tokenizer.cuh:57-76 */
    if (count == 0) return;
    if (count <= 8) c->b[c->n++] = (uint8_t)(0xF2 + count);
    else if (count < 0x80) { c->b[c->n++] = 0xF0; c->b[c->n++] = (uint8_t)count; }
    else if (count < 0x4000) { c->b[c->n++] = 0xF0; c->b[c->n++] = (uint8_t)(count | 0x80); c->b[c->n++] = (uint8_t)(count >> 7); }
    else { c->b[c->n++] = 0xF0; put_varint(c, count); }
}

static void put_lits(obuf *l, const uint8_t *src, uint32_t count) {
    memcpy(l->b + l->n, src, count);
    l->n += count;
}

/* One tile [start, end) of przm_fused_tokenizer_kernel. */
static void tok_tile(const uint8_t *in, const uint32_t *desc, uint32_t b, uint32_t start, uint32_t end,
                     obuf *cmd, obuf *off, obuf *lit) {
    int rep0 = b == 0 ? 1 : -1, rep1 = b == 0 ? 4 : -1, rep2 = b == 0 ? 8 : -1;
    uint32_t pos = start, litStart = start;
    while (pos < end) {
        uint32_t q = pos;
        while (q < end && desc[q] == 0) q++;
        if (q >= end) break;
        uint32_t mLen = desc[q] >> 20, d = desc[q] & 0xFFFFFu;
        /* lookahead, :196-216 */
        if (q + 1 < end && desc[q + 1] != 0 && (desc[q + 1] >> 20) > mLen + 1) { pos = q + 1; continue; }
        /* RLE, :218-286 */
        if (q + 12 <= end) {
            uint32_t w4 = rd32(in + q);
            uint8_t b0 = (uint8_t)w4;
            if (w4 == (uint32_t)b0 * 0x01010101u) {
                uint32_t r = 4, maxr = end - q;
                if (maxr > 65535) maxr = 65535;
                while (r < maxr && in[q + r] == b0) r++;
                if (r >= 12 && r >= mLen) {
                    if (q > litStart) {
                        put_litop(cmd, q - litStart);
                        put_lits(lit, in + litStart, q - litStart);
                    }
                    cmd->b[cmd->n++] = 0xF1;
                    put_varint(cmd, r);
                    lit->b[lit->n++] = b0;
                    pos = q + r;
                    litStart = pos;
                    continue;
                }
            }
        }
        /* match validity + extension, :289-320 */
        if (!(d > 0 && d <= q && mLen >= 4 && rd32(in + q) == rd32(in + q - d))) { pos = q + 1; continue; }
        if (q + mLen > end) mLen = end - q;
        while (q + mLen < end && in[q + mLen] == in[q - d + mLen] && mLen < 65530) mLen++;
        /* encode, :328-427 */
        int k = -1;
        if ((int)d == rep0 && rep0 > 0) k = 0;
        else if ((int)d == rep1 && rep1 > 0) k = 1;
        else if ((int)d == rep2 && rep2 > 0) k = 2;
        uint32_t litLen = q - litStart;
        uint32_t keep = k >= 0 ? (mLen <= 7 ? 7u : 15u) : 3u;
        if (litLen > keep) {
            put_litop(cmd, litLen - keep);
            put_lits(lit, in + litStart, litLen - keep);
            litStart = q - keep;
            litLen = keep;
        }
        uint32_t base = mLen - 4;
        if (base > 14) base = 15;
        if (k >= 0 && mLen <= 7) {
            cmd->b[cmd->n++] = (uint8_t)((litLen << 4) | ((mLen - 4) << 2) | (uint32_t)k);
        } else if (k >= 0) {
            cmd->b[cmd->n++] = (uint8_t)(0xC0 | k);
            cmd->b[cmd->n++] = (uint8_t)((litLen << 4) | base);
            if (base == 15) put_varint(cmd, mLen - 19);
        } else {
            cmd->b[cmd->n++] = (uint8_t)(0x80 | (litLen << 4) | base);
            if (base == 15) put_varint(cmd, mLen - 19);
        }
        put_lits(lit, in + litStart, litLen);
        if (k < 0) {
            put_varint(off, d);
            rep2 = rep1; rep1 = rep0; rep0 = (int)d;
        } else if (k == 1) {
            rep1 = rep0; rep0 = (int)d;
        } else if (k == 2) {
            rep2 = rep1; rep1 = rep0; rep0 = (int)d;
        }
        pos = q + mLen;
        litStart = pos;
    }
    if (litStart < end) { /* :440-464 */
        put_litop(cmd, end - litStart);
        put_lits(lit, in + litStart, end - litStart);
    }
}

/* Tokenize pipeline (fused tokenizer + scan + gather), przm_tokenizer.cuh:115-609.
 * Output capacities: each buffer must hold the tile-slot total
 * (36864 * tiles), the reference's own bound (gpu/bridge.go:148-153). */
void or_tokenize(const uint8_t *in, uint64_t n, const uint32_t *desc, uint8_t *cmd, uint64_t *ncmd, uint8_t *off,
                 uint64_t *noff, uint8_t *lit, uint64_t *nlit) {
    obuf c = {cmd, 0}, o = {off, 0}, l = {lit, 0};
    /* one tile at a time; streams stay contiguous (gather == concatenation) */
    uint64_t tiles = (n + OR_TILE - 1) / OR_TILE;
    uint64_t tc = 0, to = 0, tl = 0;
    for (uint64_t b = 0; b < tiles; b++) {
        uint32_t s = (uint32_t)(b * OR_TILE), e = (uint32_t)((b + 1) * OR_TILE > n ? n : (b + 1) * OR_TILE);
        obuf cc = {cmd + tc, 0}, oo = {off + to, 0}, ll = {lit + tl, 0};
        tok_tile(in, desc, (uint32_t)b, s, e, &cc, &oo, &ll);
        tc += cc.n; to += oo.n; tl += ll.n;
    }
    (void)c; (void)o; (void)l;
    *ncmd = tc; *noff = to; *nlit = tl;
}

/* Per-tile variant used by tests: lengths of each tile's streams. */
void or_tokenize_tiles(const uint8_t *in, uint64_t n, const uint32_t *desc, uint32_t *lens /* 3 per tile */) {
    uint64_t tiles = (n + OR_TILE - 1) / OR_TILE;
    uint8_t *cb = (uint8_t *)malloc(36864), *ob = (uint8_t *)malloc(36864), *lb = (uint8_t *)malloc(36864);
    for (uint64_t b = 0; b < tiles; b++) {
        uint32_t s = (uint32_t)(b * OR_TILE), e = (uint32_t)((b + 1) * OR_TILE > n ? n : (b + 1) * OR_TILE);
        obuf cc = {cb, 0}, oo = {ob, 0}, ll = {lb, 0};
        tok_tile(in, desc, (uint32_t)b, s, e, &cc, &oo, &ll);
        lens[3 * b] = cc.n; lens[3 * b + 1] = oo.n; lens[3 * b + 2] = ll.n;
    }
    free(cb); free(ob); free(lb);
}

/* ---------------------------------------------------------------------------
 * Command split, core/commands/commands.go:18-202 (opcodes produced by the
 * tokenizer only: <0x80, 0x80-0xBF, 0xC0-0xC3, 0xF0, 0xF1, 0xF3-0xFA).
 * Returns 0 on success, -1 on a malformed stream.
 * ------------------------------------------------------------------------- */
static int take_varint(const uint8_t *src, uint64_t n, uint64_t *sp, uint8_t *v, uint64_t *nv) {
    for (int i = 0; i < 4; i++) { /* consumeVarint, commands.go:187-202 */
        if (*sp >= n) return -1;
        uint8_t b = src[(*sp)++];
        v[(*nv)++] = b;
        if (!(b & 0x80)) return 0;
    }
    return -1;
}

int or_split_commands(const uint8_t *src, uint64_t n, uint8_t *op, uint64_t *nop, uint8_t *meta, uint64_t *nm,
                      uint8_t *var, uint64_t *nv) {
    uint64_t sp = 0, a = 0, b = 0, c = 0;
    while (sp < n) {
        uint8_t o = src[sp++];
        op[a++] = o;
        if (o < 0x80) continue;
        if (o < 0xC0) {
            if ((o & 15) == 15 && take_varint(src, n, &sp, var, &c)) return -1;
            continue;
        }
        if (o <= 0xC3) { /* splitLongRepeat, :70-83 */
            if (sp >= n) return -1;
            uint8_t t = src[sp++];
            meta[b++] = t;
            if ((t & 15) == 15 && take_varint(src, n, &sp, var, &c)) return -1;
            continue;
        }
        if (o == 0xF0 || o == 0xF1) { if (take_varint(src, n, &sp, var, &c)) return -1; continue; }
        if (o >= 0xF3 && o <= 0xFA) continue;
        return -1; /* opcode families the tokenizer never produces */
    }
    *nop = a; *nm = b; *nv = c;
    return 0;
}

/* ---------------------------------------------------------------------------
 * Frequency normalisation.
 * ------------------------------------------------------------------------- */

/* literals.NormalizeFrequencies + adjustFrequencySum, core/literals/literals.go:78-140 */
void or_normalize_frequencies(const uint32_t *counts_in, uint16_t *freq) {
    int64_t counts[256];
    int64_t total = 0;
    int unique = 0;
    for (int s = 0; s < 256; s++) {
        counts[s] = counts_in[s];
        freq[s] = 0;
        if (counts[s] > 0) { total += counts[s]; unique++; }
    }
    if (unique == 0) return;
    int64_t remaining = 4096 - unique;
    uint32_t sum = 0;
    for (int s = 0; s < 256; s++) {
        if (counts[s] <= 0) continue;
        int64_t share = (counts[s] * remaining) / total;
        freq[s] = (uint16_t)(1 + share);
        sum += freq[s];
    }
    int diff = 4096 - (int)(uint16_t)sum;
    if (diff > 0) {
        for (int it = 0; it < diff; it++) {
            int best = -1;
            int64_t bc = -1;
            for (int s = 0; s < 256; s++)
                if (counts[s] > bc && freq[s] > 0) { bc = counts[s]; best = s; }
            if (best >= 0) { freq[best]++; counts[best] = -1; }
        }
    } else if (diff < 0) {
        for (int it = 0; it < -diff; it++)
            for (int s = 255; s >= 0; s--)
                if (freq[s] > 1) { freq[s]--; break; }
    }
}

/* gpu.NormalizeFreq, gpu/bridge.go:2777-2829.  Its tie order comes from Go's
 * sort.Slice, which is pdqsort (Go standard library, sort/zsortfunc.go, Go >=
 * 1.19; the reference pins go 1.27 in go.mod).  The published algorithm is
 * restated below so ties between equal remainders land where Go puts them. */
typedef struct { int sym; uint64_t rem; } or_rem_t;
typedef struct { or_rem_t *v; } go_slice;

static int go_less(go_slice *d, int i, int j) { return d->v[i].rem > d->v[j].rem; }
static void go_swap(go_slice *d, int i, int j) { or_rem_t t = d->v[i]; d->v[i] = d->v[j]; d->v[j] = t; }

static void go_insertion(go_slice *d, int a, int b) {
    for (int i = a + 1; i < b; i++)
        for (int j = i; j > a && go_less(d, j, j - 1); j--) go_swap(d, j, j - 1);
}
static void go_sift_down(go_slice *d, int lo, int hi, int first) {
    int root = lo;
    for (;;) {
        int child = 2 * root + 1;
        if (child >= hi) return;
        if (child + 1 < hi && go_less(d, first + child, first + child + 1)) child++;
        if (!go_less(d, first + root, first + child)) return;
        go_swap(d, first + root, first + child);
        root = child;
    }
}
static void go_heap_sort(go_slice *d, int a, int b) {
    int first = a, lo = 0, hi = b - a;
    for (int i = (hi - 1) / 2; i >= 0; i--) go_sift_down(d, i, hi, first);
    for (int i = hi - 1; i >= 0; i--) { go_swap(d, first, first + i); go_sift_down(d, lo, i, first); }
}
static int go_bits_len(unsigned x) { int n = 0; while (x) { n++; x >>= 1; } return n; }
static void go_break_patterns(go_slice *d, int a, int b) {
    int length = b - a;
    if (length >= 8) {
        uint64_t r = (uint64_t)length;
        unsigned modulus = 1u << go_bits_len((unsigned)length);
        int idx = a + (length / 4) * 2 - 1;
        for (int i = 0; i < 3; i++) {
            r ^= r << 13; r ^= r >> 7; r ^= r << 17;
            int other = (int)((unsigned)r & (modulus - 1));
            if (other >= length) other -= length;
            go_swap(d, idx - 1 + i, a + other);
        }
    }
}
static void go_order2(go_slice *d, int *a, int *b, int *swaps) {
    if (go_less(d, *b, *a)) { int t = *a; *a = *b; *b = t; (*swaps)++; }
}
static int go_median(go_slice *d, int a, int b, int c, int *swaps) {
    go_order2(d, &a, &b, swaps);
    go_order2(d, &b, &c, swaps);
    go_order2(d, &a, &b, swaps);
    return b;
}
enum { GO_UNKNOWN = 0, GO_INCREASING = 1, GO_DECREASING = 2 };
static int go_choose_pivot(go_slice *d, int a, int b, int *hint) {
    int l = b - a, swaps = 0;
    int i = a + l / 4 * 1, j = a + l / 4 * 2, k = a + l / 4 * 3;
    if (l >= 8) {
        if (l >= 50) {
            i = go_median(d, i - 1, i, i + 1, &swaps);
            j = go_median(d, j - 1, j, j + 1, &swaps);
            k = go_median(d, k - 1, k, k + 1, &swaps);
        }
        j = go_median(d, i, j, k, &swaps);
    }
    *hint = swaps == 0 ? GO_INCREASING : (swaps == 12 ? GO_DECREASING : GO_UNKNOWN);
    return j;
}
static void go_reverse(go_slice *d, int a, int b) {
    for (int i = a, j = b - 1; i < j; i++, j--) go_swap(d, i, j);
}
static int go_partial_insertion(go_slice *d, int a, int b) {
    int i = a + 1;
    for (int step = 0; step < 5; step++) {
        while (i < b && !go_less(d, i, i - 1)) i++;
        if (i == b) return 1;
        if (b - a < 50) return 0;
        go_swap(d, i, i - 1);
        if (i - a >= 2)
            for (int j = i - 1; j >= 1; j--) { if (!go_less(d, j, j - 1)) break; go_swap(d, j, j - 1); }
        if (b - i >= 2)
            for (int j = i + 1; j < b; j++) { if (!go_less(d, j, j - 1)) break; go_swap(d, j, j - 1); }
    }
    return 0;
}
static int go_partition_equal(go_slice *d, int a, int b, int pivot) {
    go_swap(d, a, pivot);
    int i = a + 1, j = b - 1;
    for (;;) {
        while (i <= j && !go_less(d, a, i)) i++;
        while (i <= j && go_less(d, a, j)) j--;
        if (i > j) break;
        go_swap(d, i, j); i++; j--;
    }
    return i;
}
static int go_partition(go_slice *d, int a, int b, int pivot, int *already) {
    go_swap(d, a, pivot);
    int i = a + 1, j = b - 1;
    while (i <= j && go_less(d, i, a)) i++;
    while (i <= j && !go_less(d, j, a)) j--;
    if (i > j) { go_swap(d, j, a); *already = 1; return j; }
    go_swap(d, i, j); i++; j--;
    for (;;) {
        while (i <= j && go_less(d, i, a)) i++;
        while (i <= j && !go_less(d, j, a)) j--;
        if (i > j) break;
        go_swap(d, i, j); i++; j--;
    }
    go_swap(d, j, a);
    *already = 0;
    return j;
}
static void go_pdqsort(go_slice *d, int a, int b, int limit) {
    int was_balanced = 1, was_partitioned = 1;
    for (;;) {
        int length = b - a;
        if (length <= 12) { go_insertion(d, a, b); return; }
        if (limit == 0) { go_heap_sort(d, a, b); return; }
        if (!was_balanced) { go_break_patterns(d, a, b); limit--; }
        int hint;
        int pivot = go_choose_pivot(d, a, b, &hint);
        if (hint == GO_DECREASING) {
            go_reverse(d, a, b);
            pivot = (b - 1) - (pivot - a);
            hint = GO_INCREASING;
        }
        if (was_balanced && was_partitioned && hint == GO_INCREASING)
            if (go_partial_insertion(d, a, b)) return;
        if (a > 0 && !go_less(d, a - 1, pivot)) {
            a = go_partition_equal(d, a, b, pivot);
            continue;
        }
        int already;
        int mid = go_partition(d, a, b, pivot, &already);
        was_partitioned = already;
        int left = mid - a, right = b - mid, thr = length / 8;
        if (left < right) {
            was_balanced = left >= thr;
            go_pdqsort(d, a, mid, limit);
            a = mid + 1;
        } else {
            was_balanced = right >= thr;
            go_pdqsort(d, mid + 1, b, limit);
            b = mid;
        }
    }
}

void or_normalize_freq(const uint32_t *counts, uint32_t target, uint16_t *norm) {
    uint64_t total = 0;
    int active = 0;
    for (int s = 0; s < 256; s++) {
        norm[s] = 0;
        total += counts[s];
        if (counts[s]) active++;
    }
    if (total == 0 || active == 0) return;
    if ((uint32_t)active >= target) {
        for (int s = 0; s < 256; s++) norm[s] = (uint16_t)(target / 256);
        return;
    }
    uint32_t rt = target - (uint32_t)active, alloc = 0;
    or_rem_t rems[256];
    int nr = 0;
    for (int s = 0; s < 256; s++) {
        if (!counts[s]) continue;
        uint64_t prod = (uint64_t)counts[s] * rt;
        uint32_t add = (uint32_t)(prod / total);
        norm[s] = (uint16_t)(1 + add);
        alloc += 1 + add;
        rems[nr].sym = s;
        rems[nr].rem = prod % total;
        nr++;
    }
    if (alloc < target) {
        int diff = (int)(target - alloc);
        go_slice d = {rems};
        go_pdqsort(&d, 0, nr, go_bits_len((unsigned)nr));
        for (int i = 0; i < diff && i < nr; i++) norm[rems[i].sym]++;
    }
}

/* True when equal remainders straddle the +1 cutoff of NormalizeFreq, the
 * only case in which the result depends on the sort's tie order. */
int or_normalize_freq_tie_straddles(const uint32_t *counts, uint32_t target) {
    uint64_t total = 0;
    int active = 0;
    for (int s = 0; s < 256; s++) { total += counts[s]; if (counts[s]) active++; }
    if (total == 0 || (uint32_t)active >= target) return 0;
    uint32_t rt = target - (uint32_t)active, alloc = 0;
    uint64_t rem[256];
    int nr = 0;
    for (int s = 0; s < 256; s++) {
        if (!counts[s]) continue;
        uint64_t prod = (uint64_t)counts[s] * rt;
        alloc += 1 + (uint32_t)(prod / total);
        rem[nr++] = prod % total;
    }
    if (alloc >= target) return 0;
    int diff = (int)(target - alloc);
    /* sort remainders descending (plain insertion, values only) */
    for (int i = 1; i < nr; i++)
        for (int j = i; j > 0 && rem[j] > rem[j - 1]; j--) { uint64_t t = rem[j]; rem[j] = rem[j - 1]; rem[j - 1] = t; }
    return diff < nr && rem[diff - 1] == rem[diff];
}

/* BuildCDF, gpu/bridge.go:2832-2841 */
void or_build_cdf(const uint16_t *freq, uint16_t *cdf) {
    uint32_t c = 0;
    for (int s = 0; s < 256; s++) { cdf[s] = (uint16_t)c; c += freq[s]; }
    cdf[256] = (uint16_t)c;
}

/* SerializeMatrix, gpu/bridge.go:2844-2886 == EncodeJointNibbleFreq,
 * core/literals/literals.go:143-184 */
uint32_t or_serialize_matrix(const uint16_t *freq, uint8_t *out) {
    uint32_t n = 0;
    uint16_t rowMask = 0;
    for (int h = 0; h < 16; h++)
        for (int l = 0; l < 16; l++)
            if (freq[(h << 4) | l]) { rowMask |= (uint16_t)(1u << h); break; }
    out[n++] = (uint8_t)rowMask; out[n++] = (uint8_t)(rowMask >> 8);
    for (int h = 0; h < 16; h++) {
        if (!(rowMask & (1u << h))) continue;
        uint16_t colMask = 0;
        for (int l = 0; l < 16; l++) if (freq[(h << 4) | l]) colMask |= (uint16_t)(1u << l);
        out[n++] = (uint8_t)colMask; out[n++] = (uint8_t)(colMask >> 8);
        for (int l = 0; l < 16; l++) {
            if (!(colMask & (1u << l))) continue;
            uint16_t w = freq[(h << 4) | l];
            if (w < 128) out[n++] = (uint8_t)w;
            else { out[n++] = (uint8_t)(0x80 | (w >> 8)); out[n++] = (uint8_t)(w & 0xFF); }
        }
    }
    return n;
}

/* ---------------------------------------------------------------------------
 * rANS cores.
 * ------------------------------------------------------------------------- */

/* 4-lane interleaved rANS body shared by EncodeVANS4xDirect
 * (core/literals/literals.go:289-341) and przm_vans_encode4x_kernel
 * (przm_ans.cu:270-364): x = 65536 per lane, symbols in reverse, lane = i&3,
 * byte renormalisation while x > 4096*f-1, x = (x/f)*4096 + c + x%f.
 * Emitted bytes go to tmp in emission order; returns their count. */
static uint64_t rans4_emit(const uint8_t *src, uint64_t n, const uint16_t *freq, const uint16_t *cdf, uint8_t *tmp,
                           uint32_t x[4]) {
    uint64_t e = 0;
    x[0] = x[1] = x[2] = x[3] = 65536;
    for (uint64_t i = n; i-- > 0;) {
        uint32_t lane = (uint32_t)(i & 3), f = freq[src[i]], c = cdf[src[i]];
        while (x[lane] > 4096u * f - 1) { tmp[e++] = (uint8_t)x[lane]; x[lane] >>= 8; }
        x[lane] = (x[lane] / f) * 4096 + c + (x[lane] % f);
    }
    return e;
}

/* V-ANS container with a given table: 'V','A',01,flags | LE32 n | matrix |
 * 4 x LE32 state | reversed stream.  Returns the size written to dst. */
uint64_t or_vans_encode(const uint8_t *src, uint64_t n, const uint16_t *freq, uint8_t flags, uint8_t *dst) {
    uint16_t cdf[257];
    or_build_cdf(freq, cdf);
    uint8_t *tmp = (uint8_t *)malloc(2 * n + 64);
    uint32_t x[4];
    uint64_t e = rans4_emit(src, n, freq, cdf, tmp, x);
    dst[0] = 'V'; dst[1] = 'A'; dst[2] = 0x01; dst[3] = flags;
    wr32(dst + 4, (uint32_t)n);
    uint64_t p = 8 + or_serialize_matrix(freq, dst + 8);
    for (int j = 0; j < 4; j++) { wr32(dst + p, x[j]); p += 4; }
    for (uint64_t k = 0; k < e; k++) dst[p + k] = tmp[e - 1 - k];
    free(tmp);
    return p + e;
}

void or_histogram(const uint8_t *src, uint64_t n, uint32_t *counts) {
    memset(counts, 0, 256 * sizeof(uint32_t));
    for (uint64_t i = 0; i < n; i++) counts[src[i]]++;
}

/* EncodeAdaptiveVANS4x, core/literals/literals.go:368-384 (flags 0x00).
 * Returns 0 for n == 0 and UINT64_MAX when the reference would fail with
 * ErrBufferTooSmall (its emission scratch is 8 MiB, :36-37,:314-316). */
uint64_t or_adaptive_vans(const uint8_t *src, uint64_t n, uint8_t *dst) {
    if (n == 0) return 0;
    uint32_t counts[256];
    uint16_t freq[256];
    or_histogram(src, n, counts);
    or_normalize_frequencies(counts, freq);
    uint64_t sz = or_vans_encode(src, n, freq, 0x00, dst);
    uint64_t hdr = 8 + 16;
    uint8_t mat[600];
    hdr += or_serialize_matrix(freq, mat);
    if (sz - hdr > 8u * 1024 * 1024) return UINT64_MAX;
    return sz;
}

/* VANSEncode4xHost, gpu/bridge.go:3233-3322: GPU histogram, NormalizeFreq(4096),
 * BuildCDF, SerializeMatrix, przm_vans_encode4x_kernel (flags 0x01). */
uint64_t or_vans_encode_host(const uint8_t *src, uint64_t n, uint8_t *dst) {
    if (n == 0) return 0;
    uint32_t counts[256];
    uint16_t freq[256];
    or_histogram(src, n, counts);
    or_normalize_freq(counts, 4096, freq);
    return or_vans_encode(src, n, freq, 0x01, dst);
}

/* ContextMeta, core/commands/vans_meta.go:46-69 */
static inline int ctx_meta(uint8_t p) {
    if (p == 0) return 0;
    if (p < 4) return 1;
    if (p < 16) return 2;
    if (p < 32) return 3;
    if (p < 64) return 4;
    if (p < 128) return 5;
    if (p < 192) return 6;
    return 7;
}

/* EncodeVansMeta8, core/commands/vans_meta.go:78-157.  Returns the container
 * size, or UINT64_MAX when the reference's 2 MiB stream scratch
 * (varBufPool, :71-75) would overflow. */
uint64_t or_encode_meta8(const uint8_t *src, uint64_t n, uint8_t *dst) {
    uint32_t x[4] = {65536, 65536, 65536, 65536};
    uint16_t cdf[8][256];
    for (int c = 0; c < 8; c++) {
        uint32_t cum = 0;
        for (int s = 0; s < 256; s++) { cdf[c][s] = (uint16_t)cum; cum += przm_meta8_freq[c][s]; }
    }
    uint8_t *tmp = (uint8_t *)malloc(2 * n + 64);
    uint64_t e = 0;
    for (uint64_t i = n; i-- > 0;) {
        uint32_t lane = (uint32_t)(i & 3);
        int ctx = i > 0 ? ctx_meta(src[i - 1]) : 0;
        uint32_t f = przm_meta8_freq[ctx][src[i]], c = cdf[ctx][src[i]];
        while (x[lane] > 4096u * f - 1) { tmp[e++] = (uint8_t)x[lane]; x[lane] >>= 8; }
        x[lane] = (x[lane] / f) * 4096 + c + (x[lane] % f);
    }
    if (e > 2u * 1024 * 1024) { free(tmp); return UINT64_MAX; }
    dst[0] = 'V'; dst[1] = 'A'; dst[2] = 0x01; dst[3] = 0x41;
    wr32(dst + 4, (uint32_t)n);
    for (int j = 0; j < 4; j++) wr32(dst + 8 + 4 * j, x[j]);
    for (uint64_t k = 0; k < e; k++) dst[24 + k] = tmp[e - 1 - k];
    free(tmp);
    return 24 + e;
}

/* packSubstream, core/commands/commands.go:371-406 (tmp = 2 MiB). */
static uint64_t pack_substream(const uint8_t *sub, uint64_t n, uint8_t *dst) {
    const uint64_t TMP = 2u * 1024 * 1024;
    uint64_t best = 1 + n;
    uint8_t *tmp = (uint8_t *)malloc(2 * n + 1024);
    int chosen = 0;
    if (n >= 24 && n <= TMP) {
        uint64_t l = or_encode_meta8(sub, n, tmp);
        if (l != UINT64_MAX && l <= TMP && l < best) { best = l; memcpy(dst, tmp, l); chosen = 1; }
    }
    if (n >= 16 && n <= TMP) {
        uint64_t l = or_adaptive_vans(sub, n, tmp);
        if (l != UINT64_MAX && l <= TMP && l < best) { best = l; memcpy(dst, tmp, l); chosen = 1; }
    }
    free(tmp);
    if (chosen) return best;
    dst[0] = 0x09;
    memcpy(dst + 1, sub, n);
    return 1 + n;
}

/* PackCommandsMode8 (commands.go:409-444) + PackageCommandsSection
 * (:537-568).  dst capacity: 16 + n. */
uint64_t or_package_commands(const uint8_t *cmds, uint64_t n, uint8_t *dst) {
    if (n == 0) return 0;
    uint8_t *op = (uint8_t *)malloc(n), *meta = (uint8_t *)malloc(n), *var = (uint8_t *)malloc(n);
    uint64_t a, b, c;
    uint64_t out = 0;
    if (or_split_commands(cmds, n, op, &a, meta, &b, var, &c) == 0) {
        uint8_t *m8 = (uint8_t *)malloc(13 + n + 64);
        uint64_t p = 13;
        uint64_t lop = pack_substream(op, a, m8 + p); p += lop;
        uint64_t lm = pack_substream(meta, b, m8 + p); p += lm;
        p += pack_substream(var, c, m8 + p);
        m8[0] = 0x08;
        wr32(m8 + 1, (uint32_t)n); wr32(m8 + 5, (uint32_t)lop); wr32(m8 + 9, (uint32_t)lm);
        if (p < n) { memcpy(dst, m8, p); out = p; }
        free(m8);
    }
    if (!out) { dst[0] = 0x09; memcpy(dst + 1, cmds, n); out = 1 + n; }
    free(op); free(meta); free(var);
    return out;
}

/* ---------------------------------------------------------------------------
 * Section 3 distance coding (core/distance/distance.go), the offsets of a
 * frame as a distance-prefix container: a 49-bracket code per distance, its
 * extra bits MSB-first, the codes entropy-coded (Mode 12 static contexts or
 * adaptive V-ANS).  Buffer limits follow the reference's scratch sizes, since
 * running out of them changes the output (the flat fallback).
 * ------------------------------------------------------------------------- */
#define OR_DIST_SCRATCH (2u * 1024 * 1024) /* meta, varBuf, altBuf, s3Buf: distance.go:124-129, compress.go:76 */
#define OR_DIST_CODEBUF (4u * 1024 * 1024) /* cmds: distance.go:127 */

/* DistanceToCode, distance.go:165-180: code, extra bits and their count. */
uint8_t or_distance_to_code(uint32_t d, uint32_t *extra, uint32_t *nb) {
    if (d <= 4) { *extra = 0; *nb = 0; return (uint8_t)(d - 1); }
    if (d <= 16777216u) {
        const uint32_t u = d - 1;
        const uint32_t b = (uint32_t)(32 - __builtin_clz(u)) - 2;  /* bits.Len32(u) - 2, u >= 4 */
        const uint32_t half = (u >> b) & 1u;
        *nb = b;
        *extra = d - (((2u + half) << b) + 1u);
        return (uint8_t)(2 * b + 2 + half);
    }
    *nb = 24;
    *extra = d - 16777217u;
    return 48;
}

/* ContextDist, distance.go:190-202 */
static int ctx_dist(uint8_t prev) { return prev < 6 ? 0 : prev < 14 ? 1 : prev < 26 ? 2 : 3; }

/* BitWriter, distance.go:204-247: MSB-first into buf of cap bytes; a
 * write that needs a byte past cap fails (the reference's ErrBufferTooSmall). */
typedef struct { uint8_t *buf; uint64_t cap, pos; uint64_t acc; uint32_t cnt; int err; } or_bits;
static void bits_put(or_bits *w, uint32_t val, uint32_t nb) {
    if (nb == 0 || w->err) return;
    w->acc = (w->acc << nb) | ((uint64_t)val & ((1ull << nb) - 1));
    w->cnt += nb;
    while (w->cnt >= 8) {
        if (w->pos >= w->cap) { w->err = 1; return; }
        w->cnt -= 8;
        w->buf[w->pos++] = (uint8_t)(w->acc >> w->cnt);
    }
}
static void bits_flush(or_bits *w) {
    if (w->cnt > 0 && !w->err) {
        if (w->pos >= w->cap) { w->err = 1; return; }
        w->buf[w->pos++] = (uint8_t)(w->acc << (8 - w->cnt));
        w->cnt = 0;
        w->acc = 0;
    }
}

/* EncodeDistClusteredVans, distance.go:323-377: one rANS state (M = 4096,
 * L = 65536, byte renormalisation) over the codes from the last to the
 * first, each coded with the static weights of its predecessor's class;
 * 0x0C | LE32 state | reversed stream.  UINT64_MAX where the reference runs
 * out of its 2 MiB stream scratch or of dcap. */
uint64_t or_dist_mode12(const uint8_t *codes, uint64_t n, uint8_t *dst, uint64_t dcap) {
    if (n == 0) {
        if (dcap < 5) return UINT64_MAX;
        dst[0] = 0x0C;
        wr32(dst + 1, 65536);
        return 5;
    }
    uint16_t cdf[4][64];
    for (int k = 0; k < 4; k++) {
        uint16_t cum = 0;
        for (int s = 0; s < 64; s++) { cdf[k][s] = cum; cum += przm_dist_freq4[k][s]; }
    }
    uint8_t *tmp = (uint8_t *)malloc(OR_DIST_SCRATCH);
    uint64_t e = 0;
    uint32_t x = 65536;
    for (uint64_t i = n; i-- > 0;) {
        const uint8_t sym = codes[i];
        if (sym >= 64) { free(tmp); return UINT64_MAX; }
        const int k = ctx_dist(i ? codes[i - 1] : 0);
        const uint32_t f = przm_dist_freq4[k][sym], cf = cdf[k][sym];
        while (x > 4096u * f - 1) {
            if (e >= OR_DIST_SCRATCH) { free(tmp); return UINT64_MAX; }
            tmp[e++] = (uint8_t)x;
            x >>= 8;
        }
        x = (x / f) * 4096 + cf + (x % f);
    }
    if (5 + e > dcap) { free(tmp); return UINT64_MAX; }
    dst[0] = 0x0C;
    wr32(dst + 1, x);
    for (uint64_t k = 0; k < e; k++) dst[5 + k] = tmp[e - 1 - k];
    free(tmp);
    return 5 + e;
}

static uint64_t leb_len(uint32_t d) { return d <= 0x7F ? 1 : d <= 0x3FFF ? 2 : d <= 0x1FFFFF ? 3 : d <= 0x0FFFFFFF ? 4 : 5; }

/* PackDistancePrefix(mode auto, useVANS), distance.go:692-748, with
 * SelectPrefixMode :750-758 and assemblePrefixContainer :777-822:
 *   0x0B | u8 origLen | u8 count | u8 codeLen, or
 *   0x0A | LE16 x 3, or 0x06 | LE32 x 3; then the code stream, then the extra
 *   bits.  The code stream is Mode 12, or for 64 codes or more the adaptive
 *   V-ANS container of the codes when that fits 2 MiB and is smaller.
 * Returns the size, or UINT64_MAX on the reference's errors (a distance of 0
 * or above 2^24, a scratch or dst overflow). */
uint64_t or_pack_distance_prefix(const uint32_t *dist, uint64_t n, uint8_t *dst, uint64_t dcap) {
    if (n == 0) return 0;
    if (n > OR_DIST_SCRATCH) return UINT64_MAX; /* the codes' scratch (meta) */
    uint8_t *codes = (uint8_t *)malloc(n);
    uint8_t *extra = (uint8_t *)malloc(OR_DIST_SCRATCH);
    or_bits w = {extra, OR_DIST_SCRATCH, 0, 0, 0, 0};
    uint64_t orig = 0, ret = UINT64_MAX;
    uint8_t *cs = NULL, *alt = NULL;
    for (uint64_t i = 0; i < n; i++) {
        const uint32_t d = dist[i];
        if (d == 0 || d > 16777216u) goto out;
        uint32_t ex, nb;
        codes[i] = or_distance_to_code(d, &ex, &nb);
        bits_put(&w, ex, nb);
        if (w.err) goto out;
        orig += leb_len(d);
    }
    bits_flush(&w);
    if (w.err) goto out;
    cs = (uint8_t *)malloc(OR_DIST_CODEBUF);
    uint64_t cl = or_dist_mode12(codes, n, cs, OR_DIST_CODEBUF);
    if (cl == UINT64_MAX) goto out;
    if (n >= 64) {
        alt = (uint8_t *)malloc(2 * n + 1024);
        const uint64_t al = or_adaptive_vans(codes, n, alt);
        if (al != UINT64_MAX && al <= OR_DIST_SCRATCH && al < cl) { memcpy(cs, alt, al); cl = al; }
    }
    uint64_t h;
    if (orig <= 255 && n <= 255 && cl <= 255) h = 4;
    else if (orig <= 65535 && n <= 65535 && cl <= 65535) h = 7;
    else h = 13;
    if (h + cl + w.pos > dcap) goto out;
    if (h == 4) {
        dst[0] = 0x0B; dst[1] = (uint8_t)orig; dst[2] = (uint8_t)n; dst[3] = (uint8_t)cl;
    } else if (h == 7) {
        dst[0] = 0x0A;
        dst[1] = (uint8_t)orig; dst[2] = (uint8_t)(orig >> 8);
        dst[3] = (uint8_t)n; dst[4] = (uint8_t)(n >> 8);
        dst[5] = (uint8_t)cl; dst[6] = (uint8_t)(cl >> 8);
    } else {
        dst[0] = 0x06; wr32(dst + 1, (uint32_t)orig); wr32(dst + 5, (uint32_t)n); wr32(dst + 9, (uint32_t)cl);
    }
    memcpy(dst + h, cs, cl);
    memcpy(dst + h + cl, extra, w.pos);
    ret = h + cl + w.pos;
out:
    free(codes); free(extra); free(cs); free(alt);
    return ret;
}

/* PackageOffsetsSection, distance.go:825-849 (into the compressor's 2 MiB
 * s3Buf, compress.go:76,956): the distance-prefix container when it is
 * smaller than the distances as LEB128 varints, else 0x09 + those varints.
 * Returns 0 (an empty section) for no distances. dst holds 1 + 5 n bytes. */
uint64_t or_package_offsets(const uint32_t *dist, uint64_t n, uint8_t *dst) {
    if (n == 0) return 0;
    uint8_t *buf = (uint8_t *)malloc(OR_DIST_SCRATCH);
    const uint64_t pl = or_pack_distance_prefix(dist, n, buf, OR_DIST_SCRATCH);
    uint64_t raw = 0;
    for (uint64_t i = 0; i < n; i++) raw += leb_len(dist[i]);
    uint64_t w;
    if (pl != UINT64_MAX && pl < raw) {
        memcpy(dst, buf, pl);
        w = pl;
    } else {
        dst[0] = 0x09;
        w = 1;
        for (uint64_t i = 0; i < n; i++) {
            uint32_t v = dist[i];
            while (v >= 0x80) { dst[w++] = (uint8_t)(v | 0x80); v >>= 7; }
            dst[w++] = (uint8_t)v;
        }
    }
    free(buf);
    return w;
}

/* ---------------------------------------------------------------------------
 * Section 4 selection (core/literals/literals.go:600-693, sheaf.go): the
 * literals as the smallest of their adaptive V-ANS container and the four
 * étale-sheaf foliations, else raw.  A foliation sends every literal to one of
 * four fibers by the class of the literal before it (modes 0-2) or of the two
 * before it (mode 3); each fiber is V-ANS coded when that is smaller.
 * ------------------------------------------------------------------------- */
static int sheaf_ws(uint8_t b) { return b == ' ' || b == '\t' || b == '\r' || b == '\n'; }
static int sheaf_syntax(uint8_t b) {
    static const char set[] = "{}[]()<>:;,.\"'`=+-*/%&|^!~?\\#";
    return b != 0 && strchr(set, b) != NULL;
}
static int sheaf_ident(uint8_t b) { return (b >= 'a' && b <= 'z') || b == '_'; }
static int sheaf_digit(uint8_t b) { return b >= '0' && b <= '9'; }

/* ContextClassify (sheaf.go:39-88) for modes 0-2, ContextClassifyOrder2
 * (:91-107) for mode 3. */
uint8_t or_sheaf_class(uint8_t p2, uint8_t p1, int mode) {
    switch (mode) {
        case 0: return sheaf_ws(p1) ? 0 : sheaf_syntax(p1) ? 1 : sheaf_ident(p1) ? 2 : 3;
        case 1: return (p1 == '"' || p1 == ':') ? 0 : sheaf_ident(p1) ? 1 : sheaf_digit(p1) ? 2 : 3;
        case 2: return (sheaf_ws(p1) || sheaf_syntax(p1)) ? 0 : 1;
        default:
            if (sheaf_digit(p1)) return (sheaf_digit(p2) || p2 == '.' || p2 == '-') ? 0 : 1;
            if (sheaf_ident(p1)) return sheaf_ident(p2) ? 2 : 3;
            return sheaf_ws(p1) ? 0 : 1;
    }
}

/* DecomposeFibers (sheaf.go:110-137): fiber k of the literals gets the
 * literals of class k, in order; fibers[k] holds n bytes each, l[k] their
 * counts. */
void or_decompose_fibers(const uint8_t *src, uint64_t n, int mode, uint8_t *fibers[4], uint64_t l[4]) {
    uint8_t p1 = 0, p2 = 0;
    l[0] = l[1] = l[2] = l[3] = 0;
    for (uint64_t i = 0; i < n; i++) {
        const uint8_t k = or_sheaf_class(p2, p1, mode);
        fibers[k][l[k]++] = src[i];
        p2 = p1;
        p1 = src[i];
    }
}

/* EncodeVANS4x body (literals.go:344-355: the container without its 8-byte
 * header) with NormalizeFrequencies, as tryEncodeFiber (:633-643) makes it;
 * UINT64_MAX where the reference's 8 MiB emission scratch overflows. */
static uint64_t fiber_vans(const uint8_t *src, uint64_t n, uint8_t *dst) {
    uint32_t counts[256];
    uint16_t freq[256];
    or_histogram(src, n, counts);
    or_normalize_frequencies(counts, freq);
    uint8_t *tmp = (uint8_t *)malloc(2 * n + 1024);
    const uint64_t sz = or_vans_encode(src, n, freq, 0x00, tmp);
    uint8_t mat[600];
    const uint64_t hdr = 8 + 16 + or_serialize_matrix(freq, mat);
    uint64_t r = UINT64_MAX;
    if (sz - hdr <= 8u * 1024 * 1024) {
        memcpy(dst, tmp + 8, sz - 8);
        r = sz - 8;
    }
    free(tmp);
    return r;
}

/* PackEtaleSheaf (literals.go:600-631) with assembleSheafContainer (:645-662):
 * 'V','A',01, 0x01 | 0x04 | mode << 4, LE32 n, LE32 l[4], LE32 e[4], then the
 * fibers, each V-ANS coded when that is smaller (e < l), else raw (e == l).
 * dst holds 40 + 2 n + 4 x 1024 bytes. */
uint64_t or_pack_sheaf(const uint8_t *src, uint64_t n, int mode, uint8_t *dst) {
    uint8_t *fb[4];
    uint64_t l[4], e[4];
    for (int k = 0; k < 4; k++) fb[k] = (uint8_t *)malloc(n ? n : 1);
    or_decompose_fibers(src, n, mode, fb, l);
    dst[0] = 'V'; dst[1] = 'A'; dst[2] = 0x01; dst[3] = (uint8_t)(0x01 | 0x04 | ((mode & 0x0F) << 4));
    wr32(dst + 4, (uint32_t)n);
    uint64_t w = 40;
    uint8_t *enc = (uint8_t *)malloc(2 * n + 1024);
    for (int k = 0; k < 4; k++) {
        e[k] = 0;
        if (l[k] == 0) continue;
        const uint64_t el = fiber_vans(fb[k], l[k], enc);
        if (el != UINT64_MAX && el < l[k]) { memcpy(dst + w, enc, el); e[k] = el; }
        else { memcpy(dst + w, fb[k], l[k]); e[k] = l[k]; }
        w += e[k];
    }
    for (int k = 0; k < 4; k++) { wr32(dst + 8 + 4 * k, (uint32_t)l[k]); wr32(dst + 24 + 4 * k, (uint32_t)e[k]); }
    free(enc);
    for (int k = 0; k < 4; k++) free(fb[k]);
    return w;
}

/* PackageLiteralsSection (literals.go:664-693): the smallest of the adaptive
 * V-ANS container and the four foliations when one is smaller than the raw
 * literals (*nibble = FlagNibble 0x80), else the raw literals (*nibble = 0).
 * dst holds 40 + 2 n + 4 x 1024 bytes. */
uint64_t or_package_literals(const uint8_t *lits, uint64_t n, uint8_t *dst, uint8_t *nibble) {
    *nibble = 0;
    if (n == 0) return 0;
    uint8_t *cand = (uint8_t *)malloc(40 + 2 * n + 4 * 1024);
    uint64_t best = n;
    int have = 0;
    const uint64_t vl = or_adaptive_vans(lits, n, cand);
    if (vl != UINT64_MAX && vl < best) { memcpy(dst, cand, vl); best = vl; have = 1; }
    for (int mode = 0; mode <= 3; mode++) {
        const uint64_t sl = or_pack_sheaf(lits, n, mode, cand);
        if (sl < best) { memcpy(dst, cand, sl); best = sl; have = 1; }
    }
    free(cand);
    if (have) { *nibble = 0x80; return best; }
    memcpy(dst, lits, n);
    return n;
}

/* ---------------------------------------------------------------------------
 * Frames.
 * ------------------------------------------------------------------------- */

/* window-log rule of encodeD2DLocked, gpu/bridge.go:2312-2320 */
static uint32_t d2d_wlog(uint64_t n) { return n <= 65536 ? 16 : (n > 1048576 ? 23 : 20); }

static uint64_t put_header(uint8_t *dst, uint8_t flags, uint64_t n, uint64_t l2, uint64_t l3, uint32_t wlog) {
    uint64_t w = 0;
    dst[w++] = 'P'; dst[w++] = 'R'; dst[w++] = 'Z'; dst[w++] = 'M';
    dst[w++] = flags;
    dst[w++] = (uint8_t)n; dst[w++] = (uint8_t)(n >> 8); dst[w++] = (uint8_t)(n >> 16);
    if (!(flags & 0x08)) {
        dst[w++] = (uint8_t)l2; dst[w++] = (uint8_t)(l2 >> 8);
        dst[w++] = (uint8_t)l3; dst[w++] = (uint8_t)(l3 >> 8);
    } else {
        dst[w++] = (uint8_t)l2; dst[w++] = (uint8_t)(l2 >> 8); dst[w++] = (uint8_t)(l2 >> 16);
        dst[w++] = (uint8_t)l3; dst[w++] = (uint8_t)(l3 >> 8); dst[w++] = (uint8_t)(l3 >> 16);
    }
    memset(dst + w, 0, 8);
    dst[w + 1] = (uint8_t)wlog;
    return w + 8;
}

typedef struct { uint8_t *cmd, *off, *lit; uint64_t nc, no, nl; } or_tokens;

static void tokens_of(const uint8_t *in, uint64_t n, or_tokens *t) {
    uint64_t tiles = (n + OR_TILE - 1) / OR_TILE;
    uint32_t *desc = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    or_match_table(in, n, desc);
    t->cmd = (uint8_t *)malloc(tiles * 36864 + 16);
    t->off = (uint8_t *)malloc(tiles * 36864 + 16);
    t->lit = (uint8_t *)malloc(tiles * 36864 + 16);
    or_tokenize(in, n, desc, t->cmd, &t->nc, t->off, &t->no, t->lit, &t->nl);
    free(desc);
}

/* Frame bound shared with the product: worst case of either profile. */
uint64_t or_frame_bound(uint64_t n) { return 2 * n + 4096; }

/* Profile P0 == CompressD2D (gpu/bridge.go:2486-2544 -> encodeD2DLocked
 * :2287-2458): flat 0x00 Sections 2/3, raw literals, header by
 * przm_write_frame_header_kernel (przm_ans.cu:497-539). */
uint64_t or_compress_p0(const uint8_t *in, uint64_t n, uint8_t *dst) {
    if (n == 0) return 0;
    or_tokens t;
    tokens_of(in, n, &t);
    uint64_t l2 = t.nc + 5, l3 = t.no + 5;
    uint32_t wlog = d2d_wlog(n);
    uint8_t flags = (n > 65535 || l2 > 65535 || l3 > 65535 || wlog > 16) ? 0x08 : 0;
    uint64_t w = put_header(dst, flags, n, l2, l3, wlog);
    dst[w] = 0; wr32(dst + w + 1, (uint32_t)t.nc); memcpy(dst + w + 5, t.cmd, t.nc); w += l2;
    dst[w] = 0; wr32(dst + w + 1, (uint32_t)t.no); memcpy(dst + w + 5, t.off, t.no); w += l3;
    memcpy(dst + w, t.lit, t.nl); w += t.nl;
    free(t.cmd); free(t.off); free(t.lit);
    return w;
}

/* Raw Section 4 bytes that both reference decoders would read as a container
 * (core/literals/literals.go:703-734, src/przm_dec.c:853-872). */
int or_raw_literals_misparse(const uint8_t *lit, uint64_t n) {
    if (n < 8) return 0;
    if (lit[0] == 'V' && lit[1] == 'A' && lit[2] == 0x01) return 1;
    return rd32(lit + 4) == (uint32_t)(((uint64_t)rd32(lit) + 1) / 2);
}

/* Profiles P1 and P2.  P1 == match + tokenize + ANS frame (the batch
 * pipeline's entropy-coded frame format):
 *   header and Section 1 as P0;
 *   Section 2 = PackageCommandsSection(cmds) when cmds <= 2 MiB (every
 *     substream then fits the decoders' 2 MiB substream buffers), else
 *     0x09 + cmds;
 *   Section 3 = flat 0x00 offsets (as P0);
 *   Section 4 = EncodeAdaptiveVANS4x(lits) when it is smaller than the raw
 *     literals (or the raw bytes would be misread as a container) and
 *     lits <= 8 MiB (the decoders' literal buffer); else raw;
 *   flags gain FlagNibble (0x80) with a V-ANS Section 4 (compress.go:990);
 *   the frame falls back to FlagUncompressed when it would not shrink
 *     (assembleContainer, compress.go:962-985) or when neither Section 4 form
 *     is decodable.
 * n must be < 16 MiB (24-bit uSize). */
static uint64_t compress_p(const uint8_t *in, uint64_t n, uint8_t *dst, int s3_coded, int s4_full) {
    if (n == 0) return 0;
    or_tokens t;
    tokens_of(in, n, &t);
    uint8_t *s2 = (uint8_t *)malloc(t.nc + 64);
    uint64_t l2;
    if (t.nc <= 2u * 1024 * 1024) l2 = or_package_commands(t.cmd, t.nc, s2);
    else { s2[0] = 0x09; memcpy(s2 + 1, t.cmd, t.nc); l2 = 1 + t.nc; }
    uint64_t l3 = t.no + 5;
    uint8_t *s3 = NULL;
    if (s3_coded) {  /* the offset stream holds one LEB128 varint per distance */
        uint32_t *dist = (uint32_t *)malloc((t.no + 1) * sizeof(uint32_t));
        uint64_t nd = 0;
        for (uint64_t i = 0; i < t.no;) {
            uint32_t v = 0, sh = 0;
            while (t.off[i] & 0x80) { v |= (uint32_t)(t.off[i++] & 0x7F) << sh; sh += 7; }
            v |= (uint32_t)t.off[i++] << sh;
            dist[nd++] = v;
        }
        s3 = (uint8_t *)malloc(5 * nd + 64);
        l3 = or_package_offsets(dist, nd, s3);
        free(dist);
    }
    uint8_t *s4 = NULL;
    uint64_t l4 = t.nl;
    uint8_t nib = 0;
    int raw_ok = !or_raw_literals_misparse(t.lit, t.nl);
    int fallback = 0;
    if (t.nl > 0 && s4_full && t.nl <= 8u * 1024 * 1024) {
        s4 = (uint8_t *)malloc(40 + 2 * t.nl + 4 * 1024);
        l4 = or_package_literals(t.lit, t.nl, s4, &nib);
        if (!nib) {  /* raw: the same decodability guard as P1 */
            free(s4);
            s4 = NULL;
            l4 = t.nl;
        }
    }
    if (t.nl > 0 && !nib && (!s4_full || !raw_ok || t.nl > 8u * 1024 * 1024)) {
        uint64_t vl = UINT64_MAX;
        uint8_t *vb = NULL;
        if (t.nl <= 8u * 1024 * 1024) {
            vb = (uint8_t *)malloc(2 * t.nl + 1024);
            vl = or_adaptive_vans(t.lit, t.nl, vb);
        }
        if (vl != UINT64_MAX && (vl < t.nl || !raw_ok)) { s4 = vb; l4 = vl; nib = 0x80; vb = NULL; }
        else if (!raw_ok) fallback = 1;
        free(vb);
    }
    uint32_t wlog = d2d_wlog(n);
    uint8_t flags = nib | ((n > 65535 || l2 > 65535 || l3 > 65535 || wlog > 16) ? 0x08 : 0);
    uint64_t dir = (flags & 0x08) ? 6 : 4;
    uint64_t comp = 8 + dir + 8 + l2 + l3 + l4;
    uint64_t w;
    if (fallback || comp >= n) {
        memcpy(dst, "PRZM", 4);
        dst[4] = 0x04;
        dst[5] = (uint8_t)n; dst[6] = (uint8_t)(n >> 8); dst[7] = (uint8_t)(n >> 16);
        memcpy(dst + 8, in, n);
        w = 8 + n;
    } else {
        w = put_header(dst, flags, n, l2, l3, wlog);
        memcpy(dst + w, s2, l2); w += l2;
        if (s3) memcpy(dst + w, s3, l3);
        else { dst[w] = 0; wr32(dst + w + 1, (uint32_t)t.no); memcpy(dst + w + 5, t.off, t.no); }
        w += l3;
        memcpy(dst + w, s4 ? s4 : t.lit, l4); w += l4;
    }
    free(s2); free(s3); free(s4); free(t.cmd); free(t.off); free(t.lit);
    return w;
}

uint64_t or_compress_p1(const uint8_t *in, uint64_t n, uint8_t *dst) { return compress_p(in, n, dst, 0, 0); }

/* Profile P2 == P1 with Section 3 as PackageOffsetsSection of the frame's
 * distances (core/distance/distance.go:825-849, as the reference's CPU
 * compressor writes it, compress.go:956): a distance-prefix container or
 * 0x09 varints, and an empty Section 3 when the frame has no match. */
uint64_t or_compress_p2(const uint8_t *in, uint64_t n, uint8_t *dst) { return compress_p(in, n, dst, 1, 0); }

/* Profile P3 == P2 with Section 4 as PackageLiteralsSection (literals.go:
 * 664-693, as the reference's CPU compressor writes it): the smallest of the
 * adaptive V-ANS container and the four étale-sheaf foliations, else raw
 * under P1's decodability rule (the adaptive container when the raw bytes
 * would be misread as one, else a stored frame); containers only for
 * literals of at most 8 MiB (the decoders' literal and fiber buffers). */
uint64_t or_compress_p3(const uint8_t *in, uint64_t n, uint8_t *dst) { return compress_p(in, n, dst, 1, 1); }

/* Tokens only (Tokenize, gpu/bridge.go:1895), for tests. */
void or_tokenize_input(const uint8_t *in, uint64_t n, uint8_t *cmd, uint64_t *nc, uint8_t *off, uint64_t *no,
                       uint8_t *lit, uint64_t *nl) {
    uint32_t *desc = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    or_match_table(in, n, desc);
    or_tokenize(in, n, desc, cmd, nc, off, no, lit, nl);
    free(desc);
}
