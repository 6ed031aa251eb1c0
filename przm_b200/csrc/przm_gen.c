/*
 * przm_gen.c -- seeded synthetic inputs for the compression workloads.
 *
 * There is no public corpus for this path, so every workload is generated
 * from a published PRNG: xoshiro256** (Blackman & Vigna) seeded through
 * splitmix64.  The same seed gives the same bytes on every machine.
 *
 *   markov   order-1 Markov source over 64 symbols (0x20..0x5F) with
 *            Dirichlet(0.3) transition rows (normalised Gamma(0.3) draws,
 *            Marsaglia & Tsang 2000 with the a<1 boost), then copies of
 *            earlier data (length 4 + Geometric(mean 20), offset uniform in
 *            [1, 65536] clamped to the position) laid left to right until
 *            about 30% of the positions are copies;
 *   zipf     Zipf(s) over 256 ranks with a seeded rank->byte permutation;
 *   table    16 little-endian int32 columns, each a random walk with steps
 *            uniform in [-8, 8] from a uniform int32 start, row-major;
 *   records  one random 200-byte template, repeated, every byte mutated to a
 *            uniform byte with probability 0.05;
 *   uniform  uniform random bytes;
 *   mixture  one of markov/table/records/uniform with p = .4/.3/.2/.1.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { uint64_t s[4]; } rng_t;

static uint64_t splitmix64(uint64_t *x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static void rng_seed(rng_t *r, uint64_t seed) {
    for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&seed);
}
static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static inline uint64_t rng_next(rng_t *r) {
    uint64_t *s = r->s;
    uint64_t res = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return res;
}
static inline double rng_unit(rng_t *r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static inline double rng_open(rng_t *r) { return ((double)(rng_next(r) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
static inline uint32_t rng_below(rng_t *r, uint32_t n) { return (uint32_t)(((rng_next(r) >> 32) * (uint64_t)n) >> 32); }

static double rng_normal(rng_t *r) { /* Box-Muller */
    return sqrt(-2.0 * log(rng_open(r))) * cos(6.283185307179586 * rng_unit(r));
}
static double rng_gamma(rng_t *r, double a) { /* Marsaglia-Tsang */
    if (a < 1.0) return rng_gamma(r, a + 1.0) * pow(rng_open(r), 1.0 / a);
    double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
    for (;;) {
        double x = rng_normal(r), v = 1.0 + c * x;
        if (v <= 0) continue;
        v = v * v * v;
        double u = rng_open(r);
        if (log(u) < 0.5 * x * x + d - d * v + d * log(v)) return d * v;
    }
}

void przm_gen_markov(uint64_t seed, uint8_t *out, uint64_t n) {
    rng_t r;
    rng_seed(&r, seed);
    static const int K = 64;
    double cdf[64][64];
    for (int i = 0; i < K; i++) {
        double g[64], s = 0;
        for (int j = 0; j < K; j++) { g[j] = rng_gamma(&r, 0.3); s += g[j]; }
        double acc = 0;
        for (int j = 0; j < K; j++) { acc += g[j] / s; cdf[i][j] = acc; }
        cdf[i][K - 1] = 1.0;
    }
    int st = (int)rng_below(&r, K);
    for (uint64_t i = 0; i < n; i++) {
        double u = rng_unit(&r);
        int lo = 0, hi = K - 1;
        while (lo < hi) { int m = (lo + hi) >> 1; if (cdf[st][m] > u) hi = m; else lo = m + 1; }
        st = lo;
        out[i] = (uint8_t)(0x20 + st);
    }
    /* copies: start probability p with mean length 24 gives ~30% coverage */
    const double p = 0.3 / (24.0 * 0.7 + 0.3);
    uint64_t pos = 1, covered = 0, target = (uint64_t)(0.3 * (double)n);
    while (pos < n && covered < target) {
        if (rng_unit(&r) < p) {
            uint64_t L = 4;
            while (rng_unit(&r) >= 1.0 / 21.0) L++; /* Geometric on {0,1,..}, mean 20 */
            uint64_t off = 1 + rng_below(&r, 65536);
            if (off > pos) off = pos;
            if (L > n - pos) L = n - pos;
            for (uint64_t k = 0; k < L; k++) out[pos + k] = out[pos + k - off];
            pos += L;
            covered += L;
        } else {
            pos++;
        }
    }
}

void przm_gen_zipf(uint64_t seed, double s, uint8_t *out, uint64_t n) {
    rng_t r;
    rng_seed(&r, seed);
    uint8_t perm[256];
    for (int i = 0; i < 256; i++) perm[i] = (uint8_t)i;
    for (int i = 255; i > 0; i--) { int j = (int)rng_below(&r, (uint32_t)i + 1); uint8_t t = perm[i]; perm[i] = perm[j]; perm[j] = t; }
    double cdf[256], acc = 0;
    for (int k = 0; k < 256; k++) { acc += pow((double)(k + 1), -s); cdf[k] = acc; }
    for (int k = 0; k < 256; k++) cdf[k] /= acc;
    cdf[255] = 1.0;
    for (uint64_t i = 0; i < n; i++) {
        double u = rng_unit(&r);
        int lo = 0, hi = 255;
        while (lo < hi) { int m = (lo + hi) >> 1; if (cdf[m] > u) hi = m; else lo = m + 1; }
        out[i] = perm[lo];
    }
}

void przm_gen_table(uint64_t seed, uint8_t *out, uint64_t n) {
    rng_t r;
    rng_seed(&r, seed);
    uint32_t v[16];
    for (int c = 0; c < 16; c++) v[c] = (uint32_t)rng_next(&r);
    for (uint64_t i = 0; i < n; i += 4) {
        int c = (int)((i / 4) & 15);
        v[c] += (uint32_t)((int32_t)rng_below(&r, 17) - 8);
        uint8_t b[4] = {(uint8_t)v[c], (uint8_t)(v[c] >> 8), (uint8_t)(v[c] >> 16), (uint8_t)(v[c] >> 24)};
        for (int k = 0; k < 4 && i + k < n; k++) out[i + k] = b[k];
    }
}

void przm_gen_records(uint64_t seed, uint8_t *out, uint64_t n) {
    rng_t r;
    rng_seed(&r, seed);
    uint8_t tpl[200];
    for (int i = 0; i < 200; i++) tpl[i] = (uint8_t)rng_next(&r);
    for (uint64_t i = 0; i < n; i++) {
        uint8_t b = tpl[i % 200];
        if (rng_unit(&r) < 0.05) b = (uint8_t)rng_next(&r);
        out[i] = b;
    }
}

void przm_gen_uniform(uint64_t seed, uint8_t *out, uint64_t n) {
    rng_t r;
    rng_seed(&r, seed);
    uint64_t i = 0;
    for (; i + 8 <= n; i += 8) { uint64_t x = rng_next(&r); memcpy(out + i, &x, 8); }
    if (i < n) { uint64_t x = rng_next(&r); memcpy(out + i, &x, n - i); }
}

/* Returns the kind drawn: 0 markov, 1 table, 2 records, 3 uniform. */
int przm_gen_mixture(uint64_t seed, uint8_t *out, uint64_t n) {
    rng_t r;
    rng_seed(&r, seed ^ 0xA5A5A5A5A5A5A5A5ull);
    double u = rng_unit(&r);
    uint64_t sub = rng_next(&r);
    if (u < 0.4) { przm_gen_markov(sub, out, n); return 0; }
    if (u < 0.7) { przm_gen_table(sub, out, n); return 1; }
    if (u < 0.9) { przm_gen_records(sub, out, n); return 2; }
    przm_gen_uniform(sub, out, n);
    return 3;
}
