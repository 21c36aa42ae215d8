/*
 * gen.c -- the seeded synthetic graph generators, restated for the CPU side.
 *
 * TEST INFRASTRUCTURE ONLY: the reference arm of bench.py and the CPU
 * baselines make their input graphs with it, so that they load nothing from
 * the product library; tests/test_oracle.py checks that it produces the
 * product's edge lists exactly.
 *
 * Every edge is a pure function of (seed, edge number): SplitMix64's
 * finaliser (Steele, Lea & Flood, OOPSLA 2014) hashes the pair, and
 *   R-MAT    picks one quadrant per level from 32 bits of a hash (two levels
 *            per hash), thresholds a, a+b, a+b+c scaled by 2^32;
 *   uniform  takes src and dst as the high halves of 32x32-bit products
 *            of the two 32-bit hash halves with V;
 *   grid     numbers the undirected grid edges horizontal-first, keeps each
 *            with probability 1-drop (32 bits against drop*2^32), emits both
 *            directions with one weight, then adds round(shortcut*V) random
 *            vertex pairs (a salted hash), both directions;
 *   weights  wmin + floor(r * (wmax-wmin+1) / 2^32) for 32 bits r of a salted
 *            hash, as float.
 */
#include <math.h>
#include <stdint.h>

#define GEN_WEIGHT_SALT 0x5851F42D4C957F2Dull
#define GEN_SHORTCUT_SALT 0x2545F4914F6CDD1Dull

static uint64_t gen_mix(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static uint64_t gen_hash(uint64_t seed, uint64_t i) { return gen_mix(seed ^ gen_mix(i)); }

static uint32_t gen_mulhi(uint32_t r, uint32_t n) { return (uint32_t)(((uint64_t)r * n) >> 32); }

static uint64_t gen_scale32(double p)
{
    if (p <= 0) return 0;
    if (p >= 1) return 1ull << 32;
    return (uint64_t)llround(p * 4294967296.0);
}

static float gen_weight(uint64_t seed, uint64_t e, int32_t wmin, int32_t wmax)
{
    if (wmax <= 0) return 1.0f;
    uint32_t r = (uint32_t)(gen_hash(seed ^ GEN_WEIGHT_SALT, e) >> 32);
    return (float)(wmin + (int32_t)gen_mulhi(r, (uint32_t)(wmax - wmin + 1)));
}

/* R-MAT edges 0..E-1 on 2^scale vertices; w may be NULL. */
void gen_rmat(uint64_t seed, int scale, int64_t E, double a, double b, double c,
              int32_t wmin, int32_t wmax, int32_t *src, int32_t *dst, float *w)
{
    const uint64_t ta = gen_scale32(a), tab = gen_scale32(a + b), tabc = gen_scale32(a + b + c);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < E; e++) {
        uint32_t u = 0, v = 0;
        for (int l = 0; l < scale; l += 2) {
            uint64_t h = gen_hash(seed, (uint64_t)e * 32 + (uint64_t)(l >> 1));
            for (int k = 0; k < 2 && l + k < scale; k++) {
                uint64_t r = k ? (uint32_t)h : (uint32_t)(h >> 32);
                uint32_t bs = r >= tab ? 1u : 0u;
                uint32_t bd = ((r >= ta && r < tab) || r >= tabc) ? 1u : 0u;
                u = (u << 1) | bs;
                v = (v << 1) | bd;
            }
        }
        src[e] = (int32_t)u;
        dst[e] = (int32_t)v;
        if (w) w[e] = gen_weight(seed, (uint64_t)e, wmin, wmax);
    }
}

/* Uniform random edges on V vertices. */
void gen_uniform(uint64_t seed, int64_t V, int64_t E, int32_t wmin, int32_t wmax,
                 int32_t *src, int32_t *dst, float *w)
{
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < E; e++) {
        uint64_t h = gen_hash(seed, (uint64_t)e);
        src[e] = (int32_t)gen_mulhi((uint32_t)(h >> 32), (uint32_t)V);
        dst[e] = (int32_t)gen_mulhi((uint32_t)h, (uint32_t)V);
        if (w) w[e] = gen_weight(seed, (uint64_t)e, wmin, wmax);
    }
}

/* The grid; returns the edge count (src == NULL: count only). */
int64_t gen_grid(uint64_t seed, int64_t R, int64_t C, double drop, double shortcut,
                 int32_t wmin, int32_t wmax, int32_t *src, int32_t *dst, float *w)
{
    const int64_t V = R * C, nh = R * (C - 1), nv = (R - 1) * C;
    const uint64_t drop_t = (uint64_t)llround(drop * 4294967296.0);
    int64_t m = 0;
    for (int64_t i = 0; i < nh + nv; i++) {
        if ((gen_hash(seed, (uint64_t)i) >> 32) < drop_t) continue;
        int64_t u, v;
        if (i < nh) {
            u = (i / (C - 1)) * C + i % (C - 1);
            v = u + 1;
        } else {
            u = ((i - nh) / C) * C + (i - nh) % C;
            v = u + C;
        }
        if (src) {
            float x = gen_weight(seed, (uint64_t)i, wmin, wmax);
            src[m] = (int32_t)u; dst[m] = (int32_t)v;
            src[m + 1] = (int32_t)v; dst[m + 1] = (int32_t)u;
            if (w) { w[m] = x; w[m + 1] = x; }
        }
        m += 2;
    }
    const int64_t S = llround(shortcut * (double)V);
    for (int64_t k = 0; k < S; k++) {
        uint64_t h = gen_hash(seed ^ GEN_SHORTCUT_SALT, (uint64_t)k);
        int64_t u = gen_mulhi((uint32_t)(h >> 32), (uint32_t)V);
        int64_t v = gen_mulhi((uint32_t)h, (uint32_t)V);
        if (src) {
            float x = gen_weight(seed ^ GEN_SHORTCUT_SALT, (uint64_t)k, wmin, wmax);
            src[m] = (int32_t)u; dst[m] = (int32_t)v;
            src[m + 1] = (int32_t)v; dst[m + 1] = (int32_t)u;
            if (w) { w[m] = x; w[m + 1] = x; }
        }
        m += 2;
    }
    return m;
}
