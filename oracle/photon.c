/* photon.c — CPU oracle: serial restatement of the photon-walk workload (TEST
 * INFRASTRUCTURE ONLY), written independently of the spec header in plain C.
 *
 * Same physics and the same random-number keying as the spec (see
 * harmonize_b200/csrc/specs/photon.h): Philox-4x32-10 (Salmon et al., SC'11) keyed by the
 * 64-bit photon id with counter (step, phase, seed_lo, seed_hi); free path -ln(u)/mu_s
 * with ln computed as 2*atanh((m-1)/(m+1)) + e*ln2 by a truncated series; Marsaglia
 * directions; x2 splits entering flagged voxels; roulette below 1e-3 (p = 0.1, x10);
 * 2^-32 fixed-point tallies. Built with -ffp-contract=off so that every float operation
 * rounds once, like the device intrinsics. The walk keeps an explicit stack, so the order
 * of events differs from any GPU schedule while the tallies (integer sums) must agree.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    float x, y, z, dx, dy, dz, w;
    uint32_t id_lo, id_hi, step, voxel;
} oph_t;

typedef struct {
    uint32_t v[4];
} o4_t;

static o4_t o_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    o4_t c = {{c0, c1, c2, c3}};
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c.v[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c.v[2];
        o4_t n;
        n.v[0] = (uint32_t)(p1 >> 32) ^ c.v[1] ^ k0;
        n.v[1] = (uint32_t)p1;
        n.v[2] = (uint32_t)(p0 >> 32) ^ c.v[3] ^ k1;
        n.v[3] = (uint32_t)p0;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    o4_t r = o_philox(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1]);
    memcpy(out, r.v, 16);
}

static float o_u01(uint32_t r) { return (float)((r >> 8) + 1u) * (1.0f / 16777216.0f); }
static float o_upm1(uint32_t r) { return (float)(int)(r >> 8) * (1.0f / 8388608.0f) - 1.0f; }

float oracle_log(float x) {
    uint32_t b;
    memcpy(&b, &x, 4);
    int e = (int)((b >> 23) & 0xFFu) - 127;
    uint32_t mb = (b & 0x007FFFFFu) | 0x3F800000u;
    float m;
    memcpy(&m, &mb, 4);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    float s = (m - 1.0f) / (m + 1.0f);
    float z = s * s;
    float p = 0.18181818f;
    p = p * z + 0.22222222f;
    p = p * z + 0.28571429f;
    p = p * z + 0.40000000f;
    p = p * z + 0.66666667f;
    p = p * z + 2.0f;
    float lm = s * p;
    float fe = (float)e;
    return (fe * 0.693145751953125f + lm) + fe * 1.42860682030941723e-06f;
}

static uint64_t o_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

typedef struct {
    const float *mu, *ab;
    const uint8_t* sp;
    uint32_t n, s0, s1;
    uint64_t* tally;
    uint64_t calls[3]; /* move, collide, tally */
} octx_t;

static void o_dir(const octx_t* c, uint32_t lo, uint32_t hi, uint32_t step, float* dx, float* dy, float* dz) {
    for (uint32_t a = 0; a < 16; a++) {
        o4_t r = o_philox(step, 2u + a, c->s0, c->s1, lo, hi);
        for (int q = 0; q < 4; q += 2) {
            float u = o_upm1(r.v[q]), v = o_upm1(r.v[q + 1]);
            float s = u * u + v * v;
            if (s < 1.0f && s > 0.0f) {
                float f = 2.0f * sqrtf(1.0f - s);
                *dx = u * f;
                *dy = v * f;
                *dz = 1.0f - 2.0f * s;
                return;
            }
        }
    }
    *dx = 0.0f;
    *dy = 0.0f;
    *dz = 1.0f;
}

static uint64_t o_fix(float x) { return (uint64_t)(x * 4294967296.0f); }

static void o_tally(octx_t* c, uint32_t slot, uint64_t amount) {
    c->calls[2]++;
    __atomic_fetch_add(&c->tally[slot], amount, __ATOMIC_RELAXED);
}

static float o_face(float x, float d, uint32_t lo) {
    float t;
    if (d > 0.0f) {
        t = ((float)(lo + 1u) - x) / d;
        return t > 0.0f ? t : 0.0f;
    }
    if (d < 0.0f) {
        t = ((float)lo - x) / d;
        return t > 0.0f ? t : 0.0f;
    }
    return 3.0e38f;
}

typedef struct {
    oph_t* a;
    size_t n, cap;
} ostack_t;

static void o_push(ostack_t* s, oph_t p) {
    if (s->n == s->cap) {
        s->cap = s->cap ? 2 * s->cap : 1024;
        s->a = (oph_t*)realloc(s->a, s->cap * sizeof(oph_t));
    }
    s->a[s->n++] = p;
}

/* Walks one source photon and all its descendants. */
static void o_walk(octx_t* c, uint32_t id, ostack_t* st) {
    const uint32_t n = c->n, h = n / 2u, S = 1024u;
    oph_t p;
    p.x = p.y = p.z = (float)h;
    p.id_lo = id;
    p.id_hi = 0;
    p.w = 1.0f;
    o_dir(c, id, 0, 0, &p.dx, &p.dy, &p.dz);
    p.voxel = (p.dx >= 0.0f ? h : h - 1u) + n * ((p.dy >= 0.0f ? h : h - 1u) + n * (p.dz >= 0.0f ? h : h - 1u));
    p.step = 1;
    st->n = 0;
    o_push(st, p);
    while (st->n) {
        p = st->a[--st->n];
        /* move */
        for (;;) {
            c->calls[0]++;
            uint32_t ix = p.voxel % n, iy = (p.voxel / n) % n, iz = p.voxel / (n * n);
            o4_t r = o_philox(p.step, 0u, c->s0, c->s1, p.id_lo, p.id_hi);
            float dist = (0.0f - oracle_log(o_u01(r.v[0]))) / c->mu[p.voxel];
            float tx = o_face(p.x, p.dx, ix), ty = o_face(p.y, p.dy, iy), tz = o_face(p.z, p.dz, iz);
            int axis = 0;
            float tb = tx;
            if (ty < tb) { tb = ty; axis = 1; }
            if (tz < tb) { tb = tz; axis = 2; }
            p.step++;
            if (dist < tb) {
                p.x = p.x + dist * p.dx;
                p.y = p.y + dist * p.dy;
                p.z = p.z + dist * p.dz;
                /* collide */
                c->calls[1]++;
                float dep = p.w * c->ab[p.voxel];
                p.w = p.w - dep;
                o_tally(c, p.voxel, o_fix(dep));
                if (p.w < 1.0e-3f) {
                    o4_t rr = o_philox(p.step, 1u, c->s0, c->s1, p.id_lo, p.id_hi);
                    uint32_t spread = p.id_lo & (S - 1u);
                    if (o_u01(rr.v[0]) <= 0.1f) {
                        float boosted = p.w * 10.0f;
                        o_tally(c, n * n * n + 2u * S + spread, o_fix(boosted - p.w));
                        p.w = boosted;
                    } else {
                        o_tally(c, n * n * n + S + spread, o_fix(p.w));
                        break;
                    }
                }
                o_dir(c, p.id_lo, p.id_hi, p.step, &p.dx, &p.dy, &p.dz);
                p.step++;
                continue;
            }
            p.x = p.x + tb * p.dx;
            p.y = p.y + tb * p.dy;
            p.z = p.z + tb * p.dz;
            int out = 0;
            if (axis == 0) {
                if (p.dx > 0.0f) { p.x = (float)(ix + 1u); out = (ix + 1u == n); ix++; }
                else { p.x = (float)ix; out = (ix == 0u); ix--; }
            } else if (axis == 1) {
                if (p.dy > 0.0f) { p.y = (float)(iy + 1u); out = (iy + 1u == n); iy++; }
                else { p.y = (float)iy; out = (iy == 0u); iy--; }
            } else {
                if (p.dz > 0.0f) { p.z = (float)(iz + 1u); out = (iz + 1u == n); iz++; }
                else { p.z = (float)iz; out = (iz == 0u); iz--; }
            }
            if (out) {
                o_tally(c, n * n * n + (p.id_lo & (S - 1u)), o_fix(p.w));
                break;
            }
            p.voxel = ix + n * (iy + n * iz);
            if (c->sp[p.voxel]) {
                p.w = p.w * 0.5f;
                uint64_t id64 = ((uint64_t)p.id_hi << 32) | p.id_lo;
                for (uint32_t k = 0; k < 2; k++) {
                    uint64_t cid = o_mix(id64 ^ ((((uint64_t)p.step << 1) | k) * 0x9E3779B97F4A7C15ull));
                    oph_t q = p;
                    q.id_lo = (uint32_t)cid;
                    q.id_hi = (uint32_t)(cid >> 32);
                    o_push(st, q);
                }
                break;
            }
        }
    }
}

/* Walks photons [first, first+count). tally (n^3 + 3*1024 slots) must be zeroed by the
 * caller; calls[3] receives move, collide and tally call counts. Parallel over source
 * photons with OpenMP; the tallies are sums of integers, so the result does not depend
 * on the thread count. */
void oracle_photon_walk(const float* mu_s, const float* absorb, const uint8_t* split, uint32_t n, uint32_t seed_lo,
                        uint32_t seed_hi, uint32_t first, uint32_t count, uint64_t* tally, uint64_t* calls) {
    uint64_t c0 = 0, c1 = 0, c2 = 0;
#pragma omp parallel reduction(+ : c0, c1, c2)
    {
        octx_t c;
        ostack_t st = {0, 0, 0};
        c.mu = mu_s;
        c.ab = absorb;
        c.sp = split;
        c.n = n;
        c.s0 = seed_lo;
        c.s1 = seed_hi;
        c.tally = tally;
        c.calls[0] = c.calls[1] = c.calls[2] = 0;
        int64_t i;
#pragma omp for schedule(dynamic, 64)
        for (i = 0; i < (int64_t)count; i++) o_walk(&c, first + (uint32_t)i, &st);
        c0 += c.calls[0];
        c1 += c.calls[1];
        c2 += c.calls[2];
        free(st.a);
    }
    calls[0] = c0;
    calls[1] = c1;
    calls[2] = c2;
}
