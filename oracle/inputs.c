/* inputs.c — CPU oracle: the seeded photon medium restated in plain C (TEST / BENCH
 * INFRASTRUCTURE ONLY), so that the reference arm of the bench and the golden-fixture script
 * can build their inputs without loading the product library.
 *
 * Same definition as the product's generator (hrm_photon_medium): every draw is a pure
 * function of (seed, stream, voxel) through the splitmix64 finaliser (Steele, Lea and Flood,
 * OOPSLA'14), giving a double in [0, 1) from its top 53 bits; per voxel
 *   mu_s   = exp(0.5 * z), z = sqrt(-2 ln(1 - u1)) cos(2 pi u2)   (Box-Muller, streams 2, 3)
 *   absorb = 0.02 + 0.18 u                                        (stream 4)
 *   split  = u < 0.1                                               (stream 5)
 * computed in double and rounded once to float. A CPU test checks that both generators give
 * the same bytes.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

static uint64_t o_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double o_uniform(uint64_t seed, uint64_t stream, uint64_t i) {
    uint64_t z = o_mix64(seed ^ o_mix64(stream * 0x9E3779B97F4A7C15ull + i));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

int oracle_photon_medium(uint32_t n, uint64_t seed, float* mu_s, float* absorb, uint8_t* split) {
    if (n == 0 || n > 1024 || !mu_s || !absorb || !split) return 1;
    const int64_t nvox = (int64_t)n * n * n;
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < nvox; v++) {
        double u1 = o_uniform(seed, 2, (uint64_t)v);
        double u2 = o_uniform(seed, 3, (uint64_t)v);
        double z = sqrt(-2.0 * log(1.0 - u1)) * cos(6.283185307179586 * u2);
        mu_s[v] = (float)exp(0.5 * z);
        absorb[v] = (float)(0.02 + 0.18 * o_uniform(seed, 4, (uint64_t)v));
        split[v] = o_uniform(seed, 5, (uint64_t)v) < 0.1 ? 1u : 0u;
    }
    return 0;
}

/* R-MAT graph (Chakrabarti, Zhan and Faloutsos, SDM'04) restated for the oracle side: edge e
 * picks, at each of `scale` levels l, one quadrant of the adjacency matrix from the draw
 * u = uniform(seed, 1, e*scale + l): source bit 1 when u >= a+b, target bit 1 when
 * a <= u < a+b or u >= a+b+c. The CSR holds the edges sorted by (source, target). Same
 * definition as the product's generator (hrm_rmat_csr); a CPU test checks the bytes. */
static int o_cmp_u64(const void* x, const void* y) {
    uint64_t a = *(const uint64_t*)x, b = *(const uint64_t*)y;
    return a < b ? -1 : (a > b ? 1 : 0);
}

int oracle_rmat_csr(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                    uint32_t* rowptr, uint32_t* col) {
    if (scale == 0 || scale > 30 || edge_factor == 0 || !rowptr || !col) return 1;
    if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return 1;
    const uint64_t nv = 1ull << scale;
    const uint64_t ne = (uint64_t)edge_factor * nv;
    if (ne > 0xFFFFFFFFull) return 1;
    uint64_t* keys = (uint64_t*)malloc(ne * sizeof(uint64_t));
    if (!keys) return 1;
    const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)ne; e++) {
        uint64_t s = 0, d = 0;
        for (uint32_t l = 0; l < scale; l++) {
            double x = o_uniform(seed, 1, (uint64_t)e * scale + l);
            uint64_t qs = (x >= ab) ? 1u : 0u;
            uint64_t qd = ((x >= a && x < ab) || (x >= abc)) ? 1u : 0u;
            s = (s << 1) | qs;
            d = (d << 1) | qd;
        }
        keys[e] = (s << 32) | d;
    }
    qsort(keys, ne, sizeof(uint64_t), o_cmp_u64);
    for (uint64_t v = 0; v <= nv; v++) rowptr[v] = 0;
    for (uint64_t e = 0; e < ne; e++) rowptr[(keys[e] >> 32) + 1]++;
    for (uint64_t v = 0; v < nv; v++) rowptr[v + 1] += rowptr[v];
    for (uint64_t e = 0; e < ne; e++) col[e] = (uint32_t)keys[e];
    free(keys);
    return 0;
}
