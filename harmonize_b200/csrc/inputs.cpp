// inputs.cpp — seeded synthetic inputs for the built-in workloads (host code, OpenMP).
//
//  * R-MAT graphs (Chakrabarti, Zhan and Faloutsos, SDM'04): each edge picks one of the
//    four quadrants of the adjacency matrix with probabilities (a, b, c, 1-a-b-c) at each of
//    `scale` levels. Every random draw is a pure function of (seed, edge, level), so the
//    edge list does not depend on the thread count; the CSR is built from the edge list
//    sorted by (source, target), so the column order is deterministic too.
//  * Photon media: per voxel mu_s ~ lognormal(0, 0.5) (Box-Muller in double), absorbed
//    fraction ~ U[0.02, 0.2], split flag with probability 0.1.
#include <parallel/algorithm>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

namespace {

inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uniform double in [0, 1) from (seed, stream, index).
inline double uniform(uint64_t seed, uint64_t stream, uint64_t i) {
    uint64_t z = mix64(seed ^ mix64(stream * 0x9E3779B97F4A7C15ull + i));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace

extern "C" {

// rowptr[2^scale + 1], col[edge_factor * 2^scale]. Returns 0, or 1 on bad arguments.
int hrm_rmat_csr(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                 uint32_t* rowptr, uint32_t* col) {
    if (scale == 0 || scale > 30 || edge_factor == 0 || rowptr == nullptr || col == nullptr) return 1;
    if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return 1;
    const uint64_t nv = 1ull << scale;
    const uint64_t ne = (uint64_t)edge_factor * nv;
    if (ne > 0xFFFFFFFFull) return 1;
    std::vector<uint64_t> keys(ne);
    const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)ne; e++) {
        uint64_t s = 0, d = 0;
        for (uint32_t l = 0; l < scale; l++) {
            double x = uniform(seed, 1, (uint64_t)e * scale + l);
            uint64_t qs = (x >= ab) ? 1u : 0u;
            uint64_t qd = (x >= a && x < ab) || (x >= abc) ? 1u : 0u;
            s = (s << 1) | qs;
            d = (d << 1) | qd;
        }
        keys[e] = (s << 32) | d;
    }
    __gnu_parallel::sort(keys.begin(), keys.end());
    std::vector<uint32_t> deg(nv + 1, 0);
    for (uint64_t e = 0; e < ne; e++) deg[keys[e] >> 32]++;
    rowptr[0] = 0;
    for (uint64_t v = 0; v < nv; v++) rowptr[v + 1] = rowptr[v] + deg[v];
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)ne; e++) col[e] = (uint32_t)keys[e];
    return 0;
}

// mu_s, absorb, split each hold n^3 voxels. Returns 0, or 1 on bad arguments.
int hrm_photon_medium(uint32_t n, uint64_t seed, float* mu_s, float* absorb, uint8_t* split) {
    if (n == 0 || n > 1024 || mu_s == nullptr || absorb == nullptr || split == nullptr) return 1;
    const uint64_t nvox = (uint64_t)n * n * n;
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)nvox; v++) {
        double u1 = uniform(seed, 2, (uint64_t)v);
        double u2 = uniform(seed, 3, (uint64_t)v);
        double z = std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(6.283185307179586 * u2);
        mu_s[v] = (float)std::exp(0.5 * z);
        absorb[v] = (float)(0.02 + 0.18 * uniform(seed, 4, (uint64_t)v));
        split[v] = uniform(seed, 5, (uint64_t)v) < 0.1 ? 1u : 0u;
    }
    return 0;
}

}  // extern "C"
