/* collatz.c — CPU oracle for the Collatz program (TEST INFRASTRUCTURE ONLY).
 *
 * Restates the host checker of harmonize examples/cpp/collaz/collaz_hrm.cpp:157-168
 * (and collaz_std.cpp:28-39): the number of steps n -> n/2 (n even) or 3n+1 (n odd)
 * until n <= 1, with 0 and 1 taking 0 steps. Only tests/, the smoke check and the
 * bench's CPU-baseline leg use this file; the product never links it.
 */
#include <stdint.h>

uint32_t oracle_collatz_steps(uint64_t n) {
    uint32_t steps = 0;
    while (n > 1) {
        n = (n % 2 == 0) ? n / 2 : 3 * n + 1;
        steps++;
    }
    return steps;
}

/* out[i] = steps of (start + i), i < count. Parallel over i when built with OpenMP. */
void oracle_collatz_range(uint32_t start, uint32_t count, uint32_t* out) {
    int64_t i;
#pragma omp parallel for schedule(dynamic, 4096)
    for (i = 0; i < (int64_t)count; i++) {
        out[i] = oracle_collatz_steps((uint64_t)start + (uint64_t)i);
    }
}
