// spec_support.h — helpers that program specifications may use from code that must
// build both for the GPU (nvcc) and for the host executors (g++).
//
// Nothing in this header names a Harmonize API type (OpUnion, Promise, util::...), so a
// spec that includes it can be compiled against this runtime's `harmonize.h`, against
// the original Harmonize headers, or against the host executors in `oracle/`.
//
// Floating point: every helper below rounds exactly like IEEE-754 binary32 with
// round-to-nearest-even, on both sides. On the device the `__f*_rn` intrinsics are used,
// which the compiler never contracts into FMAs; on the host, plain operators are used and
// the host build must pass `-ffp-contract=off` (x86-64 without -march=native emits no FMA
// anyway). That is what makes fixed-point tallies computed from float geometry bit-exact
// between the GPU runtime and the host executors.
#ifndef HARMONIZE_SPEC_SUPPORT_H
#define HARMONIZE_SPEC_SUPPORT_H

#include <cstdint>
#include <cstring>
#include <cmath>

#if defined(__CUDACC__)
  #define HRM_HD __host__ __device__
  #define HRM_DEV __device__
  #define HRM_FI __forceinline__
#else
  #define HRM_HD
  #define HRM_DEV
  #define HRM_FI inline
#endif

namespace hrm {

// ---------------------------------------------------------------------------------------
// Atomics usable from spec code on either side.
// ---------------------------------------------------------------------------------------
HRM_HD HRM_FI unsigned long long atomic_add_u64(unsigned long long* p, unsigned long long v) {
#if defined(__CUDA_ARCH__)
    return atomicAdd(p, v);
#else
    return __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
#endif
}

HRM_HD HRM_FI unsigned int atomic_add_u32(unsigned int* p, unsigned int v) {
#if defined(__CUDA_ARCH__)
    return atomicAdd(p, v);
#else
    return __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
#endif
}

HRM_HD HRM_FI unsigned int atomic_min_u32(unsigned int* p, unsigned int v) {
#if defined(__CUDA_ARCH__)
    return atomicMin(p, v);
#else
    unsigned int cur = __atomic_load_n(p, __ATOMIC_RELAXED);
    while (v < cur && !__atomic_compare_exchange_n(p, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
    return cur;
#endif
}

HRM_HD HRM_FI unsigned int load_relaxed_u32(const unsigned int* p) {
#if defined(__CUDA_ARCH__)
    return *(volatile const unsigned int*)p;
#else
    return __atomic_load_n(p, __ATOMIC_RELAXED);
#endif
}

// ---------------------------------------------------------------------------------------
// Exactly rounded binary32 arithmetic (round to nearest even), identical on host and device.
// ---------------------------------------------------------------------------------------
HRM_HD HRM_FI float fadd(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
HRM_HD HRM_FI float fsub(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
HRM_HD HRM_FI float fmul(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
HRM_HD HRM_FI float fdiv(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
HRM_HD HRM_FI float fsqrt(float a) {
#if defined(__CUDA_ARCH__)
    return __fsqrt_rn(a);
#else
    return std::sqrt(a);
#endif
}

HRM_HD HRM_FI uint32_t float_bits(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}
HRM_HD HRM_FI float bits_float(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// Natural logarithm for finite x > 0 built only from exactly rounded +,-,*,/ and bit
// manipulation, so that host and device agree bit for bit.
//
// Method: x = 2^e * m with m in [sqrt(1/2), sqrt(2)); log(m) = 2*atanh(s) with
// s = (m-1)/(m+1), |s| <= 0.1716, summed as the Taylor series of atanh
// (2*(s + s^3/3 + s^5/5 + ...)) truncated after s^11; the truncation error is below
// 2e-11 relative, so the result is within a few ulp of the true logarithm. Subnormal
// inputs are not supported (callers pass values >= 2^-24).
HRM_HD HRM_FI float log_exact(float x) {
    uint32_t b = float_bits(x);
    int e = (int)((b >> 23) & 0xFFu) - 127;
    float m = bits_float((b & 0x007FFFFFu) | 0x3F800000u);   // m in [1, 2)
    if (m > 1.41421356f) {                                      // fold into [sqrt(1/2), sqrt(2))
        m = fmul(m, 0.5f);
        e += 1;
    }
    float s  = fdiv(fsub(m, 1.0f), fadd(m, 1.0f));
    float z  = fmul(s, s);
    // 2/(2k+1) for k = 5..0, evaluated with Horner's rule.
    float p = 0.18181818f;                       // 2/11
    p = fadd(fmul(p, z), 0.22222222f);           // 2/9
    p = fadd(fmul(p, z), 0.28571429f);           // 2/7
    p = fadd(fmul(p, z), 0.40000000f);           // 2/5
    p = fadd(fmul(p, z), 0.66666667f);           // 2/3
    p = fadd(fmul(p, z), 2.0f);                  // 2
    float log_m = fmul(s, p);
    // ln 2 split into a high part exact in 16 bits and a low correction.
    const float LN2_HI = 0.693145751953125f;
    const float LN2_LO = 1.42860682030941723e-06f;
    float fe = (float)e;
    return fadd(fadd(fmul(fe, LN2_HI), log_m), fmul(fe, LN2_LO));
}

// ---------------------------------------------------------------------------------------
// Philox-4x32-10 counter-based generator, from Salmon, Moraes, Dror and Shaw,
// "Parallel random numbers: as easy as 1, 2, 3" (SC'11), section 3.2: ten rounds of two
// 32x32->64 multiplications with multipliers 0xD2511F53 and 0xCD9E8D57, the key bumped by
// the Weyl constants 0x9E3779B9 and 0xBB67AE85 between rounds.
// ---------------------------------------------------------------------------------------
struct U32x4 { uint32_t x, y, z, w; };

HRM_HD HRM_FI U32x4 philox4x32_10(U32x4 ctr, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * ctr.x;
        uint64_t p1 = (uint64_t)M1 * ctr.z;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        U32x4 n;
        n.x = hi1 ^ ctr.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ ctr.w ^ k1;
        n.w = lo0;
        ctr = n;
        k0 += W0;
        k1 += W1;
    }
    return ctr;
}

// Uniform float in (0, 1]: the top 24 bits plus one, times 2^-24 (exact).
HRM_HD HRM_FI float u01_open0(uint32_t r) {
    return fmul((float)((r >> 8) + 1u), 1.0f / 16777216.0f);
}
// Uniform float in [-1, 1): 2*(top 24 bits)*2^-24 - 1 (exact).
HRM_HD HRM_FI float u_pm1(uint32_t r) {
    return fsub(fmul((float)(int)(r >> 8), 1.0f / 8388608.0f), 1.0f);
}

// 64-bit mixing function (the splitmix64 finaliser of Steele, Lea and Flood, OOPSLA'14).
HRM_HD HRM_FI uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace hrm

#endif
