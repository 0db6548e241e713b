// Compile-time checks of the co-residency arithmetic (hrm_capi::ctas_beside) on a B200's
// per-SM limits: 233,472 B of shared memory with 1,024 B reserved per CTA, 65,536 registers
// in four sub-partitions, 2,048 threads, 32 CTAs. The serving session sizes the resident
// kernel's share and the solo photon kernel beside it with this function.
#include "harmonize.h"
#include "../../harmonize_b200/csrc/capi_internal.h"
#include "../../harmonize_b200/csrc/specs/collatz.h"
#include "../../harmonize_b200/csrc/specs/photon.h"

using hrm_capi::ctas_beside;
using hrm_capi::CtaFootprint;
using hrm_capi::SmLimits;

constexpr SmLimits B200{233472u, 1024u, 65536u, 2048u, 32u};
constexpr CtaFootprint NONE{0u, 0u, 0u};

// Alone on an SM: the exec kernels of the tuned variants, with the registers ptxas gives them
// under their launch bounds and the stash sizes of their program types (as ncu reported them).
using hrm_capi::MinCtas;
using PhotonR4T2M11 = AsyncProgram<MinCtas<hrm_specs::PhotonSpec<4, 2>, 11>>;
using PhotonR3T2M14 = AsyncProgram<MinCtas<hrm_specs::PhotonSpec<3, 2>, 14>>;
using CollatzR3T2M14 = AsyncProgram<MinCtas<hrm_specs::CollatzSpec<3, 2>, 14>>;
static_assert(PhotonR4T2M11::SMEM_BYTES == 18176u && PhotonR3T2M14::SMEM_BYTES == 14848u &&
                  CollatzR3T2M14::SMEM_BYTES == 6880u,
              "stash bytes per CTA of 2 teams: photon R4 18,176, photon R3 14,848, Collatz R3 6,880");
static_assert(PhotonR4T2M11::CTA_THREADS == 64u && PhotonR3T2M14::MIN_CTAS_PER_SM == 14u, "2 teams; launch bound");
constexpr CtaFootprint PHOTON_R4_T2_M11{80u, 64u, PhotonR4T2M11::SMEM_BYTES};    // 12 CTAs: shared memory and registers
constexpr CtaFootprint COLLATZ_R3_T2_M14{72u, 64u, CollatzR3T2M14::SMEM_BYTES};  // 14 CTAs: registers (7 warps per sub-partition)
constexpr CtaFootprint PHOTON_R3_T2_M14{72u, 64u, PhotonR3T2M14::SMEM_BYTES};    // 14 CTAs: shared memory and registers
static_assert(ctas_beside(NONE, 0u, PHOTON_R4_T2_M11, B200) == 12u, "photon R4/T2: 12 CTAs per SM");
static_assert(ctas_beside(NONE, 0u, COLLATZ_R3_T2_M14, B200) == 14u, "Collatz R3/T2: 14 CTAs per SM");
static_assert(ctas_beside(NONE, 0u, PHOTON_R3_T2_M14, B200) == 14u, "photon R3/T2: 14 CTAs per SM");
static_assert(ctas_beside(PHOTON_R4_T2_M11, 12u, PHOTON_R4_T2_M11, B200) == 0u, "a full SM takes nothing beside");

// Registers are counted per sub-partition: 3 CTAs of a 2-warp, 126-register kernel put 2 warps
// (8,192 registers) in some sub-partition, which leaves room for 2 CTAs of 4 warps at 96
// registers (one warp each per sub-partition, 3,072 registers), not the 3 that the SM's total
// (65,536 - 24,576 registers) would suggest.
constexpr CtaFootprint MIX{126u, 64u, 0u};
constexpr CtaFootprint SOLO{96u, 128u, 0u};
static_assert(ctas_beside(MIX, 3u, SOLO, B200) == 2u, "per-sub-partition register accounting");
static_assert(ctas_beside(MIX, 4u, SOLO, B200) == 2u, "4 CTAs fill 2 warps per sub-partition too");

// The other limits: CTA slots, threads, shared memory with its per-CTA reservation.
constexpr CtaFootprint TINY{16u, 32u, 0u};
static_assert(ctas_beside(TINY, 30u, TINY, B200) == 2u, "32 CTAs per SM");
static_assert(ctas_beside(CtaFootprint{16u, 1024u, 0u}, 1u, CtaFootprint{16u, 512u, 0u}, B200) == 2u,
              "2,048 threads per SM");
static_assert(ctas_beside(NONE, 0u, CtaFootprint{16u, 32u, 115712u}, B200) == 2u &&
                  ctas_beside(NONE, 0u, CtaFootprint{16u, 32u, 115713u}, B200) == 1u,
              "two CTAs of 113 KB fit with their reservations, one byte more does not");
