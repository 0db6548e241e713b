// Compile-time checks of the optional spec members this runtime reads (no kernel runs): a
// member a spec defines is honoured, a member it leaves out takes its default, and the
// per-function forms (RING_LINKS_OF, RING_GROUP_OF, OLDEST_FIRST_OF) override the spec-wide
// ones function by function. Built with `nvcc -c`; a failed check is a compile error.
#include "harmonize.h"
#include "../../harmonize_b200/csrc/specs/mix.h"

using namespace hrm_specs;
using hrm_rt::fn_OLDEST_FIRST;
using hrm_rt::fn_RING_GROUP;
using hrm_rt::fn_RING_LINKS;

// Spec-wide values, and their defaults.
static_assert(hrm_rt::spec_RING_LINKS<PhotonSpec<4, 2>>::value == 4, "RING_LINKS from the spec");
static_assert(hrm_rt::spec_TEAMS_PER_CTA<PhotonSpec<4, 2>>::value == 2, "TEAMS_PER_CTA from the spec");
static_assert(hrm_rt::spec_MIN_CTAS_PER_SM<PhotonSpec<4, 2>>::value == 1, "MIN_CTAS_PER_SM default");
static_assert(hrm_rt::spec_COALESCE_PATIENCE<CollatzSpec<>>::value == 16, "COALESCE_PATIENCE default");
static_assert(hrm_rt::spec_OLDEST_FIRST<CollatzSpec<>>::value == 0, "OLDEST_FIRST default");
static_assert(hrm_rt::spec_OLDEST_FIRST<BfsSpec<>>::value == 1, "BFS takes oldest first");

// Per function, single-spec: every function follows the spec-wide value.
static_assert(fn_OLDEST_FIRST<BfsSpec<2, 8>, BfsRelax>::value && fn_OLDEST_FIRST<BfsSpec<2, 8>, BfsExpand>::value,
              "BFS functions oldest first");
static_assert(!fn_OLDEST_FIRST<PhotonSpec<4, 2>, PhotonMove>::value, "photon newest first");
static_assert(!fn_OLDEST_FIRST<CollatzSpec<>, CollatzOdd>::value, "Collatz newest first");
static_assert(fn_RING_LINKS<CollatzSpec<4, 2>, CollatzOdd>::value == 4, "no RING_LINKS_OF: RING_LINKS");
static_assert(fn_RING_LINKS<PhotonSpec<4, 2>, PhotonTally>::value == 4, "RING_LINKS_OF: RING_LINKS for the others");
static_assert(fn_RING_LINKS<PhotonSpec<4, 2>, PhotonCollide>::value == 2, "RING_LINKS_OF: collide half");
static_assert(fn_RING_LINKS<PhotonSpec<2, 4>, PhotonCollide>::value == 2, "RING_LINKS_OF: at least 2 links");
static_assert(fn_RING_GROUP<PhotonSpec<4, 2>, PhotonMove>::value == 0, "no RING_GROUP_OF: one group");

// Per function, the job-multiplexing spec: groups by job kind, photon rings RING links and
// the others 2*RING, BFS functions oldest first and the others newest first.
using Mix42 = MixSpec<4, 2>;
static_assert(fn_RING_GROUP<Mix42, Job<CollatzEven>>::value == JOB_COLLATZ, "Collatz group");
static_assert(fn_RING_GROUP<Mix42, Job<PhotonCollide>>::value == JOB_PHOTON, "photon group");
static_assert(fn_RING_GROUP<Mix42, Job<BfsExpand>>::value == JOB_BFS, "BFS group");
static_assert(fn_RING_LINKS<Mix42, Job<PhotonMove>>::value == 4, "photon rings");
static_assert(fn_RING_LINKS<Mix42, Job<PhotonCollide>>::value == 2, "photon collide rings: half");
static_assert(fn_RING_LINKS<Mix42, Job<CollatzEven>>::value == 8, "Collatz rings");
static_assert(fn_RING_LINKS<Mix42, Job<BfsRelax>>::value == 8, "BFS rings");
static_assert(fn_OLDEST_FIRST<Mix42, Job<BfsRelax>>::value && fn_OLDEST_FIRST<Mix42, Job<BfsExpand>>::value,
              "BFS jobs oldest first");
static_assert(!fn_OLDEST_FIRST<Mix42, Job<PhotonMove>>::value && !fn_OLDEST_FIRST<Mix42, Job<CollatzEven>>::value,
              "other jobs newest first");

// Discriminants are 0-based positions in the OpUnion, as in the original runtime.
static_assert(OpUnionLookup<PhotonTally, PhotonSpec<4, 2>::OpSet>::DISC == 2, "DISC = position");
static_assert(OpUnionLookup<Job<BfsExpand>, Mix42::OpSet>::DISC == 6, "DISC = position");

// Promises are moved as packed 32-bit words: arguments end to end in call order, each rounded
// up to whole words, with no alignment padding between them.
static_assert(Promise<CollatzEven>::WORDS == 4, "(u64, u32, u32): 4 words");
static_assert(Promise<PhotonMove>::WORDS == 11, "a moving photon: 11 words");
static_assert(Promise<PhotonCollide>::WORDS == 8, "a photon at a collision: 8 words (no direction)");
static_assert(Promise<PhotonTally>::WORDS == 2, "a tally: one 64-bit word");
static_assert(Promise<BfsRelax>::WORDS == 2 && Promise<BfsExpand>::WORDS == 4, "BFS: 2 and 4 words");
static_assert(Promise<Job<CollatzEven>>::WORDS == 5, "(u32 job, u64, u32, u32): 5 words, not the 6 of its ArgTuple");
static_assert(Promise<Job<PhotonTally>>::WORDS == 3, "(u32 job, u64): 3 words");
static_assert(ArgWordOffset<1, Promise<Job<CollatzEven>>::Args>::value == 1, "the u64 right after the job id");
static_assert(ArgWordOffset<3, Promise<Job<CollatzEven>>::Args>::value == 4, "last argument at word 4");

// Team rings need not be powers of two: a 3-link photon spec (Collide 2 links) has 96-slot Move
// and Tally rings, and ring positions wrap by one subtraction below 2 * SLOTS.
using Photon3 = AsyncProgram<PhotonSpec<3, 2>>;
static_assert(Photon3::ring_slots<0>() == 96 && Photon3::ring_slots<1>() == 64 && Photon3::ring_slots<2>() == 96,
              "3-link rings: Move 96, Collide 64, Tally 96 slots");
static_assert(Photon3::RING_WORDS == 96 * 11 + 64 * 8 + 96 * 2, "stash words of the 3-link photon spec");
static_assert(Photon3::wrap_slot<96>(95) == 95 && Photon3::wrap_slot<96>(96) == 0 && Photon3::wrap_slot<96>(191) == 95,
              "96-slot ring wraps at 96");
static_assert(Photon3::wrap_slot<128>(200) == 72 && Photon3::wrap_slot<64>(64) == 0, "power-of-two rings mask");
