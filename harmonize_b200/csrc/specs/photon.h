// photon.h — Monte Carlo optical photon random walk as a three-function async program.
//
// Workload (no counterpart file in Harmonize; the closest relative is the neutron example,
// examples/cpp/example_neutron/program.cpp:11-44, whose float tallies are not
// reproducible). Here every random number is a pure function of (photon id, step, phase)
// and tallies are integers, so results do not depend on scheduling order:
//  * an n^3 grid of unit voxels; voxel v has scattering coefficient mu_s[v], absorbed
//    fraction absorb[v] and a split flag split[v];
//  * photons start with weight 1 at the grid centre in an isotropic direction;
//  * Move: sample a free path -ln(u)/mu_s; if it ends inside the voxel, move there and
//    Collide; otherwise move to the voxel face, enter the neighbour (split x2 at half
//    weight if the neighbour is flagged, re-sample the path there) or escape the grid;
//  * Collide: deposit weight*absorb (Tally), keep the rest; below weight 1e-3 play Russian
//    roulette (survive with probability 0.1 at ten times the weight); scatter isotropically;
//  * Tally: add a 2^-32 fixed-point amount to a uint64 slot (atomic, order-independent).
// Random numbers: Philox-4x32-10 with key = 64-bit photon id and counter =
// (step, phase, seed_lo, seed_hi). Child ids are mix64 of (parent id, step, child index).
// Floating point: every operation goes through hrm::f* (exactly rounded binary32), and
// the logarithm is hrm::log_exact, so host and device results are bit-identical.
#ifndef HRM_SPECS_PHOTON_H
#define HRM_SPECS_PHOTON_H

#include "../../../include/harmonize/spec_support.h"

namespace hrm_specs {

// Tally layout: [0, n^3) voxels, then PHOTON_SPREAD slots each for escaped weight,
// roulette-killed weight and roulette-gained weight (spread to avoid one hot address).
static const unsigned int PHOTON_SPREAD = 1024u;

struct Photon {
    float x, y, z;
    float dx, dy, dz;
    float w;
    unsigned int id_lo, id_hi;
    unsigned int step;
    unsigned int voxel;
};

// A photon at a collision point. A collision redraws the direction, so a Collide promise
// carries no direction: 8 argument words instead of the 11 of a moving photon.
struct PhotonHit {
    float x, y, z;
    float w;
    unsigned int id_lo, id_hi;
    unsigned int step;
    unsigned int voxel;
};

struct PhotonState {
    const float* mu_s;
    const float* absorb;
    const unsigned char* split;
    unsigned long long* tally;                      // n^3 + 3*PHOTON_SPREAD slots
    util::iter::AtomicIter<unsigned int>* source;  // photon ids still to launch
    unsigned int n;                                 // grid edge (voxels)
    unsigned int seed_lo, seed_hi;
    unsigned int leap;                              // photons per lane per make_work call
    float load_limit;                               // stop launching above this load fraction
};

static const unsigned int PHASE_MOVE = 0u;
static const unsigned int PHASE_ROULETTE = 1u;
static const unsigned int PHASE_DIR = 2u;   // direction draws use phases 2 .. 2+15
static const float WEIGHT_CUTOFF = 1.0e-3f;
static const float ROULETTE_SURVIVAL = 0.1f;
static const float ROULETTE_BOOST = 10.0f;

HRM_HD HRM_FI hrm::U32x4 photon_rng(const PhotonState& s, unsigned int id_lo, unsigned int id_hi, unsigned int step,
                                     unsigned int phase) {
    hrm::U32x4 ctr = {step, phase, s.seed_lo, s.seed_hi};
    return hrm::philox4x32_10(ctr, id_lo, id_hi);
}

HRM_HD HRM_FI unsigned long long to_fixed(float x) {
    // x in [0, 1]; scaling by 2^32 is exact, conversion truncates on both sides.
    return (unsigned long long)hrm::fmul(x, 4294967296.0f);
}

// One Marsaglia trial on the random words (a, b): true, with the direction set, if the
// point (u, v) they give falls inside the unit disc (and is not its centre).
HRM_HD HRM_FI bool disc_trial(unsigned int a, unsigned int b, float& dx, float& dy, float& dz) {
    const float u = hrm::u_pm1(a);
    const float v = hrm::u_pm1(b);
    const float s = hrm::fadd(hrm::fmul(u, u), hrm::fmul(v, v));
    if (!(s < 1.0f && s > 0.0f)) return false;
    const float f = hrm::fmul(2.0f, hrm::fsqrt(hrm::fsub(1.0f, s)));
    dx = hrm::fmul(u, f);
    dy = hrm::fmul(v, f);
    dz = hrm::fsub(1.0f, hrm::fmul(2.0f, s));
    return true;
}

// Isotropic unit vector by Marsaglia's method (Ann. Math. Stat. 43, 1972): draw (u, v)
// uniform in the unit disc, return (2u*sqrt(1-s), 2v*sqrt(1-s), 1-2s) with s = u^2+v^2.
// Each Philox draw gives two trials, (x, y) then (z, w).
HRM_HD HRM_FI void isotropic(const PhotonState& st, unsigned int id_lo, unsigned int id_hi, unsigned int step,
                             float& dx, float& dy, float& dz) {
    for (unsigned int a = 0; a < 16u; a++) {
        const hrm::U32x4 r = photon_rng(st, id_lo, id_hi, step, PHASE_DIR + a);
        if (disc_trial(r.x, r.y, dx, dy, dz)) return;
        if (disc_trial(r.z, r.w, dx, dy, dz)) return;
    }
    dx = 0.0f;
    dy = 0.0f;
    dz = 1.0f;
}

struct PhotonMove;
struct PhotonCollide;
struct PhotonTally;

// A tally is one 64-bit word: the tally slot in bits 33-63 and the 2^-32 fixed-point amount
// in bits 0-32 (an amount is at most 2^32: photon weights never exceed 1).
HRM_HD HRM_FI unsigned long long tally_word(unsigned int slot, unsigned long long amount) {
    return ((unsigned long long)slot << 33) | amount;
}

struct PhotonTally {
    using Type = void (*)(unsigned long long);
    template <typename PROGRAM>
    HRM_DEV static void eval(PROGRAM prog, unsigned long long t) {
        hrm::atomic_add_u64(&prog.device.tally[t >> 33], t & 0x1FFFFFFFFull);
    }
};

// Distance along direction component d from coordinate x to the face of [lo, lo+1) that
// the photon is heading for (the upper face for d > 0, the lower one for d < 0). One
// division whatever the sign, so that the lanes of a warp with mixed signs share it.
HRM_HD HRM_FI float face_distance(float x, float d, unsigned int lo) {
    const bool up = d > 0.0f;
    if (!up && !(d < 0.0f)) return 3.0e38f;  // d is zero (or NaN): no face ahead
    const float face = (float)(up ? lo + 1u : lo);
    const float t = hrm::fdiv(hrm::fsub(face, x), d);
    return t > 0.0f ? t : 0.0f;
}

// Id of child c (0 or 1) of photon `id` split at step `step`.
HRM_HD HRM_FI unsigned long long child_id(unsigned long long id, unsigned int step, unsigned int c) {
    return hrm::mix64(id ^ (((unsigned long long)step << 1) | c) * 0x9E3779B97F4A7C15ull);
}

// Voxel index -> (ix, iy, iz): shifts and masks when n is a power of two (the same value for
// every lane of a batch, so the test does not diverge), else two divisions
// (v / (n*n) == (v / n) / n for unsigned v).
HRM_HD HRM_FI void voxel_coords(unsigned int v, unsigned int n, unsigned int& ix, unsigned int& iy, unsigned int& iz) {
    if ((n & (n - 1u)) == 0u) {
#if defined(__CUDA_ARCH__)
        const unsigned int s = (unsigned int)(__ffs((int)n) - 1);
#else
        const unsigned int s = (unsigned int)__builtin_ctz(n);
#endif
        ix = v & (n - 1u);
        iy = (v >> s) & (n - 1u);
        iz = v >> (2u * s);
        return;
    }
    const unsigned int q = v / n;
    ix = v - q * n;
    iz = q / n;
    iy = q - iz * n;
}

struct PhotonMove {
    using Type = void (*)(Photon);
    template <typename PROGRAM>
    HRM_DEV static void eval(PROGRAM prog, Photon p) {
        const PhotonState& s = prog.device;
        const unsigned int n = s.n;
        unsigned int ix, iy, iz;
        voxel_coords(p.voxel, n, ix, iy, iz);
        float mu = s.mu_s[p.voxel];
        hrm::U32x4 r = photon_rng(s, p.id_lo, p.id_hi, p.step, PHASE_MOVE);
        float dist = hrm::fdiv(hrm::fsub(0.0f, hrm::log_exact(hrm::u01_open0(r.x))), mu);
        float tx = face_distance(p.x, p.dx, ix);
        float ty = face_distance(p.y, p.dy, iy);
        float tz = face_distance(p.z, p.dz, iz);
        unsigned int axis = 0;
        float tb = tx;
        if (ty < tb) { tb = ty; axis = 1; }
        if (tz < tb) { tb = tz; axis = 2; }
        p.step += 1u;
        // Advance to the collision point, or to the face crossed first.
        const bool collide = dist < tb;
        const float t = collide ? dist : tb;
        p.x = hrm::fadd(p.x, hrm::fmul(t, p.dx));
        p.y = hrm::fadd(p.y, hrm::fmul(t, p.dy));
        p.z = hrm::fadd(p.z, hrm::fmul(t, p.dz));
        if (collide) {
            const PhotonHit h = {p.x, p.y, p.z, p.w, p.id_lo, p.id_hi, p.step, p.voxel};
            prog.template async<PhotonCollide>(h);
            return;
        }
        // Land exactly on the face and step the voxel index along the crossing axis (written
        // with selects, so that the lanes of a warp crossing different faces do not diverge).
        const float d_axis = axis == 0 ? p.dx : (axis == 1 ? p.dy : p.dz);
        const unsigned int c = axis == 0 ? ix : (axis == 1 ? iy : iz);
        const bool up = d_axis > 0.0f;
        const float face = (float)(up ? c + 1u : c);
        const bool out = up ? (c + 1u == n) : (c == 0u);
        const unsigned int c_next = up ? c + 1u : c - 1u;
        p.x = axis == 0 ? face : p.x;
        p.y = axis == 1 ? face : p.y;
        p.z = axis == 2 ? face : p.z;
        ix = axis == 0 ? c_next : ix;
        iy = axis == 1 ? c_next : iy;
        iz = axis == 2 ? c_next : iz;
        if (out) {
            prog.template async<PhotonTally>(tally_word(n * n * n + (p.id_lo & (PHOTON_SPREAD - 1u)), to_fixed(p.w)));
            return;
        }
        p.voxel = ix + n * (iy + n * iz);
        // Entering a flagged voxel splits the photon into two children of half weight. The
        // first call below is the photon itself or its first child, the second one the
        // second child, so that a warp with and without splits makes two calls, not three.
        const bool split = s.split[p.voxel] != 0;
        const unsigned long long id = ((unsigned long long)p.id_hi << 32) | p.id_lo;
        Photon q = p;
        if (split) {
            q.w = hrm::fmul(p.w, 0.5f);
            const unsigned long long cid = child_id(id, p.step, 0u);
            q.id_lo = (unsigned int)cid;
            q.id_hi = (unsigned int)(cid >> 32);
        }
        prog.template async<PhotonMove>(q);
        if (split) {
            const unsigned long long cid = child_id(id, p.step, 1u);
            q.id_lo = (unsigned int)cid;
            q.id_hi = (unsigned int)(cid >> 32);
            prog.template async<PhotonMove>(q);
        }
    }
};

struct PhotonCollide {
    using Type = void (*)(PhotonHit);
    template <typename PROGRAM>
    HRM_DEV static void eval(PROGRAM prog, PhotonHit h) {
        const PhotonState& s = prog.device;
        const unsigned int n = s.n;
        float dep = hrm::fmul(h.w, s.absorb[h.voxel]);
        float w = hrm::fsub(h.w, dep);
        prog.template async<PhotonTally>(tally_word(h.voxel, to_fixed(dep)));
        if (w < WEIGHT_CUTOFF) {
            // Russian roulette: a survivor tallies the weight it gains, a loser the weight it
            // loses (one call site for both, so that a warp of both kinds makes one call).
            hrm::U32x4 r = photon_rng(s, h.id_lo, h.id_hi, h.step, PHASE_ROULETTE);
            const unsigned int spread = h.id_lo & (PHOTON_SPREAD - 1u);
            const bool survive = hrm::u01_open0(r.x) <= ROULETTE_SURVIVAL;
            const float boosted = hrm::fmul(w, ROULETTE_BOOST);
            const unsigned int slot = n * n * n + (survive ? 2u : 1u) * PHOTON_SPREAD + spread;
            prog.template async<PhotonTally>(tally_word(slot, survive ? to_fixed(hrm::fsub(boosted, w)) : to_fixed(w)));
            if (!survive) return;
            w = boosted;
        }
        Photon p;
        p.x = h.x;
        p.y = h.y;
        p.z = h.z;
        p.w = w;
        p.id_lo = h.id_lo;
        p.id_hi = h.id_hi;
        p.voxel = h.voxel;
        isotropic(s, h.id_lo, h.id_hi, h.step, p.dx, p.dy, p.dz);
        p.step = h.step + 1u;
        prog.template async<PhotonMove>(p);
    }
};

// A photon launched from the grid centre (a voxel corner when n is even): it starts in
// the voxel its direction points into.
HRM_HD HRM_FI Photon photon_source(const PhotonState& s, unsigned int id) {
    Photon p;
    const unsigned int h = s.n / 2u;
    p.x = (float)h;
    p.y = (float)h;
    p.z = (float)h;
    p.id_lo = id;
    p.id_hi = 0u;
    p.step = 0u;
    p.w = 1.0f;
    isotropic(s, p.id_lo, p.id_hi, 0u, p.dx, p.dy, p.dz);
    unsigned int ix = p.dx >= 0.0f ? h : h - 1u;
    unsigned int iy = p.dy >= 0.0f ? h : h - 1u;
    unsigned int iz = p.dz >= 0.0f ? h : h - 1u;
    p.voxel = ix + s.n * (iy + s.n * iz);
    p.step = 1u;
    return p;
}

// The same walk without the async runtime: one thread follows a source photon and all of
// its split descendants (explicit stack of `cap` entries), making the same tallies in the
// same units. Used by the plain one-thread-per-photon baseline. Returns false if the stack
// overflowed (the remaining descendants are dropped).
template <unsigned int STACK = 48>
HRM_HD HRM_FI bool photon_walk_thread(const PhotonState& s, unsigned int id, unsigned long long* calls) {
    const unsigned int n = s.n;
    const unsigned int S = PHOTON_SPREAD;
    Photon stack[STACK];
    unsigned int top = 0;
    bool ok = true;
    stack[top++] = photon_source(s, id);
    unsigned long long k = 0;
    while (top) {
        Photon p = stack[--top];
        while (true) {
            k++;  // move
            unsigned int ix, iy, iz;
            voxel_coords(p.voxel, n, ix, iy, iz);
            hrm::U32x4 r = photon_rng(s, p.id_lo, p.id_hi, p.step, PHASE_MOVE);
            float dist = hrm::fdiv(hrm::fsub(0.0f, hrm::log_exact(hrm::u01_open0(r.x))), s.mu_s[p.voxel]);
            float tx = face_distance(p.x, p.dx, ix);
            float ty = face_distance(p.y, p.dy, iy);
            float tz = face_distance(p.z, p.dz, iz);
            unsigned int axis = 0;
            float tb = tx;
            if (ty < tb) { tb = ty; axis = 1; }
            if (tz < tb) { tb = tz; axis = 2; }
            p.step += 1u;
            if (dist < tb) {
                p.x = hrm::fadd(p.x, hrm::fmul(dist, p.dx));
                p.y = hrm::fadd(p.y, hrm::fmul(dist, p.dy));
                p.z = hrm::fadd(p.z, hrm::fmul(dist, p.dz));
                k++;  // collide
                float dep = hrm::fmul(p.w, s.absorb[p.voxel]);
                p.w = hrm::fsub(p.w, dep);
                k++;
                hrm::atomic_add_u64(&s.tally[p.voxel], to_fixed(dep));
                if (p.w < WEIGHT_CUTOFF) {
                    hrm::U32x4 rr = photon_rng(s, p.id_lo, p.id_hi, p.step, PHASE_ROULETTE);
                    unsigned int spread = p.id_lo & (S - 1u);
                    k++;
                    if (hrm::u01_open0(rr.x) <= ROULETTE_SURVIVAL) {
                        float boosted = hrm::fmul(p.w, ROULETTE_BOOST);
                        hrm::atomic_add_u64(&s.tally[n * n * n + 2u * S + spread], to_fixed(hrm::fsub(boosted, p.w)));
                        p.w = boosted;
                    } else {
                        hrm::atomic_add_u64(&s.tally[n * n * n + S + spread], to_fixed(p.w));
                        break;
                    }
                }
                isotropic(s, p.id_lo, p.id_hi, p.step, p.dx, p.dy, p.dz);
                p.step += 1u;
                continue;
            }
            p.x = hrm::fadd(p.x, hrm::fmul(tb, p.dx));
            p.y = hrm::fadd(p.y, hrm::fmul(tb, p.dy));
            p.z = hrm::fadd(p.z, hrm::fmul(tb, p.dz));
            bool out = false;
            if (axis == 0) {
                if (p.dx > 0.0f) { p.x = (float)(ix + 1u); out = (ix + 1u == n); ix += 1u; }
                else { p.x = (float)ix; out = (ix == 0u); ix -= 1u; }
            } else if (axis == 1) {
                if (p.dy > 0.0f) { p.y = (float)(iy + 1u); out = (iy + 1u == n); iy += 1u; }
                else { p.y = (float)iy; out = (iy == 0u); iy -= 1u; }
            } else {
                if (p.dz > 0.0f) { p.z = (float)(iz + 1u); out = (iz + 1u == n); iz += 1u; }
                else { p.z = (float)iz; out = (iz == 0u); iz -= 1u; }
            }
            if (out) {
                k++;
                hrm::atomic_add_u64(&s.tally[n * n * n + (p.id_lo & (S - 1u))], to_fixed(p.w));
                break;
            }
            p.voxel = ix + n * (iy + n * iz);
            if (s.split[p.voxel]) {
                p.w = hrm::fmul(p.w, 0.5f);
                unsigned long long id64 = ((unsigned long long)p.id_hi << 32) | p.id_lo;
                for (unsigned int c = 0; c < 2u; c++) {
                    unsigned long long cid = child_id(id64, p.step, c);
                    Photon q = p;
                    q.id_lo = (unsigned int)cid;
                    q.id_hi = (unsigned int)(cid >> 32);
                    if (top < STACK) stack[top++] = q;
                    else ok = false;
                }
                break;
            }
        }
    }
    if (calls) *calls += k;
    return ok;
}

template <size_t RING = 2, size_t TEAMS = 4>
struct PhotonSpec {
    typedef OpUnion<PhotonMove, PhotonCollide, PhotonTally> OpSet;
    typedef PhotonState DeviceState;

    static const size_t STASH_SIZE = 8;
    static const size_t FRAME_SIZE = 16069;
    static const size_t POOL_SIZE = 16069;
    static const size_t RING_LINKS = RING;
    static const size_t TEAMS_PER_CTA = TEAMS;
    // Collide has half the ring links of the others (at least 2): a batch of moves makes at
    // most one collide per lane, so two links always hold a batch's calls, and the smaller
    // stash leaves room for more teams per SM (R4/T2: 12 CTAs instead of 10).
    template <typename Op>
    struct RING_LINKS_OF {
        static const size_t value = std::is_same<Op, PhotonCollide>::value ? (RING / 2 < 2 ? 2 : RING / 2) : RING;
    };

    template <typename PROGRAM>
    HRM_DEV static void initialize(PROGRAM) {}
    template <typename PROGRAM>
    HRM_DEV static void finalize(PROGRAM) {}

    template <typename PROGRAM>
    HRM_DEV static bool make_work(PROGRAM prog) {
        // EventProgram: stop launching while the move buffer is loaded (load_fraction is NaN
        // under AsyncProgram, so the comparison is false there).
        float load = prog.template load_fraction<PhotonMove>();
        if (load > prog.device.load_limit) return false;
        util::iter::Iter<unsigned int> it = prog.device.source->leap(prog.device.leap);
        unsigned int id;
        while (it.step(id)) {
            prog.template async<PhotonMove>(photon_source(prog.device, id));
        }
        return !prog.device.source->done();
    }
};

}  // namespace hrm_specs

#endif
