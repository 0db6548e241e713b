// Every wait of the runtime is bounded: a wait that nobody will end gives up, raises
// WAIT_TIMEOUT in the instance's flags and returns an error to its caller, and the CUDA
// context stays usable. This program makes each kind of wait run out on purpose, on the
// runtime's own code (include/harmonize/runtime_common.h and event_program.h):
//   take     a consumer owns a queue position whose entry is never published;
//   push     a producer owns a position of a full queue that nobody drains;
//   barrier  the grid barrier of a cooperative EventProgram launch expects two CTAs, one comes.
// Each wait takes about SPIN_LIMIT polls (a fraction of a second). It also checks that a
// publish-then-take round trip still works and raises nothing. Prints one line per case and
// exits 0 when every case behaved as described.
#include "harmonize.h"

#include <cstdio>

using namespace hrm_rt;

struct Result {
    unsigned int ok;     // the call's own return: entry, or 1/0 for success
    unsigned int flags;  // instance flags after the call
};

__global__ void init_ring(RingSet rs, RuntimeControl* ctl) {
    ring_init_slots(rs, 1u, threadIdx.x, blockDim.x);
    if (threadIdx.x == 0) ctl->flags = 0u;
}

// Lane 0 takes position 0 of a ring to which nothing was published.
__global__ void take_unpublished(RingSet rs, RuntimeControl* ctl, Result* out) {
    if (threadIdx.x != 0) return;
    out->ok = ring_take(rs, ctl, 0u, 0u, 0u, 1u);
    __threadfence();
    out->flags = ld_relaxed(&ctl->flags);
}

// The warp publishes 32 entries (a ring of capacity 32 is then full), then lane 0 pushes one
// more: its slot still holds an entry that no consumer took.
__global__ void push_full(RingSet rs, RuntimeControl* ctl, Result* out) {
    const unsigned int lane = threadIdx.x & 31u;
    const bool first = ring_push(rs, ctl, 0u, encode_link(lane, 1u), lane, 32u, 0xFFFFFFFFu);
    if (lane == 0) {
        const bool second = ring_push(rs, ctl, 0u, encode_link(99u, 1u), 0u, 1u, 1u);
        __threadfence();
        out->ok = (first ? 2u : 0u) | (second ? 1u : 0u);
        out->flags = ld_relaxed(&ctl->flags);
    }
}

// Publish one entry, then take it back: no wait runs out.
__global__ void round_trip(RingSet rs, RuntimeControl* ctl, Result* out) {
    if (threadIdx.x != 0) return;
    const bool pushed = ring_push(rs, ctl, 0u, encode_link(7u, 3u), 0u, 1u, 1u);
    unsigned int pos = 0;
    const unsigned int got = ring_reserve(rs, 0u, 1u, pos);
    const unsigned int e = got ? ring_take(rs, ctl, 0u, pos, 0u, 1u) : 0u;
    out->ok = (pushed && got == 1u && entry_link(e) == 7u && entry_count(e) == 3u) ? 1u : 0u;
    out->flags = ld_relaxed(&ctl->flags);
}

// One CTA arrives at a grid barrier that expects two.
__global__ void lone_barrier(EventControl* ec, RuntimeControl* ctl, Result* out) {
    const bool ok = grid_barrier(ec, ctl);
    if (threadIdx.x == 0) {
        out->ok = ok ? 1u : 0u;
        out->flags = ld_relaxed(&ctl->flags);
    }
}

static bool check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    return e == cudaSuccess;
}

int main() {
    const unsigned int CAP = 32u;
    RingHead* heads = nullptr;
    unsigned long long* slots = nullptr;
    RuntimeControl* ctl = nullptr;
    EventControl* ec = nullptr;
    Result* res = nullptr;
    if (!check(cudaMalloc(&heads, sizeof(RingHead)), "malloc") ||
        !check(cudaMalloc(&slots, sizeof(unsigned long long) * CAP), "malloc") ||
        !check(cudaMalloc(&ctl, sizeof(RuntimeControl)), "malloc") ||
        !check(cudaMalloc(&ec, sizeof(EventControl)), "malloc") || !check(cudaMalloc(&res, sizeof(Result)), "malloc"))
        return 1;
    RingSet rs{heads, slots, CAP - 1u};
    Result h{};
    bool all = true;

    auto fresh = [&]() {
        check(cudaMemset(ctl, 0, sizeof(RuntimeControl)), "memset");
        check(cudaMemset(res, 0, sizeof(Result)), "memset");
        init_ring<<<1, 32>>>(rs, ctl);
        return check(cudaDeviceSynchronize(), "init");
    };
    auto read = [&](const char* name) {
        bool ok = check(cudaDeviceSynchronize(), name) && check(cudaMemcpy(&h, res, sizeof(h), cudaMemcpyDeviceToHost), name);
        return ok;
    };

    all &= fresh();
    take_unpublished<<<1, 32>>>(rs, ctl, res);
    bool c1 = read("take") && h.ok == 0u && (h.flags & WAIT_TIMEOUT_FLAG);
    std::printf("take     entry=%u flags=0x%08x %s\n", h.ok, h.flags, c1 ? "timed out as expected" : "UNEXPECTED");

    all &= fresh();
    push_full<<<1, 32>>>(rs, ctl, res);
    bool c2 = read("push") && h.ok == 2u && (h.flags & WAIT_TIMEOUT_FLAG);
    std::printf("push     first/second=%u flags=0x%08x %s\n", h.ok, h.flags, c2 ? "timed out as expected" : "UNEXPECTED");

    all &= fresh();
    check(cudaMemset(ec, 0, sizeof(EventControl)), "memset");
    EventControl ech{};
    ech.blocks = 2u;
    check(cudaMemcpy(ec, &ech, sizeof(ech), cudaMemcpyHostToDevice), "copy");
    lone_barrier<<<1, 64>>>(ec, ctl, res);
    bool c3 = read("barrier") && h.ok == 0u && (h.flags & WAIT_TIMEOUT_FLAG);
    std::printf("barrier  ok=%u flags=0x%08x %s\n", h.ok, h.flags, c3 ? "timed out as expected" : "UNEXPECTED");

    all &= fresh();
    round_trip<<<1, 32>>>(rs, ctl, res);
    bool c4 = read("round trip") && h.ok == 1u && h.flags == 0u;
    std::printf("roundtrip ok=%u flags=0x%08x %s\n", h.ok, h.flags, c4 ? "no wait ran out" : "UNEXPECTED");

    cudaFree(heads);
    cudaFree(slots);
    cudaFree(ctl);
    cudaFree(ec);
    cudaFree(res);
    bool usable = check(cudaDeviceSynchronize(), "context");
    return (all && c1 && c2 && c3 && c4 && usable) ? 0 : 1;
}
