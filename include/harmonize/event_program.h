// event_program.h — EventProgram<Spec>: generation-by-generation execution.
//
// Source-level contract kept from harmonize/cpp/program/event.h:
//  * Instance(io_size, DeviceState): each async function owns an input and an output
//    buffer of io_size promises (event.h:139-156); complete() is true when no function
//    has input left (event.h:171-205);
//  * in a generation every pending promise is evaluated once; calls made by the evals go
//    to the output buffers; a team that finds all inputs drained calls make_work until it
//    returns false or some output buffer is half full (event.h:445-472); then input and
//    output swap (event.h:500-515);
//  * exec<P>(inst, groups, chunk): the third argument is the number of promises a lane
//    takes per grab (event.h:383), as in the original;
//  * prog.load_fraction<F>() is the fill fraction of F's output buffer (event.h:540-544).
//
// Internals (B200 design):
//  * buffers are structure-of-arrays 32-bit words per function, so the 32 lanes of a
//    batch read and write 128 contiguous bytes per word;
//  * prog.async<F> reserves output slots with one atomicAdd per warp and call site
//    (active-lane popc rank), instead of one system-scope atomic per call;
//  * between generations one thread turns the per-function output counts into a prefix
//    sum of 32-promise tiles; teams then claim tiles from one counter, so every tile but
//    the last of each function is warp-full and all functions run in the same pass;
//  * generations are driven on the device: one cooperative launch runs generation after
//    generation, separated by a grid barrier whose waits are bounded, until no input is
//    left, a halt is requested or an error flag is raised;
//  * a promise that does not fit raises QUEUE_OVERFLOW_FLAG (the original printed a
//    message and dropped it, event.h:355-357).
#ifndef HARMONIZE_B200_EVENT_PROGRAM_H
#define HARMONIZE_B200_EVENT_PROGRAM_H

#include "runtime_common.h"

template <typename PROGRAM_SPEC>
class EventProgram;

namespace hrm_rt {
template <typename PROG>
__global__ void event_init_kernel(typename PROG::DeviceContext ctx);
template <typename PROG>
__global__ void __launch_bounds__(PROG::CTA_THREADS, PROG::MIN_CTAS_PER_SM)
    event_exec_kernel(typename PROG::DeviceContext ctx, typename PROG::DeviceState device, unsigned int chunk,
                      unsigned int max_generations);

// Per-function buffer bookkeeping of an EventProgram instance.
struct alignas(128) EventCounts {
    unsigned int in_count;   // promises in the current input buffer
    unsigned int out_count;  // output slots reserved so far (may exceed capacity)
    unsigned int tile_base;  // first tile of this function in the current generation
    unsigned int pad;
};

struct alignas(128) EventControl {
    unsigned int side;          // which of the two buffers is the input
    unsigned int total_tiles;   // tiles in the current generation
    unsigned int tile_next;     // next tile to claim
    unsigned int barrier_count; // arrivals at the grid barrier
    unsigned int barrier_gen;   // completed grid barriers
    unsigned int done;          // set when no input is left
    unsigned int blocks;        // CTAs in the current launch
    unsigned int pad;
};

// Grid-wide barrier for a cooperative launch. Every wait is bounded; on timeout the flag is
// raised and false returned to all threads of the CTA.
__device__ __forceinline__ bool grid_barrier(EventControl* ec, RuntimeControl* ctl) {
    __shared__ unsigned int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        unsigned int gen = ld_acquire(&ec->barrier_gen);
        __threadfence();
        unsigned int arrived = atomicAdd(&ec->barrier_count, 1u);
        if (arrived == ec->blocks - 1u) {
            atomicExch(&ec->barrier_count, 0u);
            __threadfence();
            atomicAdd(&ec->barrier_gen, 1u);
        } else {
            unsigned int spins = 0;
            while (ld_acquire(&ec->barrier_gen) == gen) {
                if (++spins > SPIN_LIMIT) {
                    raise_flag(ctl, WAIT_TIMEOUT_FLAG);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}
}  // namespace hrm_rt

template <typename PROGRAM_SPEC>
class EventProgram {
   public:
    typedef EventProgram<PROGRAM_SPEC> ProgramType;
    typedef PROGRAM_SPEC Spec;

    using AdrType = typename hrm_rt::spec_AdrType<PROGRAM_SPEC>::type;
    using OpSet = typename hrm_rt::spec_OpSet<PROGRAM_SPEC>::type;
    using DeviceState = typename hrm_rt::spec_DeviceState<PROGRAM_SPEC>::type;
    using GroupState = typename hrm_rt::spec_GroupState<PROGRAM_SPEC>::type;
    using ThreadState = typename hrm_rt::spec_ThreadState<PROGRAM_SPEC>::type;

    typedef PromiseUnion<OpSet> PromiseUnionType;
    typedef PromiseEnum<OpSet> PromiseEnumType;

    template <typename TYPE>
    struct Lookup {
        typedef typename PromiseUnionType::template Lookup<TYPE>::type type;
    };

    static const size_t GROUP_SIZE = hrm_rt::spec_GROUP_SIZE<PROGRAM_SPEC>::value;
    static const size_t WORK_GROUP_SIZE = GROUP_SIZE;
    static_assert(GROUP_SIZE == 32, "work groups are 32-lane warps");
    static const unsigned int TEAMS_PER_CTA = (unsigned int)hrm_rt::spec_TEAMS_PER_CTA<PROGRAM_SPEC>::value;
    static const unsigned int CTA_THREADS = TEAMS_PER_CTA * 32u;
    static const unsigned int MIN_CTAS_PER_SM = (unsigned int)hrm_rt::spec_MIN_CTAS_PER_SM<PROGRAM_SPEC>::value;

    static const unsigned int BAD_FUNC_ID_FLAG = hrm_rt::BAD_FUNC_ID_FLAG;
    static const unsigned int EARLY_HALT_FLAG = hrm_rt::EARLY_HALT_FLAG;
    static const unsigned int COMPLETION_FLAG = hrm_rt::COMPLETION_FLAG;

    static const unsigned char FN_ID_COUNT = (unsigned char)PromiseUnionType::Info::COUNT;
    static const unsigned int FN = FN_ID_COUNT;
    static_assert(FN >= 1 && FN <= 16, "an operation set holds 1 to 16 async functions");

    using Layout = OpLayout<OpSet>;
    static const unsigned int TOTAL_WORDS = Layout::TOTAL_WORDS;

    // Generations one exec<P> launch may run before returning to the host.
    static const unsigned int MAX_GENERATIONS_PER_EXEC = 1u << 20;

    struct ThreadContext {
        unsigned int thread_id;
        unsigned int rand_state;
        unsigned int out_side;  // buffer receiving this generation's calls
    };
    struct GroupContext {
        unsigned int unused;
    };

    struct DeviceContext {
        typedef ProgramType ParentProgramType;
        hrm_rt::RuntimeControl* ctl;
        hrm_rt::EventControl* ec;
        hrm_rt::EventCounts* counts;   // [FN]
        unsigned int* words;           // function f, side s, word w, index i:
                                       //   words[(word_base[f] + s*W_f + w) * capacity + i]
        unsigned long long* stats;
        unsigned int capacity;
    };

    struct Instance {
        size_t io_size;
        util::host::DevBuf<hrm_rt::RuntimeControl> control;
        util::host::DevBuf<hrm_rt::EventControl> event_control;
        util::host::DevBuf<hrm_rt::EventCounts> counts;
        util::host::DevBuf<unsigned int> words;
        util::host::DevBuf<unsigned long long> stats;
        DeviceState device_state;
        cudaStream_t stream = nullptr;

        __host__ Instance(size_t io, DeviceState ds)
            : io_size(io),
              control((size_t)1),
              event_control((size_t)1),
              counts((size_t)FN),
              words(io * 2u * TOTAL_WORDS),
              stats((size_t)hrm_rt::STAT_COUNT),
              device_state(ds) {
            if (io == 0 || io >= (1ull << 31)) throw std::runtime_error("EventProgram io_size must be in [1, 2^31)");
            util::host::auto_throw(cudaMemset(control.data(), 0, sizeof(hrm_rt::RuntimeControl)));
            util::host::auto_throw(cudaMemset(event_control.data(), 0, sizeof(hrm_rt::EventControl)));
            util::host::auto_throw(cudaMemset(counts.data(), 0, sizeof(hrm_rt::EventCounts) * FN));
            util::host::auto_throw(cudaMemset(stats.data(), 0, sizeof(unsigned long long) * hrm_rt::STAT_COUNT));
        }

        __host__ DeviceContext to_context() {
            DeviceContext c;
            c.ctl = control.data();
            c.ec = event_control.data();
            c.counts = counts.data();
            c.words = words.data();
            c.stats = stats.data();
            c.capacity = (unsigned int)io_size;
            return c;
        }
        __host__ unsigned int flags() {
            unsigned int f = 0;
            util::host::auto_throw(cudaMemcpy(&f, &control.data()->flags, sizeof(f), cudaMemcpyDeviceToHost));
            return f;
        }
        // True when no function has promises waiting in its input buffer. Throws if the
        // device raised an error flag, so that `do { exec } while (!complete())` host loops
        // end instead of spinning.
        __host__ bool complete() {
            unsigned int f = flags();
            if (f & hrm_rt::ERROR_MASK) hrm_rt::throw_flags(f);
            std::vector<hrm_rt::EventCounts> c(FN);
            util::host::auto_throw(
                cudaMemcpy(c.data(), counts.data(), sizeof(hrm_rt::EventCounts) * FN, cudaMemcpyDeviceToHost));
            for (unsigned int i = 0; i < FN; i++) {
                if (c[i].in_count != 0) return false;
            }
            return true;
        }
        __host__ void clear_flags() {
            util::host::auto_throw(cudaMemset(&control.data()->flags, 0, sizeof(unsigned int)));
        }
        // out[f] = promises waiting in function f's input buffer.
        __host__ std::vector<unsigned int> overview() {
            std::vector<hrm_rt::EventCounts> c(FN);
            util::host::auto_throw(
                cudaMemcpy(c.data(), counts.data(), sizeof(hrm_rt::EventCounts) * FN, cudaMemcpyDeviceToHost));
            std::vector<unsigned int> out;
            for (unsigned int f = 0; f < FN; f++) out.push_back(c[f].in_count);
            return out;
        }

        __host__ std::vector<unsigned long long> read_stats() {
            std::vector<unsigned long long> v(hrm_rt::STAT_COUNT);
            util::host::auto_throw(cudaMemcpy(v.data(), stats.data(), sizeof(unsigned long long) * hrm_rt::STAT_COUNT,
                                              cudaMemcpyDeviceToHost));
            return v;
        }
    };

    DeviceContext& _dev_ctx;
    GroupContext& _grp_ctx;
    ThreadContext& _thd_ctx;
    DeviceState& device;
    GroupState& group;
    ThreadState& thread;

    __device__ EventProgram(DeviceContext& d_c, GroupContext& g_c, ThreadContext& t_c, DeviceState& d, GroupState& g,
                            ThreadState& t)
        : _dev_ctx(d_c), _grp_ctx(g_c), _thd_ctx(t_c), device(d), group(g), thread(t) {}

    template <typename TYPE>
    __host__ __device__ static constexpr unsigned int disc_of() {
        static_assert(OpUnionLookup<TYPE, OpSet>::CONTAINED, "async function is not in the spec's OpSet");
        return OpUnionLookup<TYPE, OpSet>::DISC;
    }

    __device__ __forceinline__ unsigned int* word_ptr(unsigned int f_word_base, unsigned int side, unsigned int W,
                                                      unsigned int w, unsigned int i) {
        return _dev_ctx.words + ((size_t)(2u * f_word_base + side * W + w)) * _dev_ctx.capacity + i;
    }

    // prog.async<F>: one slot reservation per warp and call site, then SoA stores.
    template <typename TYPE>
    __device__ __forceinline__ void push_promise(const Promise<TYPE>& p) {
        constexpr unsigned int F = disc_of<TYPE>();
        constexpr unsigned int W = Promise<TYPE>::WORDS;
        constexpr unsigned int OFF = OpWordOffset<F, OpSet>::value;
        unsigned int w[W];
        p.to_words(w);
        const unsigned int mask = __activemask();
        const unsigned int rank = __popc(mask & util::lanemask_lt());
        const unsigned int leader = __ffs(mask) - 1;
        unsigned int base = 0;
        if (rank == 0) base = atomicAdd(&_dev_ctx.counts[F].out_count, (unsigned int)__popc(mask));
        base = __shfl_sync(mask, base, leader);
        const unsigned int idx = base + rank;
        const unsigned int side = _thd_ctx.out_side;
        if (idx < _dev_ctx.capacity) {
#pragma unroll
            for (unsigned int i = 0; i < W; i++) __stcg(word_ptr(OFF, side, W, i, idx), w[i]);
        } else {
            atomicOr(&_dev_ctx.ctl->flags, hrm_rt::QUEUE_OVERFLOW_FLAG);
        }
    }

    template <unsigned int I>
    __device__ __forceinline__ void push_enum(OpDisc disc, PromiseUnionType& u) {
        if constexpr (I < FN) {
            using Op = typename OpAt<I, OpSet>::type;
            if (disc == I) push_promise<Op>(u.template cast<Op>());
            else push_enum<I + 1>(disc, u);
        } else {
            atomicOr(&_dev_ctx.ctl->flags, BAD_FUNC_ID_FLAG);
        }
    }

    template <typename TYPE, typename... ARGS>
    __device__ __forceinline__ void async(ARGS... args) {
        push_promise<TYPE>(Promise<TYPE>(args...));
    }
    template <typename TYPE>
    __device__ __forceinline__ void async_call(Promise<TYPE> promise) {
        push_promise<TYPE>(promise);
    }
    __device__ void async_call(PromiseEnumType promise) { push_enum<0>(promise.disc, promise.data); }
    __device__ void async_call(OpDisc disc, int, PromiseUnionType& promise) { push_enum<0>(disc, promise); }

    template <typename TYPE, typename... ARGS>
    __device__ __forceinline__ void sync(ARGS... args) {
        Promise<TYPE>(args...)(*this);
    }
    template <typename TYPE>
    __device__ __forceinline__ void sync_call(Promise<TYPE> promise) {
        promise(*this);
    }
    template <typename TYPE>
    __device__ float load_fraction() {
        unsigned int v = hrm_rt::ld_relaxed(&_dev_ctx.counts[disc_of<TYPE>()].out_count);
        return (float)v / (float)_dev_ctx.capacity;
    }
    __device__ void halt_early() { atomicOr(&_dev_ctx.ctl->flags, EARLY_HALT_FLAG); }

    // Evaluates input tile promises [start, start+k) of function F.
    template <unsigned int F>
    __device__ __forceinline__ void run_tile(unsigned int start, unsigned int k) {
        using Op = typename OpAt<F, OpSet>::type;
        constexpr unsigned int W = Promise<Op>::WORDS;
        constexpr unsigned int OFF = OpWordOffset<F, OpSet>::value;
        const unsigned int lane = util::lane_id();
        const unsigned int side = 1u - _thd_ctx.out_side;
        if (lane < k) {
            unsigned int w[W];
#pragma unroll
            for (unsigned int i = 0; i < W; i++) w[i] = __ldcg(word_ptr(OFF, side, W, i, start + lane));
            Promise<Op> p;
            p.from_words(w);
            p(*this);
        }
        __syncwarp();
    }

    template <unsigned int I>
    __device__ __forceinline__ void run_fn(unsigned int f, unsigned int start, unsigned int k) {
        if constexpr (I < FN) {
            if (f == I) run_tile<I>(start, k);
            else run_fn<I + 1>(f, start, k);
        }
    }

    // One thread: turn output counts into the next generation's inputs and tile schedule.
    __device__ static void flip(DeviceContext ctx, bool halted) {
        hrm_rt::EventControl* ec = ctx.ec;
        unsigned int tiles = 0;
        for (unsigned int f = 0; f < FN; f++) {
            unsigned int n = atomicExch(&ctx.counts[f].out_count, 0u);
            if (n > ctx.capacity) {
                atomicOr(&ctx.ctl->flags, hrm_rt::QUEUE_OVERFLOW_FLAG);
                n = ctx.capacity;
            }
            atomicExch(&ctx.counts[f].in_count, n);
            atomicExch(&ctx.counts[f].tile_base, tiles);
            tiles += (n + 31u) / 32u;
        }
        atomicXor(&ec->side, 1u);
        atomicExch(&ec->total_tiles, tiles);
        atomicExch(&ec->tile_next, 0u);
        atomicAdd(&ctx.ctl->generation, 1u);
        if (tiles == 0 || halted) atomicExch(&ec->done, 1u);
        __threadfence();
    }

    // The device-driven generation loop.
    __device__ void exec(unsigned int chunk, unsigned int max_generations) {
        const unsigned int lane = util::lane_id();
        _thd_ctx.thread_id = blockIdx.x * blockDim.x + threadIdx.x;
        _thd_ctx.rand_state = _thd_ctx.thread_id;
        hrm_rt::call_initialize<PROGRAM_SPEC>(*this);
        __syncwarp();
        hrm_rt::EventControl* ec = _dev_ctx.ec;
        hrm_rt::RuntimeControl* ctl = _dev_ctx.ctl;
        if (chunk == 0) chunk = 1;
        unsigned long long n_evals = 0, n_batches = 0, n_full = 0, n_mw = 0, n_gen = 0;
        unsigned long long fn_evals = 0;  // lane f counts the evaluations of function f

        for (unsigned int gen = 0; gen < max_generations; gen++) {
            // This generation's schedule: lane f holds function f's first tile and count.
            const unsigned int total = hrm_rt::ld_relaxed(&ec->total_tiles);
            _thd_ctx.out_side = 1u - hrm_rt::ld_relaxed(&ec->side);
            unsigned int my_base = 0xFFFFFFFFu, my_count = 0;
            if (lane < FN) {
                my_base = hrm_rt::ld_relaxed(&_dev_ctx.counts[lane].tile_base);
                my_count = hrm_rt::ld_relaxed(&_dev_ctx.counts[lane].in_count);
            }
            while (true) {
                unsigned int t = 0;
                if (lane == 0) t = atomicAdd(&ec->tile_next, chunk);
                t = __shfl_sync(0xFFFFFFFFu, t, 0);
                if (t >= total) break;
                unsigned int t_end = min(t + chunk, total);
                for (unsigned int tt = t; tt < t_end; tt++) {
                    // The function of tile tt: the last one whose first tile is <= tt.
                    unsigned int le = __ballot_sync(0xFFFFFFFFu, lane < FN && my_base <= tt);
                    unsigned int f = 31u - __clz(le);
                    unsigned int base_f = __shfl_sync(0xFFFFFFFFu, my_base, f);
                    unsigned int count_f = __shfl_sync(0xFFFFFFFFu, my_count, f);
                    unsigned int start = (tt - base_f) * 32u;
                    unsigned int k = min(32u, count_f - start);
                    run_fn<0>(f, start, k);
                    n_evals += k;
                    n_batches += 1;
                    n_full += (k == 32u);
                    if (lane == f) fn_evals += k;
                }
            }
            // All inputs claimed: make work until told to stop or an output is half full.
            unsigned int fl = 0;
            if (lane == 0) fl = hrm_rt::ld_relaxed(&ctl->flags);
            fl = __shfl_sync(0xFFFFFFFFu, fl, 0);
            bool halted = (fl & (EARLY_HALT_FLAG | hrm_rt::ERROR_MASK)) != 0;
            bool should = !halted;
            while (should) {
                bool loaded = false;
                if (lane < FN) {
                    loaded = hrm_rt::ld_relaxed(&_dev_ctx.counts[lane].out_count) >= _dev_ctx.capacity / 2u;
                }
                if (__any_sync(0xFFFFFFFFu, loaded)) break;
                bool more = hrm_rt::call_make_work<PROGRAM_SPEC>(*this);
                should = __any_sync(0xFFFFFFFFu, more);
                n_mw++;
            }
            n_gen++;
            if (!hrm_rt::grid_barrier(ec, ctl)) break;
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                unsigned int f2 = hrm_rt::ld_relaxed(&ctl->flags);
                flip(_dev_ctx, (f2 & (EARLY_HALT_FLAG | hrm_rt::ERROR_MASK)) != 0 || gen + 1 == max_generations);
            }
            if (!hrm_rt::grid_barrier(ec, ctl)) break;
            if (hrm_rt::ld_acquire(&ec->done)) break;
        }

        hrm_rt::call_finalize<PROGRAM_SPEC>(*this);
        if (lane < FN && fn_evals != 0) atomicAdd(&_dev_ctx.stats[hrm_rt::STAT_FN_EVALS + lane], fn_evals);
        if (lane == 0) {
            unsigned long long* st = _dev_ctx.stats;
            atomicAdd(&st[hrm_rt::STAT_EVALS], n_evals);
            atomicAdd(&st[hrm_rt::STAT_BATCHES], n_batches);
            atomicAdd(&st[hrm_rt::STAT_FULL_BATCHES], n_full);
            atomicAdd(&st[hrm_rt::STAT_MAKE_WORK], n_mw);
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&st[hrm_rt::STAT_GENERATIONS], n_gen);
        }
    }

    __device__ static void init_program(DeviceContext ctx) {
        size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (tid < FN) {
            ctx.counts[tid].in_count = 0;
            ctx.counts[tid].out_count = 0;
            ctx.counts[tid].tile_base = 0;
        }
        if (tid == 0) {
            ctx.ctl->flags = 0;
            ctx.ctl->generation = 0;
            ctx.ec->side = 0;
            ctx.ec->total_tiles = 0;
            ctx.ec->tile_next = 0;
            ctx.ec->barrier_count = 0;
            ctx.ec->barrier_gen = 0;
            ctx.ec->done = 0;
        }
        if (tid < hrm_rt::STAT_COUNT) ctx.stats[tid] = 0;
    }

    static unsigned int resident_ctas() {
        static int cached_dev = -1;
        static unsigned int cached = 0;
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev != cached_dev) {
            cached = hrm_rt::max_resident_ctas(hrm_rt::event_exec_kernel<ProgramType>, (int)CTA_THREADS, 0);
            cached_dev = dev;
        }
        return cached;
    }
    static unsigned int ctas_for(size_t group_count) {
        size_t want = (group_count + TEAMS_PER_CTA - 1) / TEAMS_PER_CTA;
        if (want == 0) want = 1;
        unsigned int cap = resident_ctas();
        if (cap == 0) cap = 1;
        return (unsigned int)(want < cap ? want : cap);
    }

    static void launch_init(Instance& inst, size_t, cudaStream_t stream) {
        hrm_rt::event_init_kernel<ProgramType><<<1, 64, 0, stream>>>(inst.to_context());
    }

    // Launches the generation loop cooperatively (all CTAs co-resident) so that the grid
    // barrier is legal. If the cooperative launch is refused, LAUNCH_FLAG is raised.
    static void launch_exec(Instance& inst, size_t group_count, size_t chunk, cudaStream_t stream,
                            unsigned int max_generations = MAX_GENERATIONS_PER_EXEC) {
        unsigned int ctas = ctas_for(group_count);
        DeviceContext ctx = inst.to_context();
        unsigned int blocks = ctas;
        util::host::auto_throw(cudaMemcpyAsync(&ctx.ec->blocks, &blocks, sizeof(unsigned int),
                                               cudaMemcpyHostToDevice, stream));
        util::host::auto_throw(cudaMemsetAsync(&ctx.ec->done, 0, sizeof(unsigned int), stream));
        unsigned int ch = chunk > 0xFFFFu ? 0xFFFFu : (unsigned int)chunk;
        unsigned int mg = max_generations;
        DeviceState ds = inst.device_state;
        void* args[] = {(void*)&ctx, (void*)&ds, (void*)&ch, (void*)&mg};
        cudaError_t err = cudaLaunchCooperativeKernel((const void*)hrm_rt::event_exec_kernel<ProgramType>,
                                                      dim3(ctas), dim3(CTA_THREADS), args, 0, stream);
        if (err != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error(std::string("EventProgram cooperative launch failed: ") + cudaGetErrorString(err));
        }
    }
};

namespace hrm_rt {

template <typename PROG>
__global__ void event_init_kernel(typename PROG::DeviceContext ctx) {
    PROG::init_program(ctx);
}

template <typename PROG>
__global__ void __launch_bounds__(PROG::CTA_THREADS, PROG::MIN_CTAS_PER_SM)
    event_exec_kernel(typename PROG::DeviceContext ctx, typename PROG::DeviceState device, unsigned int chunk,
                      unsigned int max_generations) {
    __shared__ typename PROG::GroupContext grp_ctx[PROG::TEAMS_PER_CTA];
    __shared__ typename PROG::GroupState grp_state[PROG::TEAMS_PER_CTA];
    const unsigned int team = threadIdx.x >> 5;
    typename PROG::ThreadContext thd_ctx;
    typename PROG::ThreadState thd_state;
    PROG prog(ctx, grp_ctx[team], thd_ctx, device, grp_state[team], thd_state);
    prog.exec(chunk, max_generations);
    // Clear a halt request at the end of the exec call, as AsyncProgram does.
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAnd(&ctx.ctl->flags, ~EARLY_HALT_FLAG);
    }
}

}  // namespace hrm_rt

#endif
