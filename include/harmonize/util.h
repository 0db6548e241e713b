// util.h — the `util::` namespace of the Harmonize source-level API.
//
// Same names and meanings as the original (harmonize/cpp/util/mod.h:16-134,
// util/host.h:10-279, util/iter.h:13-474, util/mem.h:29-178, util/cli.h:13-498), rewritten:
//  * warp helpers use the lane index (%laneid), not threadIdx.x, so they stay correct when
//    a CTA holds several 32-lane teams;
//  * AtomicIter::leap aggregates the lanes of a warp that leap the same iterator into one
//    atomicAdd (__match_any_sync + popc rank), instead of one atomic per lane;
//  * host buffers keep the RAII/shared_ptr ownership and the `<<` / `>>` copy operators.
#ifndef HARMONIZE_B200_UTIL_H
#define HARMONIZE_B200_UTIL_H

#include "preamble.h"

namespace util {

// ---------------------------------------------------------------------------------------
// Warp helpers (harmonize/cpp/util/mod.h:16-57)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned int lane_id() {
    unsigned int l;
    asm volatile("mov.u32 %0, %%laneid;" : "=r"(l));
    return l;
}
__device__ __forceinline__ unsigned int lanemask_lt() {
    unsigned int m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Number of active lanes below this one: this lane's index among the active lanes.
static __device__ __forceinline__ unsigned int warp_inc_scan() {
    return __popc(__activemask() & lanemask_lt());
}
// Number of active lanes.
static __device__ __forceinline__ unsigned int active_count() { return __popc(__activemask()); }
// True only for the lowest active lane.
static __device__ __forceinline__ bool current_leader() {
    return (unsigned int)(__ffs(__activemask()) - 1) == lane_id();
}
static __device__ __forceinline__ unsigned int pop_count(unsigned int v) { return __popc(v); }
static __device__ __forceinline__ unsigned long long int pop_count(unsigned long long int v) {
    return __popcll(v);
}
static __device__ __forceinline__ unsigned int leading_zeros(unsigned int v) { return __clz(v); }
static __device__ __forceinline__ unsigned long long int leading_zeros(unsigned long long int v) {
    return __clzll(v);
}

// Linear congruential generators with the exact multipliers and increments of the
// original (util/mod.h:66-77); specs such as the neutron example depend on the sequence.
static __host__ __device__ __forceinline__ unsigned int random_uint(unsigned int& state) {
    state = 0x10DCDu * state + 1u;
    return state;
}
static __host__ __device__ __forceinline__ unsigned long long int random_uint(
    unsigned long long int& state) {
    state = 2971215073ull * state + 12345ull;
    return state;
}

// CUDA-event stopwatch on the default stream (util/mod.h:88-134).
struct Stopwatch {
    cudaEvent_t beg;
    cudaEvent_t end;
    float duration = 0.0f;

    Stopwatch() {
        if (cudaEventCreate(&beg) != cudaSuccess || cudaEventCreate(&end) != cudaSuccess) {
            printf("Failed to create one or more Stopwatch events\n");
            std::exit(1);
        }
    }
    ~Stopwatch() {
        cudaEventDestroy(beg);
        cudaEventDestroy(end);
    }
    Stopwatch(const Stopwatch&) = delete;
    Stopwatch& operator=(const Stopwatch&) = delete;

    bool start() { return cudaEventRecord(beg, nullptr) == cudaSuccess; }
    bool stop() {
        if (cudaEventRecord(end, nullptr) != cudaSuccess) return false;
        cudaEventSynchronize(end);
        cudaEventElapsedTime(&duration, beg, end);
        return true;
    }
    float ms_duration() { return duration; }
};

// ---------------------------------------------------------------------------------------
// Host-side device buffers (harmonize/cpp/util/host.h)
// ---------------------------------------------------------------------------------------
namespace host {

static inline bool check_error() {
    cudaError_t status = cudaGetLastError();
    if (status != cudaSuccess) {
        printf("ERROR: \"%s\"\n", cudaGetErrorString(status));
    }
    return status != cudaSuccess;
}

static inline void auto_throw(cudaError_t status) {
    if (status != cudaSuccess) {
        std::string message = "GPU Runtime Error: ";
        message += cudaGetErrorString(status);
        throw std::runtime_error(message);
    }
}

template <typename T>
T* hardMalloc(size_t size) {
    T* result = nullptr;
    if (size == 0) return nullptr;
    auto_throw(cudaMalloc((void**)&result, sizeof(T) * size));
    return result;
}

// A shared, reference-counted device array. Copies share the allocation; the last owner
// frees it. Converts implicitly to the raw device pointer.
template <typename T>
class DevBuf {
   protected:
    struct Inner {
        T* adr;
        size_t size;
        Inner(T* a, size_t s) : adr(a), size(s) {}
        ~Inner() {
            if (adr != nullptr) cudaFree(adr);
        }
    };
    std::shared_ptr<Inner> inner;

   public:
    operator T*&() { return inner->adr; }
    T* data() const { return inner->adr; }
    size_t size() const { return inner->size; }

    void resize(size_t s) {
        T* fresh = hardMalloc<T>(s);
        size_t keep = s < inner->size ? s : inner->size;
        if (keep != 0) {
            auto_throw(cudaMemcpy(fresh, inner->adr, sizeof(T) * keep, cudaMemcpyDeviceToDevice));
        }
        if (inner->adr != nullptr) auto_throw(cudaFree(inner->adr));
        inner->adr = fresh;
        inner->size = s;
    }

    void operator<<(std::vector<T>& other) {
        if (other.size() != inner->size) resize(other.size());
        if (inner->size != 0) {
            auto_throw(cudaMemcpy(inner->adr, other.data(), sizeof(T) * inner->size,
                                  cudaMemcpyHostToDevice));
        }
    }
    void operator>>(std::vector<T>& other) {
        if (other.size() != inner->size) other.resize(inner->size);
        if (inner->size != 0) {
            auto_throw(cudaMemcpy(other.data(), inner->adr, sizeof(T) * inner->size,
                                  cudaMemcpyDeviceToHost));
        }
    }
    void operator<<(T& other) {
        if (inner->size != 1) resize(1);
        auto_throw(cudaMemcpy(inner->adr, &other, sizeof(T), cudaMemcpyHostToDevice));
    }
    void operator<<(T&& other) {
        T copy = other;
        (*this) << copy;
    }
    void operator>>(T& other) {
        auto_throw(cudaMemcpy(&other, inner->adr, sizeof(T), cudaMemcpyDeviceToHost));
    }

    DevBuf(T* adr, size_t size) : inner(new Inner(adr, size)) {}
    DevBuf() : DevBuf((T*)nullptr, (size_t)0) {}
    DevBuf(size_t size) : DevBuf(hardMalloc<T>(size), size) {}
    DevBuf(T& value) : DevBuf() { (*this) << value; }
    DevBuf(T&& value) : DevBuf() { (*this) << value; }

    template <typename... ARGS>
    static DevBuf<T> make(ARGS... args) {
        return DevBuf<T>(T(args...));
    }
};

// A single device object with a host mirror. T provides host_init()/host_free(), called
// when the object is created and destroyed (util/host.h:201-279).
template <typename T>
class DevObj {
   protected:
    struct Inner {
        T* adr;
        T host_copy;
        void push_data() { auto_throw(cudaMemcpy(adr, &host_copy, sizeof(T), cudaMemcpyHostToDevice)); }
        void pull_data() { auto_throw(cudaMemcpy(&host_copy, adr, sizeof(T), cudaMemcpyDefault)); }
        template <typename... ARGS>
        Inner(T* a, ARGS... args) : adr(a), host_copy(args...) {
            host_copy.host_init();
            push_data();
        }
        ~Inner() {
            if (adr != nullptr) {
                cudaMemcpy(&host_copy, adr, sizeof(T), cudaMemcpyDefault);
                host_copy.host_free();
                cudaFree(adr);
            }
        }
    };
    std::shared_ptr<Inner> inner;

   public:
    void push_data() { inner->push_data(); }
    void pull_data() { inner->pull_data(); }
    operator T*() { return inner->adr; }
    operator T() { return inner->host_copy; }
    T& host_copy() { return inner->host_copy; }
    DevObj() = default;
    template <typename... ARGS>
    DevObj(ARGS... args) : inner(new Inner(hardMalloc<T>(1), args...)) {}
};

}  // namespace host

// ---------------------------------------------------------------------------------------
// Address and packed-pair helpers (harmonize/cpp/util/mem.h:29-178), API only.
// ---------------------------------------------------------------------------------------
namespace mem {

template <typename ADR_TYPE>
struct Adr {
    typedef ADR_TYPE AdrType;
    static const AdrType null = std::numeric_limits<AdrType>::max();
    AdrType adr;
    Adr() = default;
    __host__ __device__ Adr(AdrType a) : adr(a) {}
    __host__ __device__ bool is_null() const { return adr == null; }
    __host__ __device__ bool operator==(const Adr<AdrType>& o) const { return adr == o.adr; }
    __host__ __device__ bool operator!=(const Adr<AdrType>& o) const { return adr != o.adr; }
    __host__ __device__ operator AdrType() const { return adr; }
};

// Two 32-bit halves in one 64-bit word so that both can be swapped by one atomic.
template <typename T>
struct PairPack {
    typedef unsigned long long PairType;
    static const PairType RIGHT_MASK = 0xFFFFFFFFull;
    static const size_t RIGHT_WIDTH = 32;
    PairType data;
    PairPack() = default;
    __host__ __device__ PairPack(T left, T right)
        : data(((PairType)left << RIGHT_WIDTH) | ((PairType)right & RIGHT_MASK)) {}
    __host__ __device__ T get_left() const { return (T)(data >> RIGHT_WIDTH); }
    __host__ __device__ T get_right() const { return (T)(data & RIGHT_MASK); }
    __host__ __device__ void set_left(T v) { data = PairPack<T>(v, get_right()).data; }
    __host__ __device__ void set_right(T v) { data = PairPack<T>(get_left(), v).data; }
};

}  // namespace mem

// ---------------------------------------------------------------------------------------
// Iterators (harmonize/cpp/util/iter.h:13-474)
// ---------------------------------------------------------------------------------------
namespace iter {

template <typename INDEX_TYPE>
struct Iter {
    typedef INDEX_TYPE IndexType;
    IndexType value;
    IndexType limit;

    Iter() = default;
    __host__ __device__ Iter(IndexType v, IndexType l) : value(v), limit(l) {}

    __device__ void reset(IndexType start_val, IndexType limit_val) {
        value = start_val;
        limit = limit_val;
    }
    __host__ __device__ bool step(IndexType& out) {
        if (value >= limit) return false;
        out = value;
        value += 1;
        return true;
    }
    __host__ __device__ Iter<IndexType> leap(IndexType length) {
        IndexType sub = value + length;
        sub = (sub > limit) ? limit : sub;
        Iter<IndexType> r(value, sub);
        value = sub;
        return r;
    }
    __host__ __device__ bool done() const { return value >= limit; }
};

// A shared iterator in device memory handing out disjoint index ranges to all threads.
template <typename INDEX_TYPE>
struct AtomicIter {
    typedef INDEX_TYPE IndexType;
    IndexType value;
    IndexType limit;

    AtomicIter() = default;
    __host__ __device__ AtomicIter(IndexType start_val, IndexType limit_val)
        : value(start_val), limit(limit_val) {}
    __host__ __device__ AtomicIter(Iter<IndexType> it) : value(it.value), limit(it.limit) {}
    __host__ __device__ AtomicIter<IndexType>& operator=(Iter<IndexType> it) {
        value = it.value;
        limit = it.limit;
        return *this;
    }

    __device__ void reset(IndexType start_val, IndexType limit_val) {
        __threadfence();
        atomicExch(&limit, limit_val);
        atomicExch(&value, start_val);
        __threadfence();
    }

    // Claims up to `leap_size` consecutive indices. The lanes of a warp that leap the same
    // iterator with the same size at the same time share one atomicAdd; each lane receives
    // the same range it would have received from its own atomic, in lane order.
    __device__ Iter<IndexType> leap(IndexType leap_size) {
        IndexType cur = *(volatile IndexType*)&value;
        IndexType lim = *(volatile IndexType*)&limit;
        if (cur >= lim) return Iter<IndexType>(lim, lim);
        unsigned int active = __activemask();
        unsigned int same = __match_any_sync(active, (unsigned long long)(uintptr_t)this);
        unsigned int same_size = __match_any_sync(same, (unsigned long long)leap_size);
        unsigned int group = same & same_size;
        unsigned int rank = __popc(group & lanemask_lt());
        unsigned int n = __popc(group);
        unsigned int leader = __ffs(group) - 1;
        IndexType base = 0;
        if (rank == 0) base = atomicAdd(&value, (IndexType)(leap_size * n));
        base = __shfl_sync(group, base, leader);
        IndexType start = base + (IndexType)(leap_size * rank);
        IndexType end = start + leap_size;
        start = (start < lim) ? start : lim;
        end = (end < lim) ? end : lim;
        return Iter<IndexType>(start, end);
    }

    __device__ bool step(IndexType& out) {
        Iter<IndexType> it = leap(1);
        return it.step(out);
    }

    __device__ bool done() const {
        IndexType cur = *(volatile const IndexType*)&value;
        IndexType lim = *(volatile const IndexType*)&limit;
        return cur >= lim;
    }
};

// Per-group iterator, API only (iter.h:64-133); advances in steps of blockDim.x.
template <typename INDEX_TYPE>
struct GroupIter {
    typedef INDEX_TYPE IndexType;
    IndexType value;
    IndexType limit;
    GroupIter() = default;
    __host__ __device__ GroupIter(Iter<IndexType> it) : value(it.value), limit(it.limit) {}
    __host__ __device__ bool done() const { return value >= limit; }
};

template <typename T, template <typename> class ITER_TYPE = Iter, typename INDEX_TYPE = unsigned int>
struct ArrayIter {
    typedef INDEX_TYPE IndexType;
    typedef ITER_TYPE<IndexType> IterType;
    T* array;
    IterType iter;

    ArrayIter() = default;
    __host__ __device__ ArrayIter(T* adr, IterType it) : array(adr), iter(it) {}
    template <template <typename> class OTHER>
    __host__ __device__ ArrayIter(ArrayIter<T, OTHER, INDEX_TYPE>&& o) : array(o.array), iter(o.iter) {}
    template <template <typename> class OTHER>
    __host__ __device__ ArrayIter& operator=(ArrayIter<T, OTHER, INDEX_TYPE>&& o) {
        array = o.array;
        iter = o.iter;
        return *this;
    }
    __device__ void reset(T* a, IterType it) {
        array = a;
        iter = it;
    }
    __device__ bool step_val(T& val) {
        IndexType i;
        if (iter.step(i)) { val = array[i]; return true; }
        return false;
    }
    __device__ bool step_idx_val(IndexType& idx, T& val) {
        IndexType i;
        if (iter.step(i)) { idx = i; val = array[i]; return true; }
        return false;
    }
    __device__ bool step_ptr(T*& val) {
        IndexType i;
        if (iter.step(i)) { val = &array[i]; return true; }
        return false;
    }
    __device__ bool step_idx_ptr(IndexType& idx, T*& val) {
        IndexType i;
        if (iter.step(i)) { idx = i; val = &array[i]; return true; }
        return false;
    }
    __device__ ArrayIter<T, Iter, IndexType> leap(IndexType n) {
        return ArrayIter<T, Iter, IndexType>(array, iter.leap(n));
    }
    __device__ bool done() { return iter.done(); }
};

// Double-buffered input/output array (iter.h:320-474). Kept for specs and host code that
// name it; the EventProgram of this runtime uses its own structure-of-arrays buffers.
template <typename T, typename INDEX_TYPE = unsigned int>
struct IOBuffer {
    typedef INDEX_TYPE IndexType;
    bool toggle;
    T* data_a;
    T* data_b;
    IndexType capacity;
    AtomicIter<IndexType> input_iter;
    AtomicIter<IndexType> output_iter;

    __host__ __device__ IOBuffer()
        : toggle(false), data_a(nullptr), data_b(nullptr), capacity(0), input_iter(0, 0), output_iter(0, 0) {}
    __host__ IOBuffer(IndexType cap)
        : toggle(false), data_a(nullptr), data_b(nullptr), capacity(cap), input_iter(0, 0), output_iter(0, cap) {}
    __host__ void host_init() {
        data_a = host::hardMalloc<T>(capacity);
        data_b = host::hardMalloc<T>(capacity);
    }
    __host__ void host_free() {
        if (data_a) host::auto_throw(cudaFree(data_a));
        if (data_b) host::auto_throw(cudaFree(data_b));
    }
    __host__ __device__ T* input_pointer() { return toggle ? data_b : data_a; }
    __host__ __device__ T* output_pointer() { return toggle ? data_a : data_b; }
    __device__ ArrayIter<T, Iter, IndexType> pull_span(IndexType n) {
        return ArrayIter<T, Iter, IndexType>(input_pointer(), input_iter.leap(n));
    }
    __device__ ArrayIter<T, Iter, IndexType> push_span(IndexType n) {
        return ArrayIter<T, Iter, IndexType>(output_pointer(), output_iter.leap(n));
    }
    __device__ bool pull(T& v) {
        IndexType i;
        if (!input_iter.step(i)) return false;
        v = input_pointer()[i];
        return true;
    }
    __device__ bool pull_index(IndexType& i) { return input_iter.step(i); }
    __device__ bool push(T v) {
        IndexType i;
        if (!output_iter.step(i)) return false;
        output_pointer()[i] = v;
        return true;
    }
    __device__ bool push_index(IndexType& i) { return output_iter.step(i); }
    __device__ void flip() {
        IndexType in_count = output_iter.value >= capacity ? capacity : output_iter.value;
        toggle = !toggle;
        input_iter.reset(0, in_count);
        output_iter.reset(0, capacity);
    }
    __device__ bool input_empty() { return input_iter.done(); }
    __device__ bool output_full() { return output_iter.done(); }
    __device__ float output_fill_fraction() {
        return ((float)atomicAdd(&output_iter.value, 0u)) / ((float)capacity);
    }
};

}  // namespace iter

// ---------------------------------------------------------------------------------------
// Command-line flags (harmonize/cpp/util/cli.h:314-498): `args["flag"] | default`.
// ---------------------------------------------------------------------------------------
namespace cli {

struct ArgSet {
    int argc;
    char const** argv;

    ArgSet(int c, char const** v) : argc(c), argv(v) {}
    ArgSet(int c, char** v) : argc(c), argv((char const**)v) {}

    char const* get_flag_str(char const* flag) const {
        for (int i = 0; i < argc; i++) {
            char const* s = argv[i];
            if (s != nullptr && s[0] == '-' && strcmp(s + 1, flag) == 0) {
                return (i == argc - 1) ? "" : argv[i + 1];
            }
        }
        return nullptr;
    }

    template <typename T>
    struct ArgVal {
        T value;
        ArgVal(T v) : value(v) {}
        ArgVal<T> operator|(T) { return *this; }
        operator T() const { return value; }
    };

    struct ArgQuery {
        char const* flag_str;
        char const* value_str;
        ArgQuery(char const* f, char const* v) : flag_str(f), value_str(v) {}

        static bool parse(char const* s, bool& d) {
            if (strcmp(s, "false") == 0) { d = false; return true; }
            if (strcmp(s, "true") == 0) { d = true; return true; }
            return false;
        }
        static bool parse(char const* s, float& d) { return sscanf(s, "%f", &d) > 0; }
        static bool parse(char const* s, double& d) { return sscanf(s, "%lf", &d) > 0; }
        template <typename T>
        static bool parse(char const* s, T& d) {
            static_assert(std::is_integral<T>::value, "unsupported flag type");
            char* endp = nullptr;
            if (std::is_signed<T>::value) {
                long long v = strtoll(s, &endp, 0);
                d = (T)v;
            } else {
                unsigned long long v = strtoull(s, &endp, 0);
                d = (T)v;
            }
            return endp != s;
        }

        template <typename T>
        void scan_or_fail(T& dest) const {
            if (value_str == nullptr) {
                printf("No value provided for flag '-%s'\n", flag_str);
                std::exit(1);
            }
            if (!parse(value_str, dest)) {
                printf("Value string '%s' provided for flag '-%s' could not be parsed\n", value_str, flag_str);
                std::exit(1);
            }
        }
        void scan_or_fail(bool& dest) const { dest = (value_str != nullptr); }

        template <typename T>
        ArgVal<T> operator|(T other) {
            if (value_str == nullptr) return ArgVal<T>(other);
            T v;
            scan_or_fail(v);
            return ArgVal<T>(v);
        }
        ArgQuery operator|(ArgQuery other) { return value_str == nullptr ? other : *this; }
        template <typename T>
        operator T() const {
            T v;
            scan_or_fail(v);
            return v;
        }
    };

    ArgQuery operator[](char const* flag) const { return ArgQuery(flag, get_flag_str(flag)); }
};

// Terminal plotting, API only (cli.h:13-307): prints a plain column chart.
struct GraphStyle {
    int cols, rows;
    const char* const* tiles;
    GraphStyle(int c, int r, const char* const* t) : cols(c), rows(r), tiles(t) {}
};
struct GraphShape {
    float y_min = 0, y_max = 1, x_min = 0, x_max = 1;
    int width = 50, height = 16;
};
static const char* const Block2x2FillTiles[] = {" ", "#"};
static const GraphStyle Block2x2Fill = GraphStyle(1, 1, Block2x2FillTiles);

static inline void cli_graph(float* data, int size, GraphShape shape, GraphStyle) {
    if (size <= 0 || shape.width <= 0 || shape.height <= 0) return;
    float span = shape.y_max - shape.y_min;
    for (int row = shape.height - 1; row >= 0; row--) {
        for (int c = 0; c < shape.width; c++) {
            int i = (int)((long long)c * size / shape.width);
            float v = span > 0 ? (data[i] - shape.y_min) / span : 0.0f;
            putchar(v * shape.height > row ? '#' : ' ');
        }
        putchar('\n');
    }
}

}  // namespace cli

}  // namespace util

#endif
