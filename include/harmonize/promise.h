// promise.h — operation sets, promises and promise unions.
//
// Source-level names and discriminant rules follow harmonize/cpp/async/promise.h:
//  * OpUnion<Fns...> lists the async functions; a function's discriminant is its 0-based
//    position in the list (OpUnionLookup::DISC, promise.h:65-91);
//  * Promise<Fn> holds the arguments of one call and evaluates it with operator()(prog)
//    (promise.h:439-490);
//  * PromiseUnion<OpSet> overlays every Promise of a set, with cast / rigid_eval /
//    loose_eval / copy_as / dyn_copy_as (promise.h:503-696); PromiseEnum adds the
//    discriminant (promise.h:705-742).
//
// Storage differs from the original on purpose: the argument tuple is laid out flat
// (empty-base optimisation, no trailing 1-byte empty members) and a promise carries no
// return address, because futures are not part of this runtime. A Collatz promise
// (u64, u32, u32) is therefore 16 bytes instead of 32. The runtime moves promises as
// arrays of 32-bit words (`Promise<Fn>::WORDS`).
#ifndef HARMONIZE_B200_PROMISE_H
#define HARMONIZE_B200_PROMISE_H

#include "util.h"

using OpDisc = unsigned int;

template <typename... TYPES>
struct OpUnion {};

template <typename OPERATION>
struct Promise;

template <typename OP_UNION>
union PromiseUnion;

template <typename OP_UNION>
struct PromiseEnum;

struct VoidState {};

template <typename OP_SET, typename ADR_TYPE = unsigned int>
struct RemappingBarrier;

template <typename OP_SET, typename ADR_TYPE = unsigned int>
struct UnitBarrier;

// ---------------------------------------------------------------------------------------
// OpUnion lookup: CONTAINED, DEPTH (= list length) and DISC (= 0-based position).
// ---------------------------------------------------------------------------------------
template <typename QUERY, typename OP_UNION>
struct OpUnionLookup;

template <typename QUERY>
struct OpUnionLookup<QUERY, OpUnion<>> {
    static const bool CONTAINED = false;
    static const OpDisc DEPTH = 0;
    static const OpDisc Q_LEVEL = 0;
    static const OpDisc DISC = 0;
};

template <typename QUERY, typename HEAD, typename... TAIL>
struct OpUnionLookup<QUERY, OpUnion<HEAD, TAIL...>> {
    using Rest = OpUnionLookup<QUERY, OpUnion<TAIL...>>;
    static const bool MATCHES = std::is_same<QUERY, HEAD>::value;
    static const bool CONTAINED = MATCHES || Rest::CONTAINED;
    static const OpDisc DEPTH = Rest::DEPTH + 1;
    static const OpDisc Q_LEVEL = MATCHES ? DEPTH : Rest::Q_LEVEL;
    static const OpDisc DISC = DEPTH - Q_LEVEL;
};

// The operation at a given discriminant.
template <size_t I, typename OP_UNION>
struct OpAt;
template <typename HEAD, typename... TAIL>
struct OpAt<0, OpUnion<HEAD, TAIL...>> {
    using type = HEAD;
};
template <size_t I, typename HEAD, typename... TAIL>
struct OpAt<I, OpUnion<HEAD, TAIL...>> {
    using type = typename OpAt<I - 1, OpUnion<TAIL...>>::type;
};

template <typename OP_UNION>
struct OpCount;
template <typename... T>
struct OpCount<OpUnion<T...>> {
    static const unsigned int value = sizeof...(T);
};

// A tagged semaphore, API only (promise.h:191-200).
struct TaggedSemaphore {
    unsigned int sem;
    unsigned int tag;
    TaggedSemaphore() = default;
    __host__ __device__ TaggedSemaphore(unsigned int s, unsigned int t) : sem(s), tag(t) {}
};

// Marks an argument to be filled by an asynchronous copy from global memory (promise.h:
// 208-240 of the original, its ASYNC_LOADS form). AsyncProgram's async<F> copies such an
// argument with cp.async into the promise's shared-memory slot; everywhere else (sync,
// EventProgram, a promise that overflows to the arena) it converts to its value at the call.
template <typename TYPE>
struct LazyLoad {
    using Type = TYPE;
    Type& reference;
    __host__ __device__ LazyLoad(Type& ref) : reference(ref) {}
    __host__ __device__ operator TYPE() { return reference; }
};

template <typename... TYPES>
__host__ __device__ bool has_load(TYPES...) {
    return false;
}
template <typename HEAD, typename... TAIL>
__host__ __device__ bool has_load(LazyLoad<HEAD>, TAIL...) {
    return true;
}

// ---------------------------------------------------------------------------------------
// Flat argument tuple (element I is TupleGet<I, ArgTuple<...>>::get(t)).
// ---------------------------------------------------------------------------------------
template <typename... TS>
struct ArgTuple;

template <>
struct ArgTuple<> {
    __host__ __device__ ArgTuple() {}
};

template <typename HEAD, typename... TAIL>
struct ArgTuple<HEAD, TAIL...> : ArgTuple<TAIL...> {
    using Tail = ArgTuple<TAIL...>;
    using Head = HEAD;
    HEAD head;

    ArgTuple() = default;
    __host__ __device__ ArgTuple(HEAD h, TAIL... t) : Tail(t...), head(h) {}
};

// Element I of an ArgTuple.
template <size_t I, typename TUPLE>
struct TupleGet;
template <typename HEAD, typename... TAIL>
struct TupleGet<0, ArgTuple<HEAD, TAIL...>> {
    using type = HEAD;
    __host__ __device__ static HEAD& get(ArgTuple<HEAD, TAIL...>& t) { return t.head; }
};
template <size_t I, typename HEAD, typename... TAIL>
struct TupleGet<I, ArgTuple<HEAD, TAIL...>> {
    using Rest = TupleGet<I - 1, ArgTuple<TAIL...>>;
    using type = typename Rest::type;
    __host__ __device__ static type& get(ArgTuple<HEAD, TAIL...>& t) { return Rest::get(t); }
};

template <typename TYPE>
struct OpType;

template <typename RETURN, typename... ARGS>
struct OpType<RETURN (*)(ARGS...)> {
    typedef RETURN Return;
    typedef ArgTuple<ARGS...> Args;
    static const size_t ARITY = sizeof...(ARGS);
};

// ---------------------------------------------------------------------------------------
// Packed argument words: the runtime moves a promise as 32-bit words with its arguments laid
// end to end in call order, each rounded up to whole words and with no alignment padding
// between them (a (uint32, uint64) call is 3 words, not the 4 of its ArgTuple).
// ---------------------------------------------------------------------------------------
template <typename T>
__host__ __device__ constexpr unsigned int words_of() {
    return (unsigned int)((sizeof(T) + 3) / 4);
}

template <typename TUPLE>
struct ArgWords;

template <>
struct ArgWords<ArgTuple<>> {
    static const unsigned int COUNT = 0;
    template <unsigned int O, unsigned int N>
    __host__ __device__ static void put(const ArgTuple<>&, unsigned int (&)[N]) {}
    template <unsigned int O, unsigned int N>
    __host__ __device__ static void get(ArgTuple<>&, const unsigned int (&)[N]) {}
};

template <typename HEAD, typename... TAIL>
struct ArgWords<ArgTuple<HEAD, TAIL...>> {
    using Rest = ArgWords<ArgTuple<TAIL...>>;
    static const unsigned int HEAD_WORDS = words_of<HEAD>();
    static const unsigned int COUNT = HEAD_WORDS + Rest::COUNT;
    // Writes the arguments to words [O, O + COUNT) of w.
    template <unsigned int O, unsigned int N>
    __host__ __device__ static void put(const ArgTuple<HEAD, TAIL...>& t, unsigned int (&w)[N]) {
        unsigned int tmp[HEAD_WORDS];
        tmp[HEAD_WORDS - 1] = 0u;
        memcpy(tmp, &t.head, sizeof(HEAD));
#pragma unroll
        for (unsigned int i = 0; i < HEAD_WORDS; i++) w[O + i] = tmp[i];
        Rest::template put<O + HEAD_WORDS>(t, w);
    }
    // Reads the arguments back from words [O, O + COUNT) of w.
    template <unsigned int O, unsigned int N>
    __host__ __device__ static void get(ArgTuple<HEAD, TAIL...>& t, const unsigned int (&w)[N]) {
        unsigned int tmp[HEAD_WORDS];
#pragma unroll
        for (unsigned int i = 0; i < HEAD_WORDS; i++) tmp[i] = w[O + i];
        memcpy(&t.head, tmp, sizeof(HEAD));
        Rest::template get<O + HEAD_WORDS>(t, w);
    }
};

// First word of argument I in the packed words.
template <size_t I, typename TUPLE>
struct ArgWordOffset;
template <typename HEAD, typename... TAIL>
struct ArgWordOffset<0, ArgTuple<HEAD, TAIL...>> {
    static const unsigned int value = 0;
};
template <size_t I, typename HEAD, typename... TAIL>
struct ArgWordOffset<I, ArgTuple<HEAD, TAIL...>> {
    static const unsigned int value = words_of<HEAD>() + ArgWordOffset<I - 1, ArgTuple<TAIL...>>::value;
};

// ---------------------------------------------------------------------------------------
// Promise<Op>: the arguments of one call to Op.
// ---------------------------------------------------------------------------------------
template <typename OPERATION>
struct Promise {
    typedef typename OpType<typename OPERATION::Type>::Return Return;
    typedef typename OpType<typename OPERATION::Type>::Args Args;
    static const size_t ARITY = OpType<typename OPERATION::Type>::ARITY;

    Args args;

    // Number of 32-bit words the runtime moves for this promise (packed, see ArgWords; at
    // least one).
    static const unsigned int WORDS = ArgWords<Args>::COUNT ? ArgWords<Args>::COUNT : 1u;

    Promise() = default;
    template <typename... ARGS>
    __host__ __device__ Promise(ARGS... a) : args(a...) {}

    template <typename PROGRAM, size_t... IS>
    __device__ __forceinline__ Return call(PROGRAM program, std::index_sequence<IS...>) {
        return OPERATION::template eval<PROGRAM>(program, TupleGet<IS, Args>::get(args)...);
    }

    template <typename PROGRAM>
    __device__ __forceinline__ Return operator()(PROGRAM program) {
        return call(program, std::make_index_sequence<ARITY>{});
    }

    // Word-level access used by the runtime's queues.
    __device__ __forceinline__ void to_words(unsigned int (&w)[WORDS]) const {
        w[WORDS - 1] = 0u;
        ArgWords<Args>::template put<0>(args, w);
    }
    __device__ __forceinline__ void from_words(const unsigned int (&w)[WORDS]) {
        ArgWords<Args>::template get<0>(args, w);
    }
};

// ---------------------------------------------------------------------------------------
// PromiseUnion: one storage slot able to hold any promise of an operation set.
// ---------------------------------------------------------------------------------------
template <>
union PromiseUnion<OpUnion<>> {
    struct Info {
        static const OpDisc COUNT = 0;
    };
    template <typename PROGRAM, typename TYPE>
    __host__ __device__ void rigid_eval(PROGRAM) {}
    template <typename PROGRAM>
    __host__ __device__ void loose_eval(PROGRAM, OpDisc) {}
    __host__ __device__ void dyn_copy_as(OpDisc, PromiseUnion<OpUnion<>>&) {}
    PromiseUnion() = default;
};

template <typename HEAD, typename... TAIL>
union PromiseUnion<OpUnion<HEAD, TAIL...>> {
    using Head = Promise<HEAD>;
    using Tail = PromiseUnion<OpUnion<TAIL...>>;
    using OpSet = OpUnion<HEAD, TAIL...>;
    using TailOpSet = OpUnion<TAIL...>;

    Head head_form;
    Tail tail_form;

    struct Info {
        static const OpDisc COUNT = sizeof...(TAIL) + 1;
        static const OpDisc INDEX = 0;
    };

    template <typename TYPE>
    struct Lookup {
        typedef OpUnionLookup<TYPE, OpSet> type;
    };

    template <typename TYPE>
    __host__ __device__ typename std::enable_if<std::is_same<TYPE, HEAD>::value, Promise<TYPE>&>::type cast() {
        return head_form;
    }
    template <typename TYPE>
    __host__ __device__ typename std::enable_if<!std::is_same<TYPE, HEAD>::value, Promise<TYPE>&>::type cast() {
        static_assert(OpUnionLookup<TYPE, TailOpSet>::CONTAINED,
                      "\n\nTYPE ERROR: Promise type does not exist in union.\n\n");
        return tail_form.template cast<TYPE>();
    }

    template <typename PROGRAM, typename TYPE>
    __device__ typename std::enable_if<std::is_same<TYPE, HEAD>::value>::type rigid_eval(PROGRAM program) {
        head_form(program);
    }
    template <typename PROGRAM, typename TYPE>
    __device__ typename std::enable_if<!std::is_same<TYPE, HEAD>::value>::type rigid_eval(PROGRAM program) {
        static_assert(OpUnionLookup<TYPE, TailOpSet>::CONTAINED,
                      "\n\nTYPE ERROR: Promise type does not exist in union.\n\n");
        tail_form.template rigid_eval<PROGRAM, TYPE>(program);
    }

    // Evaluates the member selected by a runtime discriminant.
    template <typename PROGRAM>
    __device__ void loose_eval(PROGRAM program, OpDisc disc) {
        if (disc == 0) {
            head_form(program);
        } else {
            tail_form.template loose_eval<PROGRAM>(program, disc - 1);
        }
    }

    template <typename TYPE>
    __host__ __device__ void copy_as(PromiseUnion<OpSet>& other) {
        cast<TYPE>() = other.template cast<TYPE>();
    }
    __host__ __device__ void dyn_copy_as(OpDisc disc, PromiseUnion<OpSet>& other) {
        if (disc == 0) {
            head_form = other.head_form;
        } else {
            tail_form.dyn_copy_as(disc - 1, other.tail_form);
        }
    }

    __host__ __device__ PromiseUnion() : tail_form() {}

    template <typename OP_TYPE>
    __host__ __device__ PromiseUnion(Promise<OP_TYPE> prom) {
        static_assert(OpUnionLookup<OP_TYPE, OpSet>::CONTAINED,
                      "\n\nTYPE ERROR: Type of assigned promise does not exist in promise union.\n\n");
        cast<OP_TYPE>() = prom;
    }
};

template <typename OP_SET>
struct PromiseEnum {
    using UnionType = PromiseUnion<OP_SET>;
    UnionType data;
    OpDisc disc;

    PromiseEnum() = default;
    __host__ __device__ PromiseEnum(UnionType u, OpDisc d) : data(u), disc(d) {}
    template <typename OP_TYPE>
    __host__ __device__ PromiseEnum(Promise<OP_TYPE> p)
        : data(p), disc(UnionType::template Lookup<OP_TYPE>::type::DISC) {}
};

// ---------------------------------------------------------------------------------------
// Compile-time layout of an operation set in 32-bit words (used by both program types).
// ---------------------------------------------------------------------------------------
template <typename OP_SET>
struct OpLayout;

template <>
struct OpLayout<OpUnion<>> {
    static const unsigned int TOTAL_WORDS = 0;
    static const unsigned int MAX_WORDS = 0;
};

template <typename HEAD, typename... TAIL>
struct OpLayout<OpUnion<HEAD, TAIL...>> {
    using Rest = OpLayout<OpUnion<TAIL...>>;
    static const unsigned int HEAD_WORDS = Promise<HEAD>::WORDS;
    static const unsigned int TOTAL_WORDS = HEAD_WORDS + Rest::TOTAL_WORDS;
    static const unsigned int MAX_WORDS = HEAD_WORDS > Rest::MAX_WORDS ? HEAD_WORDS : Rest::MAX_WORDS;
};

// Word offset of operation I inside a per-set word array.
template <size_t I, typename OP_SET>
struct OpWordOffset;
template <typename HEAD, typename... TAIL>
struct OpWordOffset<0, OpUnion<HEAD, TAIL...>> {
    static const unsigned int value = 0;
};
template <size_t I, typename HEAD, typename... TAIL>
struct OpWordOffset<I, OpUnion<HEAD, TAIL...>> {
    static const unsigned int value = Promise<HEAD>::WORDS + OpWordOffset<I - 1, OpUnion<TAIL...>>::value;
};

#endif
