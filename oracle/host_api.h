// host_api.h — the minimal Harmonize names a spec source needs, for the CPU host executors
// (TEST INFRASTRUCTURE ONLY). Specs compiled with g++ see OpUnion, util::iter::Iter and
// util::iter::AtomicIter with the semantics of harmonize/cpp/util/iter.h:13-223 and
// harmonize/cpp/async/promise.h:16-17, implemented with host atomics.
#ifndef HRM_ORACLE_HOST_API_H
#define HRM_ORACLE_HOST_API_H

#include <cstddef>
#include <cstdint>

template <typename... TYPES>
struct OpUnion {};

namespace util {
namespace iter {

template <typename INDEX_TYPE>
struct Iter {
    typedef INDEX_TYPE IndexType;
    IndexType value;
    IndexType limit;
    Iter() = default;
    Iter(IndexType v, IndexType l) : value(v), limit(l) {}
    bool step(IndexType& out) {
        if (value >= limit) return false;
        out = value;
        value += 1;
        return true;
    }
    Iter leap(IndexType length) {
        IndexType sub = value + length;
        sub = sub > limit ? limit : sub;
        Iter r(value, sub);
        value = sub;
        return r;
    }
    bool done() const { return value >= limit; }
};

template <typename INDEX_TYPE>
struct AtomicIter {
    typedef INDEX_TYPE IndexType;
    IndexType value;
    IndexType limit;
    AtomicIter() = default;
    AtomicIter(IndexType s, IndexType l) : value(s), limit(l) {}
    Iter<IndexType> leap(IndexType n) {
        IndexType cur = __atomic_load_n(&value, __ATOMIC_RELAXED);
        if (cur >= limit) return Iter<IndexType>(limit, limit);
        IndexType s = __atomic_fetch_add(&value, n, __ATOMIC_RELAXED);
        IndexType e = s + n;
        s = s < limit ? s : limit;
        e = e < limit ? e : limit;
        return Iter<IndexType>(s, e);
    }
    bool step(IndexType& out) {
        Iter<IndexType> it = leap(1);
        return it.step(out);
    }
    bool done() const { return __atomic_load_n(&value, __ATOMIC_RELAXED) >= limit; }
};

}  // namespace iter
}  // namespace util

#endif
