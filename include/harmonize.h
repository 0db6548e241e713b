// harmonize.h — single include point of the B200-native Harmonize runtime
// (the counterpart of harmonize/cpp/harmonize.h:1-4).
//
// A program specification written for Harmonize compiles against this header unchanged:
//
//     nvcc -std=c++17 -x cu -gencode arch=compute_100a,code=sm_100a \
//          -I<repo>/include -include harmonize.h my_spec.cpp
//
// It provides OpUnion / Promise / PromiseUnion, AsyncProgram<Spec> and EventProgram<Spec>
// (one-line swappable), init<P> / exec<P>, RemappingBarrier / UnitBarrier, and the
// util:: and adapt:: namespaces.
#ifndef HARMONIZE_B200_H
#define HARMONIZE_B200_H

#include "harmonize/program.h"
#include "harmonize/barrier.h"

#endif
