// program.h — host entry points init<P>(instance, groups) and exec<P>(instance, groups, n)
// (harmonize/cpp/program/mod.h:73-80), plus stream-taking variants.
//
// init<P> resets the instance's queues and flags (one kernel launch). exec<P> launches the
// program type's persistent kernel with `groups` 32-lane work groups, clamped to what can
// be resident at once (the persistent design needs every team resident); the third
// argument is the cycle budget for AsyncProgram and the per-grab chunk for EventProgram,
// as in the original. Like the original, both are asynchronous with respect to the host.
#ifndef HARMONIZE_B200_PROGRAM_H
#define HARMONIZE_B200_PROGRAM_H

#include "async_program.h"
#include "event_program.h"

template <typename ProgType>
__host__ void init(typename ProgType::Instance& instance, size_t group_count) {
    ProgType::launch_init(instance, group_count, instance.stream);
}

template <typename ProgType>
__host__ void exec(typename ProgType::Instance& instance, size_t group_count, size_t cycle_count) {
    ProgType::launch_exec(instance, group_count, cycle_count, instance.stream);
}

template <typename ProgType>
__host__ void init(typename ProgType::Instance& instance, size_t group_count, cudaStream_t stream) {
    ProgType::launch_init(instance, group_count, stream);
}

template <typename ProgType>
__host__ void exec(typename ProgType::Instance& instance, size_t group_count, size_t cycle_count,
                   cudaStream_t stream) {
    ProgType::launch_exec(instance, group_count, cycle_count, stream);
}

#endif
