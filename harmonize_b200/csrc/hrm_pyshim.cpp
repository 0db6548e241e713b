// hrm_pyshim.cpp — the original Python front end's per-spec host symbol set
// (harmonize/python/templates.py:3-184), for the built-in specs, over the hrm_program_* life
// cycle. Declarations and the contract are in include/hrm_pyshim.h.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hrm_capi.h"
#include "../../include/hrm_pyshim.h"
#include "capi_internal.h"

namespace {

// What alloc_program_S_K returns: the program instance and the device copy of its state, which
// every init / exec reads again (the original passes the state's device address instead).
struct ShimInstance {
    hrm_program* prog = nullptr;
    const void* dev_state = nullptr;
    size_t state_size = 0;
};

bool cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    hrm_capi::set_error(HRM_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

bool reload_state(ShimInstance* in) {
    std::vector<unsigned char> host(in->state_size);
    if (!cuda_ok(cudaMemcpy(host.data(), in->dev_state, in->state_size, cudaMemcpyDeviceToHost), "state read"))
        return false;
    return hrm_program_set_state(in->prog, host.data(), in->state_size) == HRM_OK;
}

void* shim_alloc_state(size_t size) {
    void* p = nullptr;
    if (!cuda_ok(cudaMalloc(&p, size), "alloc_state")) return nullptr;
    if (!cuda_ok(cudaMemset(p, 0, size), "alloc_state")) {
        cudaFree(p);
        return nullptr;
    }
    return p;
}

void shim_free_state(void* p) {
    if (p) cuda_ok(cudaFree(p), "free_state");
}

void* shim_alloc_program(int spec, int type, void* dev_state, size_t state_size, size_t arena_or_io) {
    if (dev_state == nullptr) {
        hrm_capi::set_error(HRM_EINVAL, "alloc_program: device state is NULL");
        return nullptr;
    }
    std::vector<unsigned char> host(state_size);
    if (!cuda_ok(cudaMemcpy(host.data(), dev_state, state_size, cudaMemcpyDeviceToHost), "state read"))
        return nullptr;
    hrm_program* prog = nullptr;
    if (hrm_program_create(spec, type, arena_or_io, host.data(), state_size, &prog) != HRM_OK) return nullptr;
    auto* in = new ShimInstance;
    in->prog = prog;
    in->dev_state = dev_state;
    in->state_size = state_size;
    return in;
}

void shim_free_program(void* p) {
    auto* in = (ShimInstance*)p;
    if (!in) return;
    hrm_program_destroy(in->prog);
    delete in;
}

void shim_init(void* p, size_t grid) {
    auto* in = (ShimInstance*)p;
    if (!in) {
        hrm_capi::set_error(HRM_EINVAL, "init_program: instance is NULL");
        return;
    }
    if (!reload_state(in)) return;
    if (hrm_program_init(in->prog, grid, nullptr) != HRM_OK) return;
    cuda_ok(cudaDeviceSynchronize(), "init_program");
}

void shim_exec(void* p, size_t grid, size_t cycles) {
    auto* in = (ShimInstance*)p;
    if (!in) {
        hrm_capi::set_error(HRM_EINVAL, "exec_program: instance is NULL");
        return;
    }
    if (!reload_state(in)) return;
    if (hrm_program_exec(in->prog, grid, cycles, nullptr) != HRM_OK) return;
    cuda_ok(cudaDeviceSynchronize(), "exec_program");
}

int shim_complete(void* p) {
    auto* in = (ShimInstance*)p;
    if (!in) {
        hrm_capi::set_error(HRM_EINVAL, "complete: instance is NULL");
        return -1;
    }
    int done = 0;
    if (hrm_program_complete(in->prog, &done) != HRM_OK) return -1;
    return done ? 1 : 0;
}

void shim_clear_flags(void* p) {
    auto* in = (ShimInstance*)p;
    if (!in) {
        hrm_capi::set_error(HRM_EINVAL, "clear_flags: instance is NULL");
        return;
    }
    hrm_program_clear_flags(in->prog);
}

void shim_load(void* host, void* dev, size_t off, size_t size) {
    if (!host || !dev) {
        hrm_capi::set_error(HRM_EINVAL, "load_state: NULL pointer");
        return;
    }
    cuda_ok(cudaMemcpy(host, (char*)dev + off, size, cudaMemcpyDeviceToHost), "load_state");
}

void shim_store(void* dev, const void* host, size_t off, size_t size) {
    if (!host || !dev) {
        hrm_capi::set_error(HRM_EINVAL, "store_state: NULL pointer");
        return;
    }
    cuda_ok(cudaMemcpy((char*)dev + off, host, size, cudaMemcpyHostToDevice), "store_state");
}

void shim_store_pointer(void* dev, void* ptr, size_t off, bool is_pointer, const char* field) {
    if (!is_pointer) {
        hrm_capi::set_error(HRM_EINVAL, std::string("store_pointer_state: field '") + field +
                                            "' is not a pointer (attempted to set indirection of a non-array state field)");
        return;
    }
    if (!dev) {
        hrm_capi::set_error(HRM_EINVAL, "store_pointer_state: NULL state");
        return;
    }
    cuda_ok(cudaMemcpy((char*)dev + off, &ptr, sizeof(void*), cudaMemcpyHostToDevice), "store_pointer_state");
}

}  // namespace

#define HRM_SHIM_DEFINE_PROGRAM(S, SPEC_ID, TYPE_ID, STRUCT)                                          \
    void* alloc_state_##S(void) { return shim_alloc_state(sizeof(STRUCT)); }                         \
    void free_state_##S(void* state_ptr) { shim_free_state(state_ptr); }                             \
    void* alloc_program_##S(void* device_arg, size_t size) {                                         \
        return shim_alloc_program(SPEC_ID, TYPE_ID, device_arg, sizeof(STRUCT), size);               \
    }                                                                                                \
    void free_program_##S(void* instance_ptr) { shim_free_program(instance_ptr); }                   \
    void init_program_##S(void* instance_ptr, size_t grid_size) { shim_init(instance_ptr, grid_size); } \
    void exec_program_##S(void* instance_ptr, size_t grid_size, size_t cycle_count) {                \
        shim_exec(instance_ptr, grid_size, cycle_count);                                             \
    }                                                                                                \
    int complete_##S(void* instance_ptr) { return shim_complete(instance_ptr); }                     \
    void clear_flags_##S(void* instance_ptr) { shim_clear_flags(instance_ptr); }                     \
    void set_device_##S(int device) { hrm_set_device(device); }

#define HRM_SHIM_FIELD(STRUCT, S, F, P)                                                              \
    void load_state_##F##_##S(void* host_ptr, void* dev_ptr) {                                       \
        shim_load(host_ptr, dev_ptr, offsetof(STRUCT, F), sizeof(((STRUCT*)nullptr)->F));             \
    }                                                                                                \
    void store_state_##F##_##S(void* dev_ptr, void* host_ptr) {                                      \
        shim_store(dev_ptr, host_ptr, offsetof(STRUCT, F), sizeof(((STRUCT*)nullptr)->F));            \
    }                                                                                                \
    void store_pointer_state_##F##_##S(void* dev_ptr, void* host_ptr) {                              \
        shim_store_pointer(dev_ptr, host_ptr, offsetof(STRUCT, F), P != 0, #F);                      \
    }

#define HRM_SHIM_COLLATZ_FIELD(S, F, P) HRM_SHIM_FIELD(hrm_collatz_state, S, F, P)
#define HRM_SHIM_PHOTON_FIELD(S, F, P) HRM_SHIM_FIELD(hrm_photon_state, S, F, P)
#define HRM_SHIM_BFS_FIELD(S, F, P) HRM_SHIM_FIELD(hrm_bfs_state, S, F, P)

extern "C" {

HRM_SHIM_DEFINE_PROGRAM(collatz_event, HRM_SPEC_COLLATZ, HRM_EVENT, hrm_collatz_state)
HRM_SHIM_DEFINE_PROGRAM(collatz_async, HRM_SPEC_COLLATZ, HRM_ASYNC, hrm_collatz_state)
HRM_SHIM_DEFINE_PROGRAM(photon_event, HRM_SPEC_PHOTON, HRM_EVENT, hrm_photon_state)
HRM_SHIM_DEFINE_PROGRAM(photon_async, HRM_SPEC_PHOTON, HRM_ASYNC, hrm_photon_state)
HRM_SHIM_DEFINE_PROGRAM(bfs_event, HRM_SPEC_BFS, HRM_EVENT, hrm_bfs_state)
HRM_SHIM_DEFINE_PROGRAM(bfs_async, HRM_SPEC_BFS, HRM_ASYNC, hrm_bfs_state)

HRM_SHIM_COLLATZ_FIELDS(HRM_SHIM_COLLATZ_FIELD, collatz_event)
HRM_SHIM_COLLATZ_FIELDS(HRM_SHIM_COLLATZ_FIELD, collatz_async)
HRM_SHIM_PHOTON_FIELDS(HRM_SHIM_PHOTON_FIELD, photon_event)
HRM_SHIM_PHOTON_FIELDS(HRM_SHIM_PHOTON_FIELD, photon_async)
HRM_SHIM_BFS_FIELDS(HRM_SHIM_BFS_FIELD, bfs_event)
HRM_SHIM_BFS_FIELDS(HRM_SHIM_BFS_FIELD, bfs_async)

}  // extern "C"
