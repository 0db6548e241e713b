/* hrm_pyshim.h — the per-spec host symbol set of the original Python front end, exported by
 * libhrm.so for the built-in specs.
 *
 * The original generates, for each spec S and program kind K (S_K = "<spec>_<event|async>"),
 * a set of extern "C" host wrappers from the string templates of
 * harmonize/python/templates.py:3-184 and binds them by name with numba ExternalFunction
 * handles in harmonize/python/runtime.py:1324-1408. This header declares the same names and
 * signatures for the built-in specs collatz, photon and bfs, layered on the hrm_program_* life
 * cycle of hrm_capi.h, so that a binding written against those names can drive this runtime:
 *
 *   void* alloc_state_S_K(void)                      templates.py:73-83    device copy of the state
 *   void  free_state_S_K(void* state)                templates.py:154-159
 *   void  load_state_<field>_S_K(void* host, void* dev)          :85-104   device -> host, one field
 *   void  store_state_<field>_S_K(void* dev, void* host)         :106-125  host -> device, one field
 *   void  store_pointer_state_<field>_S_K(void* dev, void* ptr)  :128-152  store a pointer field
 *   void* alloc_program_S_K(void* dev_state, size_t arena_or_io) :43-63
 *   void  free_program_S_K(void* instance)           :65-71
 *   void  init_program_S_K(void* instance, size_t grid_size)     :3-14
 *   void  exec_program_S_K(void* instance, size_t grid_size, size_t cycles_or_chunk) :17-40
 *   int   complete_S_K(void* instance)               :161-168
 *   void  clear_flags_S_K(void* instance)            :170-177
 *   void  set_device_S_K(int device)                 :179-184
 *
 * Fields are the members of hrm_collatz_state, hrm_photon_state and hrm_bfs_state
 * (hrm_capi.h). As in the original, the program reads its state from the device copy made by
 * alloc_state_S_K: each init and exec takes the state as it is on the device at that moment,
 * and every wrapper returns after the device has finished (cudaDeviceSynchronize).
 *
 * Errors: the original lets C++ exceptions escape through these extern "C" functions. Here no
 * exception escapes: a failure records its message for hrm_last_error() (hrm_capi.h); the
 * pointer-returning wrappers then return NULL, complete_S_K returns -1 (nonzero, so a
 * `while (!complete)` loop ends), and the void wrappers return. store_pointer_state on a field
 * that is not a pointer fails the same way (the original throws "Attempted to set indirection
 * of non-array state field.").
 *
 * Not provided: the device-side entries of the generated shim (dispatch_<fn>_{async,sync}_S,
 * access_<label>_S, halt_early_S; templates.py:187-297), which numba-compiled device code
 * links against; they exist only for specs written in Python, whose front end is not part of
 * this runtime.
 */
#ifndef HRM_PYSHIM_H
#define HRM_PYSHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Field lists: X(suffix, field, is_pointer). */
#define HRM_SHIM_COLLATZ_FIELDS(X, S) \
    X(S, start, 0) X(S, limit, 0) X(S, output, 1) X(S, iterator, 1) X(S, leap, 0)
#define HRM_SHIM_PHOTON_FIELDS(X, S)                                                            \
    X(S, mu_s, 1) X(S, absorb, 1) X(S, split, 1) X(S, tally, 1) X(S, source, 1) X(S, n, 0)     \
    X(S, seed_lo, 0) X(S, seed_hi, 0) X(S, leap, 0) X(S, load_limit, 0)
#define HRM_SHIM_BFS_FIELDS(X, S) \
    X(S, rowptr, 1) X(S, col, 1) X(S, levels, 1) X(S, roots, 1) X(S, root, 0) X(S, nv, 0)

#define HRM_SHIM_DECLARE_FIELD(S, F, P)                    \
    void load_state_##F##_##S(void* host_ptr, void* dev_ptr); \
    void store_state_##F##_##S(void* dev_ptr, void* host_ptr); \
    void store_pointer_state_##F##_##S(void* dev_ptr, void* host_ptr);

#define HRM_SHIM_DECLARE_PROGRAM(S)                                              \
    void* alloc_state_##S(void);                                                 \
    void free_state_##S(void* state_ptr);                                        \
    void* alloc_program_##S(void* device_arg, size_t arena_or_io_size);          \
    void free_program_##S(void* instance_ptr);                                   \
    void init_program_##S(void* instance_ptr, size_t grid_size);                 \
    void exec_program_##S(void* instance_ptr, size_t grid_size, size_t cycle_count); \
    int complete_##S(void* instance_ptr);                                        \
    void clear_flags_##S(void* instance_ptr);                                    \
    void set_device_##S(int device);

HRM_SHIM_DECLARE_PROGRAM(collatz_event)
HRM_SHIM_DECLARE_PROGRAM(collatz_async)
HRM_SHIM_DECLARE_PROGRAM(photon_event)
HRM_SHIM_DECLARE_PROGRAM(photon_async)
HRM_SHIM_DECLARE_PROGRAM(bfs_event)
HRM_SHIM_DECLARE_PROGRAM(bfs_async)
HRM_SHIM_COLLATZ_FIELDS(HRM_SHIM_DECLARE_FIELD, collatz_event)
HRM_SHIM_COLLATZ_FIELDS(HRM_SHIM_DECLARE_FIELD, collatz_async)
HRM_SHIM_PHOTON_FIELDS(HRM_SHIM_DECLARE_FIELD, photon_event)
HRM_SHIM_PHOTON_FIELDS(HRM_SHIM_DECLARE_FIELD, photon_async)
HRM_SHIM_BFS_FIELDS(HRM_SHIM_DECLARE_FIELD, bfs_event)
HRM_SHIM_BFS_FIELDS(HRM_SHIM_DECLARE_FIELD, bfs_async)

#ifdef __cplusplus
}
#endif

#endif
