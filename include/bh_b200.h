/* Flat C ABI of the B200 Bohrium stack.
 *
 * Two boundaries are provided:
 *
 * 1. The component plugin boundary, exactly as the reference binds it: every component library
 *    (libbh_ve_cuda.so, libbh_vem_node.so) exports
 *        extern "C" bohrium::component::ComponentImpl* create(int stack_level);
 *        extern "C" void destroy(bohrium::component::ComponentImpl* self);
 *    (reference: ve/cuda/main.cpp:125-130, resolved by core/bh_component.cpp:30-61).
 *    These use the C++ classes of include/bohrium/bh_component.hpp and are declared there.
 *
 * 2. The bridge below (libbh_core.so), plain C for FFI callers (ctypes, cgo, JNI ...). It stands
 *    in for the reference's generated C bridge (bridge/c/gen_specials.py, the bhc_* functions)
 *    plus bhxx::Runtime (bridge/cxx/src/Runtime.cpp:28-140): it loads a component stack from
 *    config.ini and hands it BhIR batches. Instructions are passed in a flat int64 encoding
 *    instead of one generated function per opcode and type signature.
 *
 * Error convention: functions returning int return 0 on success and -1 on error; functions
 * returning pointers return NULL on error. bhb_last_error() returns the message of the last
 * error on the calling thread. Exceptions never cross this boundary.
 */
#ifndef BH_B200_H
#define BH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bhb_runtime bhb_runtime; /* a loaded component stack */
typedef struct bhb_ir bhb_ir;           /* a decoded, re-executable BhIR */
typedef struct bh_base bh_base;         /* a base array (struct bh_base of bohrium/bh_base.hpp) */

/* Message of the last failed call on this thread ("" if none). */
const char *bhb_last_error(void);

/* Load the stack `stack_name` of the config file `config_path` at stack level 0, the way
 * bhxx::Runtime::Runtime() does (ConfigParser(-1) + ComponentFace(child, 0)). NULL or "" use
 * $BH_CONFIG / $BH_STACK like the reference's ConfigParser (core/bh_config_parser.cpp:44-178). */
bhb_runtime *bhb_runtime_create(const char *config_path, const char *stack_name);
void bhb_runtime_destroy(bhb_runtime *rt);

/* Base arrays (bhc_new_A<type> / bhc_destroy_A<type>). dtype is the bh_type enum value
 * (BOOL=0 ... FLOAT64=10, COMPLEX64=11, COMPLEX128=12, R123=13). A base must only be destroyed
 * after a flushed BH_FREE released its data, or if it was never used. */
bh_base *bhb_base_create(int dtype, int64_t nelem);
void bhb_base_destroy(bh_base *base);
int bhb_base_dtype(const bh_base *base);
int64_t bhb_base_nelem(const bh_base *base);

/* getMemoryPointer (bhc_data_get_A<type>; ComponentImpl::getMemoryPointer): with copy2host the
 * host copy is made valid and returned (the device copy is released so the caller may write);
 * without it the device pointer is returned. */
void *bhb_data_get(bhb_runtime *rt, bh_base *base, int copy2host, int force_alloc, int nullify);
/* setMemoryPointer (bhc_data_set_A<type>; ComponentImpl::setMemoryPointer). The stack takes
 * ownership: host memory must come from bhb_host_alloc() or malloc(); device memory from
 * cudaMalloc(). */
int bhb_data_set(bhb_runtime *rt, bh_base *base, int host_ptr, void *data);
/* Page-locked host memory usable with bhb_data_set(host_ptr=1). */
void *bhb_host_alloc(bhb_runtime *rt, int64_t nbytes);
/* Copy `nbytes` of host data into the base's host storage (allocated on demand); the device copy
 * is released. */
int bhb_data_copy_in(bhb_runtime *rt, bh_base *base, const void *src, int64_t nbytes);

/* BhIR encoding (int64 words), one record per instruction:
 *   opcode, nop, const_type (-1: no constant), const_word0, const_word1,
 *   then nop operands, each: base (bh_base* as int64, 0 for the constant operand),
 *   and for a non-constant operand: start, ndim, shape[ndim], stride[ndim].
 * Strides and starts are in elements (include/bohrium/bh_view.hpp:45-62 of the reference).
 * The constant's 16 bytes are the bh_constant_value union.
 *
 * Slides (do_while sliding views, bh_slide.hpp:29-101), one record per sliding operand:
 *   instr_index, operand_index, ndims, ndims x (rank, offset_change, shape_change, stride, shape,
 *   step_delay), nresets, nresets x (dim, reset_max). */
bhb_ir *bhb_ir_create(const int64_t *words, int64_t nwords, bh_base *const *syncs, int64_t nsyncs,
                      uint64_t nrepeats, bh_base *repeat_condition, const int64_t *slides, int64_t nslide_words);
void bhb_ir_destroy(bhb_ir *ir);
/* ComponentImpl::execute of level 0 (bhc_flush / bhc_flush_and_repeat[_condition]). */
int bhb_ir_execute(bhb_runtime *rt, bhb_ir *ir);
/* Decode and execute once. */
int bhb_execute(bhb_runtime *rt, const int64_t *words, int64_t nwords, bh_base *const *syncs, int64_t nsyncs,
                uint64_t nrepeats, bh_base *repeat_condition, const int64_t *slides, int64_t nslide_words);

/* ComponentImpl::message (bhc_message). The returned string stays valid until the next call on
 * the same runtime. */
const char *bhb_message(bhb_runtime *rt, const char *msg);
/* ComponentImpl::extmethod (bhc_extmethod): register extension method `name` as `opcode`
 * (> BH_MAX_OPCODE_ID). */
int bhb_extmethod(bhb_runtime *rt, const char *name, int64_t opcode);
/* ComponentImpl::userKernel (replaces bhc_user_kernel, bridge/c/gen_specials.py:287-304, and
 * bhxx::Runtime::userKernel, bridge/cxx/src/Runtime.cpp:131-138): compile `kernel` and run its
 * function `execute` with one argument per operand, the start of that base's data, in order. The
 * caller flushes pending bytecode first, as the reference's front end does. Tag "cuda" runs on
 * this engine: `execute` is an `extern "C" __global__` function compiled with NVRTC for sm_100a,
 * launched with blocks of local_work_size threads and global_work_size / local_work_size blocks,
 * both taken from `param` ("global_work_size: 1024; local_work_size: 128", up to three numbers
 * each); `compile_cmd` is not used. Other tags go down the stack. Returns the component's message:
 * "" on success, else the error text (which the reference's front end raises); NULL when the call
 * itself failed (bhb_last_error). The string stays valid until the next call on the same
 * runtime. */
const char *bhb_user_kernel(bhb_runtime *rt, const char *kernel, int64_t nop, bh_base *const *operands,
                            const char *compile_cmd, const char *tag, const char *param);
/* ComponentImpl::getDeviceContext / setDeviceContext. */
void *bhb_get_device_context(bhb_runtime *rt);
int bhb_set_device_context(bhb_runtime *rt, void *ctx);

/* Device-side timing of the last execute on the engine's stream, in milliseconds (CUDA events;
 * 0 when the stack has no GPU engine). */
double bhb_last_execute_ms(bhb_runtime *rt);

/* Host data pointer of a base (valid after a flush that synced it; NULL without host storage). */
void *bhb_base_data(const bh_base *base);

/* --- In-tree hooks between the bridge and the engine library (not part of the reference
 * interface) --- */
/* The decoded BhIR (a BhIR*) behind a bhb_ir handle. */
void *bhb_ir_bhir(bhb_ir *ir);
/* Set the message returned by bhb_last_error() on this thread. */
void bhb_set_last_error(const char *msg);
/* Apply a bytecode filter of the filter components in place: "bcexp" (powk) with optional
 * "+sign" and "+reduce1d=<thread limit>" (e.g. "bcexp+reduce1d=32000", the reference's GPU-stack
 * setting), or "bccon" (stupidmath, collect, muladd). Returns the number of rewrites, -1 on error.
 * (The filters restate filter/bcexp/expander.cpp:42-87, expand_reduce1d.cpp:31-80 and
 * filter/bccon/contracter.cpp:46-52.) */
int bhb_ir_filter(bhb_ir *ir, const char *name);
/* Text listing of a decoded BhIR (opcode, operands with bases numbered by first appearance,
 * constant), valid until the next call on the same handle. */
const char *bhb_ir_text(bhb_ir *ir);
/* libbh_ve_cuda.so: fuse `ir`, generate the kernel sources and, if `compile` is set, compile them
 * with NVRTC for sm_100a, all without a GPU. Returns a JSON document (valid until the next call)
 * or NULL on error. `fuser_list` overrides the transformer list (NULL: the engine default). */
const char *bh_ve_cuda_dry_run(bhb_ir *ir, int compile, const char *fuser_list);

/* --- Extension methods run by the cuda engine (reference: include/bohrium/bh_extmethod.hpp:57-134;
 * the reference's GPU engines pass themselves as the `arg` of ExtmethodImpl::execute). The cuda
 * engine passes a pointer to this plain struct instead, so that an extmethod library needs no C++
 * type of the engine. --- */
typedef struct bh_ve_cuda_ext_context {
    int version;   /* 1 */
    void *engine;  /* opaque; first argument of the callbacks */
    void *stream;  /* cudaStream_t the engine runs its kernels on; extmethods enqueue on it */
    /* Device buffer of a base array (allocated, and uploaded from the host copy, on demand). */
    void *(*device_pointer)(void *engine, bh_base *base);
    /* Tell the engine that the device copy of `base` was written (its host copy is now stale). */
    void (*written)(void *engine, bh_base *base);
} bh_ve_cuda_ext_context;

/* --- libbh_ve_cuda.so: the learned fusion cost model's network (no counterpart in the reference,
 * whose fuser is the plain greedy one, core/jitk/graph.cpp:319-365). An MLP of
 * bh_ve_cuda_costmodel_nfeatures() inputs -> 64 -> 64 -> 1 (ReLU, float32) on the current
 * device; inference and minibatch Adam training run in hand-written kernels with deterministic
 * (fixed-order) reductions. Host arrays in and out; the loss is the mean squared error. Functions
 * returning int give 0 on success and -1 with bhb_last_error() set. --- */
typedef struct bh_costmodel bh_costmodel;
int bh_ve_cuda_costmodel_nfeatures(void);
int64_t bh_ve_cuda_costmodel_nparams(void);
/* He-initialised weights from `seed`; NULL on error. */
bh_costmodel *bh_ve_cuda_costmodel_create(uint64_t seed);
void bh_ve_cuda_costmodel_destroy(bh_costmodel *cm);
/* Parameters as float32[nparams]: W1[64][F], b1[64], W2[64][64], b2[64], W3[64], b3. Setting them
 * also resets the Adam moments. */
int bh_ve_cuda_costmodel_get_params(bh_costmodel *cm, float *out);
int bh_ve_cuda_costmodel_set_params(bh_costmodel *cm, const float *in);
/* y[r] = network(x[r]) for `rows` rows of F floats. */
int bh_ve_cuda_costmodel_predict(bh_costmodel *cm, const float *x, int64_t rows, float *y);
/* Gradient (float32[nparams]) and loss over all rows, without an update. */
int bh_ve_cuda_costmodel_gradient(bh_costmodel *cm, const float *x, const float *t, int64_t rows, float *grad,
                                  float *loss);
/* `epochs` passes of minibatch Adam (beta 0.9/0.999) over the rows in a seeded order; `loss_out`
 * (may be NULL) receives the final loss over all rows. */
int bh_ve_cuda_costmodel_train(bh_costmodel *cm, const float *x, const float *t, int64_t rows, int epochs,
                               int batch, float lr, uint64_t seed, float *loss_out);

/* libbh_ve_cuda.so: allocation-free sum of `n` contiguous float64 values at device address `in`,
 * written to the device address `out`, enqueued on `stream` (a cudaStream_t; NULL: the legacy
 * default stream). No counterpart in the reference: it is the engine's ADD_REDUCE grid reduction
 * with its tile partials in a fixed static device array (65,792 bytes per device) instead of
 * allocated scratch, for callers that cannot let a library allocate device memory. It calls no
 * cudaMalloc, cudaFree or other allocating routine. n is at most 16,777,216 (8,192 tiles of 2,048);
 * larger n is rejected with an error. The first call on each device, made with that device
 * current, does a one-time set-up (cudaGetSymbolAddress of the array); make it before any stream
 * capture. All calls share the array: calls whose kernels overlap on the GPU race. Returns 0, or
 * -1 with bhb_last_error() set. */
int bh_ve_cuda_sum_f64_noalloc(const double *in, int64_t n, double *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* BH_B200_H */
