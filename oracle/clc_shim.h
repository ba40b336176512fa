/*
 * Runs OpenCL C kernels of the reference on the host CPU -- TEST
 * INFRASTRUCTURE ONLY (the oracle's pin; nothing in the product loads it).
 *
 * The reference's SpMV kernels (src/library/kernels/csrmv_adaptive.cl and
 * csrmv_general.cl) are compiled as C after clc_extract.py has removed the
 * C++ raw-string delimiters the reference wraps them in. This header supplies
 * what OpenCL C takes from its runtime:
 *
 *   - work-items: on x86-64 one fiber per work-item on the calling thread
 *     (a minimal stack switch below: callee-saved registers and the stack
 *     pointer); barrier() yields, and the group's live work-items run round
 *     by round from one barrier to the next, in work-item order, so a launch
 *     is deterministic, atomics included. Elsewhere one POSIX thread per
 *     work-item. The work-groups of a launch run one after another, in group
 *     order, so the kernel's cross-group waits (the first long-row work-group
 *     releasing the others, csrmv_adaptive.cl:596-600, and the last one
 *     waiting for all, :651) are already satisfied when they are reached;
 *   - barrier(): waits for every work-item of the group that has not yet
 *     returned from the kernel (a returned work-item counts as arrived), which
 *     is how csrmv_general.cl's row loop behaves when the last group's
 *     sub-waves run different trip counts;
 *   - __local arrays declared in the kernel body become function statics
 *     (clc_extract.py), shared by the group's threads; only one group runs at
 *     a time;
 *   - 32/64-bit global atomics: GCC __atomic builtins; as_type casts: memcpy.
 *
 * Compile as C11 with -D for the kernel's own build options (VALUE_TYPE,
 * WG_SIZE, ...) exactly as the reference's host code passes them
 * (src/library/blas2/csrmv-adaptive.hpp:38-87, csrmv-vector.hpp:34-83).
 */
#ifndef CLC_SHIM_H_
#define CLC_SHIM_H_

#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---- OpenCL C scalar type names */
typedef unsigned int uint;
typedef unsigned long ulong;

/* ---- work-item state */
static __thread unsigned clc_lid, clc_gid;
static unsigned clc_ngroups, clc_wg_size;

#if defined(__x86_64__)
static unsigned clc_lid_f, clc_gid_f;
static inline size_t get_local_id(unsigned d) { return d == 0 ? clc_lid_f : 0; }
static inline size_t get_group_id(unsigned d) { return d == 0 ? clc_gid_f : 0; }
#else
static inline size_t get_local_id(unsigned d) { return d == 0 ? clc_lid : 0; }
static inline size_t get_group_id(unsigned d) { return d == 0 ? clc_gid : 0; }
#endif
static inline size_t get_local_size(unsigned d) { return d == 0 ? clc_wg_size : 1; }
static inline size_t get_num_groups(unsigned d) { return d == 0 ? clc_ngroups : 1; }
static inline size_t get_global_id(unsigned d) { return d == 0 ? get_group_id(0) * clc_wg_size + get_local_id(0) : 0; }
static inline size_t get_global_size(unsigned d) { return d == 0 ? (size_t)clc_ngroups * clc_wg_size : 1; }

/* ---- fibers (x86-64): work-items as coroutines on the calling thread */
typedef void (*clc_body_fn)(void *args);
#if defined(__x86_64__)
#define CLC_FIBERS 1
void clc_swap(void **save_sp, void *const *load_sp);
__asm__(".text\n"
        ".p2align 4\n"
        "clc_swap:\n"
        "  pushq %rbp\n  pushq %rbx\n  pushq %r12\n  pushq %r13\n  pushq %r14\n  pushq %r15\n"
        "  movq %rsp, (%rdi)\n"
        "  movq (%rsi), %rsp\n"
        "  popq %r15\n  popq %r14\n  popq %r13\n  popq %r12\n  popq %rbx\n  popq %rbp\n"
        "  ret\n");

#define CLC_MAX_WG 1024
#define CLC_STACK (64 * 1024)
static void *clc_sched_sp;
static void *clc_fib_sp[CLC_MAX_WG];
static int clc_fib_done[CLC_MAX_WG];
static char *clc_stacks;
static unsigned clc_cur;
static clc_body_fn clc_fbody;
static void *clc_fargs;
static void clc_fiber_main(void)
{
    clc_fbody(clc_fargs);
    clc_fib_done[clc_cur] = 1;
    clc_swap(&clc_fib_sp[clc_cur], &clc_sched_sp); /* never resumed */
    __builtin_unreachable();
}

static void clc_fiber_init(unsigned l)
{
    uintptr_t top = ((uintptr_t)(clc_stacks + (size_t)(l + 1) * CLC_STACK)) & ~(uintptr_t)15;
    void **sp = (void **)top;
    *--sp = 0;                          /* fake return address: entry sees rsp % 16 == 8 */
    *--sp = (void *)clc_fiber_main;     /* popped by clc_swap's ret */
    for (int k = 0; k < 6; k++) *--sp = 0; /* rbp rbx r12 r13 r14 r15 */
    clc_fib_sp[l] = sp;
    clc_fib_done[l] = 0;
}
#endif

/* ---- barrier over the work-items of the group that are still running */
static pthread_mutex_t clc_m = PTHREAD_MUTEX_INITIALIZER;
static pthread_cond_t clc_c = PTHREAD_COND_INITIALIZER;
static int clc_active, clc_arrived;
static unsigned clc_gen;

static void clc_release_locked(void)
{
    clc_arrived = 0;
    clc_gen++;
    pthread_cond_broadcast(&clc_c);
}

static void barrier(int flags)
{
    (void)flags;
#if defined(__x86_64__)
    clc_swap(&clc_fib_sp[clc_cur], &clc_sched_sp); /* back to the group's scheduler */
    return;
#endif
    pthread_mutex_lock(&clc_m);
    clc_arrived++;
    if (clc_arrived == clc_active) {
        clc_release_locked();
    } else {
        const unsigned g = clc_gen;
        while (g == clc_gen) pthread_cond_wait(&clc_c, &clc_m);
    }
    pthread_mutex_unlock(&clc_m);
}

static void mem_fence(int flags) { (void)flags; __atomic_thread_fence(__ATOMIC_SEQ_CST); }

static void clc_item_returned(void)
{
    pthread_mutex_lock(&clc_m);
    clc_active--;
    if (clc_arrived > 0 && clc_arrived == clc_active) clc_release_locked();
    pthread_mutex_unlock(&clc_m);
}

/* ---- built-in functions the kernels use */
static inline unsigned mad24(unsigned a, unsigned b, unsigned c) { return a * b + c; }
static inline unsigned clz(unsigned x) { return x ? (unsigned)__builtin_clz(x) : 32u; }
static inline unsigned long as_ulong(double v) { unsigned long u; memcpy(&u, &v, 8); return u; }
static inline double as_double(unsigned long u) { double v; memcpy(&v, &u, 8); return v; }
static inline unsigned as_uint(float v) { unsigned u; memcpy(&u, &v, 4); return u; }
static inline float as_float(unsigned u) { float v; memcpy(&v, &u, 4); return v; }

static inline unsigned long atom_xor(volatile unsigned long *p, unsigned long v)
{ return __atomic_fetch_xor(p, v, __ATOMIC_SEQ_CST); }
static inline unsigned long atom_max(volatile unsigned long *p, unsigned long v)
{
    unsigned long old = __atomic_load_n(p, __ATOMIC_SEQ_CST);
    while (old < v && !__atomic_compare_exchange_n(p, &old, v, 0, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) {
    }
    return old;
}
static inline unsigned long atom_inc(volatile unsigned long *p) { return __atomic_fetch_add(p, 1ul, __ATOMIC_SEQ_CST); }
static inline unsigned long atom_cmpxchg(volatile unsigned long *p, unsigned long cmp, unsigned long val)
{
    __atomic_compare_exchange_n(p, &cmp, val, 0, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return cmp;
}
static inline unsigned atomic_xor(volatile unsigned *p, unsigned v) { return __atomic_fetch_xor(p, v, __ATOMIC_SEQ_CST); }
static inline unsigned atomic_inc(volatile unsigned *p) { return __atomic_fetch_add(p, 1u, __ATOMIC_SEQ_CST); }
static inline unsigned atomic_cmpxchg(volatile unsigned *p, unsigned cmp, unsigned val)
{
    __atomic_compare_exchange_n(p, &cmp, val, 0, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return cmp;
}
static inline unsigned atomic_max(volatile unsigned *p, unsigned v)
{
    unsigned old = __atomic_load_n(p, __ATOMIC_SEQ_CST);
    while (old < v && !__atomic_compare_exchange_n(p, &old, v, 0, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) {
    }
    return old;
}

/* ---- launch: ngroups work-groups of wg_size work-items, groups in order */
static clc_body_fn clc_body;
static void *clc_args;
static pthread_barrier_t clc_group_bar;
static int clc_go; /* 0: wait, 1: run, 2: abandon (not every thread could be started) */

static void *clc_thread(void *arg)
{
    clc_lid = (unsigned)(uintptr_t)arg;
    pthread_mutex_lock(&clc_m);
    while (clc_go == 0) pthread_cond_wait(&clc_c, &clc_m);
    const int go = clc_go;
    pthread_mutex_unlock(&clc_m);
    if (go != 1) return NULL;
    for (unsigned g = 0; g < clc_ngroups; g++) {
        clc_gid = g;
        clc_body(clc_args);
        clc_item_returned();
        pthread_barrier_wait(&clc_group_bar); /* every work-item of group g returned */
        if (clc_lid == 0) {
            clc_active = (int)clc_wg_size;
            clc_arrived = 0;
        }
        pthread_barrier_wait(&clc_group_bar); /* state reset before group g + 1 */
    }
    return NULL;
}

#if defined(__x86_64__)
/* Runs every group's work-items as fibers: round by round, each live
 * work-item runs to its next barrier or its end, in work-item order. */
static int clc_launch_fibers(unsigned ngroups, unsigned wg_size, clc_body_fn body, void *args)
{
    if (wg_size == 0 || wg_size > CLC_MAX_WG) return -1;
    if (!clc_stacks) {
        clc_stacks = (char *)malloc((size_t)CLC_MAX_WG * CLC_STACK);
        if (!clc_stacks) return -1;
    }
    clc_ngroups = ngroups;
    clc_wg_size = wg_size;
    clc_fbody = body;
    clc_fargs = args;
    for (unsigned g = 0; g < ngroups; g++) {
        clc_gid_f = g;
        for (unsigned l = 0; l < wg_size; l++) clc_fiber_init(l);
        unsigned live = wg_size;
        while (live > 0) {
            live = 0;
            for (unsigned l = 0; l < wg_size; l++) {
                if (clc_fib_done[l]) continue;
                clc_cur = l;
                clc_lid_f = l;
                clc_swap(&clc_sched_sp, &clc_fib_sp[l]);
                if (!clc_fib_done[l]) live++;
            }
        }
    }
    return 0;
}
#endif

/* Returns 0 on success. Not reentrant: one launch at a time per library. */
static int clc_launch(unsigned ngroups, unsigned wg_size, clc_body_fn body, void *args)
{
#if defined(__x86_64__)
    return clc_launch_fibers(ngroups, wg_size, body, args);
#endif
    static pthread_mutex_t once = PTHREAD_MUTEX_INITIALIZER;
    pthread_mutex_lock(&once);
    clc_ngroups = ngroups;
    clc_wg_size = wg_size;
    clc_body = body;
    clc_args = args;
    clc_active = (int)wg_size;
    clc_arrived = 0;
    int rc = 0;
    pthread_t tid[1024];
    if (wg_size == 0 || wg_size > 1024 || pthread_barrier_init(&clc_group_bar, NULL, wg_size) != 0) {
        pthread_mutex_unlock(&once);
        return -1;
    }
    pthread_attr_t attr;
    pthread_attr_init(&attr);
    pthread_attr_setstacksize(&attr, 256 * 1024);
    unsigned started = 0;
    clc_go = 0;
    for (; started < wg_size; started++)
        if (pthread_create(&tid[started], &attr, clc_thread, (void *)(uintptr_t)started) != 0) break;
    pthread_attr_destroy(&attr);
    pthread_mutex_lock(&clc_m);
    clc_go = started == wg_size ? 1 : 2; /* a partial group would wait forever at its barriers */
    pthread_cond_broadcast(&clc_c);
    pthread_mutex_unlock(&clc_m);
    if (started != wg_size) rc = -2;
    for (unsigned k = 0; k < started; k++) pthread_join(tid[k], NULL);
    pthread_barrier_destroy(&clc_group_bar);
    pthread_mutex_unlock(&once);
    return rc;
}

/* Launch of a kernel without barriers: the work-items run one after another
 * on the calling thread (same results, far cheaper than a thread per
 * work-item). */
static int clc_launch_seq(unsigned ngroups, unsigned wg_size, clc_body_fn body, void *args)
{
    clc_ngroups = ngroups;
    clc_wg_size = wg_size;
    for (unsigned g = 0; g < ngroups; g++)
        for (unsigned l = 0; l < wg_size; l++) {
            clc_gid = g;
            clc_lid = l;
#if defined(__x86_64__)
            clc_gid_f = g;
            clc_lid_f = l;
#endif
            body(args);
        }
    return 0;
}

/* ---- OpenCL C keywords and build constants (after the shim's own code) */
#define __kernel
#define kernel
#define __global
#define global
#define __local
#define local
#define __constant const
#define restrict __restrict__
#define inline static inline
#define __attribute__(x)
#define CL_VERSION_1_0 100
#define CL_VERSION_1_1 110
#define CL_VERSION_1_2 120
#define __OPENCL_VERSION__ 120
#define cl_khr_fp64 1
#define cl_khr_int64_base_atomics 1
#define cl_khr_int64_extended_atomics 1
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2

#endif /* CLC_SHIM_H_ */
