/*
 * ref_shim.h -- OpenCL C 1.x -> host C shim for building the reference
 * KMA sources (kma.cl, clIndexedQueue.cl, clQueue.cl, clTree.cl,
 * clArrayList.cl, pma.cl) UNMODIFIED as a host shared library.
 *
 * TEST INFRASTRUCTURE ONLY.  The library built from this shim lives in
 * oracle/_ref/ (git-ignored) and is used by tests/ and bench.py's CPU
 * baseline as the checker; nothing in the product links it.
 *
 * What the shim maps (the OpenCL built-ins the reference uses):
 *   __kernel/__global/__local/__constant  -> nothing
 *   atom_cmpxchg                          -> __sync_val_compare_and_swap
 *   atom_xchg/add/or/and                  -> __atomic_*_n, seq_cst
 *   mem_fence                             -> __atomic_thread_fence(seq_cst)
 *   get_global_id/size, get_local_id/size,
 *   get_work_dim                          -> thread-local work-item ids set
 *                                            by the driver (ref_threads.c)
 *   barrier                               -> per-work-group pthread barrier
 *   malloc/free (the device heap API of clheap.h:37-39)
 *                                         -> kma_malloc/kma_free symbols so
 *                                            they do not clash with libc
 * CL_BITNESS=64 and CL_PLATFORM=0 select the reference's 64-bit, generic
 * (unbounded-loop) code paths (clQueue.h:73-78, kma.h:95-98).
 */
#ifndef ORACLE_REF_SHIM_H
#define ORACLE_REF_SHIM_H

/* All system headers first: the reference redefines NULL and uint32_t. */
#include <stdint.h>
#include <stddef.h>
#include <stdbool.h>
#include <string.h>
#include <stdlib.h>
#include <pthread.h>

#define CL_BITNESS 64
#define CL_PLATFORM 0

#define __kernel
#define __global
#define __local
#define __constant

#define CLK_GLOBAL_MEM_FENCE 1
#define CLK_LOCAL_MEM_FENCE 2

#define atom_cmpxchg(p, c, v) __sync_val_compare_and_swap((p), (c), (v))
#define atom_xchg(p, v) __atomic_exchange_n((p), (v), __ATOMIC_SEQ_CST)
#define atom_add(p, v) __atomic_fetch_add((p), (v), __ATOMIC_SEQ_CST)
#define atom_or(p, v) __atomic_fetch_or((p), (v), __ATOMIC_SEQ_CST)
#define atom_and(p, v) __atomic_fetch_and((p), (v), __ATOMIC_SEQ_CST)
#define mem_fence(f) __atomic_thread_fence(__ATOMIC_SEQ_CST)

/* Work-item identity, set per emulated work-item by the driver. */
struct oref_workitem {
	unsigned int dim;
	size_t gid[3], gsize[3], lid[3], lsize[3];
	pthread_barrier_t *group_barrier; /* NULL when the group has 1 item */
};
extern __thread struct oref_workitem oref_wi;

static inline unsigned int get_work_dim(void) { return oref_wi.dim; }
static inline size_t get_global_id(unsigned int d) { return d < 3 ? oref_wi.gid[d] : 0; }
static inline size_t get_global_size(unsigned int d) { return d < 3 ? oref_wi.gsize[d] : 1; }
static inline size_t get_local_id(unsigned int d) { return d < 3 ? oref_wi.lid[d] : 0; }
static inline size_t get_local_size(unsigned int d) { return d < 3 ? oref_wi.lsize[d] : 1; }
static inline void oref_barrier(void)
{
	__atomic_thread_fence(__ATOMIC_SEQ_CST);
	if (oref_wi.group_barrier)
		pthread_barrier_wait(oref_wi.group_barrier);
	__atomic_thread_fence(__ATOMIC_SEQ_CST);
}
#define barrier(f) oref_barrier()

/* The reference's device heap API names (clheap.h:38-39). */
#define malloc kma_malloc
#define free kma_free

#endif /* ORACLE_REF_SHIM_H */
