/*
 * kma_internal.h -- host-side handle types shared by the library's .cu files.
 */
#ifndef KMA_INTERNAL_H
#define KMA_INTERNAL_H

#include <cuda_runtime.h>
#include "kma.h"
#include "kma_device.cuh"

struct kma_heap_s {
	int device;
	void *dev_mem;       /* the single device allocation */
	size_t dev_bytes;
	kma_heap *dh;        /* device header */
	kma_heap hh;         /* host copy of the header's geometry */
};

struct kma_pma;
struct kma_pma_s {
	int device;
	void *mem;
	kma_pma *dp;         /* device header */
	unsigned char *base; /* data base */
	uint64_t bytes;      /* data bytes */
};

#define KMA_DEFAULT_SPIN (1u << 22)

static inline cudaStream_t kma_stream(void *s) { return (cudaStream_t)s; }

/* Run a CUDA call; on failure return KMA_ECUDA from the enclosing
 * function (the sticky error, if any, stays visible to cudaGetLastError). */
#define KMA_CUDA(call)                                  \
	do {                                            \
		cudaError_t e_ = (call);                \
		if (e_ != cudaSuccess)                  \
			return KMA_ECUDA;               \
	} while (0)

/* Make `dev` current for the duration of a scope. */
struct kma_device_guard {
	int prev;
	bool ok;
	explicit kma_device_guard(int dev) : prev(-1), ok(true)
	{
		if (cudaGetDevice(&prev) != cudaSuccess) {
			ok = false;
			return;
		}
		if (dev >= 0 && dev != prev && cudaSetDevice(dev) != cudaSuccess)
			ok = false;
	}
	~kma_device_guard()
	{
		int cur;
		if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev)
			cudaSetDevice(prev);
	}
};

/* host restatement of the class tables, used to fill the header */
int kma_fill_class_tables(uint32_t sb_log2, kma_heap *hh);

#endif
