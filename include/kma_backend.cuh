/*
 * kma_backend.cuh -- program composition: one device heap API over either
 * heap, chosen at compile time.
 *
 * The reference picks a program's heap by which source it concatenates
 * into the program: kma.cl or pma.cl, both defining malloc / free over an
 * opaque struct clheap (clheap.h:35-39; test/tb_clArrayList.c:170-173,
 * 221-223; test/tb_clTree.c:441-446, 478-480).  Here a heap is a type with
 * one static interface, and device code written against it runs on either:
 *
 *   template <class B> __global__ void k(typename B::heap *h, ...)
 *   {   void *p = B::alloc(h, n); ... B::release(h, p);   }
 *
 * instantiated as k<kma_backend_kma> and k<kma_backend_pma>; or, for code
 * that is not a template, against kma_clheap / kma_clheap_malloc /
 * kma_clheap_free, which name the KMA heap unless the translation unit is
 * compiled with -DKMA_BACKEND_PMA (the reference's swap of the .cl file).
 *
 *   alloc(h, n)          malloc: a block of n bytes or NULL
 *   release(h, p)        free; p may point anywhere inside the block (a
 *                        structure that aligns an object inside its block
 *                        frees by the object's address); PMA: nothing
 *   alloc_warp / release_warp   the warp-collaborative forms (any subset of
 *                        a warp may call them)
 *   free_block / free_block_warp   free, for callers holding exactly the
 *                        pointer alloc returned (no search for the block)
 *   no_request           the size a lane passes to alloc_warp when it wants
 *                        nothing (its result is NULL or to be ignored)
 *   base(h)              the address heap offsets are counted from
 */
#ifndef KMA_BACKEND_CUH
#define KMA_BACKEND_CUH

#include "kma_device.cuh"
#include "kma_structs.cuh"

#define KMA_BACKEND_ID_KMA 0
#define KMA_BACKEND_ID_PMA 1

/* kma.cl: superblock heap with free */
struct kma_backend_kma {
	typedef kma_heap heap;
	static constexpr int id = KMA_BACKEND_ID_KMA;
	static __device__ __forceinline__ void *alloc(heap *h, size_t n) { return kma_malloc(h, n); }
	static __device__ __forceinline__ void release(heap *h, void *p) { kma_free(h, block(h, p)); }
	static __device__ __forceinline__ void *alloc_warp(heap *h, size_t n) { return kma_malloc_warp(h, n); }
	static __device__ __forceinline__ void release_warp(heap *h, void *p) { kma_free_warp(h, block(h, p)); }
	static __device__ __forceinline__ void free_block(heap *h, void *p) { kma_free(h, p); }
	static __device__ __forceinline__ void free_block_warp(heap *h, void *p) { kma_free_warp(h, p); }
	static constexpr size_t no_request = ~(size_t)0; /* above every class: NULL at once */
	static __device__ __forceinline__ unsigned char *base(const heap *h) { return h->sb_base; }
	/* the largest request served (SB - 16, kma.cl:126) */
	static __device__ __forceinline__ size_t max_request(const heap *h) { return h->max_request; }
	/* the block that holds p; a pointer outside every live block is
	 * flagged as a bad free (kma_free's check), not silently dropped */
	static __device__ __forceinline__ void *block(heap *h, void *p)
	{
		if (!p)
			return nullptr;
		void *b = kma_block_of(h, p);
		if (!b)
			kma_detail::set_err(h, KMA_ERR_BADFREE);
		return b;
	}
};

/* pma.cl: bump heap, free does nothing (pma.cl:44-48) */
struct kma_backend_pma {
	typedef kma_pma heap;
	static constexpr int id = KMA_BACKEND_ID_PMA;
	static __device__ __forceinline__ void *alloc(heap *h, size_t n) { return kma_pma_malloc(h, n); }
	static __device__ __forceinline__ void release(heap *h, void *p) { kma_pma_free(h, p); }
	static __device__ __forceinline__ void *alloc_warp(heap *h, size_t n) { return kma_pma_malloc_warp(h, n); }
	static __device__ __forceinline__ void release_warp(heap *h, void *p) { kma_pma_free(h, p); }
	static __device__ __forceinline__ void free_block(heap *h, void *p) { kma_pma_free(h, p); }
	static __device__ __forceinline__ void free_block_warp(heap *h, void *p) { kma_pma_free(h, p); }
	static constexpr size_t no_request = 0; /* adds nothing to the warp's bump */
	static __device__ __forceinline__ unsigned char *base(const heap *h) { return h->base; }
	static __device__ __forceinline__ size_t max_request(const heap *) { return ~(size_t)0; }
};

/* the heap a translation unit composes with (clheap.h:37-39) */
#ifdef KMA_BACKEND_PMA
typedef kma_backend_pma kma_clheap_backend;
#else
typedef kma_backend_kma kma_clheap_backend;
#endif
typedef kma_clheap_backend::heap kma_clheap;

__device__ __forceinline__ void *kma_clheap_malloc(kma_clheap *h, size_t n)
{
	return kma_clheap_backend::alloc(h, n);
}
__device__ __forceinline__ void kma_clheap_free(kma_clheap *h, void *p) { kma_clheap_backend::release(h, p); }

/* One-thread replay of an op stream on either heap: ops[i] = {0, size}
 * mallocs (a negative size asks for more than any heap serves), {1, j}
 * frees the block op j returned (nothing when it returned NULL); out[i] =
 * the block's offset from B::base, -1 for NULL, 0 for a free.  mode
 * KMA_MODE_WARP calls the warp forms from the one thread.  The replay of
 * both heaps is this one kernel, instantiated once per backend. */
template <class B>
__global__ void kma_k_heap_replay(typename B::heap *h, const int64_t *ops, int64_t n, int64_t *out, int warp)
{
	if (blockIdx.x != 0 || threadIdx.x != 0)
		return;
	for (int64_t i = 0; i < n; i++) {
		const int64_t kind = ops[2 * i], arg = ops[2 * i + 1];
		if (kind == 0) {
			const size_t sz = arg < 0 ? ~(size_t)0 : (size_t)arg;
			void *p = warp ? B::alloc_warp(h, sz) : B::alloc(h, sz);
			out[i] = p ? (int64_t)((unsigned char *)p - B::base(h)) : -1;
		} else {
			void *q = (arg >= 0 && arg < i && out[arg] >= 0) ? B::base(h) + out[arg] : nullptr;
			if (warp)
				B::free_block_warp(h, q);
			else
				B::free_block(h, q);
			out[i] = 0;
		}
	}
}

#endif /* KMA_BACKEND_CUH */
