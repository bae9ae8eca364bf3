/*
 * ref_pma_unit.c -- the reference's poor man's allocator (pma.cl), the
 * array list over it (clQueue.cl + clArrayList.cl) and the tree driver's
 * graph build over it (clTree.cl + test/tb_clTree.cl, which the reference
 * runs on pma.cl too, test/tb_clTree.c:478-480), compiled unmodified where
 * they lie.  TEST INFRASTRUCTURE ONLY (oracle/_ref/).
 */
#include "ref_shim.h"

#include "pma.cl"
#include "clQueue.cl"
#include "clArrayList.cl"
#include "clTree.cl"
#include "test/tb_clTree.cl"

#undef malloc
#undef free

__thread struct oref_workitem oref_wi = { 1, {0, 0, 0}, {1, 1, 1}, {0, 0, 0}, {1, 1, 1}, NULL };

struct oref_pma {
	struct clheap *heap;
	void *raw;
	size_t bytes;
};

/* pma.c:31-53 + pma.cl:24-30: bytes = sblocks + sizeof(header) (so the
 * "sblocks" argument is a byte count), one work-item runs clheap_init.
 * The buffer is padded by one header so that the reference's limit check
 * (pma.cl:36, which counts the header) cannot run past it. */
void *oref_pma_create(uint64_t sblocks)
{
	struct oref_pma *p;
	size_t bytes = (size_t)sblocks + sizeof(struct clheap);
	if (sblocks == 0)
		return NULL;
	p = calloc(1, sizeof(*p));
	if (!p || posix_memalign(&p->raw, 64, bytes + sizeof(struct clheap))) {
		free(p);
		return NULL;
	}
	memset(p->raw, 0, bytes + sizeof(struct clheap));
	p->bytes = bytes;
	p->heap = p->raw;
	p->heap->bytes = bytes;
	clheap_init(p->heap);
	return p;
}
void oref_pma_destroy(void *p)
{
	struct oref_pma *q = p;
	if (!q)
		return;
	free(q->raw);
	free(q);
}
uint32_t oref_pma_header_bytes(void) { return (uint32_t)sizeof(struct clheap); }
/* offset from the heap's data base (heap->base), -1 = NULL */
int64_t oref_pma_malloc(void *p, uint64_t n)
{
	struct oref_pma *q = p;
	void *r = kma_malloc(q->heap, (size_t)n);
	if (!r)
		return -1;
	return (int64_t)((char *)r - q->heap->base);
}
void oref_pma_free(void *p, int64_t off)
{
	struct oref_pma *q = p;
	kma_free(q->heap, off < 0 ? 0 : (uintptr_t)(q->heap->base + off));
}
uint32_t oref_pma_head(void *p) { return ((struct oref_pma *)p)->heap->head; }
void oref_pma_replay(void *p, const int64_t *ops, int64_t n, int64_t *out)
{
	int64_t i;
	for (i = 0; i < n; i++) {
		if (ops[2 * i] == 0) {
			out[i] = oref_pma_malloc(p, (uint64_t)ops[2 * i + 1]);
		} else {
			int64_t a = ops[2 * i + 1];
			oref_pma_free(p, a < 0 ? -1 : out[a]);
			out[i] = 0;
		}
	}
}

/* ---- graph build (test/tb_clTree.cl:12-85) over pma.cl, one work-item -- */
void *oref_pma_heap(void *p) { return ((struct oref_pma *)p)->heap; }
uint64_t oref_pma_data_base(void *p) { return (uint64_t)(uintptr_t)((struct oref_pma *)p)->heap->base; }
void oref_pma_graph_build_serial(void *p, void *tree_root_word, const uint32_t *edges, uint32_t items)
{
	oref_wi.dim = 1;
	oref_wi.gid[0] = 0;
	oref_wi.gsize[0] = 1;
	clTree_test(((struct oref_pma *)p)->heap, tree_root_word, (struct clTree_link *)edges, items);
}
