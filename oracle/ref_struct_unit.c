/*
 * ref_struct_unit.c -- the reference's lock-free structures (clQueue.cl,
 * clIndexedQueue.cl, clTree.cl, clArrayList.cl over kma.cl, and the graph
 * kernels of test/tb_clTree.cl), compiled unmodified where they lie,
 * exported for the tests.  TEST INFRASTRUCTURE ONLY (oracle/_ref/).
 */
#include "ref_shim.h"

#include "clQueue.cl"
#include "clIndexedQueue.cl"
#include "kma.cl"
#include "clTree.cl"
#include "clArrayList.cl"
#include "test/tb_clTree.cl"

#undef malloc
#undef free

__thread struct oref_workitem oref_wi = { 1, {0, 0, 0}, {1, 1, 1}, {0, 0, 0}, {1, 1, 1}, NULL };

/* ---- clQueue (clQueue.cl:27-118) ---------------------------------- */
void *oref_q_create(void)
{
	clqueue *q = calloc(1, sizeof(*q));
	if (q)
		clQueue_init(q);
	return q;
}
void oref_q_destroy(void *q) { free(q); }
int oref_q_enqueue(void *q, void *item) { return enqueue(q, item); }
void *oref_q_dequeue(void *q) { return (void *)dequeue(q); }
uint64_t oref_q_head(void *q) { return ((clqueue *)q)->head; }
uint64_t oref_q_tail(void *q) { return ((clqueue *)q)->tail; }

/* ---- clIndexedQueue (clIndexedQueue.cl:93-290) ---------------------- */
/* items at base + (idx-1) << stride_l2; `first` becomes the dummy */
void *oref_iq_create(void *base, uint32_t stride_l2, void *first)
{
	clIndexedQueue *q = calloc(1, sizeof(*q));
	if (q)
		clIndexedQueue_init(q, base, stride_l2, first);
	return q;
}
void oref_iq_destroy(void *q) { free(q); }
int oref_iq_enqueue(void *q, void *item) { return idxd_enqueue(q, item); }
void *oref_iq_dequeue(void *q) { return (void *)idxd_dequeue(q); }
uint32_t oref_iq_head(void *q) { return ((clIndexedQueue *)q)->head; }
uint32_t oref_iq_tail(void *q) { return ((clIndexedQueue *)q)->tail; }

/* ---- clTree (clTree.cl:27-74) -------------------------------------- */
void *oref_tree_create(void) { return calloc(1, sizeof(struct clTree)); }
void oref_tree_destroy(void *t) { free(t); }
uint32_t oref_tree_node_size(void) { return (uint32_t)sizeof(struct clTree_node); }
/* node memory is the caller's; key written by the caller first */
unsigned int oref_tree_add(void *t, void *node) { return clTree_add(t, node); }
void *oref_tree_get(void *t, unsigned int key) { return (void *)clTree_get(t, key); }

/* ---- KMA heap for the array list (4 KiB superblocks) --------------- */
void *oref_heap_create(unsigned int sblocks)
{
	size_t bytes = (size_t)sblocks * KMA_SB_SIZE + sizeof(struct clheap);
	void *raw;
	if (sblocks == 0 || posix_memalign(&raw, 4096, bytes))
		return NULL;
	memset(raw, 0, bytes);
	((struct clheap *)raw)->bytes = bytes;
	clheap_init(raw);
	return raw;
}
void oref_heap_destroy(void *h) { free(h); }
/* the first superblock (offsets in the replays are measured from here) */
void *oref_heap_sb_base(void *h) { return (char *)h + sizeof(struct clheap); }
void *oref_heap_malloc(void *h, uint64_t n) { return (void *)kma_malloc(h, (size_t)n); }
void oref_heap_free(void *h, void *p) { kma_free(h, (uintptr_t)p); }

/* ---- clArrayList (clArrayList.cl:23-216) ---------------------------- */
void *oref_al_create(uint32_t objsize, void *heap)
{
	clArrayList *l = calloc(1, sizeof(*l));
	if (l)
		clArrayList_init((char *)l, objsize, heap);
	return l;
}
void oref_al_destroy(void *l) { free(l); }
uint64_t oref_al_grow(void *l, uint32_t objs) { return clArrayList_grow(l, objs); }
uint64_t oref_al_get(void *l, uint64_t i) { return clArrayList_get(l, (size_t)i); }
void oref_al_clear(void *l) { clArrayList_clear(l); }
uint64_t oref_al_head(void *l) { return ((clArrayList *)l)->queue.head; }

struct oref_group_arg {
	clArrayList *l;
	uint32_t objs;
	uint32_t lid, lsize;
	pthread_barrier_t *bar;
	uintptr_t *rmem;
	uint64_t out;
};

static void *oref_group_main(void *p)
{
	struct oref_group_arg *a = p;
	oref_wi.dim = 1;
	oref_wi.lid[0] = a->lid;
	oref_wi.lsize[0] = a->lsize;
	oref_wi.gid[0] = a->lid;
	oref_wi.gsize[0] = a->lsize;
	oref_wi.group_barrier = a->bar;
	a->out = clArrayList_grow_local(a->l, a->objs, a->rmem);
	return NULL;
}

/* One work-group of `n` work-items (n <= 64, as rMem[128] allows) calls
 * clArrayList_grow_local(l, objs[lid], rMem) together (clArrayList.cl:
 * 111-176); out[lid] receives each item's pointer. */
int oref_al_grow_local_group(void *l, uint32_t n, const uint32_t *objs, uint64_t *out)
{
	pthread_t tid[64];
	struct oref_group_arg a[64];
	pthread_barrier_t bar;
	uintptr_t rmem[128];
	uint32_t i;
	if (n == 0 || n > 64)
		return -1;
	memset(rmem, 0, sizeof(rmem));
	pthread_barrier_init(&bar, NULL, n);
	for (i = 0; i < n; i++) {
		a[i].l = l;
		a[i].objs = objs[i];
		a[i].lid = i;
		a[i].lsize = n;
		a[i].bar = n > 1 ? &bar : NULL;
		a[i].rmem = rmem;
		a[i].out = 0;
		pthread_create(&tid[i], NULL, oref_group_main, &a[i]);
	}
	for (i = 0; i < n; i++) {
		pthread_join(tid[i], NULL);
		out[i] = a[i].out;
	}
	pthread_barrier_destroy(&bar);
	return 0;
}

/* ---- graph build (test/tb_clTree.cl:12-85), serial, one work-item --- */
uint32_t oref_graph_node_size(void) { return (uint32_t)sizeof(struct clGraph_node); }
uint32_t oref_graph_link_size(void) { return (uint32_t)sizeof(struct clGraph_link); }
void oref_graph_build_serial(void *heap, void *tree, const uint32_t *edges, uint32_t items)
{
	oref_wi.dim = 1;
	oref_wi.gid[0] = 0;
	oref_wi.gsize[0] = 1;
	clTree_test(heap, tree, (struct clTree_link *)edges, items);
}
