/*
 * kma_graph.cu -- the graph-build workload (include/kma_graph.h), after the
 * reference's tree driver (test/tb_clTree.cl:12-85).
 *
 * Build: threads stride over the edges; for each, clGraph_node_ensure both
 * endpoints (tree get; else malloc a node, init its links queue, tree add;
 * free the node again when another thread added the key first) and
 * enqueue a freshly malloc'd link on the source's queue.  Every inserted
 * node is also recorded in a registry array, so the walk and the teardown
 * run one thread per node.
 *
 * Every kernel is a template on the heap backend (kma_backend.cuh), as the
 * reference's driver builds the same tb_clTree.cl over kma.cl or pma.cl
 * (test/tb_clTree.c:441-446, 478-480).
 */
#include <string.h>
#include <stdlib.h>
#include <algorithm>
#include <numeric>
#include <vector>

#include "kma_internal.h"
#include "kma_graph.h"
#include "kma_structs.h"
#include "kma_structs.cuh"
#include "kma_backend.cuh"

#define GR_LINK_REQ 16u /* the reference's clGraph_link size */

namespace {

/* 40 bytes, the reference's clGraph_node size (tb_clTree.h) */
struct gr_node {
	kma_clqueue links;
	kma_cltree_node tree;  /* key, state, left, right */
};

/* Where a node sits in its block.  KMA blocks are only 4-byte aligned, so
 * the node goes to align16(block) inside a 52-byte request, the same size
 * class as the reference's 40-byte request; PMA blocks of this build are
 * 8-byte aligned (40- and 16-byte requests from an aligned base), so the
 * node is the block and the request is the reference's own 40 bytes:
 * either way serial builds use the reference's blocks. */
template <class B> struct gr_layout;
template <> struct gr_layout<kma_backend_kma> {
	static constexpr uint32_t node_req = 52, node_align = 16;
};
template <> struct gr_layout<kma_backend_pma> {
	static constexpr uint32_t node_req = 40, node_align = 8;
};

__host__ __device__ __forceinline__ uint64_t gr_mix(uint32_t a, uint32_t b)
{
	uint64_t z = ((uint64_t)a << 32 | b) + 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

__device__ __forceinline__ gr_node *gr_of_tree(kma_cltree_node *t)
{
	return reinterpret_cast<gr_node *>(reinterpret_cast<unsigned char *>(t) - offsetof(gr_node, tree));
}

template <class B>
struct gr_dev {
	typename B::heap *h;
	kma_cltree *tree;
	gr_node **reg;               /* [cap] inserted nodes */
	unsigned long long *nreg;
	unsigned long long *acc;     /* lost_adds, nulls */
	uint32_t *qerr;
};

/* clGraph_node_ensure (tb_clTree.cl:12-38); NULL when the heap is out of
 * blocks (the reference retries forever there) */
template <class B>
__device__ gr_node *gr_ensure(const gr_dev<B> &g, uint32_t key, unsigned long long &lost, unsigned long long &nulls)
{
	for (int tries = 0; tries < 1 << 20; tries++) {
		kma_cltree_node *t = kma_cltree_get(g.tree, key);
		if (t)
			return gr_of_tree(t);
		void *b = B::alloc(g.h, gr_layout<B>::node_req);
		if (!b) {
			nulls++;
			return nullptr;
		}
		const uintptr_t al = gr_layout<B>::node_align - 1;
		gr_node *n = reinterpret_cast<gr_node *>(((uintptr_t)b + al) & ~al);
		n->tree.key = key;
		kma_clqueue_init(&n->links);
		__threadfence();
		if (kma_cltree_add(g.tree, &n->tree) == KMA_TREE_INSERTED) {
			unsigned long long i = atomicAdd(g.nreg, 1ull);
			g.reg[i] = n;
			return n;
		}
		B::release(g.h, b);
		lost++;
	}
	atomicOr(g.qerr, KMA_ERR_TIMEOUT);
	return nullptr;
}

/* clTree_test (tb_clTree.cl:40-85) */
template <class B>
__global__ void k_gr_build(gr_dev<B> g, const uint32_t *edges, uint64_t n)
{
	uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	unsigned long long lost = 0, nulls = 0;
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
		gr_node *src = gr_ensure(g, edges[2 * i], lost, nulls);
		gr_node *snk = gr_ensure(g, edges[2 * i + 1], lost, nulls);
		if (!src || !snk)
			continue;
		void *b = B::alloc(g.h, GR_LINK_REQ);
		if (!b) {
			nulls++;
			continue;
		}
		unsigned char *item = reinterpret_cast<unsigned char *>(((uintptr_t)b + 7) & ~(uintptr_t)7);
		*reinterpret_cast<uint32_t *>(item + 8) = (uint32_t)(((unsigned char *)snk - B::base(g.h)) >> 3);
		__threadfence();
		kma_clqueue_enqueue(&src->links, reinterpret_cast<kma_clqueue_item *>(item), g.qerr);
	}
	if (lost)
		atomicAdd(&g.acc[0], lost);
	if (nulls)
		atomicAdd(&g.acc[1], nulls);
}

template <class B>
__device__ __forceinline__ uint32_t gr_sink_key(const gr_dev<B> &g, const kma_clqueue_item *it)
{
	uint32_t off8 = *reinterpret_cast<const uint32_t *>(reinterpret_cast<const unsigned char *>(it) + 8);
	const gr_node *s = reinterpret_cast<const gr_node *>(B::base(g.h) + ((size_t)off8 << 3));
	return s->tree.key;
}

/* per node: links in queue order -> count, edge hashes; optionally the
 * sinks at out[start[i] ...] */
template <class B>
__global__ void k_gr_walk(gr_dev<B> g, uint64_t nodes, unsigned long long *counts, const uint64_t *start,
		uint32_t *sinks, unsigned long long *sums /* links, xor, sum */)
{
	uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long c = 0, x = 0, s = 0;
	if (i < nodes) {
		const gr_node *nd = g.reg[i];
		uint32_t key = nd->tree.key;
		for (const kma_clqueue_item *it = kma_clqueue_first(&nd->links); it && c < (1ull << 31);
		     it = kma_clqueue_next(it)) {
			uint32_t sk = gr_sink_key(g, it);
			if (sinks)
				sinks[start[i] + c] = sk;
			uint64_t m = gr_mix(key, sk);
			x ^= m;
			s += m;
			c++;
		}
		if (counts)
			counts[i] = c;
	}
	if (c)
		atomicAdd(&sums[0], c);
	if (x)
		atomicXor(&sums[1], x);
	if (s)
		atomicAdd(&sums[2], s);
}

/* offset of the block that holds node nd (PMA: of the node itself, its
 * blocks have no recorded start) */
__device__ __forceinline__ long long gr_block_off(kma_heap *h, const gr_node *nd)
{
	return (long long)((const unsigned char *)kma_block_of(h, nd) - h->sb_base);
}
__device__ __forceinline__ long long gr_block_off(kma_pma *p, const gr_node *nd)
{
	return (long long)((const unsigned char *)nd - p->base);
}

template <class B>
__global__ void k_gr_export(gr_dev<B> g, uint64_t nodes, uint32_t *keys, long long *offs)
{
	uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nodes)
		return;
	const gr_node *nd = g.reg[i];
	keys[i] = nd->tree.key;
	offs[i] = gr_block_off(g.h, nd);
}

/* in-order walk with an explicit stack: strictly increasing keys? */
__global__ void k_gr_sorted(const kma_cltree *t, unsigned long long *stack, uint64_t cap, unsigned long long *out)
{
	uint64_t sp = 0, count = 0;
	long long prev = -1;
	uint32_t sorted = 1;
	unsigned long long cur = t->root;
	while (cur || sp) {
		while (cur) {
			if (sp >= cap) {
				out[0] = 2; /* deeper than the stack: not checked */
				return;
			}
			stack[sp++] = cur;
			cur = ((const kma_cltree_node *)cur)->left;
		}
		cur = stack[--sp];
		const kma_cltree_node *nd = (const kma_cltree_node *)cur;
		if ((long long)nd->key <= prev)
			sorted = 0;
		prev = nd->key;
		count++;
		cur = nd->right;
	}
	out[0] = sorted;
	out[1] = count;
}

/* teardown: every node frees its links, then itself */
template <class B>
__global__ void k_gr_free(gr_dev<B> g, uint64_t nodes)
{
	uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nodes)
		return;
	gr_node *nd = g.reg[i];
	for (;;) {
		kma_clqueue_item *it = kma_clqueue_dequeue(&nd->links, g.qerr);
		if (!it)
			break;
		B::release(g.h, it);
	}
	B::release(g.h, nd);
}

} /* namespace */

extern "C" uint64_t kma_graph_edge_mix(uint32_t source, uint32_t sink) { return gr_mix(source, sink); }

namespace {
/* The build on heap dh (device header) of either backend; region_bytes:
 * the heap's data bytes (sink offsets are 32-bit multiples of 8 bytes). */
template <class B>
int graph_build(typename B::heap *dh, int device, uint64_t region_bytes, const uint32_t *edges, uint64_t n,
		uint32_t threads, int free_after, kma_graph_stats *st, uint32_t *keys_out, int64_t *node_off,
		uint32_t *link_sinks, uint64_t *link_start)
{
	if (!dh || !edges || !st || n == 0 || n > (1ull << 30) || threads == 0)
		return KMA_EINVAL;
	if (region_bytes > (1ull << 35))
		return KMA_EINVAL;
	if (keys_out && (!node_off || !link_sinks || !link_start))
		return KMA_EINVAL;
	kma_device_guard gd(device);
	memset(st, 0, sizeof(*st));
	uint64_t cap = 2 * n;
	void *mem = NULL;
	size_t o_tree = 0, o_reg = 256, o_nreg = o_reg + cap * 8, o_acc = o_nreg + 8, o_err = o_acc + 16,
	       o_sums = (o_err + 8 + 255) & ~(size_t)255, o_cnt = o_sums + 64, o_start = o_cnt + cap * 8,
	       o_sinks = o_start + (cap + 1) * 8, o_keys = o_sinks + n * 4, o_offs = (o_keys + cap * 4 + 7) & ~(size_t)7,
	       o_edges = o_offs + cap * 8, o_stack = o_edges + n * 8, total = o_stack + (size_t)(1 << 20) * 8;
	if (cudaMalloc(&mem, total) != cudaSuccess) {
		cudaGetLastError();
		return KMA_ENOMEM;
	}
	unsigned char *m = (unsigned char *)mem;
	int rc = KMA_OK;
	gr_dev<B> g;
	g.h = dh;
	g.tree = (kma_cltree *)(m + o_tree);
	g.reg = (gr_node **)(m + o_reg);
	g.nreg = (unsigned long long *)(m + o_nreg);
	g.acc = (unsigned long long *)(m + o_acc);
	g.qerr = (uint32_t *)(m + o_err);
	unsigned long long *sums = (unsigned long long *)(m + o_sums);
	if (cudaMemset(m, 0, o_reg) != cudaSuccess || cudaMemset(m + o_nreg, 0, o_cnt - o_nreg) != cudaSuccess ||
	    cudaMemcpy(m + o_edges, edges, n * 8, cudaMemcpyHostToDevice) != cudaSuccess)
		rc = KMA_ECUDA;
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	if (rc == KMA_OK) {
		uint32_t bd = threads < 256 ? threads : 256;
		uint32_t nb = (threads + bd - 1) / bd;
		cudaEventRecord(e0);
		k_gr_build<B><<<nb, bd>>>(g, (const uint32_t *)(m + o_edges), n);
		cudaEventRecord(e1);
		if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
			rc = KMA_ECUDA;
		cudaEventElapsedTime(&st->build_ms, e0, e1);
	}
	unsigned long long nodes = 0, acc[2] = {0, 0};
	uint32_t qerr = 0;
	if (rc == KMA_OK && (cudaMemcpy(&nodes, g.nreg, 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
			     cudaMemcpy(acc, g.acc, 16, cudaMemcpyDeviceToHost) != cudaSuccess))
		rc = KMA_ECUDA;
	uint32_t gb = (uint32_t)((nodes + 255) / 256);
	if (rc == KMA_OK && nodes) {
		unsigned long long *cnt = (unsigned long long *)(m + o_cnt);
		k_gr_walk<B><<<gb, 256>>>(g, nodes, keys_out ? cnt : NULL, NULL, NULL, sums);
		k_gr_sorted<<<1, 1>>>(g.tree, (unsigned long long *)(m + o_stack), 1 << 20, sums + 4);
		if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
			rc = KMA_ECUDA;
		unsigned long long sm[6];
		if (rc == KMA_OK && cudaMemcpy(sm, sums, sizeof(sm), cudaMemcpyDeviceToHost) != cudaSuccess)
			rc = KMA_ECUDA;
		if (rc == KMA_OK) {
			st->links = sm[0];
			st->edge_xor = sm[1];
			st->edge_sum = sm[2];
			st->sorted = (uint32_t)sm[4];
		}
		if (rc == KMA_OK && keys_out) {
			/* export: nodes in key order, links in queue order */
			std::vector<unsigned long long> c(nodes);
			std::vector<uint32_t> k(nodes);
			std::vector<long long> o(nodes);
			k_gr_export<B><<<gb, 256>>>(g, nodes, (uint32_t *)(m + o_keys), (long long *)(m + o_offs));
			if (cudaDeviceSynchronize() != cudaSuccess ||
			    cudaMemcpy(c.data(), cnt, nodes * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
			    cudaMemcpy(k.data(), m + o_keys, nodes * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
			    cudaMemcpy(o.data(), m + o_offs, nodes * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
				rc = KMA_ECUDA;
			std::vector<uint64_t> start(nodes + 1, 0);
			for (uint64_t i = 0; i < nodes; i++)
				start[i + 1] = start[i] + c[i];
			if (rc == KMA_OK && start[nodes] <= n) {
				if (cudaMemcpy(m + o_start, start.data(), (nodes + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess)
					rc = KMA_ECUDA;
				cudaMemset(sums, 0, 24);
				k_gr_walk<B><<<gb, 256>>>(g, nodes, NULL, (const uint64_t *)(m + o_start),
							 (uint32_t *)(m + o_sinks), sums);
				std::vector<uint32_t> sk(start[nodes] ? start[nodes] : 1);
				if (rc == KMA_OK && (cudaDeviceSynchronize() != cudaSuccess ||
						     cudaMemcpy(sk.data(), m + o_sinks, start[nodes] * 4,
								cudaMemcpyDeviceToHost) != cudaSuccess))
					rc = KMA_ECUDA;
				if (rc == KMA_OK) {
					std::vector<uint64_t> ord(nodes);
					std::iota(ord.begin(), ord.end(), 0);
					std::sort(ord.begin(), ord.end(), [&](uint64_t a, uint64_t b) { return k[a] < k[b]; });
					uint64_t pos = 0;
					for (uint64_t j = 0; j < nodes; j++) {
						uint64_t i = ord[j];
						keys_out[j] = k[i];
						node_off[j] = o[i];
						link_start[j] = pos;
						for (uint64_t q = start[i]; q < start[i + 1]; q++)
							link_sinks[pos++] = sk[q];
					}
					link_start[nodes] = pos;
				}
			} else if (rc == KMA_OK) {
				rc = KMA_EFAULT;
			}
		}
	}
	if (rc == KMA_OK && free_after && nodes) {
		k_gr_free<B><<<gb, 256>>>(g, nodes);
		if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
			rc = KMA_ECUDA;
	}
	if (rc == KMA_OK)
		cudaMemcpy(&qerr, g.qerr, 4, cudaMemcpyDeviceToHost);
	st->nodes = nodes;
	st->lost_adds = acc[0];
	st->nulls = acc[1];
	st->err = qerr;
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(mem);
	return rc;
}
} /* namespace */

extern "C" int kma_graph_build(kma_heap_t h, const uint32_t *edges, uint64_t n, uint32_t threads, int free_after,
		kma_graph_stats *st, uint32_t *keys_out, int64_t *node_off, uint32_t *link_sinks,
		uint64_t *link_start)
{
	if (!h)
		return KMA_EINVAL;
	return graph_build<kma_backend_kma>(h->dh, h->device, h->hh.region_bytes, edges, n, threads, free_after, st,
					    keys_out, node_off, link_sinks, link_start);
}

extern "C" int kma_graph_build_pma(kma_pma_t p, const uint32_t *edges, uint64_t n, uint32_t threads,
		kma_graph_stats *st, uint32_t *keys_out, int64_t *node_off, uint32_t *link_sinks,
		uint64_t *link_start)
{
	if (!p)
		return KMA_EINVAL;
	return graph_build<kma_backend_pma>(p->dp, p->device, p->bytes, edges, n, threads, 0, st, keys_out, node_off,
					    link_sinks, link_start);
}
