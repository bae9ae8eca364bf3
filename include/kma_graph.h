/*
 * kma_graph.h -- the graph-build workload of the reference's tree driver
 * (test/tb_clTree.cl:12-85, clTree_test / clGraph_node_ensure): for every
 * edge (source, sink) make sure both vertices exist as nodes of a clTree
 * (malloc a node, add it, free it again if another thread added the key
 * first), then malloc a link to the sink and enqueue it on the source's
 * clQueue of links.  Exercises kma_malloc, kma_free, the tree and the
 * queue together.  The reference's edge file is not shipped, so callers
 * pass synthetic edges.
 *
 * Layout: KMA heap blocks are 4-byte aligned, so a 40-byte node (its links
 * queue, then its tree node) sits at align16(block) inside a 52-byte
 * request -- the same size class as the reference's 40-byte clGraph_node;
 * on the PMA heap the node is its 40-byte block.  A link (8-byte aligned
 * queue link, then the sink's offset from the heap base / 8 as a u32) sits
 * in a 16-byte request, the reference's clGraph_link size.  Serial runs
 * therefore use the same blocks as the reference on either heap; heaps
 * hold at most 32 GiB.
 */
#ifndef KMA_GRAPH_H
#define KMA_GRAPH_H

#include <stdint.h>
#include "kma.h"
#include "kma_structs.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct kma_graph_stats {
	uint64_t nodes;          /* nodes in the tree */
	uint64_t links;          /* links found walking every node's queue */
	uint64_t lost_adds;      /* nodes freed because another thread added the key first */
	uint64_t nulls;          /* mallocs that returned NULL (edge skipped) */
	uint64_t edge_xor, edge_sum; /* over mix(source, sink) of the links found */
	uint32_t sorted;         /* 1 when the in-order walk is strictly increasing */
	uint32_t err;            /* heap / queue error flags seen */
	float build_ms;          /* device time of the build kernel */
	float pad;
} kma_graph_stats;

/* The multiset hash used for edge_xor / edge_sum: mix(source, sink). */
uint64_t kma_graph_edge_mix(uint32_t source, uint32_t sink);

/* Build the graph of `n` edges (host array of n (source, sink) u32 pairs)
 * on heap h with `threads` device threads striding over the edges
 * (threads = 1: the reference's one-work-item order).  Walk the result
 * into *st; when keys_out is non-NULL also export the nodes in key order
 * (keys_out[i], node_off[i] = the node's offset from the first superblock)
 * and each node's links in queue order (sinks of node i at
 * link_sinks[link_start[i] .. link_start[i+1])); capacities: 2n nodes, n
 * links.  free_after != 0 frees every link and node afterwards. */
int kma_graph_build(kma_heap_t h, const uint32_t *edges, uint64_t n, uint32_t threads, int free_after,
		    kma_graph_stats *st, uint32_t *keys_out, int64_t *node_off, uint32_t *link_sinks,
		    uint64_t *link_start);

/* The same build (the same kernels, instantiated for the PMA heap) on PMA
 * heap p, as the reference's driver runs tb_clTree.cl over pma.cl
 * (test/tb_clTree.c:441-446): nodes and links are bump allocations and
 * nothing is freed (a node that lost its add stays allocated; reset the
 * PMA heap to reuse it).  node_off[i] is the node's own offset from the
 * data base. */
int kma_graph_build_pma(kma_pma_t p, const uint32_t *edges, uint64_t n, uint32_t threads,
			kma_graph_stats *st, uint32_t *keys_out, int64_t *node_off, uint32_t *link_sinks,
			uint64_t *link_start);

#ifdef __cplusplus
}
#endif

#endif /* KMA_GRAPH_H */
