/*
 * kma_wl_common.cuh -- device helpers shared by the workload kernels
 * (kma_workload.cu, kma_batch.cu, kma_serve.cu): the SplitMix64 PRNG, the
 * ordered offset hash, and the warp-cooperative tag fill / verify of
 * payload blocks.
 */
#ifndef KMA_WL_COMMON_CUH
#define KMA_WL_COMMON_CUH

#include <stdint.h>

namespace kma_wl {

__device__ __forceinline__ uint64_t splitmix(uint64_t &s)
{
	uint64_t z = (s += 0x9E3779B97F4A7C15ull);
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

__device__ __forceinline__ uint64_t hash_step(uint64_t h, int64_t off)
{
	return h ^ ((uint64_t)off + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2));
}

/* Tag fill of this lane's own block (p may be NULL).  Blocks start 4 bytes
 * past a 16-byte boundary (12 + slot*size), so the head words go one at a
 * time and the rest as 16-byte stores. */
__device__ __forceinline__ void coop_fill(uint32_t mask, uint32_t lane, void *p, uint32_t n, uint32_t tag)
{
	(void)mask;
	(void)lane;
	if (!p)
		return;
	uint32_t *w = (uint32_t *)p;
	uint32_t nw = n >> 2, i = 0;
	while (i < nw && ((uintptr_t)(w + i) & 15))
		w[i++] = tag;
	uint32_t nv = (nw - i) >> 2;
	uint4 *v = reinterpret_cast<uint4 *>(w + i);
	const uint4 t4 = make_uint4(tag, tag, tag, tag);
#pragma unroll 4
	for (uint32_t k = 0; k < nv; k++)
		v[k] = t4;
	for (i += nv * 4; i < nw; i++)
		w[i] = tag;
}

/* Blocks of at least this many bytes are verified by the whole warp. */
#define WL_COOP_BYTES 256u

/* This lane's share of verifying block p (nw words) cooperatively: head
 * words up to the 16-byte boundary, 16-byte vectors lane, lane+32, ...,
 * and tail words.  Nonzero if its share differs from the tag. */
__device__ __forceinline__ uint32_t verify_share(uint32_t lane, const uint32_t *p, uint32_t nw, uint32_t tag)
{
	uint32_t head = (uint32_t)((16u - ((uintptr_t)p & 15u)) & 15u) >> 2;
	head = head < nw ? head : nw;
	uint32_t nv = (nw - head) >> 2;
	uint32_t tail = nw - head - 4 * nv;
	const uint4 *v = reinterpret_cast<const uint4 *>(p + head);
	uint32_t bad = 0;
#pragma unroll 4
	for (uint32_t k = lane; k < nv; k += 32) {
		uint4 x = v[k];
		bad |= (x.x ^ tag) | (x.y ^ tag) | (x.z ^ tag) | (x.w ^ tag);
	}
	if (lane < head)
		bad |= p[lane] ^ tag;
	if (lane < tail)
		bad |= p[head + 4 * nv + lane] ^ tag;
	return bad;
}

/* Verify every lane's block (p may be NULL) against its tag; true in the
 * owner lane of a block with a word that differs.  Small blocks: each lane
 * reads its own with 16-byte loads unrolled by eight.  Blocks of
 * WL_COOP_BYTES or more: the warp reads each together, up to four vectors
 * per lane, with no synchronisation per block -- mismatches collect in a
 * per-block bit mask reduced once at the end -- so the loads of the whole
 * pass stay in flight instead of one block's at a time. */
__device__ __forceinline__ bool coop_verify(uint32_t mask, uint32_t lane, const void *p, uint32_t n,
		uint32_t tag)
{
	const uint32_t *w = (const uint32_t *)p;
	const bool big = p && n >= WL_COOP_BYTES;
	uint32_t bad = 0;
	if (p && !big) {
		uint32_t nw = n >> 2, i = 0;
		while (i < nw && ((uintptr_t)(w + i) & 15))
			bad |= w[i++] ^ tag;
		uint32_t nv = (nw - i) >> 2;
		const uint4 *v = reinterpret_cast<const uint4 *>(w + i);
#pragma unroll 8
		for (uint32_t k = 0; k < nv; k++) {
			uint4 x = v[k];
			bad |= (x.x ^ tag) | (x.y ^ tag) | (x.z ^ tag) | (x.w ^ tag);
		}
		for (i += nv * 4; i < nw; i++)
			bad |= w[i] ^ tag;
	}
	uint32_t mb = __ballot_sync(mask, big);
	uint32_t badbits = 0;
	while (mb) {
		uint32_t j = __ffs(mb) - 1;
		mb &= mb - 1;
		const uint32_t *pj = (const uint32_t *)__shfl_sync(mask, (unsigned long long)w, j);
		uint32_t nj = __shfl_sync(mask, n, j) >> 2;
		uint32_t tj = __shfl_sync(mask, tag, j);
		if (verify_share(lane, pj, nj, tj))
			badbits |= 1u << j;
	}
	badbits = __reduce_or_sync(mask, badbits);
	return bad != 0 || ((badbits >> lane) & 1u);
}

} /* namespace kma_wl */

#endif /* KMA_WL_COMMON_CUH */
