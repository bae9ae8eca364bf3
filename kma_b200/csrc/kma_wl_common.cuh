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

/* Position of the (k+1)-th set bit of m; requires k < popc(m). */
__device__ __forceinline__ uint32_t nth_bit(uint32_t m, uint32_t k)
{
	uint32_t pos = 0;
#pragma unroll
	for (uint32_t s = 16; s; s >>= 1) {
		uint32_t lo = __popc(m & ((1u << s) - 1u));
		if (k >= lo) {
			k -= lo;
			m >>= s;
			pos += s;
		}
	}
	return pos;
}

/* Packed numbering of a full warp's work bits: the set bits of every
 * lane's `bits`, in lane order and within a lane in increasing bit index,
 * are numbered 0..total-1 by a warp prefix sum, so that pass k serves
 * numbers 32k..32k+31 with lane l taking number 32k+l.  Used for the
 * frees of a round: one pass per set bit of the busiest lane would leave
 * most lanes idle through about twice as many passes, each a chain of
 * dependent round trips (table load, payload loads, free atomics). */
struct warp_pack {
	uint32_t bits, excl, incl, total;
};

/* Every lane of the warp calls it. */
__device__ __forceinline__ warp_pack warp_pack_init(uint32_t lane, uint32_t bits)
{
	warp_pack wp;
	wp.bits = bits;
	const uint32_t c = __popc(bits);
	uint32_t incl = c;
#pragma unroll
	for (uint32_t o = 1; o < 32; o <<= 1) {
		uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o)
			incl += v;
	}
	wp.incl = incl;
	wp.excl = incl - c;
	wp.total = __shfl_sync(0xffffffffu, incl, 31);
	return wp;
}

/* Lane `lane`'s number in the pass starting at `base` (a multiple of 32
 * below total): true with the lane that owns it and its bit index, or
 * false (owner = lane) when the pass has no number for this lane.  Every
 * lane of the warp calls it. */
__device__ __forceinline__ bool warp_pack_slot(const warp_pack &wp, uint32_t lane, uint32_t base, uint32_t &owner,
		uint32_t &bit)
{
	const uint32_t full = 0xffffffffu;
	/* lanes owning numbers in this pass, and the pass slot of each one's
	 * first number (distinct slots, increasing with the lane) */
	const bool in = wp.incl > wp.excl && wp.excl < base + 32 && wp.incl > base;
	const uint32_t lanes = __ballot_sync(full, in);
	const uint32_t starts = __reduce_or_sync(full, in ? 1u << (wp.excl > base ? wp.excl - base : 0u) : 0u);
	const uint32_t s = base + lane;
	const bool mine = s < wp.total;
	owner = mine ? nth_bit(lanes, __popc(starts & (full >> (31 - lane))) - 1) : lane;
	const uint32_t o_excl = __shfl_sync(full, wp.excl, owner);
	const uint32_t o_bits = __shfl_sync(full, wp.bits, owner);
	bit = mine ? nth_bit(o_bits, s - o_excl) : 0u;
	return mine;
}

} /* namespace kma_wl */

#endif /* KMA_WL_COMMON_CUH */
