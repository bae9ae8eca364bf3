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

/* Cache policy of the payload words (tag fill and verify): 0 default,
 * 1 at L2 only (.cg), 2 streaming (.cs: evict first).  Streaming both
 * measured 1-2% faster on config 2's rounds kernel than the default;
 * .cg loads alone 1.4% slower. */
#ifndef WL_PAYLOAD_LD
#define WL_PAYLOAD_LD 2
#endif
#ifndef WL_PAYLOAD_ST
#define WL_PAYLOAD_ST 2
#endif
template <class T>
__device__ __forceinline__ T pl_ld(const T *p)
{
#if WL_PAYLOAD_LD == 1
	return __ldcg(p);
#elif WL_PAYLOAD_LD == 2
	return __ldcs(p);
#else
	return *p;
#endif
}
template <class T>
__device__ __forceinline__ void pl_st(T *p, T v)
{
#if WL_PAYLOAD_ST == 1
	__stcg(p, v);
#elif WL_PAYLOAD_ST == 2
	__stcs(p, v);
#else
	*p = v;
#endif
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
		pl_st(&w[i++], tag);
	uint32_t nv = (nw - i) >> 2;
	uint4 *v = reinterpret_cast<uint4 *>(w + i);
	const uint4 t4 = make_uint4(tag, tag, tag, tag);
#pragma unroll 4
	for (uint32_t k = 0; k < nv; k++)
		pl_st(&v[k], t4);
	for (i += nv * 4; i < nw; i++)
		pl_st(&w[i], tag);
}

/* Blocks of at least this many bytes are verified by the whole warp
 * (config 2's rounds kernel: 128 and 256 measured alike, 512 2% slower). */
#ifndef WL_COOP_BYTES
#define WL_COOP_BYTES 256u
#endif

/* The share of the r-th of `width` calling lanes in verifying block p (nw
 * words) cooperatively: head words up to the 16-byte boundary, 16-byte
 * vectors r, r+width, ..., and tail words.  Nonzero if its share differs
 * from the tag. */
__device__ __forceinline__ uint32_t verify_share(uint32_t r, uint32_t width, const uint32_t *p, uint32_t nw,
		uint32_t tag)
{
	uint32_t head = (uint32_t)((16u - ((uintptr_t)p & 15u)) & 15u) >> 2;
	head = head < nw ? head : nw;
	uint32_t nv = (nw - head) >> 2;
	uint32_t tail = nw - head - 4 * nv;
	const uint4 *v = reinterpret_cast<const uint4 *>(p + head);
	uint32_t bad = 0;
#pragma unroll 4
	for (uint32_t k = r; k < nv; k += width) {
		uint4 x = pl_ld(&v[k]);
		bad |= (x.x ^ tag) | (x.y ^ tag) | (x.z ^ tag) | (x.w ^ tag);
	}
	for (uint32_t i = r; i < head; i += width)
		bad |= pl_ld(&p[i]) ^ tag;
	for (uint32_t i = r; i < tail; i += width)
		bad |= pl_ld(&p[head + 4 * nv + i]) ^ tag;
	return bad;
}

/* Vectors each lane has in flight per batch of coop_verify_rows.  With the
 * streaming payload hints, config 2's rounds kernel (64 registers)
 * measured 7.78 / 7.93 / 8.14 / 8.13 ms per launch at 3 / 2 / 1 / 4, and
 * 8.32 ms block by block (0): deeper batches cost more spills than they
 * hide latency. */
#ifndef WL_VERIFY_SLOTS
#define WL_VERIFY_SLOTS 3
#endif

/* Verify every lane's block (p may be NULL) against its tag; true in the
 * owner lane of a block with a word that differs.  Every lane of `mask`
 * calls it.
 *
 * Small blocks: the owner reads its own, 16-byte loads unrolled by eight.
 * Blocks of WL_COOP_BYTES or more: their 16-byte aligned bodies are cut
 * into rows of one vector per calling lane, rows of all big blocks laid
 * end to end in lane order; the r-th calling lane reads vector r of each
 * row.  A batch is the next
 * WL_VERIFY_SLOTS rows, whichever blocks they belong to: every lane issues
 * all the batch's loads before it compares any, so a pass over the warp's
 * blocks costs one memory round trip per batch rather than one per block
 * (a loop over blocks consumes each block's loads before it can issue the
 * next block's).  The row schedule is the same in every lane, so which
 * block a row belongs to, its base and its tag are broadcast by shuffles;
 * the owner of a big block reads its head and tail words (the few before
 * and after the aligned body) along with the small blocks. */
#if WL_VERIFY_SLOTS > 0
__device__ __forceinline__ bool coop_verify_rows(uint32_t mask, uint32_t lane, const void *p, uint32_t n,
		uint32_t tag)
{
	const uint32_t *w = (const uint32_t *)p;
	const bool big = p && n >= WL_COOP_BYTES;
	const uint32_t nw = p ? n >> 2 : 0u;
	uint32_t head = (uint32_t)((16u - ((uintptr_t)p & 15u)) & 15u) >> 2;
	head = head < nw ? head : nw;
	const uint32_t nv = (nw - head) >> 2;
	uint32_t bad = 0;
	if (p) {
		/* head words, then (small blocks) the body, then tail words */
		for (uint32_t i = 0; i < head; i++)
			bad |= pl_ld(&w[i]) ^ tag;
		if (!big) {
			const uint4 *v = reinterpret_cast<const uint4 *>(w + head);
#pragma unroll 8
			for (uint32_t k = 0; k < nv; k++) {
				uint4 x = pl_ld(&v[k]);
				bad |= (x.x ^ tag) | (x.y ^ tag) | (x.z ^ tag) | (x.w ^ tag);
			}
		}
		for (uint32_t i = head + 4 * nv; i < nw; i++)
			bad |= pl_ld(&w[i]) ^ tag;
	}
	uint32_t mb = __ballot_sync(mask, big);
	uint32_t badbits = 0;
	const uint32_t width = __popc(mask), rank = __popc(mask & ((1u << lane) - 1u));
	/* the block whose rows are being scheduled (warp-uniform) */
	const uint4 *cb = nullptr;
	uint32_t cj = 0, cnv = 0, crow = 0, crows = 0;
	while (mb || crow < crows) {
		uint4 x[WL_VERIFY_SLOTS];
		uint32_t sj[WL_VERIFY_SLOTS];
		uint32_t valid = 0;
#pragma unroll
		for (int s = 0; s < WL_VERIFY_SLOTS; s++) {
			if (crow >= crows && mb) {
				cj = __ffs(mb) - 1;
				mb &= mb - 1;
				const uint32_t *pj = (const uint32_t *)__shfl_sync(mask, (unsigned long long)w, cj);
				cnv = __shfl_sync(mask, nv, cj);
				const uint32_t hj = __shfl_sync(mask, head, cj);
				cb = reinterpret_cast<const uint4 *>(pj + hj);
				crow = 0;
				crows = (cnv + width - 1) / width;
			}
			sj[s] = cj;
			x[s] = make_uint4(0, 0, 0, 0);
			if (crow < crows) {
				const uint32_t k = crow * width + rank;
				if (k < cnv) {
					x[s] = pl_ld(&cb[k]);
					valid |= 1u << s;
				}
				crow++;
			}
		}
#pragma unroll
		for (int s = 0; s < WL_VERIFY_SLOTS; s++) {
			const uint32_t tj = __shfl_sync(mask, tag, sj[s]);
			const uint32_t d = (x[s].x ^ tj) | (x[s].y ^ tj) | (x[s].z ^ tj) | (x[s].w ^ tj);
			if (((valid >> s) & 1u) && d)
				badbits |= 1u << sj[s];
		}
	}
	badbits = __reduce_or_sync(mask, badbits);
	return bad != 0 || ((badbits >> lane) & 1u);
}
#endif

/* Verify every lane's block (p may be NULL) against its tag; true in the
 * owner lane of a block with a word that differs.  Small blocks: each lane
 * reads its own with 16-byte loads unrolled by eight.  Blocks of
 * WL_COOP_BYTES or more: the calling lanes read each together, block by
 * block (each block's loads are consumed before the next block's are
 * issued).  coop_verify's fallback when WL_VERIFY_SLOTS is 0; with the
 * streaming payload hints the row batches measured faster in both the
 * config-2 rounds kernel and the batched form (3737 vs 3633 M ops/s). */
__device__ __forceinline__ bool coop_verify_blockwise(uint32_t mask, uint32_t lane, const void *p, uint32_t n,
		uint32_t tag)
{
	const uint32_t *w = (const uint32_t *)p;
	const bool big = p && n >= WL_COOP_BYTES;
	uint32_t bad = 0;
	if (p && !big) {
		uint32_t nw = n >> 2, i = 0;
		while (i < nw && ((uintptr_t)(w + i) & 15))
			bad |= pl_ld(&w[i++]) ^ tag;
		uint32_t nv = (nw - i) >> 2;
		const uint4 *v = reinterpret_cast<const uint4 *>(w + i);
#pragma unroll 8
		for (uint32_t k = 0; k < nv; k++) {
			uint4 x = pl_ld(&v[k]);
			bad |= (x.x ^ tag) | (x.y ^ tag) | (x.z ^ tag) | (x.w ^ tag);
		}
		for (i += nv * 4; i < nw; i++)
			bad |= pl_ld(&w[i]) ^ tag;
	}
	uint32_t mb = __ballot_sync(mask, big);
	uint32_t badbits = 0;
	const uint32_t width = __popc(mask), rank = __popc(mask & ((1u << lane) - 1u));
	while (mb) {
		uint32_t j = __ffs(mb) - 1;
		mb &= mb - 1;
		const uint32_t *pj = (const uint32_t *)__shfl_sync(mask, (unsigned long long)w, j);
		uint32_t nj = __shfl_sync(mask, n, j) >> 2;
		uint32_t tj = __shfl_sync(mask, tag, j);
		if (verify_share(rank, width, pj, nj, tj))
			badbits |= 1u << j;
	}
	badbits = __reduce_or_sync(mask, badbits);
	return bad != 0 || ((badbits >> lane) & 1u);
}

__device__ __forceinline__ bool coop_verify(uint32_t mask, uint32_t lane, const void *p, uint32_t n, uint32_t tag)
{
#if WL_VERIFY_SLOTS > 0
	return coop_verify_rows(mask, lane, p, n, tag);
#else
	return coop_verify_blockwise(mask, lane, p, n, tag);
#endif
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
