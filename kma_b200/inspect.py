"""Heap inspector: decode a heap image into the canonical form shared with
the reference, and check heap invariants.

Canonical form (implementation-neutral, what serial replay compares):
  cls[c]       superblock attached to class c, -1 empty, -2 POISON
               (a sharded heap attaches at most one superblock per class
               under serial execution; several shards holding one is
               reported as -3)
  sb_size[s]   block size of superblock s (0 if never used)
  sb_slots[s]  slots, sb_free[s] free count (kma.cl:180 packs slots<<16|free)
  freelist     superblock indices in FIFO order, the next one handed out
               (the reference's dummy, clIndexedQueue.cl:282-289) first
  region       superblock bytes with each superblock's first 12 bytes
               masked (header fields live elsewhere here), i.e. the
               bitmaps and the word-0 residue malloc/free leave in blocks
               (kma.cl:265, kma.cl:338)
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SB_HDR = 12
FREE_MASK = 0x3FFF


@dataclass
class HeapImage:
    sb_size_log2: int
    sblocks: int
    pages: int
    nclasses: int
    cls_size: list
    cls_slots: list
    cls_raw: np.ndarray          # raw class-table words, class-major
    cls_shards: list             # words (shards) per class
    state: np.ndarray            # (sblocks,) class<<28 | slots<<14 | free
    freelist: np.ndarray | None  # FIFO order; None if the list has a cycle
    region: np.ndarray | None = None


@dataclass
class Canonical:
    cls: np.ndarray
    sb_size: np.ndarray
    sb_slots: np.ndarray
    sb_free: np.ndarray
    freelist: np.ndarray
    region: np.ndarray | None = None
    notes: list = field(default_factory=list)


def decode(img: HeapImage) -> Canonical:
    raw = np.asarray(img.cls_raw, np.int64).reshape(-1)
    cls = np.full(img.nclasses, -1, np.int64)
    base = 0
    for c in range(img.nclasses):
        col = raw[base:base + img.cls_shards[c]]
        base += img.cls_shards[c]
        nz = col[col != 0]
        if len(nz) > 1:
            cls[c] = -3
        elif len(nz) == 1:
            cls[c] = -2 if nz[0] == 1 else nz[0] - 2
    st = img.state.astype(np.uint64)
    cl = (st >> 28).astype(np.int64)
    slots = ((st >> 14) & FREE_MASK).astype(np.uint32)
    free = (st & FREE_MASK).astype(np.uint32)
    sizes = np.asarray(img.cls_size + [0] * (16 - len(img.cls_size)), np.uint32)
    size = np.where(st == 0, 0, sizes[np.clip(cl, 0, 15)]).astype(np.uint32)
    canon = Canonical(cls=cls, sb_size=size, sb_slots=slots, sb_free=free,
                      freelist=np.asarray(img.freelist if img.freelist is not None else [-1],
                                          np.int64))
    if img.freelist is None:
        canon.notes.append("free list does not terminate (cycle)")
    if img.region is not None:
        canon.region = mask_headers(img.region, img.sb_size_log2)
    return canon


IMAGE_MAGIC = b"KMAHEAP1"
IMAGE_HEADER = np.dtype([
    ("magic", "S8"), ("version", "<u4"), ("header_bytes", "<u4"),
    ("sb_log2", "<u4"), ("sblocks", "<u4"), ("pages", "<u4"), ("ring", "<u4"),
    ("nclasses", "<u4"), ("cls_lines", "<u4"), ("flist_words", "<u4"), ("err", "<u4"),
    ("free_head", "<u8"), ("free_tail", "<u8"), ("ring_avail", "<u4"), ("reserved", "<u4"),
    ("cls_shards", "<u4", (16,)),
    ("off_cls", "<u8"), ("off_state", "<u8"), ("off_home", "<u8"), ("off_flist", "<u8"),
    ("off_region", "<u8"), ("total_bytes", "<u8")])
assert IMAGE_HEADER.itemsize == 184  # struct kma_image_header (kma.h)


def image_header(buf: np.ndarray) -> dict:
    """The header of a heap image (kma_image_save) as a dict."""
    buf = np.asarray(buf, np.uint8).reshape(-1)
    if buf.nbytes < IMAGE_HEADER.itemsize:
        raise ValueError("not a heap image: shorter than its header")
    h = buf[:IMAGE_HEADER.itemsize].view(IMAGE_HEADER)[0]
    if bytes(h["magic"]) != IMAGE_MAGIC:
        raise ValueError("not a heap image: bad magic")
    d = {k: (h[k].tolist() if k == "cls_shards" else (bytes(h[k]) if k == "magic" else int(h[k])))
         for k in IMAGE_HEADER.names}
    if d["total_bytes"] > buf.nbytes:
        raise ValueError("heap image truncated")
    return d


def image_from_bytes(buf: np.ndarray, cls_size: list, cls_slots: list, region: bool = True) -> HeapImage:
    """Decode a saved heap image into the HeapImage the checkers take (the
    same content kma_snapshot reports).  cls_size / cls_slots are the size
    tables of the image's superblock size (Heap.cls_size / cls_slots)."""
    buf = np.asarray(buf, np.uint8).reshape(-1)
    h = image_header(buf)
    nsb, nw = h["sblocks"], h["flist_words"]
    cls = buf[h["off_cls"]:h["off_cls"] + 4 * h["cls_lines"]].view("<u4").copy()
    state = buf[h["off_state"]:h["off_state"] + 4 * nsb].view("<u4").copy()
    words = buf[h["off_flist"]:h["off_flist"] + 8 * nw].view("<u8")
    fl: list | None = []
    if h["ring"]:
        hd, tl = h["free_head"], h["free_tail"]
        if tl - hd > nsb:
            fl = None
        else:
            fl = [int(words[p % nw]) & 0xFFFFFFFF for p in range(hd, tl)]
    else:
        idx = h["free_head"] & 0xFFFFFFFF
        while idx != 0:
            if len(fl) >= nsb or idx > nw:
                fl = None
                break
            fl.append(idx - 1)
            idx = int(words[idx - 1]) & 0xFFFFFFFF
    reg = None
    if region:
        reg = buf[h["off_region"]:h["off_region"] + (nsb << h["sb_log2"])].copy()
    nc = h["nclasses"]
    return HeapImage(sb_size_log2=h["sb_log2"], sblocks=nsb, pages=h["pages"], nclasses=nc,
                     cls_size=list(cls_size)[:nc], cls_slots=list(cls_slots)[:nc], cls_raw=cls,
                     cls_shards=h["cls_shards"][:nc], state=state,
                     freelist=None if fl is None else np.asarray(fl, np.int64), region=reg)


def mask_headers(region: np.ndarray, sb_size_log2: int) -> np.ndarray:
    """Zero the first 12 bytes of every superblock (a copy)."""
    r = np.array(region, dtype=np.uint8, copy=True).reshape(-1, 1 << sb_size_log2)
    r[:, :SB_HDR] = 0
    return r.reshape(-1)


def bitmap_words(region: np.ndarray, sb_size_log2: int, s: int, words: int) -> np.ndarray:
    """Bitmap words 0..words-1 of superblock s (word k at u32 index SB/4-1-k)."""
    sb = 1 << sb_size_log2
    w = region[s * sb:(s + 1) * sb].view(np.uint32)
    return w[::-1][:words].copy()


def check_canonical_empty(img: HeapImage, bitmaps: np.ndarray | None = None) -> list[str]:
    """The state every heap returns to once all blocks are freed: no class
    attached in any shard, every page on the free list exactly once, every
    bitmap of a used superblock clear (from img.region, or bitmaps[s, k]
    when given)."""
    c = decode(img)
    bad = []
    if np.any(np.asarray(img.cls_raw) != 0):
        bad.append(f"class table not empty: {c.cls.tolist()}")
    fl = c.freelist
    if c.notes:
        bad += c.notes
    elif len(fl) != max(img.pages, 1):
        bad.append(f"free list holds {len(fl)} superblocks, expected {max(img.pages, 1)}")
    if len(np.unique(fl)) != len(fl):
        bad.append("free list holds a superblock twice")
    if np.any(fl >= max(img.pages, 1)):
        bad.append("free list holds a superblock beyond the pages")
    used = np.nonzero(c.sb_slots)[0]
    if np.any(c.sb_free[used] != 0):
        bad.append("a recycled superblock has a non-zero free count")
    if bitmaps is not None:
        for s in used:
            words = (int(c.sb_slots[s]) + 31) // 32
            if np.any(bitmaps[s, :words]):
                bad.append(f"superblock {s} bitmap not clear")
                break
    elif img.region is not None:
        for s in used:
            words = (int(c.sb_slots[s]) + 31) // 32
            if np.any(bitmap_words(img.region, img.sb_size_log2, int(s), words)):
                bad.append(f"superblock {s} bitmap not clear")
                break
    return bad


def check_live_blocks(img: HeapImage, off: np.ndarray, size: np.ndarray,
                      bitmaps: np.ndarray | None = None) -> dict:
    """Invariants over a set of live blocks (offsets from the first
    superblock, requested sizes): no two overlap, each lies inside the data
    area of a superblock of a class at least as large as the request, on
    that class's slot grid, 4-byte aligned, and (given bitmaps[s, k]) its
    bit is set.  Returns violation counts (all zero when the heap is sound)."""
    off = np.asarray(off, np.int64)
    size = np.asarray(size, np.int64)
    sb = 1 << img.sb_size_log2
    res = {"blocks": int(len(off)), "overlap": 0, "out_of_bounds": 0, "misaligned": 0,
           "off_grid": 0, "class_too_small": 0, "bit_clear": 0, "duplicate": 0}
    if len(off) == 0:
        return res
    order = np.argsort(off, kind="stable")
    o, z = off[order], size[order]
    res["duplicate"] = int(np.sum(o[1:] == o[:-1]))
    res["overlap"] = int(np.sum(o[:-1] + z[:-1] > o[1:]))
    res["misaligned"] = int(np.sum(off % 4 != 0))
    s = off // sb
    inb = (off >= 0) & (s < img.sblocks)
    res["out_of_bounds"] += int(np.sum(~inb))
    s = np.where(inb, s, 0)
    st = img.state[s].astype(np.int64)
    cl = st >> 28
    slots = (st >> 14) & FREE_MASK
    sizes = np.asarray(img.cls_size + [0] * (16 - len(img.cls_size)), np.int64)
    csize = sizes[np.clip(cl, 0, 15)]
    within = off - s * sb - SB_HDR
    ok_state = (st != 0) & (cl < img.nclasses)
    res["out_of_bounds"] += int(np.sum(inb & (~ok_state | (within < 0))))
    good = inb & ok_state & (within >= 0) & (csize > 0)
    slot = np.where(good, within // np.where(csize > 0, csize, 1), 0)
    res["off_grid"] = int(np.sum(good & (within % np.where(csize > 0, csize, 1) != 0)))
    res["out_of_bounds"] += int(np.sum(good & (slot >= slots)))
    res["out_of_bounds"] += int(np.sum(good & (within + size > slots * csize)))
    res["class_too_small"] = int(np.sum(good & (csize < size)))
    if bitmaps is not None:
        words = bitmaps.shape[1]
        k = np.clip(slot // 32, 0, words - 1)
        bits = (bitmaps[s, k].astype(np.int64) >> (slot % 32)) & 1
        res["bit_clear"] = int(np.sum(good & (bits == 0)))
    return res


def violations(res: dict) -> int:
    return sum(v for k, v in res.items() if k != "blocks")
