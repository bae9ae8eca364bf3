"""The heap inspector's checkers, on images built from the oracle (the
mistakes are planted in oracle-side data, on the CPU)."""
import numpy as np

from kma_b200 import inspect as ins
from oracle import oracle
from opstream import make_stream


def image_from_port(p, sblocks, log2, ops, out):
    d = p.decode()
    sizes = oracle.port_tables(log2)[0]
    st = np.zeros(sblocks, np.uint32)
    for s in range(sblocks):
        if d["sb_slots"][s]:
            c = sizes.index(int(d["sb_size"][s]))
            st[s] = (c << 28) | (int(d["sb_slots"][s]) << 14) | int(d["sb_free"][s])
    cls = np.zeros((1, 16), np.uint32)
    for c, v in enumerate(d["cls"]):
        cls[0, c] = 0 if v == -1 else 1 if v == -2 else v + 2
    img = ins.HeapImage(log2, sblocks, sblocks - 1, log2 - 1, sizes,
                        oracle.port_tables(log2)[1], cls.reshape(-1)[: log2 - 1], [1] * (log2 - 1), st,
                        d["freelist"].copy(), p.region())
    return img, d


def live_set(ops, out):
    freed = {int(a) for k, a in ops if k == 1 and a >= 0}
    idx = [i for i, (k, a) in enumerate(ops) if k == 0 and out[i] >= 0 and i not in freed]
    return out[idx], ops[idx, 1]


def bitmaps_of(img):
    words = (img.cls_slots[0] + 31) // 32
    return np.stack([ins.bitmap_words(img.region, img.sb_size_log2, s, words)
                     for s in range(img.sblocks)])


def test_clean_live_set_has_no_violations():
    ops = make_stream(5, 1200, 12)
    with oracle.Port(64, 12) as p:
        out = p.replay(ops)
        img, _ = image_from_port(p, 64, 12, ops, out)
    off, size = live_set(ops, out)
    res = ins.check_live_blocks(img, off, size, bitmaps_of(img))
    assert res["blocks"] > 50 and ins.violations(res) == 0, res


def test_planted_faults_are_caught():
    ops = make_stream(6, 1200, 12)
    with oracle.Port(64, 12) as p:
        out = p.replay(ops)
        img, _ = image_from_port(p, 64, 12, ops, out)
    off, size = live_set(ops, out)
    bm = bitmaps_of(img)
    o2 = off.copy()
    o2[1] = o2[0] + 4  # overlaps block 0, off its slot grid
    r = ins.check_live_blocks(img, o2, size, bm)
    assert r["overlap"] >= 1 and r["off_grid"] >= 1
    s2 = size.copy()
    s2[0] = 5000  # request larger than any class
    assert ins.check_live_blocks(img, off, s2, bm)["class_too_small"] >= 1
    o3 = off.copy()
    o3[0] = 64 * 4096 + 12  # past the last superblock
    assert ins.check_live_blocks(img, o3, size, bm)["out_of_bounds"] >= 1
    bm2 = bm.copy()
    bm2[:] = 0  # every bit cleared
    assert ins.check_live_blocks(img, off, size, bm2)["bit_clear"] == len(off)


def test_canonical_empty_after_drain_and_not_before():
    from opstream import drain_stream
    ops = make_stream(8, 800, 12)
    with oracle.Port(40, 12) as p:
        out = p.replay(ops)
        img, _ = image_from_port(p, 40, 12, ops, out)
        assert ins.check_canonical_empty(img)  # blocks still live
    full = drain_stream(ops)
    with oracle.Port(40, 12) as p:
        out = p.replay(full)
        img, _ = image_from_port(p, 40, 12, full, out)
        assert ins.check_canonical_empty(img) == []


def encode_image(img, ring):
    """A heap image (the kma_image_save layout) of an oracle-built state,
    with the free list as ring slots or as Michael-Scott queue links."""
    al = lambda x: (x + 255) & ~255
    nsb = img.sblocks
    nw = img.pages if ring else nsb
    h = np.zeros(1, ins.IMAGE_HEADER)
    h["magic"], h["version"], h["header_bytes"] = ins.IMAGE_MAGIC, 1, ins.IMAGE_HEADER.itemsize
    h["sb_log2"], h["sblocks"], h["pages"], h["ring"] = img.sb_size_log2, nsb, img.pages, int(ring)
    h["nclasses"], h["cls_lines"], h["flist_words"] = img.nclasses, len(img.cls_raw), nw
    shards = np.zeros(16, np.uint32)
    shards[:img.nclasses] = img.cls_shards
    h["cls_shards"] = shards
    fl = np.zeros(nw, np.uint64)
    order = [int(x) for x in img.freelist]
    if ring:
        head = 5  # tickets need not start at 0: slots are taken modulo the ring size
        for k, s in enumerate(order):
            p = head + k
            fl[p % nw] = ((p + 1) << 32) | s
        h["free_head"], h["free_tail"] = head, head + len(order)
    else:
        for a, b in zip(order, order[1:]):
            fl[a] = (7 << 32) | (b + 1)
        h["free_head"], h["free_tail"] = (3 << 32) | (order[0] + 1), (9 << 32) | (order[-1] + 1)
    o = al(ins.IMAGE_HEADER.itemsize)
    h["off_cls"] = o; o = al(o + 4 * len(img.cls_raw))
    h["off_state"] = o; o = al(o + 4 * nsb)
    h["off_home"] = o; o = al(o + 2 * nsb)
    h["off_flist"] = o; o = al(o + 8 * nw)
    h["off_region"] = o; o += len(img.region)
    h["total_bytes"] = o
    buf = np.zeros(o, np.uint8)
    buf[:ins.IMAGE_HEADER.itemsize] = h.view(np.uint8)
    put = lambda off, a: buf.__setitem__(slice(off, off + a.nbytes), a.view(np.uint8))
    put(int(h["off_cls"][0]), np.asarray(img.cls_raw, "<u4"))
    put(int(h["off_state"][0]), np.asarray(img.state, "<u4"))
    put(int(h["off_flist"][0]), fl.astype("<u8"))
    put(int(h["off_region"][0]), np.asarray(img.region, np.uint8))
    return buf


def test_image_bytes_decode_to_the_oracle_state():
    ops = make_stream(9, 900, 12)
    with oracle.Port(48, 12) as p:
        out = p.replay(ops)
        img, _ = image_from_port(p, 48, 12, ops, out)
    want = ins.decode(img)
    for ring in (True, False):
        buf = encode_image(img, ring)
        got = ins.decode(ins.image_from_bytes(buf, img.cls_size, img.cls_slots))
        for f in ("cls", "sb_size", "sb_slots", "sb_free", "freelist", "region"):
            assert np.array_equal(getattr(want, f), getattr(got, f)), (ring, f)
    import pytest
    with pytest.raises(ValueError):
        ins.image_header(buf[:-1])
    bad = buf.copy()
    bad[0] ^= 1
    with pytest.raises(ValueError):
        ins.image_header(bad)
