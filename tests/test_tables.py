"""Size-class tables (kma.cl:55-148): the product's C ABI, the oracle port
and the reference build against the committed golden tables."""
import json
import os

import numpy as np
import pytest

import kma_b200
from oracle import oracle

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "tables.json")))
LOG2S = (12, 14, 16)


def expand(trans, sb):
    out = np.zeros(sb + 1, np.int32)
    for (n, c), nxt in zip(trans, trans[1:] + [[sb + 1, None]]):
        out[n:nxt[0]] = c
    return out


def test_golden_matches_reference_known_values():
    # the values the reference produces, kma.cl:55-113 at 4 KiB
    g = GOLDEN["12"]
    assert g["size_by_sbid"] == [4, 8, 16, 32, 64, 124, 252, 508, 1020, 2040, 4080]
    assert g["slots_by_size"] == [989, 502, 253, 127, 63, 32, 16, 8, 4, 2, 1]
    assert GOLDEN["14"]["size_by_sbid"][-1] == (1 << 14) - 16
    assert GOLDEN["16"]["slots_by_size"][0] == 15869


@pytest.mark.parametrize("log2", LOG2S)
def test_product_tables(log2):
    g = GOLDEN[str(log2)]
    nb = log2 - 1
    assert [kma_b200.size_by_sbid(log2, i) for i in range(nb)] == g["size_by_sbid"]
    assert [kma_b200.slots_by_size(log2, s) for s in g["size_by_sbid"]] == g["slots_by_size"]
    # sbid == nclasses divides by zero in the reference; the ABI returns 0
    assert kma_b200.size_by_sbid(log2, nb) == 0
    assert kma_b200.size_by_sbid(log2, -1) == 0
    sb = 1 << log2
    want = expand(g["sbid_transitions"], sb)
    got = np.array([kma_b200.sbid_by_size(log2, n) for n in range(sb + 1)], np.int32)
    assert np.array_equal(got, want)
    assert kma_b200.sbid_by_size(log2, 1 << 40) == -1


@pytest.mark.parametrize("log2", LOG2S)
def test_port_tables(log2):
    g = GOLDEN[str(log2)]
    sizes, slots, sbid = oracle.port_tables(log2)
    assert sizes == g["size_by_sbid"] and slots == g["slots_by_size"]
    assert np.array_equal(sbid, expand(g["sbid_transitions"], 1 << log2))


@pytest.mark.parametrize("log2", LOG2S)
def test_reference_build_reproduces_golden(log2):
    if not oracle.ref_available(log2):
        pytest.skip("reference build not present")
    g = GOLDEN[str(log2)]
    sizes, slots, sbid = oracle.ref_tables(log2)
    assert sizes == g["size_by_sbid"] and slots == g["slots_by_size"]
    assert np.array_equal(sbid, expand(g["sbid_transitions"], 1 << log2))
