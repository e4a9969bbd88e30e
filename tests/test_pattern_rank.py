"""The slot-pair pattern ranks by which a prune sorts a cluster's pruned entries (CPU test).

The packed pair kernel's source carries the rank of each of the 16 four-bit slot-pair patterns
as the nibbles of one 64-bit constant (SB_PAT_RANK in sponge_b200/csrc/sb_pair_x2.cuh), next to
the order it encodes. This checks that the constant is a permutation of 0..15 with the empty
pattern last, that it encodes the order written beside it, and restates the kernel's
pattern-of-mask mapping (a slot pair is used when either of its two slot bits is set).
"""

import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "..", "sponge_b200", "csrc", "sb_pair_x2.cuh")


def _source():
    with open(SRC) as f:
        return f.read()


def _ranks():
    m = re.search(r"#define SB_PAT_RANK (0x[0-9a-fA-F]+)ull", _source())
    assert m, "SB_PAT_RANK not found"
    v = int(m.group(1), 16)
    return [(v >> (4 * k)) & 15 for k in range(16)]


def _documented_order():
    src = _source()
    m = re.search(r"//\s+pattern:((?:\s+\d+)+)", src)
    assert m, "documented pattern order not found"
    return [int(t) for t in m.group(1).split()]


def pattern_of(mask8):
    """Bit p set when slot 2p or 2p + 1 of the entry's 8-bit mask is set."""
    return sum(1 << p for p in range(4) if (mask8 >> (2 * p)) & 3)


def test_ranks_are_a_permutation_with_empty_last():
    r = _ranks()
    assert sorted(r) == list(range(16))
    assert r[0] == 15


def test_ranks_encode_the_documented_order():
    order = _documented_order()
    assert len(order) == 15 and sorted(order) == list(range(1, 16))
    r = _ranks()
    assert [r[p] for p in order] == list(range(15))


def test_pattern_of_mask():
    assert pattern_of(0) == 0
    assert pattern_of(0b00000001) == 1 and pattern_of(0b00000010) == 1
    assert pattern_of(0b00001100) == 2
    assert pattern_of(0b11000000) == 8
    assert pattern_of(0xff) == 15
    # every mask maps to a pattern whose pairs cover exactly the mask's slots
    for m in range(256):
        p = pattern_of(m)
        cover = sum(3 << (2 * q) for q in range(4) if (p >> q) & 1)
        assert m & ~cover == 0 and all((m >> (2 * q)) & 3 for q in range(4) if (p >> q) & 1)
