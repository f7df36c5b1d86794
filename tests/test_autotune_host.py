"""Host logic of the autotuner (``shapefromcaustics_b200/autotune.py``) on the CPU: the
candidate list and the rule that picks a winner from the measured times."""
from shapefromcaustics_b200 import autotune as AT

# the library defaults of pds_config (include/pds_b200.h; min_blocks 0: the library's choice
# per direction)
DEFAULT = dict(tile=64, chunk=2048, class_bits=5, walk=3, min_blocks=0, coop_radius=-1)


def test_first_candidate_is_the_library_default_and_all_are_valid():
    assert AT.CANDIDATES[0] == DEFAULT == AT.DEFAULT
    keys = {tuple(sorted(c.items())) for c in AT.CANDIDATES}
    assert len(keys) == len(AT.CANDIDATES) == 38
    assert {c["chunk"] for c in AT.CANDIDATES} == {1024, 2048, 4096}
    for c in AT.CANDIDATES:
        assert c["tile"] in (16, 32, 64)
        assert c["chunk"] % 256 == 0
        assert 1 <= c["class_bits"] <= 6
        assert c["walk"] in (1, 2, 3, 4)
        assert c["min_blocks"] == 0 or 2 <= c["min_blocks"] <= 4
        assert c["coop_radius"] == -1 or c["coop_radius"] >= 1


def test_default_kept_within_the_margin():
    a, b, c = dict(x=0), dict(x=1), dict(x=2)
    assert AT.pick([(a, 10.0), (b, 9.9), (c, 9.85)], margin=0.02) is a


def test_fastest_beyond_the_margin_wins():
    a, b, c, d = dict(x=0), dict(x=1), dict(x=2), dict(x=3)
    assert AT.pick([(a, 10.0), (b, 9.5), (c, 9.0), (d, 9.7)], margin=0.02) is c
    # a candidate faster than the default but not beyond the margin never displaces one that is
    assert AT.pick([(a, 10.0), (b, 9.0), (c, 9.9)], margin=0.02) is b


def test_empty_and_single():
    assert AT.pick([]) is None
    a = dict(x=0)
    assert AT.pick([(a, 3.0)]) is a


def test_signature_buckets_photon_count_and_sizes():
    s1 = AT.signature([(1000, (1, 64, 64)), (3000, (1, 128, 128))], 20)
    s2 = AT.signature([(2500, (1, 128, 128)), (1200, (1, 64, 64))], 20)
    assert s1 == s2  # same log2 bucket, same set of sizes, order-free
    assert AT.signature([(1000, (1, 64, 64))], 20) != AT.signature([(1000, (1, 64, 64))], 10)
    assert AT.signature([(1 << 20, (1, 64, 64))], 20) != AT.signature([(1 << 22, (1, 64, 64))], 20)
