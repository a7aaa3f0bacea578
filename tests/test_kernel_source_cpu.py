"""CPU checks of fixed tables that live in the CUDA source.

The M-step sorts a Gaussian's bucket of up to eight (supervoxel, slot) positions with a
comparator network before visiting them in ascending order; a wrong comparator would change
the summation order of the M-step's statistics, so the network is read from the kernel source
here and checked to sort every input (by the 0-1 principle, all 2^8 inputs of zeros and ones
suffice).
"""
import itertools
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "..", "tgmm_b200", "csrc", "em_kernels.cu")


def _network():
    text = open(SRC).read()
    m = re.search(r"constexpr int kNet\[(\d+)\]\[2\] = \{(.*?)\};", text, re.S)
    assert m, "the M-step's comparator network is not in em_kernels.cu"
    pairs = [(int(a), int(b)) for a, b in re.findall(r"\{\s*(\d+)\s*,\s*(\d+)\s*\}", m.group(2))]
    assert len(pairs) == int(m.group(1))
    return pairs


def test_mstep_bucket_network_sorts_every_input():
    net = _network()
    assert all(0 <= a < b < 8 for a, b in net)
    for bits in itertools.product((0, 1), repeat=8):
        v = list(bits)
        for a, b in net:
            v[a], v[b] = min(v[a], v[b]), max(v[a], v[b])
        assert v == sorted(v), bits


def test_mstep_bucket_network_orders_positions_like_insertion():
    """Distinct positions with INT_MAX padding, as the kernel sorts them: the first n outputs
    are the n positions in ascending order (what the insertion sort of larger buckets gives)."""
    import random
    rng = random.Random(5)
    net = _network()
    for _ in range(2000):
        n = rng.randint(0, 8)
        pos = rng.sample(range(0, 5 * 40000), n)
        v = pos + [2**31 - 1] * (8 - n)
        for a, b in net:
            v[a], v[b] = min(v[a], v[b]), max(v[a], v[b])
        assert v[:n] == sorted(pos)
