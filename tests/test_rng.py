"""The transport's Philox4x32-10 (nebula_b200/csrc/device/rng.cuh) against the
published known-answer vectors of Salmon, Moraes, Dror and Shaw (SC'11,
Random123's kat_vectors for philox4x32_10), and against an independent
restatement of the algorithm on random counters and keys.  Host evaluation of
the same source the kernels compile (the 32x32 high product is exact on both
sides), so it runs on the CPU."""
import ctypes as C

import numpy as np

import nebula_b200 as nb

KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff), (0xffffffff, 0xffffffff),
     (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


def _philox(counter, key):
    out = (C.c_uint32 * 4)()
    ctr = (C.c_uint32 * 4)(*counter)
    k = (C.c_uint32 * 2)(*key)
    assert nb.lib().nbl_debug_philox(ctr, k, out) == 0
    return tuple(out)


def _restated(counter, key):
    # ten rounds: two 32x32->64 products, Weyl key bumps (Salmon et al. 2011)
    c, k = list(counter), list(key)
    for _ in range(10):
        p0, p1 = 0xD2511F53 * c[0], 0xCD9E8D57 * c[2]
        c = [(p1 >> 32) ^ c[1] ^ k[0], p1 & 0xffffffff, (p0 >> 32) ^ c[3] ^ k[1], p0 & 0xffffffff]
        k = [(k[0] + 0x9E3779B9) & 0xffffffff, (k[1] + 0xBB67AE85) & 0xffffffff]
    return tuple(c)


def test_published_known_answers():
    for counter, key, expect in KAT:
        assert _philox(counter, key) == expect
        assert _restated(counter, key) == expect


def test_random_counters_and_keys():
    rng = np.random.default_rng(5)
    for _ in range(500):
        counter = tuple(int(x) for x in rng.integers(0, 2**32, 4, dtype=np.uint64))
        key = tuple(int(x) for x in rng.integers(0, 2**32, 2, dtype=np.uint64))
        assert _philox(counter, key) == _restated(counter, key)
