"""The multiply-high division that the face and cell kernels use to split a
flat face or cell index into grid coordinates (FastDiv, kernels.cuh), on the
device, against numpy's floor division: every divisor up to 1100, random
divisors up to 2^32 - 1 and the extremes, each over the numerators that
border its multiples and random ones up to 2^32 - 1."""
import numpy as np
import pytest

from echo_gpu.lib import unit_fastdiv

pytestmark = pytest.mark.gpu


def test_fastdiv_matches_floor_division():
    rng = np.random.default_rng(5)
    d = np.concatenate([np.arange(1, 1101), rng.integers(1, 2**32, 300, dtype=np.uint64),
                        [2**31 - 1, 2**31, 2**31 + 1, 2**32 - 1]]).astype(np.uint32)
    n = np.concatenate([np.arange(0, 3000), rng.integers(0, 2**32, 3000, dtype=np.uint64),
                        [2**32 - 1, 2**32 - 2, 2**31, 2**31 - 1]]).astype(np.uint32)
    for exact in (False, True):
        q = unit_fastdiv(d, n, exact=exact)
        ref = n[None, :].astype(np.uint64) // d[:, None].astype(np.uint64)
        assert np.array_equal(q.astype(np.uint64), ref)
    # numerators at the multiples of each small divisor and one below them
    dd = np.arange(1, 257, dtype=np.uint32)
    k = np.arange(0, 2**32, 2**32 // 4096, dtype=np.uint64)
    nn = np.unique(np.concatenate([(k // 7) * 7, (k // 7) * 7 - 1, (k // 97) * 97, (k // 97) * 97 - 1]) % 2**32
                   ).astype(np.uint32)
    q = unit_fastdiv(dd, nn)
    assert np.array_equal(q.astype(np.uint64), nn[None, :].astype(np.uint64) // dd[:, None].astype(np.uint64))
