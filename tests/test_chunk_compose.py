"""The property the host-memory calls are built on, checked with the oracle on
the CPU: a stack's stream is its frame chunks' streams taken apart and put
together -- the chunks' header bytes one after the other, the zero pad to a
multiple of 4, then the chunks' payloads one after the other -- and each
chunk's own stream can be cut back out of the whole one.  (Block order is
frame-major, so a chunk of whole frames is a contiguous run of blocks.)"""
import numpy as np
import pytest

LOSSLESS = ((1, 1, 1, 1), 1.0)
LOSSY = ((3, 5, 10, 15), 0.5)


def stack(dims, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 60, size=dims).astype(np.uint16)
    a[rng.random(dims) < 0.5] = 0
    a[rng.random(dims) < 0.01] = 65535
    return a


def nblocks(dims):
    x, y, z = dims
    return x * ((y + 7) // 8) * ((z + 7) // 8)


def r4(n):
    return (n + 3) // 4 * 4


@pytest.mark.parametrize("bins,p", [LOSSLESS, LOSSY])
@pytest.mark.parametrize("dims,fpc", [((7, 9, 17), 3), ((10, 100, 130), 4), ((5, 64, 1030), 1), ((6, 13, 21), 6)])
def test_chunk_streams_compose(oracle, dims, fpc, bins, p):
    a = stack(dims, seed=sum(dims) + fpc)
    full, _ = oracle.compress(a, dims, bins, p)
    full = np.asarray(full)
    x, y, z = dims
    nb = nblocks(dims)
    headers, payloads = [], []
    for f0 in range(0, x, fpc):
        cd = (min(fpc, x - f0), y, z)
        s, _ = oracle.compress(np.ascontiguousarray(a[f0:f0 + cd[0]]), cd, bins, p)
        s = np.asarray(s)
        nb_c = nblocks(cd)
        headers.append(s[:nb_c])
        assert not s[nb_c:r4(nb_c)].any()  # each chunk's own pad is zero
        payloads.append(s[r4(nb_c):])
    composed = np.concatenate(headers + [np.zeros(r4(nb) - nb, np.uint8)] + payloads)
    assert np.array_equal(composed, full)
    # and back: every chunk's stream cut out of the whole decodes to its frames
    off = 0
    dec_full = oracle.decompress(full, dims, bins, p).reshape(dims)
    for c, f0 in enumerate(range(0, x, fpc)):
        cd = (min(fpc, x - f0), y, z)
        nb_c = nblocks(cd)
        k0 = f0 * ((y + 7) // 8) * ((z + 7) // 8)
        pay = len(payloads[c])
        cs = np.concatenate([full[k0:k0 + nb_c], np.zeros(r4(nb_c) - nb_c, np.uint8),
                             full[r4(nb) + off:r4(nb) + off + pay]])
        off += pay
        dec = oracle.decompress(cs, cd, bins, p).reshape(cd)
        assert np.array_equal(dec, dec_full[f0:f0 + cd[0]])
