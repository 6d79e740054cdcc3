"""CPU tests of the oracle (oracle/lscomp_oracle.c): hand-derived known-answer
blocks for every branch of the stream format, agreement with the independent
pure-Python restatement (tests/pyref.py), and codec properties."""
import numpy as np
import pytest

import pyref

LOSSLESS = ((1, 1, 1, 1), 1.0)
LOSSY = ((3, 5, 10, 15), 0.5)


def test_pool_threshold(oracle):
    # (float)k/64 > p  (cuLSZ_kernel.cu:920-921): smallest pooling zero count
    assert oracle.pool_min_zeros(1.0) == 65      # lossless mode never pools
    assert oracle.pool_min_zeros(0.5) == 33
    assert oracle.pool_min_zeros(0.3) == 20
    assert oracle.pool_min_zeros(0.8) == 52
    assert oracle.pool_min_zeros(0.0) == 1
    assert oracle.pool_min_zeros(-0.5) == 0
    assert oracle.pool_min_zeros(float("nan")) == 65


def test_kat_lossless_constant_block(oracle):
    # one 8x8 block of 5s: lossless bins -> choice 3 (all bin counts equal),
    # rate 3, planes 0 and 2 all ones, plane 1 all zeros
    a = np.full((1, 8, 8), 5, dtype=np.uint16)
    s, ref_size = oracle.compress(a, (1, 8, 8), *LOSSLESS)
    assert s[0] == 0x63
    assert list(s[1:4]) == [0, 0, 0]
    assert list(s[4:]) == [0xFF] * 8 + [0x00] * 8 + [0xFF] * 8
    # single reference tile: the reference reports nb (its total is never stored)
    assert ref_size == 1


def test_kat_zero_block(oracle):
    a = np.zeros((1, 8, 8), dtype=np.uint16)
    s, _ = oracle.compress(a, (1, 8, 8), *LOSSLESS)
    assert list(s) == [0x60, 0, 0, 0]
    # lossy, p = 0.5: 64 zeros pool; all bin counts 64 -> choice 3; rate 0
    s, _ = oracle.compress(a, (1, 8, 8), *LOSSY)
    assert list(s) == [0xE0, 0, 0, 0]


def test_kat_hot_pixel_rate16(oracle):
    a = np.zeros((1, 8, 8), dtype=np.uint16)
    a[0, 3, 6] = 65535
    s, _ = oracle.compress(a, (1, 8, 8), *LOSSLESS)
    assert s[0] == 0x70  # choice 3, rate 16
    pay = s[4:]
    assert len(pay) == 16 * 8
    for i in range(16):
        plane = pay[8 * i: 8 * i + 8]
        # row 3 carries the bit of column 6 at bit position 7-6 = 1
        assert list(plane) == [0, 0, 0, 0x02, 0, 0, 0, 0]


def test_kat_pooled_block(oracle):
    # p = 0.0 pools any block with a zero; pair means (a+b)//2 per row pair
    a = np.zeros((1, 8, 8), dtype=np.uint16)
    a[0, 0, 0], a[0, 0, 1] = 7, 0    # pooled value 0 -> 3
    a[0, 7, 6], a[0, 7, 7] = 2, 3    # pooled value 31 -> 2
    s, _ = oracle.compress(a, (1, 8, 8), (1, 1, 1, 1), 0.0)
    assert s[0] == 0x80 | 0x60 | 2
    pay = s[4:]
    assert len(pay) == 2 * 4
    # plane 0: value 0 (3 -> bit 1) in byte 0 bit 7; value 31 (2 -> bit 0) -> 0
    assert list(pay[0:4]) == [0x80, 0, 0, 0]
    # plane 1: value 0 bit 1 = 1 -> byte 0 bit 7; value 31 bit 1 = 1 -> byte 3 bit 0
    assert list(pay[4:8]) == [0x80, 0, 0, 0x01]


def test_kat_bin_choice(oracle):
    # bins 3 5 10 15: the smallest value >= 3 decides the bin
    for val, choice in ((4, 0), (7, 1), (12, 2), (20, 3), (2, 3)):
        a = np.full((1, 8, 8), 1, dtype=np.uint16)
        a[0, 2, 2] = val
        s, _ = oracle.compress(a, (1, 8, 8), (3, 5, 10, 15), 1.0)
        assert (s[0] >> 5) & 3 == choice, (val, s[0])
        bin_ = (3, 5, 10, 15)[choice]
        assert s[0] & 31 == (val // bin_).bit_length()


def test_kat_edge_block_padding(oracle):
    # 1 x 5 x 3: one block, 15 real values, 49 padding zeros that count as zeros
    a = np.arange(1, 16, dtype=np.uint16).reshape(1, 5, 3)
    s, _ = oracle.compress(a, (1, 5, 3), (1, 1, 1, 1), 0.7)  # 49 zeros / 64 > 0.7 -> pooled
    assert s[0] >> 7 == 1
    d = oracle.decompress(s, (1, 5, 3), (1, 1, 1, 1), 0.7)
    assert d.shape == (15,)


@pytest.mark.parametrize("dims", [(1, 8, 8), (2, 13, 21), (3, 9, 17), (1, 1, 1), (2, 16, 40), (1, 24, 5)])
@pytest.mark.parametrize("bins,p", [LOSSLESS, LOSSY, ((5, 5, 5, 5), 0.3), ((2, 7, 7, 30), 0.8),
                                    ((9, 4, 12, 3), 0.5), ((1, 1, 1, 1), 0.0)])
def test_oracle_matches_pyref(oracle, dims, bins, p):
    rng = np.random.default_rng(hash((dims, bins, p)) & 0xffffffff)
    a = rng.integers(0, 40, size=dims, dtype=np.uint16)
    a[rng.random(dims) < 0.5] = 0
    a[rng.random(dims) < 0.02] = 65535
    s_py, rs_py = pyref.compress(a, bins, p)
    s_c, rs_c = oracle.compress(a, dims, bins, p)
    assert bytes(s_c) == s_py
    nb = a.shape[0] * ((a.shape[1] + 7) // 8) * ((a.shape[2] + 7) // 8)
    # the reference reports payload + nb except for one tile (nb <= 1024): nb
    assert rs_c == (rs_py if nb > 1024 else nb)
    d_c = oracle.decompress(s_c, dims, bins, p).reshape(dims)
    d_py = pyref.decompress(s_py, dims, bins)
    assert np.array_equal(d_c, d_py)


def test_lossless_roundtrip_and_lossy_bounds(oracle):
    rng = np.random.default_rng(7)
    dims = (4, 37, 53)
    a = rng.poisson(3.0, size=dims).astype(np.uint16)
    a[:, 10:20, 10:30] = 0
    a[0, 5, 5] = 65535
    s, _ = oracle.compress(a, dims, *LOSSLESS)
    assert np.array_equal(oracle.decompress(s, dims, *LOSSLESS).reshape(dims), a)
    bins, p = LOSSY
    s, _ = oracle.compress(a, dims, bins, p)
    d = oracle.decompress(s, dims, bins, p).reshape(dims).astype(np.int64)
    hdr = s[: 4 * ((dims[1] + 7) // 8) * ((dims[2] + 7) // 8)]
    # plain blocks: 0 <= v - v' <= bin - 1
    x, y, z = dims
    byb, bzb = (y + 7) // 8, (z + 7) // 8
    for k, hb in enumerate(hdr):
        if hb >> 7:
            continue
        bx, rem = divmod(k, byb * bzb)
        by, bz = divmod(rem, bzb)
        blk = a[bx, by * 8: by * 8 + 8, bz * 8: bz * 8 + 8].astype(np.int64)
        dd = d[bx, by * 8: by * 8 + 8, bz * 8: bz * 8 + 8]
        err = blk - dd
        assert err.min() >= 0 and err.max() <= bins[(hb >> 5) & 3] - 1


def test_multi_tile_reported_size(oracle):
    # more than one 1024-block reference tile: reported size = payload + nb
    dims = (8, 128, 96)  # 8 * 16 * 12 = 1536 blocks
    rng = np.random.default_rng(3)
    a = rng.integers(0, 300, size=dims, dtype=np.uint16)
    s, rs = oracle.compress(a, dims, *LOSSLESS)
    nb = 8 * 16 * 12
    r = (nb + 3) // 4 * 4
    assert rs == len(s) - r + nb


def test_thread_count_invariance(oracle):
    rng = np.random.default_rng(11)
    dims = (8, 64, 72)
    a = rng.poisson(2.0, size=dims).astype(np.uint16)
    s1, _ = oracle.compress(a, dims, *LOSSY, threads=1)
    s4, _ = oracle.compress(a, dims, *LOSSY, threads=4)
    assert np.array_equal(s1, s4)


def test_uint32_wrap_and_rate32(oracle):
    # uint32 twin (cuLSZ_kernel.cu:4-460): pair sums wrap mod 2^32; a quotient
    # >= 2^31 gives rate 32, whose bit 5 lands in the bin field
    a = np.zeros((1, 8, 8), dtype=np.uint32)
    a[0, 0, 0] = 0xFFFFFFFF
    s, _ = oracle.compress(a, (1, 8, 8), (1, 1, 1, 1), 1.0, dtype=np.uint32)
    assert s[0] == (0x60 | 32) & 0xFF  # 0x60: rate field 0, bins 3
    assert len(s) == 4 + 32 * 8  # the tile still reserves 32 planes
    b = np.full((1, 8, 8), 0x80000001, dtype=np.uint32)
    b[0, :, 1::2] = 0x80000001
    s2, _ = oracle.compress(b, (1, 8, 8), (2, 2, 2, 2), 1.0, dtype=np.uint32)
    assert s2[0] & 31 == 31
