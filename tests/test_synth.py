"""CPU checks of the seeded synthetic stacks: determinism (seed, thread count,
frame ranges) and the value distributions the workloads specify."""
import numpy as np

import lscomp


def test_deterministic_and_thread_independent():
    dims = (3, 160, 200)  # larger than the xpcs beamstop disk (radius 60)
    for gen in (lscomp.synth_small, lscomp.synth_cssi, lscomp.synth_xpcs):
        a = gen(dims, seed=5, threads=1)
        b = gen(dims, seed=5, threads=4)
        assert np.array_equal(a, b)
        c = gen(dims, seed=6)
        assert not np.array_equal(a, c)


def test_frame_ranges_match_whole_stack():
    dims = (6, 148, 140)
    for gen in (lscomp.synth_small, lscomp.synth_cssi, lscomp.synth_xpcs):
        whole = gen(dims, seed=9).reshape(dims)
        part = gen(dims, seed=9, frames=(2, 3)).reshape(3, 148, 140)
        assert np.array_equal(whole[2:5], part)


def test_small_distribution():
    dims = (4, 256, 256)
    a = lscomp.synth_small(dims, seed=1).reshape(dims)
    hot = (a == 65535).mean()
    assert 0.0005 < hot < 0.0012           # 0.1% hot pixels (some collide)
    # Poisson(0.1) background: P(0) = 0.905 away from the spots
    assert 0.6 < (a == 0).mean() < 0.93
    assert np.median(a) == 0
    assert (a > 150).sum() > 4 * 20        # Gaussian spots present


def test_xpcs_sparse():
    dims = (8, 256, 256)
    a = lscomp.synth_xpcs(dims, seed=3).reshape(dims)
    zero = (a == 0).mean()
    assert 0.96 < zero < 0.995             # about 98% zeros
    nz = a[a > 0]
    assert (nz <= 3).mean() > 0.95         # non-zeros mostly 1-3
    # beamstop disk of radius 60 around the centre is all zeros
    assert a[:, 118:138, 118:138].max() == 0
    # frame-to-frame correlation of the speckle (AR(1) on the field): a pixel
    # lit in one frame is lit in the next about 1.8x as often as on average
    lit0, lit1 = a[:-1] > 0, a[1:] > 0
    assert (lit1 & lit0).sum() / lit0.sum() > 1.3 * lit1.mean()


def test_cssi_structure():
    dims = (2, 400, 500)
    a = lscomp.synth_cssi(dims, seed=2).reshape(dims).astype(np.float64)
    # radial falloff: centre brighter than corners; a zero beamstop near the centre
    assert a[:, 180:220, 200:300].max() > a[:, :20, :20].mean()
    assert (a == 0).any()
    assert a.max() > 400                    # rings reach hundreds+ counts
