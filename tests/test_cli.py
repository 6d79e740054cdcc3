"""The command-line tools lsCOMP_xpcs (uint16) and lsCOMP_cssi (uint32):
argument handling identical to the reference tools (checked on CPU against
the reference's own binaries, whose argument checks run before any CUDA call)
and, on a GPU, the printed compression ratio and the -o decoded file."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "sc25-lscomp_b200", "bin")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")

BAD_ARGS = [
    [],
    ["-i", "x", "-d", "1", "2", "0", "-b", "1", "1", "1", "1", "-p", "1"],
    ["-i", "x", "-d", "1", "2", "3", "-b", "1", "3", "2", "4", "-p", "1"],
    ["-i", "x", "-d", "1", "2", "3", "-b", "0", "1", "1", "1", "-p", "1"],
    ["-i", "x", "-d", "1", "2", "3", "-b", "1", "1", "1", "1", "-p", "1.5"],
    ["-i", "x", "-d", "1", "2", "3", "-b", "1", "1", "1", "1", "-p", "-0.1"],
    ["-i", "x", "-d", "1", "2", "3", "-b", "1", "1", "1", "1", "-q", "1"],
    ["-i", "x", "-d", "1", "2", "3", "-b", "1", "1", "1", "1", "-p"],
]


def run(path, args):
    return subprocess.run([path] + args, capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("tool", ["lsCOMP_xpcs", "lsCOMP_cssi"])
@pytest.mark.parametrize("args", BAD_ARGS)
def test_argument_errors(tool, args):
    ours = run(os.path.join(BIN, tool), args)
    assert ours.returncode == 1
    ref_path = os.path.join(REF_BIN, tool)
    if not os.path.exists(ref_path):
        pytest.skip("reference build not present")
    ref = run(ref_path, args)
    assert ours.returncode == ref.returncode
    # same messages up to the program name
    norm = lambda s, p: s.replace(p, "PROG")
    assert norm(ours.stderr, os.path.join(BIN, tool)) == norm(ref.stderr, ref_path)


def _ratio(out):
    return float(re.search(r"compression ratio: ([0-9.]+)", out).group(1))


@pytest.mark.gpu
@pytest.mark.parametrize("bins,p", [(("1", "1", "1", "1"), "1"), (("3", "5", "10", "15"), "0.5")])
def test_xpcs_tool_round_trip(tmp_path, oracle, bins, p):
    import lscomp

    dims = (8, 256, 260)  # 8 * 32 * 33 = 8448 blocks: several reference tiles
    a = lscomp.synth_small(dims, seed=3)
    src = tmp_path / "in.u16"
    a.tofile(src)
    dec = tmp_path / "dec.u16"
    args = ["-i", str(src), "-d", *map(str, dims), "-b", *bins, "-p", p, "-o", str(dec)]
    ours = run(os.path.join(BIN, "lsCOMP_xpcs"), args)
    assert ours.returncode == 0, ours.stderr
    assert "cuLSZ compression   end-to-end speed:" in ours.stdout
    got = np.fromfile(dec, dtype=np.uint16)
    b = tuple(int(v) for v in bins)
    s_o, rs_o = oracle.compress(a, dims, b, float(p))
    assert np.array_equal(got, oracle.decompress(s_o, dims, b, float(p)))
    assert abs(_ratio(ours.stdout) - a.size * 2 / rs_o) < 1e-4
    ref_path = os.path.join(REF_BIN, "lsCOMP_xpcs")
    if os.path.exists(ref_path):
        ref = run(ref_path, args[:-2])  # no -o: the reference leaves rate-0 blocks unwritten
        assert ref.returncode == 0, ref.stderr
        assert _ratio(ref.stdout) == _ratio(ours.stdout)


@pytest.mark.gpu
def test_cssi_tool_round_trip(tmp_path, oracle):
    import lscomp

    dims = (4, 120, 136)
    a = (lscomp.synth_cssi(dims, seed=5).astype(np.uint32) * 3000).reshape(dims)
    src = tmp_path / "in.u32"
    a.tofile(src)
    dec = tmp_path / "dec.u32"
    args = ["-i", str(src), "-d", *map(str, dims), "-b", "1", "1", "1", "1", "-p", "1", "-o", str(dec)]
    ours = run(os.path.join(BIN, "lsCOMP_cssi"), args)
    assert ours.returncode == 0, ours.stderr
    assert np.array_equal(np.fromfile(dec, dtype=np.uint32), a.ravel())
