"""Golden vectors from the reference's own CUDA build (tests/golden/*.npz,
made by tests/golden/make_golden.py on a GPU): the oracle must reproduce every
stream byte for byte, the size the reference reports and its decode; on a
GPU the B200 codec must reproduce them too."""
import glob
import os

import numpy as np
import pytest

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "*.npz")))


def load(path):
    z = np.load(path)
    t = str(z["dtype"])
    return (t, tuple(int(v) for v in z["dims"]), tuple(int(v) for v in z["bins"]), float(z["p"]), z["input"],
            z["stream"], int(z["ref_size"]), z["decode"])


def test_fixtures_present():
    assert len(GOLDEN) >= 9


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_reference_build(oracle, path):
    t, dims, bins, p, a, stream, ref_size, dec = load(path)
    dt = np.uint16 if t == "u16" else np.uint32
    s, rs = oracle.compress(a.reshape(dims), dims, bins, p, dtype=dt)
    assert np.array_equal(s, stream)
    assert rs == ref_size
    # the reference decoded into a zeroed buffer: rate-0 blocks read as zeros
    assert np.array_equal(oracle.decompress(stream, dims, bins, p, dtype=dt), dec)


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_cuda_matches_reference_build(path):
    torch = pytest.importorskip("torch")
    import lscomp

    t, dims, bins, p, a, stream, ref_size, dec = load(path)
    view, itype, esz = (np.int16, torch.int16, 2) if t == "u16" else (np.int32, torch.int32, 4)
    ws = lscomp.Workspace(0)
    d_in = torch.from_numpy(a.view(view)).cuda()
    out = torch.zeros(lscomp.max_stream_bytes(dims, esz), dtype=torch.uint8, device="cuda")
    sl, rs = lscomp.compress_into(ws, d_in, dims, bins, p, out)
    assert sl == stream.size
    assert np.array_equal(out[:sl].cpu().numpy(), stream)
    d = torch.empty(a.size, dtype=itype, device="cuda")
    lscomp.decompress_into(ws, out, sl, dims, bins, p, d)
    assert np.array_equal(d.cpu().numpy().view(dec.dtype), dec)
