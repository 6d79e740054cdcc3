"""GPU parity at the benchmark's full sizes: the CSSI-like stack 600 x 1813 x
1558 and the XPCS-like stack 512 x 1024 x 1024 (uint16, seeded synthetic
data), compressed and decompressed by this library (C ABI) and by the
reference's own CUDA build (its host API, lsCOMP/src/cuLSZ_entry.cu:93-166,
on pre-zeroed buffers) on the same device.

Checked per mode: the stream byte for byte over [0, stream length) with the
reference writing nothing past it, the reported size, the decode against the
reference's decode (and the input, lossless), and for lossy modes the bin
bound of every plain block, 0 <= v - v' <= bin - 1 (pooled blocks have no
bin bound in the reference's format)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

MODES = [((1, 1, 1, 1), 1.0), ((3, 5, 10, 15), 0.5), ((5, 10, 15, 15), 0.5), ((10, 10, 15, 15), 0.5)]
STACKS = [("cssi", (600, 1813, 1558), 2), ("xpcs", (512, 1024, 1024), 1)]


@pytest.fixture(scope="module")
def lz():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lscomp

    lscomp.load_library()
    return lscomp


@pytest.fixture(scope="module")
def ref():
    from oracle import RefLib

    return RefLib()


def bin_bound_ok(a, d, stream, dims, bins):
    """Every plain (not pooled) block's reconstruction error lies in
    [0, bin[choice] - 1]; computed on the GPU block by block."""
    x, y, z = dims
    byb, bzb = (y + 7) // 8, (z + 7) // 8
    nb = x * byb * bzb
    hdr = stream[:nb].to(torch.int32)
    binv = torch.tensor(bins, dtype=torch.int32, device="cuda")[(hdr >> 5) & 3]
    plain = (hdr & 0x80) == 0
    ok = True
    for f0 in range(0, x, 64):  # frames in slices: bounded temporaries
        f1 = min(x, f0 + 64)
        e = a[f0:f1].to(torch.int32) - d[f0:f1].to(torch.int32)
        e = torch.nn.functional.pad(e, (0, 8 * bzb - z, 0, 8 * byb - y))
        e = e.view(f1 - f0, byb, 8, bzb, 8).permute(0, 1, 3, 2, 4).reshape(-1, 64)
        k0, k1 = f0 * byb * bzb, f1 * byb * bzb
        emin, emax = e.min(dim=1).values, e.max(dim=1).values
        sel = plain[k0:k1]
        ok = ok and bool(((emin >= 0) & (emax <= binv[k0:k1] - 1))[sel].all())
    return ok


@pytest.mark.parametrize("kind,dims,seed", STACKS, ids=[s[0] for s in STACKS])
def test_full_size_vs_reference_build(lz, ref, kind, dims, seed):
    ws = lz.Workspace(0)
    a = getattr(lz, f"synth_{kind}")(dims, seed=seed)
    d_in = torch.from_numpy(a.view(np.int16)).cuda()
    del a
    cap = lz.max_stream_bytes(dims)
    ours = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    theirs = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    dec = torch.empty_like(d_in)
    dref = torch.empty_like(d_in)
    for bins, p in MODES:
        ours.fill_(0xAB)  # every byte of the stream must be written
        sl, rs = lz.compress_into(ws, d_in, dims, bins, p, ours)
        theirs.zero_()
        rs_ref = ref.compress(d_in.data_ptr(), theirs.data_ptr(), dims, bins, p)
        torch.cuda.synchronize()
        assert rs == rs_ref, (bins, p)
        assert torch.equal(ours[:sl], theirs[:sl]), (bins, p)
        assert int(theirs[sl:].count_nonzero()) == 0, (bins, p)
        dec.fill_(-1)
        lz.decompress_into(ws, ours, sl, dims, bins, p, dec)
        dref.zero_()
        ref.decompress(dref.data_ptr(), theirs.data_ptr(), rs_ref, dims, bins, p)
        torch.cuda.synchronize()
        assert torch.equal(dec, dref), (bins, p)
        if bins == (1, 1, 1, 1):
            assert torch.equal(dec, d_in)
        else:
            ai = d_in.view(dims).to(torch.int32) & 0xFFFF
            di = dec.view(dims).to(torch.int32) & 0xFFFF
            assert bin_bound_ok(ai, di, ours, dims, bins), (bins, p)
            del ai, di
    ws.close()
