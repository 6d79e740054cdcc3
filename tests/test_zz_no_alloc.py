"""GPU test of lscomp_compress_u16_noalloc, the compression entry point that
allocates nothing: its scan scratch is a fixed array inside the library, for
callers that cannot call cudaMalloc while they compress (a fixed, pre-reserved
memory budget; device memory owned by another allocator).

Called through the C ABI, its stream and sizes must equal those of the
workspace entry point (lscomp_compress_u16) byte for byte, on two calls in a
row (the second call runs on the scratch the first one left behind).  Kept in
a file of its own that pytest collects last."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOO_LARGE = 8


def _noalloc(lib):
    f = lib.lscomp_compress_u16_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                  ctypes.POINTER(ctypes.c_uint32), ctypes.c_float, ctypes.c_void_p, ctypes.c_uint64,
                  ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p]
    return f


CASES = [((6, 333, 517), (1, 1, 1, 1), 1.0, 3), ((4, 250, 1030), (3, 5, 10, 15), 0.5, 4)]


def _compare(lscomp, lib, f, ws, stream):
    for dims, bins, p, seed in CASES:  # two calls in a row
        a = lscomp.synth_cssi(dims, seed=seed)
        d_in = torch.from_numpy(a.view(np.int16)).cuda()
        cap = lscomp.max_stream_bytes(dims)
        want = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        sl_w, rs_w = lscomp.compress_into(ws, d_in, dims, bins, p, want)
        got = torch.full((cap,), 0xAB, dtype=torch.uint8, device="cuda")
        sl, rs = ctypes.c_uint64(0), ctypes.c_uint64(0)
        b = (ctypes.c_uint32 * 4)(*bins)
        st = f(ctypes.c_void_p(d_in.data_ptr()), dims[0], dims[1], dims[2], b, ctypes.c_float(p),
               ctypes.c_void_p(got.data_ptr()), ctypes.c_uint64(cap), ctypes.byref(sl), ctypes.byref(rs),
               ctypes.c_void_p(stream))
        assert st == 0, lib.lscomp_status_string(st)
        assert (sl.value, rs.value) == (sl_w, rs_w)
        assert torch.equal(got[:sl_w], want[:sl_w])


def test_noalloc_matches_workspace_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lscomp

    lib = lscomp.load_library()
    _compare(lscomp, lib, _noalloc(lib), lscomp.Workspace(0), torch.cuda.current_stream().cuda_stream)


def test_noalloc_with_tuner_table_entries(tmp_path):
    """The entry point takes the launch configuration the tuner's table holds
    for its key (another tile size, or the 13-warp groups) when the tiles fit
    its scratch; both calls must still write the same bytes."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lscomp

    lib = lscomp.load_library()
    f = _noalloc(lib)
    saved = tmp_path / "before.txt"
    lscomp.tune_save(str(saved))
    # keys "es layout pool kind vec bzb": the lossless case (layout 3, no
    # pooling, 2-byte rows, 65 blocks per block-row) and the lossy one
    # (increasing bins, pooling, 4-byte rows, 129 blocks per block-row)
    for lossless_cfg, lossy_cfg in (("0 128", "2 256"), ("1 256", "0 128")):
        table = tmp_path / "table.txt"
        table.write_text(f"2 3 0 0 2 65 -> {lossless_cfg}\n2 1 1 0 4 129 -> {lossy_cfg}\n")
        lscomp.tune_load(str(table))
        _compare(lscomp, lib, f, lscomp.Workspace(0), torch.cuda.current_stream().cuda_stream)
    lscomp.tune_clear()
    lscomp.tune_load(str(saved))


def test_noalloc_refuses_stacks_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lscomp

    f = _noalloc(lscomp.load_library())
    d = torch.zeros(16, dtype=torch.int16, device="cuda")
    o = torch.zeros(16, dtype=torch.uint8, device="cuda")
    b = (ctypes.c_uint32 * 4)(1, 1, 1, 1)
    # 300,000 frames of 8 x 2048: one tile per frame, more tiles than the
    # scratch holds; refused on the host before any GPU work
    st = f(ctypes.c_void_p(d.data_ptr()), 300000, 8, 2048, b, ctypes.c_float(1.0), ctypes.c_void_p(o.data_ptr()),
           ctypes.c_uint64(16), None, None, None)
    assert st == TOO_LARGE
