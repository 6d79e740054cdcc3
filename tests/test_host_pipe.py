"""Compression and decompression from and to host memory
(lscomp_compress_host_* / lscomp_decompress_host_*): chunks of frames
pipelined through the device.  The stream must equal the device-memory
call's byte for byte (and the oracle's), the decode must equal the input
(lossless) or the device decode (lossy), for one chunk and for many, chunks
whose block count is not a multiple of 4, pinned and pageable buffers."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

LOSSLESS = ((1, 1, 1, 1), 1.0)
LOSSY = ((3, 5, 10, 15), 0.5)


@pytest.fixture(scope="module")
def lz():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lscomp

    lscomp.load_library()
    return lscomp


def stack(dims, seed, dtype=np.uint16):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 60, size=dims).astype(dtype)
    a[rng.random(dims) < 0.5] = 0
    a[rng.random(dims) < 0.01] = np.iinfo(dtype).max if dtype == np.uint16 else (1 << 20)
    return a


def device_stream(lz, ws, a, dims, bins, p, es):
    view = np.int16 if es == 2 else np.int32
    d_in = torch.from_numpy(a.view(view).ravel()).cuda()
    out = torch.zeros(lz.max_stream_bytes(dims, es), dtype=torch.uint8, device="cuda")
    sl, rs = lz.compress_into(ws, d_in, dims, bins, p, out)
    dec = torch.empty_like(d_in)
    lz.decompress_into(ws, out, sl, dims, bins, p, dec)
    return out[:sl].cpu().numpy(), sl, rs, dec.cpu().numpy().view(a.dtype)


@pytest.mark.parametrize("chunk_frames", [0, 1, 3])
@pytest.mark.parametrize("bins,p", [LOSSLESS, LOSSY])
@pytest.mark.parametrize("dims", [(7, 9, 17), (10, 100, 130), (5, 64, 1030)])
def test_host_round_trip_u16(lz, oracle, dims, bins, p, chunk_frames):
    ws = lz.Workspace(0)
    ws.set_host_chunk(chunk_frames * dims[1] * dims[2] * 2)  # 0: one chunk (default size)
    a = stack(dims, seed=sum(dims))
    ref, sl_d, rs_d, dec_d = device_stream(lz, ws, a, dims, bins, p, 2)
    out = np.full(lz.max_stream_bytes(dims), 0xAB, dtype=np.uint8)  # pageable
    sl, rs = lz.compress_host(ws, a, dims, bins, p, out)
    assert (sl, rs) == (sl_d, rs_d)
    assert np.array_equal(out[:sl], ref)
    s_o, _ = oracle.compress(a, dims, bins, p)
    assert np.array_equal(out[:sl], np.asarray(s_o))
    dec = np.full(a.size, 0xFFFF, dtype=np.uint16)
    lz.decompress_host(ws, out, sl, dims, bins, p, dec)
    assert np.array_equal(dec, dec_d.ravel())
    if bins == LOSSLESS[0]:
        assert np.array_equal(dec, a.ravel())
    ws.close()


def test_host_pinned_many_chunks(lz):
    dims = (64, 181, 1558)
    ws = lz.Workspace(0)
    ws.set_host_chunk(5 * dims[1] * dims[2] * 2)  # 13 chunks, the last one short
    a = stack(dims, seed=5)
    h_in = torch.from_numpy(a.view(np.int16).ravel()).pin_memory()
    h_out = torch.empty(lz.max_stream_bytes(dims), dtype=torch.uint8).pin_memory()
    h_dec = torch.empty_like(h_in).pin_memory()
    for bins, p in (LOSSLESS, LOSSY):
        ref, sl_d, rs_d, dec_d = device_stream(lz, ws, a, dims, bins, p, 2)
        sl, rs = lz.compress_host(ws, h_in, dims, bins, p, h_out)
        assert (sl, rs) == (sl_d, rs_d)
        assert np.array_equal(h_out[:sl].numpy(), ref)
        lz.decompress_host(ws, h_out, sl, dims, bins, p, h_dec)
        assert np.array_equal(h_dec.numpy().view(np.uint16), dec_d.ravel())
    ws.close()


def test_host_u32(lz):
    dims = (6, 37, 530)
    ws = lz.Workspace(0)
    ws.set_host_chunk(2 * dims[1] * dims[2] * 4)
    a = stack(dims, seed=9, dtype=np.uint32)
    for bins, p in (LOSSLESS, LOSSY):
        ref, sl_d, rs_d, dec_d = device_stream(lz, ws, a, dims, bins, p, 4)
        out = np.zeros(lz.max_stream_bytes(dims, 4), dtype=np.uint8)
        sl, rs = lz.compress_host(ws, a, dims, bins, p, out)
        assert (sl, rs) == (sl_d, rs_d)
        assert np.array_equal(out[:sl], ref)
        dec = np.zeros(a.size, dtype=np.uint32)
        lz.decompress_host(ws, out, sl, dims, bins, p, dec)
        assert np.array_equal(dec, dec_d.ravel())
    ws.close()


def test_host_errors(lz):
    dims = (4, 64, 64)
    ws = lz.Workspace(0)
    ws.set_host_chunk(64 * 64 * 2)
    a = stack(dims, seed=2)
    small = np.zeros(lz.block_count(dims) + 8, dtype=np.uint8)  # header and a few payload bytes
    with pytest.raises(lz.LscompError) as e:
        lz.compress_host(ws, a, dims, *LOSSLESS, small)
    assert e.value.status == 2
    # a truncated stream is refused before any payload moves
    out = np.zeros(lz.max_stream_bytes(dims), dtype=np.uint8)
    sl, _ = lz.compress_host(ws, a, dims, *LOSSLESS, out)
    dec = np.zeros(a.size, dtype=np.uint16)
    with pytest.raises(lz.LscompError) as e:
        lz.decompress_host(ws, out, sl - 64, dims, *LOSSLESS, dec)
    assert e.value.status == 2
    # the workspace still works
    lz.decompress_host(ws, out, sl, dims, *LOSSLESS, dec)
    assert np.array_equal(dec, a.ravel())
    ws.close()
