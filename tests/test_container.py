"""The container around an lsCOMP stream: 64-byte header (include/lscomp.h,
lscomp_container_*) + the stream unchanged.  Header functions are host code
and are tested on the CPU; compression into and decompression from a
container on the GPU."""
import struct
import zlib

import numpy as np
import pytest


@pytest.fixture(scope="module")
def lz():
    import lscomp

    lscomp.load_library()
    return lscomp


def test_header_round_trip(lz):
    h = lz.container_header(2, (600, 1813, 1558), (3, 5, 10, 15), 0.5, 587054364, 587054364 - 6 + 26559000)
    assert len(h) == 64 and h[:4] == b"LSCZ"
    info = lz.parse_container(h)
    assert info["elem_bytes"] == 2 and info["dims"] == (600, 1813, 1558)
    assert info["bins"] == (3, 5, 10, 15) and info["pooling"] == 0.5
    assert info["stream_len"] == 587054364 and info["ref_size"] == 587054364 - 6 + 26559000


def test_header_layout_independent_check(lz):
    # the documented little-endian layout, rebuilt here with struct/zlib
    h = lz.container_header(4, (3, 17, 1100), (1, 2, 4, 8), 0.8, 12345, 6789)
    body = struct.pack("<4sHH3I4IfQQ", b"LSCZ", 1, 4, 3, 17, 1100, 1, 2, 4, 8, 0.8, 12345, 6789)
    assert h[:56] == body
    assert struct.unpack("<I", h[56:60])[0] == zlib.crc32(body) & 0xFFFFFFFF
    assert h[60:64] == b"\0\0\0\0"


@pytest.mark.parametrize("pos", [0, 4, 6, 9, 21, 37, 41, 57])
def test_corrupted_header_rejected(lz, pos):
    h = bytearray(lz.container_header(2, (2, 64, 64), (1, 1, 1, 1), 1.0, 5000, 4900))
    h[pos] ^= 0x10
    with pytest.raises(lz.LscompError) as e:
        lz.parse_container(bytes(h))
    assert e.value.status == 5


def test_length_checks(lz):
    h = lz.container_header(2, (2, 64, 64), (1, 1, 1, 1), 1.0, 5000, 4900)
    assert lz.parse_container(h + bytes(5000))["stream_len"] == 5000
    with pytest.raises(lz.LscompError):
        lz.parse_container(h + bytes(4999))  # body shorter than the stream
    with pytest.raises(lz.LscompError):
        lz.parse_container(h[:40])
    with pytest.raises(lz.LscompError):
        lz.container_header(3, (2, 64, 64), (1, 1, 1, 1), 1.0, 5000, 4900)  # element size
    # a stream shorter than its own header bytes is impossible
    bad = lz.container_header(2, (2, 64, 64), (1, 1, 1, 1), 1.0, 100, 100)
    with pytest.raises(lz.LscompError):
        lz.parse_container(bad)


@pytest.mark.gpu
@pytest.mark.parametrize("wide", [False, True])
@pytest.mark.parametrize("bins,p", [((1, 1, 1, 1), 1.0), ((3, 5, 10, 15), 0.5)])
def test_container_gpu(lz, wide, bins, p):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    dims = (3, 70, 190)
    rng = np.random.default_rng(3)
    a = rng.integers(0, 200, size=dims, dtype=np.uint32 if wide else np.uint16)
    a[rng.random(dims) < 0.5] = 0
    d_in = torch.from_numpy(a.view(np.int32 if wide else np.int16).ravel()).cuda()
    eb = 4 if wide else 2
    ws = lz.Workspace(0)
    plain = torch.zeros(lz.max_stream_bytes(dims, eb), dtype=torch.uint8, device="cuda")
    sl, rs = lz.compress_into(ws, d_in, dims, bins, p, plain)
    cont = torch.zeros(64 + lz.max_stream_bytes(dims, eb), dtype=torch.uint8, device="cuda")
    n = lz.compress_container(ws, d_in, dims, bins, p, cont)
    assert n == 64 + sl
    assert torch.equal(cont[64:n], plain[:sl])  # the body is the stream, unchanged
    info = lz.parse_container(cont[:n].cpu().numpy().tobytes())
    assert info["stream_len"] == sl and info["ref_size"] == rs and info["dims"] == dims
    out = torch.empty_like(d_in)
    got = lz.decompress_container(ws, cont, n, out)
    assert got["bins"] == tuple(bins)
    ref = torch.empty_like(d_in)
    lz.decompress_into(ws, plain, sl, dims, bins, p, ref)
    assert torch.equal(out, ref)
    if bins == (1, 1, 1, 1):
        assert torch.equal(out, d_in)
