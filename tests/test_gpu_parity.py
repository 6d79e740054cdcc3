"""GPU parity: the CUDA codec (through the C ABI of liblscomp.so) against the
CPU oracle and against the reference's own CUDA build on the same device.

Streams must be byte-identical, decodes bit-exact.  Sizes the oracle handles
in seconds are compared element for element; the full-size stacks are
compared with the reference build on the GPU and through round trips."""
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


@pytest.fixture(scope="module")
def ws(lz):
    return lz.Workspace(0)


@pytest.fixture(scope="module")
def ref():
    from oracle import RefLib

    return RefLib()


def to_dev(a: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int16).ravel()).cuda()


def gpu_compress(lz, ws, a, dims, bins, p):
    d_in = to_dev(a)
    out = torch.zeros(lz.max_stream_bytes(dims), dtype=torch.uint8, device="cuda")
    sl, rs = lz.compress_into(ws, d_in, dims, bins, p, out)
    return out, sl, rs


def gpu_decompress(lz, ws, stream_t, sl, dims, bins, p):
    n = dims[0] * dims[1] * dims[2]
    out = torch.full((n,), -1, dtype=torch.int16, device="cuda")  # poison: every element must be written
    lz.decompress_into(ws, stream_t, sl, dims, bins, p, out)
    return out.cpu().numpy().view(np.uint16)


def random_stack(dims, seed, zero_frac=0.5, hot=0.01, hi=40):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, hi, size=dims, dtype=np.uint16)
    a[rng.random(dims) < zero_frac] = 0
    a[rng.random(dims) < hot] = 65535
    return a


SHAPES = [
    (1, 8, 8), (1, 1, 1), (2, 13, 21), (3, 37, 53), (4, 64, 64), (2, 100, 130),
    (1, 9, 2049), (2, 17, 4100),       # chunked tiles (more than 256 blocks per block-row)
    (5, 31, 7), (64, 16, 16), (3, 250, 2), (1, 1025, 9),
]
SETTINGS = [LOSSLESS, LOSSY, ((5, 5, 5, 5), 0.3), ((2, 7, 7, 30), 0.8), ((9, 4, 12, 3), 0.5),
            ((1, 1, 1, 1), 0.0), ((1, 2, 4, 8), 1.0)]


@pytest.mark.parametrize("dims", SHAPES)
@pytest.mark.parametrize("bins,p", SETTINGS)
def test_random_shapes_vs_oracle(lz, ws, oracle, dims, bins, p):
    a = random_stack(dims, seed=hash((dims, bins, p)) & 0xffff)
    s_o, rs_o = oracle.compress(a, dims, bins, p)
    out, sl, rs = gpu_compress(lz, ws, a, dims, bins, p)
    assert sl == len(s_o)
    s_g = out[:sl].cpu().numpy()
    assert np.array_equal(s_g, s_o)
    nb = lz.block_count(dims)
    assert rs == len(s_o) - (nb + 3) // 4 * 4 + nb  # payload + nb
    if nb > 1024:
        assert rs == rs_o
    d_g = gpu_decompress(lz, ws, out, sl, dims, bins, p)
    d_o = oracle.decompress(s_o, dims, bins, p)
    assert np.array_equal(d_g, d_o)
    if bins == (1, 1, 1, 1) and p >= 1.0:
        assert np.array_equal(d_g, a.ravel())


@pytest.mark.parametrize("kind,dims", [("small", (64, 256, 256)), ("cssi", (6, 1813, 1558)),
                                       ("xpcs", (16, 1024, 1024)), ("cssi", (3, 333, 517))])
@pytest.mark.parametrize("bins,p", [LOSSLESS, LOSSY, ((5, 10, 15, 15), 0.5), ((10, 10, 15, 15), 0.5)])
def test_synthetic_vs_oracle(lz, ws, oracle, kind, dims, bins, p):
    a = getattr(lz, f"synth_{kind}")(dims).reshape(dims)
    s_o, _ = oracle.compress(a, dims, bins, p)
    out, sl, rs = gpu_compress(lz, ws, a, dims, bins, p)
    assert sl == len(s_o)
    assert torch.equal(out[:sl].cpu(), torch.from_numpy(s_o))
    d_g = gpu_decompress(lz, ws, out, sl, dims, bins, p)
    assert np.array_equal(d_g, oracle.decompress(s_o, dims, bins, p))


@pytest.mark.parametrize("dims", [(1, 8, 8), (3, 37, 53), (8, 128, 96), (64, 256, 256), (2, 17, 4100)])
@pytest.mark.parametrize("bins,p", [LOSSLESS, LOSSY, ((1, 1, 1, 1), 0.0)])
def test_vs_reference_build(lz, ws, ref, dims, bins, p):
    """Byte-identical to the reference CUDA build on pre-zeroed buffers."""
    a = random_stack(dims, seed=5, zero_frac=0.6)
    d_in = to_dev(a)
    cap = lz.max_stream_bytes(dims)
    ref_out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    rs_ref = ref.compress(d_in.data_ptr(), ref_out.data_ptr(), dims, bins, p)
    torch.cuda.synchronize()
    out, sl, rs = gpu_compress(lz, ws, a, dims, bins, p)
    assert torch.equal(out[:sl], ref_out[:sl])
    assert int(ref_out[sl:].count_nonzero()) == 0
    nb = lz.block_count(dims)
    assert rs_ref == (rs if nb > 1024 else nb)
    # decode with the reference into a zeroed buffer and with ours
    n = a.size
    dref = torch.zeros(n, dtype=torch.int16, device="cuda")
    ref.decompress(dref.data_ptr(), ref_out.data_ptr(), rs_ref, dims, bins, p)
    torch.cuda.synchronize()
    d_g = gpu_decompress(lz, ws, out, sl, dims, bins, p)
    assert np.array_equal(d_g, dref.cpu().numpy().view(np.uint16))


def test_capacity_error(lz, ws):
    dims = (4, 64, 64)
    a = random_stack(dims, seed=9, zero_frac=0.0, hi=60000)
    d_in = to_dev(a)
    small = torch.zeros(lz.block_count(dims) + 100, dtype=torch.uint8, device="cuda")
    with pytest.raises(lz.LscompError) as e:
        lz.compress_into(ws, d_in, dims, LOSSLESS[0], 1.0, small)
    assert e.value.status == 2
    # the workspace stays usable after the error
    out, sl, _ = gpu_compress(lz, ws, a, dims, *LOSSLESS)
    assert np.array_equal(gpu_decompress(lz, ws, out, sl, dims, *LOSSLESS), a.ravel())


def test_bad_arguments(lz, ws):
    d = torch.zeros(64, dtype=torch.int16, device="cuda")
    o = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    with pytest.raises(lz.LscompError):
        lz.compress_into(ws, d, (1, 8, 8), (0, 1, 1, 1), 1.0, o)
    with pytest.raises(lz.LscompError):
        lz.compress_into(ws, d, (0, 8, 8), (1, 1, 1, 1), 1.0, o)


def test_truncated_stream_rejected(lz, ws):
    dims = (2, 64, 64)
    a = random_stack(dims, seed=4, zero_frac=0.1, hi=1000)
    out, sl, _ = gpu_compress(lz, ws, a, dims, *LOSSLESS)
    d = torch.zeros(a.size, dtype=torch.int16, device="cuda")
    with pytest.raises(lz.LscompError) as e:
        lz.decompress_into(ws, out, sl - 64, dims, *LOSSLESS, d)
    assert e.value.status == 2


# ---------------------------------------------------------------- uint32 twins
U32_SETTINGS = [LOSSLESS, LOSSY, ((7, 7, 7, 7), 0.3), ((9, 4, 12, 3), 0.5), ((1, 1, 1, 1), 0.0),
                ((2, 1000, 70000, 1 << 20), 0.8)]


def random_stack32(dims, seed, hi=1 << 20):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, hi, size=dims, dtype=np.uint32)
    a[rng.random(dims) < 0.5] = 0
    a[rng.random(dims) < 0.01] = 0x7FFFFFFF
    return a


@pytest.mark.parametrize("dims", [(1, 8, 8), (2, 13, 21), (3, 37, 53), (2, 17, 1100), (4, 64, 64), (1, 1025, 9)])
@pytest.mark.parametrize("bins,p", U32_SETTINGS)
def test_u32_vs_oracle(lz, ws, oracle, dims, bins, p):
    a = random_stack32(dims, seed=hash((dims, bins, p)) & 0xffff)
    s_o, rs_o = oracle.compress(a, dims, bins, p, dtype=np.uint32)
    d_in = torch.from_numpy(a.view(np.int32).ravel()).cuda()
    out = torch.zeros(lz.max_stream_bytes(dims, 4), dtype=torch.uint8, device="cuda")
    sl, rs = lz.compress_into(ws, d_in, dims, bins, p, out)
    assert sl == len(s_o)
    assert np.array_equal(out[:sl].cpu().numpy(), s_o)
    dec = torch.full((a.size,), -1, dtype=torch.int32, device="cuda")
    lz.decompress_into(ws, out, sl, dims, bins, p, dec)
    d_o = oracle.decompress(s_o, dims, bins, p, dtype=np.uint32)
    assert np.array_equal(dec.cpu().numpy().view(np.uint32), d_o)


def test_u32_vs_reference_build(lz, ws, ref):
    dims = (8, 128, 96)
    a = random_stack32(dims, seed=12)
    d_in = torch.from_numpy(a.view(np.int32).ravel()).cuda()
    cap = lz.max_stream_bytes(dims, 4)
    ref_out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    for bins, p in (LOSSLESS, LOSSY):
        ref_out.zero_()
        rs_ref = ref.compress(d_in.data_ptr(), ref_out.data_ptr(), dims, bins, p, t="u32")
        torch.cuda.synchronize()
        out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        sl, rs = lz.compress_into(ws, d_in, dims, bins, p, out)
        assert torch.equal(out[:sl], ref_out[:sl])
        assert rs == rs_ref


def test_u32_rate32_rejected(lz, ws):
    # a quotient >= 2^31 needs 32 planes; the reference writes a stream its own
    # decoder misreads, this library reports the range error instead
    a = np.zeros((1, 8, 8), dtype=np.uint32)
    a[0, 0, 0] = 0xFFFFFFFF
    d_in = torch.from_numpy(a.view(np.int32).ravel()).cuda()
    out = torch.zeros(lz.max_stream_bytes((1, 8, 8), 4), dtype=torch.uint8, device="cuda")
    with pytest.raises(lz.LscompError) as e:
        lz.compress_into(ws, d_in, (1, 8, 8), LOSSLESS[0], 1.0, out)
    assert e.value.status == 6
    # same value with bin 2 fits in 31 planes
    sl, _ = lz.compress_into(ws, d_in, (1, 8, 8), (2, 2, 2, 2), 1.0, out)
    assert out[0].item() & 31 == 31


@pytest.mark.parametrize("in_off,out_off", [(1, 0), (3, 4), (5, 12), (0, 8)])
@pytest.mark.parametrize("dims", [(3, 37, 53), (2, 64, 64), (1, 17, 2051)])
@pytest.mark.parametrize("bins,p", [LOSSLESS, LOSSY])
def test_unaligned_pointers(lz, ws, oracle, in_off, out_off, dims, bins, p):
    """Input starting off a 16-byte boundary (the TMA fetch then copies the
    ragged ends of the array element by element) and streams at 4-byte offsets."""
    a = random_stack(dims, seed=21, zero_frac=0.4, hi=3000)
    n = a.size
    buf = torch.zeros(n + 16, dtype=torch.int16, device="cuda")
    buf[in_off:in_off + n] = to_dev(a)
    d_in = buf[in_off:in_off + n]
    cap = lz.max_stream_bytes(dims)
    obuf = torch.zeros(cap + 32, dtype=torch.uint8, device="cuda")
    out = obuf[out_off:out_off + cap]
    sl, _ = lz.compress_into(ws, d_in, dims, bins, p, out)
    s_o, _ = oracle.compress(a, dims, bins, p)
    assert np.array_equal(out[:sl].cpu().numpy(), s_o)
    dbuf = torch.full((n + 16,), -1, dtype=torch.int16, device="cuda")
    dec = dbuf[in_off:in_off + n]
    lz.decompress_into(ws, out, sl, dims, bins, p, dec)
    assert np.array_equal(dec.cpu().numpy().view(np.uint16), oracle.decompress(s_o, dims, bins, p))
    # nothing outside the output range was touched
    assert int((dbuf[:in_off] != -1).sum()) == 0 and int((dbuf[in_off + n:] != -1).sum()) == 0
