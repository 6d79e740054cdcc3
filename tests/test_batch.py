"""Batch compression (lscomp_compress_batch_u16/_u32): many stacks in one
persistent launch.  Every stack's stream and sizes must equal what the
single-stack call writes for it alone, which is itself byte-identical to
the reference (test_gpu_parity.py); a few stacks are also checked against
the oracle directly."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

LOSSLESS = ((1, 1, 1, 1), 1.0)
LOSSY = ((3, 5, 10, 15), 0.5)
GENERAL = ((9, 4, 12, 3), 0.5)

SHAPES = [
    (1, 8, 8), (1, 1, 1), (2, 13, 21), (3, 37, 53), (4, 64, 64), (2, 100, 130),
    (1, 9, 2049), (2, 17, 4100), (5, 31, 7), (64, 16, 16), (3, 250, 2), (1, 1025, 9), (6, 181, 155),
]


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


def stack16(dims, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 60, size=dims, dtype=np.uint16)
    a[rng.random(dims) < 0.55] = 0
    a[rng.random(dims) < 0.01] = 65535
    return a


def stack32(dims, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 1 << 20, size=dims, dtype=np.uint32)
    a[rng.random(dims) < 0.5] = 0
    return a


def run_batch(lz, ws, arrays, dims_list, bins, p, wide=False, poison=0xAB):
    view = np.int32 if wide else np.int16
    eb = 4 if wide else 2
    ins = [torch.from_numpy(np.ascontiguousarray(a).view(view).ravel()).cuda() for a in arrays]
    outs = [torch.full((lz.max_stream_bytes(d, eb),), poison, dtype=torch.uint8, device="cuda") for d in dims_list]
    res = lz.compress_batch(ws, list(zip(ins, dims_list, outs)), bins, p)
    return ins, outs, res


def single(lz, ws, d_in, dims, bins, p, eb):
    out = torch.zeros(lz.max_stream_bytes(dims, eb), dtype=torch.uint8, device="cuda")
    sl, rs = lz.compress_into(ws, d_in, dims, bins, p, out)
    return out[:sl].cpu().numpy(), sl, rs


@pytest.mark.parametrize("bins,p", [LOSSLESS, LOSSY, GENERAL, ((1, 1, 1, 1), 0.0)])
def test_batch_equals_single_u16(lz, ws, bins, p):
    arrays = [stack16(d, seed=i) for i, d in enumerate(SHAPES)]
    ins, outs, res = run_batch(lz, ws, arrays, SHAPES, bins, p)
    for d_in, dims, out, (sl, rs) in zip(ins, SHAPES, outs, res):
        ref, sl1, rs1 = single(lz, ws, d_in, dims, bins, p, 2)
        assert (sl, rs) == (sl1, rs1), dims
        assert np.array_equal(out[:sl].cpu().numpy(), ref), dims


@pytest.mark.parametrize("bins,p", [LOSSLESS, LOSSY])
def test_batch_equals_single_u32(lz, ws, bins, p):
    shapes = [(1, 8, 8), (2, 13, 21), (3, 37, 53), (2, 17, 1100), (4, 64, 64)]
    arrays = [stack32(d, seed=10 + i) for i, d in enumerate(shapes)]
    ins, outs, res = run_batch(lz, ws, arrays, shapes, bins, p, wide=True)
    for d_in, dims, out, (sl, rs) in zip(ins, shapes, outs, res):
        ref, sl1, rs1 = single(lz, ws, d_in, dims, bins, p, 4)
        assert (sl, rs) == (sl1, rs1), dims
        assert np.array_equal(out[:sl].cpu().numpy(), ref), dims


def test_many_small_stacks_vs_oracle(lz, ws, oracle):
    # 400 stacks of 1..6 frames with ragged frame sizes: most are a single
    # tile, so almost every tile is the first of its stack
    rng = np.random.default_rng(7)
    dims_list = [(int(rng.integers(1, 7)), int(rng.integers(1, 120)), int(rng.integers(1, 140))) for _ in range(400)]
    arrays = [stack16(d, seed=100 + i) for i, d in enumerate(dims_list)]
    bins, p = LOSSY
    ins, outs, res = run_batch(lz, ws, arrays, dims_list, bins, p)
    for i in range(0, 400, 7):  # every 7th stack against the oracle
        # (reported sizes are compared with the single-stack call below: for
        # stacks of at most 1024 blocks the oracle models the reference's own
        # report, nb, which this library replaces by payload + nb)
        s_o, _ = oracle.compress(arrays[i], dims_list[i], bins, p)
        sl, _ = res[i]
        assert sl == len(s_o)
        assert np.array_equal(outs[i][:sl].cpu().numpy(), np.asarray(s_o))
    for i in range(1, 400, 7):  # and others against the single-stack call
        ref, sl1, rs1 = single(lz, ws, ins[i], dims_list[i], bins, p, 2)
        assert res[i] == (sl1, rs1)
        assert np.array_equal(outs[i][: res[i][0]].cpu().numpy(), ref)


def test_batch_round_trip(lz, ws):
    dims_list = [(3, 200, 300), (1, 1813, 1558), (7, 64, 1030)]
    arrays = [stack16(d, seed=40 + i) for i, d in enumerate(dims_list)]
    ins, outs, res = run_batch(lz, ws, arrays, dims_list, *LOSSLESS)
    for d_in, dims, out, (sl, _) in zip(ins, dims_list, outs, res):
        dec = torch.empty_like(d_in)
        lz.decompress_into(ws, out, sl, dims, *LOSSLESS, dec)
        assert torch.equal(dec, d_in)


def test_batch_unaligned_input(lz, ws):
    # one stack's input starts 2 bytes past a 16-byte boundary: the whole
    # batch then reads rows with 2-byte accesses, same streams
    dims_list = [(2, 40, 48), (2, 33, 64)]
    arrays = [stack16(d, seed=60 + i) for i, d in enumerate(dims_list)]
    base = torch.from_numpy(np.concatenate([[0], arrays[0].ravel()]).astype(np.uint16).view(np.int16)).cuda()
    d0 = base[1:]
    d1 = torch.from_numpy(arrays[1].view(np.int16).ravel()).cuda()
    outs = [torch.zeros(lz.max_stream_bytes(d), dtype=torch.uint8, device="cuda") for d in dims_list]
    res = lz.compress_batch(ws, [(d0, dims_list[0], outs[0]), (d1, dims_list[1], outs[1])], *LOSSY)
    for d_in, dims, out, (sl, rs) in zip([d0, d1], dims_list, outs, res):
        ref, sl1, rs1 = single(lz, ws, d_in, dims, *LOSSY, 2)
        assert (sl, rs) == (sl1, rs1)
        assert np.array_equal(out[:sl].cpu().numpy(), ref)


def test_batch_errors(lz, ws):
    assert lz.compress_batch(ws, [], *LOSSY) == []
    a = stack16((2, 64, 64), seed=1)
    d = torch.from_numpy(a.view(np.int16).ravel()).cuda()
    good = torch.zeros(lz.max_stream_bytes((2, 64, 64)), dtype=torch.uint8, device="cuda")
    small = torch.zeros(lz.block_count((2, 64, 64)), dtype=torch.uint8, device="cuda")  # header only
    with pytest.raises(lz.LscompError) as e:
        lz.compress_batch(ws, [(d, (2, 64, 64), good), (d, (2, 64, 64), small)], *LOSSLESS)
    assert e.value.status == 2  # capacity
    # the workspace is usable after the failed launch
    res = lz.compress_batch(ws, [(d, (2, 64, 64), good)], *LOSSLESS)
    ref, sl1, rs1 = single(lz, ws, d, (2, 64, 64), *LOSSLESS, 2)
    assert res[0] == (sl1, rs1)
    assert np.array_equal(good[: res[0][0]].cpu().numpy(), ref)
    with pytest.raises(lz.LscompError) as e:
        lz.compress_batch(ws, [(d, (2, 64, 0), good)], *LOSSLESS)
    assert e.value.status == 1


SETTINGS = [((1, 1, 1, 1), 1.0), ((3, 5, 10, 15), 0.3), ((3, 5, 10, 15), 0.5), ((5, 10, 15, 20), 0.8),
            ((1, 1, 1, 1), 0.5), ((7, 7, 7, 7), 0.8)]


@pytest.mark.parametrize("with_general", [False, True])
def test_mixed_settings_u16(lz, ws, oracle, with_general):
    # every stack with its own bins and threshold, one launch: increasing-bins
    # kernel for the monotone mix, the general kernel once a stack's bins
    # do not increase
    rng = np.random.default_rng(11)
    settings = SETTINGS + ([GENERAL] if with_general else [])
    shapes = SHAPES + [(3, 130, 150), (2, 300, 210)]
    items, arrays, chosen = [], [], []
    for i, dims in enumerate(shapes):
        a = stack16(dims, seed=300 + i)
        b, p = settings[int(rng.integers(0, len(settings)))] if i >= len(settings) else settings[i]
        d_in = torch.from_numpy(a.view(np.int16).ravel()).cuda()
        out = torch.full((lz.max_stream_bytes(dims),), 0xAB, dtype=torch.uint8, device="cuda")
        items.append((d_in, dims, out, b, p))
        arrays.append(a)
        chosen.append((b, p))
    res = lz.compress_batch_mixed(ws, items)
    for (d_in, dims, out, b, p), a, (sl, rs) in zip(items, arrays, res):
        ref, sl1, rs1 = single(lz, ws, d_in, dims, b, p, 2)
        assert (sl, rs) == (sl1, rs1), (dims, b, p)
        assert np.array_equal(out[:sl].cpu().numpy(), ref), (dims, b, p)
        s_o, _ = oracle.compress(a, dims, b, p)
        assert np.array_equal(ref, np.asarray(s_o)), (dims, b, p)


def test_mixed_settings_u32(lz, ws):
    shapes = [(1, 8, 8), (2, 13, 21), (3, 37, 53), (2, 17, 1100), (4, 64, 64)]
    items = []
    for i, dims in enumerate(shapes):
        b, p = SETTINGS[i % len(SETTINGS)]
        d_in = torch.from_numpy(stack32(dims, seed=400 + i).view(np.int32).ravel()).cuda()
        out = torch.zeros(lz.max_stream_bytes(dims, 4), dtype=torch.uint8, device="cuda")
        items.append((d_in, dims, out, b, p))
    res = lz.compress_batch_mixed(ws, items)
    for (d_in, dims, out, b, p), (sl, rs) in zip(items, res):
        ref, sl1, rs1 = single(lz, ws, d_in, dims, b, p, 4)
        assert (sl, rs) == (sl1, rs1), (dims, b, p)
        assert np.array_equal(out[:sl].cpu().numpy(), ref), (dims, b, p)


def test_mixed_settings_plan(lz, ws):
    shapes = [(2, 100, 130), (1, 9, 2049), (5, 31, 7), (4, 64, 64), (3, 37, 53)]
    items = []
    for i, dims in enumerate(shapes):
        b, p = SETTINGS[(i + 1) % len(SETTINGS)]
        d_in = torch.from_numpy(stack16(dims, seed=500 + i).view(np.int16).ravel()).cuda()
        out = torch.zeros(lz.max_stream_bytes(dims), dtype=torch.uint8, device="cuda")
        items.append((d_in, dims, out, b, p))
    plan = lz.Plan(ws, items)
    try:
        for rnd in range(2):
            if rnd:
                for i, (d_in, dims, out, b, p) in enumerate(items):
                    d_in.copy_(torch.from_numpy(stack16(dims, seed=600 + i).view(np.int16).ravel()).cuda())
                    out.fill_(0xCD)
            res = plan.run()
            for (d_in, dims, out, b, p), (sl, rs) in zip(items, res):
                ref, sl1, rs1 = single(lz, ws, d_in, dims, b, p, 2)
                assert (sl, rs) == (sl1, rs1), (rnd, dims)
                assert np.array_equal(out[:sl].cpu().numpy(), ref), (rnd, dims)
    finally:
        plan.close()


@pytest.mark.parametrize("wide", [False, True])
def test_decompress_batch(lz, ws, wide):
    # streams of many shapes and settings decoded in one batch; each output
    # must equal the single-stream decode (every element written)
    rng = np.random.default_rng(21)
    shapes = SHAPES + [(3, 130, 150), (2, 300, 210), (40, 9, 9)]
    es = 4 if wide else 2
    items, refs = [], []
    for i, dims in enumerate(shapes):
        b, p = SETTINGS[int(rng.integers(0, len(SETTINGS)))]
        a = stack32(dims, seed=700 + i) if wide else stack16(dims, seed=700 + i)
        view = np.int32 if wide else np.int16
        d_in = torch.from_numpy(a.view(view).ravel()).cuda()
        out = torch.zeros(lz.max_stream_bytes(dims, es), dtype=torch.uint8, device="cuda")
        sl, _ = lz.compress_into(ws, d_in, dims, b, p, out)
        ref = torch.empty_like(d_in)
        lz.decompress_into(ws, out, sl, dims, b, p, ref)
        dec = torch.full_like(d_in, -1)  # poison: every element must be written
        items.append((out, sl, dims, dec, b, p))
        refs.append(ref)
    lz.decompress_batch(ws, items)
    for (out, sl, dims, dec, b, p), ref in zip(items, refs):
        assert torch.equal(dec, ref), (dims, b, p)


def test_decompress_batch_truncated(lz, ws):
    dims = (2, 64, 64)
    d_in = torch.from_numpy(stack16(dims, seed=3).view(np.int16).ravel()).cuda()
    out = torch.zeros(lz.max_stream_bytes(dims), dtype=torch.uint8, device="cuda")
    sl, _ = lz.compress_into(ws, d_in, dims, *LOSSLESS, out)
    dec = torch.empty_like(d_in)
    with pytest.raises(lz.LscompError):
        lz.decompress_batch(ws, [(out, sl - 16, dims, dec, *LOSSLESS), (out, sl, dims, torch.empty_like(d_in), *LOSSLESS)])
    # the workspace still works
    lz.decompress_batch(ws, [(out, sl, dims, dec, *LOSSLESS)])
    assert torch.equal(dec, d_in)


@pytest.mark.parametrize("wide", [False, True])
def test_stream_sizes_match_compression(lz, ws, wide):
    """lscomp_stream_sizes_batch_*: the exact bytes compression writes, per
    stack and per setting, from a pass that writes no stream; a uint32
    quotient needing 32 planes is refused as compression refuses it."""
    rng = np.random.default_rng(21)
    settings = SETTINGS + [GENERAL]
    shapes = SHAPES + [(3, 130, 150), (2, 300, 210)]
    view, eb = (np.int32, 4) if wide else (np.int16, 2)
    items = []
    for i, dims in enumerate(shapes):
        a = stack32(dims, seed=500 + i) if wide else stack16(dims, seed=500 + i)
        b, p = settings[int(rng.integers(0, len(settings)))]
        d_in = torch.from_numpy(a.view(view).ravel()).cuda()
        out = torch.zeros(lz.max_stream_bytes(dims, eb), dtype=torch.uint8, device="cuda")
        items.append((d_in, dims, out, b, p))
    sizes = lz.stream_sizes_batch(ws, items)
    res = lz.compress_batch_mixed(ws, items)
    assert sizes == [sl for sl, _ in res]
    if wide:
        a = np.zeros((1, 8, 8), dtype=np.uint32)
        a[0, 0, 0] = 0xFFFFFFFF
        d = torch.from_numpy(a.view(np.int32).ravel()).cuda()
        with pytest.raises(lz.LscompError) as e:
            lz.stream_sizes_batch(ws, items[:2] + [(d, (1, 8, 8), None, LOSSLESS[0], 1.0)])
        assert e.value.status == 6
