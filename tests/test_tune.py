"""Launch-configuration tuner and graph plans.

Every configuration the tuner may pick (encoder CTA shape x tile size,
decoder tile size) must write the same stream and the same decode, equal to
the oracle's; a configuration is forced by loading a one-line table.  The
tuner's table format round-trips on the CPU.  Graph plans (lscomp_plan_*)
must write what the ordinary calls write, again after the inputs change."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

LOSSLESS = ((1, 1, 1, 1), 1.0)
LOSSY = ((3, 5, 10, 15), 0.5)
GENERAL = ((9, 4, 12, 3), 0.5)


def layout_of(bins):
    if all(b == 1 for b in bins):
        return 3
    if len(set(bins)) == 1:
        return 0
    if list(bins) == sorted(bins):
        return 1
    return 2


def pool_of(p):
    return 1 if p < 1.0 else 0  # pool_min_zeros(p) <= 64 exactly when p < 1


def vec_of(z, es):
    if es == 2:
        return 16 if z % 8 == 0 else (4 if z % 2 == 0 else 2)
    return 16 if z % 4 == 0 else 4


@pytest.fixture(scope="module")
def lzc():
    import lscomp

    lscomp.load_library()
    return lscomp


# ---------------------------------------------------------------- host only
def test_table_roundtrip(lzc, tmp_path):
    prev = lzc.tune_mode()
    try:
        lzc.tune_clear()
        f = tmp_path / "t.txt"
        f.write_text("# comment\n2 1 1 0 16 195 -> 2 256\n2 3 0 2 16 128 -> -1 128\n4 1 1 1 16 0 -> 0 64\n")
        lzc.tune_load(str(f))
        tab = {(e["es"], e["layout"], e["pool"], e["kind"], e["vec"], e["bzb"]): (e["shape"], e["tile_blocks"])
               for e in lzc.tune_table()}
        assert tab == {(2, 1, 1, "compress", 16, 195): (2, 256), (2, 3, 0, "decompress", 16, 128): (-1, 128),
                       (4, 1, 1, "batch", 16, 0): (0, 64)}
        g = tmp_path / "g.txt"
        lzc.tune_save(str(g))
        lzc.tune_clear()
        assert lzc.tune_report() == ""
        lzc.tune_load(str(g))
        assert len(lzc.tune_table()) == 3
        # malformed or out-of-range lines change nothing
        for bad in ("2 1 1 0 16 195 -> 1 300\n", "4 1 1 0 16 9 -> 1 128\n", "2 1 1 0 16\n", "2 9 1 0 16 1 -> 0 8\n",
                    "4 1 1 0 2 9 -> 0 64\n", "2 1 1 0 8 9 -> 0 64\n",
                    "2 1 1 1 16 0 -> 2 256\n",   # 2 x 13 runs single stacks only
                    "4 1 1 0 16 9 -> 2 128\n",   # and uint16 only
                    "2 1 1 0 16 9 -> 3 256\n",   # 2 x 8 with the short paths: lossless only,
                    "2 3 0 1 16 0 -> 3 256\n",   # single stacks only,
                    "4 3 0 0 16 9 -> 3 128\n",   # uint16 only
                    "2 3 0 0 16 9 -> 4 256\n"):
            f.write_text("2 1 1 0 16 7 -> 0 8\n" + bad)
            with pytest.raises(lzc.LscompError):
                lzc.tune_load(str(f))
            assert len(lzc.tune_table()) == 3
        with pytest.raises(lzc.LscompError):
            lzc.tune_load(str(tmp_path / "missing.txt"))
        f.write_text("2 3 0 0 16 9 -> 3 256\n")  # lossless uint16 compress: accepted
        lzc.tune_load(str(f))
        assert len(lzc.tune_table()) == 4
    finally:
        lzc.tune_clear()
        lzc.tune_mode(prev)


def test_mode_switch(lzc):
    prev = lzc.tune_mode(0)
    try:
        assert lzc.tune_mode() == 0
        assert lzc.tune_mode(1) == 0
        assert lzc.tune_mode() == 1
    finally:
        lzc.tune_mode(prev)


# ---------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def lz(lzc):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return lzc


@pytest.fixture(scope="module")
def ws(lz):
    return lz.Workspace(0)


def random_stack(dims, seed, dtype=np.uint16, hi=60):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, hi, size=dims).astype(dtype)
    a[rng.random(dims) < 0.55] = 0
    a[rng.random(dims) < 0.01] = np.iinfo(dtype).max if dtype == np.uint16 else (1 << 20)
    return a


def small_value_stack(dims, seed, dtype=np.uint16):
    """Frames whose values stay below 4, 16, 128 and 300 in turn, so that the
    short paths for small values (units of rate <= 2 and <= 4, quotients of
    values below 128) and the longer ones all run; about half the values are
    zero, so blocks also pool at p = 0.5."""
    rng = np.random.default_rng(seed)
    a = np.empty(dims, dtype=dtype)
    for f in range(dims[0]):
        a[f] = rng.integers(0, (4, 16, 128, 300)[f % 4], size=dims[1:])
    a[rng.random(dims) < 0.55] = 0
    return a


def to_dev(a):
    view = np.int16 if a.dtype == np.uint16 else np.int32
    return torch.from_numpy(np.ascontiguousarray(a).view(view).ravel()).cuda()


def force(lz, tmp_path, line):
    f = tmp_path / "force.txt"
    f.write_text(line + "\n")
    lz.tune_clear()
    lz.tune_load(str(f))


CANDIDATES = {2: [(0, 256), (1, 256), (2, 256), (0, 128), (1, 128)], 4: [(0, 128), (0, 64)]}
# lossless uint16 single stacks also try 2 x 8 with the short paths for small values
CANDIDATES_LOSSLESS_U16 = [(0, 256), (1, 256), (2, 256), (3, 256), (0, 128), (1, 128)]


def candidates(es, bins):
    return CANDIDATES_LOSSLESS_U16 if es == 2 and all(x == 1 for x in bins) else CANDIDATES[es]
DEC_CANDIDATES = {2: [(-1, 256), (-1, 128)], 4: [(-1, 128), (-1, 64)]}
SHAPES = [(3, 37, 53), (2, 17, 2100), (4, 64, 1024), (2, 40, 1558), (1, 9, 2049)]
SMALL_SHAPES = [(4, 37, 53), (8, 40, 1558), (4, 64, 1024), (4, 17, 2100)]


@pytest.mark.gpu
@pytest.mark.parametrize("es", [2, 4])
@pytest.mark.parametrize("bins,p", [LOSSLESS, LOSSY, GENERAL])
@pytest.mark.parametrize("profile", ["wide", "small"])
def test_every_config_same_stream(lz, ws, oracle, tmp_path, es, bins, p, profile):
    if profile == "small" and es == 4:
        pytest.skip("the short paths for small values are uint16 only")
    dtype = np.uint16 if es == 2 else np.uint32
    # each call must use the forced line (one table hit per call)
    prev = lz.tune_mode(1)
    try:
        for i, dims in enumerate(SHAPES if profile == "wide" else SMALL_SHAPES):
            if profile == "wide":
                a = random_stack(dims, seed=100 + i, dtype=dtype)
            else:
                a = small_value_stack(dims, seed=200 + i, dtype=dtype)
            s_o, rs_o = oracle.compress(a, dims, bins, p, dtype=dtype)
            d_o = oracle.decompress(s_o, dims, bins, p, dtype=dtype)
            d_in = to_dev(a)
            bzb = (dims[2] + 7) // 8
            key = f"{es} {layout_of(bins)} {pool_of(p)}"
            for shape, tb in candidates(es, bins):
                force(lz, tmp_path, f"{key} 0 {vec_of(dims[2], es)} {bzb} -> {shape} {tb}")
                hits = lz.tune_hits()
                out = torch.full((lz.max_stream_bytes(dims, es),), 0xAB, dtype=torch.uint8, device="cuda")
                sl, rs = lz.compress_into(ws, d_in, dims, bins, p, out)
                assert sl == len(s_o), (dims, shape, tb)
                # the reference reports nb alone for stacks of at most 1024 blocks
                nb = dims[0] * ((dims[1] + 7) // 8) * bzb
                assert rs == rs_o or (nb <= 1024 and rs_o == nb), (dims, shape, tb)
                assert np.array_equal(out[:sl].cpu().numpy(), s_o), (dims, shape, tb)
                assert lz.tune_hits() == hits + 1 and len(lz.tune_table()) == 1
            stream = torch.from_numpy(s_o.copy()).cuda()
            for shape, tb in DEC_CANDIDATES[es]:
                force(lz, tmp_path, f"{key} 2 {vec_of(dims[2], es)} {bzb} -> {shape} {tb}")
                hits = lz.tune_hits()
                n = dims[0] * dims[1] * dims[2]
                dec = torch.full((n,), -1, dtype=torch.int16 if es == 2 else torch.int32, device="cuda")
                lz.decompress_into(ws, stream, len(s_o), dims, bins, p, dec)
                got = dec.cpu().numpy().view(dtype)
                assert np.array_equal(got, d_o.ravel()), (dims, tb)
                assert lz.tune_hits() == hits + 1 and len(lz.tune_table()) == 1
    finally:
        lz.tune_clear()
        lz.tune_mode(prev)


@pytest.mark.gpu
def test_autotune_times_candidates(lz, ws, oracle):
    prev = lz.tune_mode(1)
    try:
        lz.tune_clear()
        dims = (64, 256, 1024)  # 1024 tiles: large enough to be tuned
        a = random_stack(dims, seed=7)
        bins, p = LOSSY
        d_in = to_dev(a)
        out = torch.zeros(lz.max_stream_bytes(dims), dtype=torch.uint8, device="cuda")
        sl, rs = lz.compress_into(ws, d_in, dims, bins, p, out)
        s_o, rs_o = oracle.compress(a, dims, bins, p)
        assert np.array_equal(out[:sl].cpu().numpy(), s_o) and rs == rs_o
        tab = lz.tune_table()
        assert len(tab) == 1
        e = tab[0]
        assert (e["es"], e["layout"], e["pool"], e["kind"], e["vec"], e["bzb"]) == (2, 1, 1, "compress", 16, 128)
        assert [(t["shape"], t["tile_blocks"]) for t in e["times"]] == CANDIDATES[2]
        best = min(e["times"], key=lambda t: t["ms"])
        assert (e["shape"], e["tile_blocks"]) == (best["shape"], best["tile_blocks"])
        assert all(t["ms"] > 0 for t in e["times"])
        # a second call uses the table and tunes nothing
        hits = lz.tune_hits()
        lz.compress_into(ws, d_in, dims, bins, p, out)
        assert lz.tune_table() == tab and lz.tune_hits() == hits + 1
        # small stacks are never tuned
        small = (2, 64, 64)
        o_small = torch.zeros(lz.max_stream_bytes(small), dtype=torch.uint8, device="cuda")
        lz.compress_into(ws, to_dev(random_stack(small, seed=8)), small, bins, p, o_small)
        assert lz.tune_table() == tab
        # decompress and batch keys are tuned on their first call too
        dec = torch.empty(dims[0] * dims[1] * dims[2], dtype=torch.int16, device="cuda")
        lz.decompress_into(ws, out, sl, dims, bins, p, dec)
        assert np.array_equal(dec.cpu().numpy().view(np.uint16), oracle.decompress(s_o, dims, bins, p).ravel())
        o2 = torch.zeros_like(out)
        res = lz.compress_batch(ws, [(d_in, dims, out), (d_in, dims, o2)], bins, p)
        assert res == [(sl, rs), (sl, rs)]
        assert torch.equal(out[:sl], o2[:sl])
        kinds = sorted(t["kind"] for t in lz.tune_table())
        assert kinds == ["batch", "compress", "decompress"]
    finally:
        lz.tune_clear()
        lz.tune_mode(prev)


@pytest.mark.gpu
@pytest.mark.parametrize("bins,p", [LOSSLESS, LOSSY])
def test_plan_replays(lz, ws, bins, p):
    shapes = [(1, 8, 8), (3, 37, 53), (2, 100, 130), (1, 9, 2049), (5, 31, 7), (4, 64, 64)]
    arrays = [random_stack(d, seed=i) for i, d in enumerate(shapes)]
    ins = [to_dev(a) for a in arrays]
    outs = [torch.zeros(lz.max_stream_bytes(d), dtype=torch.uint8, device="cuda") for d in shapes]
    plan = lz.Plan(ws, list(zip(ins, shapes, outs)), bins, p)
    try:
        for rnd in range(3):
            if rnd:
                # new contents in the same buffers
                for i, (d, t) in enumerate(zip(shapes, ins)):
                    t.copy_(to_dev(random_stack(d, seed=1000 * rnd + i)))
                for o in outs:
                    o.fill_(0xCD)
            res = plan.run()
            for d_in, dims, out, (sl, rs) in zip(ins, shapes, outs, res):
                ref = torch.zeros_like(out)
                sl1, rs1 = lz.compress_into(ws, d_in, dims, bins, p, ref)
                assert (sl, rs) == (sl1, rs1), (rnd, dims)
                assert torch.equal(out[:sl], ref[:sl]), (rnd, dims)
    finally:
        plan.close()


@pytest.mark.gpu
@pytest.mark.parametrize("es", [2, 4])
def test_plan_single_stack(lz, ws, oracle, es):
    dtype = np.uint16 if es == 2 else np.uint32
    dims = (6, 181, 1558)
    bins, p = LOSSY
    a = random_stack(dims, seed=3, dtype=dtype)
    d_in = to_dev(a)
    out = torch.zeros(lz.max_stream_bytes(dims, es), dtype=torch.uint8, device="cuda")
    plan = lz.Plan(ws, [(d_in, dims, out)], bins, p)
    try:
        for rnd in range(2):
            out.fill_(0xEE)
            (sl, rs), = plan.run()
            s_o, rs_o = oracle.compress(a, dims, bins, p, dtype=dtype)
            assert sl == len(s_o) and rs == rs_o
            assert np.array_equal(out[:sl].cpu().numpy(), s_o)
            a = random_stack(dims, seed=50 + rnd, dtype=dtype)
            d_in.copy_(to_dev(a))
    finally:
        plan.close()


@pytest.mark.gpu
def test_plan_rejects_bad_arguments(lz, ws):
    dims = (2, 16, 16)
    d_in = to_dev(random_stack(dims, seed=1))
    small = torch.zeros(8, dtype=torch.uint8, device="cuda")
    with pytest.raises(lz.LscompError):
        lz.Plan(ws, [(d_in, dims, small)], *LOSSY)
    with pytest.raises(ValueError):
        lz.Plan(ws, [], *LOSSY)


@pytest.mark.gpu
def test_workspace_without_tuning(lz, oracle):
    prev = lz.tune_mode(1)
    ws2 = lz.Workspace(0)
    try:
        lz.tune_clear()
        ws2.set_tuning(False)
        dims = (64, 256, 1024)
        a = random_stack(dims, seed=9)
        out = torch.zeros(lz.max_stream_bytes(dims), dtype=torch.uint8, device="cuda")
        sl, _ = lz.compress_into(ws2, to_dev(a), dims, *LOSSLESS, out)
        assert lz.tune_table() == []
        s_o, _ = oracle.compress(a, dims, *LOSSLESS)
        assert np.array_equal(out[:sl].cpu().numpy(), s_o)
        ws2.set_tuning(True)
        lz.compress_into(ws2, to_dev(a), dims, *LOSSLESS, out)
        assert len(lz.tune_table()) == 1
    finally:
        ws2.close()
        lz.tune_clear()
        lz.tune_mode(prev)
