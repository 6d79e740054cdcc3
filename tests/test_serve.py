"""The serving loop (lscomp_server_*): host buffers in and out, admission
into a fixed device arena, continuous batching of compress requests.

A served request's output must not depend on what it was batched with: every
served container is compared byte for byte with lscomp_compress_container on
the same stack alone, and decompress requests with the stack."""
import threading

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


def stack(dims, seed, wide=False):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 300, size=dims, dtype=np.uint32 if wide else np.uint16)
    a[rng.random(dims) < 0.5] = 0
    return a


def alone(lz, ws, a, dims, bins, p):
    """Container of one stack made by the single-stack call."""
    view = np.int32 if a.itemsize == 4 else np.int16
    d_in = torch.from_numpy(np.ascontiguousarray(a).view(view).ravel()).cuda()
    out = torch.zeros(64 + lz.max_stream_bytes(dims, a.itemsize), dtype=torch.uint8, device="cuda")
    n = lz.compress_container(ws, d_in, dims, bins, p, out)
    return out[:n].cpu().numpy()


def requests(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        dims = (int(rng.integers(1, 6)), int(rng.integers(1, 300)), int(rng.integers(1, 400)))
        wide = bool(i % 5 == 4)
        bins, p = (LOSSLESS, LOSSY, ((5, 10, 15, 20), 0.3))[i % 3]
        out.append((stack(dims, seed * 1000 + i, wide), dims, bins, p))
    return out


def test_alone_vs_mix_bit_exact(lz):
    reqs = requests(60, seed=1)
    ws = lz.Workspace(0)
    srv = lz.Server(0, arena_bytes=1 << 30)
    outs, ids = [], []
    for a, dims, bins, p in reqs:  # all submitted before any is waited for: mixed rounds
        o = np.zeros(64 + lz.max_stream_bytes(dims, a.itemsize), dtype=np.uint8)
        outs.append(o)
        ids.append(srv.submit_compress(a, dims, bins, p, o))
    res = [srv.wait(i) for i in ids]
    st = srv.stats()
    assert st["batched_requests"] == len(reqs) and st["batches"] < len(reqs)  # requests were batched
    for (a, dims, bins, p), o, r in zip(reqs, outs, res):
        assert r["status"] == 0
        ref = alone(lz, ws, a, dims, bins, p)
        assert r["out_len"] == len(ref)
        assert np.array_equal(o[: r["out_len"]], ref)
    # and back: decompress requests of the served containers
    decs, ids = [], []
    for (a, dims, bins, p), o, r in zip(reqs, outs, res):
        d = np.zeros_like(a)
        decs.append(d)
        ids.append(srv.submit_decompress(o[: r["out_len"]], d))
    for (a, dims, bins, p), d, i, o, r in zip(reqs, decs, ids, outs, res):
        rr = srv.wait(i)
        assert rr["status"] == 0 and rr["out_len"] == a.nbytes
        if bins == (1, 1, 1, 1):
            assert np.array_equal(d, a)
        else:
            view = np.int32 if a.itemsize == 4 else np.int16
            cont = torch.from_numpy(o[: r["out_len"]].copy()).cuda()
            ref = torch.empty(a.size, dtype=torch.int32 if a.itemsize == 4 else torch.int16, device="cuda")
            lz.decompress_container(ws, cont, r["out_len"], ref)
            assert np.array_equal(d.view(view).ravel(), ref.cpu().numpy())
    srv.close()


def test_admission_small_arena(lz):
    # the arena holds only a few requests at a time: many rounds, same outputs
    reqs = requests(40, seed=2)
    ws = lz.Workspace(0)
    srv = lz.Server(0, arena_bytes=8 << 20)
    outs = [np.zeros(64 + lz.max_stream_bytes(d, a.itemsize), dtype=np.uint8) for a, d, _, _ in reqs]
    ids = [srv.submit_compress(a, d, b, p, o) for (a, d, b, p), o in zip(reqs, outs)]
    res = [srv.wait(i) for i in ids]
    assert srv.stats()["rounds"] > 1
    for (a, d, b, p), o, r in zip(reqs, outs, res):
        assert r["status"] == 0
        assert np.array_equal(o[: r["out_len"]], alone(lz, ws, a, d, b, p))
    # larger than the whole arena: refused at submission
    big = np.zeros((16, 512, 512), dtype=np.uint16)
    with pytest.raises(lz.LscompError) as e:
        srv.submit_compress(big, big.shape, *LOSSLESS, np.zeros(1 << 24, dtype=np.uint8))
    assert e.value.status == 8
    # output buffer too small for the container: that request fails alone
    a, d, b, p = reqs[0]
    rid = srv.submit_compress(a, d, b, p, np.zeros(70, dtype=np.uint8))
    assert srv.wait(rid)["status"] == 2
    srv.close()


def test_threads(lz):
    reqs = requests(48, seed=3)
    ws = lz.Workspace(0)
    srv = lz.Server(0, arena_bytes=256 << 20)
    outs = [np.zeros(64 + lz.max_stream_bytes(d, a.itemsize), dtype=np.uint8) for a, d, _, _ in reqs]
    results = [None] * len(reqs)

    def client(k):
        for i in range(k, len(reqs), 4):
            a, d, b, p = reqs[i]
            results[i] = srv.wait(srv.submit_compress(a, d, b, p, outs[i]))

    th = [threading.Thread(target=client, args=(k,)) for k in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for (a, d, b, p), o, r in zip(reqs, outs, results):
        assert r["status"] == 0
        assert np.array_equal(o[: r["out_len"]], alone(lz, ws, a, d, b, p))
    srv.close()


def test_bad_request_fails_alone(lz):
    """A uint32 request whose quotient needs 32 bit planes (the 5-bit rate
    field cannot say so: LSCOMP_ERR_RANGE) is batched with valid requests;
    only it fails, and the others' containers equal the single calls'."""
    reqs = requests(12, seed=4)
    bad = np.zeros((1, 8, 8), dtype=np.uint32)
    bad[0, 0, 0] = 0xFFFFFFFF
    ws = lz.Workspace(0)
    srv = lz.Server(0, arena_bytes=1 << 30)
    # two uint32 requests around the bad one, so it shares their batch
    reqs.insert(3, (bad, bad.shape, LOSSLESS[0], 1.0))
    reqs.insert(2, (stack((2, 17, 33), 77, wide=True), (2, 17, 33), *LOSSY))
    reqs.insert(5, (stack((1, 40, 9), 78, wide=True), (1, 40, 9), *LOSSLESS))
    outs = [np.zeros(64 + lz.max_stream_bytes(d, a.itemsize), dtype=np.uint8) for a, d, _, _ in reqs]
    ids = [srv.submit_compress(a, d, b, p, o) for (a, d, b, p), o in zip(reqs, outs)]
    res = [srv.wait(i) for i in ids]
    for (a, d, b, p), o, r in zip(reqs, outs, res):
        if a is bad:
            assert r["status"] == 6 and r["out_len"] == 0
        else:
            assert r["status"] == 0
            assert np.array_equal(o[: r["out_len"]], alone(lz, ws, a, d, b, p))
    srv.close()


def test_admitted_while_others_in_flight(lz):
    """A request submitted while a large one is being served is admitted
    (and so starts its upload) before the large one completes."""
    srv = lz.Server(0, arena_bytes=4 << 30)
    big = np.random.default_rng(9).integers(0, 50, size=(64, 1024, 1024), dtype=np.uint16)  # 128 MB
    small = stack((1, 64, 64), 10)
    ob = np.zeros(64 + lz.max_stream_bytes(big.shape), dtype=np.uint8)
    os_ = np.zeros(64 + lz.max_stream_bytes(small.shape), dtype=np.uint8)
    rb = srv.submit_compress(big, big.shape, *LOSSY, ob)
    rs = srv.submit_compress(small, small.shape, *LOSSLESS, os_)
    r_small, r_big = srv.wait(rs), srv.wait(rb)
    assert r_small["status"] == 0 and r_big["status"] == 0
    assert r_small["admit_ns"] < r_big["done_ns"]
    srv.close()


def test_second_waiter_refused(lz):
    """Two threads wait for the same request: one gets the result, the other
    LSCOMP_ERR_ARG (while the first waits, or after it released the request)."""
    srv = lz.Server(0, arena_bytes=1 << 30)
    a = np.random.default_rng(12).integers(0, 50, size=(32, 1024, 1024), dtype=np.uint16)
    o = np.zeros(64 + lz.max_stream_bytes(a.shape), dtype=np.uint8)
    rid = srv.submit_compress(a, a.shape, *LOSSLESS, o)
    got = []

    def waiter():
        try:
            got.append(srv.wait(rid)["status"])
        except lz.LscompError as e:
            got.append(-e.status)

    th = [threading.Thread(target=waiter) for _ in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert sorted(got) == [-1, 0]
    srv.close()


def pinned(a):
    """A copy of a in page-locked host memory (a numpy view of a pinned
    tensor, which the view keeps alive)."""
    v = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True).numpy().view(a.dtype).reshape(a.shape)
    v[...] = a
    return v


def test_pinned_buffers_direct(lz):
    """Page-locked client buffers are copied by the device directly (no
    staging): mixed with pageable ones in the same batches, every container
    still equals the single-call container and every decode the input;
    stacks larger than one staging slot (32 MB) included."""
    reqs = requests(24, seed=7)
    rng = np.random.default_rng(8)
    big = rng.integers(0, 40, size=(24, 1024, 1024), dtype=np.uint16)  # 48 MB: more than one slot
    reqs.append((big, big.shape, LOSSLESS[0], LOSSLESS[1]))
    ws = lz.Workspace(0)
    srv = lz.Server(0, arena_bytes=1 << 30)
    ins, outs, ids = [], [], []
    for i, (a, dims, bins, p) in enumerate(reqs):
        pin_in, pin_out = i % 2 == 0, i % 3 != 1  # every combination of pinned and pageable
        h_in = pinned(a) if pin_in else a
        o = np.zeros(64 + lz.max_stream_bytes(dims, a.itemsize), dtype=np.uint8)
        o = pinned(o) if pin_out else o
        ins.append(h_in)
        outs.append(o)
        ids.append(srv.submit_compress(h_in, dims, bins, p, o))
    res = [srv.wait(i) for i in ids]
    conts = []
    for (a, dims, bins, p), o, r in zip(reqs, outs, res):
        assert r["status"] == 0
        ref = alone(lz, ws, a, dims, bins, p)
        assert r["out_len"] == len(ref)
        assert np.array_equal(o[: r["out_len"]], ref)
        conts.append(ref)
    decs, ids = [], []
    for i, ((a, dims, bins, p), c) in enumerate(zip(reqs, conts)):
        c_in = pinned(c) if i % 3 == 0 else c
        d = np.full(a.shape, 0xFF, dtype=a.dtype)
        d = pinned(d) if i % 2 == 1 else d
        decs.append((c_in, d))
        ids.append(srv.submit_decompress(c_in, d))
    for (a, dims, bins, p), (c_in, d), i in zip(reqs, decs, ids):
        r = srv.wait(i)
        assert r["status"] == 0
        if bins == LOSSLESS[0]:
            assert np.array_equal(d, a)
        else:
            view = np.int32 if a.itemsize == 4 else np.int16
            cont = torch.from_numpy(np.array(c_in)).cuda()
            ref = torch.empty(a.size, dtype=torch.int32 if a.itemsize == 4 else torch.int16, device="cuda")
            lz.decompress_container(ws, cont, len(c_in), ref)
            assert np.array_equal(d.view(view).ravel(), ref.cpu().numpy())
    srv.close()
