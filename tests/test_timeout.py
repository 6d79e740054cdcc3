"""Device-side failure detection without a GPU fault.

Every wait in the kernels is bounded and watches a launch-wide abort flag;
the reference's look-back spins without a bound
(lsCOMP/src/cuLSZ_kernel.cu:1001-1004).  Here one launch is made to wait for
a look-back predecessor that never publishes: lscomp_workspace_stall_next
starts the launch's tile tickets at 1, so tile 0 (the decoder's offsets
kernel: segment 0) is never claimed, and limits every wait to a short time.
The call must come back with LSCOMP_ERR_TIMEOUT after about that limit --
no trap, no hang -- and the same workspace must serve the next call
normally."""
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TIMEOUT = 4
WAIT_NS = 50_000_000  # 50 ms, against the default limit of 2 s


@pytest.fixture(scope="module")
def lz():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lscomp

    lscomp.load_library()
    return lscomp


@pytest.mark.parametrize("bins,p", [((1, 1, 1, 1), 1.0), ((3, 5, 10, 15), 0.5)])
def test_lookback_timeout_then_recovery(lz, oracle, bins, p):
    dims = (64, 256, 256)  # 256 tiles of 256 blocks: 8 segments of the offsets kernel
    a = lz.synth_small(dims, seed=3)
    d_in = torch.from_numpy(a.view(np.int16)).cuda()
    ws = lz.Workspace(0)
    ws.set_tuning(False)  # a tuning run would take the injected launch
    out = torch.zeros(lz.max_stream_bytes(dims), dtype=torch.uint8, device="cuda")

    ws.stall_next(WAIT_NS)
    t0 = time.perf_counter()
    with pytest.raises(lz.LscompError) as e:
        lz.compress_into(ws, d_in, dims, bins, p, out)
    took = time.perf_counter() - t0
    assert e.value.status == TIMEOUT
    assert took < 1.5, f"the encoder's look-back waited {took:.2f} s, not the injected limit"

    # the next ordinary call on the same workspace is exact
    sl, _ = lz.compress_into(ws, d_in, dims, bins, p, out)
    s_o, _ = oracle.compress(a, dims, bins, p)
    assert np.array_equal(out[:sl].cpu().numpy(), s_o)

    dec = torch.empty_like(d_in)
    ws.stall_next(WAIT_NS)
    t0 = time.perf_counter()
    with pytest.raises(lz.LscompError) as e:
        lz.decompress_into(ws, out, sl, dims, bins, p, dec)
    took = time.perf_counter() - t0
    assert e.value.status == TIMEOUT
    assert took < 1.5, f"the decoder's look-back waited {took:.2f} s, not the injected limit"

    dec.fill_(-1)
    lz.decompress_into(ws, out, sl, dims, bins, p, dec)
    assert np.array_equal(dec.cpu().numpy().view(np.uint16), oracle.decompress(s_o, dims, bins, p))
    ws.close()


def test_stall_next_argument_checks(lz):
    ws = lz.Workspace(0)
    for bad in (0, 999_999, 2_000_000_001):
        with pytest.raises(lz.LscompError) as e:
            ws.stall_next(bad)
        assert e.value.status == 1
    ws.close()
