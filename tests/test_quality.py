"""Lossy quality report (PSNR / SSIM with the definitions of the reference's
host utilities, lsCOMP/src/cuLSZ_utility.cu:757-946).

CPU: this library's host computePSNR / computeSSIM (include/cuLSZ_utility.h)
equal, double for double, the reference's own functions built from its
sources (oracle/_ref/libculsz_util_ref.so).  GPU: lscomp_quality_* equals the
host functions up to the order of the final sums."""
import ctypes
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "sc25-lscomp_b200", "liblscomp.so")
REF = os.path.join(ROOT, "oracle", "_ref", "libculsz_util_ref.so")


def host_fns(path):
    lib = ctypes.CDLL(path)
    psnr = getattr(lib, "_Z11computePSNRmPfS_")
    psnr.restype = ctypes.POINTER(ctypes.c_double)
    psnr.argtypes = [ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    ssim = getattr(lib, "_Z11computeSSIMPfS_mmm")
    ssim.restype = ctypes.c_double
    ssim.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t]
    return psnr, ssim


def host_report(path, a, b):
    psnr, ssim = host_fns(path)
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    p = psnr(a.size, a.ctypes.data, b.ctypes.data)
    return [p[i] for i in range(6)], ssim(a.ctypes.data, b.ctypes.data, *a.shape)


def pair(dims, seed, noise=3, top=4000):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, top, size=dims).astype(np.uint16)
    b = np.clip(a.astype(np.int64) + rng.integers(-noise, noise + 1, size=dims), 0, 65535).astype(np.uint16)
    return a, b


@pytest.mark.skipif(not os.path.exists(REF), reason="reference utilities not built (oracle/Makefile ref)")
@pytest.mark.parametrize("dims", [(7, 7, 7), (9, 21, 17), (12, 33, 40), (8, 10, 30)])
def test_host_functions_equal_reference(dims):
    a, b = pair(dims, seed=sum(dims))
    po, so = host_report(OURS, a, b)
    pr, sr = host_report(REF, a, b)
    assert po == pr
    assert so == sr


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(7, 7, 7), (9, 21, 17), (16, 64, 70), (3, 40, 40)])
def test_gpu_quality_equals_host(dims):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lscomp

    a, b = pair(dims, seed=7 + sum(dims))
    da = torch.from_numpy(a.view(np.int16).ravel()).cuda()
    db = torch.from_numpy(b.view(np.int16).ravel()).cuda()
    q = lscomp.quality(da, db, dims)
    p, s = host_report(OURS, a, b)
    got = [q["mse"], q["range"], q["psnr"], q["l2_error"], q["l2_error_rel"], q["nrmse"]]
    assert np.allclose(got, p, rtol=1e-12, atol=0)
    if min(dims) < 7:
        assert np.isnan(q["ssim"]) and np.isnan(s)
    else:
        assert abs(q["ssim"] - s) <= 1e-12


@pytest.mark.gpu
def test_gpu_quality_of_a_lossy_round_trip():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lscomp

    dims = (8, 181, 155)
    a = lscomp.synth_cssi(dims, seed=3).reshape(dims)
    d = torch.from_numpy(a.view(np.int16).ravel()).cuda()
    ws = lscomp.Workspace(0)
    out = torch.zeros(lscomp.max_stream_bytes(dims), dtype=torch.uint8, device="cuda")
    sl, _ = lscomp.compress_into(ws, d, dims, (3, 5, 10, 15), 0.5, out)
    dec = torch.empty_like(d)
    lscomp.decompress_into(ws, out, sl, dims, (3, 5, 10, 15), 0.5, dec)
    q = lscomp.quality(d, dec, dims)
    p, s = host_report(OURS, a, dec.cpu().numpy().view(np.uint16).reshape(dims))
    assert np.allclose([q["mse"], q["psnr"]], [p[0], p[2]], rtol=1e-12)
    assert abs(q["ssim"] - s) <= 1e-12
    assert 0 < q["ssim"] <= 1 and q["psnr"] > 20
