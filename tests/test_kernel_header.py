"""GPU parity of the kernels of include/cuLSZ_kernel.h (the reference's public
kernel header, lsCOMP/include/cuLSZ_kernel.h:9-36), launched as a caller of
that header launches them: one 32-thread CTA per 1024 blocks and three
zeroed scratch arrays (tests/culsz_kernel_driver.cu, built here with nvcc
and linked with liblscomp_kernels.a, the static archive of these kernels).

Streams must equal the oracle's byte for byte, the size read from
cmpOffset[grid] must be payload + nb (also for one-CTA grids, where the
reference leaves it 0), and decodes must equal the oracle's."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sc25-lscomp_b200")

LOSSLESS = ((1, 1, 1, 1), 1.0)
LOSSY = ((3, 5, 10, 15), 0.5)
SETTINGS = [LOSSLESS, LOSSY, ((9, 4, 12, 3), 0.5), ((1, 1, 1, 1), 0.0), ((5, 5, 5, 5), 0.3)]
SHAPES = [(1, 8, 8), (1, 1, 1), (3, 37, 53), (8, 128, 96), (64, 256, 256), (2, 17, 4100), (5, 31, 7)]


@pytest.fixture(scope="module")
def kdrv(tmp_path_factory):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lscomp

    lscomp.load_library()
    so = str(tmp_path_factory.mktemp("kdrv") / "libkdrv.so")
    # linked with the static kernel archive, as a program built against the
    # reference's static library links its kernels
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler",
                    "-fPIC", "-shared", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "culsz_kernel_driver.cu"), os.path.join(PKG, "liblscomp_kernels.a"),
                    "-o", so], check=True)
    lib = ctypes.CDLL(so)
    vp, u, f32 = ctypes.c_void_p, ctypes.c_uint, ctypes.c_float
    pint = ctypes.POINTER(ctypes.c_int)
    for t in ("u16", "u32"):
        getattr(lib, f"kdrv_compress_{t}").argtypes = [vp, vp, ctypes.POINTER(ctypes.c_size_t), u, u, u, vp, f32,
                                                       pint]
        getattr(lib, f"kdrv_decompress_{t}").argtypes = [vp, vp, u, u, u, vp, f32, pint]
    return lib


def stack(dims, seed, wide=False):
    rng = np.random.default_rng(seed)
    dt = np.uint32 if wide else np.uint16
    a = rng.integers(0, 1 << 20 if wide else 3000, size=dims, dtype=dt)
    a[rng.random(dims) < 0.5] = 0
    a[rng.random(dims) < 0.01] = (1 << 30) if wide else 65535
    return a


def run(kdrv, t, a, dims, bins, p):
    view, tt = (np.int32, torch.int32) if t == "u32" else (np.int16, torch.int16)
    d_in = torch.from_numpy(np.ascontiguousarray(a).view(view).ravel()).cuda()
    nb = dims[0] * ((dims[1] + 7) // 8) * ((dims[2] + 7) // 8)
    cap = (nb + 3) // 4 * 4 + (248 if t == "u32" else 128) * nb
    cmp = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    b = np.asarray(bins, dtype=np.uint32)
    cs, fl = ctypes.c_size_t(0), ctypes.c_int(0)
    st = getattr(kdrv, f"kdrv_compress_{t}")(d_in.data_ptr(), cmp.data_ptr(), ctypes.byref(cs), *dims,
                                             b.ctypes.data, ctypes.c_float(p), ctypes.byref(fl))
    assert st == 0
    dec = torch.full((a.size,), -1, dtype=tt, device="cuda")
    fl2 = ctypes.c_int(0)
    if fl.value >= 0:
        st = getattr(kdrv, f"kdrv_decompress_{t}")(dec.data_ptr(), cmp.data_ptr(), *dims, b.ctypes.data,
                                                   ctypes.c_float(p), ctypes.byref(fl2))
        assert st == 0 and fl2.value >= 0
    return cmp, int(cs.value), fl.value, dec.cpu().numpy().view(np.uint32 if t == "u32" else np.uint16), nb


@pytest.mark.parametrize("dims", SHAPES)
@pytest.mark.parametrize("bins,p", SETTINGS)
def test_kernel_header_u16_vs_oracle(kdrv, oracle, dims, bins, p):
    a = stack(dims, seed=hash((dims, bins, p)) & 0xffff)
    s_o, _ = oracle.compress(a, dims, bins, p)
    cmp, cs, fl, dec, nb = run(kdrv, "u16", a, dims, bins, p)
    assert fl >= 0
    assert cs == len(s_o) - (nb + 3) // 4 * 4 + nb  # payload + nb
    assert np.array_equal(cmp[:len(s_o)].cpu().numpy(), s_o)
    assert np.array_equal(dec, oracle.decompress(s_o, dims, bins, p))


@pytest.mark.parametrize("dims", [(1, 8, 8), (3, 37, 53), (2, 17, 1100), (4, 64, 64)])
@pytest.mark.parametrize("bins,p", [LOSSLESS, LOSSY, ((9, 4, 12, 3), 0.5)])
def test_kernel_header_u32_vs_oracle(kdrv, oracle, dims, bins, p):
    a = stack(dims, seed=hash((dims, bins, p, 32)) & 0xffff, wide=True)
    s_o, _ = oracle.compress(a, dims, bins, p, dtype=np.uint32)
    cmp, cs, fl, dec, nb = run(kdrv, "u32", a, dims, bins, p)
    assert fl >= 0
    assert cs == len(s_o) - (nb + 3) // 4 * 4 + nb
    assert np.array_equal(cmp[:len(s_o)].cpu().numpy(), s_o)
    assert np.array_equal(dec, oracle.decompress(s_o, dims, bins, p, dtype=np.uint32))


def test_kernel_header_u32_range_reported(kdrv):
    """A quotient that needs 32 bit planes: the launch is aborted (sign bit of
    flag[grid]) instead of writing a header the 5-bit rate field cannot hold."""
    a = np.zeros((1, 8, 8), dtype=np.uint32)
    a[0, 0, 0] = 0xFFFFFFFF
    _, _, fl, _, _ = run(kdrv, "u32", a, (1, 8, 8), *LOSSLESS)
    assert fl < 0
