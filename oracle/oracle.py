"""TEST INFRASTRUCTURE: ctypes front ends for the two checkers.

* ``Oracle``  -- liblscomp_oracle.so, the C/OpenMP restatement of the lsCOMP
  codec in lscomp_oracle.c (see that file for the reference lines it follows).
* ``RefLib``  -- _ref/libculsz_ref.so, the unmodified reference CUDA sources
  built for sm_100a plus the C-linkage forwarders in ref_driver.cu.  It runs
  the reference's own host API on the GPU.

Only tests/, __graft_entry__.smoke() and bench.py (CPU baseline and the
reference arm) import this module.  The product library never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liblscomp_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libculsz_ref.so")
REF_LIB_DEFAULT = os.path.join(HERE, "_ref", "libculsz_ref_default.so")


class Oracle:
    def __init__(self, path: str = ORACLE_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle not built: {path} (make -C oracle oracle)")
        lib = ctypes.CDLL(path)
        vp, u32, f32, i32, sz = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_float, ctypes.c_int, ctypes.c_size_t
        psz = ctypes.POINTER(ctypes.c_size_t)
        for t in ("u16", "u32"):
            f = getattr(lib, f"lsc_oracle_compress_{t}")
            f.restype = i32
            f.argtypes = [vp, u32, u32, u32, vp, f32, vp, sz, psz, psz, i32]
            f = getattr(lib, f"lsc_oracle_decompress_{t}")
            f.restype = i32
            f.argtypes = [vp, sz, u32, u32, u32, vp, f32, vp, i32, i32]
        lib.lsc_oracle_pool_min_zeros.restype = i32
        lib.lsc_oracle_pool_min_zeros.argtypes = [f32]
        lib.lsc_oracle_max_threads.restype = i32
        lib.lsc_oracle_headers_u16.restype = i32
        lib.lsc_oracle_headers_u16.argtypes = [vp, u32, u32, u32, vp, f32, vp, vp]
        self.lib = lib

    @staticmethod
    def _bins(bins):
        return np.ascontiguousarray(np.asarray(bins, dtype=np.uint32))

    def max_threads(self) -> int:
        return int(self.lib.lsc_oracle_max_threads())

    def pool_min_zeros(self, p: float) -> int:
        return int(self.lib.lsc_oracle_pool_min_zeros(ctypes.c_float(p)))

    def compress(self, data: np.ndarray, dims, bins, p: float, threads: int = 0, dtype=np.uint16):
        """Returns (stream bytes as uint8 array, ref_size)."""
        x, y, z = (int(v) for v in dims)
        data = np.ascontiguousarray(data, dtype=dtype)
        nb = x * ((y + 7) // 8) * ((z + 7) // 8)
        per = 128 if dtype == np.uint16 else 256
        cap = (nb + 3) // 4 * 4 + per * nb
        out = np.empty(cap, dtype=np.uint8)
        sl, rs = ctypes.c_size_t(0), ctypes.c_size_t(0)
        b = self._bins(bins)
        t = "u16" if dtype == np.uint16 else "u32"
        st = getattr(self.lib, f"lsc_oracle_compress_{t}")(
            data.ctypes.data, x, y, z, b.ctypes.data, ctypes.c_float(p), out.ctypes.data, cap,
            ctypes.byref(sl), ctypes.byref(rs), threads)
        if st != 0:
            raise RuntimeError(f"oracle compress failed ({st})")
        return out[: sl.value].copy(), int(rs.value)

    def decompress(self, stream: np.ndarray, dims, bins, p: float, threads: int = 0, dtype=np.uint16,
                   write_zero_blocks: bool = True, out=None):
        x, y, z = (int(v) for v in dims)
        stream = np.ascontiguousarray(stream, dtype=np.uint8)
        if out is None:
            out = np.zeros(x * y * z, dtype=dtype)
        b = self._bins(bins)
        t = "u16" if dtype == np.uint16 else "u32"
        st = getattr(self.lib, f"lsc_oracle_decompress_{t}")(
            stream.ctypes.data, stream.size, x, y, z, b.ctypes.data, ctypes.c_float(p), out.ctypes.data,
            1 if write_zero_blocks else 0, threads)
        if st != 0:
            raise RuntimeError(f"oracle decompress failed ({st})")
        return out

    def headers(self, data: np.ndarray, dims, bins, p: float):
        x, y, z = (int(v) for v in dims)
        nb = x * ((y + 7) // 8) * ((z + 7) // 8)
        data = np.ascontiguousarray(data, dtype=np.uint16)
        hdr = np.empty(nb, dtype=np.uint8)
        sizes = np.empty(nb, dtype=np.uint32)
        b = self._bins(bins)
        st = self.lib.lsc_oracle_headers_u16(data.ctypes.data, x, y, z, b.ctypes.data, ctypes.c_float(p),
                                             hdr.ctypes.data, sizes.ctypes.data)
        if st != 0:
            raise RuntimeError(f"oracle headers failed ({st})")
        return hdr, sizes


class RefLib:
    """The reference's own host API (GPU), through ref_driver.cu."""

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference build missing: {path} (make -C oracle ref)")
        lib = ctypes.CDLL(path)
        vp, u32, f32, sz = ctypes.c_void_p, ctypes.c_uint, ctypes.c_float, ctypes.c_size_t
        for t in ("u16", "u32"):
            f = getattr(lib, f"ref_compress_{t}")
            f.restype = ctypes.c_int
            f.argtypes = [vp, vp, ctypes.POINTER(sz), u32, u32, u32, vp, f32, vp]
            f = getattr(lib, f"ref_decompress_{t}")
            f.restype = ctypes.c_int
            f.argtypes = [vp, vp, sz, u32, u32, u32, vp, f32, vp]
        self.lib = lib
        self._keep = []

    def compress(self, d_in_ptr: int, d_cmp_ptr: int, dims, bins, p: float, stream: int = 0, t: str = "u16"):
        x, y, z = (int(v) for v in dims)
        b = (ctypes.c_uint * 4)(*[int(v) for v in bins])
        cs = ctypes.c_size_t(0)
        st = getattr(self.lib, f"ref_compress_{t}")(ctypes.c_void_p(d_in_ptr), ctypes.c_void_p(d_cmp_ptr),
                                                      ctypes.byref(cs), x, y, z, b, ctypes.c_float(p),
                                                      ctypes.c_void_p(stream))
        if st != 0:
            raise RuntimeError(f"reference compress: cuda error {st}")
        return int(cs.value)

    def decompress(self, d_out_ptr: int, d_cmp_ptr: int, cmp_size: int, dims, bins, p: float, stream: int = 0,
                   t: str = "u16"):
        x, y, z = (int(v) for v in dims)
        b = (ctypes.c_uint * 4)(*[int(v) for v in bins])
        st = getattr(self.lib, f"ref_decompress_{t}")(ctypes.c_void_p(d_out_ptr), ctypes.c_void_p(d_cmp_ptr),
                                                        ctypes.c_size_t(cmp_size), x, y, z, b, ctypes.c_float(p),
                                                        ctypes.c_void_p(stream))
        if st != 0:
            raise RuntimeError(f"reference decompress: cuda error {st}")
