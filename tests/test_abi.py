"""CPU checks of the drop-in boundary: liblscomp.so loads without a GPU and
exports every entry point the public headers declare (the C ABI by name,
the reference-compatible C++ API by its mangled names, which must equal the
reference's own)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "sc25-lscomp_b200", "liblscomp.so")

# Itanium-mangled names of lsCOMP/include/cuLSZ_entry.h:8-11 (uint3/uint4 by
# value, CUstream_st* stream)
REFERENCE_MANGLED = [
    "_Z32cuLSZ_compression_uint16_bsize64PtPhPm5uint35uint4fP11CUstream_st",
    "_Z34cuLSZ_decompression_uint16_bsize64PtPhm5uint35uint4fP11CUstream_st",
    "_Z32cuLSZ_compression_uint32_bsize64PjPhPm5uint35uint4fP11CUstream_st",
    "_Z34cuLSZ_decompression_uint32_bsize64PjPhm5uint35uint4fP11CUstream_st",
]


def c_functions(header):
    text = open(os.path.join(INC, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lscomp_\w+)\s*\(", text)))


def exported():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_library_loads_without_gpu():
    lib = ctypes.CDLL(LIB)
    lib.lscomp_version.restype = ctypes.c_int
    assert lib.lscomp_version() >= 100
    lib.lscomp_block_count.restype = ctypes.c_uint64
    lib.lscomp_block_count.argtypes = [ctypes.c_uint32] * 3
    assert lib.lscomp_block_count(600, 1813, 1558) == 26559000
    lib.lscomp_max_stream_bytes_u16.restype = ctypes.c_uint64
    lib.lscomp_max_stream_bytes_u16.argtypes = [ctypes.c_uint32] * 3
    assert lib.lscomp_max_stream_bytes_u16(1, 8, 8) == 4 + 128


@pytest.mark.parametrize("header", sorted(h for h in os.listdir(INC) if h.startswith("lscomp")))
def test_c_abi_exports_every_declared_function(header):
    names = c_functions(header)
    assert names, header
    missing = [n for n in names if n not in exported()]
    assert not missing, missing


def test_reference_cpp_api_exported():
    syms = exported()
    missing = [m for m in REFERENCE_MANGLED if m not in syms]
    assert not missing, missing


def test_status_strings():
    lib = ctypes.CDLL(LIB)
    lib.lscomp_status_string.restype = ctypes.c_char_p
    for s in range(8):
        assert lib.lscomp_status_string(s)


# host-side launch stubs of the four __global__ kernels of
# lsCOMP/include/cuLSZ_kernel.h:9-36 (include/cuLSZ_kernel.h)
REFERENCE_KERNELS = [
    "_Z39cuLSZ_compression_kernel_uint16_bsize64PKtPhPVmS3_PVij5uint35uint4f",
    "_Z41cuLSZ_decompression_kernel_uint16_bsize64PtPKhPVmS3_PVij5uint35uint4f",
    "_Z39cuLSZ_compression_kernel_uint32_bsize64PKjPhPVjS3_PVij5uint35uint4f",
    "_Z41cuLSZ_decompression_kernel_uint32_bsize64PjPKhPVjS3_PVij5uint35uint4f",
]


def test_reference_kernel_header_in_archive():
    """The kernels of include/cuLSZ_kernel.h are defined in the static archive
    callers link (liblscomp_kernels.a), with the reference's mangled names."""
    arc = os.path.join(ROOT, "sc25-lscomp_b200", "liblscomp_kernels.a")
    out = subprocess.run(["nm", "--defined-only", arc], capture_output=True, text=True, check=True).stdout
    syms = {line.split()[-1] for line in out.splitlines() if len(line.split()) >= 3}
    missing = [m for m in REFERENCE_KERNELS if m not in syms]
    assert not missing, missing
