"""Python host interface of the B200 lsCOMP codec (uint16 detector stacks).

Mirrors the reference's host API (lsCOMP/include/cuLSZ_entry.h:8-11):

    compress(data, dims, bins, pooling)   ~ cuLSZ_compression_uint16_bsize64
    decompress(stream, dims, bins, pooling) ~ cuLSZ_decompression_uint16_bsize64

with the same argument meaning (dims = (x, y, z), z fastest; four
quantisation bins; the -p pooling threshold) and the same stream format.
Device buffers are torch tensors on a CUDA device (uint16 data is carried in
int16 tensors, bit for bit).  Every call goes through the C ABI of
liblscomp.so (include/lscomp.h); there is no other implementation, so a
missing or unloadable library raises instead of falling back.

The synthetic stack generators used by the tests and the benchmark live in
liblscomp_synth.so and are exposed as synth_small / synth_cssi / synth_xpcs.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# LSCOMP_LIBRARY selects another build of the same library (tuning variants)
LIB_PATH = os.environ.get("LSCOMP_LIBRARY", os.path.join(_HERE, "liblscomp.so"))
SYNTH_PATH = os.path.join(_HERE, "liblscomp_synth.so")

STATUS = {
    0: "ok",
    1: "invalid argument",
    2: "buffer too small for the stream",
    3: "CUDA runtime error",
    4: "bounded wait in kernel timed out",
    5: "stream inconsistent with the geometry",
    6: "value range not representable",
    7: "out of memory",
    8: "stack too large for the fixed scratch area",
}


class LscompError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, 'unknown')} (status {status})")


_lib = None
_synth_lib = None


class ContainerInfo(ctypes.Structure):
    """struct lscomp_container_info of include/lscomp.h."""
    _fields_ = [("elem_bytes", ctypes.c_uint32), ("x", ctypes.c_uint32), ("y", ctypes.c_uint32),
                ("z", ctypes.c_uint32), ("bins", ctypes.c_uint32 * 4), ("pooling", ctypes.c_float),
                ("stream_len", ctypes.c_uint64), ("ref_size", ctypes.c_uint64)]

    def as_dict(self):
        return {"elem_bytes": self.elem_bytes, "dims": (self.x, self.y, self.z), "bins": tuple(self.bins),
                "pooling": self.pooling, "stream_len": self.stream_len, "ref_size": self.ref_size}


class ServerResult(ctypes.Structure):
    """struct lscomp_server_result of include/lscomp.h."""
    _fields_ = [("status", ctypes.c_int), ("out_len", ctypes.c_uint64), ("queued_ns", ctypes.c_uint64),
                ("service_ns", ctypes.c_uint64), ("admit_ns", ctypes.c_uint64), ("done_ns", ctypes.c_uint64)]


class LscompStack(ctypes.Structure):
    """struct lscomp_stack of include/lscomp.h (one stack of a batch)."""
    _fields_ = [("d_in", ctypes.c_void_p), ("x", ctypes.c_uint32), ("y", ctypes.c_uint32), ("z", ctypes.c_uint32),
                ("d_out", ctypes.c_void_p), ("cap", ctypes.c_uint64)]


def _u32(x):
    return ctypes.c_uint32(int(x))


def load_library() -> ctypes.CDLL:
    """Load liblscomp.so (built by `make -C sc25-lscomp_b200`)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"liblscomp.so not built: {LIB_PATH} (run __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    vp, u32, u64, f32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_float
    pu64 = ctypes.POINTER(ctypes.c_uint64)
    bins_t = ctypes.POINTER(ctypes.c_uint32)
    lib.lscomp_version.restype = ctypes.c_int
    lib.lscomp_status_string.restype = ctypes.c_char_p
    lib.lscomp_status_string.argtypes = [ctypes.c_int]
    lib.lscomp_block_count.restype = u64
    lib.lscomp_block_count.argtypes = [u32, u32, u32]
    lib.lscomp_max_stream_bytes_u16.restype = u64
    lib.lscomp_max_stream_bytes_u16.argtypes = [u32, u32, u32]
    lib.lscomp_launch_count.restype = u64
    lib.lscomp_workspace_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int]
    lib.lscomp_workspace_destroy.argtypes = [vp]
    lib.lscomp_workspace_check.argtypes = [vp, vp]
    lib.lscomp_workspace_set_tuning.argtypes = [vp, ctypes.c_int]
    lib.lscomp_workspace_set_host_chunk.argtypes = [vp, u64]
    lib.lscomp_compress_u16.argtypes = [vp, vp, u32, u32, u32, bins_t, f32, vp, u64, pu64, pu64, vp]
    lib.lscomp_compress_u16_async.argtypes = [vp, vp, u32, u32, u32, bins_t, f32, vp, u64, vp, vp]
    lib.lscomp_decompress_u16.argtypes = [vp, vp, u64, u32, u32, u32, bins_t, f32, vp, vp]
    lib.lscomp_decompress_u16_async.argtypes = [vp, vp, u64, u32, u32, u32, bins_t, f32, vp, vp]
    lib.lscomp_max_stream_bytes_u32.restype = u64
    lib.lscomp_max_stream_bytes_u32.argtypes = [u32, u32, u32]
    lib.lscomp_compress_u32.argtypes = [vp, vp, u32, u32, u32, bins_t, f32, vp, u64, pu64, pu64, vp]
    lib.lscomp_compress_u32_async.argtypes = [vp, vp, u32, u32, u32, bins_t, f32, vp, u64, vp, vp]
    lib.lscomp_decompress_u32.argtypes = [vp, vp, u64, u32, u32, u32, bins_t, f32, vp, vp]
    lib.lscomp_decompress_u32_async.argtypes = [vp, vp, u64, u32, u32, u32, bins_t, f32, vp, vp]
    lib.lscomp_container_header_bytes.restype = u32
    lib.lscomp_container_write_header.argtypes = [vp, u32, u32, u32, u32, bins_t, f32, u64, u64]
    lib.lscomp_container_read_header.argtypes = [vp, u64, ctypes.POINTER(ContainerInfo)]
    lib.lscomp_compress_container.argtypes = [vp, u32, vp, u32, u32, u32, bins_t, f32, vp, u64, pu64, vp]
    lib.lscomp_decompress_container.argtypes = [vp, vp, u64, vp, u64, ctypes.POINTER(ContainerInfo), vp]
    lib.lscomp_server_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, u64]
    lib.lscomp_server_destroy.argtypes = [vp]
    lib.lscomp_server_submit_compress.restype = ctypes.c_int64
    lib.lscomp_server_submit_compress.argtypes = [vp, u32, vp, u32, u32, u32, bins_t, f32, vp, u64]
    lib.lscomp_server_submit_decompress.restype = ctypes.c_int64
    lib.lscomp_server_submit_decompress.argtypes = [vp, vp, u64, vp, u64]
    lib.lscomp_server_wait.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(ServerResult)]
    lib.lscomp_server_stats.argtypes = [vp, pu64, pu64, pu64]
    for sfx in ("u16", "u32"):
        getattr(lib, f"lscomp_quality_{sfx}").argtypes = [vp, vp, u32, u32, u32, ctypes.POINTER(ctypes.c_double),
                                                          ctypes.POINTER(ctypes.c_double), vp]
    for sfx in ("u16", "u32"):
        getattr(lib, f"lscomp_compress_batch_{sfx}").argtypes = [vp, ctypes.POINTER(LscompStack), u32, bins_t, f32,
                                                                 pu64, pu64, vp]
        getattr(lib, f"lscomp_plan_create_{sfx}").argtypes = [vp, ctypes.POINTER(LscompStack), u32, bins_t, f32, vp,
                                                              ctypes.POINTER(vp)]
        getattr(lib, f"lscomp_compress_batch_ex_{sfx}").argtypes = [vp, ctypes.POINTER(LscompStack), u32,
                                                                    ctypes.POINTER(u32), ctypes.POINTER(f32),
                                                                    pu64, pu64, vp]
        getattr(lib, f"lscomp_decompress_batch_{sfx}").argtypes = [vp, ctypes.POINTER(LscompStack), u32,
                                                                   ctypes.POINTER(u32), ctypes.POINTER(f32), vp]
        getattr(lib, f"lscomp_stream_sizes_batch_{sfx}").argtypes = [vp, ctypes.POINTER(LscompStack), u32,
                                                                     ctypes.POINTER(u32), ctypes.POINTER(f32), pu64, vp]
        getattr(lib, f"lscomp_plan_create_ex_{sfx}").argtypes = [vp, ctypes.POINTER(LscompStack), u32,
                                                                 ctypes.POINTER(u32), ctypes.POINTER(f32), vp,
                                                                 ctypes.POINTER(vp)]
    lib.lscomp_plan_run.argtypes = [vp, vp, pu64, pu64]
    lib.lscomp_plan_destroy.argtypes = [vp]
    for sfx in ("u16", "u32"):
        getattr(lib, f"lscomp_compress_host_{sfx}").argtypes = [vp, vp, u32, u32, u32, bins_t, f32, vp, u64, pu64,
                                                               pu64, vp]
        getattr(lib, f"lscomp_decompress_host_{sfx}").argtypes = [vp, vp, u64, u32, u32, u32, bins_t, f32, vp, vp]
    lib.lscomp_tune_mode.argtypes = [ctypes.c_int]
    lib.lscomp_tune_hits.restype = u64
    lib.lscomp_tune_report.restype = u64
    lib.lscomp_tune_report.argtypes = [ctypes.c_char_p, u64]
    lib.lscomp_tune_save.argtypes = [ctypes.c_char_p]
    lib.lscomp_tune_load.argtypes = [ctypes.c_char_p]
    lib.lscomp_workspace_stall_next.argtypes = [vp, u64]
    _lib = lib
    return lib


def _check(st: int, what: str):
    if st != 0:
        raise LscompError(st, what)


def _bins(bins: Sequence[int]):
    if len(bins) != 4:
        raise ValueError("bins must have four entries")
    arr = (ctypes.c_uint32 * 4)(*[int(b) for b in bins])
    return arr


def block_count(dims: Sequence[int]) -> int:
    x, y, z = dims
    return x * ((y + 7) // 8) * ((z + 7) // 8)


def max_stream_bytes(dims: Sequence[int], elem_bytes: int = 2) -> int:
    nb = block_count(dims)
    return (nb + 3) // 4 * 4 + (128 if elem_bytes == 2 else 248) * nb


def launch_count() -> int:
    return int(load_library().lscomp_launch_count())


class Workspace:
    """Scan state for a sequence of ordered calls on one device."""

    def __init__(self, device: int = -1):
        lib = load_library()
        self._ws = ctypes.c_void_p()
        _check(lib.lscomp_workspace_create(ctypes.byref(self._ws), int(device)), "lscomp_workspace_create")

    @property
    def handle(self):
        return self._ws

    def set_host_chunk(self, nbytes: int) -> None:
        """Input bytes per chunk of compress_host / decompress_host (0: default)."""
        _check(load_library().lscomp_workspace_set_host_chunk(self._ws, ctypes.c_uint64(int(nbytes))),
               "lscomp_workspace_set_host_chunk")

    def set_tuning(self, allow: bool) -> None:
        """False: calls through this workspace never run the tuner."""
        _check(load_library().lscomp_workspace_set_tuning(self._ws, 1 if allow else 0), "lscomp_workspace_set_tuning")

    def stall_next(self, wait_ns: int) -> None:
        """Failure injection: the next launch leaves tile 0 unclaimed and limits
        every wait to wait_ns, so its look-back times out (LSCOMP_ERR_TIMEOUT)."""
        _check(load_library().lscomp_workspace_stall_next(self._ws, ctypes.c_uint64(int(wait_ns))),
               "lscomp_workspace_stall_next")

    def close(self):
        if self._ws:
            load_library().lscomp_workspace_destroy(self._ws)
            self._ws = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, stream: int = 0):
        _check(load_library().lscomp_workspace_check(self._ws, ctypes.c_void_p(stream)), "lscomp_workspace_check")


def _stream_handle(stream) -> int:
    if stream is None:
        import torch

        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _suffix(t) -> str:
    return "u32" if t.element_size() == 4 else "u16"


def compress_into(ws: Workspace, d_in, dims, bins, pooling: float, d_out, stream=None) -> Tuple[int, int]:
    """Compress device tensor d_in (X*Y*Z values: uint16 carried in int16, or
    uint32 carried in int32) into d_out (uint8).

    Returns (stream_len, ref_size): the stream's length in bytes and the size
    the reference's host API reports (payload + nb)."""
    lib = load_library()
    x, y, z = (int(v) for v in dims)
    sl, rs = ctypes.c_uint64(0), ctypes.c_uint64(0)
    st = getattr(lib, f"lscomp_compress_{_suffix(d_in)}")(
        ws.handle, ctypes.c_void_p(d_in.data_ptr()), x, y, z, _bins(bins), ctypes.c_float(pooling),
        ctypes.c_void_p(d_out.data_ptr()), ctypes.c_uint64(d_out.numel() * d_out.element_size()),
        ctypes.byref(sl), ctypes.byref(rs), ctypes.c_void_p(_stream_handle(stream)))
    _check(st, f"lscomp_compress_{_suffix(d_in)}")
    return int(sl.value), int(rs.value)


def _stack_array(items):
    n = len(items)
    sfx = _suffix(items[0][0])
    arr = (LscompStack * n)()
    for i, it in enumerate(items):
        d_in, dims, d_out = it[0], it[1], it[2]
        if _suffix(d_in) != sfx:
            raise ValueError("a batch holds one element type")
        x, y, z = (int(v) for v in dims)
        arr[i] = LscompStack(d_in.data_ptr(), x, y, z, d_out.data_ptr(), d_out.numel() * d_out.element_size())
    return sfx, arr


def _per_stack_settings(items):
    n = len(items)
    bins = (ctypes.c_uint32 * (4 * n))()
    pool = (ctypes.c_float * n)()
    for i, it in enumerate(items):
        b, p = it[3], it[4]
        for k in range(4):
            bins[4 * i + k] = int(b[k])
        pool[i] = float(p)
    return bins, pool


def stream_sizes_batch(ws: Workspace, items, stream=None):
    """Exact stream lengths of many stacks without compressing them:
    items = [(d_in, dims, d_out or None, bins, pooling), ...] (one element
    type; d_out is not used).  Returns [stream_len, ...], the bytes
    compress_batch_mixed / compress_into would write."""
    lib = load_library()
    n = len(items)
    if n == 0:
        return []
    sfx = _suffix(items[0][0])
    arr = (LscompStack * n)()
    for i, it in enumerate(items):
        if _suffix(it[0]) != sfx:
            raise ValueError("a batch holds one element type")
        x, y, z = (int(v) for v in it[1])
        arr[i] = LscompStack(it[0].data_ptr(), x, y, z, None, 0)
    bins, pool = _per_stack_settings(items)
    sl = (ctypes.c_uint64 * n)()
    st = getattr(lib, f"lscomp_stream_sizes_batch_{sfx}")(ws.handle, arr, n, bins, pool, sl,
                                                          ctypes.c_void_p(_stream_handle(stream)))
    _check(st, f"lscomp_stream_sizes_batch_{sfx}")
    return [int(v) for v in sl]


def compress_batch_mixed(ws: Workspace, items, stream=None):
    """Compress many stacks in one launch, each with its own settings:
    items = [(d_in, dims, d_out, bins, pooling), ...] (one element type).
    Returns [(stream_len, ref_size), ...]; each stream is the one
    compress_into writes for that stack alone with its settings."""
    lib = load_library()
    n = len(items)
    if n == 0:
        return []
    sfx, arr = _stack_array(items)
    bins, pool = _per_stack_settings(items)
    sl = (ctypes.c_uint64 * n)()
    rs = (ctypes.c_uint64 * n)()
    st = getattr(lib, f"lscomp_compress_batch_ex_{sfx}")(ws.handle, arr, n, bins, pool, sl, rs,
                                                         ctypes.c_void_p(_stream_handle(stream)))
    _check(st, f"lscomp_compress_batch_ex_{sfx}")
    return [(int(sl[i]), int(rs[i])) for i in range(n)]


def _host_buffer(a):
    """(address, bytes, element bytes) of a host buffer: a numpy array or a
    CPU torch tensor (pinned ones let the copies overlap)."""
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("host buffer must be contiguous")
        return a.ctypes.data, a.nbytes, a.itemsize
    if getattr(a, "is_cuda", False):
        raise ValueError("expected a host buffer")
    return a.data_ptr(), a.numel() * a.element_size(), a.element_size()


def compress_host(ws: Workspace, h_in, dims, bins, pooling: float, h_out, stream=None) -> Tuple[int, int]:
    """Compress a stack in host memory (uint16 / uint32 values, or int16 /
    int32 carrying them) into host buffer h_out (bytes).  Returns
    (stream_len, ref_size), as compress_into."""
    lib = load_library()
    pi, ni, es = _host_buffer(h_in)
    po, no, _ = _host_buffer(h_out)
    x, y, z = (int(v) for v in dims)
    if ni < x * y * z * es:
        raise ValueError("input smaller than the dims")
    sfx = "u32" if es == 4 else "u16"
    sl, rs = ctypes.c_uint64(0), ctypes.c_uint64(0)
    _check(getattr(lib, f"lscomp_compress_host_{sfx}")(ws.handle, ctypes.c_void_p(pi), x, y, z, _bins(bins),
                                                       ctypes.c_float(pooling), ctypes.c_void_p(po),
                                                       ctypes.c_uint64(no), ctypes.byref(sl), ctypes.byref(rs),
                                                       ctypes.c_void_p(_stream_handle(stream))),
           f"lscomp_compress_host_{sfx}")
    return int(sl.value), int(rs.value)


def decompress_host(ws: Workspace, h_cmp, cmp_len: int, dims, bins, pooling: float, h_out, stream=None) -> None:
    """Decompress a stream in host memory (cmp_len readable bytes) into the
    host buffer h_out (X*Y*Z values of 2 or 4 bytes)."""
    lib = load_library()
    pi, ni, _ = _host_buffer(h_cmp)
    po, no, es = _host_buffer(h_out)
    x, y, z = (int(v) for v in dims)
    if no < x * y * z * es or ni < cmp_len:
        raise ValueError("buffer smaller than the dims or the stream")
    sfx = "u32" if es == 4 else "u16"
    _check(getattr(lib, f"lscomp_decompress_host_{sfx}")(ws.handle, ctypes.c_void_p(pi), ctypes.c_uint64(int(cmp_len)),
                                                         x, y, z, _bins(bins), ctypes.c_float(pooling),
                                                         ctypes.c_void_p(po), ctypes.c_void_p(_stream_handle(stream))),
           f"lscomp_decompress_host_{sfx}")


def decompress_batch(ws: Workspace, items, stream=None) -> None:
    """Decode many streams in two launches: items = [(d_stream, cmp_len, dims,
    d_out, bins, pooling), ...], d_out int16 (uint16 data) or int32 (uint32)
    tensors of one type."""
    lib = load_library()
    n = len(items)
    if n == 0:
        return
    sfx = _suffix(items[0][3])
    arr = (LscompStack * n)()
    for i, (d_s, ln, dims, d_out, b, p) in enumerate(items):
        if _suffix(d_out) != sfx:
            raise ValueError("a batch holds one element type")
        x, y, z = (int(v) for v in dims)
        arr[i] = LscompStack(d_s.data_ptr(), x, y, z, d_out.data_ptr(), int(ln))
    bins, pool = _per_stack_settings([(None, None, None, it[4], it[5]) for it in items])
    _check(getattr(lib, f"lscomp_decompress_batch_{sfx}")(ws.handle, arr, n, bins, pool,
                                                          ctypes.c_void_p(_stream_handle(stream))),
           f"lscomp_decompress_batch_{sfx}")


def compress_batch(ws: Workspace, items, bins, pooling: float, stream=None):
    """Compress many stacks in one launch: items = [(d_in, dims, d_out), ...],
    all uint16 (int16 tensors) or all uint32 (int32 tensors), with the same
    bins and pooling threshold.  Returns [(stream_len, ref_size), ...]; each
    stack's stream is the one compress_into writes for it alone."""
    lib = load_library()
    n = len(items)
    if n == 0:
        return []
    sfx = _suffix(items[0][0])
    arr = (LscompStack * n)()
    for i, (d_in, dims, d_out) in enumerate(items):
        if _suffix(d_in) != sfx:
            raise ValueError("a batch holds one element type")
        x, y, z = (int(v) for v in dims)
        arr[i] = LscompStack(d_in.data_ptr(), x, y, z, d_out.data_ptr(), d_out.numel() * d_out.element_size())
    sl = (ctypes.c_uint64 * n)()
    rs = (ctypes.c_uint64 * n)()
    st = getattr(lib, f"lscomp_compress_batch_{sfx}")(ws.handle, arr, n, _bins(bins), ctypes.c_float(pooling), sl, rs,
                                                      ctypes.c_void_p(_stream_handle(stream)))
    _check(st, f"lscomp_compress_batch_{sfx}")
    return [(int(sl[i]), int(rs[i])) for i in range(n)]


class Plan:
    """A compression captured once as a CUDA graph (lscomp_plan_*): the same
    items as compress_batch (one item: the single-stack kernel), replayed by
    run() on new contents of the same buffers.  Creating it runs one ordinary
    call through ws (the streams are written)."""

    def __init__(self, ws: Workspace, items, bins=None, pooling: Optional[float] = None, stream=None):
        """items = [(d_in, dims, d_out), ...] with bins and pooling for all,
        or [(d_in, dims, d_out, bins, pooling), ...] with bins=None."""
        lib = load_library()
        self._lib = lib
        self.handle = None
        n = len(items)
        if n == 0:
            raise ValueError("a plan holds at least one stack")
        sfx, arr = _stack_array(items)
        self.n = n
        self._keep = items  # the buffers must outlive the plan
        h = ctypes.c_void_p()
        hs = ctypes.c_void_p(_stream_handle(stream))
        if bins is None:
            pb, pp = _per_stack_settings(items)
            st = getattr(lib, f"lscomp_plan_create_ex_{sfx}")(ws.handle, arr, n, pb, pp, hs, ctypes.byref(h))
        else:
            st = getattr(lib, f"lscomp_plan_create_{sfx}")(ws.handle, arr, n, _bins(bins), ctypes.c_float(pooling),
                                                           hs, ctypes.byref(h))
        _check(st, f"lscomp_plan_create_{sfx}")
        self.handle = h

    def run(self, stream=None):
        """Replay; returns [(stream_len, ref_size), ...]."""
        sl = (ctypes.c_uint64 * self.n)()
        rs = (ctypes.c_uint64 * self.n)()
        _check(self._lib.lscomp_plan_run(self.handle, ctypes.c_void_p(_stream_handle(stream)), sl, rs),
               "lscomp_plan_run")
        return [(int(sl[i]), int(rs[i])) for i in range(self.n)]

    def close(self):
        if self.handle:
            self._lib.lscomp_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tune_mode(mode: Optional[int] = None) -> int:
    """Launch-configuration tuning: 1 on (tune keys on first use), 0 off;
    None only queries.  Returns the previous mode."""
    return int(load_library().lscomp_tune_mode(-1 if mode is None else int(mode)))


def tune_hits() -> int:
    """Calls so far that used a configuration from the tuner's table."""
    return int(load_library().lscomp_tune_hits())


def tune_clear() -> None:
    _check(load_library().lscomp_tune_clear(), "lscomp_tune_clear")


def tune_report() -> str:
    """The tuner's table as text (see lscomp_tune_report in include/lscomp.h)."""
    lib = load_library()
    n = int(lib.lscomp_tune_report(None, 0))
    buf = ctypes.create_string_buffer(n)
    lib.lscomp_tune_report(buf, n)
    return buf.value.decode()


def tune_table() -> list:
    """The tuner's table parsed: one dict per key."""
    out = []
    for line in tune_report().splitlines():
        head, *cands = line.split(" | ")
        key, cfg = head.split(" -> ")
        es, layout, pool, kind, vec, bzb = (int(v) for v in key.split())
        shape, tb = (int(v) for v in cfg.split())
        times = []
        for c in cands:
            cs, ct, ms = c.split()
            times.append({"shape": int(cs), "tile_blocks": int(ct), "ms": float(ms)})
        out.append({"es": es, "layout": layout, "pool": pool, "kind": ("compress", "batch", "decompress")[kind],
                    "vec": vec, "bzb": bzb, "shape": shape, "tile_blocks": tb, "times": times})
    return out


def tune_save(path: str) -> None:
    _check(load_library().lscomp_tune_save(os.fsencode(path)), "lscomp_tune_save")


def tune_load(path: str) -> None:
    _check(load_library().lscomp_tune_load(os.fsencode(path)), "lscomp_tune_load")


def container_header(elem_bytes: int, dims, bins, pooling: float, stream_len: int, ref_size: int) -> bytes:
    """The 64-byte container header for a stream (host only)."""
    lib = load_library()
    buf = ctypes.create_string_buffer(int(lib.lscomp_container_header_bytes()))
    x, y, z = (int(v) for v in dims)
    _check(lib.lscomp_container_write_header(buf, elem_bytes, x, y, z, _bins(bins), ctypes.c_float(pooling),
                                             ctypes.c_uint64(stream_len), ctypes.c_uint64(ref_size)),
           "lscomp_container_write_header")
    return buf.raw


def parse_container(buf: bytes, length: Optional[int] = None) -> dict:
    """Parse and check a container header (host only); length defaults to
    len(buf), i.e. a whole container, or a header alone when len(buf) == 64."""
    lib = load_library()
    info = ContainerInfo()
    raw = ctypes.create_string_buffer(bytes(buf), len(buf))
    _check(lib.lscomp_container_read_header(raw, ctypes.c_uint64(len(buf) if length is None else length),
                                            ctypes.byref(info)), "lscomp_container_read_header")
    return info.as_dict()


def compress_container(ws: Workspace, d_in, dims, bins, pooling: float, d_out, stream=None) -> int:
    """Compress into a container (header + unchanged stream) in d_out; returns its length."""
    lib = load_library()
    x, y, z = (int(v) for v in dims)
    n = ctypes.c_uint64(0)
    _check(lib.lscomp_compress_container(ws.handle, d_in.element_size(), ctypes.c_void_p(d_in.data_ptr()), x, y, z,
                                         _bins(bins), ctypes.c_float(pooling), ctypes.c_void_p(d_out.data_ptr()),
                                         ctypes.c_uint64(d_out.numel() * d_out.element_size()), ctypes.byref(n),
                                         ctypes.c_void_p(_stream_handle(stream))), "lscomp_compress_container")
    return int(n.value)


def decompress_container(ws: Workspace, d_cont, length: int, d_out, stream=None) -> dict:
    """Decompress a container of `length` bytes into d_out; returns its header."""
    lib = load_library()
    info = ContainerInfo()
    _check(lib.lscomp_decompress_container(ws.handle, ctypes.c_void_p(d_cont.data_ptr()), ctypes.c_uint64(length),
                                           ctypes.c_void_p(d_out.data_ptr()),
                                           ctypes.c_uint64(d_out.numel() * d_out.element_size()), ctypes.byref(info),
                                           ctypes.c_void_p(_stream_handle(stream))), "lscomp_decompress_container")
    return info.as_dict()


class Server:
    """The serving loop of liblscomp.so (lscomp_server_*): submit requests with
    numpy host buffers from any thread, wait for them in any order.  The
    buffers are kept alive here until the request is waited for."""

    def __init__(self, device: int = 0, arena_bytes: int = 1 << 30):
        lib = load_library()
        h = ctypes.c_void_p()
        _check(lib.lscomp_server_create(ctypes.byref(h), device, ctypes.c_uint64(arena_bytes)), "lscomp_server_create")
        self._h = h
        self._keep = {}

    def submit_compress(self, h_in: np.ndarray, dims, bins, pooling: float, h_out: np.ndarray) -> int:
        assert h_in.flags["C_CONTIGUOUS"] and h_out.flags["C_CONTIGUOUS"] and h_in.itemsize in (2, 4)
        x, y, z = (int(v) for v in dims)
        rid = load_library().lscomp_server_submit_compress(self._h, h_in.itemsize, h_in.ctypes.data, x, y, z,
                                                           _bins(bins), ctypes.c_float(pooling), h_out.ctypes.data,
                                                           ctypes.c_uint64(h_out.nbytes))
        if rid < 0:
            raise LscompError(int(-rid), "lscomp_server_submit_compress")
        self._keep[rid] = (h_in, h_out)
        return int(rid)

    def submit_decompress(self, container: np.ndarray, h_out: np.ndarray) -> int:
        assert container.flags["C_CONTIGUOUS"] and h_out.flags["C_CONTIGUOUS"]
        rid = load_library().lscomp_server_submit_decompress(self._h, container.ctypes.data,
                                                             ctypes.c_uint64(container.nbytes), h_out.ctypes.data,
                                                             ctypes.c_uint64(h_out.nbytes))
        if rid < 0:
            raise LscompError(int(-rid), "lscomp_server_submit_decompress")
        self._keep[rid] = (container, h_out)
        return int(rid)

    def wait(self, rid: int) -> dict:
        r = ServerResult()
        _check(load_library().lscomp_server_wait(self._h, ctypes.c_int64(rid), ctypes.byref(r)), "lscomp_server_wait")
        self._keep.pop(rid, None)
        return {"status": r.status, "out_len": int(r.out_len), "queued_ns": int(r.queued_ns),
                "service_ns": int(r.service_ns), "admit_ns": int(r.admit_ns), "done_ns": int(r.done_ns)}

    def stats(self) -> dict:
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(load_library().lscomp_server_stats(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
               "lscomp_server_stats")
        return {"rounds": a.value, "batches": b.value, "batched_requests": c.value}

    def close(self):
        if self._h:
            load_library().lscomp_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def quality(d_ori, d_dec, dims, ssim: bool = True, stream=None) -> dict:
    """PSNR report and (optionally) the 7x7x7 SSIM of an original stack and its
    decoded copy, on the GPU (lscomp_quality_*): the reference's computePSNR /
    computeSSIM definitions on float copies of the values."""
    lib = load_library()
    x, y, z = (int(v) for v in dims)
    p = (ctypes.c_double * 6)()
    sv = ctypes.c_double(0.0)
    _check(getattr(lib, f"lscomp_quality_{_suffix(d_ori)}")(
        ctypes.c_void_p(d_ori.data_ptr()), ctypes.c_void_p(d_dec.data_ptr()), x, y, z, p,
        ctypes.byref(sv) if ssim else None, ctypes.c_void_p(_stream_handle(stream))), f"lscomp_quality_{_suffix(d_ori)}")
    out = {"mse": p[0], "range": p[1], "psnr": p[2], "l2_error": p[3], "l2_error_rel": p[4], "nrmse": p[5]}
    if ssim:
        out["ssim"] = sv.value
    return out


def compress_async(ws: Workspace, d_in, dims, bins, pooling: float, d_out, d_sizes=None, stream=None):
    """Enqueue a compression without host synchronisation; d_sizes (2 x uint64
    in an int64 tensor) receives {stream_len, payload bytes}."""
    lib = load_library()
    x, y, z = (int(v) for v in dims)
    st = getattr(lib, f"lscomp_compress_{_suffix(d_in)}_async")(
        ws.handle, ctypes.c_void_p(d_in.data_ptr()), x, y, z, _bins(bins), ctypes.c_float(pooling),
        ctypes.c_void_p(d_out.data_ptr()), ctypes.c_uint64(d_out.numel() * d_out.element_size()),
        ctypes.c_void_p(d_sizes.data_ptr() if d_sizes is not None else 0),
        ctypes.c_void_p(_stream_handle(stream)))
    _check(st, f"lscomp_compress_{_suffix(d_in)}_async")


def decompress_into(ws: Workspace, d_cmp, cmp_len: int, dims, bins, pooling: float, d_out, stream=None):
    """Decompress the stream in device tensor d_cmp (cmp_len readable bytes)
    into d_out (X*Y*Z values, int16 for uint16 data or int32 for uint32)."""
    lib = load_library()
    x, y, z = (int(v) for v in dims)
    st = getattr(lib, f"lscomp_decompress_{_suffix(d_out)}")(
        ws.handle, ctypes.c_void_p(d_cmp.data_ptr()), ctypes.c_uint64(int(cmp_len)), x, y, z, _bins(bins),
        ctypes.c_float(pooling), ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(_stream_handle(stream)))
    _check(st, f"lscomp_decompress_{_suffix(d_out)}")


def decompress_async(ws: Workspace, d_cmp, cmp_len: int, dims, bins, pooling: float, d_out, stream=None):
    lib = load_library()
    x, y, z = (int(v) for v in dims)
    st = getattr(lib, f"lscomp_decompress_{_suffix(d_out)}_async")(
        ws.handle, ctypes.c_void_p(d_cmp.data_ptr()), ctypes.c_uint64(int(cmp_len)), x, y, z, _bins(bins),
        ctypes.c_float(pooling), ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(_stream_handle(stream)))
    _check(st, f"lscomp_decompress_{_suffix(d_out)}_async")


_default_ws = {}


def _ws_for(device: int) -> Workspace:
    if device not in _default_ws:
        _default_ws[device] = Workspace(device)
    return _default_ws[device]


def compress(data, dims, bins, pooling: float, out=None, stream=None):
    """Reference-style call: returns (stream tensor, cmp_size) where cmp_size
    is what cuLSZ_compression_uint16_bsize64 reports; the stream tensor is
    trimmed to the true stream length."""
    import torch

    dev = data.device.index if data.device.index is not None else torch.cuda.current_device()
    if out is None:
        out = torch.empty(max_stream_bytes(dims), dtype=torch.uint8, device=data.device)
    sl, rs = compress_into(_ws_for(dev), data, dims, bins, pooling, out, stream)
    return out[:sl], rs


def decompress(stream_t, dims, bins, pooling: float, out=None, stream=None):
    import torch

    dev = stream_t.device.index if stream_t.device.index is not None else torch.cuda.current_device()
    if out is None:
        n = int(dims[0]) * int(dims[1]) * int(dims[2])
        out = torch.empty(n, dtype=torch.int16, device=stream_t.device)
    decompress_into(_ws_for(dev), stream_t, stream_t.numel(), dims, bins, pooling, out, stream)
    return out


# --------------------------------------------------------------- synthetic data
def _load_synth():
    global _synth_lib
    if _synth_lib is None:
        if not os.path.exists(SYNTH_PATH):
            raise ImportError(f"liblscomp_synth.so not built: {SYNTH_PATH}")
        s = ctypes.CDLL(SYNTH_PATH)
        for name in ("lsc_synth_small", "lsc_synth_cssi", "lsc_synth_xpcs"):
            f = getattr(s, name)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                          ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int]
        _synth_lib = s
    return _synth_lib


def _synth(kind: str, dims, seed: int, frames: Optional[Tuple[int, int]] = None, out=None, threads: int = 0):
    x, y, z = (int(v) for v in dims)
    x0, nx = frames if frames is not None else (0, x)
    if out is None:
        out = np.empty(nx * y * z, dtype=np.uint16)
    assert out.dtype == np.uint16 and out.size >= nx * y * z and out.flags["C_CONTIGUOUS"]
    f = getattr(_load_synth(), f"lsc_synth_{kind}")
    st = f(out.ctypes.data, x, y, z, x0, nx, ctypes.c_uint64(seed), threads)
    if st != 0:
        raise RuntimeError(f"lsc_synth_{kind} failed ({st})")
    return out


def synth_small(dims, seed: int = 1, frames=None, out=None, threads: int = 0):
    """Poisson(0.1) background, 20 Gaussian spots per frame, 0.1% hot pixels."""
    return _synth("small", dims, seed, frames, out, threads)


def synth_cssi(dims, seed: int = 2, frames=None, out=None, threads: int = 0):
    """Radial Poisson background 50 -> 0.5, 3-8 diffraction rings, beamstop."""
    return _synth("cssi", dims, seed, frames, out, threads)


def synth_xpcs(dims, seed: int = 3, frames=None, out=None, threads: int = 0):
    """Sparse AR(1) speckle (mean 0.02, rho 0.9), beamstop disk r = 60 px."""
    return _synth("xpcs", dims, seed, frames, out, threads)
