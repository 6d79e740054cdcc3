"""Generate tests/golden/*.npz from the reference's own CUDA build.

Runs the unmodified reference (oracle/_ref/libculsz_ref.so, built from
lsCOMP/src/cuLSZ_kernel.cu and cuLSZ_entry.cu by oracle/Makefile) through its
host API on small seeded inputs that cover every branch of the stream format,
on a CUDA GPU, and stores input, stream, reported size and the reference's
decode.  The output buffers are zeroed before each call (the reference leaves
header pad bytes and rate-0 blocks unwritten).

    python tests/golden/make_golden.py OUT_DIR
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "sc25-lscomp_b200"))


def cases():
    import lscomp

    rng = np.random.default_rng(20261203)

    def rand16(dims, hi, zero, hot):
        a = rng.integers(0, hi, size=dims, dtype=np.uint16)
        a[rng.random(dims) < zero] = 0
        a[rng.random(dims) < hot] = 65535
        return a

    def rand32(dims, hi, zero):
        a = rng.integers(0, hi, size=dims, dtype=np.uint32)
        a[rng.random(dims) < zero] = 0
        return a

    yield "u16_small_lossless", "u16", (3, 37, 53), lscomp.synth_small((3, 37, 53), seed=11), (1, 1, 1, 1), 1.0
    yield "u16_small_lossy", "u16", (3, 37, 53), lscomp.synth_small((3, 37, 53), seed=11), (3, 5, 10, 15), 0.5
    yield "u16_pool_all", "u16", (2, 64, 72), rand16((2, 64, 72), 50, 0.5, 0.01), (1, 1, 1, 1), 0.0
    yield "u16_multitile", "u16", (8, 128, 96), rand16((8, 128, 96), 400, 0.4, 0.002), (2, 7, 7, 30), 0.8
    yield "u16_cssi_wide", "u16", (1, 9, 2049), lscomp.synth_cssi((1, 9, 2049), seed=4), (5, 10, 15, 15), 0.3
    yield "u16_xpcs", "u16", (4, 200, 136), lscomp.synth_xpcs((4, 200, 136), seed=6), (3, 5, 10, 15), 0.5
    yield "u16_unsorted_bins", "u16", (2, 40, 48), rand16((2, 40, 48), 60, 0.3, 0.0), (9, 4, 12, 3), 0.5
    yield "u32_lossless", "u32", (2, 40, 48), rand32((2, 40, 48), 1 << 20, 0.5), (1, 1, 1, 1), 1.0
    yield "u32_lossy", "u32", (2, 40, 48), rand32((2, 40, 48), 1 << 20, 0.5), (7, 7, 7, 7), 0.3


def stream_length(hdr, nb):
    sizes = (hdr & 0x1F).astype(np.int64) * np.where(hdr & 0x80, 4, 8)
    return (nb + 3) // 4 * 4 + int(sizes.sum())


def main(out_dir):
    import torch

    from oracle import RefLib

    ref = RefLib()
    os.makedirs(out_dir, exist_ok=True)
    for name, t, dims, a, bins, p in cases():
        x, y, z = dims
        nb = x * ((y + 7) // 8) * ((z + 7) // 8)
        itype = torch.int16 if t == "u16" else torch.int32
        view = np.int16 if t == "u16" else np.int32
        d_in = torch.from_numpy(np.ascontiguousarray(a).view(view).ravel()).cuda()
        cap = (nb + 3) // 4 * 4 + 256 * nb
        d_cmp = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        size = ref.compress(d_in.data_ptr(), d_cmp.data_ptr(), dims, bins, p, t=t)
        torch.cuda.synchronize()
        buf = d_cmp.cpu().numpy()
        slen = stream_length(buf[:nb], nb)
        d_dec = torch.zeros(a.size, dtype=itype, device="cuda")
        ref.decompress(d_dec.data_ptr(), d_cmp.data_ptr(), size, dims, bins, p, t=t)
        torch.cuda.synchronize()
        dec = d_dec.cpu().numpy().view(np.uint16 if t == "u16" else np.uint32)
        np.savez_compressed(os.path.join(out_dir, name + ".npz"), input=np.ascontiguousarray(a).ravel(),
                            dims=np.array(dims), bins=np.array(bins, dtype=np.uint32), p=np.float32(p),
                            stream=buf[:slen], ref_size=np.int64(size), decode=dec, dtype=t)
        print(name, dims, bins, p, "stream", slen, "reported", size)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
