"""Pure-Python restatement of the lsCOMP block codec for tiny inputs (test
infrastructure).  Written independently of oracle/lscomp_oracle.c so the two
checkers can be compared with each other; it follows the same reference
lines: lsCOMP/src/cuLSZ_kernel.cu:868-957 (block statistics and header),
:1100-1276 (packing), :1322-1640 (decode) and lsCOMP/src/cuLSZ_entry.cu:97-125.
uint16 data only."""
import numpy as np


def _blocks(dims):
    x, y, z = dims
    byb, bzb = (y + 7) // 8, (z + 7) // 8
    for bx in range(x):
        for by in range(byb):
            for bz in range(bzb):
                yield bx, by, bz


def _gather(a, bx, by, bz):
    x, y, z = a.shape
    v = [0] * 64
    for i in range(8):
        for k in range(8):
            yy, zz = by * 8 + i, bz * 8 + k
            if yy < y and zz < z:
                v[i * 8 + k] = int(a[bx, yy, zz])
    return v


def _pool_from_p(p):
    p32 = np.float32(p)
    for k in range(65):
        if np.float32(k) / np.float32(64) > p32:
            return k
    return 65


def header(v, bins, p):
    zc = sum(1 for t in v if t == 0)
    cnt = [sum(1 for t in v if t < b) for b in bins]
    max1 = max(v)
    max2 = max((v[i - 1] + v[i]) // 2 for i in range(1, 64, 2))
    pool = zc >= _pool_from_p(p)
    c = 0
    if cnt[1] == cnt[0]:
        c = 1
        if cnt[2] == cnt[1]:
            c = 2
            if cnt[3] == cnt[2]:
                c = 3
    m = (max2 if pool else max1) // bins[c]
    rate = m.bit_length()
    return (0x80 if pool else 0) | (c << 5) | rate


def pack(v, hb, bins):
    pool, c, rate = hb >> 7, (hb >> 5) & 3, hb & 31
    out = bytearray()
    if pool:
        q = [((v[2 * i] + v[2 * i + 1]) // 2) // bins[c] for i in range(32)]
        for i in range(rate):
            for b in range(4):
                out.append(sum(((q[8 * b + k] >> i) & 1) << (7 - k) for k in range(8)))
    else:
        q = [t // bins[c] for t in v]
        for i in range(rate):
            for r in range(8):
                out.append(sum(((q[8 * r + k] >> i) & 1) << (7 - k) for k in range(8)))
    return bytes(out)


def compress(a, bins, p):
    """a: uint16 array of shape (x, y, z).  Returns (stream bytes, payload+nb)."""
    dims = a.shape
    hdrs, pays = [], []
    for bx, by, bz in _blocks(dims):
        v = _gather(a, bx, by, bz)
        hb = header(v, bins, p)
        hdrs.append(hb)
        pays.append(pack(v, hb, bins))
    nb = len(hdrs)
    r = (nb + 3) // 4 * 4
    payload = b"".join(pays)
    return bytes(hdrs) + bytes(r - nb) + payload, len(payload) + nb


def decompress(stream, dims, bins):
    x, y, z = dims
    out = np.zeros((x, y, z), dtype=np.uint16)
    nb = x * ((y + 7) // 8) * ((z + 7) // 8)
    off = (nb + 3) // 4 * 4
    for k, (bx, by, bz) in enumerate(_blocks(dims)):
        hb = stream[k]
        pool, c, rate = hb >> 7, (hb >> 5) & 3, hb & 31
        vals = [0] * 64
        if pool:
            for m in range(32):
                q = 0
                for i in range(rate):
                    q |= ((stream[off + 4 * i + m // 8] >> (7 - m % 8)) & 1) << i
                vals[2 * m] = vals[2 * m + 1] = (q * bins[c]) & 0xFFFF
            off += 4 * rate
        else:
            for e in range(64):
                q = 0
                for i in range(rate):
                    q |= ((stream[off + 8 * i + e // 8] >> (7 - e % 8)) & 1) << i
                vals[e] = (q * bins[c]) & 0xFFFF
            off += 8 * rate
        for i in range(8):
            for kk in range(8):
                yy, zz = by * 8 + i, bz * 8 + kk
                if yy < y and zz < z:
                    out[bx, yy, zz] = vals[i * 8 + kk]
    return out
