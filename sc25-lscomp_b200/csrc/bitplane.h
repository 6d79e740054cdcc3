// bitplane.h -- register-level bit-plane transposes shared by the encoder and
// decoder kernels (and compiled on the host by the unit test of the format).
//
// Stream format of one 8x8 block (lsCOMP/src/cuLSZ_kernel.cu:1100-1276):
//   plain block,  plane i (least significant first) = 8 bytes, byte r = row r,
//                 bit (7-k) of that byte = bit i of the quantised value at col k;
//   pooled block, plane i = 4 bytes, byte b = pooled values 8b..8b+7, the first
//                 value in the most significant bit.
// Here one thread holds the 8 quantised values of one row (or of one pooled
// row pair) as four packed words w0..w3 (w0 = q0 | q1 << 16, ...).  The
// functions below turn them into the 8 plane bytes for planes 0-7 (low value
// bytes) or 8-15 (high value bytes), and back.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define LSC_HD __host__ __device__ __forceinline__
#else
#define LSC_HD static inline
#endif

// Byte permute with the semantics of the PRMT instruction / __byte_perm:
// result byte n = byte (sel >> 4n) & 7 of the 8-byte value {b:a}.
LSC_HD uint32_t lsc_prmt(uint32_t a, uint32_t b, uint32_t sel)
{
#if defined(__CUDA_ARCH__)
    return __byte_perm(a, b, sel);
#else
    uint64_t v = ((uint64_t)b << 32) | a;
    uint32_t r = 0;
    for (int n = 0; n < 4; n++) {
        uint32_t s = (sel >> (4 * n)) & 7;
        r |= (uint32_t)((v >> (8 * s)) & 0xff) << (8 * n);
    }
    return r;
#endif
}

// 8x8 bit-matrix transpose of the 64-bit value {hi:lo}: bit (8a + b) moves to
// bit (8b + a).  Three rounds of masked swaps (rows 1 apart, 2 apart, 4 apart);
// the last round exchanges nibbles between the two 32-bit halves.  It is its
// own inverse.
LSC_HD void lsc_transpose8x8(uint32_t &lo, uint32_t &hi)
{
    uint32_t t;
    t = (lo ^ (lo >> 7)) & 0x00AA00AAu; lo ^= t ^ (t << 7);
    t = (hi ^ (hi >> 7)) & 0x00AA00AAu; hi ^= t ^ (t << 7);
    t = (lo ^ (lo >> 14)) & 0x0000CCCCu; lo ^= t ^ (t << 14);
    t = (hi ^ (hi >> 14)) & 0x0000CCCCu; hi ^= t ^ (t << 14);
    t = (lo ^ (hi << 4)) & 0xF0F0F0F0u; lo ^= t; hi ^= t >> 4;
}

// Plane bytes of one row: w0..w3 hold q0..q7 (q_k in 16-bit half k&1 of
// w[k>>1]).  high=0 gives planes 0-7, high=1 planes 8-15; on return p_lo holds
// planes {0,1,2,3}(+8) in bytes 0..3 and p_hi planes {4,5,6,7}(+8).
// The value bytes are laid out in reverse (q7 first) so that after the
// transpose value k lands in bit 7-k of each plane byte.
LSC_HD void lsc_row_planes(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, int high, uint32_t &p_lo,
                           uint32_t &p_hi)
{
    uint32_t sel = high ? 0x5713u : 0x4602u;
    uint32_t lo = lsc_prmt(w3, w2, sel); // q7 q6 q5 q4
    uint32_t hi = lsc_prmt(w1, w0, sel); // q3 q2 q1 q0
    lsc_transpose8x8(lo, hi);
    p_lo = lo;
    p_hi = hi;
}

// Inverse of lsc_row_planes for both halves at once: from the plane bytes of
// planes 0-7 (l_lo, l_hi) and 8-15 (h_lo, h_hi) rebuild w0..w3.
LSC_HD void lsc_row_values(uint32_t l_lo, uint32_t l_hi, uint32_t h_lo, uint32_t h_hi, uint32_t &w0,
                           uint32_t &w1, uint32_t &w2, uint32_t &w3)
{
    lsc_transpose8x8(l_lo, l_hi); // value low bytes: l_lo = q7 q6 q5 q4, l_hi = q3 q2 q1 q0
    lsc_transpose8x8(h_lo, h_hi); // value high bytes
    w3 = lsc_prmt(l_lo, h_lo, 0x4051u);
    w2 = lsc_prmt(l_lo, h_lo, 0x6273u);
    w1 = lsc_prmt(l_hi, h_hi, 0x4051u);
    w0 = lsc_prmt(l_hi, h_hi, 0x6273u);
}

// The first two rounds of lsc_transpose8x8 on one word: a 4x4 bit transpose
// of the low nibbles (bit c of byte a <-> bit a of byte c, a, c < 4) and one
// of the high nibbles.  Its own inverse.
LSC_HD uint32_t lsc_transpose4x4x2(uint32_t x)
{
    uint32_t t;
    t = (x ^ (x >> 7)) & 0x00AA00AAu; x ^= t ^ (t << 7);
    t = (x ^ (x >> 14)) & 0x0000CCCCu; x ^= t ^ (t << 14);
    return x;
}

// Values below 16: the 8 values of a row as nibbles of one word, byte a
// holding q(7-a) in its low nibble and q(3-a) in its high nibble.
LSC_HD uint32_t lsc_row_nibbles(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3)
{
    return lsc_prmt(w3 | (w1 << 4), w2 | (w0 << 4), 0x4602u);
}

// Values below 16: planes 0-3 of a row (p_lo of lsc_row_planes, high=0).
// With the high value nibbles zero, the third round of the 8x8 transpose
// only merges the two halves, so it is done first, by lsc_row_nibbles.
LSC_HD uint32_t lsc_row_planes4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3)
{
    return lsc_transpose4x4x2(lsc_row_nibbles(w0, w1, w2, w3));
}

// Values below 4, two rows a and b: bytes 0-3 = plane 0 of a, plane 1 of a,
// plane 0 of b, plane 1 of b.  Row b's two bits sit above row a's in every
// nibble, so one pair of 4x4 transposes serves both rows.
LSC_HD uint32_t lsc_rows_planes2(const uint32_t a[4], const uint32_t b[4])
{
    const uint32_t na = lsc_row_nibbles(a[0], a[1], a[2], a[3]);
    const uint32_t nb = lsc_row_nibbles(b[0], b[1], b[2], b[3]);
    return lsc_transpose4x4x2(na | (nb << 2));
}

// Inverse of lsc_row_planes4: planes 0-3 of a row back to w0..w3.
LSC_HD void lsc_row_values4(uint32_t p, uint32_t &w0, uint32_t &w1, uint32_t &w2, uint32_t &w3)
{
    const uint32_t x = lsc_transpose4x4x2(p);
    const uint32_t L = x & 0x0f0f0f0fu, H = (x >> 4) & 0x0f0f0f0fu;  // q7 q6 q5 q4 / q3 q2 q1 q0
    w3 = lsc_prmt(L, 0u, 0x4051u);
    w2 = lsc_prmt(L, 0u, 0x6273u);
    w1 = lsc_prmt(H, 0u, 0x4051u);
    w0 = lsc_prmt(H, 0u, 0x6273u);
}

// Inverse of lsc_rows_planes2: rows a and b back from their planes 0 and 1.
LSC_HD void lsc_rows_values2(uint32_t p, uint32_t a[4], uint32_t b[4])
{
    const uint32_t x = lsc_transpose4x4x2(p);
    const uint32_t La = x & 0x03030303u, Ha = (x >> 4) & 0x03030303u;
    const uint32_t Lb = (x >> 2) & 0x03030303u, Hb = (x >> 6) & 0x03030303u;
    a[3] = lsc_prmt(La, 0u, 0x4051u);
    a[2] = lsc_prmt(La, 0u, 0x6273u);
    a[1] = lsc_prmt(Ha, 0u, 0x4051u);
    a[0] = lsc_prmt(Ha, 0u, 0x6273u);
    b[3] = lsc_prmt(Lb, 0u, 0x4051u);
    b[2] = lsc_prmt(Lb, 0u, 0x6273u);
    b[1] = lsc_prmt(Hb, 0u, 0x4051u);
    b[0] = lsc_prmt(Hb, 0u, 0x6273u);
}

// Quotients of both 16-bit halves of w when every value is below 128:
// floor(v / bin) = (v * m) >> s with m <= 511, so both products stay inside
// their halves and one multiply serves the pair; the mask drops the bits the
// high product shifts into the low half.  qsm = m | s << 16 from
// lsc_small_quant_magic.
LSC_HD uint32_t lsc_quant7x2(uint32_t w, uint32_t qsm)
{
    const uint32_t s = qsm >> 16;
    return ((w * (qsm & 0xffffu)) >> s) & ((0xffffu >> s) | 0xffff0000u);
}

// m and s for lsc_quant7x2: s = bit length of 128 * bin - 1 (so 2^s >= 128 *
// bin > 127 * (m * bin - 2^s), which makes the quotient exact for v < 128)
// and m = ceil(2^s / bin); bins of 128 and more give 0 for every such value.
LSC_HD uint32_t lsc_small_quant_magic(uint32_t bin)
{
    if (bin >= 128u) return 0u;
    uint32_t s = 0;
    while ((1u << s) < 128u * bin) s++;
    const uint32_t m = ((1u << s) + bin - 1u) / bin;
    return m | (s << 16);
}

// Byte selectors of the 4x4 byte transpose across four threads r = 0..3
// (see xpose4 in the kernels).  Step A exchanges with thread r^2: threads 0,1
// keep their bytes 0,1 and take the partner's bytes 0,1; threads 2,3 take the
// partner's bytes 2,3 and keep their own bytes 2,3.  Step B exchanges with
// thread r^1 and interleaves single bytes.  Each selector applies to
// {partner : own}, so one PRMT per step with a per-thread selector.
#define LSC_XP_A_LOW 0x5410u   // r < 2:  own0 own1 prt0 prt1
#define LSC_XP_A_HIGH 0x3276u  // r >= 2: prt2 prt3 own2 own3
#define LSC_XP_B_EVEN 0x6240u  // r even: own0 prt0 own2 prt2
#define LSC_XP_B_ODD 0x3715u   // r odd:  prt1 own1 prt3 own3
