// CPU check of the register bit-plane transposes (sc25-lscomp_b200/csrc/bitplane.h)
// against a direct restatement of the plane format
// (lsCOMP/src/cuLSZ_kernel.cu:1189-1267: plane i byte of row r holds bit i of
// the value at column k in bit 7-k), and of the 4x4 byte-transpose network
// the kernels run across four lanes.  Built and run by tests/test_bitplane.py.
#include <stdio.h>
#include <stdint.h>
#include "bitplane.h"

static uint64_t state = 0x9e3779b97f4a7c15ull;
static uint32_t rnd(void)
{
    state ^= state << 13; state ^= state >> 7; state ^= state << 17;
    return (uint32_t)state;
}

int main(void)
{
    int bad = 0;
    for (int it = 0; it < 200000; it++) {
        uint32_t q[8];
        for (int k = 0; k < 8; k++) q[k] = rnd() & 0xffffu;
        uint32_t w0 = q[0] | q[1] << 16, w1 = q[2] | q[3] << 16, w2 = q[4] | q[5] << 16, w3 = q[6] | q[7] << 16;
        for (int high = 0; high < 2; high++) {
            uint32_t plo, phi;
            lsc_row_planes(w0, w1, w2, w3, high, plo, phi);
            for (int i = 0; i < 8; i++) {
                int plane = i + 8 * high;
                uint32_t want = 0;
                for (int k = 0; k < 8; k++) want |= ((q[k] >> plane) & 1u) << (7 - k);
                uint32_t got = (i < 4) ? (plo >> (8 * i)) & 0xffu : (phi >> (8 * (i - 4))) & 0xffu;
                bad += got != want;
            }
        }
        uint32_t a, b, c, d, r0, r1, r2, r3;
        lsc_row_planes(w0, w1, w2, w3, 0, a, b);
        lsc_row_planes(w0, w1, w2, w3, 1, c, d);
        lsc_row_values(a, b, c, d, r0, r1, r2, r3);
        bad += (r0 != w0) + (r1 != w1) + (r2 != w2) + (r3 != w3);
    }
    // narrow values: planes 0-3 of values below 16, planes 0-1 of two rows
    // of values below 4, and back
    for (int it = 0; it < 200000; it++) {
        uint32_t q[8], u[8];
        for (int k = 0; k < 8; k++) {
            q[k] = rnd() & 0xfu;
            u[k] = rnd() & 0x3u;
        }
        const uint32_t w[4] = {q[0] | q[1] << 16, q[2] | q[3] << 16, q[4] | q[5] << 16, q[6] | q[7] << 16};
        const uint32_t v[4] = {u[0] | u[1] << 16, u[2] | u[3] << 16, u[4] | u[5] << 16, u[6] | u[7] << 16};
        uint32_t plo, phi;
        lsc_row_planes(w[0], w[1], w[2], w[3], 0, plo, phi);
        bad += lsc_row_planes4(w[0], w[1], w[2], w[3]) != plo;
        uint32_t r0, r1, r2, r3;
        lsc_row_values4(plo, r0, r1, r2, r3);
        bad += (r0 != w[0]) + (r1 != w[1]) + (r2 != w[2]) + (r3 != w[3]);
        // two rows: w's two low bits as row a, v as row b
        uint32_t a2[4], ra[4], rb[4];
        for (int i = 0; i < 4; i++) a2[i] = w[i] & 0x00030003u;
        const uint32_t m = lsc_rows_planes2(a2, v);
        for (int i = 0; i < 4; i++) {
            const uint32_t *src = i < 2 ? a2 : v;
            const int plane = i & 1;
            uint32_t want = 0;
            for (int k = 0; k < 8; k++)
                want |= ((((src[k >> 1] >> (16 * (k & 1))) & 0xffffu) >> plane) & 1u) << (7 - k);
            bad += ((m >> (8 * i)) & 0xffu) != want;
        }
        lsc_rows_values2(m, ra, rb);
        for (int i = 0; i < 4; i++) bad += (ra[i] != a2[i]) + (rb[i] != v[i]);
    }
    // the paired quotient of values below 128, every bin it serves
    for (uint32_t bin = 1; bin < 300; bin++) {
        const uint32_t qsm = lsc_small_quant_magic(bin);
        bad += (qsm & 0xffffu) > 511u;
        for (uint32_t x = 0; x < 128; x++)
            for (uint32_t y = 0; y < 128; y += 7) {
                const uint32_t got = lsc_quant7x2(x | y << 16, qsm);
                bad += got != ((x / bin) | (y / bin) << 16);
            }
    }
    for (int it = 0; it < 10000; it++) {
        uint32_t x[4], z[4], y[4];
        for (int r = 0; r < 4; r++) x[r] = rnd();
        for (int r = 0; r < 4; r++) z[r] = lsc_prmt(x[r], x[r ^ 2], r < 2 ? LSC_XP_A_LOW : LSC_XP_A_HIGH);
        for (int r = 0; r < 4; r++) y[r] = lsc_prmt(z[r], z[r ^ 1], (r & 1) ? LSC_XP_B_ODD : LSC_XP_B_EVEN);
        for (int r = 0; r < 4; r++)
            for (int c2 = 0; c2 < 4; c2++) bad += ((x[c2] >> (8 * r)) & 0xffu) != ((y[r] >> (8 * c2)) & 0xffu);
    }
    printf("mismatches %d\n", bad);
    return bad != 0;
}
