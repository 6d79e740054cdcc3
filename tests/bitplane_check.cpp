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
