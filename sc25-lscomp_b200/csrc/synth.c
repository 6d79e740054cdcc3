/*
 * synth.c -- seeded synthetic light-source detector stacks (uint16, z fastest).
 *
 * The datasets the lsCOMP paper measured on (CSSI, XPCS beamline captures)
 * are not public; these generators stand in for them with the shapes and
 * value distributions of the workloads this library is measured on:
 *
 *   small : Poisson(0.1) background, 20 Gaussian spots per frame with peak
 *           U(200,5000) counts and sigma U(1.5,4) px, 0.1% hot pixels = 65535.
 *   cssi  : per-frame Poisson background whose mean falls radially from 50
 *           at the beam centre to 0.5 at the far corner, 3-8 concentric rings
 *           with Gaussian radial profile and peak U(500,20000) counts, and a
 *           rectangular beamstop of zeros.
 *   xpcs  : speckle intensity = 0.02 * |A|^2 with A a unit complex Gaussian
 *           per pixel that follows A_t = rho*A_{t-1} + sqrt(1-rho^2)*eps_t
 *           (rho = 0.9) from frame to frame, Poisson-sampled (about 98% zeros),
 *           and a zero beamstop disk of radius 60 px.
 *
 * Every random draw is a pure function of (seed, frame, pixel, draw index)
 * (a SplitMix64 counter hash), so the output does not depend on the number
 * of threads, and any frame range can be generated on its own.
 */
#include <stdint.h>
#include <stddef.h>
#include <math.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static inline uint64_t mix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

/* uniform in (0,1) from a counter */
static inline double unif(uint64_t key, uint64_t ctr)
{
    uint64_t r = mix64(key ^ mix64(ctr));
    return ((double)(r >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

static inline uint64_t stream_key(uint64_t seed, uint64_t tag)
{
    return mix64(seed * 0x632be59bd9b4e019ull + tag);
}

/* standard normal from two counter uniforms (Box-Muller) */
static inline double gauss(uint64_t key, uint64_t ctr)
{
    double u1 = unif(key, 2 * ctr), u2 = unif(key, 2 * ctr + 1);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

/* Poisson(lambda) from one uniform by CDF inversion for small means and a
   rounded normal approximation above 30 counts. */
static inline uint32_t poisson(double lambda, uint64_t key, uint64_t ctr)
{
    if (lambda <= 0.0) return 0;
    if (lambda > 30.0) {
        double v = lambda + sqrt(lambda) * gauss(key, ctr) + 0.5;
        if (v < 0.0) v = 0.0;
        if (v > 65535.0) v = 65535.0;
        return (uint32_t)v;
    }
    double u = unif(key, ctr);
    double p = exp(-lambda), F = p;
    uint32_t k = 0;
    while (u > F && k < 200) {
        k++;
        p *= lambda / k;
        F += p;
    }
    return k;
}

static inline uint16_t clamp16(double v)
{
    if (v <= 0.0) return 0;
    if (v >= 65535.0) return 65535;
    return (uint16_t)v;
}

static void set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ---------------------------------------------------------------- small */
int lsc_synth_small(uint16_t *out, uint32_t X, uint32_t Y, uint32_t Z, uint32_t x0, uint32_t nx,
                    uint64_t seed, int nthreads)
{
    if (!out || x0 + nx > X) return -1;
    set_threads(nthreads);
    const uint64_t HW = (uint64_t)Y * Z;
    int64_t f;
#pragma omp parallel for schedule(dynamic, 1)
    for (f = 0; f < (int64_t)nx; f++) {
        uint64_t x = x0 + (uint64_t)f;
        uint16_t *fr = out + (uint64_t)f * HW;
        uint64_t kb = stream_key(seed, 0x100000000ull + x);
        for (uint64_t i = 0; i < HW; i++) {
            /* Poisson(0.1) by inversion */
            double u = unif(kb, i);
            double p = 0.9048374180359595, F = p; /* exp(-0.1) */
            uint32_t k = 0;
            while (u > F && k < 20) { k++; p *= 0.1 / k; F += p; }
            fr[i] = (uint16_t)k;
        }
        uint64_t ks = stream_key(seed, 0x200000000ull + x);
        for (int s = 0; s < 20; s++) {
            double cy = unif(ks, 8 * s) * Y, cz = unif(ks, 8 * s + 1) * Z;
            double amp = 200.0 + 4800.0 * unif(ks, 8 * s + 2);
            double sig = 1.5 + 2.5 * unif(ks, 8 * s + 3);
            int r = (int)ceil(4.0 * sig);
            for (int dy = -r; dy <= r; dy++) {
                int64_t yy = (int64_t)floor(cy) + dy;
                if (yy < 0 || yy >= (int64_t)Y) continue;
                for (int dz = -r; dz <= r; dz++) {
                    int64_t zz = (int64_t)floor(cz) + dz;
                    if (zz < 0 || zz >= (int64_t)Z) continue;
                    double ddy = yy + 0.5 - cy, ddz = zz + 0.5 - cz;
                    double v = amp * exp(-(ddy * ddy + ddz * ddz) / (2.0 * sig * sig));
                    uint64_t idx = (uint64_t)yy * Z + (uint64_t)zz;
                    fr[idx] = clamp16((double)fr[idx] + v);
                }
            }
        }
        uint64_t kh = stream_key(seed, 0x300000000ull + x);
        uint64_t nhot = HW / 1000;
        for (uint64_t h = 0; h < nhot; h++) {
            uint64_t idx = mix64(kh ^ mix64(h)) % HW;
            fr[idx] = 65535;
        }
    }
    return 0;
}

/* ----------------------------------------------------------------- cssi */
typedef struct {
    double cy, cz, rmax;
    int nrings;
    double rad[8], wid[8], amp[8];
    int64_t bs_y0, bs_y1, bs_z0, bs_z1;
} cssi_scene;

static void cssi_make_scene(cssi_scene *s, uint32_t Y, uint32_t Z, uint64_t seed)
{
    uint64_t k = stream_key(seed, 0x400000000ull);
    s->cy = Y * (0.45 + 0.1 * unif(k, 0));
    s->cz = Z * (0.45 + 0.1 * unif(k, 1));
    double dy = (s->cy > Y - s->cy) ? s->cy : Y - s->cy;
    double dz = (s->cz > Z - s->cz) ? s->cz : Z - s->cz;
    s->rmax = sqrt(dy * dy + dz * dz);
    s->nrings = 3 + (int)(unif(k, 2) * 6.0);
    if (s->nrings > 8) s->nrings = 8;
    for (int j = 0; j < s->nrings; j++) {
        s->rad[j] = s->rmax * (0.08 + 0.8 * unif(k, 10 + 3 * j));
        s->wid[j] = 1.5 + 6.0 * unif(k, 11 + 3 * j);
        s->amp[j] = 500.0 + 19500.0 * unif(k, 12 + 3 * j);
    }
    double hy = (Y < 64 ? Y : 64) * (0.4 + 0.6 * unif(k, 40));
    double hz = (Z < 96 ? Z : 96) * (0.4 + 0.6 * unif(k, 41));
    s->bs_y0 = (int64_t)(s->cy - hy / 2);
    s->bs_y1 = (int64_t)(s->cy + hy / 2);
    s->bs_z0 = (int64_t)(s->cz - hz / 2);
    s->bs_z1 = (int64_t)(s->cz + hz / 2);
}

int lsc_synth_cssi(uint16_t *out, uint32_t X, uint32_t Y, uint32_t Z, uint32_t x0, uint32_t nx,
                   uint64_t seed, int nthreads)
{
    if (!out || x0 + nx > X) return -1;
    set_threads(nthreads);
    cssi_scene s;
    cssi_make_scene(&s, Y, Z, seed);
    const uint64_t HW = (uint64_t)Y * Z;
    float *bg = (float *)malloc(HW * sizeof(float));
    float *ring = (float *)malloc(HW * sizeof(float));
    if (!bg || !ring) { free(bg); free(ring); return -2; }
    int64_t yy;
#pragma omp parallel for schedule(static)
    for (yy = 0; yy < (int64_t)Y; yy++) {
        for (uint64_t z = 0; z < Z; z++) {
            double dy = yy + 0.5 - s.cy, dz = z + 0.5 - s.cz;
            double r = sqrt(dy * dy + dz * dz);
            uint64_t i = (uint64_t)yy * Z + z;
            bg[i] = (float)(50.0 * pow(0.01, r / s.rmax));
            double rv = 0.0;
            for (int j = 0; j < s.nrings; j++) {
                double d = (r - s.rad[j]) / s.wid[j];
                if (d > -6.0 && d < 6.0) rv += s.amp[j] * exp(-0.5 * d * d);
            }
            ring[i] = (float)rv;
            if (yy >= s.bs_y0 && yy < s.bs_y1 && (int64_t)z >= s.bs_z0 && (int64_t)z < s.bs_z1) {
                bg[i] = -1.0f; /* beamstop marker */
                ring[i] = 0.0f;
            }
        }
    }
    int64_t t;
    const uint64_t rows = (uint64_t)nx * Y;
#pragma omp parallel for schedule(dynamic, 8)
    for (t = 0; t < (int64_t)rows; t++) {
        uint64_t f = (uint64_t)t / Y, y = (uint64_t)t % Y;
        uint64_t x = x0 + f;
        double scale = 0.8 + 0.4 * unif(stream_key(seed, 0x500000000ull), x);
        uint64_t key = stream_key(seed, 0x600000000ull + x);
        uint16_t *row = out + f * HW + y * Z;
        for (uint64_t z = 0; z < Z; z++) {
            uint64_t i = y * Z + z;
            if (bg[i] < 0.0f) { row[z] = 0; continue; }
            double lam = (double)bg[i] + scale * (double)ring[i];
            row[z] = clamp16((double)poisson(lam, key, i));
        }
    }
    free(bg);
    free(ring);
    return 0;
}

/* ----------------------------------------------------------------- xpcs */
int lsc_synth_xpcs(uint16_t *out, uint32_t X, uint32_t Y, uint32_t Z, uint32_t x0, uint32_t nx,
                   uint64_t seed, int nthreads)
{
    if (!out || x0 + nx > X) return -1;
    set_threads(nthreads);
    const double rho = 0.9, innov = sqrt(1.0 - rho * rho), mean = 0.02;
    const uint64_t HW = (uint64_t)Y * Z;
    const double cy = Y * 0.5, cz = Z * 0.5, r2stop = 60.0 * 60.0;
    int64_t pix;
#pragma omp parallel for schedule(static)
    for (pix = 0; pix < (int64_t)HW; pix++) {
        uint64_t y = (uint64_t)pix / Z, z = (uint64_t)pix % Z;
        double dy = y + 0.5 - cy, dz = z + 0.5 - cz;
        int stop = dy * dy + dz * dz < r2stop;
        uint64_t kA = stream_key(seed, 0x700000000ull + (uint64_t)pix);
        /* A_0 ~ CN(0,1): real and imaginary parts N(0, 1/2) */
        double ar = gauss(kA, 0) * 0.7071067811865476, ai = gauss(kA, 1) * 0.7071067811865476;
        uint64_t kP = stream_key(seed, 0x800000000ull + (uint64_t)pix);
        for (uint64_t x = 0; x < x0 + nx; x++) {
            if (x > 0) {
                ar = rho * ar + innov * 0.7071067811865476 * gauss(kA, 2 * x);
                ai = rho * ai + innov * 0.7071067811865476 * gauss(kA, 2 * x + 1);
            }
            if (x < x0) continue;
            uint16_t v = 0;
            if (!stop) {
                double lam = mean * (ar * ar + ai * ai);
                double u = unif(kP, x);
                double p = exp(-lam), F = p;
                uint32_t k = 0;
                while (u > F && k < 64) { k++; p *= lam / k; F += p; }
                v = (uint16_t)k;
            }
            out[(x - x0) * HW + (uint64_t)pix] = v;
        }
    }
    return 0;
}
