// culsz_utility.cpp -- the host utilities declared in include/cuLSZ_utility.h
// (the reference's lsCOMP/include/cuLSZ_utility.h interface).
//
// File I/O: raw native-order binary files.  The *_Yafan readers of the
// reference read in the host's byte order unless its data/system endian
// flags differ (lsCOMP/src/cuLSZ_utility.cu:25-26, both 0), so here the
// plain readers and the *_systemEndian_* readers are the same operation.
// Status values follow the reference: 0 success, -2 file error on reads,
// 1 file error on writes.
//
// Quality measures (lossy reports): PSNR and the 7x7x7-window SSIM with
// stride 2, with the definitions of lsCOMP/src/cuLSZ_utility.cu:757-946.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "cuLSZ_utility.h"

namespace {
constexpr int kReadOk = 0;
constexpr int kReadFileError = -2;
constexpr int kWriteOk = 0;
constexpr int kWriteFileError = 1;

// whole file into a malloc'd buffer of `elem`-byte elements
void *read_file(const char *path, size_t elem, size_t *count, int *status)
{
    *count = 0;
    FILE *f = fopen(path, "rb");
    if (!f) {
        printf("Failed to open input file %s\n", path);
        *status = kReadFileError;
        return nullptr;
    }
    fseek(f, 0, SEEK_END);
    long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (size <= 0) {
        printf("Error: input file %s is empty or unreadable\n", path);
        fclose(f);
        *status = kReadFileError;
        return nullptr;
    }
    size_t n = (size_t)size / elem;
    void *buf = malloc(n * elem > 0 ? n * elem : 1);
    if (!buf) {
        fclose(f);
        *status = kReadFileError;
        return nullptr;
    }
    size_t got = fread(buf, elem, n, f);
    fclose(f);
    *count = got;
    *status = got == n ? kReadOk : kReadFileError;
    return buf;
}

void write_file(const void *data, size_t bytes, const char *path, int *status)
{
    FILE *f = fopen(path, "wb");
    if (!f) {
        printf("Failed to open output file %s\n", path);
        *status = kWriteFileError;
        return;
    }
    size_t put = fwrite(data, 1, bytes, f);
    fclose(f);
    *status = put == bytes ? kWriteOk : kWriteFileError;
}

template <int N>
void reverse_bytes(unsigned char *d)
{
    for (int i = 0; i < N / 2; i++) {
        unsigned char t = d[i];
        d[i] = d[N - 1 - i];
        d[N - 1 - i] = t;
    }
}
}  // namespace

void symTransform_2bytes(unsigned char data[2]) { reverse_bytes<2>(data); }
void symTransForm_4Bytes(unsigned char data[4]) { reverse_bytes<4>(data); }
void symTransform_8bytes(unsigned char data[8]) { reverse_bytes<8>(data); }

void convertUShortArrayToBytes(unsigned short *states, size_t stateLength, unsigned char *bytes)
{
    memcpy(bytes, states, stateLength * sizeof(unsigned short));
}

void convertUIntArrayToBytes(unsigned int *states, size_t stateLength, unsigned char *bytes)
{
    memcpy(bytes, states, stateLength * sizeof(unsigned int));
}

unsigned char *readByteData_Yafan(char *srcFilePath, size_t *byteLength, int *status)
{
    return static_cast<unsigned char *>(read_file(srcFilePath, 1, byteLength, status));
}

uint16_t *readUInt16Data_systemEndian_Yafan(char *srcFilePath, size_t *nbEle, int *status)
{
    return static_cast<uint16_t *>(read_file(srcFilePath, 2, nbEle, status));
}

uint16_t *readUInt16Data_Yafan(char *srcFilePath, size_t *nbEle, int *status)
{
    return readUInt16Data_systemEndian_Yafan(srcFilePath, nbEle, status);
}

uint32_t *readUInt32Data_systemEndian_Yafan(char *srcFilePath, size_t *nbEle, int *status)
{
    return static_cast<uint32_t *>(read_file(srcFilePath, 4, nbEle, status));
}

uint32_t *readUInt32Data_Yafan(char *srcFilePath, size_t *nbEle, int *status)
{
    return readUInt32Data_systemEndian_Yafan(srcFilePath, nbEle, status);
}

float *readFloatData_systemEndian_Yafan(char *srcFilePath, size_t *nbEle, int *status)
{
    return static_cast<float *>(read_file(srcFilePath, sizeof(float), nbEle, status));
}

float *readFloatData_Yafan(char *srcFilePath, size_t *nbEle, int *status)
{
    return readFloatData_systemEndian_Yafan(srcFilePath, nbEle, status);
}

double *readDoubleData_systemEndian_Yafan(char *srcFilePath, size_t *nbEle, int *status)
{
    return static_cast<double *>(read_file(srcFilePath, sizeof(double), nbEle, status));
}

double *readDoubleData_Yafan(char *srcFilePath, size_t *nbEle, int *status)
{
    return readDoubleData_systemEndian_Yafan(srcFilePath, nbEle, status);
}

void writeByteData_Yafan(unsigned char *bytes, size_t byteLength, char *tgtFilePath, int *status)
{
    write_file(bytes, byteLength, tgtFilePath, status);
}

void writeUShortData_inBytes_Yafan(unsigned short *states, size_t stateLength, char *tgtFilePath, int *status)
{
    write_file(states, stateLength * sizeof(unsigned short), tgtFilePath, status);
}

void writeUIntData_inBytes_Yafan(unsigned int *states, size_t stateLength, char *tgtFilePath, int *status)
{
    write_file(states, stateLength * sizeof(unsigned int), tgtFilePath, status);
}

void writeFloatData_inBytes_Yafan(float *data, size_t nbEle, char *tgtFilePath, int *status)
{
    write_file(data, nbEle * sizeof(float), tgtFilePath, status);
}

void writeDoubleData_inBytes_Yafan(double *data, size_t nbEle, char *tgtFilePath, int *status)
{
    write_file(data, nbEle * sizeof(double), tgtFilePath, status);
}

// SSIM of one window [offset, offset + window) of two 3-D arrays (size0
// fastest): luminance x contrast x structure with K1 = 0.01, K2 = 0.03 scaled
// by the original's value range in the window (1 when the range is 0), and
// population statistics.
double SSIM_3d_calcWindow_float(float *data, float *other, size_t size1, size_t size0, int offset0, int offset1,
                                int offset2, int windowSize0, int windowSize1, int windowSize2)
{
    double sx = 0, sy = 0;
    float xmin = data[offset0 + size0 * (offset1 + size1 * offset2)], xmax = xmin;
    int np = 0;
    for (int i2 = offset2; i2 < offset2 + windowSize2; i2++)
        for (int i1 = offset1; i1 < offset1 + windowSize1; i1++)
            for (int i0 = offset0; i0 < offset0 + windowSize0; i0++) {
                size_t k = i0 + size0 * (i1 + size1 * i2);
                xmin = data[k] < xmin ? data[k] : xmin;
                xmax = data[k] > xmax ? data[k] : xmax;
                sx += data[k];
                sy += other[k];
                np++;
            }
    const double mx = sx / np, my = sy / np;
    double vx = 0, vy = 0, cxy = 0;
    for (int i2 = offset2; i2 < offset2 + windowSize2; i2++)
        for (int i1 = offset1; i1 < offset1 + windowSize1; i1++)
            for (int i0 = offset0; i0 < offset0 + windowSize0; i0++) {
                size_t k = i0 + size0 * (i1 + size1 * i2);
                vx += (data[k] - mx) * (data[k] - mx);
                vy += (other[k] - my) * (other[k] - my);
                cxy += (data[k] - mx) * (other[k] - my);
            }
    vx /= np;
    vy /= np;
    cxy /= np;
    const double sdx = sqrt(vx), sdy = sqrt(vy);
    // constants evaluated in the reference's order (float range, then
    // K^2 * range * range in double)
    const float range = xmax - xmin;
    const double c1 = range == 0 ? 0.01 * 0.01 : 0.01 * 0.01 * range * range;
    const double c2 = range == 0 ? 0.03 * 0.03 : 0.03 * 0.03 * range * range;
    const double c3 = c2 / 2;
    const double lum = (2 * mx * my + c1) / (mx * mx + my * my + c1);
    const double con = (2 * sdx * sdy + c2) / (sdx * sdx + sdy * sdy + c2);
    const double str = (cxy + c3) / (sdx * sdy + c3);
    return lum * con * str;
}

// Mean SSIM over 7x7x7 windows moved in steps of 2 along every axis.
double computeSSIM(float *oriData, float *decData, size_t size2, size_t size1, size_t size0)
{
    const int w = 7, step = 2;
    if ((size_t)w > size0 || (size_t)w > size1 || (size_t)w > size2)
        printf("ERROR: a dimension is smaller than the SSIM window (%d)\n", w);
    double sum = 0;
    long nw = 0;
    for (size_t o2 = 0; o2 + w <= size2; o2 += step)
        for (size_t o1 = 0; o1 + w <= size1; o1 += step)
            for (size_t o0 = 0; o0 + w <= size0; o0 += step) {
                sum += SSIM_3d_calcWindow_float(oriData, decData, size1, size0, (int)o0, (int)o1, (int)o2, w, w, w);
                nw++;
            }
    return sum / nw;
}

// {MSE, value range, PSNR, L2 error norm, L2 norm of the error over the L2
// norm of the decoded data, NRMSE} in a malloc'd array of 6 doubles.
double *computePSNR(size_t nbEle, float *ori_data, float *data)
{
    double lo = ori_data[0], hi = ori_data[0];
    double se = 0, s22 = 0;
    for (size_t i = 0; i < nbEle; i++) {
        lo = ori_data[i] < lo ? ori_data[i] : lo;
        hi = ori_data[i] > hi ? ori_data[i] : hi;
        // squares formed in float, accumulated in double, as the
        // reference's quality report does
        const float e = fabsf(data[i] - ori_data[i]);
        se += e * e;
        s22 += data[i] * data[i];
    }
    const double mse = se / nbEle, range = hi - lo;
    double *r = (double *)malloc(6 * sizeof(double));
    r[0] = mse;
    r[1] = range;
    r[2] = 20 * log10(range) - 10 * log10(mse);
    r[3] = sqrt(se);
    r[4] = sqrt(se) / sqrt(s22);
    r[5] = sqrt(mse) / range;
    return r;
}
