// fvm2d_io.cuh -- frames and state files.
//
// Frames replace the reference's OpenCV recorder (src/wrappers.cuh:253-260,
// 323-345): density as a viridis image, the density range stretched over the
// 256 colours (cv::normalize NORM_MINMAX to 8 bits, then applyColorMap).
// The colour map is rendered on the device into an RGB byte buffer; the host
// writes it as a PNG with stored (uncompressed) deflate blocks, so neither
// OpenCV nor zlib is needed.  The viridis map is taken as linear
// interpolation between its ten published stops at 0, 1/9, ..., 1, which is
// close to, not byte-identical with, OpenCV's 256-entry table.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <vector>

namespace fvm2d {
namespace io {

// Per-block min and max of the density plane, as floats (the reference
// converts the density to CV_32F before normalising).
template <typename T, int NT>
__global__ void density_range_blocks(const T *__restrict__ rho, int pitch, int nx, int ny, float *__restrict__ out)
{
    __shared__ float lo[NT], hi[NT];
    float a = INFINITY, b = -INFINITY;
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < n; k += (long long)gridDim.x * NT) {
        const float v = float(rho[(k / nx) * pitch + k % nx]);
        a = fminf(a, v);
        b = fmaxf(b, v);
    }
    lo[threadIdx.x] = a;
    hi[threadIdx.x] = b;
    __syncthreads();
    for (int s = NT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            lo[threadIdx.x] = fminf(lo[threadIdx.x], lo[threadIdx.x + s]);
            hi[threadIdx.x] = fmaxf(hi[threadIdx.x], hi[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[2 * blockIdx.x] = lo[0];
        out[2 * blockIdx.x + 1] = hi[0];
    }
}

// Viridis at ten evenly spaced stops (RGB).
__constant__ unsigned char kViridis[10][3] = {
    {68, 1, 84},    {72, 40, 120},  {62, 73, 137},  {49, 104, 142}, {38, 130, 142},
    {31, 158, 137}, {53, 183, 121}, {110, 206, 88}, {181, 222, 43}, {253, 231, 37},
};

// Pixel (i, j) of row j: level = round((rho - min) * 255 / (max - min)),
// colour = viridis(level / 255).  nblocks partial ranges are folded first.
template <typename T>
__global__ void render_density(const T *__restrict__ rho, int pitch, int nx, int ny, const float *__restrict__ parts,
                               int nblocks, unsigned char *__restrict__ rgb)
{
    float lo = INFINITY, hi = -INFINITY;
    for (int b = 0; b < nblocks; ++b) {
        lo = fminf(lo, parts[2 * b]);
        hi = fmaxf(hi, parts[2 * b + 1]);
    }
    const double scale = hi > lo ? 255.0 / (double(hi) - double(lo)) : 0.0;
    const double shift = -double(lo) * scale;
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const float v = float(rho[(k / nx) * pitch + k % nx]);
        double level = rint(double(v) * scale + shift);
        level = level < 0.0 ? 0.0 : (level > 255.0 ? 255.0 : level);
        const double pos = level * 9.0 / 255.0;
        int s = int(pos);
        if (s > 8) s = 8;
        const double f = pos - s;
        for (int c = 0; c < 3; ++c) {
            const double x = kViridis[s][c] + f * (double(kViridis[s + 1][c]) - double(kViridis[s][c]));
            rgb[3 * k + c] = (unsigned char)rint(x);
        }
    }
}

// ---- PNG (RFC 2083) with a zlib stream (RFC 1950) of stored deflate blocks
// (RFC 1951, BTYPE 00) -----------------------------------------------------
inline uint32_t crc32_update(uint32_t crc, const unsigned char *p, size_t n)
{
    static uint32_t table[256];
    static bool ready = false;
    if (!ready) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[i] = c;
        }
        ready = true;
    }
    for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xFF] ^ (crc >> 8);
    return crc;
}

inline void put_be32(std::vector<unsigned char> &v, uint32_t x)
{
    v.push_back((unsigned char)(x >> 24));
    v.push_back((unsigned char)(x >> 16));
    v.push_back((unsigned char)(x >> 8));
    v.push_back((unsigned char)x);
}

inline void put_chunk(FILE *f, const char *type, const std::vector<unsigned char> &data)
{
    std::vector<unsigned char> head;
    put_be32(head, (uint32_t)data.size());
    fwrite(head.data(), 1, 4, f);
    fwrite(type, 1, 4, f);
    if (!data.empty()) fwrite(data.data(), 1, data.size(), f);
    uint32_t crc = crc32_update(0xFFFFFFFFu, reinterpret_cast<const unsigned char *>(type), 4);
    crc = crc32_update(crc, data.data(), data.size()) ^ 0xFFFFFFFFu;
    std::vector<unsigned char> tail;
    put_be32(tail, crc);
    fwrite(tail.data(), 1, 4, f);
}

// Writes width x height RGB pixels (rows top to bottom).  Returns false on an
// I/O error.
inline bool write_png_rgb(const char *path, int width, int height, const unsigned char *rgb)
{
    FILE *f = std::fopen(path, "wb");
    if (!f) return false;
    static const unsigned char sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    fwrite(sig, 1, 8, f);
    std::vector<unsigned char> ihdr;
    put_be32(ihdr, (uint32_t)width);
    put_be32(ihdr, (uint32_t)height);
    ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});  // 8 bits, RGB, deflate, adaptive filters, no interlace
    put_chunk(f, "IHDR", ihdr);
    // raw scanlines: filter byte 0 + the row
    const size_t row = 3 * (size_t)width, raw = (row + 1) * (size_t)height;
    std::vector<unsigned char> idat;
    idat.reserve(raw + raw / 65535 * 5 + 16);
    idat.push_back(0x78);  // zlib: deflate, 32 KB window
    idat.push_back(0x01);  // check bits, no dictionary, fastest
    uint32_t a = 1, b = 0;  // Adler-32
    size_t done = 0, in_block = 0;
    auto open_block = [&](size_t len, bool last) {
        idat.push_back(last ? 1 : 0);
        idat.push_back((unsigned char)(len & 0xFF));
        idat.push_back((unsigned char)(len >> 8));
        idat.push_back((unsigned char)(~len & 0xFF));
        idat.push_back((unsigned char)((~len >> 8) & 0xFF));
        in_block = len;
    };
    auto emit = [&](unsigned char byte) {
        if (in_block == 0) {
            const size_t left = raw - done;
            const size_t len = left < 65535 ? left : 65535;
            open_block(len, len == left);
        }
        idat.push_back(byte);
        --in_block;
        ++done;
        a = (a + byte) % 65521u;
        b = (b + a) % 65521u;
    };
    for (int j = 0; j < height; ++j) {
        emit(0);
        const unsigned char *r = rgb + row * (size_t)j;
        for (size_t i = 0; i < row; ++i) emit(r[i]);
    }
    put_be32(idat, (b << 16) | a);
    put_chunk(f, "IDAT", idat);
    put_chunk(f, "IEND", {});
    const bool ok = std::ferror(f) == 0;
    return std::fclose(f) == 0 && ok;
}

// ---- state files ------------------------------------------------------------
// "FVM2DST1", int32 nx, int32 ny, double t, int64 steps, then ny*nx cells of
// four doubles (rho, p, u, v), row by row, little-endian.
struct StateFileHeader {
    char magic[8];
    int32_t nx, ny;
    double t;
    int64_t steps;
};

} // namespace io
} // namespace fvm2d
