// tonemap.cu - Pencil's HDR -> 8-bit output path on the device
// (write_image / color_to_rgb8, src/image_io.hpp:40-113; tone curves,
// src/tonemap.hpp:27-61): exposure, tone curve, clamp, gamma 2.2, 8 bits.
//
// Exposure, ACES and Reinhard are plain float arithmetic and round on the
// device as on the host (--fmad=false, IEEE division). The gamma step calls
// the host's powf, whose last bits the device's powf need not match. The
// 8-bit result of that step is a non-decreasing function of the clamped
// value, so it is fully described by 255 thresholds: t[k] is the smallest
// float whose byte is >= k under the host's own powf. They are computed on
// the host by bisection over float bit patterns, once per process, and the
// kernel counts the thresholds at or below each value: the bytes equal the
// host's for every input (tests check the monotonicity over all floats in
// [0, 1] and the bytes against the oracle).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

namespace pgpu {

struct GammaThresholds {
    float t[256];   // t[0] unused; t[k], k = 1..255
};

namespace {

uint8_t host_gamma_byte(float x) {
    x = x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x);
    x = std::pow(x, 1.0f / 2.2f);
    return (uint8_t)(x * 255.0f + 0.5f);
}

float bits_float(uint32_t b) {
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

const GammaThresholds& thresholds() {
    static GammaThresholds g;
    static std::once_flag once;
    std::call_once(once, [] {
        g.t[0] = 0.0f;
        const uint32_t one = 0x3f800000u;   // 1.0f; non-negative floats order as their bits
        for (int k = 1; k < 256; ++k) {
            uint32_t lo = 0, hi = one;       // host_gamma_byte(1) = 255 >= k
            while (lo < hi) {
                const uint32_t mid = lo + (hi - lo) / 2;
                if (host_gamma_byte(bits_float(mid)) >= k) hi = mid;
                else lo = mid + 1;
            }
            g.t[k] = bits_float(lo);
        }
    });
    return g;
}

}  // namespace

// mode: 0 none, 1 ACES, 2 Reinhard (pencil::ToneMap order). `thr`: the 256
// thresholds in device memory, staged in shared memory per block.
__global__ void tm_rgb8(const float* __restrict__ hdr, long long n3, float e, int mode,
                        const float* __restrict__ thr, uint8_t* __restrict__ out) {
    __shared__ float t[256];
    for (int k = threadIdx.x; k < 256; k += blockDim.x) t[k] = thr[k];
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3;
         i += (long long)gridDim.x * blockDim.x) {
        float x = hdr[i] * e;
        if (mode == 1) {
            const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, f = 0.14f;
            const float y = (x * (a * x + b)) / (x * (c * x + d) + f);
            x = 0.0f < y ? y : 0.0f;                       // std::max(0.0f, y)
        } else if (mode == 2) {
            x = x / (1.0f + x);
        }
        x = (x < 0.0f) ? 0.0f : (x > 1.0f) ? 1.0f : x;     // clampf
        int lo = 0, hi = 255;                              // largest k with t[k] <= x
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (t[mid] <= x) lo = mid;
            else hi = mid - 1;
        }
        out[i] = (uint8_t)lo;
    }
}

// The 256 thresholds (t[0] unused) for upload to the device.
const float* gamma_thresholds_host() { return thresholds().t; }

cudaError_t launch_tonemap(const float* d_hdr, long long n_pixels, int mode, float exposure,
                           uint8_t* d_out, const float* d_thr, cudaStream_t st) {
    const float e = std::pow(2.0f, exposure);             // tonemap_color's exposure
    const long long n3 = 3 * n_pixels;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long blocks = (n3 + 255) / 256;
    const int grid = (int)(blocks < (long long)sms * 16 ? (blocks > 0 ? blocks : 1) : sms * 16);
    tm_rgb8<<<grid, 256, 0, st>>>(d_hdr, n3, e, mode, d_thr, d_out);
    return cudaGetLastError();
}

}  // namespace pgpu
