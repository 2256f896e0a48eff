// quant.cu -- 16-bit affine sinogram storage (no counterpart in the reference).
//
// A sinogram is stored as one unsigned 16-bit code per sample plus, per view
// of each batch item (the nv x nu samples of that view), an FP32 offset and
// step: value = lo + step * code, with lo the view's minimum and step its
// range / 65535.  The rounding error of a sample is at most step / 2, i.e.
// 1/131070 of its view's range: for line integrals of 0-8 that is 3e-5, where
// FP16 rounds a value near 6 by up to 2e-3 and BF16 by up to 1.6e-2.  It halves
// the bytes of FP32 storage like the two 16-bit float formats, and keeps a
// reconstruction from it within 1e-4 of the FP32-input one (the float formats
// do not: the ramp filter and the back projection magnify their rounding).
//
//   quantize_u16_kernel   one CTA per view: min / max reduction, then codes
//   dequantize_u16_kernel grid-stride: y = lo + step * code (or y -= ...)
// The exact ramp filter reads the codes directly (fbp.cu, ramp_filter_u16).
#include <cuda_runtime.h>

#include <cfloat>

#include "ctp_common.cuh"

namespace ctp {

namespace {

__global__ void __launch_bounds__(256) quantize_u16_kernel(unsigned short* __restrict__ code,
                                                           float* __restrict__ lo, float* __restrict__ step,
                                                           const float* __restrict__ y, size_t row_len) {
    __shared__ float s_min[8], s_max[8];
    const size_t row = blockIdx.x;
    const float* src = y + row * row_len;
    unsigned short* dst = code + row * row_len;
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (size_t i = threadIdx.x; i < row_len; i += blockDim.x) {
        const float v = __ldg(src + i);
        mn = fminf(mn, v);
        mx = fmaxf(mx, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_min[warp] = mn;
        s_max[warp] = mx;
    }
    __syncthreads();
    mn = s_min[0];
    mx = s_max[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
        mn = fminf(mn, s_min[w]);
        mx = fmaxf(mx, s_max[w]);
    }
    const float range = mx - mn;
    const float st = range > 0.f ? range / 65535.f : 0.f;
    const float inv = range > 0.f ? 65535.f / range : 0.f;
    if (threadIdx.x == 0) {
        lo[row] = mn;
        step[row] = st;
    }
    for (size_t i = threadIdx.x; i < row_len; i += blockDim.x) {
        const float q = rintf((__ldg(src + i) - mn) * inv);
        dst[i] = (unsigned short)fminf(fmaxf(q, 0.f), 65535.f);
    }
}

template <bool kSubtract>
__global__ void dequantize_u16_kernel(float* __restrict__ y, const unsigned short* __restrict__ code,
                                      const float* __restrict__ lo, const float* __restrict__ step, size_t n,
                                      size_t row_len) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t row = i / row_len;
        const float v = fmaf(__ldg(step + row), (float)__ldg(code + i), __ldg(lo + row));
        if (kSubtract)
            y[i] -= v;
        else
            y[i] = v;
    }
}

unsigned grid_for(size_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t want = (n + 255) / 256, cap = (size_t)sms * 8;
    return (unsigned)(want < cap ? (want ? want : 1) : cap);
}

}  // namespace

int quantize_u16(unsigned short* code, float* lo, float* step, const float* y, size_t nrows, size_t row_len,
                 cudaStream_t s) {
    if (nrows == 0 || row_len == 0) return CTP_OK;
    if (!code || !lo || !step || !y) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (nrows > 0x7fffffffULL) return set_error(CTP_ERR_TOO_LARGE, "quantize: %zu rows", nrows);
    quantize_u16_kernel<<<(unsigned)nrows, 256, 0, s>>>(code, lo, step, y, row_len);
    return check_launch("quantize_u16_kernel");
}

int dequantize_u16(float* y, const unsigned short* code, const float* lo, const float* step, size_t nrows,
                   size_t row_len, bool subtract, cudaStream_t s) {
    const size_t n = nrows * row_len;
    if (n == 0) return CTP_OK;
    if (!code || !lo || !step || !y) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    const unsigned grid = grid_for(n);
    if (subtract)
        dequantize_u16_kernel<true><<<grid, 256, 0, s>>>(y, code, lo, step, n, row_len);
    else
        dequantize_u16_kernel<false><<<grid, 256, 0, s>>>(y, code, lo, step, n, row_len);
    return check_launch("dequantize_u16_kernel");
}

}  // namespace ctp
