// tv.cu -- separable-quadratic-surrogate terms of the anisotropic TV prior,
// sm_100a.
//
// Reference: Variation3DKernel and TVSQS3DKernel
// (kernel/prior/cuda/TotalVariation.cu:21-149 of the reference), computed
// there in two passes.  Here one pass: each thread owns one voxel, computes
// its variation and that of its three forward neighbours (whose backward
// differences it can form from the same cached neighbourhood), and writes the
// surrogate numerator s1, denominator s2 and the variation map.  x is the
// fastest index, so every load and store is coalesced; the image is read from
// HBM once (neighbour reads hit L1/L2).
#include <cuda_runtime.h>
#include <math.h>

#include "ctp_common.cuh"

namespace ctp {

namespace {

struct Vol {
    const float* __restrict__ p;
    int nx, ny, nz;
    size_t nxy;
};

__device__ __forceinline__ float at(const Vol& v, int ix, int iy, int iz) {
    return __ldg(v.p + (size_t)iz * v.nxy + (size_t)iy * v.nx + ix);
}

// sqrt(wx dx^2 + wy dy^2 + wz dz^2 + eps) with backward differences, zero at
// the low borders (TotalVariation.cu:21-55).
__device__ __forceinline__ float variation(const Vol& v, int ix, int iy, int iz, float wx, float wy, float wz,
                                           float eps) {
    float x = at(v, ix, iy, iz);
    float dx = ix > 0 ? x - at(v, ix - 1, iy, iz) : 0.f;
    float dy = iy > 0 ? x - at(v, ix, iy - 1, iz) : 0.f;
    float dz = iz > 0 ? x - at(v, ix, iy, iz - 1) : 0.f;
    return sqrtf(wx * dx * dx + wy * dy * dy + wz * dz * dz + eps);
}

__global__ void tv_sqs_kernel(float* __restrict__ s1, float* __restrict__ s2, float* __restrict__ var,
                              const float* __restrict__ img, float wx, float wy, float wz, int nx, int ny, int nz,
                              float eps) {
    int ix = blockIdx.x * blockDim.x + threadIdx.x;
    int iy = blockIdx.y * blockDim.y + threadIdx.y;
    int bz = blockIdx.z;
    int iz = bz % nz, b = bz / nz;
    if (ix >= nx || iy >= ny) return;
    size_t nxy = (size_t)nx * ny;
    size_t base = (size_t)b * nz * nxy;
    Vol v{img + base, nx, ny, nz, nxy};
    size_t ind = (size_t)iz * nxy + (size_t)iy * nx + ix;
    float x = at(v, ix, iy, iz);
    float vv = variation(v, ix, iy, iz, wx, wy, wz, eps);
    // TotalVariation.cu:69-149: forward neighbour's variation, or this voxel's at the high border
    float dx0 = 0.f, dx1 = 0.f, dy0 = 0.f, dy1 = 0.f, dz0 = 0.f, dz1 = 0.f;
    float varx = vv, vary = vv, varz = vv;
    if (ix > 0) dx0 = x - at(v, ix - 1, iy, iz);
    if (ix < nx - 1) {
        dx1 = x - at(v, ix + 1, iy, iz);
        varx = variation(v, ix + 1, iy, iz, wx, wy, wz, eps);
    }
    if (iy > 0) dy0 = x - at(v, ix, iy - 1, iz);
    if (iy < ny - 1) {
        dy1 = x - at(v, ix, iy + 1, iz);
        vary = variation(v, ix, iy + 1, iz, wx, wy, wz, eps);
    }
    if (iz > 0) dz0 = x - at(v, ix, iy, iz - 1);
    if (iz < nz - 1) {
        dz1 = x - at(v, ix, iy, iz + 1);
        varz = variation(v, ix, iy, iz + 1, wx, wy, wz, eps);
    }
    dx0 *= wx;
    dx1 *= wx;
    dy0 *= wy;
    dy1 *= wy;
    dz0 *= wz;
    dz1 *= wz;
    s1[base + ind] = (dx0 + dy0 + dz0) / vv + dx1 / varx + dy1 / vary + dz1 / varz;
    s2[base + ind] = (wx + wy + wz) / vv + wx / varx + wy / vary + wz / varz;
    var[base + ind] = vv;
}


// One SQS iteration with the TV prior, fused: x_out = x - (bp + beta s1(x)) /
// (norm + beta s2(x)), with s1, s2 those of tv_sqs_kernel.  The slices are a
// flat array; zlink[i] bit 0 says slice i has its z neighbour i-1 in the same
// volume and bit 1 the neighbour i+1, so volumes of different depths packed
// back to back keep the reference's border rule (zero backward difference at
// the first slice, own variation past the last) at their own borders.
struct Slices {
    const float* __restrict__ p;
    int nx, ny;
    size_t nxy;
};

__device__ __forceinline__ float at_s(const Slices& v, int ix, int iy, int is) {
    return __ldg(v.p + (size_t)is * v.nxy + (size_t)iy * v.nx + ix);
}

// variation at (ix, iy, slice is); has_prev: slice is-1 belongs to the same volume
__device__ __forceinline__ float variation_s(const Slices& v, int ix, int iy, int is, bool has_prev, float wx,
                                             float wy, float wz, float eps) {
    float x = at_s(v, ix, iy, is);
    float dx = ix > 0 ? x - at_s(v, ix - 1, iy, is) : 0.f;
    float dy = iy > 0 ? x - at_s(v, ix, iy - 1, is) : 0.f;
    float dz = has_prev ? x - at_s(v, ix, iy, is - 1) : 0.f;
    return sqrtf(wx * dx * dx + wy * dy * dy + wz * dz * dz + eps);
}

template <typename Tlp>
__global__ void sqs_tv_update_kernel(float* __restrict__ x_out, Tlp* __restrict__ x_lp, const float* __restrict__ x,
                                     const float* __restrict__ bp, const float* __restrict__ norm, int norm_slices,
                                     const unsigned char* __restrict__ zlink, float wx, float wy, float wz,
                                     float beta, float eps, int nx, int ny) {
    int ix = blockIdx.x * blockDim.x + threadIdx.x;
    int iy = blockIdx.y * blockDim.y + threadIdx.y;
    int is = blockIdx.z;
    if (ix >= nx || iy >= ny) return;
    size_t nxy = (size_t)nx * ny;
    Slices v{x, nx, ny, nxy};
    const unsigned link = zlink ? zlink[is] : 0u;
    const bool prev = link & 1u, next = link & 2u;
    size_t ind = (size_t)is * nxy + (size_t)iy * nx + ix;
    float xv = at_s(v, ix, iy, is);
    float vv = variation_s(v, ix, iy, is, prev, wx, wy, wz, eps);
    float dx0 = 0.f, dx1 = 0.f, dy0 = 0.f, dy1 = 0.f, dz0 = 0.f, dz1 = 0.f;
    float varx = vv, vary = vv, varz = vv;
    if (ix > 0) dx0 = xv - at_s(v, ix - 1, iy, is);
    if (ix < nx - 1) {
        dx1 = xv - at_s(v, ix + 1, iy, is);
        varx = variation_s(v, ix + 1, iy, is, prev, wx, wy, wz, eps);
    }
    if (iy > 0) dy0 = xv - at_s(v, ix, iy - 1, is);
    if (iy < ny - 1) {
        dy1 = xv - at_s(v, ix, iy + 1, is);
        vary = variation_s(v, ix, iy + 1, is, prev, wx, wy, wz, eps);
    }
    if (prev) dz0 = xv - at_s(v, ix, iy, is - 1);
    if (next) {
        dz1 = xv - at_s(v, ix, iy, is + 1);
        varz = variation_s(v, ix, iy, is + 1, true, wx, wy, wz, eps);
    }
    float s1 = (wx * dx0 + wy * dy0 + wz * dz0) / vv + wx * dx1 / varx + wy * dy1 / vary + wz * dz1 / varz;
    float s2 = (wx + wy + wz) / vv + wx / varx + wy / vary + wz / varz;
    float nv = __ldg(norm + (size_t)(is % norm_slices) * nxy + (size_t)iy * nx + ix);
    float out = xv - (__ldg(bp + ind) + beta * s1) / (nv + beta * s2);
    x_out[ind] = out;
    if (x_lp) stf(x_lp + ind, out);
}

}  // namespace

int tv_sqs(float* s1, float* s2, float* var, const float* img, float wx, float wy, float wz, size_t nb, size_t nx,
           size_t ny, size_t nz, float eps, cudaStream_t s) {
    if (nb == 0) return CTP_OK;
    if (!s1 || !s2 || !var || !img) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (nx == 0 || ny == 0 || nz == 0) return set_error(CTP_ERR_INVALID_ARGUMENT, "zero image extent");
    if (nb * nz > 65535 * 64) return set_error(CTP_ERR_INVALID_ARGUMENT, "too many slices");
    dim3 block(32, 8);
    dim3 grid((unsigned)((nx + 31) / 32), (unsigned)((ny + 7) / 8), (unsigned)(nb * nz));
    tv_sqs_kernel<<<grid, block, 0, s>>>(s1, s2, var, img, wx, wy, wz, (int)nx, (int)ny, (int)nz, eps);
    return check_launch("tv_sqs_kernel");
}

int sqs_tv_update(float* x_out, void* x_lp, const float* x, const float* bp, const float* norm, size_t norm_slices,
                  const unsigned char* zlink, float wx, float wy, float wz, float beta, float eps, size_t nx,
                  size_t ny, size_t nslices, unsigned flags, cudaStream_t s) {
    if (nslices == 0) return CTP_OK;
    if (!x_out || !x || !bp || !norm) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (x_out == x) return set_error(CTP_ERR_INVALID_ARGUMENT, "x_out must not alias x (neighbours are read)");
    if (nx == 0 || ny == 0 || norm_slices == 0) return set_error(CTP_ERR_INVALID_ARGUMENT, "zero extent");
    if (nslices > 65535u * 64u) return set_error(CTP_ERR_INVALID_ARGUMENT, "too many slices");
    const bool bf = flags & CTP_FLAG_OUT_BF16, hf = flags & CTP_FLAG_OUT_FP16;
    if (x_lp && bf == hf) return set_error(CTP_ERR_INVALID_ARGUMENT, "x_lp needs exactly one of OUT_BF16/OUT_FP16");
    dim3 block(32, 8);
    dim3 grid((unsigned)((nx + 31) / 32), (unsigned)((ny + 7) / 8), (unsigned)nslices);
    if (x_lp && bf)
        sqs_tv_update_kernel<__nv_bfloat16><<<grid, block, 0, s>>>(x_out, static_cast<__nv_bfloat16*>(x_lp), x, bp,
                                                                  norm, (int)norm_slices, zlink, wx, wy, wz, beta,
                                                                  eps, (int)nx, (int)ny);
    else if (x_lp)
        sqs_tv_update_kernel<__half><<<grid, block, 0, s>>>(x_out, static_cast<__half*>(x_lp), x, bp, norm,
                                                           (int)norm_slices, zlink, wx, wy, wz, beta, eps, (int)nx,
                                                           (int)ny);
    else
        sqs_tv_update_kernel<float><<<grid, block, 0, s>>>(x_out, nullptr, x, bp, norm, (int)norm_slices, zlink, wx,
                                                          wy, wz, beta, eps, (int)nx, (int)ny);
    return check_launch("sqs_tv_update_kernel");
}

}  // namespace ctp
