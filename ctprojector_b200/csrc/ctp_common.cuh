// ctp_common.cuh -- shared types and helpers of the sm_100a projector pair.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/ctp.h"

namespace ctp {

// Blend band of the distance-driven tracer (distanceDriven2DBoxInt.cu:18).
constexpr float kDDMargin = 0.12f;
constexpr double kDDMarginD = 0.12;

// ---------------------------------------------------------------- host side
int set_error(int code, const char* fmt, ...);
// Reports a launch failure of the kernels just enqueued (cudaGetLastError).
int check_launch(const char* what);
// Validates pointers/sizes shared by every entry.  Returns CTP_OK or sets the
// error and returns CTP_ERR_INVALID_ARGUMENT.
int check_geometry(const ctp_geometry* g, bool need_image, bool need_detector);

inline size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

// staging.cu: the library's stream-ordered scratch pool (plain
// cudaMallocAsync under graph capture), and copies between pageable host
// arrays and the device through pinned chunks (synchronous for downloads).
int scratch_alloc(void** p, size_t bytes, cudaStream_t s);
unsigned long long scratch_allocations();  // successful scratch_alloc calls since load
int staged_upload(void* dst, const void* src, size_t bytes, cudaStream_t s);
int staged_download(void* dst, const void* src, size_t bytes, cudaStream_t s);

// Scratch memory for one call: the caller's workspace when given, otherwise a
// stream-ordered pool allocation released on the same stream.
class Scratch {
   public:
    Scratch() = default;
    Scratch(const Scratch&) = delete;
    Scratch& operator=(const Scratch&) = delete;
    ~Scratch();
    int acquire(void* user, size_t user_bytes, size_t need, cudaStream_t s);
    char* base() const { return static_cast<char*>(ptr_); }

   private:
    void* ptr_ = nullptr;
    bool owned_ = false;
    cudaStream_t stream_ = nullptr;
};

// Element size of the storage type selected by the IN/OUT flags.
inline int elem_size_in(unsigned flags) { return (flags & (CTP_FLAG_IN_BF16 | CTP_FLAG_IN_FP16)) ? 2 : 4; }
inline int elem_size_out(unsigned flags) { return (flags & (CTP_FLAG_OUT_BF16 | CTP_FLAG_OUT_FP16)) ? 2 : 4; }

// ---------------------------------------------------------------- device side
struct Grid {
    int nx, ny, nz;
    float dx, dy, dz, cx, cy, cz;
};

struct Det {
    int nu, nv;
    float du, dv, off_u, off_v;
};

inline Grid make_grid(const ctp_geometry& g) {
    return Grid{(int)g.nx, (int)g.ny, (int)g.nz, g.dx, g.dy, g.dz, g.cx, g.cy, g.cz};
}
inline Det make_det(const ctp_geometry& g) { return Det{(int)g.nu, (int)g.nv, g.du, g.dv, g.off_u, g.off_v}; }

__device__ __forceinline__ float ldf(const float* p) { return __ldg(p); }
__device__ __forceinline__ float ldf(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
__device__ __forceinline__ float ldf(const __half* p) { return __half2float(__ldg(p)); }

__device__ __forceinline__ void stf(float* p, float v) { *p = v; }
__device__ __forceinline__ void stf(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
__device__ __forceinline__ void stf(__half* p, float v) { *p = __float2half_rn(v); }

__device__ __forceinline__ float rdf(const float* p) { return *p; }
__device__ __forceinline__ float rdf(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ float rdf(const __half* p) { return __half2float(*p); }

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// Exact integral over [lo, hi], clamped to [0, n], of a line of n cells
// whose cell i holds p[i*stride]: the pixel sum minus the partial edges, as
// in IntegralBoxX/IntegralBoxY (cudaMath.cu:533-601).
template <typename T>
__device__ __forceinline__ float box_line(const T* p, int stride, float lo, float hi, int n) {
    lo = clampf(lo, 0.f, (float)n);
    hi = clampf(hi, 0.f, (float)n);
    if (hi <= lo) return 0.f;
    int i1 = min((int)lo, n - 1);
    int i2 = min((int)hi, n - 1);
    float s = 0.f;
    for (int i = i1; i <= i2; ++i) s += ldf(p + (size_t)i * stride);
    s -= ldf(p + (size_t)i1 * stride) * (lo - (float)i1);
    s -= ldf(p + (size_t)i2 * stride) * ((float)(i2 + 1) - hi);
    return s;
}

// Same on a shared-memory line (plain loads).
__device__ __forceinline__ float box_line_smem(const float* p, float lo, float hi, int n) {
    lo = clampf(lo, 0.f, (float)n);
    hi = clampf(hi, 0.f, (float)n);
    if (hi <= lo) return 0.f;
    int i1 = min((int)lo, n - 1);
    int i2 = min((int)hi, n - 1);
    float s = 0.f;
    for (int i = i1; i <= i2; ++i) s += p[i];
    s -= p[i1] * (lo - (float)i1);
    s -= p[i2] * ((float)(i2 + 1) - hi);
    return s;
}

}  // namespace ctp
