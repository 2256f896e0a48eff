// siddon.cu -- Siddon cone-beam projector pair for arbitrary trajectories,
// sm_100a.
//
// Reference: siddon.cu (InboundAlpha :37, InboundFirstVoxel :59,
// OutboundFirstVoxel :78, GetAlpha :95, InitializeSiddon :104, SiddonRayTracing
// :175, SiddonRayTracingTransposeAtomicAdd :259, MoveSourceDstNearGrid :342)
// and siddonCone.cu:12-74 (one ray per detector cell; u,v measured from the
// detector centre along det_u / det_v).
//
// The ray set-up (near-grid move, entry/exit parameters, first voxel) and the
// alpha recurrences run in FP64, so segment lengths do not drift along the
// walk; the line integral accumulates in FP32.  Forward and back projection
// share the same walk function, so the back projector is the exact transpose
// of the forward projector up to FP32 rounding of the accumulation.
// One thread per ray; a 32x8 block covers a detector tile so that a warp's
// rays traverse neighbouring voxels.
#include <cuda_runtime.h>
#include <math.h>

#include "ctp_common.cuh"

namespace ctp {

namespace {

constexpr double kEps = 1e-6;  // siddon.cu:35

struct Ray {
    double alpha[3], dalpha[3];
    int ng[3];
    int step[3];  // voxel index step along x, y, z (+-1, or 0)
    double aprev;
    bool hit;
};

// Ray end points for cell (iu, iv) of a view, moved near the grid.
__device__ void ray_ends(double src[3], double dst[3], int view, int iu, int iv, const float* __restrict__ dc,
                         const float* __restrict__ du_, const float* __restrict__ dv_,
                         const float* __restrict__ sr, const Grid& g, const Det& d) {
    double u = ((double)iu - d.off_u - (d.nu - 1) / 2.0) * d.du;
    double v = ((double)iv - d.off_v - (d.nv - 1) / 2.0) * d.dv;
    for (int k = 0; k < 3; ++k) {
        src[k] = (double)sr[view * 3 + k];
        dst[k] = (double)dc[view * 3 + k] + (double)du_[view * 3 + k] * u + (double)dv_[view * 3 + k] * v;
    }
    // MoveSourceDstNearGrid, siddon.cu:342-362
    double ex = (double)g.nx * g.dx, ey = (double)g.ny * g.dy, ez = (double)g.nz * g.dz;
    double r = sqrt(ex * ex + ey * ey + ez * ez);
    double dd[3] = {dst[0] - src[0], dst[1] - src[1], dst[2] - src[2]};
    double len = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
    if (len >= 1e-6)
        for (int k = 0; k < 3; ++k) dd[k] /= len;
    double t0 = (g.cx - src[0]) * dd[0] + (g.cy - src[1]) * dd[1] + (g.cz - src[2]) * dd[2];
    double t1 = (dst[0] - g.cx) * dd[0] + (dst[1] - g.cy) * dd[1] + (dst[2] - g.cz) * dd[2];
    if (t0 > r)
        for (int k = 0; k < 3; ++k) src[k] += (t0 - r) * dd[k];
    if (t1 > r)
        for (int k = 0; k < 3; ++k) dst[k] -= (t1 - r) * dd[k];
}

// InitializeSiddon, siddon.cu:104-173 (alphas scaled by the ray length).
__device__ Ray init_ray(const double src[3], const double dst[3], const Grid& g) {
    Ray R;
    R.hit = false;
    double dist = sqrt((src[0] - dst[0]) * (src[0] - dst[0]) + (src[1] - dst[1]) * (src[1] - dst[1]) +
                       (src[2] - dst[2]) * (src[2] - dst[2]));
    double cen[3] = {(double)g.cx, (double)g.cy, (double)g.cz};
    double sp[3] = {(double)g.dx, (double)g.dy, (double)g.dz};
    int n[3] = {g.nx, g.ny, g.nz};
    double s[3], dd[3], a0[3] = {1, 1, 1}, a1[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) {
        s[k] = (src[k] - cen[k]) / sp[k] + 0.5 * n[k];
        double e = (dst[k] - cen[k]) / sp[k] + 0.5 * n[k];
        dd[k] = e - s[k];
        if (fabs(dd[k]) > kEps) {
            a0[k] = (0 - s[k]) / dd[k];
            a1[k] = (n[k] - s[k]) / dd[k];
        } else if (s[k] < 0 || s[k] > n[k]) {
            return R;
        }
    }
    double amin = 0, amax = 1;
    for (int k = 0; k < 3; ++k) {
        amin = fmax(amin, fmin(a0[k], a1[k]));
        amax = fmin(amax, fmax(a0[k], a1[k]));
    }
    if (amax <= amin) return R;
    for (int k = 0; k < 3; ++k) {
        double p0 = s[k] + amin * dd[k];
        int v = (int)p0;
        if (fabs(dd[k]) > kEps) v = v < 0 ? 0 : (v >= n[k] ? n[k] - 1 : v);
        if (v < 0 || v >= n[k]) return R;
        R.ng[k] = v;
        double p1 = dd[k] > kEps ? (double)(v + 1) : (double)v;
        if (fabs(dd[k]) > kEps) {
            R.alpha[k] = (p1 - s[k]) / dd[k] * dist;
            R.dalpha[k] = dist / fabs(dd[k]);
        } else {
            R.alpha[k] = 2.0 * dist;
            R.dalpha[k] = 0;
        }
        R.step[k] = dd[k] > 0 ? 1 : -1;
    }
    R.aprev = amin * dist;
    R.hit = true;
    return R;
}

// The walk of SiddonRayTracing (siddon.cu:187-252): pick the nearest
// crossing (ties go to the later axis), emit the segment in the current voxel,
// step, stop when the index leaves the grid.  The crossing parameters are
// exact in FP64 (an axis' k-th crossing is its first one plus k steps); the
// walk itself runs in FP32 on their offsets from an anchor, the previous
// crossing, re-anchored every kAnchorSteps crossings so that the offsets stay
// within a few voxels (a segment's FP32 rounding is then ~1e-7 of that).  The
// axis is chosen by selects, not branches, so the rays of a warp step
// together, and the FP32 arithmetic keeps the walk off the FP64 pipe.
// IdxT: int when the volume has fewer than 2^31 voxels, else long long.
constexpr int kAnchorSteps = 16;

// One span of the walk: per axis k, crossing m (0-based) lies at
// a0[k] + m da[k]; taken[k] crossings are behind the start, rem[k] more stay
// inside the span (the next one after those leaves it); idx is the start
// voxel and mv[k] the index step of a crossing; ta is the start parameter.
template <typename IdxT, typename F>
__device__ __forceinline__ void walk_span(const double a0[3], const double da[3], const int taken[3], int r0, int r1,
                                          int r2, IdxT idx, const IdxT mv[3], double ta, F&& emit) {
    const int q0 = r0 + taken[0], q1 = r1 + taken[1], q2 = r2 + taken[2];  // crossings taken = q - r
    const float d0 = (float)da[0], d1 = (float)da[1], d2 = (float)da[2];
    for (;;) {
        // offsets of the next crossings from the anchor (never behind it)
        float l0 = fmaxf((float)(fma((double)(q0 - r0), da[0], a0[0]) - ta), 0.f);
        float l1 = fmaxf((float)(fma((double)(q1 - r1), da[1], a0[1]) - ta), 0.f);
        float l2 = fmaxf((float)(fma((double)(q2 - r2), da[2], a0[2]) - ta), 0.f);
        float lp = 0.f;
#pragma unroll 4
        for (int k = 0; k < kAnchorSteps; ++k) {
            const bool bx = l0 < l1 && l0 < l2;
            const bool by = !bx && l1 < l2;
            const bool bz = !bx && !by;
            const float m = bx ? l0 : (by ? l1 : l2);
            emit(idx, m - lp);
            lp = m;
            l0 = bx ? l0 + d0 : l0;
            l1 = by ? l1 + d1 : l1;
            l2 = bz ? l2 + d2 : l2;
            r0 -= bx;
            r1 -= by;
            r2 -= bz;
            idx += bx ? mv[0] : (by ? mv[1] : mv[2]);
            if ((r0 | r1 | r2) < 0) return;
        }
        ta += (double)lp;
    }
}

// The whole walk of a ray over a volume with index strides (sx, sy, sz).
template <typename IdxT, typename F>
__device__ __forceinline__ void walk_strided(const Ray& R, const Grid& g, IdxT sx, IdxT sy, IdxT sz, F&& emit) {
    // crossings left on each axis before its index leaves the grid
    const int r0 = R.step[0] > 0 ? g.nx - 1 - R.ng[0] : R.ng[0];
    const int r1 = R.step[1] > 0 ? g.ny - 1 - R.ng[1] : R.ng[1];
    const int r2 = R.step[2] > 0 ? g.nz - 1 - R.ng[2] : R.ng[2];
    const IdxT mv[3] = {(IdxT)R.step[0] * sx, (IdxT)R.step[1] * sy, (IdxT)R.step[2] * sz};
    const IdxT idx = (IdxT)R.ng[0] * sx + (IdxT)R.ng[1] * sy + (IdxT)R.ng[2] * sz;
    const int taken[3] = {0, 0, 0};
    walk_span<IdxT>(R.alpha, R.dalpha, taken, r0, r1, r2, idx, mv, R.aprev, emit);
}

// The walk over the volume's own [z][y][x] layout.
template <typename IdxT, typename F>
__device__ __forceinline__ void walk(const Ray& R, const Grid& g, F&& emit) {
    walk_strided<IdxT>(R, g, (IdxT)1, (IdxT)g.nx, (IdxT)g.nx * g.ny, emit);
}

// Five CTAs per SM (48 registers): the walk is latency-bound on its
// dependent loads, and the extra warps hide ~1% more of it.
template <typename Tin, typename Tout, typename IdxT>
__global__ void __launch_bounds__(256, 5) siddon_fp_kernel(Tout* __restrict__ prj, const Tin* __restrict__ img,
                                                        const float* __restrict__ dc, const float* __restrict__ du_,
                                                        const float* __restrict__ dv_, const float* __restrict__ sr,
                                                        int nview, Grid g, Det d, int accumulate) {
    int iu = blockIdx.x * 32 + (threadIdx.x & 31);
    int iv = blockIdx.y * 8 + (threadIdx.x >> 5);
    int view = blockIdx.z % nview, b = blockIdx.z / nview;
    if (iu >= d.nu || iv >= d.nv) return;
    double src[3], dst[3];
    ray_ends(src, dst, view, iu, iv, dc, du_, dv_, sr, g, d);
    Ray R = init_ray(src, dst, g);
    float acc = 0.f;
    if (R.hit) {
        const Tin* vol = img + (size_t)b * g.nx * g.ny * g.nz;
        // each sample is added one step later, so its load overlaps the next
        // step's arithmetic; the summation order is unchanged
        float pv = 0.f, pl = 0.f;
        walk<IdxT>(R, g, [&](IdxT idx, float len) {
            const float v = ldf(vol + idx);
            acc = fmaf(pv, pl, acc);
            pv = v;
            pl = len;
        });
        acc = fmaf(pv, pl, acc);
    }
    Tout* o = prj + (((size_t)b * nview + view) * d.nv + iv) * d.nu + iu;
    stf(o, (accumulate ? rdf(o) : 0.f) + acc);
}

// Transpose: scatter prj * length into the volume (FP32 atomics, as the
// reference's SiddonRayTracingTransposeAtomicAdd, siddon.cu:332).  The lanes
// of a warp are neighbouring detector cells, so at a given step they sit on
// voxels next to each other across the rays, along the detector's u
// direction.  When u runs mainly along y, those voxels are a row apart in the
// [z][y][x] volume and every lane's reduction is a separate L2 sector; such
// views scatter into imgT, laid out [z][x][y] (when given), where they are
// adjacent and share sectors, and imgT is added back transposed at the end.
template <typename Tin, typename IdxT>
__global__ void __launch_bounds__(256) siddon_bp_kernel(float* __restrict__ img, float* __restrict__ imgT,
                                                        const Tin* __restrict__ prj, const float* __restrict__ dc,
                                                        const float* __restrict__ du_, const float* __restrict__ dv_,
                                                        const float* __restrict__ sr, int nview, Grid g, Det d) {
    int iu = blockIdx.x * 32 + (threadIdx.x & 31);
    int iv = blockIdx.y * 8 + (threadIdx.x >> 5);
    int view = blockIdx.z % nview, b = blockIdx.z / nview;
    if (iu >= d.nu || iv >= d.nv) return;
    float p = ldf(prj + (((size_t)b * nview + view) * d.nv + iv) * d.nu + iu);
    if (p == 0.f) return;
    double src[3], dst[3];
    ray_ends(src, dst, view, iu, iv, dc, du_, dv_, sr, g, d);
    Ray R = init_ray(src, dst, g);
    if (!R.hit) return;
    const bool across_y = imgT && fabsf(du_[view * 3 + 1]) > fabsf(du_[view * 3]);
    float* vol = (across_y ? imgT : img) + (size_t)b * g.nx * g.ny * g.nz;
    if (across_y)
        walk_strided<IdxT>(R, g, (IdxT)g.ny, (IdxT)1, (IdxT)g.nx * g.ny,
                           [&](IdxT idx, float len) { atomicAdd(vol + idx, p * len); });
    else
        walk<IdxT>(R, g, [&](IdxT idx, float len) { atomicAdd(vol + idx, p * len); });
}

// img[b][z][y][x] += imgT[b][z][x][y], through 32x32 shared tiles.
__global__ void __launch_bounds__(256) add_transposed_kernel(float* __restrict__ img, const float* __restrict__ imgT,
                                                             int nx, int ny) {
    __shared__ float t[32][33];
    const size_t plane = (size_t)blockIdx.z * nx * ny;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += 8) {  // read rows of imgT: x fixed, y contiguous
        const int x = x0 + k, y = y0 + threadIdx.x;
        if (x < nx && y < ny) t[k][threadIdx.x] = imgT[plane + (size_t)x * ny + y];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int y = y0 + k, x = x0 + threadIdx.x;
        if (x < nx && y < ny) img[plane + (size_t)y * nx + x] += t[threadIdx.x][k];
    }
}

__global__ void __launch_bounds__(256) siddon_count_kernel(unsigned long long* __restrict__ count,
                                                           const float* __restrict__ dc, const float* __restrict__ du_,
                                                           const float* __restrict__ dv_,
                                                           const float* __restrict__ sr, int nview, Grid g, Det d) {
    int iu = blockIdx.x * 32 + (threadIdx.x & 31);
    int iv = blockIdx.y * 8 + (threadIdx.x >> 5);
    int view = blockIdx.z;
    unsigned long long c = 0;
    if (iu < d.nu && iv < d.nv) {
        double src[3], dst[3];
        ray_ends(src, dst, view, iu, iv, dc, du_, dv_, sr, g, d);
        Ray R = init_ray(src, dst, g);
        if (R.hit) walk<long long>(R, g, [&](long long, float) { ++c; });
    }
    __shared__ unsigned long long blk;
    if (threadIdx.x == 0) blk = 0;
    __syncthreads();
    if (c) atomicAdd(&blk, c);
    __syncthreads();
    if (threadIdx.x == 0 && blk) atomicAdd(count, blk);
}

// Fan-beam rays (SiddonFanProjectionKernel, siddonFan.cu:12-44): source on
// the circle of radius dso, detector cell on the arc of radius dsd at angle
// a = (-(iu - (nu-1)/2) - off_u) da, both at height z = (iv - (nv-1)/2 + off_v)
// dv, rotated by the view angle (trigonometry in FP64); the end points are not
// moved towards the grid, as in the reference's fan kernels.
__device__ void fan_ray_ends(double src[3], double dst[3], float deg, int iu, int iv, const Det& d, double dsd,
                             double dso) {
    double s, c, sa, ca;
    sincos((double)deg, &s, &c);
    const double a = (-((double)iu - (d.nu - 1) / 2.0) - d.off_u) * d.du;
    sincos(a, &sa, &ca);
    const double z = ((double)iv - (d.nv - 1) / 2.0 + d.off_v) * d.dv;
    const double rx = dsd * sa, ry = -dso + dsd * ca;
    src[0] = dso * s;
    src[1] = -dso * c;
    src[2] = z;
    dst[0] = rx * c - ry * s;
    dst[1] = rx * s + ry * c;
    dst[2] = z;
}

template <typename IdxT>
__global__ void __launch_bounds__(256) siddon_fan_fp_kernel(float* __restrict__ prj, const float* __restrict__ img,
                                                            const float* __restrict__ deg, int nview, Grid g, Det d,
                                                            double dsd, double dso, int accumulate) {
    int iu = blockIdx.x * 32 + (threadIdx.x & 31);
    int iv = blockIdx.y * 8 + (threadIdx.x >> 5);
    int view = blockIdx.z % nview, b = blockIdx.z / nview;
    if (iu >= d.nu || iv >= d.nv) return;
    double src[3], dst[3];
    fan_ray_ends(src, dst, deg[view], iu, iv, d, dsd, dso);
    Ray R = init_ray(src, dst, g);
    float acc = 0.f;
    if (R.hit) {
        const float* vol = img + (size_t)b * g.nx * g.ny * g.nz;
        float pv = 0.f, pl = 0.f;
        walk<IdxT>(R, g, [&](IdxT idx, float len) {
            const float v = __ldg(vol + idx);
            acc = fmaf(pv, pl, acc);
            pv = v;
            pl = len;
        });
        acc = fmaf(pv, pl, acc);
    }
    float* o = prj + (((size_t)b * nview + view) * d.nv + iv) * d.nu + iu;
    *o = (accumulate ? *o : 0.f) + acc;
}

// As siddon_bp_kernel: views whose detector tangent runs mainly along y
// scatter into the [z][x][y] copy imgT (when given).
template <typename IdxT>
__global__ void __launch_bounds__(256) siddon_fan_bp_kernel(float* __restrict__ img, float* __restrict__ imgT,
                                                            const float* __restrict__ prj,
                                                            const float* __restrict__ deg, int nview, Grid g, Det d,
                                                            double dsd, double dso) {
    int iu = blockIdx.x * 32 + (threadIdx.x & 31);
    int iv = blockIdx.y * 8 + (threadIdx.x >> 5);
    int view = blockIdx.z % nview, b = blockIdx.z / nview;
    if (iu >= d.nu || iv >= d.nv) return;
    float p = __ldg(prj + (((size_t)b * nview + view) * d.nv + iv) * d.nu + iu);
    if (p == 0.f) return;
    double src[3], dst[3];
    fan_ray_ends(src, dst, deg[view], iu, iv, d, dsd, dso);
    Ray R = init_ray(src, dst, g);
    if (!R.hit) return;
    const float th = deg[view];
    const bool across_y = imgT && fabsf(sinf(th)) > fabsf(cosf(th));
    float* vol = (across_y ? imgT : img) + (size_t)b * g.nx * g.ny * g.nz;
    if (across_y)
        walk_strided<IdxT>(R, g, (IdxT)g.ny, (IdxT)1, (IdxT)g.nx * g.ny,
                           [&](IdxT idx, float len) { atomicAdd(vol + idx, p * len); });
    else
        walk<IdxT>(R, g, [&](IdxT idx, float len) { atomicAdd(vol + idx, p * len); });
}

dim3 ray_grid(const ctp_geometry& g, size_t nz_mult) {
    return dim3((unsigned)((g.nu + 31) / 32), (unsigned)((g.nv + 7) / 8), (unsigned)(g.nview * nz_mult));
}

// 32-bit voxel indices when one volume has fewer than 2^31 voxels.
bool small_volume(const ctp_geometry& g) { return (unsigned long long)g.nx * g.ny * g.nz < (1ull << 31); }

template <typename IdxT>
int launch_siddon_fp(void* prj, const void* img, const float* dc, const float* du_, const float* dv_, const float* sr,
                     const ctp_geometry& g, unsigned flags, cudaStream_t s) {
    int acc = (flags & CTP_FLAG_ZERO_OUT) ? 0 : 1;
    dim3 grid = ray_grid(g, g.nbatch);
    Grid gr = make_grid(g);
    Det dt = make_det(g);
    int nv = (int)g.nview;
    if (flags & CTP_FLAG_IN_BF16) {
        if (flags & CTP_FLAG_OUT_BF16)
            siddon_fp_kernel<__nv_bfloat16, __nv_bfloat16, IdxT><<<grid, 256, 0, s>>>(
                (__nv_bfloat16*)prj, (const __nv_bfloat16*)img, dc, du_, dv_, sr, nv, gr, dt, acc);
        else
            siddon_fp_kernel<__nv_bfloat16, float, IdxT><<<grid, 256, 0, s>>>(
                (float*)prj, (const __nv_bfloat16*)img, dc, du_, dv_, sr, nv, gr, dt, acc);
    } else if (flags & CTP_FLAG_IN_FP16) {
        if (flags & CTP_FLAG_OUT_FP16)
            siddon_fp_kernel<__half, __half, IdxT><<<grid, 256, 0, s>>>((__half*)prj, (const __half*)img, dc, du_, dv_,
                                                                        sr, nv, gr, dt, acc);
        else
            siddon_fp_kernel<__half, float, IdxT><<<grid, 256, 0, s>>>((float*)prj, (const __half*)img, dc, du_, dv_,
                                                                       sr, nv, gr, dt, acc);
    } else {
        if (flags & (CTP_FLAG_OUT_BF16 | CTP_FLAG_OUT_FP16))
            return set_error(CTP_ERR_UNSUPPORTED, "siddon_fp: FP32 input with 16-bit output is not supported");
        siddon_fp_kernel<float, float, IdxT><<<grid, 256, 0, s>>>((float*)prj, (const float*)img, dc, du_, dv_, sr,
                                                                  nv, gr, dt, acc);
    }
    return check_launch("siddon_fp_kernel");
}

template <typename IdxT>
int launch_siddon_bp(void* img, const void* prj, const float* dc, const float* du_, const float* dv_,
                     const float* sr, const ctp_geometry& g, unsigned flags, cudaStream_t s) {
    dim3 grid = ray_grid(g, g.nbatch);
    // the transposed scatter target (zeroed), when the scratch can be had
    const size_t vox = g.nbatch * g.nz * g.ny * g.nx;
    Scratch scr;
    float* imgT = nullptr;
    if (!scr.acquire(nullptr, 0, vox * sizeof(float), s)) {
        imgT = reinterpret_cast<float*>(scr.base());
        cudaError_t e = cudaMemsetAsync(imgT, 0, vox * sizeof(float), s);
        if (e != cudaSuccess) return set_error((int)e, "siddon_bp memset: %s", cudaGetErrorString(e));
    } else {
        cudaGetLastError();  // fall back to the plain layout
    }
    if (flags & CTP_FLAG_IN_BF16)
        siddon_bp_kernel<__nv_bfloat16, IdxT><<<grid, 256, 0, s>>>((float*)img, imgT, (const __nv_bfloat16*)prj, dc,
                                                                   du_, dv_, sr, (int)g.nview, make_grid(g),
                                                                   make_det(g));
    else if (flags & CTP_FLAG_IN_FP16)
        siddon_bp_kernel<__half, IdxT><<<grid, 256, 0, s>>>((float*)img, imgT, (const __half*)prj, dc, du_, dv_, sr,
                                                            (int)g.nview, make_grid(g), make_det(g));
    else
        siddon_bp_kernel<float, IdxT><<<grid, 256, 0, s>>>((float*)img, imgT, (const float*)prj, dc, du_, dv_, sr,
                                                           (int)g.nview, make_grid(g), make_det(g));
    int rc = check_launch("siddon_bp_kernel");
    if (rc || !imgT) return rc;
    add_transposed_kernel<<<dim3((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 31) / 32),
                                 (unsigned)(g.nbatch * g.nz)),
                            dim3(32, 8), 0, s>>>((float*)img, imgT, (int)g.nx, (int)g.ny);
    return check_launch("add_transposed_kernel");
}

}  // namespace

int siddon_fp(void* prj, const void* img, const float* dc, const float* du_, const float* dv_, const float* sr,
              const ctp_geometry& g, unsigned flags, cudaStream_t s) {
    return small_volume(g) ? launch_siddon_fp<int>(prj, img, dc, du_, dv_, sr, g, flags, s)
                           : launch_siddon_fp<long long>(prj, img, dc, du_, dv_, sr, g, flags, s);
}

int siddon_bp(void* img, const void* prj, const float* dc, const float* du_, const float* dv_, const float* sr,
              const ctp_geometry& g, unsigned flags, cudaStream_t s) {
    if (flags & (CTP_FLAG_OUT_BF16 | CTP_FLAG_OUT_FP16))
        return set_error(CTP_ERR_UNSUPPORTED, "siddon_bp accumulates in FP32: 16-bit output is not supported");
    if (flags & CTP_FLAG_ZERO_OUT) {
        cudaError_t e = cudaMemsetAsync(img, 0, g.nbatch * g.nz * g.ny * g.nx * sizeof(float), s);
        if (e != cudaSuccess) return set_error((int)e, "siddon_bp memset: %s", cudaGetErrorString(e));
    }
    return small_volume(g) ? launch_siddon_bp<int>(img, prj, dc, du_, dv_, sr, g, flags, s)
                           : launch_siddon_bp<long long>(img, prj, dc, du_, dv_, sr, g, flags, s);
}

int siddon_nnz(unsigned long long* nnz_host, const float* dc, const float* du_, const float* dv_, const float* sr,
               const ctp_geometry& g, cudaStream_t s) {
    if (!nnz_host) return set_error(CTP_ERR_INVALID_ARGUMENT, "nnz output pointer is null");
    Scratch scr;
    int rc = scr.acquire(nullptr, 0, 256, s);
    if (rc) return rc;
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(scr.base());
    cudaMemsetAsync(cnt, 0, sizeof(*cnt), s);
    siddon_count_kernel<<<ray_grid(g, 1), 256, 0, s>>>(cnt, dc, du_, dv_, sr, (int)g.nview, make_grid(g),
                                                      make_det(g));
    if ((rc = check_launch("siddon_count_kernel"))) return rc;
    cudaError_t e = cudaMemcpyAsync(nnz_host, cnt, sizeof(*cnt), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_error((int)e, "siddon_nnz: %s", cudaGetErrorString(e));
    return CTP_OK;
}

// Fan-beam Siddon pair (siddonFan.cu:12-274); g.du is the angular cell size.
int siddon_fan_fp(float* prj, const float* img, const float* deg, const ctp_geometry& g, unsigned flags,
                  cudaStream_t s) {
    const int acc = (flags & CTP_FLAG_ZERO_OUT) ? 0 : 1;
    if (small_volume(g))
        siddon_fan_fp_kernel<int><<<ray_grid(g, g.nbatch), 256, 0, s>>>(prj, img, deg, (int)g.nview, make_grid(g),
                                                                       make_det(g), (double)g.dsd, (double)g.dso, acc);
    else
        siddon_fan_fp_kernel<long long><<<ray_grid(g, g.nbatch), 256, 0, s>>>(
            prj, img, deg, (int)g.nview, make_grid(g), make_det(g), (double)g.dsd, (double)g.dso, acc);
    return check_launch("siddon_fan_fp_kernel");
}

int siddon_fan_bp(float* img, const float* prj, const float* deg, const ctp_geometry& g, unsigned flags,
                  cudaStream_t s) {
    if (flags & CTP_FLAG_ZERO_OUT) {
        cudaError_t e = cudaMemsetAsync(img, 0, g.nbatch * g.nz * g.ny * g.nx * sizeof(float), s);
        if (e != cudaSuccess) return set_error((int)e, "siddon_fan_bp memset: %s", cudaGetErrorString(e));
    }
    const size_t vox = g.nbatch * g.nz * g.ny * g.nx;
    Scratch scr;
    float* imgT = nullptr;
    if (!scr.acquire(nullptr, 0, vox * sizeof(float), s)) {
        imgT = reinterpret_cast<float*>(scr.base());
        cudaError_t e = cudaMemsetAsync(imgT, 0, vox * sizeof(float), s);
        if (e != cudaSuccess) return set_error((int)e, "siddon_fan_bp memset: %s", cudaGetErrorString(e));
    } else {
        cudaGetLastError();  // fall back to the plain layout
    }
    if (small_volume(g))
        siddon_fan_bp_kernel<int><<<ray_grid(g, g.nbatch), 256, 0, s>>>(img, imgT, prj, deg, (int)g.nview,
                                                                       make_grid(g), make_det(g), (double)g.dsd,
                                                                       (double)g.dso);
    else
        siddon_fan_bp_kernel<long long><<<ray_grid(g, g.nbatch), 256, 0, s>>>(
            img, imgT, prj, deg, (int)g.nview, make_grid(g), make_det(g), (double)g.dsd, (double)g.dso);
    int rc = check_launch("siddon_fan_bp_kernel");
    if (rc || !imgT) return rc;
    add_transposed_kernel<<<dim3((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 31) / 32),
                                 (unsigned)(g.nbatch * g.nz)),
                            dim3(32, 8), 0, s>>>(img, imgT, (int)g.nx, (int)g.ny);
    return check_launch("add_transposed_kernel");
}

}  // namespace ctp
