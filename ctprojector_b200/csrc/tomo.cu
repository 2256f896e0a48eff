// tomo.cu -- distance-driven tomosynthesis projector pair (z main axis,
// detector u = (1,0,0), v = (0,1,0)), sm_100a.
//
// Reference: DDFPConeBoxIntKernelXY distanceDriven3DBoxInt.cu:28-117,
// DDBPConeBoxIntCartKernelXY :170-216, PreweightBPCartKernelXY
// distanceDriven3DUtils.cu:10-31, ProjectConeToDetCart :45-56, and the 2D box
// integral IntegralBoxXY cudaMath.cu:336-404.
//
// Forward: one thread per ray; per z plane the normalised integral of the
// plane over the footprint rectangle of the cell.  Back projection
// (reference-parity form): one thread per voxel; per view the normalised
// integral of the length-weighted projection over the voxel's projected
// rectangle.  The per-cell ray-length weight is applied once in a pre-pass
// into the workspace.  Unlike the reference, every batch item reads its own
// weighted projections (the reference reads item 0's for all items,
// distanceDriven3DBoxInt.cu:257-259).
#include <cuda_runtime.h>
#include <math.h>

#include "ctp_common.cuh"

namespace ctp {

namespace {

// Exact integral of an (ny, nx) plane over the clamped rectangle.
__device__ float box2d(const float* __restrict__ p, float x1, float y1, float x2, float y2, int nx, int ny) {
    x1 = clampf(x1, 0.f, (float)nx);
    y1 = clampf(y1, 0.f, (float)ny);
    x2 = clampf(x2, 0.f, (float)nx);
    y2 = clampf(y2, 0.f, (float)ny);
    if (x2 <= x1 || y2 <= y1) return 0.f;
    int ix1 = min((int)x1, nx - 1), iy1 = min((int)y1, ny - 1);
    int ix2 = min((int)x2, nx - 1), iy2 = min((int)y2, ny - 1);
    float v = 0.f;
    for (int iy = iy1; iy <= iy2; ++iy) {
        float wy = 1.f;
        if (iy == iy1) wy -= (y1 - (float)iy1);
        if (iy == iy2) wy -= ((float)(iy2 + 1) - y2);
        const float* row = p + (size_t)iy * nx;
        float r = 0.f;
        for (int ix = ix1; ix <= ix2; ++ix) r += __ldg(row + ix);
        r -= __ldg(row + ix1) * (x1 - (float)ix1);
        r -= __ldg(row + ix2) * ((float)(ix2 + 1) - x2);
        v += r * wy;
    }
    return v;
}

// The same integral when the rectangle spans at most K pixels along each axis
// (x2 - x1 <= K - 1 and y2 - y1 <= K - 1, K = 2 or 3): the pixel weights are
// the overlaps of the clamped rectangle with K consecutive columns and rows,
// straight-line code with K*K loads (indices clamped, weights 0 past the
// edge) instead of the general loops.
template <int K>
__device__ __forceinline__ float box2d_small(const float* __restrict__ p, float x1, float y1, float x2, float y2,
                                             int nx, int ny) {
    x1 = clampf(x1, 0.f, (float)nx);
    y1 = clampf(y1, 0.f, (float)ny);
    x2 = clampf(x2, 0.f, (float)nx);
    y2 = clampf(y2, 0.f, (float)ny);
    if (x2 <= x1 || y2 <= y1) return 0.f;
    const int ix = min((int)x1, nx - 1), iy = min((int)y1, ny - 1);
    float wx[K], wy[K];
    int cx[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        // overlap of [x1, x2] with column ix + k (and of [y1, y2] with row iy + k)
        wx[k] = fmaxf(fminf(x2, (float)(ix + k + 1)) - fmaxf(x1, (float)(ix + k)), 0.f);
        wy[k] = fmaxf(fminf(y2, (float)(iy + k + 1)) - fmaxf(y1, (float)(iy + k)), 0.f);
        cx[k] = min(ix + k, nx - 1);
    }
    float v = 0.f;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const float* row = p + (size_t)min(iy + j, ny - 1) * nx;
        float r = 0.f;
#pragma unroll
        for (int k = 0; k < K; ++k) r = fmaf(wx[k], __ldg(row + cx[k]), r);
        v = fmaf(wy[j], r, v);
    }
    return v;
}

__global__ void __launch_bounds__(256) tomo_fp_kernel(float* __restrict__ prj, const float* __restrict__ img,
                                                      const float* __restrict__ dc, const float* __restrict__ sr,
                                                      int nview, Grid g, Det d, int accumulate) {
    int iu = blockIdx.x * 32 + (threadIdx.x & 31);
    int iv = blockIdx.y * 8 + (threadIdx.x >> 5);
    int view = blockIdx.z % nview, b = blockIdx.z / nview;
    if (iu >= d.nu || iv >= d.nv) return;
    double u = ((double)iu - d.off_u - (d.nu - 1) / 2.0) * d.du;
    double v = ((double)iv - d.off_v - (d.nv - 1) / 2.0) * d.dv;
    double C[3] = {dc[view * 3], dc[view * 3 + 1], dc[view * 3 + 2]};
    double S[3] = {sr[view * 3], sr[view * 3 + 1], sr[view * 3 + 2]};
    // image coordinates of the source and of the four cell-edge mid points
    auto ix_ = [&](double x) { return (x - g.cx) / g.dx + 0.5 * g.nx; };
    auto iy_ = [&](double y) { return (y - g.cy) / g.dy + 0.5 * g.ny; };
    auto iz_ = [&](double z) { return (z - g.cz) / g.dz + 0.5 * g.nz; };
    double sx = ix_(S[0]), sy = iy_(S[1]), sz = iz_(S[2]);
    double cz = iz_(C[2]);
    double xa = ix_(C[0] + u - d.du / 2.0), xb = ix_(C[0] + u + d.du / 2.0);
    double ya = iy_(C[1] + v - d.dv / 2.0), yb = iy_(C[1] + v + d.dv / 2.0);
    if (xa > xb) { double t = xa; xa = xb; xb = t; }
    if (ya > yb) { double t = ya; ya = yb; yb = t; }
    double rx1 = (xa - sx) / (cz - sz), rx2 = (xb - sx) / (cz - sz);
    double ry1 = (ya - sy) / (cz - sz), ry2 = (yb - sy) / (cz - sz);
    const float* vol = img + (size_t)b * g.nx * g.ny * g.nz;
    float val = 0.f;
    // footprint widths grow linearly with the distance from the source: the
    // widest is on the end plane farther from it
    const double dmax = fmax(fabs(0.0 - sz), fabs((double)(g.nz - 1) - sz));
    if (fabs(rx2 - rx1) * dmax <= 1.0 && fabs(ry2 - ry1) * dmax <= 1.0) {
        // at most 2 x 2 pixels per plane; edges in FP32 from per-ray FP32
        // coefficients (the width and the integral see the same rounded edges)
        const float fsx = (float)sx, fsy = (float)sy, fsz = (float)sz;
        const float frx1 = (float)rx1, frx2 = (float)rx2, fry1 = (float)ry1, fry2 = (float)ry2;
        for (int iz = 0; iz < g.nz; ++iz) {
            const float dz = (float)iz - fsz;
            const float x1 = fmaf(frx1, dz, fsx), x2 = fmaf(frx2, dz, fsx);
            const float y1 = fmaf(fry1, dz, fsy), y2 = fmaf(fry2, dz, fsy);
            val += __fdividef(box2d_small<2>(vol + (size_t)iz * g.nx * g.ny, x1, y1, x2, y2, g.nx, g.ny),
                              (x2 - x1) * (y2 - y1));
        }
    } else {
        for (int iz = 0; iz < g.nz; ++iz) {
            double dz = iz - sz;
            float x1 = (float)(sx + rx1 * dz), x2 = (float)(sx + rx2 * dz);
            float y1 = (float)(sy + ry1 * dz), y2 = (float)(sy + ry2 * dz);
            val += box2d(vol + (size_t)iz * g.nx * g.ny, x1, y1, x2, y2, g.nx, g.ny) / ((x2 - x1) * (y2 - y1));
        }
    }
    double D[3] = {C[0] + u, C[1] + v, C[2]};
    double L = sqrt((S[2] - D[2]) * (S[2] - D[2]) + (S[1] - D[1]) * (S[1] - D[1]) + (S[0] - D[0]) * (S[0] - D[0]));
    val *= (float)(g.dz / fabs(S[2] - D[2]) * L);
    float* o = prj + (((size_t)b * nview + view) * d.nv + iv) * d.nu + iu;
    *o = (accumulate ? *o : 0.f) + val;
}

__global__ void tomo_preweight_kernel(float* __restrict__ out, const float* __restrict__ prj,
                                      const float* __restrict__ dc, const float* __restrict__ sr, int nview, Det d,
                                      float dz, size_t total) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= total) return;
    int iu = (int)(i % d.nu);
    int iv = (int)((i / d.nu) % d.nv);
    int view = (int)((i / ((size_t)d.nu * d.nv)) % nview);
    double u = ((double)iu - d.off_u - (d.nu - 1) / 2.0) * d.du;
    double v = ((double)iv - d.off_v - (d.nv - 1) / 2.0) * d.dv;
    double D[3] = {dc[view * 3] + u, dc[view * 3 + 1] + v, (double)dc[view * 3 + 2]};
    double S[3] = {sr[view * 3], sr[view * 3 + 1], sr[view * 3 + 2]};
    double L = sqrt((S[2] - D[2]) * (S[2] - D[2]) + (S[1] - D[1]) * (S[1] - D[1]) + (S[0] - D[0]) * (S[0] - D[0]));
    out[i] = prj[i] * (float)(dz / fabs(S[2] - D[2]) * L);
}

__global__ void __launch_bounds__(256) tomo_bp_kernel(float* __restrict__ img, const float* __restrict__ wprj,
                                                      const float* __restrict__ dc, const float* __restrict__ sr,
                                                      int nview, Grid g, Det d, int accumulate) {
    int ix = blockIdx.x * 32 + (threadIdx.x & 31);
    int iy = blockIdx.y * 8 + (threadIdx.x >> 5);
    int iz = blockIdx.z % g.nz, b = blockIdx.z / g.nz;
    if (ix >= g.nx || iy >= g.ny) return;
    float x = ((float)ix - (g.nx - 1) / 2.0f) * g.dx + g.cx;
    float y = ((float)iy - (g.ny - 1) / 2.0f) * g.dy + g.cy;
    float z = ((float)iz - (g.nz - 1) / 2.0f) * g.dz + g.cz;
    const float* pb = wprj + (size_t)b * nview * d.nv * d.nu;
    // fast divides and reciprocals of the cell sizes (a few ulp each)
    const float idu = 1.f / d.du, idv = 1.f / d.dv;
    float val = 0.f;
    for (int view = 0; view < nview; ++view) {
        float Sx = sr[view * 3], Sy = sr[view * 3 + 1], Sz = sr[view * 3 + 2];
        float Cx = dc[view * 3], Cy = dc[view * 3 + 1], Cz = dc[view * 3 + 2];
        float r = __fdividef(Cz - Sz, z - Sz);
        float u1 = (Sx - Cx + r * (x - g.dx / 2 - Sx)) * idu + d.off_u + (d.nu - 1) / 2.0f;
        float u2 = (Sx - Cx + r * (x + g.dx / 2 - Sx)) * idu + d.off_u + (d.nu - 1) / 2.0f;
        float v1 = (Sy - Cy + r * (y - g.dy / 2 - Sy)) * idv + d.off_v + (d.nv - 1) / 2.0f;
        float v2 = (Sy - Cy + r * (y + g.dy / 2 - Sy)) * idv + d.off_v + (d.nv - 1) / 2.0f;
        const float* pv = pb + (size_t)view * d.nv * d.nu;
        const float w = fabsf(u2 - u1), h = fabsf(v2 - v1);
        float box;
        if (w <= 1.f && h <= 1.f) box = box2d_small<2>(pv, u1, v1, u2, v2, d.nu, d.nv);
        else if (w <= 2.f && h <= 2.f) box = box2d_small<3>(pv, u1, v1, u2, v2, d.nu, d.nv);
        else box = box2d(pv, u1, v1, u2, v2, d.nu, d.nv);
        val += __fdividef(box, (u2 - u1) * (v2 - v1));
    }
    float* o = img + (((size_t)b * g.nz + iz) * g.ny + iy) * g.nx + ix;
    *o = (accumulate ? *o : 0.f) + val;
}

}  // namespace

int tomo_fp(float* prj, const float* img, const float* dc, const float* sr, const ctp_geometry& g, unsigned flags,
            cudaStream_t s) {
    dim3 grid((unsigned)((g.nu + 31) / 32), (unsigned)((g.nv + 7) / 8), (unsigned)(g.nview * g.nbatch));
    // the reference overwrites; CTP_FLAG_ZERO_OUT is the default here
    tomo_fp_kernel<<<grid, 256, 0, s>>>(prj, img, dc, sr, (int)g.nview, make_grid(g), make_det(g), 0);
    (void)flags;
    return check_launch("tomo_fp_kernel");
}

size_t tomo_bp_workspace(const ctp_geometry& g) { return align_up(g.nbatch * g.nview * g.nv * g.nu * sizeof(float)); }

int tomo_bp(float* img, const float* prj, const float* dc, const float* sr, const ctp_geometry& g, unsigned flags,
            void* workspace, size_t workspace_bytes, cudaStream_t s) {
    Scratch scr;
    int rc = scr.acquire(workspace, workspace_bytes, tomo_bp_workspace(g), s);
    if (rc) return rc;
    float* wprj = reinterpret_cast<float*>(scr.base());
    size_t total = g.nbatch * g.nview * g.nv * g.nu;
    tomo_preweight_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(wprj, prj, dc, sr, (int)g.nview,
                                                                         make_det(g), g.dz, total);
    if ((rc = check_launch("tomo_preweight_kernel"))) return rc;
    dim3 grid((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 7) / 8), (unsigned)(g.nz * g.nbatch));
    (void)flags;
    tomo_bp_kernel<<<grid, 256, 0, s>>>(img, wprj, dc, sr, (int)g.nview, make_grid(g), make_det(g), 0);
    return check_launch("tomo_bp_kernel");
}

}  // namespace ctp
