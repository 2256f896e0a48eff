// dd2d.cu -- distance-driven fan-beam (equiangular) and parallel-beam
// projector pair for sm_100a.
//
// Operator (reference: distanceDriven2DBoxInt.cu:21-235, the box-integral
// DDFPTracing with the 0.12 blend band; distanceDriven2DUtils.cu for the
// back-projection pre-weights and detector mappings):
//
//   prj[ray] = wx * Ly * sum_rows  int_{x1(row)}^{x2(row)} img_row / |x2-x1|
//            + (1-wx) * Lx * sum_cols int_{y1(col)}^{y2(col)} img_col / |y2-y1|
//
// with the two detector-cell edge rays intersected with every row (column)
// centre and z linearly interpolated between two slices.
//
// Design:
//  * dd_table_kernel evaluates, once per call and in FP64, the footprint edges
//    of every detector-cell edge ray of every view as lines x(row) = A + B*t in
//    image coordinates (t = row - anchor) and the ray-length factor L per
//    cell.  The forward projector
//    and its exact transpose read the same FP32 table entries, so both see
//    bit-identical footprints.
//  * Forward projection: one thread per ray, rows read with coalesced loads
//    (adjacent threads = adjacent cells).  Views traced along x read a
//    transposed copy of the image so that those walks are row reads too.
//  * Back projection is a gather (no atomics): a CTA owns a 16x16 pixel tile,
//    streams chunks of views and stages, per view, only the window of
//    detector cells that the tile projects onto in shared memory.  Two modes:
//      - reference parity: the normalised detector-space box integral of
//        DDBPFanKernel / DDBPParallelKernel (distanceDriven2DBoxInt.cu:319,409),
//      - exact adjoint: the transpose of the forward projector, with the
//        image-space overlaps taken from the same edge table.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <type_traits>

#include "ctp_common.cuh"

namespace ctp {

namespace {

constexpr int kTile = 16;       // back-projection pixel tile edge
constexpr int kBPViews = 32;    // views per staged chunk (parity)
constexpr int kAdjViews = 8;    // views per staged chunk (adjoint)
constexpr int kMaxWin = 192;    // largest staged detector window (cells)
constexpr int kFPThreads = 128;

struct DDTab {
    const float* eA[2];  // [nview][nu+1] edge position at the anchor row/col
    const float* eB[2];  // [nview][nu+1] edge slope per row/col
    const float* cL[2];  // [nview][nu] ray length factor dy/|cos| or dx/|sin|
    const float* wx;     // [nview] blend weight of the row (y main axis) sweep
    const float* sP[2];  // [nview] fan source: position across the lines
    const float* sS[2];  // [nview] fan source: line coordinate from the anchor line's centre
    int ym, xm;          // anchor row / column
};

struct DDTabW {
    float* eA[2];
    float* eB[2];
    float* cL[2];
    float* wx;
    float* sP[2];
    float* sS[2];
};

size_t table_floats(size_t nview, size_t nu) { return 2 * (2 * nview * (nu + 1) + nview * nu) + 5 * nview; }

// Table carve-out in a float buffer; the same layout for readers and writers.
void carve_table(float* base, size_t nview, size_t nu, DDTabW& w) {
    size_t ne = nview * (nu + 1), nc = nview * nu;
    float* p = base;
    for (int o = 0; o < 2; ++o) {
        w.eA[o] = p; p += ne;
        w.eB[o] = p; p += ne;
        w.cL[o] = p; p += nc;
    }
    w.wx = p; p += nview;
    for (int o = 0; o < 2; ++o) {
        w.sP[o] = p; p += nview;
        w.sS[o] = p; p += nview;
    }
}

DDTab as_read(const DDTabW& w, int ym, int xm) {
    DDTab t;
    for (int o = 0; o < 2; ++o) {
        t.eA[o] = w.eA[o]; t.eB[o] = w.eB[o];
        t.cL[o] = w.cL[o];
        t.sP[o] = w.sP[o]; t.sS[o] = w.sS[o];
    }
    t.wx = w.wx;
    t.ym = ym;
    t.xm = xm;
    return t;
}

// Two points of the edge ray of detector edge j in image coordinates.
// Fan: source (dso sin, -dso cos) and the arc point at angle e_j
// (distanceDriven2DBoxInt.cu:213-226).  Parallel: the two virtual points at
// +-(nx dx + ny dy) along the rotated axis (:143-163).  Edge j sits at
// e_j = (-(j - nu/2) - off_u) du, so cell k spans edges k and k+1.
__device__ void edge_ray(int geom, double th, int j, const Grid& g, const Det& d, double dsd, double dso,
                         double& sx, double& sy, double& ex, double& ey) {
    double s, c;
    sincos(th, &s, &c);
    double e = (-((double)j - 0.5 * d.nu) - (double)d.off_u) * (double)d.du;
    if (geom == 0) {
        sx = dso * s;
        sy = -dso * c;
        double lx = dsd * sin(e), ly = -dso + dsd * cos(e);
        ex = lx * c - ly * s;
        ey = lx * s + ly * c;
    } else {
        double r = (double)g.nx * g.dx + (double)g.ny * g.dy;
        sx = e * c + r * s;
        sy = e * s - r * c;
        ex = e * c - r * s;
        ey = e * s + r * c;
    }
    sx = (sx - g.cx) / g.dx + 0.5 * g.nx;
    sy = (sy - g.cy) / g.dy + 0.5 * g.ny;
    ex = (ex - g.cx) / g.dx + 0.5 * g.nx;
    ey = (ey - g.cy) / g.dy + 0.5 * g.ny;
}

// hard != 0: the branchless tracer's weights (distanceDriven2DBranchless.cu:
// 68-118): the main axis alone, chosen by |__cosf| > |__sinf| as there.
__global__ void dd_table_kernel(DDTabW t, const float* __restrict__ deg, int nview, Grid g, Det d, double dsd,
                                double dso, int geom, int ym, int xm, int hard) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    int view = blockIdx.y;
    if (j > d.nu || view >= nview) return;
    double th = (double)deg[view];
    double sx, sy, ex, ey;
    edge_ray(geom, th, j, g, d, dsd, dso, sx, sy, ex, ey);
    double by = (ex - sx) / (ey - sy), bx = (ey - sy) / (ex - sx);
    if (geom != 0) {
        // parallel rays: one slope per view, the same float for every edge
        // (the parallel forward projector relies on equal footprint widths)
        double s, c;
        sincos(th, &s, &c);
        by = -(s * g.dy) / (c * g.dx);
        bx = -(c * g.dx) / (s * g.dy);
    }
    double ay = sx + by * (ym + 0.5 - sy), ax = sy + bx * (xm + 0.5 - sx);
    size_t ie = (size_t)view * (d.nu + 1) + j;
    t.eA[0][ie] = (float)ay;
    t.eB[0][ie] = (float)by;
    t.eA[1][ie] = (float)ax;
    t.eB[1][ie] = (float)bx;
    if (j < d.nu) {
        size_t ic = (size_t)view * d.nu + j;
        double a = geom == 0 ? (-((double)j - 0.5 * (d.nu - 1)) - (double)d.off_u) * (double)d.du : 0.0;
        t.cL[0][ic] = (float)((double)g.dy / fabs(cos(th - a)));
        t.cL[1][ic] = (float)((double)g.dx / fabs(sin(th - a)));
    }
    if (j == 0) {
        double s, c;
        sincos(th, &s, &c);
        double r = (fabs(c) - fabs(s) + kDDMarginD) / (2 * kDDMarginD);
        t.wx[view] = hard ? (fabsf(__cosf(deg[view])) > fabsf(__sinf(deg[view])) ? 1.f : 0.f)
                          : (float)(r < 0 ? 0.0 : (r > 1 ? 1.0 : r));
        // fan source in line coordinates: edge j sits at sP + eB_j (t - sS) on
        // line t (counted from the anchor line)
        t.sP[0][view] = (float)sx;
        t.sS[0][view] = (float)(sy - ym - 0.5);
        t.sP[1][view] = (float)sy;
        t.sS[1][view] = (float)(sx - xm - 0.5);
    }
}

// The reference decides its hard axis switches (fan back projection,
// back-projection pre-weights) on |__cosf(deg)| > |__sinf(deg)|
// (distanceDriven2DBoxInt.cu:362, distanceDriven2DUtils.cu:22,54).  At views
// within rounding of 45 degrees the outcome depends on those fast intrinsics,
// so the same comparison is made here; the geometry itself uses accurate
// trigonometry.
__device__ __forceinline__ bool ref_y_main(float deg) { return fabsf(__cosf(deg)) > fabsf(__sinf(deg)); }

// [nslice][ny][nx] -> [nslice][nx][ny]
template <typename T>
__global__ void transpose_kernel(T* __restrict__ out, const T* __restrict__ in, int nx, int ny) {
    __shared__ T tile[32][33];
    size_t slice = blockIdx.z;
    const T* src = in + slice * (size_t)nx * ny;
    T* dst = out + slice * (size_t)nx * ny;
    int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        int x = x0 + threadIdx.x, y = y0 + k;
        if (x < nx && y < ny) tile[k][threadIdx.x] = src[(size_t)y * nx + x];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        int y = y0 + threadIdx.x, x = x0 + k;
        if (x < nx && y < ny) dst[(size_t)x * ny + y] = tile[threadIdx.x][k];
    }
}

// z interpolation of one detector row, in the reference's float arithmetic
// (distanceDriven2DBoxInt.cu:35-42, :214, :227).
__device__ __forceinline__ void row_z(int iv, const Grid& g, const Det& d, int& iz, int& iz1, float& wz) {
    float z = ((float)iv - (d.nv - 1) / 2.0f + d.off_v) * d.dv;
    z = (z - g.cz) / g.dz + g.nz / 2.f - 0.5f;
    z = clampf(z, 0.f, (float)g.nz);
    int a = (int)z;
    int b = a + 1;
    a = min(max(a, 0), g.nz - 1);
    b = min(max(b, 0), g.nz - 1);
    iz = a;
    iz1 = b;
    wz = z - (float)a;
}

// One sweep of one ray over the lines of a slice pair.  Lines are rows of the
// image (n = nx cells per line, nl = ny lines) or rows of the transposed image.
template <typename Tin, bool COUNT>
__device__ __forceinline__ float sweep(const Tin* __restrict__ s0, const Tin* __restrict__ s1, float wz, int n,
                                       int nl, int anchor, float Aa, float Ba, float Ab, float Bb,
                                       unsigned long long& cnt) {
    float sum = 0.f;
    for (int l = 0; l < nl; ++l) {
        float t = (float)(l - anchor);
        float xa = fmaf(Ba, t, Aa);
        float xb = fmaf(Bb, t, Ab);
        float lo = fminf(xa, xb), hi = fmaxf(xa, xb);
        if (COUNT) {
            float c1 = clampf(lo, 0.f, (float)n), c2 = clampf(hi, 0.f, (float)n);
            if (c2 > c1) cnt += (unsigned long long)(min((int)c2, n - 1) - min((int)c1, n - 1) + 1) * (wz != 0.f ? 2 : 1);
            continue;
        }
        float v = box_line(s0 + (size_t)l * n, 1, lo, hi, n);
        if (wz != 0.f) v = v * (1.f - wz) + box_line(s1 + (size_t)l * n, 1, lo, hi, n) * wz;
        // normalised by the width of the rounded footprint, as the reference
        // does (:63-66): the ratio is the mean of the line over the interval,
        // which edge rounding only shifts instead of rescaling
        sum += __fdividef(v, hi - lo);
    }
    return sum;
}

template <typename Tin, typename Tout, bool COUNT>
__global__ void __launch_bounds__(kFPThreads) dd2d_fp_kernel(Tout* __restrict__ prj, const Tin* __restrict__ img,
                                                             const Tin* __restrict__ imgT, DDTab tab, Grid g,
                                                             Det d, int nview, const float* __restrict__ deg,
                                                             int unweight_par, int accumulate,
                                                             unsigned long long* __restrict__ count) {
    int iu = blockIdx.x * blockDim.x + threadIdx.x;
    int view = blockIdx.y;
    int bz = blockIdx.z;
    unsigned long long cnt = 0;
    if (iu < d.nu) {
        int iv = bz % d.nv, b = bz / d.nv;
        int iz, iz1;
        float wz;
        row_z(iv, g, d, iz, iz1, wz);
        float wx = tab.wx[view];
        float acc = 0.f;
        size_t ie = (size_t)view * (d.nu + 1) + iu;
        size_t ic = (size_t)view * d.nu + iu;
        size_t plane = (size_t)g.nx * g.ny;
        if (wx > 0.f) {
            const Tin* s0 = img + ((size_t)b * g.nz + iz) * plane;
            const Tin* s1 = img + ((size_t)b * g.nz + iz1) * plane;
            float sum = sweep<Tin, COUNT>(s0, s1, wz, g.nx, g.ny, tab.ym, tab.eA[0][ie], tab.eB[0][ie],
                                          tab.eA[0][ie + 1], tab.eB[0][ie + 1], cnt);
            acc += sum * tab.cL[0][ic] * wx;
        }
        if (wx < 1.f) {
            const Tin* s0 = imgT + ((size_t)b * g.nz + iz) * plane;
            const Tin* s1 = imgT + ((size_t)b * g.nz + iz1) * plane;
            float sum = sweep<Tin, COUNT>(s0, s1, wz, g.ny, g.nx, tab.xm, tab.eA[1][ie], tab.eB[1][ie],
                                          tab.eA[1][ie + 1], tab.eB[1][ie + 1], cnt);
            acc += sum * tab.cL[1][ic] * (1.f - wx);
        }
        if (!COUNT) {
            if (unweight_par) {
                // FORCE_FBP on parallel FP: cancel the ray-length weight
                // (ReverseWeightBPParallelKernel, distanceDriven2DUtils.cu:68).
                float s, c;
                sincosf(deg[view], &s, &c);
                acc /= ref_y_main(deg[view]) ? g.dy / fabsf(c) : g.dx / fabsf(s);
            }
            Tout* o = prj + (((size_t)b * nview + view) * d.nv + iv) * d.nu + iu;
            if (accumulate) acc += rdf(o);
            stf(o, acc);
        }
    }
    if (COUNT) {
        __shared__ unsigned long long blk;
        if (threadIdx.x == 0) blk = 0;
        __syncthreads();
        if (cnt) atomicAdd(&blk, cnt);
        __syncthreads();
        if (threadIdx.x == 0 && blk) atomicAdd(count, blk);
    }
}


// Fan pre-weight of the copied sinogram for the normalised back projection
// (PreweightBPKernel, distanceDriven2DUtils.cu:8-33): hard switch on the view
// angle, weight from the ray angle.
template <typename Tin>
__global__ void fan_preweight_kernel(float* __restrict__ out, const Tin* __restrict__ prj,
                                     const float* __restrict__ deg, int nview, Det d, Grid g, size_t total) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= total) return;
    int iu = (int)(i % d.nu);
    int view = (int)((i / ((size_t)d.nu * d.nv)) % nview);
    float th = deg[view];
    float a = (-((float)iu - (d.nu - 1) / 2.0f) - d.off_u) * d.du;
    float sa, ca;
    sincosf(th - a, &sa, &ca);
    float w = ref_y_main(th) ? g.dy / fabsf(ca) : g.dx / fabsf(sa);
    out[i] = ldf(prj + i) * w;
}

// Detector edge coordinate (cell k spans [k, k+1]) of a physical point for
// one view: fan atan(rx/(ry+dso)) (distanceDriven2DUtils.cu:96-101),
// parallel x cos + y sin (:104-107), then -(a/du + off_u) + nu/2.
__device__ __forceinline__ float det_coord(bool fan, float x, float y, float c, float s, float dso, const Det& d) {
    float a;
    if (fan) {
        float rx = x * c + y * s;
        float ry = -x * s + y * c;
        a = atanf(rx / (ry + dso));
    } else {
        a = x * c + y * s;
    }
    return -(a / d.du + d.off_u) + d.nu / 2.0f;
}

__device__ __forceinline__ double det_coord_d(bool fan, double x, double y, double c, double s, double dso,
                                              const Det& d) {
    double a;
    if (fan) {
        double rx = x * c + y * s;
        double ry = -x * s + y * c;
        a = atan(rx / (ry + dso));
    } else {
        a = x * c + y * s;
    }
    return -(a / d.du + (double)d.off_u) + 0.5 * d.nu;
}

// Window of detector cells covering a pixel tile for one view: the tile
// corners' detector coordinates (extreme over a convex tile) with a margin.
__device__ void tile_window(bool fan, int tx0, int ty0, const Grid& g, const Det& d, double c, double s,
                            double dso, int win, int& w0, int& ok) {
    int tx1 = min(tx0 + kTile, g.nx), ty1 = min(ty0 + kTile, g.ny);
    double xs[2] = {(tx0 - 0.5 * g.nx) * g.dx + g.cx, (tx1 - 0.5 * g.nx) * g.dx + g.cx};
    double ys[2] = {(ty0 - 0.5 * g.ny) * g.dy + g.cy, (ty1 - 0.5 * g.ny) * g.dy + g.cy};
    double jmin = 1e300, jmax = -1e300;
    bool good = true;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            if (fan && (-xs[a] * s + ys[b] * c) + dso <= 0) good = false;
            double j = det_coord_d(fan, xs[a], ys[b], c, s, dso, d);
            jmin = fmin(jmin, j);
            jmax = fmax(jmax, j);
        }
    if (!(jmin > -1e9 && jmax < 1e9)) good = false;
    if (good) {
        w0 = (int)floor(jmin) - 2;
        good = ((int)ceil(jmax) + 2 - w0) <= win;
    } else {
        w0 = 0;
    }
    ok = good ? 1 : 0;
}

// Reference-parity normalised back projection (and FBP mode).
//   fan:      DDBPFanKernel distanceDriven2DBoxInt.cu:319-396
//   parallel: DDBPParallelKernel :409-497
// src is the (pre-weighted, for fan non-FBP) sinogram of this batch item.
// branchless != 0: the reference's branchless back projection
// (distanceDriven2DBranchless.cu:384-530): the parallel beam's main axis alone
// (no blend band), and the detector row interpolated linearly at the pixel's
// v between the two nearest rows (clamped to [0, nv-1]) instead of truncated.
template <bool FAN, typename Tp, typename Tout>
__global__ void __launch_bounds__(kTile* kTile) dd2d_bp_parity_kernel(
    Tout* __restrict__ img, const Tp* __restrict__ src, const float* __restrict__ deg, int nview, Grid g, Det d,
    float dso, int fbp, int accumulate, int win, int branchless) {
    extern __shared__ float smem[];
    float* s_win = smem;                               // [kBPViews][win]
    float* s_cos = s_win + kBPViews * win;             // [kBPViews]
    float* s_sin = s_cos + kBPViews;
    int* s_w0 = (int*)(s_sin + kBPViews);
    int* s_ok = s_w0 + kBPViews;
    int* s_ym = s_ok + kBPViews;

    int tiles_x = (g.nx + kTile - 1) / kTile;
    int tx0 = (blockIdx.x % tiles_x) * kTile, ty0 = (blockIdx.x / tiles_x) * kTile;
    int bz = blockIdx.y;
    int iz = bz % g.nz, b = bz / g.nz;
    int tid = threadIdx.x;
    int ix = tx0 + (tid % kTile), iy = ty0 + (tid / kTile);

    // pixel geometry (ImgToPhysics + half pixel, :340-350)
    float xc = ((float)ix - g.nx / 2.f) * g.dx + g.cx + g.dx / 2;
    float yc = ((float)iy - g.ny / 2.f) * g.dy + g.cy + g.dy / 2;
    float zc = ((float)iz - g.nz / 2.f) * g.dz + g.cz + g.dz / 2;
    float x1 = xc - g.dx / 2.0f, x2 = xc + g.dx / 2.0f;
    float y1 = yc - g.dy / 2.0f, y2 = yc + g.dy / 2.0f;
    float ivf = zc / d.dv + d.off_v + d.nv / 2.f - 0.5f;
    int iv = (int)ivf;  // float passed to an int parameter: truncation (:383)
    bool row_ok = iv >= 0 && iv < d.nv;
    float wrow = 1.f;    // weight of the row of this pass
    int npass = 1, iv_next = iv;
    float w_next = 0.f;
    if (branchless) {  // InterpolateXY of the row prefix sums, cudaMath.cu:227-258
        const float v = clampf(ivf, 0.f, (float)d.nv);
        const int i0 = min((int)v, d.nv - 1), i1 = min((int)v + 1, d.nv - 1);
        w_next = v - (float)i0;
        iv = i0;
        row_ok = true;
        wrow = 1.f - w_next;
        iv_next = i1;
        npass = (w_next != 0.f && i1 != i0) ? 2 : 1;
        if (npass == 1) wrow = 1.f;
    }
    size_t view_stride = (size_t)d.nv * d.nu;

    float acc = 0.f;
    for (int pass = 0; pass < npass; ++pass) {
    if (pass == 1) {
        iv = iv_next;
        wrow = w_next;
    }
    const Tp* rows = src + ((size_t)b * nview * d.nv + (row_ok ? iv : 0)) * d.nu;
    for (int v0 = 0; v0 < nview && row_ok; v0 += kBPViews) {
        int nvc = min(kBPViews, nview - v0);
        if (tid < nvc) {
            double s, c;
            sincos((double)deg[v0 + tid], &s, &c);
            s_cos[tid] = (float)c;
            s_sin[tid] = (float)s;
            int w0, ok;
            tile_window(FAN, tx0, ty0, g, d, c, s, dso, win, w0, ok);
            s_w0[tid] = w0;
            s_ok[tid] = ok;
            s_ym[tid] = ref_y_main(deg[v0 + tid]) ? 1 : 0;
        }
        __syncthreads();
        for (int i = tid; i < nvc * win; i += blockDim.x) {
            int vi = i / win, k = i - vi * win;
            int cell = s_w0[vi] + k;
            float val = 0.f;
            if (s_ok[vi] && cell >= 0 && cell < d.nu) val = ldf(rows + (size_t)(v0 + vi) * view_stride + cell);
            s_win[i] = val;
        }
        __syncthreads();
        if (ix < g.nx && iy < g.ny) {
            for (int vi = 0; vi < nvc; ++vi) {
                float c = s_cos[vi], s = s_sin[vi];
                const float* w = s_win + vi * win;
                float off = (float)s_w0[vi];
                bool ok = s_ok[vi] != 0;
                const Tp* grow = rows + (size_t)(v0 + vi) * view_stride;
                if (FAN) {
                    float a1, a2;
                    if (s_ym[vi]) {
                        a1 = det_coord(true, x1, yc, c, s, dso, d);
                        a2 = det_coord(true, x2, yc, c, s, dso, d);
                    } else {
                        a1 = det_coord(true, xc, y1, c, s, dso, d);
                        a2 = det_coord(true, xc, y2, c, s, dso, d);
                    }
                    float lo = fminf(a1, a2), hi = fmaxf(a1, a2);
                    float val = ok ? box_line_smem(w, lo - off, hi - off, win) : box_line(grow, 1, lo, hi, d.nu);
                    val = val / (hi - lo);
                    if (fbp) {
                        float rx = xc * c + yc * s, ry = -xc * s + yc * c;
                        val *= dso * dso / (rx * rx + (dso + ry) * (dso + ry));
                    }
                    acc += val * wrow;
                } else {
                    float valx = 0.f, valy = 0.f;
                    const float wx = branchless ? (s_ym[vi] ? 1.f : 0.f)
                                                : clampf((fabsf(c) - fabsf(s) + kDDMargin) / (2 * kDDMargin), 0.f, 1.f);
                    if (wx > 0.f) {
                        float u1 = det_coord(false, x1, yc, c, s, dso, d);
                        float u2 = det_coord(false, x2, yc, c, s, dso, d);
                        float lo = fminf(u1, u2), hi = fmaxf(u1, u2);
                        valx = (ok ? box_line_smem(w, lo - off, hi - off, win) : box_line(grow, 1, lo, hi, d.nu)) /
                               (hi - lo);
                    }
                    if (wx < 1.f) {
                        float u1 = det_coord(false, xc, y1, c, s, dso, d);
                        float u2 = det_coord(false, xc, y2, c, s, dso, d);
                        float lo = fminf(u1, u2), hi = fmaxf(u1, u2);
                        valy = (ok ? box_line_smem(w, lo - off, hi - off, win) : box_line(grow, 1, lo, hi, d.nu)) /
                               (hi - lo);
                    }
                    float val = valx * wx + valy * (1 - wx);
                    if (!fbp) val *= s_ym[vi] ? g.dy / fabsf(c) : g.dx / fabsf(s);  // :39-65
                    acc += val * wrow;
                }
            }
        }
        __syncthreads();
    }
    }
    if (ix < g.nx && iy < g.ny) {
        Tout* o = img + (((size_t)b * g.nz + iz) * g.ny + iy) * g.nx + ix;
        if (accumulate) acc += rdf(o);
        stf(o, acc);
    }
}

// Exact transpose of dd2d_fp_kernel, as a gather over a pixel tile.
// For each pixel and view, the candidate cells come from the pixel's detector
// coordinates (+-1 cell); the weight of cell k is the image-space overlap of
// the pixel with the cell's footprint on the pixel's row (column) divided by
// the footprint width, times L and the blend weight -- the forward
// projector's coefficient, from the same table entries.
template <bool FAN, typename Tp, typename Tout>
__global__ void __launch_bounds__(kTile* kTile) dd2d_bp_adjoint_kernel(
    Tout* __restrict__ img, const Tp* __restrict__ prj, const float* __restrict__ deg, DDTab tab, int nview, Grid g,
    Det d, float dso, int accumulate, int win) {
    extern __shared__ float smem[];
    // per view: p[win], then per orientation: A[win+1], B[win+1], L[win]
    const int per_o = 2 * (win + 1) + win;
    const int per_v = win + 2 * per_o;
    float* s_view = smem;                           // [kAdjViews][per_v]
    float* s_cos = s_view + kAdjViews * per_v;      // [kAdjViews]
    float* s_sin = s_cos + kAdjViews;
    float* s_wx = s_sin + kAdjViews;
    int* s_w0 = (int*)(s_wx + kAdjViews);
    int* s_ok = s_w0 + kAdjViews;

    int tiles_x = (g.nx + kTile - 1) / kTile;
    int tx0 = (blockIdx.x % tiles_x) * kTile, ty0 = (blockIdx.x / tiles_x) * kTile;
    int bz = blockIdx.y;
    int iz = bz % g.nz, b = bz / g.nz;
    int tid = threadIdx.x;
    int ix = tx0 + (tid % kTile), iy = ty0 + (tid / kTile);
    float xc = ((float)ix - g.nx / 2.f) * g.dx + g.cx + g.dx / 2;
    float yc = ((float)iy - g.ny / 2.f) * g.dy + g.cy + g.dy / 2;
    float x1 = xc - g.dx / 2.0f, x2 = xc + g.dx / 2.0f;
    float y1 = yc - g.dy / 2.0f, y2 = yc + g.dy / 2.0f;
    float ty = (float)(iy - tab.ym), tx = (float)(ix - tab.xm);
    float fx = (float)ix, fy = (float)iy;

    float acc = 0.f;
    for (int iv = 0; iv < d.nv; ++iv) {
        // weight of slice iz in the z interpolation of detector row iv
        int za, zb;
        float wz;
        row_z(iv, g, d, za, zb, wz);
        float om = (za == iz ? 1.f - wz : 0.f) + ((zb == iz && wz != 0.f) ? wz : 0.f);
        if (om == 0.f) continue;
        const Tp* rows = prj + ((size_t)b * nview * d.nv + iv) * d.nu;
        for (int v0 = 0; v0 < nview; v0 += kAdjViews) {
            int nvc = min(kAdjViews, nview - v0);
            if (tid < nvc) {
                double s, c;
                sincos((double)deg[v0 + tid], &s, &c);
                s_cos[tid] = (float)c;
                s_sin[tid] = (float)s;
                s_wx[tid] = tab.wx[v0 + tid];
                int w0, ok;
                tile_window(FAN, tx0, ty0, g, d, c, s, dso, win, w0, ok);
                s_w0[tid] = w0;
                s_ok[tid] = ok;
            }
            __syncthreads();
            for (int i = tid; i < nvc * per_v; i += blockDim.x) {
                int vi = i / per_v, r = i - vi * per_v;
                int view = v0 + vi;
                int w0 = s_w0[vi];
                float val = 0.f;
                if (s_ok[vi]) {
                    if (r < win) {
                        int cell = w0 + r;
                        if (cell >= 0 && cell < d.nu) val = ldf(rows + (size_t)view * d.nv * d.nu + cell) * om;
                    } else {
                        int q = r - win;
                        int o = q / per_o;
                        q -= o * per_o;
                        if (q < 2 * (win + 1)) {
                            int e = w0 + (q % (win + 1));
                            if (e >= 0 && e <= d.nu) {
                                size_t ie = (size_t)view * (d.nu + 1) + e;
                                val = (q < win + 1) ? tab.eA[o][ie] : tab.eB[o][ie];
                            }
                        } else {
                            int cell = w0 + (q - 2 * (win + 1));
                            if (cell >= 0 && cell < d.nu) val = tab.cL[o][(size_t)view * d.nu + cell];
                        }
                    }
                }
                s_view[i] = val;
            }
            __syncthreads();
            if (ix < g.nx && iy < g.ny) {
                for (int vi = 0; vi < nvc; ++vi) {
                    int view = v0 + vi;
                    float c = s_cos[vi], s = s_sin[vi], wx = s_wx[vi];
                    int w0 = s_w0[vi];
                    bool ok = s_ok[vi] != 0;
                    const float* sv = s_view + vi * per_v;
                    for (int o = 0; o < 2; ++o) {
                        float wo = o == 0 ? wx : 1.f - wx;
                        if (!(wo > 0.f)) continue;
                        float j1, j2, t, pmin;
                        if (o == 0) {
                            j1 = det_coord(FAN, x1, yc, c, s, dso, d);
                            j2 = det_coord(FAN, x2, yc, c, s, dso, d);
                            t = ty;
                            pmin = fx;
                        } else {
                            j1 = det_coord(FAN, xc, y1, c, s, dso, d);
                            j2 = det_coord(FAN, xc, y2, c, s, dso, d);
                            t = tx;
                            pmin = fy;
                        }
                        int kmin = max((int)floorf(fminf(j1, j2)) - 1, 0);
                        int kmax = min((int)floorf(fmaxf(j1, j2)) + 1, d.nu - 1);
                        float sum = 0.f;
                        const float* sp = sv;
                        const float* sA = sv + win + o * per_o;
                        const float* sB = sA + (win + 1);
                        const float* sL = sB + (win + 1);
                        for (int k = kmin; k <= kmax; ++k) {
                            float Aa, Ba, Ab, Bb, L, p;
                            int kk = k - w0;
                            if (ok && kk >= 0 && kk < win) {
                                Aa = sA[kk]; Ba = sB[kk]; Ab = sA[kk + 1]; Bb = sB[kk + 1];
                                L = sL[kk]; p = sp[kk];
                            } else {
                                size_t ie = (size_t)view * (d.nu + 1) + k, ic = (size_t)view * d.nu + k;
                                Aa = tab.eA[o][ie]; Ba = tab.eB[o][ie]; Ab = tab.eA[o][ie + 1]; Bb = tab.eB[o][ie + 1];
                                L = tab.cL[o][ic];
                                p = ldf(rows + (size_t)view * d.nv * d.nu + k) * om;
                            }
                            float xa = fmaf(Ba, t, Aa), xb = fmaf(Bb, t, Ab);
                            float lo = fminf(xa, xb), hi = fmaxf(xa, xb);
                            float ov = fminf(hi, pmin + 1.f) - fmaxf(lo, pmin);
                            // the forward projector's coefficient: overlap over the
                            // width of the same rounded footprint
                            if (ov > 0.f) sum += p * L * __fdividef(ov, hi - lo);
                        }
                        acc += sum * wo;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (ix < g.nx && iy < g.ny) {
        Tout* o = img + (((size_t)b * g.nz + iz) * g.ny + iy) * g.nx + ix;
        if (accumulate) acc += rdf(o);
        stf(o, acc);
    }
}

// ---------------------------------------------------------------------------
// Forward projection, fast path (fan and parallel, z slices projected one to
// one onto detector rows).
//
// A CTA owns a group of views of one slice and streams the image through
// shared memory a few lines at a time (rows of the image for the views traced
// along y, rows of the transposed image for those traced along x).  Each staged
// line is stored as its running integral F in FP64 plus the pixel value r, so
// the integral of the line over [a, b] is F(b) - F(a) with no cancellation.
// Detector cells share their edges, so each lane of a warp evaluates F at one
// edge: 31 rays per warp, one table read per ray and line.  On every line the
// footprint of a cell is the same multiple of one per-ray constant (parallel
// beams: the width itself; fan beams: the slope difference of the two edge
// rays times the line's distance tau from the source), so each lane sums F at
// its own edge over the lines, weighted by 1/tau for fan beams, and the cell
// is the difference of two neighbouring sums taken once, after the last line:
// no shuffle or divide per line (fp_line).  The normalisation by the
// footprint width, the ray-length factor and the blend weight are those of
// DDFPTracing (distanceDriven2DBoxInt.cu:21-106).
constexpr int kFMaxItems = 16;  // edge groups (of 32 edges) per warp

// Running integral along a line from its midpoint table.  The line of n
// cells gets a zero cell on each side (cells -1 and n); table entry k = i + 1
// of cell i in [-1, n] holds M_i = C_i + r_i/2 and r_i, C_i the integral up
// to cell i, so F(x) = M_i + r_i (x' - i) at x' = x - 1/2 for the cell i
// nearest x'.  Edge positions are normalised, xn = (x' + 1) / (n + 1), and
// clamped to [0, 1] by the saturating FP32 fused multiply-add that computes
// them, so the clamped x' = xn (n + 1) - 1 spans [-1, n] and every lookup
// stays inside the table (NaN saturates to 0).  The nearest integer comes
// from the float adder in the same kind of instruction: xn (n + 1) +
// (1.5*2^23 - 1) rounds x' to an integer in the low mantissa bits, and
// xn (n + 1) + (1.5*2^23 - 1 - that sum) is its fraction, both from the exact
// product; the mantissa bits, times the entry size, plus a base offset are
// the entry's shared-memory address.
constexpr float kRoundMagic = 12582912.0f;  // 1.5 * 2^23
constexpr unsigned kRoundMagicBits = 0x4B400000u;

// Approximate reciprocal (the PTX rcp.approx instruction, flushing
// subnormals): one instruction, relative error about 1 ulp.
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// a * b + c rounded once, clamped to [0, 1] (NaN to 0)
__device__ __forceinline__ float fma_sat(float a, float b, float c) {
    float y;
    asm("fma.rn.sat.f32 %0, %1, %2, %3;" : "=f"(y) : "f"(a), "f"(b), "f"(c));
    return y;
}

__device__ __forceinline__ double lds_f64(unsigned addr) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr));
    return v;
}

__device__ __forceinline__ float lds_f32(unsigned addr) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
    return v;
}

// Layout of one line's midpoint table (n cells, entries 0..n+1): n + 2 FP64
// values M_i padded to an even count, then n + 2 FP32 cell values r_i padded
// to a multiple of four.  Both parts, and so every line of a stack of tables,
// start on a 16-byte boundary, as bulk copies require.  A warp reads 8 + 4
// bytes per edge in two accesses: the edges of a warp spread over more
// entries than lanes, so the wavefronts of a read grow with the bytes
// spanned, and 12 bytes span fewer than one 16-byte entry would.
__host__ __device__ __forceinline__ int line_nf(int n) { return (n + 3) & ~1; }
__host__ __device__ __forceinline__ int line_nr(int n) { return (n + 5) & ~3; }
__host__ __device__ __forceinline__ size_t line_bytes(int n) { return (size_t)8 * line_nf(n) + (size_t)4 * line_nr(n); }

// Shared-memory base offsets of a line table for the lookup of fp_line: the
// address of the entry of cell i is base + size * (kRoundMagicBits + i) + size
// (32-bit arithmetic, modulo 2^32).
struct LineBase {
    unsigned f, r;
};
__device__ __forceinline__ LineBase line_base(const unsigned char* line, int n) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(line);
    return {a + 8u - 8u * kRoundMagicBits, a + 8u * (unsigned)line_nf(n) + 4u - 4u * kRoundMagicBits};
}

// Edge group q of a warp: its view within the CTA (vi) and its group of 31
// cells within the view (m).  wpv > 0: each view has wpv consecutive warps
// and a warp's groups all belong to one view (fan beams share the line's
// weight across them); wpv == 0: the CTA's edge groups are numbered view by
// view across the 8 warps, it = warp + 8 q (parallel beams, densest packing).
// The group is real if vi < the CTA's views and m < the groups per view.
__device__ __forceinline__ void fp_item(int warp, int q, int ipv, int wpv, int& vi, int& m) {
    if (wpv > 0) {
        vi = warp / wpv;
        m = warp - vi * wpv + wpv * q;
    } else {
        const int it = warp + 8 * q;
        vi = it / ipv;
        m = it - vi * ipv;
    }
}

// One image line's contribution to a thread's NI edge groups.  L is the
// line's table, t the line's coordinate from the anchor line, W = n + 1 and
// Cm = 1.5*2^23 - 1.  Positions and slopes are normalised (xn above):
//   parallel: edge position A + B t, A on the anchor line (fp_norm_grid) and
//        the same slope B for every edge of a view, so a cell's footprint
//        has the same width on every line; the lane adds F at its edge
//        (accd += M in FP64, the small r * frac part in FP32 in alo, folded
//        into accd every 16 lines).
//   FAN: edge position A + B tau with A, S the source's position and line
//        coordinate and tau = t - S the line's distance from the source
//        (the same for every edge of the view), so the footprint between
//        edges j and j+1 is (B_j+1 - B_j) tau wide, and the rounding of the
//        common A cancels in it; the lane adds F / tau (the FP32 weight
//        1/tau is common to the cell's two edges, so its rounding only
//        reweights the line).
// Fan beams: every edge group of the warp belongs to the same view (fp_item;
// dummy groups past the view included, whose results are dropped), so tau and
// its weight are computed once per line from group 0's source coordinate.
template <bool FAN, int NI>
__device__ __forceinline__ void fp_line(LineBase L, float t, float W, float Cm, const float (&A)[NI],
                                        const float (&B)[NI], const float (&S)[NI], double (&accd)[NI],
                                        float (&alo)[NI]) {
    float tau = t, wgt = 1.f;
    if constexpr (FAN) {
        tau = t - S[0];  // |tau| >= 1/2 (a dummy warp) or the source's distance
        wgt = rcp_approx(tau);
    }
    const double wd = (double)wgt;
#pragma unroll
    for (int q = 0; q < NI; ++q) {
        const float xn = fma_sat(B[q], tau, A[q]);
        const float tt = fmaf(xn, W, Cm);
        const unsigned bits = __float_as_uint(tt);
        const double F = lds_f64(L.f + 8u * bits);
        const float r = lds_f32(L.r + 4u * bits);
        const float frac = fmaf(xn, W, Cm - tt);
        if constexpr (FAN) {
            accd[q] = fma(wd, F, accd[q]);
            alo[q] = fmaf(wgt * r, frac, alo[q]);
        } else {
            accd[q] += F;
            alo[q] = fmaf(r, frac, alo[q]);
        }
    }
}

// Fold the FP32 parts (at most 16 lines of r * frac) into the FP64 sums.
template <int NI>
__device__ __forceinline__ void fp_renorm(double (&accd)[NI], float (&alo)[NI]) {
#pragma unroll
    for (int q = 0; q < NI; ++q) {
        accd[q] += (double)alo[q];
        alo[q] = 0.f;
    }
}

// Normalised edge coordinate of fp_line on a line of n cells: (v + add) /
// (n + 1) in FP64 (inv = 1 / (n + 1)), rounded to FP32 (add = 1/2 for a
// position, 0 for a slope).
__device__ __forceinline__ float fp_norm(double v, double add, double inv) { return (float)((v + add) * inv); }

// Normalised position of a parallel-beam edge on the anchor line, on the
// grid of multiples of 2^-24 (fp_norm, then rounded to that grid): the
// positions A_j + B t of a view's edges share B t, so with every A_j on a
// grid no finer than that of the sums, the sums of one binade round alike
// and the footprint widths between the edges stay exactly A_j+1 - A_j, the
// widths fp_cell_sum divides by.
__device__ __forceinline__ float fp_norm_grid(double v, double add, double inv) {
    constexpr double kGrid = 16777216.0;  // 2^24
    return (float)(rint((v + add) * inv * kGrid) / kGrid);
}

// Sum over lines of the cell integral over the footprint width, for the cell
// between this lane's edge and the next lane's (all lanes call it, sums
// renormalised first): the difference of the two edge sums over the
// difference of W, the edge's normalised position at the anchor line
// (parallel) or its normalised slope (fan); the caller divides by n + 1.
__device__ __forceinline__ float fp_cell_sum(double accd, float W) {
    const double dn = __shfl_down_sync(0xffffffffu, accd, 1);
    const float Wn = __shfl_down_sync(0xffffffffu, W, 1);
    return __fdividef((float)(dn - accd), Wn - W);
}

// FP64 midpoint table of one line, built by one warp: entries k = 0..n+1 of
// cells i = k - 1 (zero cells at -1 and n), M_i = C_i + r_i/2 and r_i, C_i
// the integral over cells [0, i) and r_i the cell value; the padding entries
// are zero.
template <typename Cell>
__device__ __forceinline__ void build_line_fp64(unsigned char* __restrict__ line, int n, int lane, Cell cell) {
    double* Fm = reinterpret_cast<double*>(line);
    float* Rc = reinterpret_cast<float*>(line + 8 * line_nf(n));
    const int ne = n + 2;
    const int E = (ne + 31) / 32;
    const int k0 = lane * E;
    double tot = 0.0;
    for (int q = 0; q < E; ++q) {
        const int i = k0 + q - 1;
        if (i >= 0 && i < n) tot += (double)cell(i);
    }
    double inc = tot;  // inclusive scan of the lane totals
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    double c = inc - tot;
    for (int q = 0; q < E; ++q) {
        const int k = k0 + q, i = k - 1;
        if (k < ne) {
            const float r = (i >= 0 && i < n) ? cell(i) : 0.f;
            Fm[k] = c + 0.5 * (double)r;
            Rc[k] = r;
            c += (double)r;
        }
    }
    if (ne + lane < line_nf(n)) Fm[ne + lane] = 0.0;
    if (ne + lane < line_nr(n)) Rc[ne + lane] = 0.f;
}

// The same from a row of the image in global memory.
template <typename Tin>
__device__ __forceinline__ void stage_line_fp64(unsigned char* __restrict__ line, const Tin* __restrict__ row,
                                                int n, int lane) {
    build_line_fp64(line, n, lane, [&](int i) { return ldf(row + i); });
}

// Stage lines (length n, stride n between lines) into consecutive tables.
template <typename Tin>
__device__ void stage_lines(unsigned char* __restrict__ tab, const Tin* __restrict__ src, int nlines, int n,
                            int warp, int lane, int nwarps) {
    for (int l = warp; l < nlines; l += nwarps)
        stage_line_fp64(tab + (size_t)l * line_bytes(n), src + (size_t)l * n, n, lane);
}

// Shared memory of one warp of line_tables_kernel: a line's table, then its
// cells (both multiples of 16 bytes).
__host__ __device__ __forceinline__ size_t line_tables_warp_bytes(int n) {
    return line_bytes(n) + (((size_t)n * 4 + 15) & ~(size_t)15);
}

// The tables of every line of a stack of slices (one warp per line), for the
// forward projector that streams them into shared memory.  The warp reads the
// line's cells into shared memory with coalesced loads, builds the table
// there (each lane scans a run of consecutive entries) and writes it out with
// coalesced 16-byte stores.
template <typename Tin>
__global__ void __launch_bounds__(256) line_tables_kernel(unsigned char* __restrict__ out,
                                                          const Tin* __restrict__ src, long long nlines, int n) {
    extern __shared__ float4 s_lt4[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t lb = line_bytes(n);
    unsigned char* tab = reinterpret_cast<unsigned char*>(s_lt4) + warp * line_tables_warp_bytes(n);
    float* cells = reinterpret_cast<float*>(tab + lb);
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long l = w0; l < nlines; l += nw) {
        const Tin* row = src + l * n;
        for (int i = lane; i < n; i += 32) cells[i] = ldf(row + i);
        __syncwarp();
        build_line_fp64(tab, n, lane, [&](int i) { return cells[i]; });
        __syncwarp();
        const uint4* from = reinterpret_cast<const uint4*>(tab);
        uint4* to = reinterpret_cast<uint4*>(out + l * lb);
        for (int i = lane; i < (int)(lb / 16); i += 32) to[i] = from[i];
        __syncwarp();
    }
}

// NI = edge groups per warp (compile time, so the group loop is straight-line
// code with independent dependency chains); groups beyond the CTA's views are
// harmless dummies whose results are dropped.
// An edge group holds five registers (position, slope, the FP64 sum and its
// FP32 part; fan beams add the source's line coordinate): above 4 groups per
// warp the staged kernel runs two CTAs per SM.
template <bool FAN, int NI>
constexpr int fp_fast_min_blocks() { return NI <= 4 ? 3 : 2; }

template <bool FAN, int NI, typename Tin, typename Tout>
__global__ void __launch_bounds__(256, (fp_fast_min_blocks<FAN, NI>())) dd2d_fp_fast_kernel(Tout* __restrict__ prj, const Tin* __restrict__ img,
                                                           const Tin* __restrict__ imgT, DDTab tab, Grid g, Det d,
                                                           int nview, int vgroup, int wpv, int nrows_chunk,
                                                           const float* __restrict__ deg, int unweight_par) {
    extern __shared__ float4 s_lines4[];
    unsigned char* s_lines = reinterpret_cast<unsigned char*>(s_lines4);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int v0 = blockIdx.x * vgroup;
    const int nvg = min(vgroup, nview - v0);
    const int slice = blockIdx.y;  // b * nz + iz, detector row iv = iz
    const int iz = slice % g.nz, b = slice / g.nz;
    const int ipv = (d.nu + 30) / 31;  // edge groups per view

    for (int o = 0; o < 2; ++o) {
        const int n = o == 0 ? g.nx : g.ny;   // cells per line
        const int nl = o == 0 ? g.ny : g.nx;  // lines
        const int anchor = o == 0 ? tab.ym : tab.xm;
        const Tin* src = (o == 0 ? img : imgT) + (size_t)slice * g.nx * g.ny;
        float A[NI], B[NI], S[NI], alo[NI];
        double accd[NI];
        bool any = false;
        const double inv = 1.0 / (double)(n + 1);
#pragma unroll
        for (int q = 0; q < NI; ++q) {
            int vi, m;
            fp_item(warp, q, ipv, wpv, vi, m);
            // dummy edges (results dropped): positions in range, tau never 0
            A[q] = 0.5f;
            B[q] = 0.f;
            S[q] = 0.5f;
            accd[q] = 0.0;
            alo[q] = 0.f;
            if (vi < nvg && m < ipv) {
                const int view = v0 + vi;
                const float wx = tab.wx[view];
                const bool active = o == 0 ? wx > 0.f : wx < 1.f;
                const int j = 31 * m + lane;
                if (active && j <= d.nu) {
                    const size_t ie = (size_t)view * (d.nu + 1) + j;
                    A[q] = FAN ? fp_norm(tab.sP[o][view], 0.5, inv) : fp_norm_grid(tab.eA[o][ie], 0.5, inv);
                    B[q] = fp_norm((double)tab.eB[o][ie], 0.0, inv);
                    if (FAN) S[q] = tab.sS[o][view];
                    any = true;
                }
            }
        }
        // every warp takes part in staging whether or not it has work
        if (!__syncthreads_or(any)) continue;
        const float W = (float)(n + 1), Cm = kRoundMagic - 1.f;
        const int renorm = max(1, 16 / nrows_chunk);  // chunks between renormalisations
        for (int l0 = 0, c = 0; l0 < nl; l0 += nrows_chunk, ++c) {
            const int nlc = min(nrows_chunk, nl - l0);
            __syncthreads();
            stage_lines<Tin>(s_lines, src + (size_t)l0 * n, nlc, n, warp, lane, 8);
            __syncthreads();
            for (int r = 0; r < nlc; ++r)
                fp_line<FAN, NI>(line_base(s_lines + (size_t)r * line_bytes(n), n), (float)(l0 + r - anchor),
                                       W, Cm, A, B, S, accd, alo);
            if ((c + 1) % renorm == 0) fp_renorm<NI>(accd, alo);
        }
        fp_renorm<NI>(accd, alo);
#pragma unroll
        for (int q = 0; q < NI; ++q) {
            int vi, m;
            fp_item(warp, q, ipv, wpv, vi, m);
            if (vi >= nvg || m >= ipv) continue;
            const float sum = fp_cell_sum(accd[q], FAN ? B[q] : A[q]) / W;
            const int view = v0 + vi;
            const int k = 31 * m + lane;
            const float wx = tab.wx[view];
            const bool active = o == 0 ? wx > 0.f : wx < 1.f;
            if (!active || lane >= 31 || k >= d.nu) continue;
            float v = sum * tab.cL[o][(size_t)view * d.nu + k] * (o == 0 ? wx : 1.f - wx);
            Tout* dst = prj + (((size_t)b * nview + view) * d.nv + iz) * d.nu + k;
            if (o == 1 && wx > 0.f) v += rdf(dst);  // the row sweep of this view wrote first
            stf(dst, v);
        }
    }
    if (unweight_par) {
        // FORCE_FBP on parallel FP: cancel the ray-length weight
        // (ReverseWeightBPParallelKernel, distanceDriven2DUtils.cu:68-94)
        for (int q = 0; q < NI; ++q) {
            int vi, m;
            fp_item(warp, q, ipv, wpv, vi, m);
            if (vi >= nvg || m >= ipv) continue;
            const int view = v0 + vi;
            const int k = 31 * m + lane;
            if (lane >= 31 || k >= d.nu) continue;
            float sn, cs;
            sincosf(deg[view], &sn, &cs);
            Tout* dst = prj + (((size_t)b * nview + view) * d.nv + iz) * d.nu + k;
            stf(dst, rdf(dst) / (ref_y_main(deg[view]) ? g.dy / fabsf(cs) : g.dx / fabsf(sn)));
        }
    }
}

// ---------------------------------------------------------------------------
// Forward projection, streamed-table path.  Same arithmetic as
// dd2d_fp_fast_kernel, but the midpoint tables of every image line are built
// once per slice by line_tables_kernel and streamed into a two-buffer ring in
// shared memory with bulk asynchronous copies (cp.async.bulk, completion on an
// mbarrier): while the warps integrate one chunk of lines, the copy of the
// next chunk is in flight, and no warp spends instructions on staging.
__device__ unsigned int g_wait_timeouts;  // bounded waits that gave up (read by ctp_wait_timeouts)

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// bytes and both addresses are multiples of 16
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar`, giving up (and counting it) after a bounded
// number of polls instead of spinning forever.
constexpr unsigned kWaitPolls = CTP_WAIT_POLLS_DEFAULT;
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned polls = kWaitPolls) {
    for (unsigned i = 0; i < polls; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    atomicAdd(&g_wait_timeouts, 1u);
    return false;
}

// Poll limit of each CTA's first chunk wait (ctp_set_wait_limit).  Lowering it
// lets a test make that wait give up; the waits that let in-flight copies land
// before a CTA exits keep kWaitPolls.
__device__ unsigned int g_first_wait_polls = kWaitPolls;

// Above 8 edge groups per warp (five or six registers per group) two CTAs
// per SM.
template <bool FAN, int NI>
constexpr int fp_stream_min_blocks() { return NI <= 8 ? 3 : 2; }

// The views in the order the streamed forward projector takes them: those of
// the blend band (0 < wx < 1), which sweep both orientations and so take
// about twice as long, first, then the others, each in their original order
// (a stable partition).  The launch dispatches view groups in this order, so
// its longest CTAs start in the first wave instead of trailing the last.
// One CTA; ballots and per-warp counts give each view its position.
__global__ void __launch_bounds__(1024) blend_first_kernel(int* __restrict__ order, const float* __restrict__ wx,
                                                           int nview) {
    __shared__ int s_cnt[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    auto in_band = [&](int v) { return v < nview && wx[v] > 0.f && wx[v] < 1.f; };
    int nband = 0;
    for (int t0 = 0; t0 < nview; t0 += blockDim.x) nband += __syncthreads_count(in_band(t0 + threadIdx.x));
    int placed_band = 0, placed_rest = 0;
    for (int t0 = 0; t0 < nview; t0 += blockDim.x) {
        const int v = t0 + threadIdx.x;
        const bool in = v < nview, band = in_band(v);
        const unsigned mb = __ballot_sync(0xffffffffu, band), mi = __ballot_sync(0xffffffffu, in);
        const unsigned below = (1u << lane) - 1u;
        if (lane == 0) s_cnt[warp] = __popc(mb) | (__popc(mi) << 16);
        __syncthreads();
        int band_before = __popc(mb & below), all_before = __popc(mi & below), tile_band = 0, tile_all = 0;
        for (int w = 0; w < nw; ++w) {
            const int c = s_cnt[w];
            if (w < warp) {
                band_before += c & 0xffff;
                all_before += c >> 16;
            }
            tile_band += c & 0xffff;
            tile_all += c >> 16;
        }
        if (in)
            order[band ? placed_band + band_before : nband + placed_rest + (all_before - band_before)] = v;
        placed_band += tile_band;
        placed_rest += tile_all - tile_band;
        __syncthreads();
    }
}

template <bool FAN, int NI, typename Tout>
__global__ void __launch_bounds__(256, (fp_stream_min_blocks<FAN, NI>())) dd2d_fp_stream_kernel(Tout* __restrict__ prj, const unsigned char* __restrict__ ltab0,
                                                             const unsigned char* __restrict__ ltab1, DDTab tab, Grid g,
                                                             Det d, int nview, int vgroup, int wpv, int rchunk, int slice0,
                                                             const int* __restrict__ order, const float* __restrict__ deg,
                                                             int unweight_par) {
    extern __shared__ float4 s_ring4[];  // [2][rchunk line tables of max(nx, ny) cells]
    unsigned char* s_ring = reinterpret_cast<unsigned char*>(s_ring4);
    __shared__ __align__(8) unsigned long long s_bar[2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // view group blockIdx.y of the views in `order` (blend-band views first),
    // slice b * nz + iz (detector row iv = iz) whose tables are the launch's
    // blockIdx.x-th
    const int v0 = blockIdx.y * vgroup;
    const int nvg = min(vgroup, nview - v0);
    const int slice = slice0 + (int)blockIdx.x;
    const int iz = slice % g.nz, b = slice / g.nz;
    const int ipv = (d.nu + 30) / 31;  // edge groups per view
    const size_t ring = (size_t)rchunk * line_bytes(max(g.nx, g.ny));  // bytes per buffer

    // orientations with work in this CTA: rows (o = 0) for views traced along
    // y, columns (o = 1) for views traced along x, both in the blend band
    bool act0 = false, act1 = false;
    for (int vi = threadIdx.x; vi < nvg; vi += blockDim.x) {
        const float wx = tab.wx[order[v0 + vi]];
        act0 |= wx > 0.f;
        act1 |= wx < 1.f;
    }
    act0 = __syncthreads_or(act0);
    act1 = __syncthreads_or(act1);
    const int nc0 = act0 ? (g.ny + rchunk - 1) / rchunk : 0;
    const int nc1 = act1 ? (g.nx + rchunk - 1) / rchunk : 0;
    const int K = nc0 + nc1;
    const unsigned char* src0 = ltab0 + (size_t)blockIdx.x * g.ny * line_bytes(g.nx);
    const unsigned char* src1 = ltab1 + (size_t)blockIdx.x * g.nx * line_bytes(g.ny);

    auto issue = [&](int k) {
        const int o = k < nc0 ? 0 : 1;
        const int c = o == 0 ? k : k - nc0;
        const int n = o == 0 ? g.nx : g.ny, nl = o == 0 ? g.ny : g.nx;
        const int l0 = c * rchunk, nlc = min(rchunk, nl - l0);
        const unsigned bytes = (unsigned)((size_t)nlc * line_bytes(n));
        unsigned long long* bar = &s_bar[k & 1];
        mbar_expect_tx(bar, bytes);
        bulk_copy_g2s(s_ring + (k & 1) * ring, (o == 0 ? src0 : src1) + (size_t)l0 * line_bytes(n), bytes, bar);
    };
    if (threadIdx.x == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (K > 0) issue(0);
        if (K > 1) issue(1);
    }

    // per edge group: edge position and slope, and the sums of fp_line
    float A[NI], B[NI], S[NI], alo[NI];
    double accd[NI];
    const int renorm = max(1, 16 / rchunk);  // chunks between renormalisations of (acc, alo)
    const unsigned first_polls = g_first_wait_polls;
    bool failed = false;
    int k = 0;
    for (; k < K; ++k) {
        const int o = k < nc0 ? 0 : 1;
        const int c = o == 0 ? k : k - nc0;
        const int n = o == 0 ? g.nx : g.ny, nl = o == 0 ? g.ny : g.nx;
        const int last = (o == 0 ? nc0 : nc1) - 1;
        if (c == 0) {
            const double inv = 1.0 / (double)(n + 1);
#pragma unroll
            for (int q = 0; q < NI; ++q) {
                int vi, m;
                fp_item(warp, q, ipv, wpv, vi, m);
                // dummy edges (results dropped): positions in range, tau never 0
                A[q] = 0.5f;
                B[q] = 0.f;
                S[q] = 0.5f;
                accd[q] = 0.0;
                alo[q] = 0.f;
                if (vi < nvg && m < ipv) {
                    const int view = order[v0 + vi];
                    const float wx = tab.wx[view];
                    const bool active = o == 0 ? wx > 0.f : wx < 1.f;
                    const int j = 31 * m + lane;
                    if (active && j <= d.nu) {
                        const size_t ie = (size_t)view * (d.nu + 1) + j;
                        A[q] = FAN ? fp_norm(tab.sP[o][view], 0.5, inv) : fp_norm_grid(tab.eA[o][ie], 0.5, inv);
                        B[q] = fp_norm((double)tab.eB[o][ie], 0.0, inv);
                        if (FAN) S[q] = tab.sS[o][view];
                    }
                }
            }
        }
        if (!mbar_wait_bounded(&s_bar[k & 1], (k >> 1) & 1, k == 0 ? first_polls : kWaitPolls)) failed = true;
        failed = __any_sync(0xffffffffu, failed);  // the cell sums shuffle: whole warps stop together
        const unsigned char* buf = s_ring + (k & 1) * ring;
        const int anchor = o == 0 ? tab.ym : tab.xm;
        const int l0 = c * rchunk, nlc = min(rchunk, nl - l0);
        const float W = (float)(n + 1), Cm = kRoundMagic - 1.f;
        float tl = (float)(l0 - anchor);  // line coordinate, stepped exactly
        LineBase L = line_base(buf, n);
        const unsigned lb = (unsigned)line_bytes(n);
        for (int r = 0; r < nlc && !failed; ++r, tl += 1.f, L.f += lb, L.r += lb)
            fp_line<FAN, NI>(L, tl, W, Cm, A, B, S, accd, alo);
        if ((c + 1) % renorm == 0 || c == last) fp_renorm<NI>(accd, alo);
        if (c == last && !failed) {
#pragma unroll
            for (int q = 0; q < NI; ++q) {
                int vi, m;
                fp_item(warp, q, ipv, wpv, vi, m);
                if (vi >= nvg || m >= ipv) continue;
                const float sum = fp_cell_sum(accd[q], FAN ? B[q] : A[q]) / (float)(n + 1);
                const int view = order[v0 + vi];
                const int kk = 31 * m + lane;
                const float wx = tab.wx[view];
                const bool active = o == 0 ? wx > 0.f : wx < 1.f;
                if (!active || lane >= 31 || kk >= d.nu) continue;
                float v = sum * tab.cL[o][(size_t)view * d.nu + kk] * (o == 0 ? wx : 1.f - wx);
                Tout* dst = prj + (((size_t)b * nview + view) * d.nv + iz) * d.nu + kk;
                if (o == 1 && wx > 0.f) v += rdf(dst);  // the row pass of this view wrote first
                stf(dst, v);
            }
        }
        // every warp is done with buffer k & 1 before it is refilled
        failed = __syncthreads_or(failed);
        if (failed) break;
        if (threadIdx.x == 0 && k + 2 < K) issue(k + 2);
    }
    if (failed) {
        // chunks k and k + 1 may still be in flight: let them land (bounded) before exiting
        if (threadIdx.x == 0)
            for (int j = k; j < min(k + 2, K); ++j) mbar_wait_bounded(&s_bar[j & 1], (j >> 1) & 1);
        return;
    }
    if (unweight_par) {
        // FORCE_FBP on parallel FP: cancel the ray-length weight
        // (ReverseWeightBPParallelKernel, distanceDriven2DUtils.cu:68-94)
        for (int q = 0; q < NI; ++q) {
            int vi, m;
            fp_item(warp, q, ipv, wpv, vi, m);
            if (vi >= nvg || m >= ipv) continue;
            const int view = order[v0 + vi];
            const int kk = 31 * m + lane;
            if (lane >= 31 || kk >= d.nu) continue;
            float sn, cs;
            sincosf(deg[view], &sn, &cs);
            Tout* dst = prj + (((size_t)b * nview + view) * d.nv + iz) * d.nu + kk;
            stf(dst, rdf(dst) / (ref_y_main(deg[view]) ? g.dy / fabsf(cs) : g.dx / fabsf(sn)));
        }
    }
}

// ---------------------------------------------------------------------------
// Parallel-beam normalised back projection, fast path.
//
// For a parallel beam the detector coordinate of a pixel centre,
// jc = -((x cos + y sin)/du + off_u) + nu/2, is linear in (ix, iy) with steps
// jx = -dx cos/du and jy = -dy sin/du, and the footprint of the pixel's
// x-edges is [jc - |jx|/2, jc + |jx|/2] (of its y-edges, jc -+ |jy|/2).  The
// reference's normalised box integral (DDBPParallelKernel,
// distanceDriven2DBoxInt.cu:409-497) is then (F(e1) - F(e0)) / (e1 - e0) with
// F the running integral of the detector row, and neighbouring pixels share
// footprint edges: pixels ix and ix+1 meet at jc + jx/2.  So a thread that
// owns 4 consecutive pixels along x evaluates F at 5 edges for the x-edge
// term, and one that owns 4 consecutive pixels along y does the same for the
// y-edge term.  Each thread holds one pixel run of each kind (x-layout and
// y-layout accumulators) and the two are added through shared memory at the
// end.
//
// A CTA owns a 32x32 tile of one slice.  Per chunk of 32 views: one thread per
// view computes the view's constants in FP64 (tile-origin coordinate, steps,
// blend weights, staged window); each warp then stages, for its views, the
// window of cells the tile projects onto as a midpoint table of window-local
// running sums (small, so FP32 keeps them accurate); then every thread adds
// the views to its 8 pixels with table lookups only.  No atomics.
constexpr int kPT = 32;        // tile edge
constexpr int kPViews = 32;    // views per staged chunk
constexpr int kPMaxWin = 255;  // staged cells per view (table holds win+1 entries)

// Window tables of the fast back projectors, staged by one warp M at a time:
// for each item, entries k = 0 .. win of (running sum of the window cells
// before k + value/2, value) for the cells w0 .. w0 + win - 1 of the detector
// row at `row` (cells off the detector, and the entry past the window, are
// zero; ok = false stages zeros, valid = false writes nothing).  Lane l scans
// the PER consecutive entries from l PER of every item: it issues all M PER
// loads before it sums, so that the items' load latencies overlap, then the
// warp scans the lane sums and the lane writes its entries.
template <typename Tp>
struct WinItem {
    float2* T;
    const Tp* row;
    int w0;
    bool ok, valid;
};
// Windows a warp stages together: on the parallel 16 x 512^2, 720-view batch
// the back projection takes 1.97, 1.75 and 1.90 ms with 1, 2 and 4 (4 spills).
constexpr int kStageBatch = 2;

template <int PER, int M, typename Tp>
__device__ __forceinline__ void stage_windows_per(const WinItem<Tp> (&it)[M], int win, int nu, int lane) {
    const int k0 = lane * PER;
    float v[M][PER];
    float run[M], incl[M];
#pragma unroll
    for (int m = 0; m < M; ++m)
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int k = k0 + q, cell = it[m].w0 + k;
            v[m][q] = (it[m].ok && k < win && cell >= 0 && cell < nu) ? ldf(it[m].row + cell) : 0.f;
        }
#pragma unroll
    for (int m = 0; m < M; ++m) {
        run[m] = 0.f;
#pragma unroll
        for (int q = 0; q < PER; ++q) run[m] += v[m][q];
        incl[m] = run[m];
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const float t = __shfl_up_sync(0xffffffffu, incl[m], o);
            if (lane >= o) incl[m] += t;
        }
#pragma unroll
    for (int m = 0; m < M; ++m) {
        if (!it[m].valid) continue;
        float base = incl[m] - run[m];
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int k = k0 + q;
            if (k <= win) it[m].T[k] = make_float2(fmaf(0.5f, v[m][q], base), v[m][q]);
            base += v[m][q];
        }
    }
}

// The same for any window of up to 255 cells: PER = ceil((win + 1) / 32),
// a compile-time count, so a lane issues exactly its loads.
template <int M, typename Tp>
__device__ __forceinline__ void stage_windows(const WinItem<Tp> (&it)[M], int win, int nu, int lane) {
    switch ((win + 1 + 31) / 32) {
        case 1: stage_windows_per<1>(it, win, nu, lane); break;
        case 2: stage_windows_per<2>(it, win, nu, lane); break;
        case 3: stage_windows_per<3>(it, win, nu, lane); break;
        case 4: stage_windows_per<4>(it, win, nu, lane); break;
        case 5: stage_windows_per<5>(it, win, nu, lane); break;
        case 6: stage_windows_per<6>(it, win, nu, lane); break;
        case 7: stage_windows_per<7>(it, win, nu, lane); break;
        default: stage_windows_per<8>(it, win, nu, lane); break;
    }
}

struct ParView {
    float jb, jx, jy, sx;  // jb: window coordinate - 1/2 of the tile's first pixel centre
    float sy, jc, hx, hy;  // sx, sy: signed normalisations (0 = term inactive); jc: absolute coordinate
};

inline size_t par_fast_smem(int win, int S) {
    return (size_t)S * kPViews * (win + 1) * sizeof(float2) + kPViews * sizeof(ParView) + kPViews * sizeof(int) +
           (size_t)S * kPT * (kPT + 1) * sizeof(float);
}

// S slices of the same geometry per CTA: the per-view constants, the edge
// positions and each lookup's index and fraction are shared; only the table
// reads and the sums repeat per slice.
// Views are split over blockIdx.z in parts of vper (a multiple of kPViews)
// when the tile grid alone leaves SMs idle or fills its last wave poorly
// (bp_view_parts); part z writes its own partial volume at
// img + z * part_elems (summed by bp_parts_sum_kernel).
template <typename Tp, typename Tout, int S>
__global__ void __launch_bounds__(256) dd2d_bp_par_fast_kernel(Tout* __restrict__ img, const Tp* __restrict__ prj,
                                                               const float* __restrict__ deg, int nview, Grid g,
                                                               Det d, int fbp, int accumulate, int win,
                                                               int nslices, int vper, size_t part_elems) {
    extern __shared__ float4 smem_f4[];
    const int stride = win + 1;
    float2* s_tab = reinterpret_cast<float2*>(smem_f4);                       // [S][kPViews][stride]
    ParView* s_par = reinterpret_cast<ParView*>(s_tab + S * kPViews * stride);  // 16-byte aligned: 256 * S * stride bytes before
    int* s_w0 = reinterpret_cast<int*>(s_par + kPViews);                      // window start, INT_MIN = not staged
    float* s_acc = reinterpret_cast<float*>(s_w0 + kPViews);                  // [S][kPT][kPT + 1] merge buffer

    const int tiles_x = (g.nx + kPT - 1) / kPT;
    const int tx0 = (blockIdx.x % tiles_x) * kPT, ty0 = (blockIdx.x / tiles_x) * kPT;
    const int s0 = blockIdx.y * S;  // first slice (b * nz + iz) of this CTA
    const int ns = min(S, nslices - s0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // x-layout: 4 pixels along x; a half warp spans 16 columns x 4 rows, so its
    // table reads fall on distinct banks.  y-layout: 4 pixels along y, lane = column.
    const int xl_row = warp * 4 + ((lane >> 2) & 3);
    const int xl_col = ((lane >> 4) * 4 + (lane & 3)) * 4;
    const int yl_col = lane, yl_row = warp * 4;

    // detector row of each slice (truncation, :383); a slice off the detector stages zeros
    const Tp* rows[S];
    bool row_ok[S];
    bool any_row = false;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int slice = s0 + min(s, ns - 1), iz = slice % g.nz, b = slice / g.nz;
        const float zc = ((float)iz - g.nz / 2.f) * g.dz + g.cz + g.dz / 2;
        const int iv = (int)(zc / d.dv + d.off_v + d.nv / 2.f - 0.5f);
        row_ok[s] = s < ns && iv >= 0 && iv < d.nv;
        rows[s] = prj + ((size_t)b * nview * d.nv + (row_ok[s] ? iv : 0)) * d.nu;
        any_row |= row_ok[s];
    }
    float ax[S][4], ay[S][4];
#pragma unroll
    for (int s = 0; s < S; ++s)
#pragma unroll
        for (int k = 0; k < 4; ++k) ax[s][k] = ay[s][k] = 0.f;
    const size_t vstride = (size_t)d.nv * d.nu;
    const size_t tstride = (size_t)kPViews * stride;  // per slice

    img += blockIdx.z * part_elems;
    const int vb = blockIdx.z * vper, ve = min(nview, vb + vper);
    for (int v0 = vb; v0 < ve && any_row; v0 += kPViews) {
        const int nvc = min(kPViews, ve - v0);
        if (threadIdx.x < nvc) {
            const int vi = threadIdx.x, view = v0 + vi;
            double s, c;
            sincos((double)deg[view], &s, &c);
            const double du = d.du;
            const double jx = -c * g.dx / du, jy = -s * g.dy / du;
            const double xc0 = (tx0 + 0.5 - 0.5 * g.nx) * g.dx + g.cx;
            const double yc0 = (ty0 + 0.5 - 0.5 * g.ny) * g.dy + g.cy;
            const double j00 = -((xc0 * c + yc0 * s) / du + d.off_u) + 0.5 * d.nu;
            const double ac = fabs(c), as = fabs(s);
            const bool ya = ac > as - kDDMarginD, xa = ac < as + kDDMarginD;
            const double r = (ac - as + kDDMarginD) / (2 * kDDMarginD);
            const double wx = r < 0 ? 0.0 : (r > 1 ? 1.0 : r);
            const double hx = 0.5 * g.dx * ac / du, hy = 0.5 * g.dy * as / du;
            const double hm = fmax(ya ? hx : 0.0, xa ? hy : 0.0);
            const double pw = fbp ? 1.0 : (ref_y_main(deg[view]) ? g.dy / ac : g.dx / as);  // Utils.cu:39-65
            const double jmin = j00 + fmin(0.0, (kPT - 1) * jx) + fmin(0.0, (kPT - 1) * jy);
            const double jmax = j00 + fmax(0.0, (kPT - 1) * jx) + fmax(0.0, (kPT - 1) * jy);
            bool ok = isfinite(j00) && isfinite(hm);
            int w0 = 0;
            if (ok) {
                // two spare cells on each side: every edge lookup lands in [1.5, win - 2.5]
                w0 = (int)floor(jmin - hm) - 2;
                ok = ((int)ceil(jmax + hm) + 2 - w0) <= win;
            }
            ParView P;
            P.jb = (float)(j00 - w0 - 0.5);
            P.jx = (float)jx;
            P.jy = (float)jy;
            P.sx = ya ? (float)(pw * wx / jx) : 0.f;
            P.sy = xa ? (float)(pw * (1 - wx) / jy) : 0.f;
            P.jc = (float)j00;
            P.hx = (float)hx;
            P.hy = (float)hy;
            s_par[vi] = P;
            s_w0[vi] = ok ? w0 : INT_MIN;
        }
        __syncthreads();
        // stage (running sum + value/2, value) for window cells w0 .. w0+win-1; entry win = (total, 0)
        for (int sv0 = warp; sv0 < S * nvc; sv0 += 8 * kStageBatch) {
            WinItem<Tp> it[kStageBatch];
#pragma unroll
            for (int m = 0; m < kStageBatch; ++m) {
                const int sv = sv0 + 8 * m;
                const int s = sv / nvc, vi = sv - s * nvc;
                const Tp* srow = rows[0];
                bool rok = row_ok[0];
#pragma unroll
                for (int q = 1; q < S; ++q)
                    if (s == q) {
                        srow = rows[q];
                        rok = row_ok[q];
                    }
                it[m].valid = sv < S * nvc;
                it[m].w0 = s_w0[vi];
                it[m].ok = it[m].valid && it[m].w0 != INT_MIN && rok;
                it[m].T = s_tab + s * tstride + vi * stride;
                it[m].row = srow + (size_t)(v0 + vi) * vstride;
            }
            stage_windows(it, win, d.nu, lane);
        }
        __syncthreads();
        for (int vi = 0; vi < nvc; ++vi) {
            const ParView P = s_par[vi];
            const float2* T = s_tab + vi * stride;
            if (s_w0[vi] != INT_MIN) {
                if (P.sx != 0.f) {
                    const float e0 = fmaf((float)xl_col - 0.5f, P.jx, fmaf((float)xl_row, P.jy, P.jb));
                    float f[S][5];
#pragma unroll
                    for (int k = 0; k < 5; ++k) {
                        const float xs = fmaf((float)k, P.jx, e0);
                        const float tt = xs + kRoundMagic;
                        const int i = __float_as_int(tt) - kRoundMagicBits;
                        const float fr = xs - (tt - kRoundMagic);
#pragma unroll
                        for (int s = 0; s < S; ++s) {
                            const float2 e = T[s * tstride + i];
                            f[s][k] = fmaf(e.y, fr, e.x);
                        }
                    }
#pragma unroll
                    for (int s = 0; s < S; ++s)
#pragma unroll
                        for (int k = 0; k < 4; ++k) ax[s][k] = fmaf(f[s][k + 1] - f[s][k], P.sx, ax[s][k]);
                }
                if (P.sy != 0.f) {
                    const float e0 = fmaf((float)yl_row - 0.5f, P.jy, fmaf((float)yl_col, P.jx, P.jb));
                    float f[S][5];
#pragma unroll
                    for (int k = 0; k < 5; ++k) {
                        const float xs = fmaf((float)k, P.jy, e0);
                        const float tt = xs + kRoundMagic;
                        const int i = __float_as_int(tt) - kRoundMagicBits;
                        const float fr = xs - (tt - kRoundMagic);
#pragma unroll
                        for (int s = 0; s < S; ++s) {
                            const float2 e = T[s * tstride + i];
                            f[s][k] = fmaf(e.y, fr, e.x);
                        }
                    }
#pragma unroll
                    for (int s = 0; s < S; ++s)
#pragma unroll
                        for (int k = 0; k < 4; ++k) ay[s][k] = fmaf(f[s][k + 1] - f[s][k], P.sy, ay[s][k]);
                }
            } else {
                // window larger than the staging buffer: integrate the rows in global memory
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    if (!row_ok[s]) continue;
                    const Tp* grow = rows[s] + (size_t)(v0 + vi) * vstride;
                    if (P.sx != 0.f) {
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            float jc = P.jc + (float)(xl_col + k) * P.jx + (float)xl_row * P.jy;
                            ax[s][k] += box_line(grow, 1, jc - P.hx, jc + P.hx, d.nu) * fabsf(P.sx);
                        }
                    }
                    if (P.sy != 0.f) {
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            float jc = P.jc + (float)yl_col * P.jx + (float)(yl_row + k) * P.jy;
                            ay[s][k] += box_line(grow, 1, jc - P.hy, jc + P.hy, d.nu) * fabsf(P.sy);
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    // add the x-layout sums to the y-layout ones and store rows coalesced
#pragma unroll
    for (int s = 0; s < S; ++s)
#pragma unroll
        for (int k = 0; k < 4; ++k) s_acc[(s * kPT + xl_row) * (kPT + 1) + xl_col + k] = ax[s][k];
    __syncthreads();
    const int ix = tx0 + yl_col;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        if (s >= ns) continue;
        const int slice = s0 + s, iz = slice % g.nz, b = slice / g.nz;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            int iy = ty0 + yl_row + k;
            if (ix < g.nx && iy < g.ny) {
                Tout* o = img + (((size_t)b * g.nz + iz) * g.ny + iy) * g.nx + ix;
                float a = ay[s][k] + s_acc[(s * kPT + yl_row + k) * (kPT + 1) + yl_col];
                if (accumulate) a += rdf(o);
                stf(o, a);
            }
        }
    }
}

// Fan-beam normalised back projection (and FBP weighting), fast path.
// DDBPFanKernel (distanceDriven2DBoxInt.cu:319-396): per pixel and view, the
// pixel's x-edges at its centre row (or y-edges at its centre column, by the
// reference's intrinsic axis switch) are mapped to the detector with
// atan(rx / (ry + dso)) (distanceDriven2DUtils.cu:96-101) and the pre-weighted
// row is integrated between them and normalised by the mapped width.  Pixels
// next to each other along the switched axis share an edge point, so a thread
// owning 4 consecutive pixels along that axis maps 5 edge points, not 8: the
// x-layout of the parallel path for x-edge views, the y-layout for y-edge
// views, merged through shared memory at the end.  Same tiling and window
// tables as the parallel fast path; src is the pre-weighted sinogram (or the
// plain one in FBP mode).
struct FanView {
    float c, s;
    int w0;  // window start, INT_MIN = not staged
    int ym;  // x-edges at the centre row (1) or y-edges at the centre column (0)
};

inline size_t fan_fast_smem(int win, int S) {
    return (size_t)S * kPViews * (win + 1) * sizeof(float2) + kPViews * sizeof(FanView) +
           (size_t)S * kPT * (kPT + 1) * sizeof(float);
}

// S slices of the same geometry per CTA: the atan mappings of the edge points,
// the footprint widths, the FBP weights and each lookup's index and fraction
// are shared; only the table reads and sums repeat per slice.
template <typename Tp, typename Tout, int S>
__global__ void __launch_bounds__(256) dd2d_bp_fan_fast_kernel(Tout* __restrict__ img, const Tp* __restrict__ src,
                                                               const float* __restrict__ deg, int nview, Grid g,
                                                               Det d, float dso, int fbp, int accumulate, int win,
                                                               int nslices, int vper, size_t part_elems) {
    extern __shared__ float4 smem_f4[];
    const int stride = win + 1;
    float2* s_tab = reinterpret_cast<float2*>(smem_f4);                        // [S][kPViews][stride]
    FanView* s_view = reinterpret_cast<FanView*>(s_tab + S * kPViews * stride);
    float* s_acc = reinterpret_cast<float*>(s_view + kPViews);                 // [S][kPT][kPT + 1] merge buffer

    const int tiles_x = (g.nx + kPT - 1) / kPT;
    const int tx0 = (blockIdx.x % tiles_x) * kPT, ty0 = (blockIdx.x / tiles_x) * kPT;
    const int s0 = blockIdx.y * S;
    const int ns = min(S, nslices - s0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int xl_row = warp * 4 + ((lane >> 2) & 3);
    const int xl_col = ((lane >> 4) * 4 + (lane & 3)) * 4;
    const int yl_col = lane, yl_row = warp * 4;

    const Tp* rows[S];
    bool row_ok[S];
    bool any_row = false;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int slice = s0 + min(s, ns - 1), iz = slice % g.nz, b = slice / g.nz;
        const float zc = ((float)iz - g.nz / 2.f) * g.dz + g.cz + g.dz / 2;
        const int iv = (int)(zc / d.dv + d.off_v + d.nv / 2.f - 0.5f);
        row_ok[s] = s < ns && iv >= 0 && iv < d.nv;
        rows[s] = src + ((size_t)b * nview * d.nv + (row_ok[s] ? iv : 0)) * d.nu;
        any_row |= row_ok[s];
    }
    const size_t vstride = (size_t)d.nv * d.nu;
    const size_t tstride = (size_t)kPViews * stride;
    const float hdx = g.dx / 2.0f, hdy = g.dy / 2.0f;
    // x-layout: pixel centres (xs0 + k dx, ysx); y-layout: (xsy, ys0 + k dy)
    const float xs0 = ((float)(tx0 + xl_col) - g.nx / 2.f) * g.dx + g.cx + hdx;
    const float ysx = ((float)(ty0 + xl_row) - g.ny / 2.f) * g.dy + g.cy + hdy;
    const float xsy = ((float)(tx0 + yl_col) - g.nx / 2.f) * g.dx + g.cx + hdx;
    const float ys0 = ((float)(ty0 + yl_row) - g.ny / 2.f) * g.dy + g.cy + hdy;
    const float jscale = -1.f / d.du, joff = -d.off_u + d.nu / 2.0f;
    const float dso2 = dso * dso;
    float ax[S][4], ay[S][4];
#pragma unroll
    for (int s = 0; s < S; ++s)
#pragma unroll
        for (int k = 0; k < 4; ++k) ax[s][k] = ay[s][k] = 0.f;

    img += blockIdx.z * part_elems;
    const int vb = blockIdx.z * vper, ve = min(nview, vb + vper);
    for (int v0 = vb; v0 < ve && any_row; v0 += kPViews) {
        const int nvc = min(kPViews, ve - v0);
        if (threadIdx.x < nvc) {
            const int vi = threadIdx.x, view = v0 + vi;
            double s, c;
            sincos((double)deg[view], &s, &c);
            // window: detector coordinates of the tile's corner edges
            double xs[2] = {(tx0 - 0.5 * g.nx) * g.dx + g.cx, (tx0 + kPT - 0.5 * g.nx) * g.dx + g.cx};
            double ys[2] = {(ty0 - 0.5 * g.ny) * g.dy + g.cy, (ty0 + kPT - 0.5 * g.ny) * g.dy + g.cy};
            double jmin = 1e300, jmax = -1e300;
            bool ok = true;
            for (int a = 0; a < 2; ++a)
                for (int q = 0; q < 2; ++q) {
                    double ry = -xs[a] * s + ys[q] * c + dso;
                    if (!(ry > 0)) ok = false;
                    double j = -(atan((xs[a] * c + ys[q] * s) / ry) / d.du + (double)d.off_u) + 0.5 * d.nu;
                    jmin = fmin(jmin, j);
                    jmax = fmax(jmax, j);
                }
            int w0 = 0;
            if (ok && isfinite(jmin) && isfinite(jmax)) {
                w0 = (int)floor(jmin) - 2;
                ok = ((int)ceil(jmax) + 2 - w0) <= win;
            } else {
                ok = false;
            }
            FanView V;
            V.c = (float)c;
            V.s = (float)s;
            V.w0 = ok ? w0 : INT_MIN;
            V.ym = ref_y_main(deg[view]) ? 1 : 0;
            s_view[vi] = V;
        }
        __syncthreads();
        for (int sv0 = warp; sv0 < S * nvc; sv0 += 8 * kStageBatch) {
            WinItem<Tp> it[kStageBatch];
#pragma unroll
            for (int m = 0; m < kStageBatch; ++m) {
                const int sv = sv0 + 8 * m;
                const int s = sv / nvc, vi = sv - s * nvc;
                const Tp* srow = rows[0];
                bool rok = row_ok[0];
#pragma unroll
                for (int q = 1; q < S; ++q)
                    if (s == q) {
                        srow = rows[q];
                        rok = row_ok[q];
                    }
                it[m].valid = sv < S * nvc;
                it[m].w0 = s_view[vi].w0;
                it[m].ok = it[m].valid && it[m].w0 != INT_MIN && rok;
                it[m].T = s_tab + s * tstride + vi * stride;
                it[m].row = srow + (size_t)(v0 + vi) * vstride;
            }
            stage_windows(it, win, d.nu, lane);
        }
        __syncthreads();
        for (int vi = 0; vi < nvc; ++vi) {
            const FanView V = s_view[vi];
            const float2* T = s_tab + vi * stride;
            const float fw0 = (float)V.w0 + 0.5f;  // window origin, shifted for the midpoint tables
            // edge points p_k = p_0 + k * step, k = 0..4, rotated: (rx, ry)
            float px, py, sx, sy;
            if (V.ym) {
                px = xs0 - hdx; py = ysx; sx = g.dx; sy = 0.f;
            } else {
                px = xsy; py = ys0 - hdy; sx = 0.f; sy = g.dy;
            }
            const float rx0 = px * V.c + py * V.s, ry0 = -px * V.s + py * V.c;
            const float drx = sx * V.c + sy * V.s, dry = -sx * V.s + sy * V.c;
            float j[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                const float rx = fmaf((float)k, drx, rx0), ry = fmaf((float)k, dry, ry0);
                j[k] = fmaf(atanf(__fdividef(rx, ry + dso)), jscale, joff);  // fast divide: a few ulp
            }
            float wgt[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                wgt[k] = 1.f;
                if (fbp) {
                    const float rxc = fmaf((float)k + 0.5f, drx, rx0), ryc = fmaf((float)k + 0.5f, dry, ry0);
                    wgt[k] = __fdividef(dso2, rxc * rxc + (dso + ryc) * (dso + ryc));
                }
            }
            float val[S][4];
            if (V.w0 != INT_MIN) {
                float f[S][5];
#pragma unroll
                for (int k = 0; k < 5; ++k) {
                    const float xs = j[k] - fw0;
                    const float tt = xs + kRoundMagic;
                    const int i = __float_as_int(tt) - kRoundMagicBits;
                    const float fr = xs - (tt - kRoundMagic);
#pragma unroll
                    for (int s = 0; s < S; ++s) {
                        const float2 e = T[s * tstride + i];
                        f[s][k] = fmaf(e.y, fr, e.x);
                    }
                }
#pragma unroll
                for (int s = 0; s < S; ++s)
#pragma unroll
                    for (int k = 0; k < 4; ++k) val[s][k] = __fdividef(f[s][k + 1] - f[s][k], j[k + 1] - j[k]);
            } else {
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    const Tp* grow = rows[s] + (size_t)(v0 + vi) * vstride;
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const float lo = fminf(j[k], j[k + 1]), hi = fmaxf(j[k], j[k + 1]);
                        val[s][k] = row_ok[s] ? __fdividef(box_line(grow, 1, lo, hi, d.nu), hi - lo) : 0.f;
                    }
                }
            }
            if (V.ym) {
#pragma unroll
                for (int s = 0; s < S; ++s)
#pragma unroll
                    for (int k = 0; k < 4; ++k) ax[s][k] = fmaf(val[s][k], wgt[k], ax[s][k]);
            } else {
#pragma unroll
                for (int s = 0; s < S; ++s)
#pragma unroll
                    for (int k = 0; k < 4; ++k) ay[s][k] = fmaf(val[s][k], wgt[k], ay[s][k]);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int s = 0; s < S; ++s)
#pragma unroll
        for (int k = 0; k < 4; ++k) s_acc[(s * kPT + xl_row) * (kPT + 1) + xl_col + k] = ax[s][k];
    __syncthreads();
    const int ix = tx0 + yl_col;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        if (s >= ns) continue;
        const int slice = s0 + s, iz = slice % g.nz, b = slice / g.nz;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            int iy = ty0 + yl_row + k;
            if (ix < g.nx && iy < g.ny) {
                Tout* o = img + (((size_t)b * g.nz + iz) * g.ny + iy) * g.nx + ix;
                float a = ay[s][k] + s_acc[(s * kPT + yl_row + k) * (kPT + 1) + yl_col];
                if (accumulate) a += rdf(o);
                stf(o, a);
            }
        }
    }
}

// Staged window for the fast fan path: angular size of a 32x32 tile seen from
// the nearest source position, in cells, or 0 if it does not fit.
int fan_fast_window(const ctp_geometry& g) {
    double hx = 0.5 * g.nx * g.dx, hy = 0.5 * g.ny * g.dy;
    double rmax = sqrt((fabs(g.cx) + hx) * (fabs(g.cx) + hx) + (fabs(g.cy) + hy) * (fabs(g.cy) + hy));
    double diag = kPT * sqrt((double)g.dx * g.dx + (double)g.dy * g.dy);
    double near = (double)g.dso - rmax;
    if (near <= diag) return 0;
    double cells = 2 * atan(0.5 * diag / near) / fabs((double)g.du);
    int win = (int)ceil(cells) + 8;
    return win <= kPMaxWin ? win : 0;
}

// Staged window for the fast parallel path (cells), or 0 if it does not fit.
int par_fast_window(const ctp_geometry& g) {
    double du = fabs((double)g.du);
    double w = ((kPT - 1) * ((double)g.dx + g.dy) + fmax(g.dx, g.dy)) / du;
    int win = (int)ceil(w) + 8;
    return win <= kPMaxWin ? win : 0;
}

// Staged window (cells) needed by a 16x16 tile, from a conservative bound on
// the tile's projected size.  0 means "read the sinogram from global memory".
int window_cells(const ctp_geometry& g, int geom) {
    double diag = kTile * sqrt((double)g.dx * g.dx + (double)g.dy * g.dy);
    double cells;
    if (geom == 0) {
        double hx = 0.5 * g.nx * g.dx, hy = 0.5 * g.ny * g.dy;
        double rmax = sqrt((fabs(g.cx) + hx) * (fabs(g.cx) + hx) + (fabs(g.cy) + hy) * (fabs(g.cy) + hy));
        double near = (double)g.dso - rmax;
        if (near <= diag) return 0;
        cells = 2 * atan(0.5 * diag / near) / fabs((double)g.du);
    } else {
        cells = diag / fabs((double)g.du);
    }
    int w = (int)ceil(cells) + 8;
    return w <= kMaxWin ? w : 0;
}

template <typename T>
const T* cptr(const void* p) { return static_cast<const T*>(p); }
template <typename T>
T* mptr(void* p) { return static_cast<T*>(p); }

// Scratch of the forward projector.  Every path starts with the edge table
// and the order in which the streamed path takes the views.  The staged and
// general kernels then read the transposed image of every slice
// (fp_workspace_min).  The streamed path runs in chunks of slices: per chunk
// the transposed slices and the row and column line tables
// (fp_stream_bytes), rebuilt in the same buffer for each chunk.
size_t fp_edge_table_bytes(const ctp_geometry& g) {
    return align_up(table_floats(g.nview, g.nu) * sizeof(float)) + align_up(g.nview * sizeof(int));
}

size_t fp_workspace_min(const ctp_geometry& g) {
    return fp_edge_table_bytes(g) + align_up(g.nbatch * g.nz * g.ny * g.nx * 4);
}

size_t fp_slice_tables_bytes(const ctp_geometry& g) {
    return g.ny * line_bytes((int)g.nx) + g.nx * line_bytes((int)g.ny);
}

size_t fp_stream_bytes(const ctp_geometry& g, size_t chunk) {
    return fp_edge_table_bytes(g) + align_up(chunk * g.ny * g.nx * 4) + align_up(chunk * fp_slice_tables_bytes(g));
}

// Largest chunk of the streamed path (transposed slices and line tables,
// about 7.3 MB per 512 x 512 slice).  Measured on the 16-slice 512^2,
// 720-view batch (B200, warm caches, every launch of one call): chunks of 4
// slices stay resident in the L2 between the launches that write the
// tables and the sweep that reads them, 73 MB of DRAM traffic per call (1.4x
// the image and projections) at 3.27 ms; chunks of 8, 220 MB at 2.95 ms; one
// chunk of 16, 576 MB at 2.86 ms.  The sweep is bound by shared memory and
// instruction issue (576 MB in 2.86 ms is 3% of the HBM bandwidth), and a
// chunk's launch of 2 waves pays its tail, so the default takes large
// chunks; smaller workspaces (and ctp_set_fp_stream_slices) take smaller ones.
constexpr size_t kFPChunkBytes = (size_t)256 << 20;

// Cap on the slices per chunk (ctp_set_fp_stream_slices): negative = none,
// 0 = no streamed path.
std::atomic<int> g_fp_stream_cap{-1};

// Slices per chunk of the streamed path with `ws` bytes of scratch: the
// largest count up to the chunk limit (and the cap) whose scratch fits,
// evened out over the chunks the stack then takes; 0 if one slice does not
// fit.
int fp_stream_slices(const ctp_geometry& g, size_t ws) {
    const size_t nslices = g.nbatch * g.nz;
    const size_t per = g.ny * g.nx * 4 + fp_slice_tables_bytes(g);
    if (nslices == 0 || per == 0) return 0;
    size_t c = std::min(nslices, std::max<size_t>(1, kFPChunkBytes / per));
    const int cap = g_fp_stream_cap.load();
    if (cap >= 0) c = std::min(c, (size_t)cap);
    while (c > 0 && fp_stream_bytes(g, c) > ws) --c;
    if (c == 0) return 0;
    const size_t nchunks = (nslices + c - 1) / c;
    return (int)((nslices + nchunks - 1) / nchunks);
}

// Lines per chunk of the streamed path's two-buffer ring, or 0 if one line
// per buffer does not fit.
int fp_stream_chunk(const ctp_geometry& g) {
    size_t line = line_bytes((int)std::max(g.nx, g.ny));
    if (2 * line > 200 * 1024) return 0;
    int r = (int)((66 * 1024) / (2 * line));
    return std::max(1, std::min(r, 8));
}

// hard != 0: the branchless tracer's per-view weights (main axis alone)
int build_table(float* base, const float* deg, const ctp_geometry& g, int geom, cudaStream_t s, DDTab& tab,
                int hard = 0) {
    DDTabW w;
    carve_table(base, g.nview, g.nu, w);
    int ym = (int)(g.ny / 2), xm = (int)(g.nx / 2);
    double dsd = geom == 0 ? g.dsd : 1000.0, dso = geom == 0 ? g.dso : 500.0;
    dim3 grid((unsigned)((g.nu + 1 + 127) / 128), (unsigned)g.nview);
    dd_table_kernel<<<grid, 128, 0, s>>>(w, deg, (int)g.nview, make_grid(g), make_det(g), dsd, dso, geom, ym, xm,
                                         hard);
    tab = as_read(w, ym, xm);
    return check_launch("dd_table_kernel");
}

// The fast forward projector handles slices projected one to one onto
// detector rows (nz == nv and the z interpolation of every row landing exactly
// on its own slice, as for single-slice and matched stacks) and at most
// kFMaxItems edge groups per warp.
bool fp_fast_ok(const ctp_geometry& g, int& vgroup, int& nrows) {
    // also reached from the workspace query, before the geometry is validated
    if (g.nu == 0 || g.nview == 0 || g.nx == 0 || g.ny == 0 || g.nz == 0) return false;
    if (g.nz != g.nv) return false;
    for (size_t iv = 0; iv < g.nv; ++iv) {
        double z = ((double)iv - (g.nv - 1) / 2.0 + g.off_v) * g.dv;
        z = (z - g.cz) / g.dz + g.nz / 2.0 - 0.5;
        if (fabs(z - (double)iv) > 1e-6) return false;
    }
    int ipv = (int)((g.nu + 30) / 31);
    // views per CTA: the largest count whose edge groups fill the warps of one
    // of the compiled group counts (4, 8, 12, 16 per warp) with the least waste
    vgroup = 0;
    double best = 1e30;
    for (int v = 1; v * ipv <= kFMaxItems * 8 && v <= (int)g.nview; ++v) {
        int per_warp = (v * ipv + 7) / 8;
        int ni = per_warp <= 4 ? 4 : per_warp <= 8 ? 8 : per_warp <= 12 ? 12 : 16;
        double waste = (double)(ni * 8) / (v * ipv) + 0.05 / v;  // prefer more views per staged image
        if (waste < best) {
            best = waste;
            vgroup = v;
        }
    }
    if (vgroup < 1) return false;
    size_t line = line_bytes((int)std::max(g.nx, g.ny));
    nrows = 8;
    while (nrows > 1 && nrows * line > 110 * 1024) nrows /= 2;
    return nrows * line <= 200 * 1024;
}

// View group and edge groups per warp (one of the compiled counts, at most
// max_ni) of the streamed forward projector: the most views per CTA whose
// edge groups fill the 8 warps with the least waste.
bool fp_stream_shape(const ctp_geometry& g, int& vgroup, int& ni, int max_ni = 16) {
    static const int set[4] = {4, 8, 12, 16};
    const int ipv = (int)((g.nu + 30) / 31);
    vgroup = 0;
    ni = 0;
    if (ipv == 0 || g.nview == 0) return false;
    double best = 1e30;
    for (int v = 1; v * ipv <= max_ni * 8 && v <= (int)g.nview; ++v) {
        const int per_warp = (v * ipv + 7) / 8;
        int n = 0;
        for (int i = 0; i < 4 && !n; ++i)
            if (set[i] >= per_warp && set[i] <= max_ni) n = set[i];
        if (!n) continue;
        const double waste = (double)(n * 8) / (v * ipv) + 0.05 / v;  // prefer more views per table chunk
        if (waste < best) {
            best = waste;
            vgroup = v;
            ni = n;
        }
    }
    return vgroup > 0;
}

// Views per CTA and edge groups per warp of the fan forward projectors.
// Each of the v views of a CTA (1, 2, 4 or 8) gets 8 / v consecutive warps,
// so that a warp's edge groups share the per-line weight and the source
// coordinate (fp_item, fp_line); a view's groups take ceil(ipv v / 8) per
// warp, rounded up to a compiled count (4, 8, 12 or 16).  The kernels are
// issue-bound, so the launch's time goes as its CTAs times a CTA's groups per
// warp plus the per-line work they share (measured at about half a group on
// the 4 x 512^2, 984-view, 888-cell fan workload: 1.85, 1.81 and 1.75 ms for
// 1, 2 and 4 views per CTA); the cheapest shape wins, the larger view group
// on a tie (fewer copies of the slice's tables), among those that keep at
// least two CTAs per SM.  False if one view does not fit 16 groups per warp
// (detectors of more than 128 groups of 31 cells).
bool fan_shape(const ctp_geometry& g, int nslices, int sms, int& vgroup, int& ni) {
    const int ipv = (int)((g.nu + 30) / 31);
    vgroup = 0;
    ni = 0;
    if (ipv == 0 || g.nview == 0 || nslices <= 0) return false;
    long long best = -1;
    for (int v = 1; v <= 8 && v <= (int)g.nview; v *= 2) {
        const int per_warp = (ipv * v + 7) / 8;
        const int n = per_warp <= 4 ? 4 : per_warp <= 8 ? 8 : per_warp <= 12 ? 12 : per_warp <= 16 ? 16 : 0;
        if (!n) continue;
        const long long units = (long long)((g.nview + v - 1) / v) * nslices;
        if (v > 1 && units < 2LL * std::max(sms, 1)) break;
        const long long cost = units * (2 * n + 1);
        if (best < 0 || cost <= best) {
            best = cost;
            vgroup = v;
            ni = n;
        }
    }
    return vgroup > 0;
}

template <typename Tin, typename Tout>
int launch_fp(void* prj, const void* img, const float* deg, const ctp_geometry& g, int geom, int type,
              unsigned flags, char* ws, size_t ws_bytes, cudaStream_t s) {
    DDTab tab;
    int rc = build_table(reinterpret_cast<float*>(ws), deg, g, geom, s, tab, (type & CTP_TYPE_BRANCHLESS) ? 1 : 0);
    if (rc) return rc;
    Tin* imgT = reinterpret_cast<Tin*>(ws + fp_edge_table_bytes(g));
    const size_t slice_px = g.ny * g.nx;
    auto transpose = [&](const Tin* from, int nsl) {
        dim3 tg((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 31) / 32), (unsigned)nsl);
        transpose_kernel<Tin><<<tg, dim3(32, 8), 0, s>>>(imgT, from, (int)g.nx, (int)g.ny);
        return check_launch("transpose_kernel");
    };
    int unweight = (geom == 1) && (type & CTP_TYPE_FORCE_FBP);
    int vgroup = 0, nrows = 0;
    const int rchunk = fp_stream_chunk(g);
    const int nslices = (int)(g.nbatch * g.nz);
    // the streamed path is the faster one from a single slice up (the tables
    // are built once per slice instead of once per view group); it runs in
    // chunks of slices sized to the workspace (fp_stream_slices), and a
    // workspace without room for one slice's tables runs the staged kernel
    const bool fast = fp_fast_ok(g, vgroup, nrows);
    const int chunk = fast && rchunk > 0 ? fp_stream_slices(g, ws_bytes) : 0;
    // views per CTA and edge groups per warp, for the slices of one launch
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int launch_slices = chunk > 0 ? chunk : nslices;
    int sv = 0, ni = 0;
    const bool shaped = fast && (geom == 0 ? fan_shape(g, launch_slices, sms, sv, ni)
                                           : fp_stream_shape(g, sv, ni, kFMaxItems));
    if (shaped && chunk > 0) {
        // streamed path: per chunk, the line tables of rows (from the image)
        // and columns (from its transpose), then the sweep
        unsigned char* lt0 =
            reinterpret_cast<unsigned char*>(ws + fp_edge_table_bytes(g) + align_up(chunk * slice_px * 4));
        unsigned char* lt1 = lt0 + (size_t)chunk * g.ny * line_bytes((int)g.nx);
        // warps per CTA: as many as 96 KB of shared memory holds (at least one)
        const size_t wb = line_tables_warp_bytes((int)std::max(g.nx, g.ny));
        const int lt_warps = (int)std::max<size_t>(1, std::min<size_t>(8, (96 * 1024) / wb));
        const size_t lt_shm = (size_t)lt_warps * wb;
        cudaFuncSetAttribute(line_tables_kernel<Tin>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lt_shm);
        // one slice per CTA (sharing the edge work across two slices halves the
        // lines per table chunk, and the warps then wait on the copies instead)
        if (geom != 0) {
            // a grid short of one wave of resident CTAs (few slices) takes
            // smaller view groups: more CTAs, each streaming the slice's tables
            for (int cap = 8; cap >= 4 && ((g.nview + sv - 1) / sv) * (size_t)chunk < 2 * (size_t)sms; cap /= 2) {
                int sv2 = 0, ni2 = 0;
                if (!fp_stream_shape(g, sv2, ni2, cap)) break;
                sv = sv2;
                ni = ni2;
            }
        }
        const int rc_s = rchunk;
        size_t shm = 2 * (size_t)rc_s * line_bytes((int)std::max(g.nx, g.ny));
        const bool fan = geom == 0;
        const int wpv = fan ? 8 / sv : 0;  // fan beams: warps per view (fp_item)
        int* order = reinterpret_cast<int*>(ws + align_up(table_floats(g.nview, g.nu) * sizeof(float)));
        blend_first_kernel<<<1, 1024, 0, s>>>(order, tab.wx, (int)g.nview);
        if ((rc = check_launch("blend_first_kernel"))) return rc;
        for (int s0 = 0; s0 < nslices; s0 += chunk) {
            const int cs = std::min(chunk, nslices - s0);
            const Tin* from = cptr<Tin>(img) + (size_t)s0 * slice_px;
            if ((rc = transpose(from, cs))) return rc;
            const long long rows = (long long)cs * g.ny, cols = (long long)cs * g.nx;
            const unsigned rgrid = (unsigned)std::min<long long>((rows + lt_warps - 1) / lt_warps, 148 * 8);
            const unsigned cgrid = (unsigned)std::min<long long>((cols + lt_warps - 1) / lt_warps, 148 * 8);
            line_tables_kernel<Tin><<<rgrid, 32 * lt_warps, lt_shm, s>>>(lt0, from, rows, (int)g.nx);
            line_tables_kernel<Tin><<<cgrid, 32 * lt_warps, lt_shm, s>>>(lt1, imgT, cols, (int)g.ny);
            if ((rc = check_launch("line_tables_kernel"))) return rc;
            // slices along x, view groups along y: CTAs are dispatched view
            // group by view group, the blend band's first
            dim3 fg((unsigned)cs, (unsigned)((g.nview + sv - 1) / sv));
            auto launch = [&](auto kern) {
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
                cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
                kern<<<fg, 256, shm, s>>>(mptr<Tout>(prj), lt0, lt1, tab, make_grid(g), make_det(g), (int)g.nview,
                                          sv, wpv, rc_s, s0, order, deg, unweight);
            };
#define CTP_FP_STREAM(NI_)                                                       \
    if (fan) launch(dd2d_fp_stream_kernel<true, NI_, Tout>);                     \
    else launch(dd2d_fp_stream_kernel<false, NI_, Tout>)
            if (ni == 4) { CTP_FP_STREAM(4); }
            else if (ni == 8) { CTP_FP_STREAM(8); }
            else if (ni == 12) { CTP_FP_STREAM(12); }
            else { CTP_FP_STREAM(16); }
#undef CTP_FP_STREAM
            if ((rc = check_launch("dd2d_fp_stream_kernel"))) return rc;
        }
        return CTP_OK;
    }
    // the staged and general kernels read the transposed image of every slice
    if (ws_bytes < fp_workspace_min(g))
        return set_error(CTP_ERR_INVALID_ARGUMENT, "dd2d_fp: workspace of %zu bytes, the kernel needs %zu", ws_bytes,
                         fp_workspace_min(g));
    if ((rc = transpose(cptr<Tin>(img), nslices))) return rc;
    if (shaped) {
        size_t shm = (size_t)nrows * line_bytes((int)std::max(g.nx, g.ny));
        dim3 fg((unsigned)((g.nview + sv - 1) / sv), (unsigned)(g.nbatch * g.nz));
        const bool fan = geom == 0;
        const int wpv = fan ? 8 / sv : 0;  // fan beams: warps per view (fp_item)
        auto launch = [&](auto kern) {
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
            cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
            kern<<<fg, 256, shm, s>>>(mptr<Tout>(prj), cptr<Tin>(img), imgT, tab, make_grid(g), make_det(g),
                                      (int)g.nview, sv, wpv, nrows, deg, unweight);
        };
#define CTP_FP_STAGED(NI_)                                                       \
    if (fan) launch(dd2d_fp_fast_kernel<true, NI_, Tin, Tout>);                  \
    else launch(dd2d_fp_fast_kernel<false, NI_, Tin, Tout>)
        if (ni == 4) { CTP_FP_STAGED(4); }
        else if (ni == 8) { CTP_FP_STAGED(8); }
        else if (ni == 12) { CTP_FP_STAGED(12); }
        else { CTP_FP_STAGED(16); }
#undef CTP_FP_STAGED
        return check_launch("dd2d_fp_fast_kernel");
    }
    dim3 grid((unsigned)((g.nu + kFPThreads - 1) / kFPThreads), (unsigned)g.nview, (unsigned)(g.nbatch * g.nv));
    dd2d_fp_kernel<Tin, Tout, false><<<grid, kFPThreads, 0, s>>>(
        mptr<Tout>(prj), cptr<Tin>(img), imgT, tab, make_grid(g), make_det(g), (int)g.nview, deg, unweight,
        (flags & CTP_FLAG_ZERO_OUT) ? 0 : 0, nullptr);
    return check_launch("dd2d_fp_kernel");
}

}  // namespace

// ------------------------------------------------------------------ launchers
namespace {
// The streamed forward projector applies (slices projected one to one onto
// detector rows, at most 128 edge groups per view, a line table pair fits
// the shared-memory ring).
bool fp_streamable(const ctp_geometry& g) {
    int vgroup = 0, nrows = 0;
    return fp_fast_ok(g, vgroup, nrows) && fp_stream_chunk(g) > 0 && (g.nu + 30) / 31 <= 8 * kFMaxItems;
}

// The least workspace a caller may pass: one slice per chunk of the streamed
// path where it applies, else the staged and general kernels' minimum.
size_t fp_workspace_least(const ctp_geometry& g) {
    return fp_streamable(g) && g_fp_stream_cap.load() != 0 ? std::min(fp_workspace_min(g), fp_stream_bytes(g, 1))
                                                            : fp_workspace_min(g);
}
}  // namespace

void set_fp_stream_cap(int max_slices) { g_fp_stream_cap.store(max_slices < 0 ? -1 : max_slices); }

// The workspace of the fastest path: the streamed one in its largest chunks.
size_t dd2d_fp_workspace(const ctp_geometry& g, int, int, unsigned) {
    const int c = fp_streamable(g) ? fp_stream_slices(g, SIZE_MAX) : 0;
    return c > 0 ? fp_stream_bytes(g, (size_t)c) : fp_workspace_min(g);
}

int dd2d_fp(void* prj, const void* img, const float* deg, const ctp_geometry& g, int geom, int type,
            unsigned flags, void* workspace, size_t workspace_bytes, cudaStream_t s) {
    if (geom != 0 && geom != 1) return set_error(CTP_ERR_INVALID_ARGUMENT, "geom must be 0 (fan) or 1 (parallel)");
    Scratch scr;
    // a caller's workspace runs the streamed path in chunks of as many slices
    // as it holds (the staged kernel if not one), scratch taken here the
    // largest chunks of the workspace query
    const size_t full = dd2d_fp_workspace(g, geom, type, flags);
    const size_t have = workspace ? workspace_bytes : full;
    int rc = scr.acquire(workspace, workspace_bytes, workspace ? fp_workspace_least(g) : full, s);
    if (rc) return rc;
    bool in16 = flags & (CTP_FLAG_IN_BF16 | CTP_FLAG_IN_FP16);
    bool out16 = flags & (CTP_FLAG_OUT_BF16 | CTP_FLAG_OUT_FP16);
    if (!in16 && !out16) return launch_fp<float, float>(prj, img, deg, g, geom, type, flags, scr.base(), have, s);
    if ((flags & CTP_FLAG_IN_BF16) && (flags & CTP_FLAG_OUT_BF16))
        return launch_fp<__nv_bfloat16, __nv_bfloat16>(prj, img, deg, g, geom, type, flags, scr.base(), have, s);
    if ((flags & CTP_FLAG_IN_FP16) && (flags & CTP_FLAG_OUT_FP16))
        return launch_fp<__half, __half>(prj, img, deg, g, geom, type, flags, scr.base(), have, s);
    if ((flags & CTP_FLAG_IN_BF16) && !out16)
        return launch_fp<__nv_bfloat16, float>(prj, img, deg, g, geom, type, flags, scr.base(), have, s);
    if ((flags & CTP_FLAG_IN_FP16) && !out16)
        return launch_fp<__half, float>(prj, img, deg, g, geom, type, flags, scr.base(), have, s);
    return set_error(CTP_ERR_UNSUPPORTED, "dd2d_fp: unsupported storage type combination (flags 0x%x)", flags);
}

int dd2d_nnz(unsigned long long* nnz_host, const float* deg, const ctp_geometry& g, int geom, cudaStream_t s) {
    if (!nnz_host) return set_error(CTP_ERR_INVALID_ARGUMENT, "nnz output pointer is null");
    Scratch scr;
    size_t need = align_up(table_floats(g.nview, g.nu) * sizeof(float)) + 256;
    int rc = scr.acquire(nullptr, 0, need, s);
    if (rc) return rc;
    DDTab tab;
    if ((rc = build_table(reinterpret_cast<float*>(scr.base()), deg, g, geom, s, tab))) return rc;
    unsigned long long* cnt =
        reinterpret_cast<unsigned long long*>(scr.base() + align_up(table_floats(g.nview, g.nu) * sizeof(float)));
    cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s);
    dim3 grid((unsigned)((g.nu + kFPThreads - 1) / kFPThreads), (unsigned)g.nview, (unsigned)g.nv);
    dd2d_fp_kernel<float, float, true><<<grid, kFPThreads, 0, s>>>(nullptr, nullptr, nullptr, tab, make_grid(g),
                                                                    make_det(g), (int)g.nview, deg, 0, 0, cnt);
    if ((rc = check_launch("dd2d_fp_kernel<count>"))) return rc;
    cudaError_t e = cudaMemcpyAsync(nnz_host, cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_error((int)e, "dd2d_nnz: %s", cudaGetErrorString(e));
    return CTP_OK;
}

namespace {

// Sum of the view parts of a split back projection into the output.
template <typename Tout>
__global__ void bp_parts_sum_kernel(Tout* __restrict__ img, const float* __restrict__ parts, int nparts,
                                    size_t elems, int accumulate) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < elems; i += (size_t)gridDim.x * blockDim.x) {
        float a = accumulate ? rdf(img + i) : 0.f;
        for (int q = 0; q < nparts; ++q) a += parts[(size_t)q * elems + i];
        stf(img + i, a);
    }
}

// View parts of a fast back projection whose grid (ctas) leaves SMs idle:
// enough parts of whole kPViews chunks (at most 8) for about two CTAs per SM.
// vper receives the views per part.
int bp_view_parts(size_t ctas, int nview, int& vper) {
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int chunks = (nview + kPViews - 1) / kPViews;
    if (chunks <= 0) {
        vper = kPViews;
        return 1;
    }
    int parts = 1;
    if (ctas > 0 && ctas < (size_t)sms) {
        parts = (int)std::min<size_t>(8, (2 * (size_t)sms + ctas - 1) / ctas);
    } else if (ctas >= 2 * (size_t)sms && ctas < 6 * (size_t)sms) {
        // A grid of one to three waves of equal CTAs (2 resident per SM: the
        // fast kernels' registers and shared memory) whose last wave is far
        // from full leaves SMs idle at the end: split the views into the
        // parts (up to 8) that fill the waves best, summed by one more pass
        // over the output.  Measured: the 4-slice 512^2 fan batch (512 CTAs,
        // 1.7 waves) 1.60 -> 1.39 ms with 4 parts; the 16-slice parallel
        // batch (1024 CTAs, 3.5 waves, whose tail is already spread over the
        // SMs) unchanged with 2.
        const double slots = 2.0 * sms;
        auto fill = [&](int p) {
            const double waves = (double)ctas * p / slots;
            return waves / std::ceil(waves);
        };
        if (fill(1) < 0.95)
            for (int p = 2; p <= 8; ++p)
                if (fill(p) > fill(parts) + 0.02) parts = p;
    }
    parts = std::max(1, std::min(parts, chunks));
    vper = ((chunks + parts - 1) / parts) * kPViews;
    return (nview + vper - 1) / vper;
}

// CTAs of the fast back-projection grid (0 when the fast path does not apply).
size_t bp_fast_ctas(const ctp_geometry& g, int geom) {
    const size_t nslices = g.nbatch * g.nz;
    const size_t tiles = ((g.nx + kPT - 1) / kPT) * ((g.ny + kPT - 1) / kPT);
    if (geom == 0) {
        if (fan_fast_window(g) <= 0) return 0;
        return tiles * ((nslices + (nslices >= 2 ? 1 : 0)) / (nslices >= 2 ? 2 : 1));
    }
    if (par_fast_window(g) <= 0) return 0;
    const size_t S = nslices >= 4 ? 4 : nslices >= 2 ? 2 : 1;
    return tiles * ((nslices + S - 1) / S);
}

size_t bp_pre_bytes(const ctp_geometry& g, int geom, int type) {
    bool fbp = type & (CTP_TYPE_FBP | CTP_TYPE_FORCE_FBP);
    return (geom == 0 && !fbp) ? align_up(g.nbatch * g.nview * g.nv * g.nu * sizeof(float)) : 0;
}

size_t bp_workspace(const ctp_geometry& g, int geom, int type, unsigned flags) {
    if (flags & CTP_FLAG_ADJOINT) return align_up(table_floats(g.nview, g.nu) * sizeof(float));
    size_t need = bp_pre_bytes(g, geom, type);
    const size_t ctas = bp_fast_ctas(g, geom);
    int vper = 0;
    const int parts = ctas ? bp_view_parts(ctas, (int)g.nview, vper) : 1;
    if (parts > 1) need += align_up((size_t)parts * g.nbatch * g.nz * g.ny * g.nx * sizeof(float));
    return need;
}

template <typename Tin, typename Tout>
int launch_bp(void* img, const void* prj, const float* deg, const ctp_geometry& g, int geom, int type,
              unsigned flags, char* ws, cudaStream_t s) {
    Grid gr = make_grid(g);
    Det dt = make_det(g);
    int nview = (int)g.nview;
    float dso = geom == 0 ? g.dso : 500.0f;
    int accumulate = (flags & CTP_FLAG_ZERO_OUT) ? 0 : 1;
    int tiles = (int)(((g.nx + kTile - 1) / kTile) * ((g.ny + kTile - 1) / kTile));
    dim3 grid((unsigned)tiles, (unsigned)(g.nbatch * g.nz));
    int win = window_cells(g, geom);
    int wl = win > 0 ? win : 1;
    int rc;
    if (flags & CTP_FLAG_ADJOINT) {
        DDTab tab;
        if ((rc = build_table(reinterpret_cast<float*>(ws), deg, g, geom, s, tab))) return rc;
        int per_v = wl + 2 * (2 * (wl + 1) + wl);
        size_t shm = (size_t)kAdjViews * per_v * 4 + kAdjViews * 5 * 4;
        if (geom == 0) {
            auto k = dd2d_bp_adjoint_kernel<true, Tin, Tout>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
            k<<<grid, kTile * kTile, shm, s>>>(mptr<Tout>(img), cptr<Tin>(prj), deg, tab, nview, gr, dt, dso,
                                               accumulate, win > 0 ? win : 0);
        } else {
            auto k = dd2d_bp_adjoint_kernel<false, Tin, Tout>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
            k<<<grid, kTile * kTile, shm, s>>>(mptr<Tout>(img), cptr<Tin>(prj), deg, tab, nview, gr, dt, dso,
                                               accumulate, win > 0 ? win : 0);
        }
        return check_launch("dd2d_bp_adjoint_kernel");
    }
    int fbp = (type & (CTP_TYPE_FBP | CTP_TYPE_FORCE_FBP)) ? 1 : 0;
    // branchless: the same operator as the box integral for a fan beam with
    // one detector row; otherwise the general kernel in its branchless mode
    const int bl = (type & CTP_TYPE_BRANCHLESS) ? 1 : 0;
    size_t shm = (size_t)kBPViews * wl * 4 + kBPViews * 5 * 4;
    if (geom == 0) {
        int fwin = (bl && g.nv > 1) ? 0 : fan_fast_window(g);
        int tiles_f = (int)(((g.nx + kPT - 1) / kPT) * ((g.ny + kPT - 1) / kPT));
        // two slices per CTA for stacks (shared edge mappings), one otherwise
        const int nslices = (int)(g.nbatch * g.nz);
        const int FS = nslices >= 2 ? 2 : 1;
        size_t fshm = fan_fast_smem(fwin, FS);
        // few tiles and slices: the views split into parts summed at the end
        int vper = nview;
        const int parts = fwin > 0 ? bp_view_parts(bp_fast_ctas(g, 0), nview, vper) : 1;
        const size_t elems = g.nbatch * g.nz * g.ny * g.nx;
        float* partial = reinterpret_cast<float*>(ws + bp_pre_bytes(g, geom, type));
        dim3 fgrid((unsigned)tiles_f, (unsigned)((nslices + FS - 1) / FS), (unsigned)parts);
        auto fan_fast = [&](auto k1, auto k2, auto kp1, auto kp2, const auto* srcp, int fbp_mode) {
            if (parts == 1) {
                auto k = FS == 2 ? k2 : k1;
                cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fshm);
                k<<<fgrid, 256, fshm, s>>>(mptr<Tout>(img), srcp, deg, nview, gr, dt, dso, fbp_mode, accumulate, fwin,
                                           nslices, nview, (size_t)0);
                return check_launch("dd2d_bp_fan_fast_kernel");
            }
            auto k = FS == 2 ? kp2 : kp1;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fshm);
            k<<<fgrid, 256, fshm, s>>>(partial, srcp, deg, nview, gr, dt, dso, fbp_mode, 0, fwin, nslices, vper,
                                       elems);
            int r = check_launch("dd2d_bp_fan_fast_kernel");
            if (r) return r;
            bp_parts_sum_kernel<Tout><<<(unsigned)std::min<size_t>((elems + 255) / 256, 148 * 8), 256, 0, s>>>(
                mptr<Tout>(img), partial, parts, elems, accumulate);
            return check_launch("bp_parts_sum_kernel");
        };
        if (fwin > 0 && !fbp) {
            float* wprj = reinterpret_cast<float*>(ws);
            size_t total = g.nbatch * g.nview * g.nv * g.nu;
            fan_preweight_kernel<Tin><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(wprj, cptr<Tin>(prj), deg,
                                                                                    nview, dt, gr, total);
            if ((rc = check_launch("fan_preweight_kernel"))) return rc;
            return fan_fast(dd2d_bp_fan_fast_kernel<float, Tout, 1>, dd2d_bp_fan_fast_kernel<float, Tout, 2>,
                            dd2d_bp_fan_fast_kernel<float, float, 1>, dd2d_bp_fan_fast_kernel<float, float, 2>,
                            (const float*)wprj, 0);
        }
        if (fwin > 0)
            return fan_fast(dd2d_bp_fan_fast_kernel<Tin, Tout, 1>, dd2d_bp_fan_fast_kernel<Tin, Tout, 2>,
                            dd2d_bp_fan_fast_kernel<Tin, float, 1>, dd2d_bp_fan_fast_kernel<Tin, float, 2>,
                            cptr<Tin>(prj), 1);
        if (!fbp) {
            float* wprj = reinterpret_cast<float*>(ws);
            size_t total = g.nbatch * g.nview * g.nv * g.nu;
            fan_preweight_kernel<Tin><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(wprj, cptr<Tin>(prj), deg,
                                                                                    nview, dt, gr, total);
            if ((rc = check_launch("fan_preweight_kernel"))) return rc;
            auto k = dd2d_bp_parity_kernel<true, float, Tout>;
            k<<<grid, kTile * kTile, shm, s>>>(mptr<Tout>(img), wprj, deg, nview, gr, dt, dso, 0, accumulate,
                                               win > 0 ? win : 0, bl);
        } else {
            auto k = dd2d_bp_parity_kernel<true, Tin, Tout>;
            k<<<grid, kTile * kTile, shm, s>>>(mptr<Tout>(img), cptr<Tin>(prj), deg, nview, gr, dt, dso, 1,
                                               accumulate, win > 0 ? win : 0, bl);
        }
    } else {
        int pwin = bl ? 0 : par_fast_window(g);
        if (pwin > 0) {
            int tiles_p = (int)(((g.nx + kPT - 1) / kPT) * ((g.ny + kPT - 1) / kPT));
            // slices per CTA for stacks (shared per-view work): 4, 2 or 1
            const int nslices = (int)(g.nbatch * g.nz);
            const int S = nslices >= 4 ? 4 : nslices >= 2 ? 2 : 1;
            size_t pshm = par_fast_smem(pwin, S);
            // few tiles and slices: the views split into parts summed at the end
            int vper = nview;
            const int parts = bp_view_parts(bp_fast_ctas(g, 1), nview, vper);
            const size_t elems = g.nbatch * g.nz * g.ny * g.nx;
            float* partial = reinterpret_cast<float*>(ws + bp_pre_bytes(g, geom, type));
            dim3 pg((unsigned)tiles_p, (unsigned)((nslices + S - 1) / S), (unsigned)parts);
            auto par_fast = [&](auto kout, auto kpart) {
                if (parts == 1) {
                    cudaFuncSetAttribute(kout, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pshm);
                    kout<<<pg, 256, pshm, s>>>(mptr<Tout>(img), cptr<Tin>(prj), deg, nview, gr, dt, fbp, accumulate,
                                               pwin, nslices, nview, (size_t)0);
                    return check_launch("dd2d_bp_par_fast_kernel");
                }
                cudaFuncSetAttribute(kpart, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pshm);
                kpart<<<pg, 256, pshm, s>>>(partial, cptr<Tin>(prj), deg, nview, gr, dt, fbp, 0, pwin, nslices, vper,
                                            elems);
                int r = check_launch("dd2d_bp_par_fast_kernel");
                if (r) return r;
                bp_parts_sum_kernel<Tout><<<(unsigned)std::min<size_t>((elems + 255) / 256, 148 * 8), 256, 0, s>>>(
                    mptr<Tout>(img), partial, parts, elems, accumulate);
                return check_launch("bp_parts_sum_kernel");
            };
            if (S == 4) return par_fast(dd2d_bp_par_fast_kernel<Tin, Tout, 4>, dd2d_bp_par_fast_kernel<Tin, float, 4>);
            if (S == 2) return par_fast(dd2d_bp_par_fast_kernel<Tin, Tout, 2>, dd2d_bp_par_fast_kernel<Tin, float, 2>);
            return par_fast(dd2d_bp_par_fast_kernel<Tin, Tout, 1>, dd2d_bp_par_fast_kernel<Tin, float, 1>);
        }
        auto k = dd2d_bp_parity_kernel<false, Tin, Tout>;
        k<<<grid, kTile * kTile, shm, s>>>(mptr<Tout>(img), cptr<Tin>(prj), deg, nview, gr, dt, dso, fbp,
                                           accumulate, win > 0 ? win : 0, bl);
    }
    return check_launch("dd2d_bp_parity_kernel");
}

}  // namespace

size_t dd2d_bp_workspace(const ctp_geometry& g, int geom, int type, unsigned flags) {
    return bp_workspace(g, geom, type, flags);
}

int dd2d_bp(void* img, const void* prj, const float* deg, const ctp_geometry& g, int geom, int type,
            unsigned flags, void* workspace, size_t workspace_bytes, cudaStream_t s) {
    if (geom != 0 && geom != 1) return set_error(CTP_ERR_INVALID_ARGUMENT, "geom must be 0 (fan) or 1 (parallel)");
    Scratch scr;
    size_t need = bp_workspace(g, geom, type, flags);
    int rc = scr.acquire(workspace, workspace_bytes, need, s);
    if (rc) return rc;
    bool in16 = flags & (CTP_FLAG_IN_BF16 | CTP_FLAG_IN_FP16);
    bool out16 = flags & (CTP_FLAG_OUT_BF16 | CTP_FLAG_OUT_FP16);
    if (!in16 && !out16) return launch_bp<float, float>(img, prj, deg, g, geom, type, flags, scr.base(), s);
    if ((flags & CTP_FLAG_IN_BF16) && (flags & CTP_FLAG_OUT_BF16))
        return launch_bp<__nv_bfloat16, __nv_bfloat16>(img, prj, deg, g, geom, type, flags, scr.base(), s);
    if ((flags & CTP_FLAG_IN_FP16) && (flags & CTP_FLAG_OUT_FP16))
        return launch_bp<__half, __half>(img, prj, deg, g, geom, type, flags, scr.base(), s);
    if ((flags & CTP_FLAG_IN_BF16) && !out16)
        return launch_bp<__nv_bfloat16, float>(img, prj, deg, g, geom, type, flags, scr.base(), s);
    if ((flags & CTP_FLAG_IN_FP16) && !out16)
        return launch_bp<__half, float>(img, prj, deg, g, geom, type, flags, scr.base(), s);
    return set_error(CTP_ERR_UNSUPPORTED, "dd2d_bp: unsupported storage type combination (flags 0x%x)", flags);
}

// ---------------------------------------------------------------------------
// Forward projection without any allocation.
//
// Some callers cannot allocate device memory at call time: a process whose GPU
// memory is owned by another allocator (frameworks that reserve most of the
// device at start-up, so a cudaMalloc from inside their custom ops fails or
// fragments their pool), or an acquisition/reconstruction service that
// forbids allocation once it is running.  For them, this variant of the DD
// forward projector takes its scratch (the edge table and the transposed
// image) from a fixed array in the library's device memory instead of the
// caller's workspace or the stream-ordered pool.  Every GPU that loads the
// library holds the array until the process exits.  All calls on a device
// share it, so calls that overlap on that GPU (for example from two streams)
// race and must be ordered by the caller; nothing in it needs to start at
// zero, because every call rewrites all the scratch it reads.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB

static __device__ __align__(256) unsigned char g_fp_scratch[kNoAllocScratchBytes];

// Device address of g_fp_scratch on the current device (the host-side symbol
// is only a stand-in, not a device address).  Looked up on every call: the
// lookup allocates nothing, and a cached address would go stale if the
// device were reset and the module loaded again.
static int fp_scratch_address(void** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_fp_scratch);
    if (e != cudaSuccess) return set_error((int)e, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    *out = p;
    return CTP_OK;
}

int dd2d_fp_noalloc(void* prj, const void* img, const float* deg, const ctp_geometry& g, int geom, int type,
                    unsigned flags, cudaStream_t s) {
    size_t need = fp_workspace_least(g);
    if (need > kNoAllocScratchBytes)
        return set_error(CTP_ERR_TOO_LARGE,
                         "ctp_dd2d_fp_noalloc needs %zu bytes of scratch; its fixed buffer holds %zu "
                         "(use ctp_dd2d_fp with a workspace)",
                         need, kNoAllocScratchBytes);
    void* scratch = nullptr;
    int rc = fp_scratch_address(&scratch);
    if (rc) return rc;
    return dd2d_fp(prj, img, deg, g, geom, type, flags, scratch, kNoAllocScratchBytes, s);
}

size_t dd2d_fp_noalloc_capacity() { return kNoAllocScratchBytes; }

int set_first_wait_polls(unsigned polls) {
    cudaError_t e = cudaMemcpyToSymbol(g_first_wait_polls, &polls, sizeof(unsigned));
    if (e != cudaSuccess) return set_error((int)e, "setting the wait limit: %s", cudaGetErrorString(e));
    return CTP_OK;
}

int wait_timeouts(unsigned* count) {
    if (!count) return set_error(CTP_ERR_INVALID_ARGUMENT, "count pointer is null");
    cudaError_t e = cudaMemcpyFromSymbol(count, g_wait_timeouts, sizeof(unsigned));
    if (e != cudaSuccess) return set_error((int)e, "reading the wait-timeout counter: %s", cudaGetErrorString(e));
    return CTP_OK;
}

}  // namespace ctp
