/*
 * ctp_oracle.c -- CPU FP64 restatement of the CTProjector projector pair.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the parity tests,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py check the CUDA
 * product against.  Nothing in ctprojector_b200 links, loads or calls it.
 *
 * Every function restates one reference kernel in double precision and cites
 * the reference file:line it follows.  Paths are relative to
 * src/ct_projector/kernel/projector/cuda/ in wudufan/CTProjector.
 *
 * Conventions (projector.h:7-28, 64-97):
 *   image    [batch][nz][ny][nx], image coordinates put the corner of pixel 0
 *            at the origin: X = (x - cx)/dx + nx/2.
 *   sinogram [batch][nview][nv][nu].
 * Trigonometry is evaluated exactly in double, not with fast intrinsics.
 *
 * OpenMP parallelises over rays (forward projectors) and pixel rows
 * (back projectors).  Scatter-style transposes parallelise over views with
 * a private accumulator per thread and a fixed-order reduction, so results
 * do not depend on the thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define DD_MARGIN 0.12 /* distanceDriven2DBoxInt.cu:18 */
#define SIDDON_EPS 1e-6 /* siddon.cu:35 */

typedef struct {
    long nx, ny, nz;
    double dx, dy, dz, cx, cy, cz;
} og_grid;

typedef struct {
    long nu, nv;
    double du, dv, off_u, off_v;
} og_det;

static inline double clampd(double x, double lo, double hi) /* cudaMath.cu:164 */
{
    return x < lo ? lo : (x > hi ? hi : x);
}

static inline long clampi(long x, long lo, long end) /* cudaMath.cu:182, [lo, end) */
{
    return x < lo ? lo : (x >= end ? end - 1 : x);
}

/* Exact integral of a piecewise-constant line of n cells (stride s) over
 * [x1, x2] after clamping both ends to [0, n].  cudaMath.cu:533-565
 * (IntegralBoxX / IntegralBoxY: pixel sum minus the two partial edges). */
static double box1d(const double* p, long s, double x1, double x2, long n)
{
    x1 = clampd(x1, 0, (double)n);
    x2 = clampd(x2, 0, (double)n);
    if (x2 <= x1) return 0;
    long i1 = clampi((long)x1, 0, n);
    long i2 = clampi((long)x2, 0, n);
    double v = 0;
    for (long i = i1; i <= i2; i++) v += p[i * s];
    v -= p[i1 * s] * (x1 - i1);
    v -= p[i2 * s] * (i2 + 1 - x2);
    return v;
}

/* Exact integral over the clamped rectangle [x1,x2]x[y1,y2] of an (ny, nx)
 * plane.  cudaMath.cu:336-404 (IntegralBoxXY, inclusion-exclusion). */
static double box2d(const double* p, double x1, double y1, double x2, double y2, long nx, long ny)
{
    x1 = clampd(x1, 0, (double)nx);
    y1 = clampd(y1, 0, (double)ny);
    x2 = clampd(x2, 0, (double)nx);
    y2 = clampd(y2, 0, (double)ny);
    long ix1 = clampi((long)x1, 0, nx), iy1 = clampi((long)y1, 0, ny);
    long ix2 = clampi((long)x2, 0, nx), iy2 = clampi((long)y2, 0, ny);
    if (x2 <= x1 || y2 <= y1) return 0;
    double v = 0;
    for (long iy = iy1; iy <= iy2; iy++) {
        double wy = 1.0;
        if (iy == iy1) wy -= (y1 - iy1);
        if (iy == iy2) wy -= (iy2 + 1 - y2);
        double r = 0;
        for (long ix = ix1; ix <= ix2; ix++) {
            double wx = 1.0;
            if (ix == ix1) wx -= (x1 - ix1);
            if (ix == ix2) wx -= (ix2 + 1 - x2);
            r += p[iy * nx + ix] * wx;
        }
        v += r * wy;
    }
    return v;
}

/* ------------------------------------------------------------------------ */
/* Distance-driven 2D (fan / parallel) forward projection                    */
/* ------------------------------------------------------------------------ */

/* z interpolation of DDFPTracing, distanceDriven2DBoxInt.cu:35-42 */
static void z_interp(double z, long nz, long* iz, long* iz1, double* wz)
{
    z = clampd(z, 0, (double)nz);
    long a = (long)z;
    long b = a + 1;
    a = clampi(a, 0, nz);
    b = clampi(b, 0, nz);
    *iz = a;
    *iz1 = b;
    *wz = z - a;
}

/* Ray footprint for one detector cell: the two edge rays src_k -> dst_k in
 * image coordinates. */
typedef struct {
    double s1x, s1y, s2x, s2y; /* sources of edge 1 / edge 2 */
    double d1x, d1y, d2x, d2y; /* destinations */
} og_cell_rays;

static void to_img2(double* x, double* y, const og_grid* g)
{
    *x = (*x - g->cx) / g->dx + g->nx / 2.0;
    *y = (*y - g->cy) / g->dy + g->ny / 2.0;
}

/* Fan cell geometry, DDFPFanKernel distanceDriven2DBoxInt.cu:209-227. */
static void fan_cell(og_cell_rays* r, double* a_out, double deg, long iu, const og_grid* g,
                     const og_det* d, double dsd, double dso)
{
    double c = cos(deg), s = sin(deg);
    double a = (-(iu - (d->nu - 1) / 2.0) - d->off_u) * d->du;
    double sx = dso * s, sy = -dso * c;
    double e1x = dsd * sin(a - d->du / 2), e1y = -dso + dsd * cos(a - d->du / 2);
    double e2x = dsd * sin(a + d->du / 2), e2y = -dso + dsd * cos(a + d->du / 2);
    r->d1x = e1x * c - e1y * s;
    r->d1y = e1x * s + e1y * c;
    r->d2x = e2x * c - e2y * s;
    r->d2y = e2x * s + e2y * c;
    r->s1x = r->s2x = sx;
    r->s1y = r->s2y = sy;
    to_img2(&r->s1x, &r->s1y, g);
    to_img2(&r->s2x, &r->s2y, g);
    to_img2(&r->d1x, &r->d1y, g);
    to_img2(&r->d2x, &r->d2y, g);
    *a_out = a;
}

/* Parallel cell geometry, DDFPParallelKernel distanceDriven2DBoxInt.cu:139-164:
 * two virtual sources at distance nx*dx + ny*dy. */
static void par_cell(og_cell_rays* r, double deg, long iu, const og_grid* g, const og_det* d)
{
    double c = cos(deg), s = sin(deg);
    double u = (-(iu - (d->nu - 1) / 2.0) - d->off_u) * d->du;
    double dsov = g->nx * g->dx + g->ny * g->dy;
    double p[4][2] = {{u - d->du / 2, -dsov}, {u + d->du / 2, -dsov}, {u - d->du / 2, dsov}, {u + d->du / 2, dsov}};
    double q[4][2];
    for (int k = 0; k < 4; k++) {
        q[k][0] = p[k][0] * c - p[k][1] * s;
        q[k][1] = p[k][0] * s + p[k][1] * c;
        to_img2(&q[k][0], &q[k][1], g);
    }
    r->s1x = q[0][0]; r->s1y = q[0][1];
    r->s2x = q[1][0]; r->s2y = q[1][1];
    r->d1x = q[2][0]; r->d1y = q[2][1];
    r->d2x = q[3][0]; r->d2y = q[3][1];
}

/* Visitor used by the forward projector, its exact transpose and the nnz count.
 * mode 0: return sum (forward), mode 1: scatter val into out, mode 2: count. */
typedef struct {
    int mode;
    const double* img; /* slice pointers resolved by caller */
    double* out;
    double val;
    long long count;
} og_visit;

/* Row-wise (y main axis) or column-wise (x main axis) box-integral sweep of
 * one cell over one slice pair; returns sum_rows integral/width for mode 0.
 * distanceDriven2DBoxInt.cu:47-98. */
static double dd_sweep(const og_cell_rays* r, int ymain, const double* s0, const double* s1, double w0,
                       double w1, double* o0, double* o1, double scat, long long* cnt, int mode,
                       const og_grid* g)
{
    double acc = 0;
    long nx = g->nx, ny = g->ny;
    if (ymain) {
        double r1 = (r->d1x - r->s1x) / (r->d1y - r->s1y);
        double r2 = (r->d2x - r->s2x) / (r->d2y - r->s2y);
        for (long iy = 0; iy < ny; iy++) {
            double x1 = r->s1x + r1 * (iy + 0.5 - r->s1y);
            double x2 = r->s2x + r2 * (iy + 0.5 - r->s2y);
            if (x1 > x2) { double t = x1; x1 = x2; x2 = t; }
            double w = x2 - x1;
            if (mode == 0) {
                double v = box1d(s0 + iy * nx, 1, x1, x2, nx) * w0;
                if (w1 != 0) v += box1d(s1 + iy * nx, 1, x1, x2, nx) * w1;
                acc += v / w;
            } else {
                double c1 = clampd(x1, 0, (double)nx), c2 = clampd(x2, 0, (double)nx);
                if (c2 <= c1) continue;
                long i1 = clampi((long)c1, 0, nx), i2 = clampi((long)c2, 0, nx);
                if (mode == 2) { *cnt += (i2 - i1 + 1) * (w1 != 0 ? 2 : 1); continue; }
                for (long i = i1; i <= i2; i++) {
                    double ov = 1.0;
                    if (i == i1) ov -= (c1 - i1);
                    if (i == i2) ov -= (i2 + 1 - c2);
                    o0[iy * nx + i] += scat * w0 * ov / w;
                    if (w1 != 0) o1[iy * nx + i] += scat * w1 * ov / w;
                }
            }
        }
    } else {
        double r1 = (r->d1y - r->s1y) / (r->d1x - r->s1x);
        double r2 = (r->d2y - r->s2y) / (r->d2x - r->s2x);
        for (long ix = 0; ix < nx; ix++) {
            double y1 = r->s1y + r1 * (ix + 0.5 - r->s1x);
            double y2 = r->s2y + r2 * (ix + 0.5 - r->s2x);
            if (y1 > y2) { double t = y1; y1 = y2; y2 = t; }
            double w = y2 - y1;
            if (mode == 0) {
                double v = box1d(s0 + ix, nx, y1, y2, ny) * w0;
                if (w1 != 0) v += box1d(s1 + ix, nx, y1, y2, ny) * w1;
                acc += v / w;
            } else {
                double c1 = clampd(y1, 0, (double)ny), c2 = clampd(y2, 0, (double)ny);
                if (c2 <= c1) continue;
                long i1 = clampi((long)c1, 0, ny), i2 = clampi((long)c2, 0, ny);
                if (mode == 2) { *cnt += (i2 - i1 + 1) * (w1 != 0 ? 2 : 1); continue; }
                for (long i = i1; i <= i2; i++) {
                    double ov = 1.0;
                    if (i == i1) ov -= (c1 - i1);
                    if (i == i2) ov -= (i2 + 1 - c2);
                    o0[i * nx + ix] += scat * w0 * ov / w;
                    if (w1 != 0) o1[i * nx + ix] += scat * w1 * ov / w;
                }
            }
        }
    }
    return acc;
}

/* One ray of DDFPTracing (distanceDriven2DBoxInt.cu:21-106) in any mode.
 * hard != 0: the branchless tracer's axis choice (distanceDriven2DBranchless.cu
 * :56-120): the main axis alone by |cos| > |sin|, no blend band. */
static double dd_ray(const og_cell_rays* r, double deg, double a, double z, const double* vol, double* out,
                     double scat, long long* cnt, int mode, const og_grid* g, int hard)
{
    long iz, iz1;
    double wz;
    z_interp(z, g->nz, &iz, &iz1, &wz);
    long nxy = g->nx * g->ny;
    const double* s0 = vol ? vol + iz * nxy : NULL;
    const double* s1 = vol ? vol + iz1 * nxy : NULL;
    double* o0 = out ? out + iz * nxy : NULL;
    double* o1 = out ? out + iz1 * nxy : NULL;
    double c = cos(deg), s = sin(deg);
    double ac = fabs(c), as = fabs(s);
    double wx = hard ? (ac > as ? 1.0 : 0.0) : clampd((ac - as + DD_MARGIN) / (2 * DD_MARGIN), 0, 1);
    double valx = 0, valy = 0;
    if (wx > 0) {
        double L = g->dy / fabs(cos(deg - a));
        valx = dd_sweep(r, 1, s0, s1, 1 - wz, wz, o0, o1, scat * L * wx, cnt, mode, g) * L;
    }
    if (wx < 1) {
        double L = g->dx / fabs(sin(deg - a));
        valy = dd_sweep(r, 0, s0, s1, 1 - wz, wz, o0, o1, scat * L * (1 - wx), cnt, mode, g) * L;
    }
    return valx * wx + valy * (1 - wx);
}

static double fan_zpos(long iv, const og_det* d, const og_grid* g) /* distanceDriven2DBoxInt.cu:214,227 */
{
    double z = (iv - (d->nv - 1) / 2.0 + d->off_v) * d->dv;
    return (z - g->cz) / g->dz + g->nz / 2.0 - 0.5;
}

/* fan: geom 0, parallel: geom 1.  Forward projection, writes prj (=);
 * branchless != 0 traces like distanceDriven2DBranchless.cu:56-258 (the
 * prefix-sum interpolation there is the same clamped box integral). */
void oracle_dd2d_fp_mode(double* prj, const double* img, const double* deg, long nb, og_grid g, og_det d,
                         long nview, double dsd, double dso, int geom, int branchless)
{
    long nxyz = g.nx * g.ny * g.nz;
    long nrays = d.nu * d.nv * nview;
#pragma omp parallel for schedule(dynamic, 64)
    for (long t = 0; t < nb * nrays; t++) {
        long ib = t / nrays, k = t % nrays;
        long iview = k / (d.nu * d.nv), iv = (k / d.nu) % d.nv, iu = k % d.nu;
        og_cell_rays r;
        double a = 0;
        if (geom == 0) fan_cell(&r, &a, deg[iview], iu, &g, &d, dsd, dso);
        else par_cell(&r, deg[iview], iu, &g, &d);
        prj[t] = dd_ray(&r, deg[iview], a, fan_zpos(iv, &d, &g), img + ib * nxyz, NULL, 0, NULL, 0, &g, branchless);
    }
}

void oracle_dd2d_fp(double* prj, const double* img, const double* deg, long nb, og_grid g, og_det d,
                    long nview, double dsd, double dso, int geom)
{
    oracle_dd2d_fp_mode(prj, img, deg, nb, g, d, nview, dsd, dso, geom, 0);
}

/* Exact transpose of oracle_dd2d_fp: img += A^T prj. */
void oracle_dd2d_bp_adjoint(double* img, const double* prj, const double* deg, long nb, og_grid g, og_det d,
                            long nview, double dsd, double dso, int geom)
{
    long nxyz = g.nx * g.ny * g.nz;
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    double* priv = (double*)calloc((size_t)nt * nxyz, sizeof(double));
    for (long ib = 0; ib < nb; ib++) {
        memset(priv, 0, sizeof(double) * nt * nxyz);
#pragma omp parallel
        {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            double* acc = priv + (size_t)tid * nxyz;
#pragma omp for schedule(static)
            for (long iview = 0; iview < nview; iview++) {
                for (long iv = 0; iv < d.nv; iv++) {
                    for (long iu = 0; iu < d.nu; iu++) {
                        double p = prj[((ib * nview + iview) * d.nv + iv) * d.nu + iu];
                        if (p == 0) continue;
                        og_cell_rays r;
                        double a = 0;
                        if (geom == 0) fan_cell(&r, &a, deg[iview], iu, &g, &d, dsd, dso);
                        else par_cell(&r, deg[iview], iu, &g, &d);
                        dd_ray(&r, deg[iview], a, fan_zpos(iv, &d, &g), NULL, acc, p, NULL, 1, &g, 0);
                    }
                }
            }
        }
        for (int t = 0; t < nt; t++)
            for (long i = 0; i < nxyz; i++) img[ib * nxyz + i] += priv[(size_t)t * nxyz + i];
    }
    free(priv);
}

/* Operator nonzeros: sum over rays and main-axis lines of the pixels in the
 * clamped footprint, both axes inside the blend band, both z slices when the
 * interpolation weight is nonzero. */
long long oracle_dd2d_nnz(const double* deg, og_grid g, og_det d, long nview, double dsd, double dso, int geom)
{
    long long total = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : total)
    for (long iview = 0; iview < nview; iview++) {
        long long cnt = 0;
        for (long iv = 0; iv < d.nv; iv++)
            for (long iu = 0; iu < d.nu; iu++) {
                og_cell_rays r;
                double a = 0;
                if (geom == 0) fan_cell(&r, &a, deg[iview], iu, &g, &d, dsd, dso);
                else par_cell(&r, deg[iview], iu, &g, &d);
                dd_ray(&r, deg[iview], a, fan_zpos(iv, &d, &g), NULL, NULL, 0, &cnt, 2, &g, 0);
            }
        total += cnt;
    }
    return total;
}

/* ------------------------------------------------------------------------ */
/* Distance-driven 2D back projection, reference-parity (normalised) mode.   */
/* ------------------------------------------------------------------------ */

/* Pre-weight of the copied sinogram, distanceDriven2DUtils.cu:8-65 (hard
 * switch on |cos| > |sin| of the view angle). */
static double preweight(double deg, long iu, const og_det* d, const og_grid* g, int geom)
{
    double a = geom == 0 ? (-(iu - (d->nu - 1) / 2.0) - d->off_u) * d->du : 0.0;
    if (fabs(cos(deg)) > fabs(sin(deg))) return g->dy / fabs(cos(deg - a));
    return g->dx / fabs(sin(deg - a));
}

/* Normalised box integral of one pre-weighted detector row over the
 * projection of pixel (xc, yc) for one view: DDBPFanKernel
 * distanceDriven2DBoxInt.cu:354-390 + utils :96-116 (fan, hard axis switch),
 * DDBPParallelKernel :440-491 (parallel: blend band, or the branchless hard
 * switch, distanceDriven2DBranchless.cu:509-530). */
static double bp_row(const double* row, const double* wr, double c, double s, double xc, double yc,
                     const og_grid* g, const og_det* d, double dso, int geom, int fbp, int hard)
{
    double x1 = xc - g->dx / 2, x2 = xc + g->dx / 2, y1 = yc - g->dy / 2, y2 = yc + g->dy / 2;
    if (geom == 0) {
        double a1, a2;
        if (fabs(c) > fabs(s)) {
            a1 = atan((x1 * c + yc * s) / ((-x1 * s + yc * c) + dso));
            a2 = atan((x2 * c + yc * s) / ((-x2 * s + yc * c) + dso));
        } else {
            a1 = atan((xc * c + y1 * s) / ((-xc * s + y1 * c) + dso));
            a2 = atan((xc * c + y2 * s) / ((-xc * s + y2 * c) + dso));
        }
        a1 = -(a1 / d->du + d->off_u) + d->nu / 2.0;
        a2 = -(a2 / d->du + d->off_u) + d->nu / 2.0;
        if (a1 > a2) { double t = a1; a1 = a2; a2 = t; }
        /* integral of the pre-weighted row */
        double v = 0;
        double c1 = clampd(a1, 0, (double)d->nu), c2 = clampd(a2, 0, (double)d->nu);
        if (c2 > c1) {
            long i1 = clampi((long)c1, 0, d->nu), i2 = clampi((long)c2, 0, d->nu);
            for (long i = i1; i <= i2; i++) v += row[i] * wr[i];
            v -= row[i1] * wr[i1] * (c1 - i1) + row[i2] * wr[i2] * (i2 + 1 - c2);
        }
        v /= (a2 - a1);
        if (fbp) {
            double rx = xc * c + yc * s, ry = -xc * s + yc * c;
            v *= dso * dso / (rx * rx + (dso + ry) * (dso + ry));
        }
        return v;
    }
    double valx = 0, valy = 0;
    double wv = wr[0];
    double wx = hard ? (fabs(c) > fabs(s) ? 1.0 : 0.0) : clampd((fabs(c) - fabs(s) + DD_MARGIN) / (2 * DD_MARGIN), 0, 1);
    if (wx > 0) {
        double u1 = -((x1 * c + yc * s) / d->du + d->off_u) + d->nu / 2.0;
        double u2 = -((x2 * c + yc * s) / d->du + d->off_u) + d->nu / 2.0;
        if (u1 > u2) { double t = u1; u1 = u2; u2 = t; }
        valx = box1d(row, 1, u1, u2, d->nu) * wv / (u2 - u1);
    }
    if (wx < 1) {
        double u1 = -((xc * c + y1 * s) / d->du + d->off_u) + d->nu / 2.0;
        double u2 = -((xc * c + y2 * s) / d->du + d->off_u) + d->nu / 2.0;
        if (u1 > u2) { double t = u1; u1 = u2; u2 = t; }
        valy = box1d(row, 1, u1, u2, d->nu) * wv / (u2 - u1);
    }
    return valx * wx + valy * (1 - wx);
}

/* Fan: DDBPFanKernel distanceDriven2DBoxInt.cu:319-396 + utils :96-116.
 * Parallel: DDBPParallelKernel :409-497.  img += BP(prj).
 * fbp != 0 selects the FBP weighting (no pre-weight; fan adds dso^2/L^2).
 * branchless != 0: distanceDriven2DBranchless.cu:384-530 -- the parallel
 * beam's hard axis switch, and the detector row interpolated linearly at the
 * pixel's v (InterpolateXY of the row prefix sums, cudaMath.cu:227-258: rows
 * clamped to [0, nv-1]) where the box-integral mode truncates it. */
void oracle_dd2d_bp_mode(double* img, const double* prj, const double* deg, long nb, og_grid g, og_det d,
                         long nview, double dsd, double dso, int geom, int fbp, int branchless)
{
    (void)dsd;
    long nxyz = g.nx * g.ny * g.nz;
    long nprj = nview * d.nv * d.nu;
    double* w = (double*)malloc(sizeof(double) * nview * d.nu);
    for (long iview = 0; iview < nview; iview++)
        for (long iu = 0; iu < d.nu; iu++) w[iview * d.nu + iu] = fbp ? 1.0 : preweight(deg[iview], iu, &d, &g, geom);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (long ib = 0; ib < nb; ib++)
        for (long iz = 0; iz < g.nz; iz++) {
            const double* p = prj + ib * nprj;
            double zc = (iz - g.nz / 2.0) * g.dz + g.cz + g.dz / 2;
            double ivf = zc / d.dv + d.off_v + d.nv / 2.0 - 0.5;
            long iv0, iv1;
            double wv1;
            if (branchless) {
                double v = clampd(ivf, 0, (double)d.nv);
                iv0 = (long)v;
                iv1 = clampi(iv0 + 1, 0, d.nv);
                iv0 = clampi(iv0, 0, d.nv);
                wv1 = v - iv0;
            } else {
                iv0 = iv1 = (long)ivf; /* float -> int parameter: truncation, :383 */
                wv1 = 0;
                if (iv0 < 0 || iv0 >= d.nv) continue; /* reference reads outside the view here */
            }
            for (long iy = 0; iy < g.ny; iy++)
                for (long ix = 0; ix < g.nx; ix++) {
                    double xc = (ix - g.nx / 2.0) * g.dx + g.cx + g.dx / 2;
                    double yc = (iy - g.ny / 2.0) * g.dy + g.cy + g.dy / 2;
                    double acc = 0;
                    for (long iview = 0; iview < nview; iview++) {
                        double c = cos(deg[iview]), s = sin(deg[iview]);
                        const double* wr = w + iview * d.nu;
                        double v0 = bp_row(p + (iview * d.nv + iv0) * d.nu, wr, c, s, xc, yc, &g, &d, dso, geom, fbp,
                                           branchless);
                        if (wv1 != 0)
                            v0 = v0 * (1 - wv1) + wv1 * bp_row(p + (iview * d.nv + iv1) * d.nu, wr, c, s, xc, yc,
                                                               &g, &d, dso, geom, fbp, branchless);
                        acc += v0;
                    }
                    img[ib * nxyz + (iz * g.ny + iy) * g.nx + ix] += acc;
                }
        }
    free(w);
}

void oracle_dd2d_bp(double* img, const double* prj, const double* deg, long nb, og_grid g, og_det d,
                    long nview, double dsd, double dso, int geom, int fbp)
{
    oracle_dd2d_bp_mode(img, prj, deg, nb, g, d, nview, dsd, dso, geom, fbp, 0);
}

/* ------------------------------------------------------------------------ */
/* Pixel-driven fan FBP back projection, fbp.cu:265-337 (bpFanKernel3D with  */
/* isFBP = true, bilinear InterpolateXY(truncate=true) cudaMath.cu:227-260). */
/* ------------------------------------------------------------------------ */
void oracle_fbp_fan_bp(double* img, const double* prj, const double* deg, long nb, og_grid g, og_det d,
                       long nview, double dsd, double dso)
{
    (void)dsd;
    long nxyz = g.nx * g.ny * g.nz;
    long nprj = nview * d.nv * d.nu;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (long ib = 0; ib < nb; ib++)
        for (long iy = 0; iy < g.ny; iy++)
            for (long ix = 0; ix < g.nx; ix++) {
                double x = (ix + 0.5 - g.nx / 2.0) * g.dx + g.cx;
                double y = (iy + 0.5 - g.ny / 2.0) * g.dy + g.cy;
                for (long iz = 0; iz < g.nz; iz++) {
                    double z = (iz + 0.5 - g.nz / 2.0) * g.dz + g.cz;
                    double acc = 0;
                    for (long iview = 0; iview < nview; iview++) {
                        double c = cos(deg[iview]), s = sin(deg[iview]);
                        double rx = x * c + y * s, ry = -x * s + y * c;
                        double a = atan(rx / (ry + dso));
                        double dist = dso * dso / (rx * rx + (dso + ry) * (dso + ry));
                        double pu = -(a / d.du + d.off_u) + (d.nu - 1.0) / 2.0;
                        double pv = z / d.dv + d.off_v + (d.nv - 1.0) / 2.0;
                        if (pu < 0 || pu >= d.nu || pv < 0 || pv >= d.nv) continue;
                        long i0 = (long)pu, j0 = (long)pv;
                        long i1 = clampi(i0 + 1, 0, d.nu), j1 = clampi(j0 + 1, 0, d.nv);
                        double wu = pu - i0, wv = pv - j0;
                        const double* p = prj + ib * nprj + iview * d.nv * d.nu;
                        double v = p[j0 * d.nu + i0] * (1 - wu) * (1 - wv) + p[j0 * d.nu + i1] * wu * (1 - wv) +
                                   p[j1 * d.nu + i0] * (1 - wu) * wv + p[j1 * d.nu + i1] * wu * wv;
                        acc += v * dist;
                    }
                    img[ib * nxyz + (iz * g.ny + iy) * g.nx + ix] += acc;
                }
            }
}

/* ------------------------------------------------------------------------ */
/* Siddon cone-beam, arbitrary trajectory.  siddon.cu:35-362,                */
/* siddonCone.cu:12-74.  Geometry arrays are [nview][3] as (x, y, z).        */
/* ------------------------------------------------------------------------ */

/* MoveSourceDstNearGrid, siddon.cu:342-362 */
static void move_near_grid(double* src, double* dst, const og_grid* g)
{
    double ex = g->nx * g->dx, ey = g->ny * g->dy, ez = g->nz * g->dz;
    double r = sqrt(ex * ex + ey * ey + ez * ez);
    double d[3] = {dst[0] - src[0], dst[1] - src[1], dst[2] - src[2]};
    double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (len >= 1e-6)
        for (int k = 0; k < 3; k++) d[k] /= len;
    double t0 = (g->cx - src[0]) * d[0] + (g->cy - src[1]) * d[1] + (g->cz - src[2]) * d[2];
    double t1 = (dst[0] - g->cx) * d[0] + (dst[1] - g->cy) * d[1] + (dst[2] - g->cz) * d[2];
    if (t0 > r)
        for (int k = 0; k < 3; k++) src[k] += (t0 - r) * d[k];
    if (t1 > r)
        for (int k = 0; k < 3; k++) dst[k] -= (t1 - r) * d[k];
}

/* Siddon walk (InitializeSiddon siddon.cu:104-173 and SiddonRayTracing
 * :175-257).  mode 0 returns sum img*len, mode 1 scatters val*len into out,
 * mode 2 returns the segment count. */
static double siddon_walk(const double* img, double* out, double val, long long* cnt, int mode, double* src,
                          double* dst, const og_grid* g)
{
    double dist = sqrt((src[0] - dst[0]) * (src[0] - dst[0]) + (src[1] - dst[1]) * (src[1] - dst[1]) +
                       (src[2] - dst[2]) * (src[2] - dst[2]));
    double s[3] = {(src[0] - g->cx) / g->dx + g->nx / 2.0, (src[1] - g->cy) / g->dy + g->ny / 2.0,
                   (src[2] - g->cz) / g->dz + g->nz / 2.0};
    double e[3] = {(dst[0] - g->cx) / g->dx + g->nx / 2.0, (dst[1] - g->cy) / g->dy + g->ny / 2.0,
                   (dst[2] - g->cz) / g->dz + g->nz / 2.0};
    long n[3] = {g->nx, g->ny, g->nz};
    double dd[3], a0[3] = {1, 1, 1}, a1[3] = {0, 0, 0};
    for (int k = 0; k < 3; k++) {
        dd[k] = e[k] - s[k];
        if (fabs(dd[k]) > SIDDON_EPS) { /* InboundAlpha :37-56 */
            a0[k] = (0 - s[k]) / dd[k];
            a1[k] = (n[k] - s[k]) / dd[k];
        } else if (s[k] < 0 || s[k] > n[k]) {
            return 0;
        }
    }
    double amin = 0, amax = 1;
    for (int k = 0; k < 3; k++) {
        double lo = a0[k] < a1[k] ? a0[k] : a1[k];
        double hi = a0[k] < a1[k] ? a1[k] : a0[k];
        if (lo > amin) amin = lo;
        if (hi < amax) amax = hi;
    }
    if (amax <= amin) return 0;
    long ng[3];
    double alpha[3], dalpha[3];
    int pos[3];
    for (int k = 0; k < 3; k++) {
        double p0 = s[k] + amin * dd[k];
        long v = (long)p0; /* InboundFirstVoxel :59-75 */
        if (fabs(dd[k]) > SIDDON_EPS) {
            if (v < 0) v = 0;
            else if (v >= n[k]) v = n[k] - 1;
        }
        ng[k] = v;
        double p1 = dd[k] > SIDDON_EPS ? (double)(v + 1) : (double)v; /* OutboundFirstVoxel :78-92 */
        alpha[k] = 2.0;
        dalpha[k] = 0;
        if (fabs(dd[k]) > SIDDON_EPS) { /* GetAlpha :95-102 */
            alpha[k] = (p1 - s[k]) / dd[k];
            dalpha[k] = 1 / fabs(dd[k]);
        }
        alpha[k] *= dist;
        dalpha[k] *= dist;
        pos[k] = dd[k] > 0;
    }
    for (int k = 0; k < 3; k++)
        if (ng[k] < 0 || ng[k] >= n[k]) return 0; /* :179-185 */
    double aprev = amin * dist, anow;
    double acc = 0;
    int tracing = 1;
    while (tracing) {
        int k;
        if (alpha[0] < alpha[1] && alpha[0] < alpha[2]) k = 0;
        else if (alpha[1] < alpha[2]) k = 1;
        else k = 2;
        long idx = (ng[2] * g->ny + ng[1]) * g->nx + ng[0];
        anow = alpha[k];
        alpha[k] += dalpha[k];
        if (pos[k]) {
            if (++ng[k] >= n[k]) tracing = 0;
        } else {
            if (--ng[k] < 0) tracing = 0;
        }
        double len = anow - aprev;
        if (mode == 0) acc += img[idx] * len;
        else if (mode == 1) out[idx] += val * len;
        else *cnt += 1;
        aprev = anow;
    }
    return acc;
}

static void siddon_ray_ends(double* src, double* dst, long iview, long iu, long iv, const float* dc,
                            const float* du_, const float* dv_, const float* sr, const og_det* d, const og_grid* g)
{
    /* siddonCone.cu:33-38 and UVToCart cudaMath.h:104-117 */
    double u = (iu - d->off_u - (d->nu - 1) / 2.0) * d->du;
    double v = (iv - d->off_v - (d->nv - 1) / 2.0) * d->dv;
    for (int k = 0; k < 3; k++) {
        src[k] = sr[iview * 3 + k];
        dst[k] = dc[iview * 3 + k] + du_[iview * 3 + k] * u + dv_[iview * 3 + k] * v;
    }
    move_near_grid(src, dst, g);
}

/* prj += FP(img)  (siddon.cu:254: the reference accumulates into prj) */
void oracle_siddon_fp(double* prj, const double* img, const float* det_center, const float* det_u,
                      const float* det_v, const float* src, long nb, og_grid g, og_det d, long nview)
{
    long nxyz = g.nx * g.ny * g.nz;
    long nrays = nview * d.nv * d.nu;
#pragma omp parallel for schedule(dynamic, 64)
    for (long t = 0; t < nb * nrays; t++) {
        long ib = t / nrays, k = t % nrays;
        long iview = k / (d.nu * d.nv), iv = (k / d.nu) % d.nv, iu = k % d.nu;
        double s[3], e[3];
        siddon_ray_ends(s, e, iview, iu, iv, det_center, det_u, det_v, src, &d, &g);
        prj[t] += siddon_walk(img + ib * nxyz, NULL, 0, NULL, 0, s, e, &g);
    }
}

/* img += BP(prj): the transpose with the same segment lengths. */
void oracle_siddon_bp(double* img, const double* prj, const float* det_center, const float* det_u,
                      const float* det_v, const float* src, long nb, og_grid g, og_det d, long nview)
{
    long nxyz = g.nx * g.ny * g.nz;
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    double* priv = (double*)calloc((size_t)nt * nxyz, sizeof(double));
    for (long ib = 0; ib < nb; ib++) {
        memset(priv, 0, sizeof(double) * nt * nxyz);
#pragma omp parallel
        {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            double* acc = priv + (size_t)tid * nxyz;
#pragma omp for schedule(static)
            for (long iview = 0; iview < nview; iview++)
                for (long iv = 0; iv < d.nv; iv++)
                    for (long iu = 0; iu < d.nu; iu++) {
                        double p = prj[((ib * nview + iview) * d.nv + iv) * d.nu + iu];
                        double s[3], e[3];
                        siddon_ray_ends(s, e, iview, iu, iv, det_center, det_u, det_v, src, &d, &g);
                        siddon_walk(NULL, acc, p, NULL, 1, s, e, &g);
                    }
        }
        for (int t = 0; t < nt; t++)
            for (long i = 0; i < nxyz; i++) img[ib * nxyz + i] += priv[(size_t)t * nxyz + i];
    }
    free(priv);
}

/* Fan-beam Siddon rays (SiddonFanProjectionKernel, siddonFan.cu:12-44): the
 * source on the circle of radius dso, the detector cell on the arc of radius
 * dsd at angle a = (-(iu - (nu-1)/2) - off_u) da, both at height
 * z = (iv - (nv-1)/2 + off_v) dv, rotated by the view angle; the end points
 * are not moved towards the grid. */
static void siddon_fan_ray_ends(double* src, double* dst, double deg, long iu, long iv, const og_det* d, double dsd,
                                double dso)
{
    double c = cos(deg), s = sin(deg);
    double a = (-(iu - (d->nu - 1) / 2.0) - d->off_u) * d->du;
    double z = (iv - (d->nv - 1) / 2.0 + d->off_v) * d->dv;
    double rx = dsd * sin(a), ry = -dso + dsd * cos(a);
    src[0] = dso * s;
    src[1] = -dso * c;
    src[2] = z;
    dst[0] = rx * c - ry * s;
    dst[1] = rx * s + ry * c;
    dst[2] = z;
}

/* prj = FP(img) for fan-beam Siddon (the reference's host entry zeroes prj). */
void oracle_siddon_fan_fp(double* prj, const double* img, const double* deg, long nb, og_grid g, og_det d,
                          long nview, double dsd, double dso)
{
    long nxyz = g.nx * g.ny * g.nz;
    long nrays = nview * d.nv * d.nu;
#pragma omp parallel for schedule(dynamic, 64)
    for (long t = 0; t < nb * nrays; t++) {
        long ib = t / nrays, k = t % nrays;
        long iview = k / (d.nu * d.nv), iv = (k / d.nu) % d.nv, iu = k % d.nu;
        double s[3], e[3];
        siddon_fan_ray_ends(s, e, deg[iview], iu, iv, &d, dsd, dso);
        prj[t] = siddon_walk(img + ib * nxyz, NULL, 0, NULL, 0, s, e, &g);
    }
}

/* img = BP(prj) for fan-beam Siddon: the transpose with the same segments. */
void oracle_siddon_fan_bp(double* img, const double* prj, const double* deg, long nb, og_grid g, og_det d,
                          long nview, double dsd, double dso)
{
    long nxyz = g.nx * g.ny * g.nz;
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    double* priv = (double*)calloc((size_t)nt * nxyz, sizeof(double));
    for (long ib = 0; ib < nb; ib++) {
        memset(priv, 0, sizeof(double) * nt * nxyz);
#pragma omp parallel
        {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            double* acc = priv + (size_t)tid * nxyz;
#pragma omp for schedule(static)
            for (long iview = 0; iview < nview; iview++)
                for (long iv = 0; iv < d.nv; iv++)
                    for (long iu = 0; iu < d.nu; iu++) {
                        double p = prj[((ib * nview + iview) * d.nv + iv) * d.nu + iu];
                        double s[3], e[3];
                        siddon_fan_ray_ends(s, e, deg[iview], iu, iv, &d, dsd, dso);
                        siddon_walk(NULL, acc, p, NULL, 1, s, e, &g);
                    }
        }
        for (long i = 0; i < nxyz; i++) {
            double v = 0;
            for (int t = 0; t < nt; t++) v += priv[(size_t)t * nxyz + i];
            img[ib * nxyz + i] = v;
        }
    }
    free(priv);
}

long long oracle_siddon_nnz(const float* det_center, const float* det_u, const float* det_v, const float* src,
                            og_grid g, og_det d, long nview)
{
    long long total = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total)
    for (long iview = 0; iview < nview; iview++) {
        long long cnt = 0;
        for (long iv = 0; iv < d.nv; iv++)
            for (long iu = 0; iu < d.nu; iu++) {
                double s[3], e[3];
                siddon_ray_ends(s, e, iview, iu, iv, det_center, det_u, det_v, src, &d, &g);
                siddon_walk(NULL, NULL, 0, &cnt, 2, s, e, &g);
            }
        total += cnt;
    }
    return total;
}

/* ------------------------------------------------------------------------ */
/* Tomosynthesis distance driven (z main axis, detector u=(1,0,0) v=(0,1,0)) */
/* ------------------------------------------------------------------------ */

/* prj = FP(img): DDFPConeBoxIntKernelXY distanceDriven3DBoxInt.cu:28-117 */
void oracle_tomo_fp(double* prj, const double* img, const float* det_center, const float* src, long nb,
                    og_grid g, og_det d, long nview)
{
    long nxyz = g.nx * g.ny * g.nz;
    long nrays = nview * d.nv * d.nu;
#pragma omp parallel for schedule(dynamic, 64)
    for (long t = 0; t < nb * nrays; t++) {
        long ib = t / nrays, k = t % nrays;
        long iview = k / (d.nu * d.nv), iv = (k / d.nu) % d.nv, iu = k % d.nu;
        double u = (iu - d.off_u - (d.nu - 1) / 2.0) * d.du;
        double v = (iv - d.off_v - (d.nv - 1) / 2.0) * d.dv;
        double C[3] = {det_center[iview * 3], det_center[iview * 3 + 1], det_center[iview * 3 + 2]};
        double S[3] = {src[iview * 3], src[iview * 3 + 1], src[iview * 3 + 2]};
        double ax1[3] = {C[0] + u - d.du / 2, C[1] + v, C[2]};
        double ax2[3] = {C[0] + u + d.du / 2, C[1] + v, C[2]};
        double ay1[3] = {C[0] + u, C[1] + v - d.dv / 2, C[2]};
        double ay2[3] = {C[0] + u, C[1] + v + d.dv / 2, C[2]};
        double Si[3];
        double* pts[5] = {Si, ax1, ax2, ay1, ay2};
        Si[0] = S[0]; Si[1] = S[1]; Si[2] = S[2];
        for (int q = 0; q < 5; q++) {
            pts[q][0] = (pts[q][0] - g.cx) / g.dx + g.nx / 2.0;
            pts[q][1] = (pts[q][1] - g.cy) / g.dy + g.ny / 2.0;
            pts[q][2] = (pts[q][2] - g.cz) / g.dz + g.nz / 2.0;
        }
        if (ax1[0] > ax2[0]) for (int q = 0; q < 3; q++) { double tt = ax1[q]; ax1[q] = ax2[q]; ax2[q] = tt; }
        if (ay1[1] > ay2[1]) for (int q = 0; q < 3; q++) { double tt = ay1[q]; ay1[q] = ay2[q]; ay2[q] = tt; }
        double rx1 = (ax1[0] - Si[0]) / (ax1[2] - Si[2]);
        double rx2 = (ax2[0] - Si[0]) / (ax2[2] - Si[2]);
        double ry1 = (ay1[1] - Si[1]) / (ay1[2] - Si[2]);
        double ry2 = (ay2[1] - Si[1]) / (ay2[2] - Si[2]);
        double val = 0;
        const double* vol = img + ib * nxyz;
        for (long iz = 0; iz < g.nz; iz++) {
            double x1 = Si[0] + rx1 * (iz - Si[2]);
            double x2 = Si[0] + rx2 * (iz - Si[2]);
            double y1 = Si[1] + ry1 * (iz - Si[2]);
            double y2 = Si[1] + ry2 * (iz - Si[2]);
            val += box2d(vol + iz * g.nx * g.ny, x1, y1, x2, y2, g.nx, g.ny) / ((x2 - x1) * (y2 - y1));
        }
        double D[3] = {C[0] + u, C[1] + v, C[2]};
        double L = sqrt((S[2] - D[2]) * (S[2] - D[2]) + (S[1] - D[1]) * (S[1] - D[1]) +
                        (S[0] - D[0]) * (S[0] - D[0]));
        prj[t] = val * g.dz / fabs(S[2] - D[2]) * L;
    }
}

/* img = BP(prj), reference-parity mode: PreweightBPCartKernelXY
 * distanceDriven3DUtils.cu:10-31 then DDBPConeBoxIntCartKernelXY
 * distanceDriven3DBoxInt.cu:170-216 with ProjectConeToDetCart
 * distanceDriven3DUtils.cu:45-56.  Every batch uses its own projections (the
 * reference reads batch 0's weighted projections for every batch). */
void oracle_tomo_bp(double* img, const double* prj, const float* det_center, const float* src, long nb,
                    og_grid g, og_det d, long nview)
{
    long nxyz = g.nx * g.ny * g.nz;
    long nprj = nview * d.nv * d.nu;
    double* w = (double*)malloc(sizeof(double) * nprj);
    for (long iview = 0; iview < nview; iview++)
        for (long iv = 0; iv < d.nv; iv++)
            for (long iu = 0; iu < d.nu; iu++) {
                double u = (iu - d.off_u - (d.nu - 1) / 2.0) * d.du;
                double v = (iv - d.off_v - (d.nv - 1) / 2.0) * d.dv;
                double D[3] = {det_center[iview * 3] + u, det_center[iview * 3 + 1] + v, det_center[iview * 3 + 2]};
                double S[3] = {src[iview * 3], src[iview * 3 + 1], src[iview * 3 + 2]};
                double L = sqrt((S[2] - D[2]) * (S[2] - D[2]) + (S[1] - D[1]) * (S[1] - D[1]) +
                                (S[0] - D[0]) * (S[0] - D[0]));
                w[(iview * d.nv + iv) * d.nu + iu] = g.dz / fabs(S[2] - D[2]) * L;
            }
    double* wp = (double*)malloc(sizeof(double) * nprj);
    for (long ib = 0; ib < nb; ib++) {
        for (long i = 0; i < nprj; i++) wp[i] = prj[ib * nprj + i] * w[i];
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
        for (long iz = 0; iz < g.nz; iz++)
            for (long iy = 0; iy < g.ny; iy++)
                for (long ix = 0; ix < g.nx; ix++) {
                    double x = (ix - (g.nx - 1) / 2.0) * g.dx + g.cx;
                    double y = (iy - (g.ny - 1) / 2.0) * g.dy + g.cy;
                    double z = (iz - (g.nz - 1) / 2.0) * g.dz + g.cz;
                    double val = 0;
                    for (long iview = 0; iview < nview; iview++) {
                        double S[3] = {src[iview * 3], src[iview * 3 + 1], src[iview * 3 + 2]};
                        double C[3] = {det_center[iview * 3], det_center[iview * 3 + 1], det_center[iview * 3 + 2]};
                        double r = (C[2] - S[2]) / (z - S[2]);
                        double u1 = (S[0] - C[0] + r * (x - g.dx / 2 - S[0])) / d.du + d.off_u + (d.nu - 1) / 2.0;
                        double u2 = (S[0] - C[0] + r * (x + g.dx / 2 - S[0])) / d.du + d.off_u + (d.nu - 1) / 2.0;
                        double v1 = (S[1] - C[1] + r * (y - g.dy / 2 - S[1])) / d.dv + d.off_v + (d.nv - 1) / 2.0;
                        double v2 = (S[1] - C[1] + r * (y + g.dy / 2 - S[1])) / d.dv + d.off_v + (d.nv - 1) / 2.0;
                        val += box2d(wp + iview * d.nv * d.nu, u1, v1, u2, v2, d.nu, d.nv) / ((u2 - u1) * (v2 - v1));
                    }
                    img[ib * nxyz + (iz * g.ny + iy) * g.nx + ix] = val;
                }
    }
    free(wp);
    free(w);
}

int oracle_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
