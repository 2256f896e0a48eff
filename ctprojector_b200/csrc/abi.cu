// abi.cu -- the exported C ABI of libctp.so (declared in include/ctp.h).
//
// Reference-compatible entries keep the reference symbols, argument order and
// output semantics (see include/ctp.h); extended ctp_* entries take an
// explicit stream, workspace and flags and never synchronise.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include "ctp_common.cuh"

namespace ctp {

// launchers defined in dd2d.cu, fbp.cu, siddon.cu, tomo.cu
int dd2d_fp(void*, const void*, const float*, const ctp_geometry&, int, int, unsigned, void*, size_t, cudaStream_t);
size_t dd2d_fp_workspace(const ctp_geometry&, int, int, unsigned);
void set_fp_stream_cap(int max_slices);
int dd2d_bp(void*, const void*, const float*, const ctp_geometry&, int, int, unsigned, void*, size_t, cudaStream_t);
size_t dd2d_bp_workspace(const ctp_geometry&, int, int, unsigned);
int dd2d_nnz(unsigned long long*, const float*, const ctp_geometry&, int, cudaStream_t);
int dd2d_fp_noalloc(void*, const void*, const float*, const ctp_geometry&, int, int, unsigned, cudaStream_t);
size_t dd2d_fp_noalloc_capacity();
int ramp_filter(float*, const float*, const ctp_geometry&, int, int, unsigned, void*, size_t, cudaStream_t);
size_t ramp_filter_workspace(const ctp_geometry&, int, int, unsigned);
int fbp_fan_bp(float*, const float*, const float*, const ctp_geometry&, unsigned, cudaStream_t);
int siddon_fp(void*, const void*, const float*, const float*, const float*, const float*, const ctp_geometry&,
              unsigned, cudaStream_t);
int siddon_bp(void*, const void*, const float*, const float*, const float*, const float*, const ctp_geometry&,
              unsigned, cudaStream_t);
int siddon_nnz(unsigned long long*, const float*, const float*, const float*, const float*, const ctp_geometry&,
               cudaStream_t);
int tomo_fp(float*, const float*, const float*, const float*, const ctp_geometry&, unsigned, cudaStream_t);
int tomo_bp(float*, const float*, const float*, const float*, const ctp_geometry&, unsigned, void*, size_t,
            cudaStream_t);
size_t tomo_bp_workspace(const ctp_geometry&);
int wait_timeouts(unsigned*);
int set_first_wait_polls(unsigned);
int quantize_u16(unsigned short*, float*, float*, const float*, size_t, size_t, cudaStream_t);
int dequantize_u16(float*, const unsigned short*, const float*, const float*, size_t, size_t, bool, cudaStream_t);
int ramp_filter_u16(float*, const unsigned short*, const float*, const float*, const ctp_geometry&, int, int,
                    cudaStream_t);
int siddon_fan_fp(float*, const float*, const float*, const ctp_geometry&, unsigned, cudaStream_t);
int siddon_fan_bp(float*, const float*, const float*, const ctp_geometry&, unsigned, cudaStream_t);
int pixel_bp_parallel(float*, const float*, const float*, const ctp_geometry&, unsigned, cudaStream_t);
size_t tomo_filter_workspace(const ctp_geometry&);
int tomo_filter(float*, const float*, const float*, const float*, const ctp_geometry&, int, float, float, unsigned,
                void*, size_t, cudaStream_t);
int sqs_tv_update(float*, void*, const float*, const float*, const float*, size_t, const unsigned char*, float, float,
                  float, float, float, size_t, size_t, size_t, unsigned, cudaStream_t);
int tv_sqs(float*, float*, float*, const float*, float, float, float, size_t, size_t, size_t, size_t, float,
           cudaStream_t);

static thread_local char t_err[512] = "";

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_err, sizeof(t_err), fmt, ap);
    va_end(ap);
    return code;
}

const char* last_error() { return t_err; }

int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error((int)e, "%s: %s", what, cudaGetErrorString(e));
    return CTP_OK;
}

int check_geometry(const ctp_geometry* g, bool need_image, bool need_detector) {
    if (!g) return set_error(CTP_ERR_INVALID_ARGUMENT, "geometry pointer is null");
    if (need_image && (g->nx == 0 || g->ny == 0 || g->nz == 0))
        return set_error(CTP_ERR_INVALID_ARGUMENT, "image size (%zu, %zu, %zu) has a zero extent", g->nz, g->ny,
                         g->nx);
    if (need_detector && (g->nu == 0 || g->nv == 0 || g->nview == 0))
        return set_error(CTP_ERR_INVALID_ARGUMENT, "sinogram size (%zu, %zu, %zu) has a zero extent", g->nview,
                         g->nv, g->nu);
    if (g->nx > (1u << 20) || g->ny > (1u << 20) || g->nz > (1u << 20) || g->nu > (1u << 20) || g->nv > (1u << 20) ||
        g->nview > 65535)
        return set_error(CTP_ERR_INVALID_ARGUMENT, "geometry extent out of range");
    return CTP_OK;
}

Scratch::~Scratch() {
    if (owned_ && ptr_) cudaFreeAsync(ptr_, stream_);
}

int Scratch::acquire(void* user, size_t user_bytes, size_t need, cudaStream_t s) {
    stream_ = s;
    if (need == 0) return CTP_OK;
    if (user) {
        if (user_bytes < need)
            return set_error(CTP_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu bytes required",
                             user_bytes, need);
        ptr_ = user;
        return CTP_OK;
    }
    int rc = scratch_alloc(&ptr_, need, s);
    if (rc) return rc;
    owned_ = true;
    return CTP_OK;
}

}  // namespace ctp

using namespace ctp;

namespace {

ctp_geometry make_geom(size_t nb, size_t nx, size_t ny, size_t nz, float dx, float dy, float dz, float cx, float cy,
                       float cz, size_t nu, size_t nv, size_t nview, float du, float dv, float off_u, float off_v,
                       float dsd, float dso) {
    ctp_geometry g;
    g.nbatch = nb;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.dx = dx; g.dy = dy; g.dz = dz;
    g.cx = cx; g.cy = cy; g.cz = cz;
    g.nu = nu; g.nv = nv; g.nview = nview;
    g.du = du; g.dv = dv; g.off_u = off_u; g.off_v = off_v;
    g.dsd = dsd; g.dso = dso;
    return g;
}

// Synchronous completion of a reference-compatible device-pointer call: the
// reference synchronises after every batch item and returns the last error.
int finish_sync(int rc, cudaStream_t s) {
    if (rc) return rc;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_error((int)e, "%s", cudaGetErrorString(e));
    return CTP_OK;
}

// Synchronous forward projections: a bounded device wait that gave up during
// the call (its CTA leaves its part of the output unwritten) is reported as
// CTP_ERR_WAIT_TIMEOUT, from the device counter read before and after.
struct WaitCheck {
    unsigned before = 0;
    bool armed = false;
    WaitCheck() { armed = wait_timeouts(&before) == CTP_OK; }
    int finish(int rc) {
        if (rc || !armed) return rc;
        unsigned after = before;
        if (wait_timeouts(&after) != CTP_OK) return CTP_OK;
        if (after != before)
            return set_error(CTP_ERR_WAIT_TIMEOUT,
                             "%u bounded device waits gave up during the forward projection; its output is "
                             "incomplete",
                             after - before);
        return CTP_OK;
    }
};

// Host-pointer call: pooled device buffers, copies in (through pinned
// staging chunks), op, copy out.
struct HostCall {
    cudaStream_t s = cudaStreamPerThread;
    void* bufs[8] = {nullptr};
    int n = 0;
    int rc = CTP_OK;
    template <typename T>
    T* dev(size_t count) {
        if (rc) return nullptr;
        void* p = nullptr;
        if ((rc = scratch_alloc(&p, count * sizeof(T) + 16, s))) return nullptr;
        bufs[n++] = p;
        return static_cast<T*>(p);
    }
    template <typename T>
    T* upload(const T* host, size_t count) {
        T* d = dev<T>(count);
        if (rc) return nullptr;
        rc = staged_upload(d, host, count * sizeof(T), s);
        return d;
    }
    template <typename T>
    T* zeros(size_t count) {
        T* d = dev<T>(count);
        if (rc) return nullptr;
        cudaError_t e = cudaMemsetAsync(d, 0, count * sizeof(T), s);
        if (e != cudaSuccess) rc = set_error((int)e, "memset: %s", cudaGetErrorString(e));
        return d;
    }
    template <typename T>
    void download(T* host, const T* d, size_t count) {
        if (rc) return;
        rc = staged_download(host, d, count * sizeof(T), s);
    }
    int finish() {
        for (int i = 0; i < n; ++i) cudaFreeAsync(bufs[i], s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (!rc && e != cudaSuccess) rc = set_error((int)e, "%s", cudaGetErrorString(e));
        return rc;
    }
};

}  // namespace

namespace ctp {
const char* last_error();
}

#define CTP_GEOM_ARGS                                                                                             \
    size_t nBatches, size_t nx, size_t ny, size_t nz, float dx, float dy, float dz, float cx, float cy, float cz, \
        size_t nu, size_t nv, size_t nview
#define CTP_GEOM(du_, dv_, ou_, ov_, dsd_, dso_) \
    make_geom(nBatches, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, nv, nview, du_, dv_, ou_, ov_, dsd_, dso_)

extern "C" {

const char* ctpGetLastErrorString(void) { return ctp::last_error(); }

const char* ctpVersion(void) { return "ctprojector_b200 0.1.0 (sm_100a)"; }

int SetDevice(int device) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return set_error((int)e, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    return CTP_OK;
}

// ------------------------------------------------------------ DD 2D (device)
static int dd_fp_dev(float* prj, const float* img, const float* deg, const ctp_geometry& g, int geom, int type) {
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    WaitCheck wc;
    return wc.finish(finish_sync(dd2d_fp(prj, img, deg, g, geom, type, 0, nullptr, 0, 0), 0));
}

static int dd_bp_dev(float* img, const float* prj, const float* deg, const ctp_geometry& g, int geom, int type) {
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    return finish_sync(dd2d_bp(img, prj, deg, g, geom, type, 0, nullptr, 0, 0), 0);
}

int cupyDistanceDrivenFanProjection(float* prj, const float* img, const float* deg, CTP_GEOM_ARGS, float da, float dv,
                                    float off_a, float off_v, float dsd, float dso, int typeProjector) {
    return dd_fp_dev(prj, img, deg, CTP_GEOM(da, dv, off_a, off_v, dsd, dso), 0, typeProjector);
}

int cupyDistanceDrivenParallelProjection(float* prj, const float* img, const float* deg, CTP_GEOM_ARGS, float du,
                                         float dv, float off_u, float off_v, int typeProjector) {
    return dd_fp_dev(prj, img, deg, CTP_GEOM(du, dv, off_u, off_v, 1000.f, 500.f), 1, typeProjector);
}

int cupyDistanceDrivenFanBackprojection(float* img, const float* prj, const float* deg, CTP_GEOM_ARGS, float da,
                                        float dv, float off_a, float off_v, float dsd, float dso, int typeProjector) {
    return dd_bp_dev(img, prj, deg, CTP_GEOM(da, dv, off_a, off_v, dsd, dso), 0, typeProjector);
}

int cupyDistanceDrivenParallelBackprojection(float* img, const float* prj, const float* deg, CTP_GEOM_ARGS, float du,
                                             float dv, float off_u, float off_v, int typeProjector) {
    return dd_bp_dev(img, prj, deg, CTP_GEOM(du, dv, off_u, off_v, 1000.f, 500.f), 1, typeProjector);
}

// ------------------------------------------------------------ DD 2D (host)
static int dd_fp_host(float* prj, const float* img, const float* deg, const ctp_geometry& g, int geom, int type) {
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    WaitCheck wc;
    HostCall hc;
    size_t ni = g.nbatch * g.nz * g.ny * g.nx, np = g.nbatch * g.nview * g.nv * g.nu;
    float* dimg = hc.upload(img, ni);
    float* ddeg = hc.upload(deg, g.nview);
    float* dprj = hc.dev<float>(np);
    if (!hc.rc) hc.rc = dd2d_fp(dprj, dimg, ddeg, g, geom, type, 0, nullptr, 0, hc.s);
    hc.download(prj, dprj, np);
    return wc.finish(hc.finish());
}

static int dd_bp_host(float* img, const float* prj, const float* deg, const ctp_geometry& g, int geom, int type) {
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    HostCall hc;
    size_t ni = g.nbatch * g.nz * g.ny * g.nx, np = g.nbatch * g.nview * g.nv * g.nu;
    float* dprj = hc.upload(prj, np);
    float* ddeg = hc.upload(deg, g.nview);
    float* dimg = hc.dev<float>(ni);
    if (!hc.rc) hc.rc = dd2d_bp(dimg, dprj, ddeg, g, geom, type, CTP_FLAG_ZERO_OUT, nullptr, 0, hc.s);
    hc.download(img, dimg, ni);
    return hc.finish();
}

int cDistanceDrivenFanProjection(float* prj, const float* img, const float* deg, CTP_GEOM_ARGS, float da, float dv,
                                 float off_a, float off_v, float dsd, float dso, int typeProjector) {
    return dd_fp_host(prj, img, deg, CTP_GEOM(da, dv, off_a, off_v, dsd, dso), 0, typeProjector);
}

int cDistanceDrivenParallelProjection(float* prj, const float* img, const float* deg, CTP_GEOM_ARGS, float du,
                                      float dv, float off_u, float off_v, int typeProjector) {
    return dd_fp_host(prj, img, deg, CTP_GEOM(du, dv, off_u, off_v, 1000.f, 500.f), 1, typeProjector);
}

int cDistanceDrivenFanBackprojection(float* img, const float* prj, const float* deg, CTP_GEOM_ARGS, float da,
                                     float dv, float off_a, float off_v, float dsd, float dso, int typeProjector) {
    return dd_bp_host(img, prj, deg, CTP_GEOM(da, dv, off_a, off_v, dsd, dso), 0, typeProjector);
}

int cDistanceDrivenParallelBackprojection(float* img, const float* prj, const float* deg, CTP_GEOM_ARGS, float du,
                                          float dv, float off_u, float off_v, int typeProjector) {
    return dd_bp_host(img, prj, deg, CTP_GEOM(du, dv, off_u, off_v, 1000.f, 500.f), 1, typeProjector);
}

// ------------------------------------------------------------ tomo
int cupyDistanceDrivenTomoProjection(float* prj, const float* img, const float* detCenter, const float* src,
                                     CTP_GEOM_ARGS, float du, float dv, float off_u, float off_v, int) {
    ctp_geometry g = CTP_GEOM(du, dv, off_u, off_v, 0.f, 0.f);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !detCenter || !src) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    return finish_sync(tomo_fp(prj, img, detCenter, src, g, 0, 0), 0);
}

int cupyDistanceDrivenTomoBackprojection(float* img, const float* prj, const float* detCenter, const float* src,
                                         CTP_GEOM_ARGS, float du, float dv, float off_u, float off_v, int) {
    ctp_geometry g = CTP_GEOM(du, dv, off_u, off_v, 0.f, 0.f);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !detCenter || !src) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    return finish_sync(tomo_bp(img, prj, detCenter, src, g, 0, nullptr, 0, 0), 0);
}

int cDistanceDrivenTomoProjection(float* prj, const float* img, const float* detCenter, const float* src,
                                  CTP_GEOM_ARGS, float du, float dv, float off_u, float off_v, int) {
    ctp_geometry g = CTP_GEOM(du, dv, off_u, off_v, 0.f, 0.f);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !detCenter || !src) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    HostCall hc;
    size_t ni = g.nbatch * g.nz * g.ny * g.nx, np = g.nbatch * g.nview * g.nv * g.nu;
    float* dimg = hc.upload(img, ni);
    float* dc = hc.upload(detCenter, 3 * g.nview);
    float* ds = hc.upload(src, 3 * g.nview);
    float* dprj = hc.dev<float>(np);
    if (!hc.rc) hc.rc = tomo_fp(dprj, dimg, dc, ds, g, 0, hc.s);
    hc.download(prj, dprj, np);
    return hc.finish();
}

int cDistanceDrivenTomoBackprojection(float* img, const float* prj, const float* detCenter, const float* src,
                                      CTP_GEOM_ARGS, float du, float dv, float off_u, float off_v, int) {
    ctp_geometry g = CTP_GEOM(du, dv, off_u, off_v, 0.f, 0.f);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !detCenter || !src) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    HostCall hc;
    size_t ni = g.nbatch * g.nz * g.ny * g.nx, np = g.nbatch * g.nview * g.nv * g.nu;
    float* dprj = hc.upload(prj, np);
    float* dc = hc.upload(detCenter, 3 * g.nview);
    float* ds = hc.upload(src, 3 * g.nview);
    float* dimg = hc.dev<float>(ni);
    if (!hc.rc) hc.rc = tomo_bp(dimg, dprj, dc, ds, g, 0, nullptr, 0, hc.s);
    hc.download(img, dimg, ni);
    return hc.finish();
}

// ------------------------------------------------------------ Siddon cone
#define SIDDON_ARGS                                                                                              \
    const float *detCenter, const float *detU, const float *detV, const float *src, CTP_GEOM_ARGS, float du, \
        float dv, float off_u, float off_v

int cupySiddonConeProjectionArbitrary(float* prj, const float* img, SIDDON_ARGS) {
    ctp_geometry g = CTP_GEOM(du, dv, off_u, off_v, 0.f, 0.f);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !detCenter || !detU || !detV || !src)
        return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    return finish_sync(siddon_fp(prj, img, detCenter, detU, detV, src, g, 0, 0), 0);
}

int cupySiddonConeBackprojectionArbitrary(float* img, const float* prj, SIDDON_ARGS) {
    ctp_geometry g = CTP_GEOM(du, dv, off_u, off_v, 0.f, 0.f);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !detCenter || !detU || !detV || !src)
        return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    return finish_sync(siddon_bp(img, prj, detCenter, detU, detV, src, g, 0, 0), 0);
}

int cSiddonConeProjectionArbitrary(float* prj, const float* img, SIDDON_ARGS) {
    ctp_geometry g = CTP_GEOM(du, dv, off_u, off_v, 0.f, 0.f);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !detCenter || !detU || !detV || !src)
        return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    HostCall hc;
    size_t ni = g.nbatch * g.nz * g.ny * g.nx, np = g.nbatch * g.nview * g.nv * g.nu;
    float* dimg = hc.upload(img, ni);
    float* dc = hc.upload(detCenter, 3 * g.nview);
    float* du_ = hc.upload(detU, 3 * g.nview);
    float* dv_ = hc.upload(detV, 3 * g.nview);
    float* ds = hc.upload(src, 3 * g.nview);
    float* dprj = hc.dev<float>(np);
    if (!hc.rc) hc.rc = siddon_fp(dprj, dimg, dc, du_, dv_, ds, g, CTP_FLAG_ZERO_OUT, hc.s);
    hc.download(prj, dprj, np);
    return hc.finish();
}

int cSiddonConeBackprojectionArbitrary(float* img, const float* prj, SIDDON_ARGS) {
    ctp_geometry g = CTP_GEOM(du, dv, off_u, off_v, 0.f, 0.f);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!prj || !img || !detCenter || !detU || !detV || !src)
        return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    HostCall hc;
    size_t ni = g.nbatch * g.nz * g.ny * g.nx, np = g.nbatch * g.nview * g.nv * g.nu;
    float* dprj = hc.upload(prj, np);
    float* dc = hc.upload(detCenter, 3 * g.nview);
    float* du_ = hc.upload(detU, 3 * g.nview);
    float* dv_ = hc.upload(detV, 3 * g.nview);
    float* ds = hc.upload(src, 3 * g.nview);
    float* dimg = hc.dev<float>(ni);
    if (!hc.rc) hc.rc = siddon_bp(dimg, dprj, dc, du_, dv_, ds, g, CTP_FLAG_ZERO_OUT, hc.s);
    hc.download(img, dimg, ni);
    return hc.finish();
}

// ------------------------------------------------------------ filters and fbp_bp
static int filter_dev(float* out, const float* in, const ctp_geometry& g, int geom, int filter, cudaStream_t s) {
    int rc = check_geometry(&g, false, true);
    if (rc) return rc;
    if (!out || !in) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    return ramp_filter(out, in, g, geom, filter, 0, nullptr, 0, s);
}

static ctp_geometry filter_geom(int nBatches, size_t nu, size_t nv, size_t nview, float du, float dv, float off_u,
                                float off_v, float dsd, float dso) {
    return make_geom(nBatches < 0 ? 0 : (size_t)nBatches, 1, 1, 1, 1, 1, 1, 0, 0, 0, nu, nv, nview, du, dv, off_u,
                     off_v, dsd, dso);
}

int cupyfbpFanFilter(float* pFPrj, const float* pPrj, int nBatches, size_t nu, size_t nv, size_t nview, float da,
                     float dv, float off_a, float off_v, float dsd, float dso, int typeFilter) {
    ctp_geometry g = filter_geom(nBatches, nu, nv, nview, da, dv, off_a, off_v, dsd, dso);
    return finish_sync(filter_dev(pFPrj, pPrj, g, 0, typeFilter, 0), 0);
}

int cupyfbpParallelFilter(float* pFPrj, const float* pPrj, int nBatches, size_t nu, size_t nv, size_t nview,
                          float du, float dv, float off_u, float off_v, int typeFilter) {
    ctp_geometry g = filter_geom(nBatches, nu, nv, nview, du, dv, off_u, off_v, 0.f, 0.f);
    return finish_sync(filter_dev(pFPrj, pPrj, g, 1, typeFilter, 0), 0);
}

static int filter_host(float* out, const float* in, const ctp_geometry& g, int geom, int filter,
                       unsigned flags = 0) {
    int rc = check_geometry(&g, false, true);
    if (rc) return rc;
    if (!out || !in) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    HostCall hc;
    size_t np = g.nbatch * g.nview * g.nv * g.nu;
    float* din = hc.upload(in, np);
    float* dout = hc.dev<float>(np);
    if (!hc.rc) hc.rc = ramp_filter(dout, din, g, geom, filter, flags, nullptr, 0, hc.s);
    hc.download(out, dout, np);
    return hc.finish();
}

int cfbpFanFilter(float* pFPrj, const float* pPrj, int nBatches, size_t nu, size_t nv, size_t nview, float da,
                  float dv, float off_a, float off_v, float dsd, float dso, int typeFilter) {
    return filter_host(pFPrj, pPrj, filter_geom(nBatches, nu, nv, nview, da, dv, off_a, off_v, dsd, dso), 0,
                       typeFilter);
}

int cfbpParallelFilter(float* pFPrj, const float* pPrj, int nBatches, size_t nu, size_t nv, size_t nview, float du,
                       float dv, float off_u, float off_v, int typeFilter) {
    return filter_host(pFPrj, pPrj, filter_geom(nBatches, nu, nv, nview, du, dv, off_u, off_v, 0.f, 0.f), 1,
                       typeFilter);
}

int cupyfbpFanBackprojection(float* pImg, const float* pPrj, const float* pDeg, CTP_GEOM_ARGS, float da, float dv,
                             float off_a, float off_v, float dsd, float dso) {
    ctp_geometry g = CTP_GEOM(da, dv, off_a, off_v, dsd, dso);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!pImg || !pPrj || !pDeg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    return finish_sync(fbp_fan_bp(pImg, pPrj, pDeg, g, 0, 0), 0);
}

int cfbpFanBackprojection(float* pImg, const float* pPrj, const float* pDeg, CTP_GEOM_ARGS, float da, float dv,
                          float off_a, float off_v, float dsd, float dso) {
    ctp_geometry g = CTP_GEOM(da, dv, off_a, off_v, dsd, dso);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!pImg || !pPrj || !pDeg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    HostCall hc;
    size_t ni = g.nbatch * g.nz * g.ny * g.nx, np = g.nbatch * g.nview * g.nv * g.nu;
    float* dprj = hc.upload(pPrj, np);
    float* ddeg = hc.upload(pDeg, g.nview);
    float* dimg = hc.dev<float>(ni);
    if (!hc.rc) hc.rc = fbp_fan_bp(dimg, dprj, ddeg, g, CTP_FLAG_ZERO_OUT, hc.s);
    hc.download(pImg, dimg, ni);
    return hc.finish();
}

// Fan-beam Siddon pair, host pointers (siddonFan.cu:127-274; nBatches is an
// int there).  The reference zeroes the device output before tracing.
static int siddon_fan_host(bool fp, float* out, const float* in, const float* deg, int nBatches, size_t nx, size_t ny,
                           size_t nz, float dx, float dy, float dz, float cx, float cy, float cz, size_t nu, size_t nv,
                           size_t nview, float da, float dv, float off_a, float off_v, float dsd, float dso) {
    if (nBatches < 0) return set_error(CTP_ERR_INVALID_ARGUMENT, "negative batch count");
    ctp_geometry g = make_geom((size_t)nBatches, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, nv, nview, da, dv, off_a,
                               off_v, dsd, dso);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!out || !in || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    HostCall hc;
    size_t ni = g.nbatch * g.nz * g.ny * g.nx, np = g.nbatch * g.nview * g.nv * g.nu;
    float* din = hc.upload(in, fp ? ni : np);
    float* ddeg = hc.upload(deg, g.nview);
    float* dout = hc.dev<float>(fp ? np : ni);
    if (!hc.rc)
        hc.rc = fp ? siddon_fan_fp(dout, din, ddeg, g, CTP_FLAG_ZERO_OUT, hc.s)
                   : siddon_fan_bp(dout, din, ddeg, g, CTP_FLAG_ZERO_OUT, hc.s);
    hc.download(out, dout, fp ? np : ni);
    return hc.finish();
}

int cSiddonFanProjection(float* prj, const float* img, const float* deg, int nBatches, size_t nx, size_t ny,
                         size_t nz, float dx, float dy, float dz, float cx, float cy, float cz, size_t nu, size_t nv,
                         size_t nview, float da, float dv, float off_a, float off_v, float dsd, float dso) {
    return siddon_fan_host(true, prj, img, deg, nBatches, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, nv, nview, da, dv,
                           off_a, off_v, dsd, dso);
}

int cSiddonFanBackprojection(float* img, const float* prj, const float* deg, int nBatches, size_t nx, size_t ny,
                             size_t nz, float dx, float dy, float dz, float cx, float cy, float cz, size_t nu,
                             size_t nv, size_t nview, float da, float dv, float off_a, float off_v, float dsd,
                             float dso) {
    return siddon_fan_host(false, img, prj, deg, nBatches, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, nv, nview, da, dv,
                           off_a, off_v, dsd, dso);
}

// Pixel-driven parallel back projection, host pointers (fbpParallel.cu:271-345).
int cfbpParallelBackprojection(float* pImg, const float* pPrj, const float* pDeg, CTP_GEOM_ARGS, float du, float dv,
                               float off_u, float off_v, int typeProjector) {
    (void)typeProjector;  // the reference reads no bit of it here
    ctp_geometry g = CTP_GEOM(du, dv, off_u, off_v, 1000.f, 500.f);
    int rc = check_geometry(&g, true, true);
    if (rc) return rc;
    if (!pImg || !pPrj || !pDeg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nbatch == 0) return CTP_OK;
    HostCall hc;
    size_t ni = g.nbatch * g.nz * g.ny * g.nx, np = g.nbatch * g.nview * g.nv * g.nu;
    float* dprj = hc.upload(pPrj, np);
    float* ddeg = hc.upload(pDeg, g.nview);
    float* dimg = hc.dev<float>(ni);
    if (!hc.rc) hc.rc = pixel_bp_parallel(dimg, dprj, ddeg, g, CTP_FLAG_ZERO_OUT, hc.s);
    hc.download(pImg, dimg, ni);
    return hc.finish();
}

// ============================================================ extended entries
static cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int ctp_siddon_fan_fp(float* prj, const float* img, const float* deg, const ctp_geometry* g, unsigned flags,
                      void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!prj || !img || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return siddon_fan_fp(prj, img, deg, *g, flags, as_stream(stream));
}

int ctp_siddon_fan_bp(float* img, const float* prj, const float* deg, const ctp_geometry* g, unsigned flags,
                      void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!prj || !img || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return siddon_fan_bp(img, prj, deg, *g, flags, as_stream(stream));
}

int ctp_pixel_bp_parallel(float* img, const float* prj, const float* deg, const ctp_geometry* g, unsigned flags,
                          void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!prj || !img || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return pixel_bp_parallel(img, prj, deg, *g, flags, as_stream(stream));
}

int ctp_dd2d_fp(void* prj, const void* img, const float* deg, const ctp_geometry* g, int geom, int typeProjector,
                unsigned flags, void* workspace, size_t workspace_bytes, void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!prj || !img || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return dd2d_fp(prj, img, deg, *g, geom, typeProjector, flags, workspace, workspace_bytes, as_stream(stream));
}

size_t ctp_dd2d_fp_workspace(const ctp_geometry* g, int geom, int typeProjector, unsigned flags) {
    return g ? dd2d_fp_workspace(*g, geom, typeProjector, flags) : 0;
}

int ctp_dd2d_bp(void* img, const void* prj, const float* deg, const ctp_geometry* g, int geom, int typeProjector,
                unsigned flags, void* workspace, size_t workspace_bytes, void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!prj || !img || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return dd2d_bp(img, prj, deg, *g, geom, typeProjector, flags, workspace, workspace_bytes, as_stream(stream));
}

size_t ctp_dd2d_bp_workspace(const ctp_geometry* g, int geom, int typeProjector, unsigned flags) {
    return g ? dd2d_bp_workspace(*g, geom, typeProjector, flags) : 0;
}

int ctp_dd2d_fp_noalloc(void* prj, const void* img, const float* deg, const ctp_geometry* g, int geom,
                        int typeProjector, unsigned flags, void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!prj || !img || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return dd2d_fp_noalloc(prj, img, deg, *g, geom, typeProjector, flags, as_stream(stream));
}

size_t ctp_dd2d_fp_noalloc_capacity(void) { return dd2d_fp_noalloc_capacity(); }

int ctp_dd2d_nnz(unsigned long long* nnz_host, const float* deg, const ctp_geometry* g, int geom, void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (!deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null angle pointer");
    return dd2d_nnz(nnz_host, deg, *g, geom, as_stream(stream));
}

int ctp_ramp_filter(float* fprj, const float* prj, const ctp_geometry* g, int geom, int typeFilter, unsigned flags,
                    void* workspace, size_t workspace_bytes, void* stream) {
    int rc = check_geometry(g, false, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!fprj || !prj) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return ramp_filter(fprj, prj, *g, geom, typeFilter, flags, workspace, workspace_bytes, as_stream(stream));
}

int ctp_ramp_filter_host(float* fprj, const float* prj, const ctp_geometry* g, int geom, int typeFilter,
                         unsigned flags) {
    if (!g) return set_error(CTP_ERR_INVALID_ARGUMENT, "geometry pointer is null");
    if (geom != 0 && geom != 1) return set_error(CTP_ERR_INVALID_ARGUMENT, "geom must be 0 (fan) or 1 (parallel)");
    return filter_host(fprj, prj, *g, geom, typeFilter, flags);
}

size_t ctp_ramp_filter_workspace(const ctp_geometry* g, int geom, int typeFilter, unsigned flags) {
    return g ? ramp_filter_workspace(*g, geom, typeFilter, flags) : 0;
}

int ctp_fbp_fan_bp(float* img, const float* prj, const float* deg, const ctp_geometry* g, unsigned flags,
                   void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!img || !prj || !deg) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return fbp_fan_bp(img, prj, deg, *g, flags, as_stream(stream));
}

int ctp_siddon_fp(void* prj, const void* img, const float* detCenter, const float* detU, const float* detV,
                  const float* src, const ctp_geometry* g, unsigned flags, void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!prj || !img || !detCenter || !detU || !detV || !src)
        return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return siddon_fp(prj, img, detCenter, detU, detV, src, *g, flags, as_stream(stream));
}

int ctp_siddon_bp(void* img, const void* prj, const float* detCenter, const float* detU, const float* detV,
                  const float* src, const ctp_geometry* g, unsigned flags, void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!prj || !img || !detCenter || !detU || !detV || !src)
        return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return siddon_bp(img, prj, detCenter, detU, detV, src, *g, flags, as_stream(stream));
}

int ctp_siddon_nnz(unsigned long long* nnz_host, const float* detCenter, const float* detU, const float* detV,
                   const float* src, const ctp_geometry* g, void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (!detCenter || !detU || !detV || !src) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return siddon_nnz(nnz_host, detCenter, detU, detV, src, *g, as_stream(stream));
}

int ctp_tomo_fp(float* prj, const float* img, const float* detCenter, const float* src, const ctp_geometry* g,
                unsigned flags, void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!prj || !img || !detCenter || !src) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return tomo_fp(prj, img, detCenter, src, *g, flags, as_stream(stream));
}

int ctp_tomo_bp(float* img, const float* prj, const float* detCenter, const float* src, const ctp_geometry* g,
                unsigned flags, void* workspace, size_t workspace_bytes, void* stream) {
    int rc = check_geometry(g, true, true);
    if (rc) return rc;
    if (g->nbatch == 0) return CTP_OK;
    if (!prj || !img || !detCenter || !src) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    return tomo_bp(img, prj, detCenter, src, *g, flags, workspace, workspace_bytes, as_stream(stream));
}

size_t ctp_tomo_bp_workspace(const ctp_geometry* g) { return g ? tomo_bp_workspace(*g) : 0; }

// ------------------------------------------------------------ TV prior
int cupyTVSQS3D(float* s1, float* s2, float* var, const float* img, float wx, float wy, float wz, size_t nBatches,
                size_t nx, size_t ny, size_t nz, float eps) {
    return finish_sync(tv_sqs(s1, s2, var, img, wx, wy, wz, nBatches, nx, ny, nz, eps, 0), 0);
}

int cTVSQS3D(float* s1, float* s2, float* var, const float* img, float wx, float wy, float wz, size_t nBatches,
             size_t nx, size_t ny, size_t nz, float eps) {
    if (nBatches == 0) return CTP_OK;
    if (!s1 || !s2 || !var || !img) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    HostCall hc;
    size_t n = nBatches * nx * ny * nz;
    float* dimg = hc.upload(img, n);
    float* d1 = hc.dev<float>(n);
    float* d2 = hc.dev<float>(n);
    float* dv = hc.dev<float>(n);
    if (!hc.rc) hc.rc = tv_sqs(d1, d2, dv, dimg, wx, wy, wz, nBatches, nx, ny, nz, eps, hc.s);
    hc.download(s1, d1, n);
    hc.download(s2, d2, n);
    hc.download(var, dv, n);
    return hc.finish();
}

int ctp_tv_sqs(float* s1, float* s2, float* var, const float* img, float wx, float wy, float wz, size_t nbatch,
               size_t nx, size_t ny, size_t nz, float eps, void* stream) {
    return tv_sqs(s1, s2, var, img, wx, wy, wz, nbatch, nx, ny, nz, eps, as_stream(stream));
}

int ctp_sqs_tv_update(float* x_out, void* x_lp, const float* x, const float* bp, const float* norm,
                      size_t norm_slices, const unsigned char* zlink, float wx, float wy, float wz, float beta,
                      float eps, size_t nx, size_t ny, size_t nslices, unsigned flags, void* stream) {
    return sqs_tv_update(x_out, x_lp, x, bp, norm, norm_slices, zlink, wx, wy, wz, beta, eps, nx, ny, nslices, flags,
                         as_stream(stream));
}

int ctp_wait_timeouts(unsigned int* count) { return wait_timeouts(count); }

int ctp_set_wait_limit(unsigned int first_chunk_polls) { return set_first_wait_polls(first_chunk_polls); }

int ctp_set_fp_stream_slices(int max_slices) {
    set_fp_stream_cap(max_slices);
    return CTP_OK;
}

int ctp_quantize_u16(unsigned short* code, float* lo, float* step, const float* y, size_t nrows, size_t row_len,
                     void* stream) {
    return quantize_u16(code, lo, step, y, nrows, row_len, as_stream(stream));
}

int ctp_dequantize_u16(float* y, const unsigned short* code, const float* lo, const float* step, size_t nrows,
                       size_t row_len, unsigned flags, void* stream) {
    return dequantize_u16(y, code, lo, step, nrows, row_len, (flags & CTP_FLAG_SUBTRACT) != 0, as_stream(stream));
}

int ctp_ramp_filter_u16(float* fprj, const unsigned short* code, const float* lo, const float* step,
                        const ctp_geometry* g, int geom, int typeFilter, void* stream) {
    int rc = check_geometry(g, false, true);
    if (rc) return rc;
    if (!fprj || !code || !lo || !step) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g->nbatch == 0) return CTP_OK;
    return ramp_filter_u16(fprj, code, lo, step, *g, geom, typeFilter, as_stream(stream));
}

int ctp_scratch_allocations(unsigned long long* count) {
    if (!count) return set_error(CTP_ERR_INVALID_ARGUMENT, "count pointer is null");
    *count = scratch_allocations();
    return CTP_OK;
}

int cupyFbpTomoFilter(float* fprj, const float* prj, const float* detCenter, const float* src, int nBatches,
                      size_t nu, size_t nv, size_t nview, float du, float dx, float dz, int typeFilter,
                      float cutoffX, float cutoffZ) {
    if (nBatches < 0) return set_error(CTP_ERR_INVALID_ARGUMENT, "negative batch count");
    ctp_geometry g = make_geom((size_t)nBatches, 1, 1, 1, dx, 1.f, dz, 0.f, 0.f, 0.f, nu, nv, nview, du, 1.f, 0.f, 0.f,
                               0.f, 0.f);
    return finish_sync(tomo_filter(fprj, prj, detCenter, src, g, typeFilter, cutoffX, cutoffZ, 0, nullptr, 0, 0), 0);
}

int ctp_tomo_filter(float* fprj, const float* prj, const float* detCenter, const float* src, const ctp_geometry* g,
                    int filter, float cutoff_x, float cutoff_z, unsigned flags, void* workspace,
                    size_t workspace_bytes, void* stream) {
    if (!g) return set_error(CTP_ERR_INVALID_ARGUMENT, "geometry pointer is null");
    return tomo_filter(fprj, prj, detCenter, src, *g, filter, cutoff_x, cutoff_z, flags, workspace, workspace_bytes,
                       as_stream(stream));
}

size_t ctp_tomo_filter_workspace(const ctp_geometry* g) { return g ? tomo_filter_workspace(*g) : 0; }

}  // extern "C"
