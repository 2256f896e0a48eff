// fbp.cu -- ramp filtering (parallel / equiangular fan) and the pixel-driven
// fan FBP back projector for sm_100a.
//
// Ramp filter (reference: GetRamp fbpMath.cu:90-267, fbpParallel::Filter
// fbpParallel.cu:14-109, fbpFan::Filter fbp.cu:15-162).  The reference builds a
// spatial ramp h of length L = 2nu-1 (offset k = i-(nu-1)), applies the window
// in the L-point frequency domain, and convolves every zero-padded detector
// row with the result, keeping outputs nu-1 .. 2nu-2.  That is the linear
// convolution
//      out[i] = scale * sum_j p[j] g[i-j],   g = real(IDFT_L(DFT_L(h) W)),
// which this file evaluates as a circular convolution of size N >= 2nu-1
// (N = 2^a 3^b), exact because g has support [-(nu-1), nu-1]:
//   * g is computed once per (nu, da, window, geometry) on the host in FP64
//     and its N-point spectrum (real: g is even) cached on the device;
//   * the transforms and the spectrum product run in FP64 (this path is the
//     accuracy reference; the default path replays the reference's FP32
//     construction further below);
//   * one pad/weight kernel writes all rows of the batch into an in-place
//     R2C layout, cuFFT runs batched R2C and C2R over every row at once, a
//     multiply kernel scales the spectrum, and a crop kernel writes the first
//     nu samples of each row.
#include <cufft.h>
#include <cmath>
#include <cuda_runtime.h>
#include <math.h>

#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "ctp_common.cuh"

namespace ctp {

namespace {

int fft_size(int nu) {
    int need = 2 * nu - 1, best = 1 << 30;
    for (long p2 = 1; p2 < (1L << 30); p2 *= 2)
        for (long p3 = p2; p3 < (1L << 30); p3 *= 3) {
            if (p3 >= need && p3 < best) best = (int)p3;
            if (p3 >= need) break;
        }
    return best;
}

// Windowed ramp g[k], k = 0..nu-1 (g is even), FP64, following GetRamp.
std::vector<double> ramp_kernel(int nu, double da, int filter, bool equiangular) {
    const int L = 2 * nu - 1;
    std::vector<double> h(L), w(L), cosL(L), sinL(L);
    for (int i = 0; i < L; ++i) {
        long k = (long)i - (nu - 1);
        if (k == 0)
            h[i] = 1.0 / (4 * da * da);
        else if (k % 2 != 0)
            h[i] = equiangular ? -1.0 / (M_PI * M_PI * sin(k * da) * sin(k * da))
                               : -1.0 / (M_PI * M_PI * (double)k * (double)k * da * da);
        else
            h[i] = 0;
        double t = 2 * M_PI * i / L;
        switch (filter) {  // fbpMath.cu:178-208
            case 1: w[i] = 0.54 + 0.46 * cos(t); break;
            case 2: w[i] = 0.5 + 0.5 * cos(t); break;
            case 3: w[i] = fabs(cos(M_PI * i / L)); break;
            default: w[i] = 1.0;
        }
        cosL[i] = cos(t);
        sinL[i] = sin(t);
    }
    // H = DFT_L(h);  g = real(IDFT_L(H .* w)) / L
    std::vector<double> Hr(L), Hi(L);
    for (int m = 0; m < L; ++m) {
        double re = 0, im = 0;
        long idx = 0;
        for (int n = 0; n < L; ++n) {
            re += h[n] * cosL[idx];
            im -= h[n] * sinL[idx];
            idx += m;
            if (idx >= L) idx -= L;
        }
        Hr[m] = re * w[m];
        Hi[m] = im * w[m];
    }
    std::vector<double> g(nu);
    for (int k = 0; k < nu; ++k) {
        // average of offsets +k and -k (exactly equal in exact arithmetic)
        double acc = 0;
        for (int sgn = -1; sgn <= 1; sgn += 2) {
            long n = (long)(nu - 1) + sgn * k;
            double re = 0;
            long idx = 0;
            for (int m = 0; m < L; ++m) {
                re += Hr[m] * cosL[idx] - Hi[m] * sinL[idx];
                idx += n;
                idx %= L;
            }
            acc += re / L;
            if (k == 0) { acc *= 2; break; }
        }
        g[k] = acc / 2;
    }
    return g;
}

struct Spectrum {
    double* dev = nullptr;  // N/2+1 real coefficients
    int n = 0;
};

std::mutex g_spec_mu;
std::map<std::tuple<int, int, long long, int, int, int>, Spectrum> g_spec;

// Device spectrum of g for this (device, nu, da, filter, kind, N); built once.
int get_spectrum(int nu, double da, int filter, bool equiangular, int N, const double** out) {
    int dev = 0;
    cudaGetDevice(&dev);
    long long dkey;
    memcpy(&dkey, &da, sizeof(dkey));
    auto key = std::make_tuple(dev, nu, dkey, filter, (int)equiangular, N);
    std::lock_guard<std::mutex> lk(g_spec_mu);
    auto it = g_spec.find(key);
    if (it != g_spec.end()) {
        *out = it->second.dev;
        return CTP_OK;
    }
    std::vector<double> g = ramp_kernel(nu, da, filter, equiangular);
    int M = N / 2 + 1;
    std::vector<double> G(M);
    std::vector<double> cosN(N);
    for (int i = 0; i < N; ++i) cosN[i] = cos(2 * M_PI * i / N);
    for (int m = 0; m < M; ++m) {
        double acc = g[0];
        long long idx = 0;
        for (int k = 1; k < nu; ++k) {
            idx += m;
            if (idx >= N) idx -= N;
            acc += 2 * g[k] * cosN[idx];
        }
        G[m] = acc;
    }
    Spectrum sp;
    sp.n = M;
    cudaError_t e = cudaMalloc(&sp.dev, sizeof(double) * M);  // one-time table, kept for the process
    if (e == cudaSuccess) e = cudaMemcpy(sp.dev, G.data(), sizeof(double) * M, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_error((int)e, "ramp spectrum upload: %s", cudaGetErrorString(e));
    g_spec[key] = sp;
    *out = sp.dev;
    return CTP_OK;
}

struct Plan {
    cufftHandle fwd = 0, inv = 0;
    size_t work = 0;
    std::mutex mu;
};

std::mutex g_plan_mu;
std::map<std::tuple<int, int, int>, std::unique_ptr<Plan>> g_plans;

int get_plan(int N, int batch, Plan** out) {
    int dev = 0;
    cudaGetDevice(&dev);
    auto key = std::make_tuple(dev, N, batch);
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_plans.find(key);
    if (it != g_plans.end()) {
        *out = it->second.get();
        return CTP_OK;
    }
    std::unique_ptr<Plan> p(new Plan());
    int n[1] = {N};
    int rembed[1] = {2 * (N / 2 + 1)}, cembed[1] = {N / 2 + 1};
    size_t w1 = 0, w2 = 0;
    if (cufftCreate(&p->fwd) != CUFFT_SUCCESS || cufftCreate(&p->inv) != CUFFT_SUCCESS)
        return set_error(CTP_ERR_CUFFT, "cufftCreate failed");
    cufftSetAutoAllocation(p->fwd, 0);
    cufftSetAutoAllocation(p->inv, 0);
    if (cufftMakePlanMany(p->fwd, 1, n, rembed, 1, rembed[0], cembed, 1, cembed[0], CUFFT_D2Z, batch, &w1) !=
            CUFFT_SUCCESS ||
        cufftMakePlanMany(p->inv, 1, n, cembed, 1, cembed[0], rembed, 1, rembed[0], CUFFT_Z2D, batch, &w2) !=
            CUFFT_SUCCESS)
        return set_error(CTP_ERR_CUFFT, "cufftMakePlanMany failed (N=%d, batch=%d)", N, batch);
    p->work = w1 > w2 ? w1 : w2;
    *out = p.get();
    g_plans[key] = std::move(p);
    return CTP_OK;
}

constexpr int kMaxRowsPerExec = 32768;

// Zero-pad and pre-weight rows (FP64) into the in-place D2Z layout.
__global__ void pad_kernel(double* __restrict__ buf, const float* __restrict__ prj, int nu, int N, int stride,
                           size_t rows, int fan, double da, double off_u) {
    size_t r = blockIdx.y + (size_t)blockIdx.z * gridDim.y;
    if (r >= rows) return;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < stride; n += gridDim.x * blockDim.x) {
        double v = 0.0;
        if (n < nu) {
            v = (double)prj[r * nu + n];
            if (fan) v *= cos(((n - (nu - 1) / 2.0) - off_u) * da);  // fbp.cu:62-66
        }
        buf[r * stride + n] = v;
    }
}

__global__ void spectrum_mul_kernel(double2* __restrict__ spec, const double* __restrict__ G, int M, size_t rows,
                                    double scale) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= rows * M) return;
    double g = G[i % M] * scale;
    double2 v = spec[i];
    spec[i] = make_double2(v.x * g, v.y * g);
}

__global__ void crop_kernel(float* __restrict__ out, const double* __restrict__ buf, int nu, int stride, size_t rows) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= rows * nu) return;
    size_t r = i / nu;
    int n = (int)(i - r * nu);
    out[i] = (float)buf[r * stride + n];
}

// ------------------------------------------------------------------ reference construction
// The reference builds the windowed ramp in FP32 (GetRamp, fbpMath.cu:90-241):
// float spatial ramp on the host, length-L C2C FFT, float window product on
// the host, inverse C2C, real part / L, length-L R2C.  Rows are then filtered
// with length-L R2C/C2R transforms in batches of nview rows
// (fbpParallel.cu:44-86, fbp.cu:81-134).  Replaying those steps in the same
// float operation order keeps the output within FP32 rounding of the
// reference.
struct RefFilter {
    cufftComplex* spec = nullptr;  // [nu] frequency kernel
    float* weight = nullptr;       // [nu] fan pre-weight (cos), or null
};

std::mutex g_ref_mu;
std::map<std::tuple<int, int, unsigned, int, int, unsigned>, RefFilter> g_ref;

int build_ref_filter(int nu, float da, int filter, bool fan, float off_u, RefFilter* out) {
    const int L = 2 * nu - 1;
    const float PIf = 3.141592657f;  // projector.h:5
    std::vector<cufftComplex> ramp(L), win(L);
    for (int i = 0; i < L; i++) {
        int k = i - (nu - 1);
        if (k == 0)
            ramp[i].x = 1 / (4 * da * da);
        else if (k % 2 != 0)
            ramp[i].x = fan ? -1 / (PIf * PIf * sinf(k * da) * sinf(k * da)) : -1 / (PIf * PIf * k * k * da * da);
        else
            ramp[i].x = 0;
        ramp[i].y = 0;
        switch (filter) {
            case 1: win[i].x = 0.54f + 0.46f * cosf(2 * PIf * i / (float)L); break;
            case 2: win[i].x = 0.5f + 0.5f * cosf(2 * PIf * i / (float)L); break;
            case 3: win[i].x = fabsf(cosf(PIf * i / (float)L)); break;
            default: win[i].x = 1;
        }
        win[i].y = 0;
    }
    cufftHandle c2c = 0, r2c = 0;
    cufftComplex* d = nullptr;
    float* dk = nullptr;
    int rc = CTP_OK;
    // one-time table construction for this geometry; kept for the process
    if (cudaMalloc(&d, sizeof(cufftComplex) * L) != cudaSuccess || cudaMalloc(&dk, sizeof(float) * L) != cudaSuccess ||
        cudaMalloc(&out->spec, sizeof(cufftComplex) * nu) != cudaSuccess)
        rc = set_error(cudaErrorMemoryAllocation, "ramp table allocation failed");
    if (!rc && (cufftPlan1d(&c2c, L, CUFFT_C2C, 1) != CUFFT_SUCCESS || cufftPlan1d(&r2c, L, CUFFT_R2C, 1) != CUFFT_SUCCESS))
        rc = set_error(CTP_ERR_CUFFT, "ramp table plan failed");
    if (!rc) {
        cudaMemcpy(d, ramp.data(), sizeof(cufftComplex) * L, cudaMemcpyHostToDevice);
        cufftExecC2C(c2c, d, d, CUFFT_FORWARD);
        cudaMemcpy(ramp.data(), d, sizeof(cufftComplex) * L, cudaMemcpyDeviceToHost);
        for (int i = 0; i < L; i++) {
            float re = ramp[i].x * win[i].x - ramp[i].y * win[i].y;
            float im = ramp[i].x * win[i].y + ramp[i].y * win[i].x;
            ramp[i].x = re;
            ramp[i].y = im;
        }
        cudaMemcpy(d, ramp.data(), sizeof(cufftComplex) * L, cudaMemcpyHostToDevice);
        cufftExecC2C(c2c, d, d, CUFFT_INVERSE);
        cudaMemcpy(ramp.data(), d, sizeof(cufftComplex) * L, cudaMemcpyDeviceToHost);
        std::vector<float> k(L);
        for (int i = 0; i < L; i++) k[i] = ramp[i].x / L;
        cudaMemcpy(dk, k.data(), sizeof(float) * L, cudaMemcpyHostToDevice);
        if (cufftExecR2C(r2c, dk, out->spec) != CUFFT_SUCCESS) rc = set_error(CTP_ERR_CUFFT, "ramp R2C failed");
        cudaError_t e = cudaDeviceSynchronize();
        if (!rc && e != cudaSuccess) rc = set_error((int)e, "ramp table: %s", cudaGetErrorString(e));
    }
    if (!rc && fan) {
        std::vector<float> w(nu);
        for (int i = 0; i < nu; i++) w[i] = cosf(((i - (nu - 1) / 2.f) - off_u) * da);  // fbp.cu:62-66
        if (cudaMalloc(&out->weight, sizeof(float) * nu) != cudaSuccess)
            rc = set_error(cudaErrorMemoryAllocation, "ramp weight allocation failed");
        else
            cudaMemcpy(out->weight, w.data(), sizeof(float) * nu, cudaMemcpyHostToDevice);
    }
    if (c2c) cufftDestroy(c2c);
    if (r2c) cufftDestroy(r2c);
    if (d) cudaFree(d);
    if (dk) cudaFree(dk);
    return rc;
}

int get_ref_filter(int nu, float da, int filter, bool fan, float off_u, RefFilter* out) {
    int dev = 0;
    cudaGetDevice(&dev);
    unsigned dbits, obits;
    memcpy(&dbits, &da, 4);
    memcpy(&obits, &off_u, 4);
    auto key = std::make_tuple(dev, nu, dbits, filter, (int)fan, fan ? obits : 0u);
    std::lock_guard<std::mutex> lk(g_ref_mu);
    auto it = g_ref.find(key);
    if (it != g_ref.end()) {
        *out = it->second;
        return CTP_OK;
    }
    RefFilter f;
    int rc = build_ref_filter(nu, da, filter, fan, off_u, &f);
    if (rc) return rc;
    g_ref[key] = f;
    *out = f;
    return CTP_OK;
}

struct RefPlan {
    cufftHandle fwd = 0, inv = 0;
    size_t work = 0;
    std::mutex mu;
};
std::mutex g_rplan_mu;
std::map<std::tuple<int, int, int>, std::unique_ptr<RefPlan>> g_rplans;

// cufftPlanMany with the reference's layout: real rows of length L (idist L),
// complex rows of nu bins (odist nu), batch nview.
int get_ref_plan(int L, int nu, int batch, RefPlan** out) {
    int dev = 0;
    cudaGetDevice(&dev);
    auto key = std::make_tuple(dev, L, batch);
    std::lock_guard<std::mutex> lk(g_rplan_mu);
    auto it = g_rplans.find(key);
    if (it != g_rplans.end()) {
        *out = it->second.get();
        return CTP_OK;
    }
    std::unique_ptr<RefPlan> p(new RefPlan());
    int n[1] = {L};
    size_t w1 = 0, w2 = 0;
    if (cufftCreate(&p->fwd) != CUFFT_SUCCESS || cufftCreate(&p->inv) != CUFFT_SUCCESS)
        return set_error(CTP_ERR_CUFFT, "cufftCreate failed");
    cufftSetAutoAllocation(p->fwd, 0);
    cufftSetAutoAllocation(p->inv, 0);
    if (cufftMakePlanMany(p->fwd, 1, n, nullptr, 1, L, nullptr, 1, nu, CUFFT_R2C, batch, &w1) != CUFFT_SUCCESS ||
        cufftMakePlanMany(p->inv, 1, n, nullptr, 1, nu, nullptr, 1, L, CUFFT_C2R, batch, &w2) != CUFFT_SUCCESS)
        return set_error(CTP_ERR_CUFFT, "cufftMakePlanMany failed (L=%d, batch=%d)", L, batch);
    p->work = w1 > w2 ? w1 : w2;
    *out = p.get();
    g_rplans[key] = std::move(p);
    return CTP_OK;
}

// CopyPrjToPad + Multiply2D (fbpMath.cu:59-72, cudaMath.cu:28-49): one pass over all rows.
__global__ void ref_pad_kernel(float* __restrict__ pad, const float* __restrict__ prj, const float* __restrict__ w,
                               int nu, int L, size_t rows) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= rows * L) return;
    size_t r = i / L;
    int n = (int)(i - r * L);
    float v = 0.f;
    if (n < nu) {
        v = prj[r * nu + n];
        if (w) v = v * w[n];
    }
    pad[i] = v;
}

// ComplexMultiply2D (fbpMath.cu:12-33) against the kernel replicated over rows.
__global__ void ref_cmul_kernel(cufftComplex* __restrict__ f, const cufftComplex* __restrict__ k, int nu,
                                size_t rows) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= rows * nu) return;
    cufftComplex val1 = f[i];
    cufftComplex val2 = k[i % nu];
    cufftComplex val;
    val.x = val1.x * val2.x - val1.y * val2.y;
    val.y = val1.x * val2.y + val1.y * val2.x;
    f[i] = val;
}

// Scale2D + CopyPadToPrj (cudaMath.cu:76-97, fbpMath.cu:74-87).
__global__ void ref_crop_kernel(float* __restrict__ out, const float* __restrict__ pad, int nu, int L, size_t rows,
                                float scale) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= rows * nu) return;
    size_t r = i / nu;
    int n = (int)(i - r * nu);
    out[i] = pad[r * L + nu - 1 + n] * scale;
}

size_t ref_workspace(const ctp_geometry& g) {
    size_t nu = g.nu, L = 2 * nu - 1, rows = g.nbatch * g.nview * g.nv;
    RefPlan* p = nullptr;
    if (get_ref_plan((int)L, (int)nu, (int)g.nview, &p)) return 0;
    return align_up(rows * L * sizeof(float)) + align_up(rows * nu * sizeof(cufftComplex)) + align_up(p->work);
}

int ramp_filter_reference(float* fprj, const float* prj, const ctp_geometry& g, int geom, int filter,
                          void* workspace, size_t workspace_bytes, cudaStream_t s) {
    int nu = (int)g.nu, L = 2 * nu - 1, nview = (int)g.nview;
    size_t rows = g.nbatch * g.nview * g.nv;
    bool fan = geom == 0;
    RefFilter rf;
    int rc = get_ref_filter(nu, g.du, filter, fan, g.off_u, &rf);
    if (rc) return rc;
    RefPlan* plan = nullptr;
    if ((rc = get_ref_plan(L, nu, nview, &plan))) return rc;
    Scratch scr;
    size_t pad_b = align_up(rows * L * sizeof(float)), frq_b = align_up(rows * nu * sizeof(cufftComplex));
    if ((rc = scr.acquire(workspace, workspace_bytes, pad_b + frq_b + align_up(plan->work), s))) return rc;
    float* pad = reinterpret_cast<float*>(scr.base());
    cufftComplex* frq = reinterpret_cast<cufftComplex*>(scr.base() + pad_b);
    void* work = scr.base() + pad_b + frq_b;
    const float PIf = 3.141592657f;
    // fbpParallel.cu:59, fbp.cu:103 (float arithmetic)
    float scale = fan ? PIf / g.nview * g.du / g.dso / L : PIf / g.nview * g.du / L;
    size_t np = rows * L;
    ref_pad_kernel<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(pad, prj, fan ? rf.weight : nullptr, nu, L, rows);
    if ((rc = check_launch("ref_pad_kernel"))) return rc;
    {
        std::lock_guard<std::mutex> lk(plan->mu);
        cufftSetStream(plan->fwd, s);
        cufftSetStream(plan->inv, s);
        cufftSetWorkArea(plan->fwd, work);
        cufftSetWorkArea(plan->inv, work);
        for (size_t r0 = 0; r0 < rows; r0 += nview)
            if (cufftExecR2C(plan->fwd, pad + r0 * L, frq + r0 * nu) != CUFFT_SUCCESS)
                return set_error(CTP_ERR_CUFFT, "cufftExecR2C failed");
        size_t nf = rows * nu;
        ref_cmul_kernel<<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(frq, rf.spec, nu, rows);
        if ((rc = check_launch("ref_cmul_kernel"))) return rc;
        for (size_t r0 = 0; r0 < rows; r0 += nview)
            if (cufftExecC2R(plan->inv, frq + r0 * nu, pad + r0 * L) != CUFFT_SUCCESS)
                return set_error(CTP_ERR_CUFFT, "cufftExecC2R failed");
    }
    size_t no = rows * nu;
    ref_crop_kernel<<<(unsigned)((no + 255) / 256), 256, 0, s>>>(fprj, pad, nu, L, rows, scale);
    return check_launch("ref_crop_kernel");
}

// ------------------------------------------------------------------ exact mode: one-launch row convolution
// The exact filter evaluates  out[i] = scale * sum_j w_j p[j] g[i-j]  (g the
// FP64 windowed ramp, w the fan pre-weight) as a circular convolution of a
// smooth size N = 2^a 3^b >= 2nu-1 (exact, since g spans offsets
// -(nu-1)..nu-1), in FP64 arithmetic, in one launch over every row of the
// batch with no scratch memory: a CTA takes two detector rows as the real and
// imaginary parts of one complex row (a convolution with a real kernel acts
// on both parts separately), zero pads it to N in shared memory, transforms
// it (Stockham autosort, radix 8/4/3/2 stages ping-ponging between two
// shared-memory buffers), multiplies by the kernel's spectrum, transforms back
// (the inverse as the conjugate of the forward transform of the conjugate),
// and writes the first nu samples of both parts, scaled and cropped.
constexpr int kConvMaxN = 6912;  // two FP64 complex buffers of N fit 227 KB of shared memory
constexpr int kConvMaxStages = 16;

struct ConvPlan {
    int n = 0;                    // transform size
    int nstages = 0;              // number of radix stages
    unsigned long long code = 0;  // the radices, 4 bits each, first stage lowest
};

// The smooth size with the least work (elements x passes over shared memory)
// and its radices (8s first, then a 4 or a 2, then 3s); n = 0 if 2nu-1 >
// kConvMaxN.
ConvPlan conv_plan(int nu) {
    ConvPlan best;
    long best_cost = -1;
    const long need = 2L * nu - 1;
    for (long p2 = 1, a = 0; p2 <= kConvMaxN; p2 *= 2, ++a)
        for (long p3 = p2, b = 0; p3 <= kConvMaxN; p3 *= 3, ++b) {
            if (p3 < need) continue;
            int radix[kConvMaxStages], ns = 0;
            for (long i = 0; i < a / 3; ++i) radix[ns++] = 8;
            if (a % 3) radix[ns++] = a % 3 == 2 ? 4 : 2;
            for (long i = 0; i < b; ++i) radix[ns++] = 3;
            long cost = p3 * (ns + 1);
            if (best_cost < 0 || cost < best_cost || (cost == best_cost && p3 < best.n)) {
                best = ConvPlan();
                best.n = (int)p3;
                best.nstages = ns;
                for (int i = 0; i < ns; ++i) best.code |= (unsigned long long)radix[i] << (4 * i);
                best_cost = cost;
            }
            break;  // larger powers of 3 at this power of 2 only cost more
        }
    return best;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }  // a * (-i)

// In-register DFT of length R, forward sign (exp(-2 pi i nk/R)).
template <int R>
__device__ __forceinline__ void small_dft(double2* v);

template <>
__device__ __forceinline__ void small_dft<2>(double2* v) {
    const double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <>
__device__ __forceinline__ void small_dft<4>(double2* v) {
    const double2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    const double2 s13 = cadd(v[1], v[3]), d13 = mul_mi(csub(v[1], v[3]));
    v[0] = cadd(s02, s13);
    v[2] = csub(s02, s13);
    v[1] = cadd(d02, d13);
    v[3] = csub(d02, d13);
}

template <>
__device__ __forceinline__ void small_dft<8>(double2* v) {
    double2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    small_dft<4>(e);
    small_dft<4>(o);
    const double h = 0.70710678118654752440;  // cos(pi/4)
    const double2 o1 = make_double2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));   // * exp(-i pi/4)
    const double2 o2 = mul_mi(o[2]);                                                // * exp(-i pi/2)
    const double2 o3 = make_double2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));  // * exp(-3i pi/4)
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
}

template <>
__device__ __forceinline__ void small_dft<3>(double2* v) {
    const double s = 0.86602540378443864676;  // sin(pi/3)
    const double2 t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    const double2 m = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
    const double2 r = make_double2(s * t2.y, -s * t2.x);  // -i s t2
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
}

// Shared-memory slot of element i: i with its low three bits XORed by the
// next three, a permutation within each aligned group of 8 (buffers are
// rounded up to a multiple of 8).  The first stage writes each thread's
// outputs 8 elements apart, which would put the 8 threads of a 16-byte
// access phase on the same banks; swizzled they are spread over all banks,
// while the contiguous accesses of the other stages stay contiguous.
__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 3) & 7); }

// One radix-R stage: sub-transforms of length ns are merged R at a time.
// The twiddles of a butterfly are the powers w, w^2, ... of
// w = tw[k * n / (ns R)] (tw[t] = exp(-2 pi i t / n)): one table load, the
// other powers by FP64 complex products (their rounding, ~R ulp, is far below
// the FP32 output's).
template <int R>
__device__ __forceinline__ void fft_stage(const double2* __restrict__ src, double2* __restrict__ dst,
                                          const double2* __restrict__ tw, int n, int ns) {
    const int nr = n / R, tstep = n / (ns * R);
    for (int j = threadIdx.x; j < nr; j += blockDim.x) {
        const int k = j % ns;
        double2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[swz(j + r * nr)];
        if (ns > 1) {
            const double2 w = __ldg(tw + k * tstep);
            double2 wr = w;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                v[r] = cmul(v[r], wr);
                if (r + 1 < R) wr = cmul(wr, w);
            }
        }
        small_dft<R>(v);
        const int d = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[swz(d + r * ns)] = v[r];
    }
}

// Forward transform of the buffer at offset a of smem (the other buffer at
// offset b); returns the offset of the buffer that holds the result.
__device__ __forceinline__ int fft_forward(double2* smem, int a, int b, const double2* __restrict__ tw,
                                           const ConvPlan& plan) {
    int ns = 1;
    unsigned long long code = plan.code;
    for (int s = 0; s < plan.nstages; ++s, code >>= 4) {
        const int R = (int)(code & 15);
        if (R == 8)
            fft_stage<8>(smem + a, smem + b, tw, plan.n, ns);
        else if (R == 4)
            fft_stage<4>(smem + a, smem + b, tw, plan.n, ns);
        else if (R == 3)
            fft_stage<3>(smem + a, smem + b, tw, plan.n, ns);
        else
            fft_stage<2>(smem + a, smem + b, tw, plan.n, ns);
        __syncthreads();
        const int t = a;
        a = b;
        b = t;
        ns *= R;
    }
    return a;
}

// Input rows of the filter: FP32 samples, or 16-bit affine codes with one
// offset and step per view (quant.cu), dequantized as they are read.
struct RowsF32 {
    const float* p;
    __device__ __forceinline__ float load(size_t row, int j, int nu) const { return __ldg(p + row * nu + j); }
};
struct RowsU16 {
    const unsigned short* code;
    const float* lo;
    const float* step;
    int nv;  // detector rows per view (one offset and step each view)
    __device__ __forceinline__ float load(size_t row, int j, int nu) const {
        const size_t v = row / (size_t)nv;
        return fmaf(__ldg(step + v), (float)__ldg(code + row * nu + j), __ldg(lo + v));
    }
};

// fbpParallel.cu:44-86 / fbp.cu:81-134 for every row of the batch at once:
// pre-weight (fan), convolution with the windowed ramp, crop and scale.
template <typename Rows>
__global__ void __launch_bounds__(256) conv_rows_kernel(float* __restrict__ out, const Rows in,
                                                        const double* __restrict__ weight,
                                                        const double* __restrict__ spec,
                                                        const double2* __restrict__ tw, const ConvPlan plan, int nu,
                                                        size_t rows, double scale) {
    extern __shared__ double2 conv_smem[];
    const size_t r0 = (size_t)blockIdx.x * 2;
    const bool two = r0 + 1 < rows;
    for (int j = threadIdx.x; j < plan.n; j += blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        if (j < nu) {
            const double w = weight ? __ldg(weight + j) : 1.0;
            v.x = (double)in.load(r0, j, nu) * w;
            v.y = two ? (double)in.load(r0 + 1, j, nu) * w : 0.0;
        }
        conv_smem[swz(j)] = v;
    }
    __syncthreads();
    const int stride = (plan.n + 7) & ~7;  // one buffer, rounded up for the swizzle
    int a = fft_forward(conv_smem, 0, stride, tw, plan);
    double2* buf = conv_smem + a;
    for (int j = threadIdx.x; j < plan.n; j += blockDim.x) {
        const double k = __ldg(spec + j);
        const double2 y = buf[swz(j)];
        buf[swz(j)] = make_double2(y.x * k, -y.y * k);  // conjugate of the product with the real spectrum
    }
    __syncthreads();
    a = fft_forward(conv_smem, a, stride - a, tw, plan);
    buf = conv_smem + a;
    float* y0 = out + r0 * nu;
    float* y1 = y0 + nu;
    for (int n = threadIdx.x; n < nu; n += blockDim.x) {
        const double2 v = buf[swz(n)];
        y0[n] = (float)(v.x * scale);
        if (two) y1[n] = (float)(-v.y * scale);
    }
}

// Cached per (device, nu, da, filter, kind, off_u): plan, spectrum, twiddles
// and the fan pre-weight, all FP64.
struct ConvTables {
    ConvPlan plan;
    double* spec = nullptr;   // [N] DFT_N of the circular kernel (real: g is even)
    double2* tw = nullptr;    // [N] exp(-2 pi i t / N)
    double* weight = nullptr; // [nu] fan pre-weight, or null
};

std::mutex g_conv_mu;
std::map<std::tuple<int, int, long long, int, int, long long>, ConvTables> g_conv;

int get_conv_tables(int nu, double da, int filter, bool fan, double off_u, const ConvPlan& plan,
                    ConvTables* out) {
    int dev = 0;
    cudaGetDevice(&dev);
    long long dkey, okey;
    memcpy(&dkey, &da, sizeof(dkey));
    memcpy(&okey, &off_u, sizeof(okey));
    auto key = std::make_tuple(dev, nu, dkey, filter, (int)fan, fan ? okey : 0LL);
    std::lock_guard<std::mutex> lk(g_conv_mu);
    auto it = g_conv.find(key);
    if (it != g_conv.end()) {
        *out = it->second;
        return CTP_OK;
    }
    const int N = plan.n;
    std::vector<double> g = ramp_kernel(nu, da, filter, fan);
    std::vector<double> c(N), spec(N), w(nu);
    std::vector<double2> tw(N);
    for (int t = 0; t < N; ++t) {
        c[t] = cos(2 * M_PI * t / N);
        tw[t] = make_double2(c[t], -sin(2 * M_PI * t / N));
    }
    for (int m = 0; m < N; ++m) {
        double acc = g[0];
        long long idx = 0;
        for (int k = 1; k < nu; ++k) {
            idx += m;
            if (idx >= N) idx -= N;
            acc += 2 * g[k] * c[idx];
        }
        spec[m] = acc;
    }
    for (int n = 0; n < nu; ++n) w[n] = cos(((n - (nu - 1) / 2.0) - off_u) * da);  // fbp.cu:62-66
    ConvTables t;
    t.plan = plan;
    // one-time tables for this geometry, kept for the process
    cudaError_t e = cudaMalloc(&t.spec, sizeof(double) * N);
    if (e == cudaSuccess) e = cudaMalloc(&t.tw, sizeof(double2) * N);
    if (e == cudaSuccess && fan) e = cudaMalloc(&t.weight, sizeof(double) * nu);
    if (e == cudaSuccess) e = cudaMemcpy(t.spec, spec.data(), sizeof(double) * N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t.tw, tw.data(), sizeof(double2) * N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && fan) e = cudaMemcpy(t.weight, w.data(), sizeof(double) * nu, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_error((int)e, "ramp convolution tables: %s", cudaGetErrorString(e));
    g_conv[key] = t;
    *out = t;
    return CTP_OK;
}

template <typename Rows>
int ramp_filter_conv(float* fprj, const Rows prj, const ctp_geometry& g, bool fan, int filter,
                     const ConvPlan& plan, cudaStream_t s) {
    const int nu = (int)g.nu, N = plan.n;
    const size_t rows = g.nbatch * g.nview * g.nv;
    if (rows == 0) return CTP_OK;
    ConvTables t;
    int rc = get_conv_tables(nu, (double)g.du, filter, fan, (double)g.off_u, plan, &t);
    if (rc) return rc;
    const double scale = M_PI / (double)g.nview * (double)g.du / (fan ? (double)g.dso : 1.0) / N;
    int threads = (N / 8 + 31) / 32 * 32;
    threads = threads < 64 ? 64 : threads > 256 ? 256 : threads;
    const size_t smem = 2 * sizeof(double2) * (size_t)((N + 7) & ~7);
    if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(conv_rows_kernel<Rows>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return set_error((int)e, "conv_rows_kernel shared memory: %s", cudaGetErrorString(e));
    }
    const size_t blocks = (rows + 1) / 2;
    if (blocks > 0x7fffffffULL) return set_error(CTP_ERR_TOO_LARGE, "ramp filter: %zu rows", rows);
    conv_rows_kernel<Rows><<<(unsigned)blocks, threads, smem, s>>>(fprj, prj, t.weight, t.spec, t.tw, plan, nu,
                                                                   rows, scale);
    return check_launch("conv_rows_kernel");
}

size_t exact_workspace(const ctp_geometry& g) {
    if (conv_plan((int)g.nu).n > 0) return 0;  // conv_rows_kernel needs no scratch
    size_t rows = g.nbatch * g.nview * g.nv;
    int N = fft_size((int)g.nu);
    size_t chunk = rows < (size_t)kMaxRowsPerExec ? rows : (size_t)kMaxRowsPerExec;
    Plan* p = nullptr;
    if (chunk == 0 || get_plan(N, (int)chunk, &p)) return 0;
    return align_up(chunk * 2 * (N / 2 + 1) * sizeof(double)) + align_up(p->work);
}

int ramp_filter_exact(float* fprj, const float* prj, const ctp_geometry& g, int geom, int filter, void* workspace,
                      size_t workspace_bytes, cudaStream_t s) {
    const ConvPlan cp = conv_plan((int)g.nu);
    if (cp.n > 0) return ramp_filter_conv(fprj, RowsF32{prj}, g, geom == 0, filter, cp, s);
    // wider detectors: batched FP64 cuFFT transforms of the same convolution
    int nu = (int)g.nu;
    size_t rows = g.nbatch * g.nview * g.nv;
    int N = fft_size(nu), M = N / 2 + 1, stride = 2 * M;
    size_t chunk = rows < (size_t)kMaxRowsPerExec ? rows : (size_t)kMaxRowsPerExec;
    Plan* plan = nullptr;
    int rc = get_plan(N, (int)chunk, &plan);
    if (rc) return rc;
    const double* G = nullptr;
    bool fan = geom == 0;
    if ((rc = get_spectrum(nu, (double)g.du, filter, fan, N, &G))) return rc;
    Scratch scr;
    size_t buf_bytes = align_up(chunk * stride * sizeof(double));
    if ((rc = scr.acquire(workspace, workspace_bytes, buf_bytes + align_up(plan->work), s))) return rc;
    double* buf = reinterpret_cast<double*>(scr.base());
    void* work = scr.base() + buf_bytes;
    double scale = M_PI / (double)g.nview * (double)g.du / (fan ? (double)g.dso : 1.0) / N;
    for (size_t r0 = 0; r0 < rows; r0 += chunk) {
        size_t nr = rows - r0 < chunk ? rows - r0 : chunk;
        dim3 pg((unsigned)((stride + 255) / 256 > 8 ? 8 : (stride + 255) / 256), (unsigned)(nr < 65535 ? nr : 65535),
                (unsigned)((nr + 65534) / 65535));
        pad_kernel<<<pg, 256, 0, s>>>(buf, prj + r0 * nu, nu, N, stride, nr, fan ? 1 : 0, (double)g.du,
                                      (double)g.off_u);
        if ((rc = check_launch("pad_kernel"))) return rc;
        {
            std::lock_guard<std::mutex> lk(plan->mu);
            cufftSetStream(plan->fwd, s);
            cufftSetStream(plan->inv, s);
            cufftSetWorkArea(plan->fwd, work);
            cufftSetWorkArea(plan->inv, work);
            if (nr != chunk) cudaMemsetAsync(buf + nr * stride, 0, (chunk - nr) * stride * sizeof(double), s);
            if (cufftExecD2Z(plan->fwd, buf, reinterpret_cast<cufftDoubleComplex*>(buf)) != CUFFT_SUCCESS)
                return set_error(CTP_ERR_CUFFT, "cufftExecD2Z failed");
            size_t ns = nr * (size_t)M;
            spectrum_mul_kernel<<<(unsigned)((ns + 255) / 256), 256, 0, s>>>(reinterpret_cast<double2*>(buf), G, M,
                                                                           nr, scale);
            if ((rc = check_launch("spectrum_mul_kernel"))) return rc;
            if (cufftExecZ2D(plan->inv, reinterpret_cast<cufftDoubleComplex*>(buf), buf) != CUFFT_SUCCESS)
                return set_error(CTP_ERR_CUFFT, "cufftExecZ2D failed");
        }
        size_t no = nr * (size_t)nu;
        crop_kernel<<<(unsigned)((no + 255) / 256), 256, 0, s>>>(fprj + r0 * nu, buf, nu, stride, nr);
        if ((rc = check_launch("crop_kernel"))) return rc;
    }
    return CTP_OK;
}

}  // namespace

// The exact filter of a sinogram in 16-bit affine storage (quant.cu): one
// offset and step per view of each batch item.
int ramp_filter_u16(float* fprj, const unsigned short* code, const float* lo, const float* step,
                    const ctp_geometry& g, int geom, int filter, cudaStream_t s) {
    if (geom != 0 && geom != 1) return set_error(CTP_ERR_INVALID_ARGUMENT, "geom must be 0 (fan) or 1 (parallel)");
    const ConvPlan cp = conv_plan((int)g.nu);
    if (cp.n == 0)
        return set_error(CTP_ERR_UNSUPPORTED, "16-bit sinogram filter: %zu cells exceed the one-launch filter", g.nu);
    return ramp_filter_conv(fprj, RowsU16{code, lo, step, (int)g.nv}, g, geom == 0, filter, cp, s);
}

size_t ramp_filter_workspace(const ctp_geometry& g, int, int, unsigned flags) {
    return (flags & CTP_FLAG_FILTER_EXACT) ? exact_workspace(g) : ref_workspace(g);
}

int ramp_filter(float* fprj, const float* prj, const ctp_geometry& g, int geom, int filter, unsigned flags,
                void* workspace, size_t workspace_bytes, cudaStream_t s) {
    if (geom != 0 && geom != 1) return set_error(CTP_ERR_INVALID_ARGUMENT, "geom must be 0 (fan) or 1 (parallel)");
    if (flags & CTP_FLAG_FILTER_EXACT)
        return ramp_filter_exact(fprj, prj, g, geom, filter, workspace, workspace_bytes, s);
    return ramp_filter_reference(fprj, prj, g, geom, filter, workspace, workspace_bytes, s);
}

// ------------------------------------------------------------------ tomosynthesis FBP filter
// fbpTomo::Filter and GetRampTomo (fbpTomo.cu:50-384): every view has its own
// kernel.  The view's tilt (from the source-to-detector-centre direction in
// the x-z plane) gives a virtual detector pitch vdu = du cos(tilt); the ramp
// at that pitch is transformed, windowed by the product of an x window and a z
// window whose frequencies scale with cos and sin of the tilt (both clamped
// above at their cut-offs), transformed back, divided by L and transformed to
// the R2C spectrum.  The rows of each view are zero padded to L = 2nu-1,
// multiplied by the view's spectrum, transformed back, scaled by
// pi / nview * vdu / L and cropped at nu-1.  The construction and the row
// transforms replay the reference's FP32 steps and cuFFT plan shapes (one
// length-L transform per view for the kernel, nv rows per transform for the
// data), so the output stays within FP32 rounding of the reference.
namespace {

float tomo_frequency(int i, int L, float du, float dx, float angle_weight, float cutoff) {  // :50-68
    float fu;
    if (i > (L + 1) / 2)
        fu = (i - L) / float(L) / du;
    else
        fu = i / float(L) / du;
    float wx = fu * angle_weight * dx * 2;
    if (wx > cutoff) wx = cutoff;
    return wx;
}

struct TomoView {
    float vdu, sin_t, cos_t;
};

TomoView tomo_view(float3 src, float3 det, float du) {  // :127-135
    float r = sqrtf((det.x - src.x) * (det.x - src.x) + (det.z - src.z) * (det.z - src.z));
    TomoView v;
    v.sin_t = (det.x - src.x) / r;
    v.cos_t = (src.z - det.z) / r;
    v.vdu = du * v.cos_t;
    return v;
}

// Spectra [nview][nu] of the per-view kernels, built on the device.
int build_tomo_spectra(cufftComplex* spec, const std::vector<TomoView>& views, int nu, float dx, float dz,
                       float cutoff_x, float cutoff_z, int filter) {
    const int L = 2 * nu - 1;
    const float PIf = 3.141592657f;  // projector.h:5
    cufftHandle c2c = 0, r2c = 0;
    cufftComplex* d = nullptr;
    float* dk = nullptr;
    int rc = CTP_OK;
    if (cudaMalloc(&d, sizeof(cufftComplex) * L) != cudaSuccess || cudaMalloc(&dk, sizeof(float) * L) != cudaSuccess)
        rc = set_error(cudaErrorMemoryAllocation, "tomo ramp allocation failed");
    if (!rc && (cufftPlan1d(&c2c, L, CUFFT_C2C, 1) != CUFFT_SUCCESS || cufftPlan1d(&r2c, L, CUFFT_R2C, 1) != CUFFT_SUCCESS))
        rc = set_error(CTP_ERR_CUFFT, "tomo ramp plan failed");
    std::vector<cufftComplex> ramp(L), win(L);
    std::vector<float> k(L);
    for (size_t iv = 0; iv < views.size() && !rc; ++iv) {
        const float vdu = views[iv].vdu;
        for (int i = 0; i < L; i++) {
            int kk = i - (nu - 1);
            if (kk == 0)
                ramp[i].x = 1 / (4 * vdu * vdu);
            else if (kk % 2 != 0)
                ramp[i].x = -1 / (PIf * PIf * kk * kk * vdu * vdu);
            else
                ramp[i].x = 0;
            ramp[i].y = 0;
        }
        cudaMemcpy(d, ramp.data(), sizeof(cufftComplex) * L, cudaMemcpyHostToDevice);
        cufftExecC2C(c2c, d, d, CUFFT_FORWARD);
        cudaMemcpy(ramp.data(), d, sizeof(cufftComplex) * L, cudaMemcpyDeviceToHost);
        for (int i = 0; i < L; i++) {
            if (filter == 1 || filter == 2) {
                float wx = tomo_frequency(i, L, vdu, dx, views[iv].cos_t, cutoff_x);
                float wz = tomo_frequency(i, L, vdu, dz, views[iv].sin_t, cutoff_z);
                win[i].x = filter == 1
                               ? (0.54f + 0.46f * cosf(PIf * wx / cutoff_x)) * (0.54f + 0.46f * cosf(PIf * wz / cutoff_z))
                               : (0.5f + 0.5f * cosf(PIf * wx / cutoff_x)) * (0.5f + 0.5f * cosf(PIf * wz / cutoff_z));
            } else {
                win[i].x = 1;
            }
            win[i].y = 0;
            float re = ramp[i].x * win[i].x - ramp[i].y * win[i].y;
            float im = ramp[i].x * win[i].y + ramp[i].y * win[i].x;
            ramp[i].x = re;
            ramp[i].y = im;
        }
        cudaMemcpy(d, ramp.data(), sizeof(cufftComplex) * L, cudaMemcpyHostToDevice);
        cufftExecC2C(c2c, d, d, CUFFT_INVERSE);
        cudaMemcpy(ramp.data(), d, sizeof(cufftComplex) * L, cudaMemcpyDeviceToHost);
        for (int i = 0; i < L; i++) k[i] = ramp[i].x / L;
        cudaMemcpy(dk, k.data(), sizeof(float) * L, cudaMemcpyHostToDevice);
        if (cufftExecR2C(r2c, dk, spec + iv * nu) != CUFFT_SUCCESS) rc = set_error(CTP_ERR_CUFFT, "tomo ramp R2C failed");
        cudaError_t e = cudaDeviceSynchronize();
        if (!rc && e != cudaSuccess) rc = set_error((int)e, "tomo ramp: %s", cudaGetErrorString(e));
    }
    if (c2c) cufftDestroy(c2c);
    if (r2c) cufftDestroy(r2c);
    if (d) cudaFree(d);
    if (dk) cudaFree(dk);
    return rc;
}

// FilterByFreqMultiply1D against the kernel of each row's view.
__global__ void tomo_cmul_kernel(cufftComplex* __restrict__ f, const cufftComplex* __restrict__ spec, int nu, int nv,
                                 int nview, size_t rows) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= rows * nu) return;
    size_t r = i / nu;
    int n = (int)(i - r * nu);
    int view = (int)((r / nv) % nview);
    cufftComplex a = f[i], b = spec[(size_t)view * nu + n], v;
    v.x = a.x * b.x - a.y * b.y;
    v.y = a.x * b.y + a.y * b.x;
    f[i] = v;
}

__global__ void tomo_crop_kernel(float* __restrict__ out, const float* __restrict__ pad, const float* __restrict__ scale,
                                 int nu, int L, int nv, int nview, size_t rows) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= rows * nu) return;
    size_t r = i / nu;
    int n = (int)(i - r * nu);
    out[i] = pad[r * L + nu - 1 + n] * scale[(r / nv) % nview];
}

}  // namespace

size_t tomo_filter_workspace(const ctp_geometry& g) {
    size_t nu = g.nu, L = 2 * nu - 1, rows = g.nbatch * g.nview * g.nv;
    RefPlan* p = nullptr;
    if (nu == 0 || g.nv == 0 || get_ref_plan((int)L, (int)nu, (int)g.nv, &p)) return 0;
    return align_up(rows * L * sizeof(float)) + align_up(rows * nu * sizeof(cufftComplex)) + align_up(p->work) +
           align_up(g.nview * nu * sizeof(cufftComplex)) + align_up(g.nview * sizeof(float));
}

int tomo_filter(float* fprj, const float* prj, const float* det_center, const float* src, const ctp_geometry& g,
                int filter, float cutoff_x, float cutoff_z, unsigned flags, void* workspace, size_t workspace_bytes,
                cudaStream_t s) {
    if (g.nbatch == 0) return CTP_OK;
    if (!fprj || !prj || !det_center || !src) return set_error(CTP_ERR_INVALID_ARGUMENT, "null array pointer");
    if (g.nu == 0 || g.nv == 0 || g.nview == 0) return set_error(CTP_ERR_INVALID_ARGUMENT, "zero detector extent");
    if (!(cutoff_x > 0) || !(cutoff_z > 0)) return set_error(CTP_ERR_INVALID_ARGUMENT, "cut-offs must be positive");
    const int nu = (int)g.nu, L = 2 * nu - 1, nv = (int)g.nv, nview = (int)g.nview;
    const size_t rows = g.nbatch * g.nview * g.nv;
    // view geometry on the host (fbpTomo.cu:285-290 copies it back too)
    std::vector<float3> hd(nview), hs(nview);
    cudaError_t e = cudaMemcpyAsync(hd.data(), det_center, sizeof(float3) * nview, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hs.data(), src, sizeof(float3) * nview, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_error((int)e, "tomo filter geometry: %s", cudaGetErrorString(e));
    std::vector<TomoView> views(nview);
    std::vector<float> scale(nview);
    const float PIf = 3.141592657f;
    for (int v = 0; v < nview; ++v) {
        views[v] = tomo_view(hs[v], hd[v], g.du);
        if (!(views[v].vdu != 0.f) || !std::isfinite(views[v].vdu))
            return set_error(CTP_ERR_INVALID_ARGUMENT, "view %d: source and detector centre give no tilt", v);
        scale[v] = PIf / g.nview * views[v].vdu / L;  // fbpTomo.cu:311
    }
    RefPlan* plan = nullptr;
    int rc = get_ref_plan(L, nu, nv, &plan);
    if (rc) return rc;
    Scratch scr;
    size_t pad_b = align_up(rows * L * sizeof(float)), frq_b = align_up(rows * nu * sizeof(cufftComplex));
    size_t work_b = align_up(plan->work), spec_b = align_up(g.nview * nu * sizeof(cufftComplex));
    if ((rc = scr.acquire(workspace, workspace_bytes, pad_b + frq_b + work_b + spec_b + align_up(g.nview * sizeof(float)),
                          s)))
        return rc;
    float* pad = reinterpret_cast<float*>(scr.base());
    cufftComplex* frq = reinterpret_cast<cufftComplex*>(scr.base() + pad_b);
    void* work = scr.base() + pad_b + frq_b;
    cufftComplex* spec = reinterpret_cast<cufftComplex*>(scr.base() + pad_b + frq_b + work_b);
    float* dscale = reinterpret_cast<float*>(scr.base() + pad_b + frq_b + work_b + spec_b);
    // the view kernels are built with synchronous copies and transforms (as in
    // the reference; the filter is not on a hot path): the scratch must exist first
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_error((int)e, "tomo filter: %s", cudaGetErrorString(e));
    // the reference multiplies every view by the first view's kernel (fbpTomo.cu:323)
    const bool first_only = flags & CTP_FLAG_TOMO_FIRST_VIEW_KERNEL;
    const std::vector<TomoView> kviews = first_only ? std::vector<TomoView>(1, views[0]) : views;
    if ((rc = build_tomo_spectra(spec, kviews, nu, g.dx, g.dz, cutoff_x, cutoff_z, filter))) return rc;
    e = cudaMemcpyAsync(dscale, scale.data(), sizeof(float) * nview, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_error((int)e, "tomo filter scales: %s", cudaGetErrorString(e));
    ref_pad_kernel<<<(unsigned)((rows * L + 255) / 256), 256, 0, s>>>(pad, prj, nullptr, nu, L, rows);
    if ((rc = check_launch("ref_pad_kernel"))) return rc;
    {
        std::lock_guard<std::mutex> lk(plan->mu);
        cufftSetStream(plan->fwd, s);
        cufftSetStream(plan->inv, s);
        cufftSetWorkArea(plan->fwd, work);
        cufftSetWorkArea(plan->inv, work);
        for (size_t r0 = 0; r0 < rows; r0 += nv)
            if (cufftExecR2C(plan->fwd, pad + r0 * L, frq + r0 * nu) != CUFFT_SUCCESS)
                return set_error(CTP_ERR_CUFFT, "cufftExecR2C failed");
        tomo_cmul_kernel<<<(unsigned)((rows * nu + 255) / 256), 256, 0, s>>>(frq, spec, nu, nv,
                                                                           first_only ? 1 : nview, rows);
        if ((rc = check_launch("tomo_cmul_kernel"))) return rc;
        for (size_t r0 = 0; r0 < rows; r0 += nv)
            if (cufftExecC2R(plan->inv, frq + r0 * nu, pad + r0 * L) != CUFFT_SUCCESS)
                return set_error(CTP_ERR_CUFFT, "cufftExecC2R failed");
    }
    tomo_crop_kernel<<<(unsigned)((rows * nu + 255) / 256), 256, 0, s>>>(fprj, pad, dscale, nu, L, nv, nview, rows);
    return check_launch("tomo_crop_kernel");
}

// ------------------------------------------------------------------ fbp_bp
namespace {

constexpr int kFbpViews = 64;
constexpr int kFbpZ = 4;

// Pixel-driven fan back projection with the FBP distance weight,
// bpFanKernel3D fbp.cu:265-337; bilinear InterpolateXY(truncate = true),
// cudaMath.cu:227-260.  One thread per pixel and kFbpZ slices.
__global__ void fbp_fan_bp_kernel(float* __restrict__ img, const float* __restrict__ prj,
                                  const float* __restrict__ deg, int nview, Grid g, Det d, float dso,
                                  int accumulate) {
    __shared__ float s_c[kFbpViews], s_s[kFbpViews];
    int ix = blockIdx.x * 32 + (threadIdx.x & 31);
    int iy = blockIdx.y * 8 + (threadIdx.x >> 5);
    int zb = blockIdx.z % ((g.nz + kFbpZ - 1) / kFbpZ);
    int b = blockIdx.z / ((g.nz + kFbpZ - 1) / kFbpZ);
    int iz0 = zb * kFbpZ;
    float x = ((float)ix + 0.5f - g.nx / 2.f) * g.dx + g.cx;
    float y = ((float)iy + 0.5f - g.ny / 2.f) * g.dy + g.cy;
    float z0 = ((float)iz0 + 0.5f - g.nz / 2.f) * g.dz + g.cz;
    float acc[kFbpZ];
#pragma unroll
    for (int q = 0; q < kFbpZ; ++q) acc[q] = 0.f;
    const float inv_du = 1.f / d.du;
    const float* pb = prj + (size_t)b * nview * d.nv * d.nu;
    for (int v0 = 0; v0 < nview; v0 += kFbpViews) {
        int nvc = min(kFbpViews, nview - v0);
        if (threadIdx.x < nvc) {
            double s, c;
            sincos((double)deg[v0 + threadIdx.x], &s, &c);
            s_c[threadIdx.x] = (float)c;
            s_s[threadIdx.x] = (float)s;
        }
        __syncthreads();
        if (ix < g.nx && iy < g.ny) {
            for (int vi = 0; vi < nvc; ++vi) {
                float c = s_c[vi], s = s_s[vi];
                float rx = x * c + y * s, ry = -x * s + y * c;
                // fast divides and a reciprocal for 1/du: a few ulp, against
                // the IEEE divide sequences of the reference's expressions
                float a = atanf(__fdividef(rx, ry + dso));
                float dist = __fdividef(dso * dso, rx * rx + (dso + ry) * (dso + ry));
                float pu = -(a * inv_du + d.off_u) + (d.nu - 1.0f) / 2.0f;
                if (pu < 0 || pu >= d.nu) continue;
                int i0 = (int)pu;
                int i1 = min(i0 + 1, d.nu - 1);
                float wu = pu - (float)i0;
                const float* pv_base = pb + (size_t)(v0 + vi) * d.nv * d.nu;
#pragma unroll
                for (int q = 0; q < kFbpZ; ++q) {
                    float pv = (z0 + q * g.dz) / d.dv + d.off_v + (d.nv - 1.0f) / 2.f;
                    if (pv < 0 || pv >= d.nv) continue;
                    int j0 = (int)pv;
                    int j1 = min(j0 + 1, d.nv - 1);
                    float wv = pv - (float)j0;
                    const float* r0 = pv_base + (size_t)j0 * d.nu;
                    const float* r1 = pv_base + (size_t)j1 * d.nu;
                    float v = __ldg(r0 + i0) * (1 - wu) * (1 - wv) + __ldg(r0 + i1) * wu * (1 - wv) +
                              __ldg(r1 + i0) * (1 - wu) * wv + __ldg(r1 + i1) * wu * wv;
                    acc[q] += v * dist;
                }
            }
        }
        __syncthreads();
    }
    if (ix < g.nx && iy < g.ny) {
#pragma unroll
        for (int q = 0; q < kFbpZ; ++q) {
            int iz = iz0 + q;
            if (iz >= g.nz) break;
            float* o = img + (((size_t)b * g.nz + iz) * g.ny + iy) * g.nx + ix;
            *o = (accumulate ? *o : 0.f) + acc[q];
        }
    }
}

// Pixel-driven parallel back projection without weights (the numpy
// module's pixel_driven_bp; bpParallelKernel3D, fbpParallel.cu:200-250):
// pu = -((x cos + y sin)/du + off_u) + (nu-1)/2 and the same truncating
// bilinear interpolation as fbp_fan_bp_kernel.
__global__ void pixel_bp_par_kernel(float* __restrict__ img, const float* __restrict__ prj,
                                    const float* __restrict__ deg, int nview, Grid g, Det d, int accumulate) {
    __shared__ float s_c[kFbpViews], s_s[kFbpViews];
    int ix = blockIdx.x * 32 + (threadIdx.x & 31);
    int iy = blockIdx.y * 8 + (threadIdx.x >> 5);
    int zb = blockIdx.z % ((g.nz + kFbpZ - 1) / kFbpZ);
    int b = blockIdx.z / ((g.nz + kFbpZ - 1) / kFbpZ);
    int iz0 = zb * kFbpZ;
    float x = ((float)ix + 0.5f - g.nx / 2.f) * g.dx + g.cx;
    float y = ((float)iy + 0.5f - g.ny / 2.f) * g.dy + g.cy;
    float z0 = ((float)iz0 + 0.5f - g.nz / 2.f) * g.dz + g.cz;
    float acc[kFbpZ];
#pragma unroll
    for (int q = 0; q < kFbpZ; ++q) acc[q] = 0.f;
    const float inv_du = 1.f / d.du;
    const float* pb = prj + (size_t)b * nview * d.nv * d.nu;
    for (int v0 = 0; v0 < nview; v0 += kFbpViews) {
        int nvc = min(kFbpViews, nview - v0);
        if (threadIdx.x < nvc) {
            double s, c;
            sincos((double)deg[v0 + threadIdx.x], &s, &c);
            s_c[threadIdx.x] = (float)c;
            s_s[threadIdx.x] = (float)s;
        }
        __syncthreads();
        if (ix < g.nx && iy < g.ny) {
            for (int vi = 0; vi < nvc; ++vi) {
                float pu = -((x * s_c[vi] + y * s_s[vi]) * inv_du + d.off_u) + (d.nu - 1.0f) / 2.0f;
                if (pu < 0 || pu >= d.nu) continue;
                int i0 = (int)pu;
                int i1 = min(i0 + 1, d.nu - 1);
                float wu = pu - (float)i0;
                const float* pv_base = pb + (size_t)(v0 + vi) * d.nv * d.nu;
#pragma unroll
                for (int q = 0; q < kFbpZ; ++q) {
                    float pv = (z0 + q * g.dz) / d.dv + d.off_v + (d.nv - 1.0f) / 2.f;
                    if (pv < 0 || pv >= d.nv) continue;
                    int j0 = (int)pv;
                    int j1 = min(j0 + 1, d.nv - 1);
                    float wv = pv - (float)j0;
                    const float* r0 = pv_base + (size_t)j0 * d.nu;
                    const float* r1 = pv_base + (size_t)j1 * d.nu;
                    acc[q] += __ldg(r0 + i0) * (1 - wu) * (1 - wv) + __ldg(r0 + i1) * wu * (1 - wv) +
                              __ldg(r1 + i0) * (1 - wu) * wv + __ldg(r1 + i1) * wu * wv;
                }
            }
        }
        __syncthreads();
    }
    if (ix < g.nx && iy < g.ny) {
#pragma unroll
        for (int q = 0; q < kFbpZ; ++q) {
            int iz = iz0 + q;
            if (iz >= g.nz) break;
            float* o = img + (((size_t)b * g.nz + iz) * g.ny + iy) * g.nx + ix;
            *o = (accumulate ? *o : 0.f) + acc[q];
        }
    }
}

}  // namespace

int fbp_fan_bp(float* img, const float* prj, const float* deg, const ctp_geometry& g, unsigned flags,
               cudaStream_t s) {
    int zb = (int)((g.nz + kFbpZ - 1) / kFbpZ);
    dim3 grid((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 7) / 8), (unsigned)(g.nbatch * zb));
    fbp_fan_bp_kernel<<<grid, 256, 0, s>>>(img, prj, deg, (int)g.nview, make_grid(g), make_det(g), g.dso,
                                           (flags & CTP_FLAG_ZERO_OUT) ? 0 : 1);
    return check_launch("fbp_fan_bp_kernel");
}

int pixel_bp_parallel(float* img, const float* prj, const float* deg, const ctp_geometry& g, unsigned flags,
                      cudaStream_t s) {
    int zb = (int)((g.nz + kFbpZ - 1) / kFbpZ);
    dim3 grid((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 7) / 8), (unsigned)(g.nbatch * zb));
    pixel_bp_par_kernel<<<grid, 256, 0, s>>>(img, prj, deg, (int)g.nview, make_grid(g), make_det(g),
                                             (flags & CTP_FLAG_ZERO_OUT) ? 0 : 1);
    return check_launch("pixel_bp_par_kernel");
}

}  // namespace ctp
