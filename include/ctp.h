/*
 * ctp.h -- C ABI of libctp.so, the sm_100a projector pair (ctprojector_b200).
 *
 * Two families of entry points:
 *
 *  1. Reference-compatible entries.  Same symbol names, argument order and
 *     meaning as the reference libprojector.so (wudufan/CTProjector,
 *     src/ct_projector/kernel/projector/cuda/), so a caller that binds the
 *     reference library through ctypes can load this library instead.
 *       c*    take HOST pointers: device buffers are taken from a
 *             stream-ordered pool, data is copied in and out, and the call
 *             returns when the result is on the host.
 *       cupy* take DEVICE pointers and run asynchronously on the legacy
 *             default stream, like the reference (which also synchronises).
 *     Each returns 0 on success, a CUDA error code, or a CTP_ERR_* code.
 *     Output semantics follow the reference: DD and tomo forward projection
 *     and tomo back projection overwrite the output; DD back projection,
 *     Siddon forward/back projection and fbp_bp accumulate into it; the
 *     filters overwrite.
 *
 *  2. Extended entries (ctp_*): explicit cudaStream_t (as void*), caller
 *     workspace, and flags.  They never synchronise the device.  A NULL
 *     workspace makes the library take scratch from the stream-ordered pool
 *     (cudaMallocAsync/cudaFreeAsync on the same stream).
 *
 * Array layouts (row-major, float32 unless a flag says otherwise):
 *   image    [nbatch][nz][ny][nx]
 *   sinogram [nbatch][nview][nv][nu]
 *   angles   [nview] radians
 *   cone/tomo geometry arrays [nview][3] as (x, y, z) in mm.
 */
#ifndef CTP_H
#define CTP_H

#include <stddef.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (CUDA runtime codes pass through unchanged) ---------- */
#define CTP_OK 0
#define CTP_ERR_INVALID_ARGUMENT 1001 /* null pointer, zero or inconsistent size */
#define CTP_ERR_UNSUPPORTED 1002      /* flag or geometry this build does not handle */
#define CTP_ERR_WORKSPACE 1003        /* caller workspace smaller than required */
#define CTP_ERR_CUFFT 1004            /* cuFFT plan or execution failure */
#define CTP_ERR_TOO_LARGE 1005        /* request exceeds a fixed-size internal buffer */
#define CTP_ERR_WAIT_TIMEOUT 1006     /* a bounded device-side wait gave up during a synchronous call; the
                                         output is incomplete (see ctp_wait_timeouts) */

/* Default poll limit of the bounded device-side waits (ctp_set_wait_limit). */
#define CTP_WAIT_POLLS_DEFAULT 4194304u

/* ---- flags for the extended entries ------------------------------------ */
#define CTP_FLAG_ZERO_OUT 0x1  /* treat the output as zero (write instead of accumulate) */
#define CTP_FLAG_ADJOINT 0x2   /* DD back projection: exact transpose of the forward projector */
#define CTP_FLAG_TOMO_FIRST_VIEW_KERNEL 0x200 /* tomo filter: every view uses the first view's kernel, as the
                                                 reference computes (fbpTomo.cu:323); default: each view its own */
#define CTP_FLAG_IN_BF16 0x10  /* the input array is bfloat16 (FP32 accumulation) */
#define CTP_FLAG_IN_FP16 0x20  /* the input array is float16 */
#define CTP_FLAG_OUT_BF16 0x40 /* the output array is bfloat16 */
#define CTP_FLAG_OUT_FP16 0x80 /* the output array is float16 */
#define CTP_FLAG_FILTER_EXACT 0x100 /* ramp filter: FP64 windowed kernel, smooth FFT size
                                       (default: the reference's FP32 construction) */
#define CTP_FLAG_SUBTRACT 0x400 /* ctp_dequantize_u16: subtract the values from the output */

/* typeProjector bits of the DD 2D entries, as in the reference
 * (distanceDriven2D.cu:12-25): bit0 FBP weighting, bit1 branchless,
 * bit2 force FBP weighting.  Branchless is the reference's branchless tracer
 * (distanceDriven2DBranchless.cu): the forward projector traces the main axis
 * alone (no 0.12 blend band), the parallel back projector likewise, and the
 * back projectors interpolate the detector row at each pixel's v instead of
 * truncating it.  Its prefix-sum interpolation is the same clamped box
 * integral, evaluated here in FP64-accurate form rather than from FP32 prefix
 * sums.  (Tomo entries: typeProjector 1 selects the reference's branchless
 * tomo tracer, the same operator as the box integral.) */
#define CTP_TYPE_FBP 0x1
#define CTP_TYPE_BRANCHLESS 0x2
#define CTP_TYPE_FORCE_FBP 0x4

/* Geometry of one call (mirrors the reference Grid/Detector structs,
 * projector.h:7-28, plus batch, view count and source distances). */
typedef struct ctp_geometry {
    size_t nbatch;
    size_t nx, ny, nz;
    float dx, dy, dz;
    float cx, cy, cz;
    size_t nu, nv, nview;
    float du, dv;
    float off_u, off_v;
    float dsd, dso;
} ctp_geometry;

/* Last error message of the calling thread ("" when none). */
const char* ctpGetLastErrorString(void);
/* Library version string. */
const char* ctpVersion(void);

/* ======================================================================== */
/* 1. Reference-compatible entries                                          */
/* ======================================================================== */

/* projector.cu:12 */
int SetDevice(int device);

/* distanceDriven2D.cu:109 (cupy*) / :205 (c*): fan-beam equiangular DD
 * forward projection; da is the angular cell size du/dsd. */
int cupyDistanceDrivenFanProjection(float* prj, const float* img, const float* deg, size_t nBatches, size_t nx,
                                    size_t ny, size_t nz, float dx, float dy, float dz, float cx, float cy,
                                    float cz, size_t nu, size_t nv, size_t nview, float da, float dv, float off_a,
                                    float off_v, float dsd, float dso, int typeProjector);
int cDistanceDrivenFanProjection(float* prj, const float* img, const float* deg, size_t nBatches, size_t nx,
                                 size_t ny, size_t nz, float dx, float dy, float dz, float cx, float cy, float cz,
                                 size_t nu, size_t nv, size_t nview, float da, float dv, float off_a, float off_v,
                                 float dsd, float dso, int typeProjector);

/* distanceDriven2D.cu:158 (cupy*) / :285 (c*): parallel-beam DD forward
 * projection (the reference injects dsd=1000, dso=500, :187). */
int cupyDistanceDrivenParallelProjection(float* prj, const float* img, const float* deg, size_t nBatches,
                                         size_t nx, size_t ny, size_t nz, float dx, float dy, float dz, float cx,
                                         float cy, float cz, size_t nu, size_t nv, size_t nview, float du, float dv,
                                         float off_u, float off_v, int typeProjector);
int cDistanceDrivenParallelProjection(float* prj, const float* img, const float* deg, size_t nBatches, size_t nx,
                                      size_t ny, size_t nz, float dx, float dy, float dz, float cx, float cy,
                                      float cz, size_t nu, size_t nv, size_t nview, float du, float dv, float off_u,
                                      float off_v, int typeProjector);

/* distanceDriven2D.cu:384 (cupy*) / :482 (c*): fan DD back projection,
 * accumulates into img. */
int cupyDistanceDrivenFanBackprojection(float* img, const float* prj, const float* deg, size_t nBatches, size_t nx,
                                        size_t ny, size_t nz, float dx, float dy, float dz, float cx, float cy,
                                        float cz, size_t nu, size_t nv, size_t nview, float da, float dv,
                                        float off_a, float off_v, float dsd, float dso, int typeProjector);
int cDistanceDrivenFanBackprojection(float* img, const float* prj, const float* deg, size_t nBatches, size_t nx,
                                     size_t ny, size_t nz, float dx, float dy, float dz, float cx, float cy, float cz,
                                     size_t nu, size_t nv, size_t nview, float da, float dv, float off_a,
                                     float off_v, float dsd, float dso, int typeProjector);

/* distanceDriven2D.cu:434 (cupy*) / :560 (c*): parallel DD back projection,
 * accumulates into img. */
int cupyDistanceDrivenParallelBackprojection(float* img, const float* prj, const float* deg, size_t nBatches,
                                             size_t nx, size_t ny, size_t nz, float dx, float dy, float dz,
                                             float cx, float cy, float cz, size_t nu, size_t nv, size_t nview,
                                             float du, float dv, float off_u, float off_v, int typeProjector);
int cDistanceDrivenParallelBackprojection(float* img, const float* prj, const float* deg, size_t nBatches,
                                          size_t nx, size_t ny, size_t nz, float dx, float dy, float dz, float cx,
                                          float cy, float cz, size_t nu, size_t nv, size_t nview, float du, float dv,
                                          float off_u, float off_v, int typeProjector);

/* distanceDriven3D.cu:184 (c*) / :264 (cupy*): tomosynthesis DD forward
 * projection (detector u=(1,0,0), v=(0,1,0)), overwrites prj.  detCenter and
 * src are [nview][3].  typeProjector 1 (branchless) selects the same
 * operator. */
int cupyDistanceDrivenTomoProjection(float* prj, const float* img, const float* detCenter, const float* src,
                                     size_t nBatches, size_t nx, size_t ny, size_t nz, float dx, float dy, float dz,
                                     float cx, float cy, float cz, size_t nu, size_t nv, size_t nview, float du,
                                     float dv, float off_u, float off_v, int typeProjector);
int cDistanceDrivenTomoProjection(float* prj, const float* img, const float* detCenter, const float* src,
                                  size_t nBatches, size_t nx, size_t ny, size_t nz, float dx, float dy, float dz,
                                  float cx, float cy, float cz, size_t nu, size_t nv, size_t nview, float du,
                                  float dv, float off_u, float off_v, int typeProjector);

/* distanceDriven3D.cu:312 (c*) / :393 (cupy*): tomosynthesis DD back
 * projection, overwrites img. */
int cupyDistanceDrivenTomoBackprojection(float* img, const float* prj, const float* detCenter, const float* src,
                                         size_t nBatches, size_t nx, size_t ny, size_t nz, float dx, float dy,
                                         float dz, float cx, float cy, float cz, size_t nu, size_t nv, size_t nview,
                                         float du, float dv, float off_u, float off_v, int typeProjector);
int cDistanceDrivenTomoBackprojection(float* img, const float* prj, const float* detCenter, const float* src,
                                      size_t nBatches, size_t nx, size_t ny, size_t nz, float dx, float dy, float dz,
                                      float cx, float cy, float cz, size_t nu, size_t nv, size_t nview, float du,
                                      float dv, float off_u, float off_v, int typeProjector);

/* siddonCone.cu:137 (c*) / :233 (cupy*): Siddon cone-beam forward projection
 * for arbitrary trajectories; accumulates into prj. */
int cupySiddonConeProjectionArbitrary(float* prj, const float* img, const float* detCenter, const float* detU,
                                      const float* detV, const float* src, size_t nBatches, size_t nx, size_t ny,
                                      size_t nz, float dx, float dy, float dz, float cx, float cy, float cz, size_t nu,
                                      size_t nv, size_t nview, float du, float dv, float off_u, float off_v);
int cSiddonConeProjectionArbitrary(float* prj, const float* img, const float* detCenter, const float* detU,
                                   const float* detV, const float* src, size_t nBatches, size_t nx, size_t ny,
                                   size_t nz, float dx, float dy, float dz, float cx, float cy, float cz, size_t nu,
                                   size_t nv, size_t nview, float du, float dv, float off_u, float off_v);

/* siddonCone.cu:282 (c*) / :378 (cupy*): Siddon cone-beam back projection
 * (transpose, same segment lengths); accumulates into img. */
int cupySiddonConeBackprojectionArbitrary(float* img, const float* prj, const float* detCenter, const float* detU,
                                          const float* detV, const float* src, size_t nBatches, size_t nx,
                                          size_t ny, size_t nz, float dx, float dy, float dz, float cx, float cy,
                                          float cz, size_t nu, size_t nv, size_t nview, float du, float dv,
                                          float off_u, float off_v);
int cSiddonConeBackprojectionArbitrary(float* img, const float* prj, const float* detCenter, const float* detU,
                                       const float* detV, const float* src, size_t nBatches, size_t nx, size_t ny,
                                       size_t nz, float dx, float dy, float dz, float cx, float cy, float cz,
                                       size_t nu, size_t nv, size_t nview, float du, float dv, float off_u,
                                       float off_v);

/* fbp.cu:165 (cupy*) / :204 (c*): equiangular fan ramp filter; typeFilter
 * 1 hamming, 2 hann, 3 cosine, else Ram-Lak.  Overwrites pFPrj. */
int cupyfbpFanFilter(float* pFPrj, const float* pPrj, int nBatches, size_t nu, size_t nv, size_t nview, float da,
                     float dv, float off_a, float off_v, float dsd, float dso, int typeFilter);
int cfbpFanFilter(float* pFPrj, const float* pPrj, int nBatches, size_t nu, size_t nv, size_t nview, float da,
                  float dv, float off_a, float off_v, float dsd, float dso, int typeFilter);

/* fbpParallel.cu:111 (cupy*) / :146 (c*): parallel-beam ramp filter. */
int cupyfbpParallelFilter(float* pFPrj, const float* pPrj, int nBatches, size_t nu, size_t nv, size_t nview,
                          float du, float dv, float off_u, float off_v, int typeFilter);
int cfbpParallelFilter(float* pFPrj, const float* pPrj, int nBatches, size_t nu, size_t nv, size_t nview, float du,
                       float dv, float off_u, float off_v, int typeFilter);

/* fbp.cu:362 (cupy*) / :409 (c*): pixel-driven fan FBP back projection,
 * accumulates into pImg. */
int cupyfbpFanBackprojection(float* pImg, const float* pPrj, const float* pDeg, size_t nBatches, size_t nx,
                             size_t ny, size_t nz, float dx, float dy, float dz, float cx, float cy, float cz,
                             size_t nu, size_t nv, size_t nview, float da, float dv, float off_a, float off_v,
                             float dsd, float dso);
int cfbpFanBackprojection(float* pImg, const float* pPrj, const float* pDeg, size_t nBatches, size_t nx, size_t ny,
                          size_t nz, float dx, float dy, float dz, float cx, float cy, float cz, size_t nu,
                          size_t nv, size_t nview, float da, float dv, float off_a, float off_v, float dsd,
                          float dso);

/* TotalVariation.cu:185 (cupy*) / :213 (c*) of the reference prior library
 * (libprior.so): SQS surrogate terms of the anisotropic TV prior.  s1, s2 and
 * var are [nBatches][nz][ny][nx]; wx, wy, wz weight the x, y, z differences.
 * (The reference host entry sizes its buffers for one batch item; this one
 * handles every item.) */
int cupyTVSQS3D(float* s1, float* s2, float* var, const float* img, float wx, float wy, float wz, size_t nBatches,
                size_t nx, size_t ny, size_t nz, float eps);
int cTVSQS3D(float* s1, float* s2, float* var, const float* img, float wx, float wy, float wz, size_t nBatches,
             size_t nx, size_t ny, size_t nz, float eps);

/* ======================================================================== */
/* 2. Extended entries: explicit stream, workspace and flags                */
/* ======================================================================== */
/* geom 0 = fan (g->du is the angular cell size), 1 = parallel.
 * Replaces the cupyDistanceDriven{Fan,Parallel}Projection path
 * (distanceDriven2D.cu:109-200).  Default: overwrite prj.  workspace may be
 * NULL (the library's stream-ordered pool supplies the scratch); otherwise
 * it holds workspace_bytes, at least a minimum that depends on the geometry.
 * The streamed projector runs in chunks of slices, as many per chunk as the
 * workspace holds up to 256 MiB of line tables and transposed slices;
 * ctp_dd2d_fp_workspace returns the size of the largest chunks.  Smaller
 * workspaces take smaller chunks, and one without room for a single slice's
 * tables runs the staged kernel.  Every path gives the same result. */
int ctp_dd2d_fp(void* prj, const void* img, const float* deg, const ctp_geometry* g, int geom, int typeProjector,
                unsigned flags, void* workspace, size_t workspace_bytes, void* stream);
size_t ctp_dd2d_fp_workspace(const ctp_geometry* g, int geom, int typeProjector, unsigned flags);

/* Caps the slices per chunk of the streamed forward projector of this
 * process (max_slices > 0), makes it run the staged kernel (0), or lifts the
 * cap (negative, the default).  Four slices of 512 x 512 per chunk keep the
 * line tables resident in the L2 (a seventh of the DRAM traffic, about 14%
 * more time).  For tests and tuning; no counterpart in the reference. */
int ctp_set_fp_stream_slices(int max_slices);

/* DD back projection (distanceDriven2D.cu:384-478).  Default: img += BP(prj)
 * in the reference's normalised form; CTP_FLAG_ADJOINT gives the exact
 * transpose of ctp_dd2d_fp. */
int ctp_dd2d_bp(void* img, const void* prj, const float* deg, const ctp_geometry* g, int geom, int typeProjector,
                unsigned flags, void* workspace, size_t workspace_bytes, void* stream);
size_t ctp_dd2d_bp_workspace(const ctp_geometry* g, int geom, int typeProjector, unsigned flags);

/* The DD forward projection of ctp_dd2d_fp for callers that cannot allocate
 * device memory at call time (their GPU memory is owned by another allocator,
 * or allocation is not allowed once their service runs).  It allocates
 * nothing: its scratch is a fixed 32 MiB array inside the library's device
 * memory, held by every GPU that loads the library until the process exits
 * (ctp_dd2d_fp_noalloc_capacity() returns the size).  The driver commits that
 * memory when it loads the library's device code on a device -- with lazy
 * module loading (CUDA_MODULE_LOADING=LAZY, the default) that can be the first
 * call of any entry of this library on the device -- so callers make one
 * early call (for example at start-up, before they reserve the rest of the
 * GPU, and before any stream capture).  Each call looks up the array's device
 * address (the lookup allocates nothing).  Requests needing more scratch
 * return CTP_ERR_TOO_LARGE.  All calls on a device share the array: calls that
 * overlap on the GPU race, so the caller must order them (one stream, or
 * events).  Output semantics and flags as ctp_dd2d_fp.  This entry has no
 * counterpart in the reference. */
int ctp_dd2d_fp_noalloc(void* prj, const void* img, const float* deg, const ctp_geometry* g, int geom,
                        int typeProjector, unsigned flags, void* stream);
size_t ctp_dd2d_fp_noalloc_capacity(void);

/* Number of operator nonzeros of the DD forward projector for one batch
 * item (the pixel count of every ray footprint on every main-axis line). */
int ctp_dd2d_nnz(unsigned long long* nnz_host, const float* deg, const ctp_geometry* g, int geom, void* stream);

/* Ramp filter (fbp.cu:15-162 fan, fbpParallel.cu:14-109 parallel); overwrites
 * fprj.  geom 0 = fan (g->du angular), 1 = parallel.  By default the windowed
 * ramp is built and applied in FP32 with transforms of length 2nu-1, the
 * construction of the reference (fbpMath.cu:90-241), which reproduces the
 * reference's own FP32 rounding (its output is 1-2e-5 from the exact result
 * at 700-900 cells).  CTP_FLAG_FILTER_EXACT builds the kernel in FP64 and
 * applies it in FP64 arithmetic: one launch over every row with no scratch
 * (workspace 0) up to 3456 cells, batched FP64 transforms above. */
int ctp_ramp_filter(float* fprj, const float* prj, const ctp_geometry* g, int geom, int typeFilter, unsigned flags,
                    void* workspace, size_t workspace_bytes, void* stream);
size_t ctp_ramp_filter_workspace(const ctp_geometry* g, int geom, int typeFilter, unsigned flags);
/* The same on host arrays, synchronous, as cfbpFanFilter / cfbpParallelFilter
 * (fbp.cu:204, fbpParallel.cu:146) with flags; no counterpart entry in the
 * reference. */
int ctp_ramp_filter_host(float* fprj, const float* prj, const ctp_geometry* g, int geom, int typeFilter,
                         unsigned flags);

/* Pixel-driven fan FBP back projection (fbp.cu:265-359); img += BP. */
int ctp_fbp_fan_bp(float* img, const float* prj, const float* deg, const ctp_geometry* g, unsigned flags,
                   void* stream);

/* Siddon cone-beam projector pair (siddonCone.cu:12-135). */
int ctp_siddon_fp(void* prj, const void* img, const float* detCenter, const float* detU, const float* detV,
                  const float* src, const ctp_geometry* g, unsigned flags, void* stream);
int ctp_siddon_bp(void* img, const void* prj, const float* detCenter, const float* detU, const float* detV,
                  const float* src, const ctp_geometry* g, unsigned flags, void* stream);
int ctp_siddon_nnz(unsigned long long* nnz_host, const float* detCenter, const float* detU, const float* detV,
                   const float* src, const ctp_geometry* g, void* stream);

/* Tomosynthesis DD projector pair (distanceDriven3DBoxInt.cu:28-280). */
int ctp_tomo_fp(float* prj, const float* img, const float* detCenter, const float* src, const ctp_geometry* g,
                unsigned flags, void* stream);
int ctp_tomo_bp(float* img, const float* prj, const float* detCenter, const float* src, const ctp_geometry* g,
                unsigned flags, void* workspace, size_t workspace_bytes, void* stream);
size_t ctp_tomo_bp_workspace(const ctp_geometry* g);

/* TV-SQS surrogate terms (TotalVariation.cu:21-149) on a stream. */
int ctp_tv_sqs(float* s1, float* s2, float* var, const float* img, float wx, float wy, float wz, size_t nbatch,
               size_t nx, size_t ny, size_t nz, float eps, void* stream);

/* Tomosynthesis FBP filter, fbpTomo.cu:386 (cupyFbpTomoFilter, device
   pointers; nBatches is an int in the reference's C signature).  Per view the
   ramp at the virtual pitch du*cos(tilt), windowed (typeFilter 1 Hamming,
   2 Hann, else none) with x/z cut-offs; fprj is overwritten.  Each view is
   filtered with its own kernel; the reference applies the first view's
   kernel to every view (CTP_FLAG_TOMO_FIRST_VIEW_KERNEL reproduces that). */
int cupyFbpTomoFilter(float* fprj, const float* prj, const float* detCenter, const float* src, int nBatches,
                      size_t nu, size_t nv, size_t nview, float du, float dx, float dz, int typeFilter,
                      float cutoffX, float cutoffZ);
/* The same with a ctp_geometry (nbatch, nu, nv, nview, du, dx, dz), a caller
   workspace (size from ctp_tomo_filter_workspace) and a stream. */
int ctp_tomo_filter(float* fprj, const float* prj, const float* detCenter, const float* src, const ctp_geometry* g,
                    int filter, float cutoff_x, float cutoff_z, unsigned flags, void* workspace,
                    size_t workspace_bytes, void* stream);
size_t ctp_tomo_filter_workspace(const ctp_geometry* g);

/* Fan-beam Siddon pair, host pointers: siddonFan.cu:127 (cSiddonFanProjection)
   and :201 (cSiddonFanBackprojection); da = du / dsd; outputs overwritten. */
int cSiddonFanProjection(float* prj, const float* img, const float* deg, int nBatches, size_t nx, size_t ny,
                         size_t nz, float dx, float dy, float dz, float cx, float cy, float cz, size_t nu, size_t nv,
                         size_t nview, float da, float dv, float off_a, float off_v, float dsd, float dso);
int cSiddonFanBackprojection(float* img, const float* prj, const float* deg, int nBatches, size_t nx, size_t ny,
                             size_t nz, float dx, float dy, float dz, float cx, float cy, float cz, size_t nu,
                             size_t nv, size_t nview, float da, float dv, float off_a, float off_v, float dsd,
                             float dso);
/* Pixel-driven parallel back projection, host pointers: fbpParallel.cu:271
   (cfbpParallelBackprojection); img overwritten. */
int cfbpParallelBackprojection(float* pImg, const float* pPrj, const float* pDeg, size_t nBatches, size_t nx,
                               size_t ny, size_t nz, float dx, float dy, float dz, float cx, float cy, float cz,
                               size_t nu, size_t nv, size_t nview, float du, float dv, float off_u, float off_v,
                               int typeProjector);
/* The same three on device pointers and a stream (no counterpart entries in
   the reference, which has only the host-pointer ones); g->du is the angular
   cell size for the fan pair; CTP_FLAG_ZERO_OUT writes instead of adding. */
int ctp_siddon_fan_fp(float* prj, const float* img, const float* deg, const ctp_geometry* g, unsigned flags,
                      void* stream);
int ctp_siddon_fan_bp(float* img, const float* prj, const float* deg, const ctp_geometry* g, unsigned flags,
                      void* stream);
int ctp_pixel_bp_parallel(float* img, const float* prj, const float* deg, const ctp_geometry* g, unsigned flags,
                          void* stream);

/* Bounded device-side waits that gave up on the current device since the
   library was loaded (the streamed forward projector polls an mbarrier for
   each chunk of line tables with an iteration limit, and counts a limit that
   ran out instead of spinning for ever; a CTA whose wait gave up lets its
   in-flight copies land and exits without writing its part of the output).
   0 in a healthy process.  The synchronous entries (c*, cupy*) compare this
   counter before and after the call and return CTP_ERR_WAIT_TIMEOUT when it
   went up; the asynchronous ctp_* entries return before their kernels run,
   so their callers read the counter.  No counterpart in the reference.
   Synchronises with the device. */
int ctp_wait_timeouts(unsigned int* count);

/* Poll limit of the first chunk wait of every CTA of the streamed forward
   projector on the current device (default CTP_WAIT_POLLS_DEFAULT).  A test
   of the failure path sets 0, so that the wait gives up at once (the waits
   that let in-flight copies land before a CTA exits keep the default), and
   restores CTP_WAIT_POLLS_DEFAULT afterwards.  No counterpart in the
   reference. */
int ctp_set_wait_limit(unsigned int first_chunk_polls);

/* 16-bit affine sinogram storage (no counterpart in the reference).  Each of
 * nrows rows of row_len samples (a view of one batch item: nv x nu samples)
 * keeps lo = its minimum and step = (maximum - minimum) / 65535; a sample is
 * the code round((y - lo) / step), read back as lo + step * code (error at
 * most step / 2).  Half the bytes of FP32, like BF16/FP16, with a rounding
 * error of 1/131070 of the view's range instead of the float formats'
 * 2^-9 (BF16) or 2^-12 (FP16) of each value.  Asynchronous on the stream. */
int ctp_quantize_u16(unsigned short* code, float* lo, float* step, const float* y, size_t nrows, size_t row_len,
                     void* stream);
/* y = lo + step * code, or y -= lo + step * code with CTP_FLAG_SUBTRACT (the
 * residual A x - y of an SQS iteration). */
int ctp_dequantize_u16(float* y, const unsigned short* code, const float* lo, const float* step, size_t nrows,
                       size_t row_len, unsigned flags, void* stream);
/* The exact (FP64) ramp filter of ctp_ramp_filter with CTP_FLAG_FILTER_EXACT
 * on a sinogram in 16-bit affine storage (one lo / step per view of each batch
 * item), dequantized as it is read; up to 3456 cells (CTP_ERR_UNSUPPORTED
 * above). */
int ctp_ramp_filter_u16(float* fprj, const unsigned short* code, const float* lo, const float* step,
                        const ctp_geometry* g, int geom, int typeFilter, void* stream);

/* Number of scratch allocations the library has made since it was loaded
   (stream-ordered pool, or cudaMallocAsync under graph capture), on every
   device: calls that get a workspace, and ctp_dd2d_fp_noalloc, add none.  No
   counterpart in the reference. */
int ctp_scratch_allocations(unsigned long long* count);

/* One SQS iteration with the TV prior, fused into one pass (no counterpart
   entry in the reference: there it is sqs_one_step, recon/cupy/sqs_algorithms.py
   :22-57, calling the TV-SQS terms of TotalVariation.cu:21-149, in several
   array operations):
       x_out = x - (bp + beta s1(x)) / (norm + beta s2(x))
   over nslices slices of ny x nx.  zlink[i] (may be NULL: no z coupling) bit 0
   says slice i has its z neighbour i-1 in the same volume, bit 1 the
   neighbour i+1.  norm holds norm_slices slices, read at slice i % norm_slices.
   x_out must not alias x.  x_lp (may be NULL) also receives x_out in bf16
   (flags CTP_FLAG_OUT_BF16) or fp16 (CTP_FLAG_OUT_FP16). */
int ctp_sqs_tv_update(float* x_out, void* x_lp, const float* x, const float* bp, const float* norm,
                      size_t norm_slices, const unsigned char* zlink, float wx, float wy, float wz, float beta,
                      float eps, size_t nx, size_t ny, size_t nslices, unsigned flags, void* stream);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* CTP_H */
