/*
 * vct.h -- C ABI of the B200-native MBFPA + FBP library (libvct.so).
 *
 * Drop-in boundary for the two hot paths of hagaakihiro/VirtualCT:
 *   MBFPA  Release_MBFPA_CPU_human/main.cpp:492-530  (energy loop over
 *          reprojection_TOMO, spectral sum, max-normalisation, gaussiannoise0)
 *   FBP    Release_FBP_CPU/main.cpp:137-167          (filterSinogram +
 *          reconstructImage)
 *
 * Conventions
 *   - Every function returns VCT_OK (0) or a negative VCT_E_* code; the text of
 *     the last error on the calling thread is available from vct_last_error().
 *   - Pointers without a _dev suffix are host pointers.  *_dev functions take
 *     device pointers on the context's device and enqueue on the context's
 *     stream (vct_set_stream); they return once the work is enqueued.
 *   - The caller owns every buffer it passes; the context owns its device
 *     scratch.  One host thread per context.
 *   - Layouts are the reference's raw file layouts: sinograms float32
 *     [views][width] (row = view), images float32 [N][N], element maps int16
 *     [M][N][N] holding element partial density x 1000 (g/cm^3).
 */
#ifndef VCT_H
#define VCT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VCT_OK 0
#define VCT_E_ARG (-1)         /* invalid argument or size */
#define VCT_E_CUDA (-2)        /* CUDA runtime error (message in vct_last_error) */
#define VCT_E_TIMEOUT (-3)     /* a bounded device wait gave up */
#define VCT_E_NOMEM (-4)       /* host or device allocation failed */
#define VCT_E_IO (-5)          /* file missing, short or malformed */
#define VCT_E_STATE (-6)       /* call order: e.g. forward before maps are set */
#define VCT_E_UNSUPPORTED (-7) /* configuration outside this build's limits */
#define VCT_E_RANGE (-8)       /* a measured value outside the range the reference accepts */

#define VCT_MAX_MATERIALS 8
#define VCT_MAX_BINS 1024 /* the reference's spectrum buffers hold 1024 bins (MB/main.cpp:338-339) */

/* Fan-beam geometry.  The first block holds the compile-time macros of
 * physParamsTOMO.h as runtime fields; the second block the input-txt fields
 * the hot path reads.  vct_geometry_default() fills the shipped values. */
typedef struct vct_geometry {
  double sid_cm;         /* DIST_BTWN_SRC_AND_ISOCENT_CM 85.0           MB/physParamsTOMO.h:25 */
  double det_radius_cm;  /* DETECTOR_RADIUS_CURVATURE_CM 142.6          MB/physParamsTOMO.h:27 */
  double det_src_iso_cm; /* DIST_BTWN_DETERCTORSRC_AND_ISOCENT_CM 85.0  MB/physParamsTOMO.h:28 */
  int start_channel;     /* Start_Channel 0                             MB/physParamsTOMO.h:43 */
  int end_channel;       /* End_Channel 609                             MB/physParamsTOMO.h:46 */
  double iso_channel;    /* isocenter_channel 304.5                     MB/physParamsTOMO.h:47 */
  double max_alpha;      /* Max_alpha 0.326086956                       MB/physParamsTOMO.h:56 */
  double max_beta;       /* Max_beta 0.326086956                        FBP/physParamsTOMO.h:50 */
  int views;             /* projImgHeight = GantryRotationPeriod*DataSamplingRate */
  int width;             /* projImgWidth: sinogram row stride (>= end_channel) */
  double start_view_deg; /* StartViewAngle */
  int recon_size;        /* reconSize N (square image) */
  double pixel_cm;       /* reconPixSize */
  int xfactor;           /* "Factor for output CT value" */
} vct_geometry;

/* Replaces the physParamsTOMO.h defaults + the shipped txt (800 views x 609
 * channels, 512 x 512 at 0.1 cm, xfactor 1). */
void vct_geometry_default(vct_geometry* g);

const char* vct_strerror(int code);
const char* vct_last_error(void);

typedef struct vct_ctx vct_ctx;

/* Creates a context on CUDA device `device` for geometry g.  Precomputes the
 * view trig tables (MB/projectionDataTOMO.cpp:362-368, MB/misc_TOMO.cpp:82-100)
 * and detector tables on the host and uploads them, and lists (one kernel on
 * the context's stream, then a wait for it) the rays the fast walk hands to
 * the exact walk, which the forward walks a warp per ray. */
int vct_create(const vct_geometry* g, int device, vct_ctx** out);
void vct_destroy(vct_ctx* ctx);
/* cudaStream_t passed as an opaque pointer; NULL = the context's own stream
 * (so the legacy default stream, whose handle is also NULL, is named by
 * cudaStreamLegacy, (void*)1). */
int vct_set_stream(vct_ctx* ctx, void* stream);
int vct_synchronize(vct_ctx* ctx);

/* ---------------------------------------------------------------- spectrum
 * Host-side restatement of attenuation_coefficient
 * (MB/prior_weight_production.cpp:180-297): reads the spectrum txt
 * (one header line, then "E_lo E_hi weight" in MeV), normalises the pdf in
 * float and fills the analytic mass attenuation table mu[M][NE] (cm^2/g) for
 * the elements given by atomic number Z (A = the reference's table for
 * H,C,N,O,P,Ca and Mg=24, Si=28).  pdf must hold VCT_MAX_BINS floats and mu
 * M*VCT_MAX_BINS floats.  Results are bit-identical to the reference. */
int vct_attenuation_coefficient(const char* spectrum_path, int nthin, const int* Z, int M,
                                float* mu, float* pdf, int* NE);

/* ----------------------------------------------------------------- MBFPA
 * Uploads the element maps int16 [M][N][N] (value = partial density x 1000;
 * the reference reads them with fread as short, MB/main.cpp:421-429, and
 * divides by 1000, :103).  Negative entries contribute nothing, as in
 * MB/reprojection_TOMO.cpp:151-155. */
int vct_set_maps(vct_ctx* ctx, const int16_t* maps, int M);
/* Stored map units per g/cm^3 (default 1000, the reference's "density x
 * 1000").  A finer scale (e.g. 16384: densities up to 2 g/cm^3 in steps of
 * 6e-5) lets iterative callers take small steps; no counterpart in the
 * reference.  Applies to the maps of every later call. */
int vct_set_density_scale(vct_ctx* ctx, double units_per_gcc);
int vct_set_maps_dev(vct_ctx* ctx, const int16_t* d_maps, int M);

/* Uploads mu [M][NE] (bin fastest, the Attenuation layout of
 * MB/reprojection_TOMO.cpp:156) and pdf [NE]. */
int vct_set_spectrum(vct_ctx* ctx, const float* mu, const float* pdf, int M, int NE);

/* Spectral summation mode of the forward epilogue. */
#define VCT_SUM_COMPENSATED 0 /* bins summed in an FP64 accumulator (default) */
#define VCT_SUM_REFERENCE 1   /* each bin rounded to float and summed in float in
                                 bin order, as MB/main.cpp:504 */
int vct_set_sum_mode(vct_ctx* ctx, int mode);

/* Ray-walk mode.  Both walk the reference's segments (MB/reprojection_TOMO.cpp
 * :113-283) with the same set-up, loop test and crossing rule.
 * VCT_WALK_EXACT evaluates every segment with the reference's own double
 * expressions (divisions and square roots included), so segment boundaries
 * match it bit for bit.  VCT_WALK_FAST (default) advances the minor
 * coordinate incrementally, tracks the next gridline, uses one precomputed
 * step length and splits crossing steps in 31-bit fixed point; rays whose
 * first major gridline is not a pixel boundary (pixel sizes that do not
 * divide 1 cm) and geometries where the rmax test can fire take the exact
 * walk.  Densities enter as s/1000 exactly in both modes. */
#define VCT_WALK_FAST 0
#define VCT_WALK_EXACT 1
int vct_set_walk_mode(vct_ctx* ctx, int mode);

/* Polyenergetic forward projection, un-normalised:
 *   sino[v][c] = sum_E pdf[E] * exp(-sum_m mu_m(E) * L_m(v,c) / xfactor)
 * with L_m the line integrals of the reference's ray walk
 * (MB/reprojection_TOMO.cpp:13-289, one walk per ray for all bins).
 * Rows v >= views/2*2 and channels outside [start_channel, end_channel) are 0,
 * as the reference leaves them.  With VCT_SUM_COMPENSATED each bin's
 * exponential is 2^-y, y = transp*log2(e) in FP64 split into integer and
 * fraction (the fraction through the SFU), and bins are summed in FP64. */
int vct_forward(vct_ctx* ctx, float* sino_out);
int vct_forward_dev(vct_ctx* ctx, float* d_sino_out);

/* Per-ray line integrals only: lint[v][c][m] in g/cm^2 (FP64). */
int vct_line_integrals_dev(vct_ctx* ctx, double* d_lint_out);

/* Full MBFPA as MB/main.cpp:492-530: forward, divide by the global maximum,
 * then additive Gaussian noise of standard deviation sigma with the
 * reference's clamps (p < 0 -> projection_min/10, p > 1 -> 1).  Noise is
 * counter-based Philox4x32-10 keyed by (seed, view, channel); sigma <= 0
 * skips it.  stats (optional, 3 floats) receives {max, min_normalised,
 * sum-of-segments as float}. */
int vct_mbfpa(vct_ctx* ctx, double sigma, uint64_t seed, float* sino_out, float* stats);
int vct_mbfpa_dev(vct_ctx* ctx, double sigma, uint64_t seed, float* d_sino_out);

/* vct_set_maps + vct_mbfpa for n slices of this context's geometry and
 * spectrum, pipelined (no counterpart in the reference, which projects one
 * slice per process): slice i's maps ([M][N][N] int16 at maps[i]) go
 * host->device on one copy stream while slice i-1 is projected and slice
 * i-2's sinogram ([views][width] float to out[i]) comes back on another, so
 * with pinned host buffers the copies hide behind the projections (pageable
 * buffers give the same results, with the copies serialised).  Slice i's
 * noise uses seed + i.  stats (optional): [n][3] as vct_mbfpa's.  Returns
 * when every sinogram is in host memory; the context keeps the last slice's
 * maps. */
int vct_mbfpa_many(vct_ctx* ctx, int n, const int16_t* const* maps, int M, double sigma, uint64_t seed,
                   float* const* out, float* stats);

/* One slice over several GPUs (no counterpart in the reference): each rank
 * projects some views, the ranks combine (max, min) and normalise their own
 * rows, and each backprojects one band of the image; virtualct_b200.sharded
 * does the collectives.  Pieced together, the results are bit-identical to
 * vct_mbfpa_dev and vct_fbp_dev on one GPU.
 *   vct_forward_views_dev: the un-normalised forward of views [v0, v1) of
 *     the views/2*2 used into those rows of d_out ([views][width]; other
 *     rows untouched), and the rows' (max, min) into d_maxmin (2 device
 *     floats, 8-byte aligned).
 *   vct_normalize_noise_rows_dev: max-normalisation and noise of rows
 *     [r0, r1) of [0, views) in place, with the global (max, min) in
 *     d_maxmin (the element-wise max of the ranks' max, min of their min);
 *     slice-wide noise keyed by (seed, view, channel) as vct_mbfpa_dev's.
 *   vct_fbp_band_count: the bands vct_fbp_band_dev splits the image into
 *     (N/2 orbit rows of the quarter-turn backprojector when views % 4 == 0
 *     and N is even, else N image rows).
 *   vct_fbp_band_dev: vct_fbp_dev's image for bands [band0, band1) only;
 *     other pixels are not written. */
int vct_forward_views_dev(vct_ctx* ctx, int v0, int v1, float* d_out, float* d_maxmin);
int vct_normalize_noise_rows_dev(vct_ctx* ctx, float* d_sino, int r0, int r1, const float* d_maxmin, double sigma,
                                 uint64_t seed);
int vct_fbp_band_count(vct_ctx* ctx, int* count);
int vct_fbp_band_dev(vct_ctx* ctx, const float* d_sino, int filter, int in_mode, int band0, int band1,
                     float* d_img);

/* lengthproj_TOMO (MB/lengthproj_TOMO.cpp:14-185; the reference's main calls
 * it at MB/main.cpp:407 and writes npf_float.raw): for every pixel of the
 * reconstruction circle, npf = sum over the views/2*2 views used of
 * (float)(lerp(proj, dj) * rr) -- rr the pixel-width chord of the line from
 * the source to the pixel centre, dj the channel where that line meets the
 * curved detector, edge channels clamped -- in float, in view order.
 * proj: [views/2*2][width], row k = the k-th view used (as main.cpp:354-370
 * builds it); z and couch_speed are the txt's reconstruction z and couch
 * speed.  The first view is the reference's (int)(z/pitch - views/2 + 1e-8)
 * (pitch = couch_speed/views), wrapped into the rotation; with couch_speed 0
 * (where the reference divides 0/0) the views start at 0.  npf: [N][N], 0
 * outside the circle.  The reference's [N][N][V] side tables are not kept. */
int vct_lengthproj(vct_ctx* ctx, const float* proj, double z, double couch_speed, float* npf);
int vct_lengthproj_dev(vct_ctx* ctx, const float* d_proj, double z, double couch_speed, float* d_npf);

/* The reference's iterative step (MB/main.cpp:432-600):
 *  - vct_lengthproj2: lengthproj_TOMO_2 (MB/lengthproj_TOMO.cpp:188-276), the
 *    same sum over the rows (ite-1)%thinout + k*thinout, k < (views/2*2)/
 *    thinout, with chord and channel rounded to float as the reference's
 *    side tables hold them (recomputed here, never stored);
 *  - vct_ir_update_dev: IR_ImageTOMO (MB/IR_ImageTOMO.cpp:19-72) on one
 *    N x N map: per mask pixel lambda = w_tv TV + w_prior TV(image - prior)
 *    + 1e-6, after = max(0, before + w (npf_re - npf/thinout + lambda)),
 *    w = wbefore (before / (npf/thinout - lambda) past iteration 300);
 *    d_prior may be NULL (zeros); pixels outside the mask are not written;
 *  - vct_squdiff_dev: calc_squdiff_quad (MB/main.cpp:111-134): d_out2[0] =
 *    sum (p - r)^2 and d_out2[1] = sum 0.5 p ln(p/r)^2 (only when
 *    ite == num_ite, else 0) over the rows of iteration ite, channels
 *    [start, end). */
int vct_lengthproj2(vct_ctx* ctx, const float* proj, double z, double couch_speed, int ite, int thinout, float* npf);
int vct_lengthproj2_dev(vct_ctx* ctx, const float* d_proj, double z, double couch_speed, int ite, int thinout,
                        float* d_npf);
int vct_ir_update_dev(vct_ctx* ctx, const float* d_before, const float* d_prior, const float* d_npf,
                      const float* d_npf_re, double wbefore, double w_tv, double w_prior, int ite, int thinout,
                      float* d_after);
int vct_squdiff_dev(vct_ctx* ctx, const float* d_proj, const float* d_reproj, int ite, int thinout, int num_ite,
                    double* d_out2);
/* One pass of the iterative step (MB/main.cpp:432-600, ite >= 1), host
 * buffers: the context's last energy bin alone projected (the un-normalised,
 * per-bin float sinogram the reference's step reads), calc_squdiff_quad
 * against proj ([views/2*2][width], the measured sinogram; *objective holds
 * the previous value on entry and the new one on return, *quadratic
 * optional), update_wbefore (MB/main.cpp:136-150) on *wbefore,
 * lengthproj_TOMO_2 of the projected bin, and IR_ImageTOMO from `before`
 * (the first element's map, g/cm^3) into `after` ([N][N]; values outside the
 * mask are kept).  npf: lengthproj_TOMO of the measured sinogram; prior may
 * be NULL. */
int vct_ir_step(vct_ctx* ctx, const float* proj, const float* npf, const float* before, const float* prior, double z,
                double couch_speed, int ite, int thinout, int num_ite, double w_tv, double w_prior, double* wbefore,
                double* objective, double* quadratic, float* after);

/* Only the normalisation + noise step on a device sinogram (in place). */
int vct_normalize_noise_dev(vct_ctx* ctx, float* d_sino, double sigma, uint64_t seed);

/* ------------------------------------------------------------------- FBP
 * filterSinogram + reconstructImage (Release_FBP_CPU/main.cpp:137-167) for
 * one slice.  filter: 1 Ram-Lak, 2 Shepp-Logan (prepareConstMap,
 * FBP/filterSinogramTOMO.cpp:9-138).  in_mode != 0 applies the "IN" class
 * window (filtered values outside [1000, 3e5] -> 0, :250-255).
 * sino: [views][width] transmission values p; img_out: [N][N]. */
int vct_fbp(vct_ctx* ctx, const float* sino, int filter, int in_mode, float* img_out);
int vct_fbp_dev(vct_ctx* ctx, const float* d_sino, int filter, int in_mode, float* d_img_out);
/* FBP that allocates nothing (no counterpart in the reference).  For callers
 * that cannot allocate device memory at the point where they reconstruct: a
 * process whose device memory is owned by another allocator or a fixed
 * budget, a real-time loop that must not wait on an allocation, library code
 * that may not fail on one.  The result equals vct_fbp_dev's within the FBP
 * tolerance (its filter and trig tables are built on the device, in double,
 * where vct_fbp_dev uploads host-built ones), without a context: g gives the
 * geometry (the limits of vct_create apply), d_sino [views][width] and d_img
 * [N][N] are the caller's device buffers on the current device, stream is a
 * cudaStream_t (NULL: the legacy default stream); the call returns once the
 * work is enqueued.  The intermediate buffers are static device arrays of
 * libvct, about 8 MB, limited to views <= 4096, channels <= 2048 and
 * views*channels <= 1048576; larger sizes return VCT_E_ARG.  The first call
 * on a device looks up those arrays' device addresses there, and with CUDA's
 * lazy module loading (the default) that is when the driver allocates them,
 * so it can fail with VCT_E_NOMEM: make it at start-up, before any stream
 * capture.  Later calls allocate nothing.  A call made after the device's
 * context was reset (cudaDeviceReset) repeats that set-up.  All calls share
 * the arrays (each call rewrites every element it reads), so calls that
 * overlap on the GPU -- on different streams, or from several threads --
 * race. */
int vct_fbp_noalloc(const vct_geometry* g, const float* d_sino, int filter, int in_mode, float* d_img,
                    void* stream);
/* Beam-hardening correction, MB/beam_hardening_correction.cpp:21-69 (the
 * reference's separate program on reprojection_float.raw): every
 * transmission p becomes exp(-(|y| + alpha |y|^beta)), y = -ln p (logarithm
 * in single precision, as the reference's C++ resolves log() of a float),
 * stored as float.  vct_beam_hardening works on [views][width] host buffers
 * (sino and out may alias), vct_beam_hardening_dev in place on the device.
 * vct_set_beam_hardening(ctx, alpha, beta) makes every later vct_fbp* apply
 * the same correction to its line integrals on the way into the filter (one
 * pass fewer over the sinogram; alpha 0 turns it off, the default). */
int vct_beam_hardening(vct_ctx* ctx, const float* sino, double alpha, double beta, float* out);
int vct_beam_hardening_dev(vct_ctx* ctx, float* d_sino, double alpha, double beta);
int vct_set_beam_hardening(vct_ctx* ctx, double alpha, double beta);

/* Transpose of the FBP (no counterpart in the reference).  With in_mode 0
 * the FBP image is linear in lam = -ln p: img = B F W lam (weight W,
 * filter F, backprojection B).  vct_fbp_transpose returns
 * lam_adj = W^T F^T B^T u for an image-space u [N][N], as [views][width]
 * (0 outside [start_channel, end_channel) and in rows >= views/2*2); the
 * gradient of a loss on the image w.r.t. p is then -lam_adj / p.  B^T is a
 * gather (one thread per view and detector bin, no atomics). */
int vct_fbp_transpose(vct_ctx* ctx, const float* u, int filter, float* lam_adj);
int vct_fbp_transpose_dev(vct_ctx* ctx, const float* d_u, int filter, float* d_lam_adj);
/* The filtered sinogram of the last vct_fbp* call, [views][C]. */
int vct_fbp_filtered_dev(vct_ctx* ctx, const float** d_fltd);

/* ---------------------------------------------------------------- adjoint
 * No counterpart in the reference (it has no gradient).  The model is the
 * forward of vct_forward: line integrals L = A rho of the reference walk
 * (A linear in the densities rho_m = maps_m / 1000, g/cm^3) and the
 * polyenergetic intensity y = sum_E pdf exp(-sum_m mu_m(E) L_m / xfactor).
 * The loss is the weighted log least squares of MB/main.cpp:125-126 with
 * y / ynorm (ynorm = sum_E pdf, the un-attenuated intensity) as the
 * normalised reprojection:
 *     l = 1/2 sum_i w_i (ln(y_i / ynorm) - ln p_i)^2
 * over rays (v < views/2*2, start_channel <= c < end_channel) with p_i > 0;
 * w_i = p_i when weights is NULL.  grad receives dl/drho_m, [M][N][N]
 * float, per g/cm^3 (divide by 1000 for per map unit).  A^T is the exact
 * transpose of the walk (its lumped first segment and folded border cells
 * included), computed pixel by pixel with no atomics; the result does not
 * depend on scheduling.  Uses the maps and spectrum set on the context.
 * Requires det_src_iso_cm == sid_cm (a fan centred on the source, as the
 * reference's geometry) and returns VCT_E_UNSUPPORTED otherwise.  The first
 * adjoint call of a context plans every ray once and waits for it.
 * meas, weights: [views][width]; loss (optional): FP64. */
int vct_forward_adjoint(vct_ctx* ctx, const float* meas, const float* weights, float* grad, double* loss);
/* Device buffers; d_loss (optional) is a device double; nothing waits. */
int vct_forward_adjoint_dev(vct_ctx* ctx, const float* d_meas, const float* d_weights, float* d_grad,
                            double* d_loss);
/* Vector-Jacobian product of the normalised forward: given d_dy = dl/d(y/ynorm)
 * [views][width], d_grad = dl/drho_m [M][N][N]. */
int vct_forward_vjp_dev(vct_ctx* ctx, const float* d_dy, float* d_grad);
/* A^T alone: d_out[m][pix] = sum_rays d_g[ray][m] * len(ray, pix) for
 * per-ray, per-element weights d_g [views/2*2][end-start][M] (float), M the
 * maps' element count; the transpose of vct_line_integrals_dev. */
int vct_adjoint_rays_dev(vct_ctx* ctx, const float* d_g, float* d_out);

/* Helical z-interpolation, MB/main.cpp:347-371 (start_angle_num 0,
 * UsedReconAngle 2): from a measured volume [rotations][views][width]
 * (vct_load_measured), the sinogram [views][width] of one reconstruction z.
 * View j < (views/2*2)/2 is blended with view j of the next rotation,
 * (1 - w) a + w b in FP64 with w = 0.5 |j - views/2| / (views/2), where the
 * next rotation exists within the volume (j + views <= (rotations-1)*views);
 * every other view is (1 - w) a + w a.  Rows from views/2*2 on are left as
 * they are in out.  _dev: device buffers, enqueued on stream (NULL: legacy
 * default stream); the host form copies through the given device. */
int vct_helical_sinogram(const float* volume, int rotations, int views, int width, float* out, int device);
int vct_helical_sinogram_dev(const float* d_volume, int rotations, int views, int width, float* d_out,
                             void* stream);

/* One projected gradient-descent step on device densities (no counterpart in
 * the reference): rho[i] = max(0, rho[i] - step * (grad_a[i] + grad_b[i]))
 * for i < count (grad_b may be NULL: one gradient), then maps[i] =
 * rho[i] * units rounded to nearest and clamped to [0, 32767], ready for
 * vct_set_maps_dev.  Enqueued on stream (a cudaStream_t, NULL: legacy
 * default stream); allocates nothing. */
/* Index checks (no counterpart in the reference).  libvct_bounds.so, built
 * beside libvct.so with -DVCT_BOUNDS=1, checks the kernels' computed indices
 * (the walks' map gathers, the adjoint's staged rays, the backprojector's
 * rows, lengthproj's views and channels, the measured-data planes); an access
 * whose check fails is skipped and counted.  Returns the count since the last
 * call on the current device (and clears it) and, in *where, unit * 100000 +
 * source line of a failing check (units: 1 forward, 2 adjoint, 3 FBP,
 * 4 lengthproj, 5 measured data).  libvct.so returns VCT_E_UNSUPPORTED. */
int vct_bounds_violations(unsigned long long* hits, int* where);

int vct_descent_step_dev(float* d_rho, const float* d_grad_a, const float* d_grad_b, double step, double units,
                         int16_t* d_maps, long long count, void* stream);
/* The same step with a diagonal scale (a preconditioner, no counterpart in
 * the reference): rho[i] = max(0, rho[i] - step * grad[i] * scale[i % period]),
 * then maps[i] as above.  period is the scale table's length (M*N*N for one
 * table shared by every slice of a [S][M][N][N] block).  Allocates nothing. */
int vct_descent_step_scaled_dev(float* d_rho, const float* d_grad, const float* d_scale, long long period,
                                double step, double units, int16_t* d_maps, long long count, void* stream);

/* ------------------------------------------------------------------ batch
 * Many slices of uneven size (geometry, grid, spectrum) in one captured CUDA
 * graph; no counterpart in the reference, which runs one slice per process.
 * A job either runs vct_mbfpa (+ vct_fbp) -- d_sino set, d_grad NULL -- or
 * the adjoint -- d_grad set.  All jobs of a batch have M elements and run
 * the same kind of work.  One run of an MBFPA batch packs every job's maps,
 * walks the rays of all jobs in ONE persistent launch (tiles of rays taken
 * from a global counter, so uneven jobs share the GPU without a tail per
 * job), then normalises, adds noise and reconstructs each job on parallel
 * streams.  An adjoint batch runs each job's vct_forward_adjoint_dev on the
 * parallel streams.  Device buffers are the caller's and are read or
 * written at every run; the maps may change between runs, the geometry and
 * spectrum may not.  With tune != 0, creation times candidate ray-tile sizes
 * of the persistent launch and view splits of the backprojector on the batch
 * itself and keeps the fastest. */
typedef struct vct_job {
  vct_geometry geo;
  const int16_t* d_maps;  /* device [M][N][N], density x 1000 */
  const float* mu;        /* host [M][NE], copied at creation */
  const float* pdf;       /* host [NE] */
  int NE;
  /* MBFPA jobs */
  double sigma;           /* noise standard deviation; <= 0: none */
  uint64_t seed;
  float* d_sino;          /* device [views][width]: the vct_mbfpa result */
  float* d_img;           /* device [N][N]: FBP of d_sino, or NULL */
  int filter;             /* 1 Ram-Lak, 2 Shepp-Logan (with d_img) */
  /* adjoint jobs (vct_forward_adjoint_dev) */
  const float* d_meas;    /* device [views][width] */
  const float* d_weights; /* device [views][width] or NULL */
  float* d_grad;          /* device [M][N][N] */
  double* d_loss;         /* device double, or NULL */
  double density_units;   /* map units per g/cm^3; 0 means 1000 (vct_set_density_scale) */
} vct_job;
typedef struct vct_batch vct_batch;
int vct_batch_create(const vct_job* jobs, int n, int M, int device, int tune, vct_batch** out);
/* Enqueue one run on stream (NULL: the batch's own stream). */
int vct_batch_run(vct_batch* b, void* stream);
/* Wait for runs on the batch's own stream. */
int vct_batch_synchronize(vct_batch* b);
/* The chosen launch parameters and the number of kernel nodes per run. */
int vct_batch_config(const vct_batch* b, int* tile_rays, int* blocks_per_sm, int* view_groups, int* kernels);
void vct_batch_destroy(vct_batch* b);
/* create (untuned) + run + wait + destroy. */
int vct_forward_batched(const vct_job* jobs, int n, int M, int device);

/* ------------------------------------------------------------ inspection */
/* Per-stage device times (no counterpart in the reference, whose only timers
 * are the clock() laps of FBP/misc.cpp:196-215).  With on != 0, every later
 * forward, FBP, FBP transpose and adjoint call on ctx records a CUDA event on
 * its stream before its first kernel stage and after each stage;
 * vct_stage_times waits for the last such call's events and returns, for up
 * to cap stages, the stage names (static strings) and milliseconds, with the
 * stage count in *n.  Off (the default), nothing is recorded. */
int vct_set_stage_timing(vct_ctx* ctx, int on);
int vct_stage_times(vct_ctx* ctx, int cap, const char** names, float* ms, int* n);
/* Number of in-grid walk segments of the last forward (the algorithmic work
 * unit of the forward kernel). */
int vct_last_segment_count(vct_ctx* ctx, long long* segments);
/* Number of kernels this context has launched since creation. */
long long vct_kernel_launches(vct_ctx* ctx);
int vct_version(void);
/* Philox4x32-10 (the noise generator of vct_mbfpa) evaluated on the host,
 * for known-answer tests. */
void vct_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

#ifdef __cplusplus
}
#endif
#endif /* VCT_H */
