/*
 * vct_oracle.h -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * A plain-C restatement of the reference's MBFPA and FBP arithmetic
 * (hagaakihiro/VirtualCT), used only as the checker by tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py.  The product
 * library (virtualct_b200/) never links, loads or calls it.
 *
 * Every function names the reference lines it restates.  Operation order and
 * types follow the reference exactly (double geometry, float densities and mu,
 * float accumulators where the reference has them), and the file is compiled
 * with -ffp-contract=off so rounding matches the reference's x86-64 -O2 build.
 *
 * Parity pin: tests/test_oracle_pin.py compares these functions with the
 * reference itself, compiled from its sources by oracle/Makefile into
 * oracle/_ref/, and with the golden outputs the reference ships.
 */
#ifndef VCT_ORACLE_H
#define VCT_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Runtime copy of the physParamsTOMO.h geometry macros plus the txt fields
 * the hot path reads.  orc_geom_default() gives the shipped values. */
typedef struct orc_geom {
  int start_channel;   /* Start_Channel 0          MB/physParamsTOMO.h:43 */
  int end_channel;     /* End_Channel 609          :46 */
  double iso_channel;  /* isocenter_channel 304.5  :47 */
  double max_alpha;    /* Max_alpha 0.326086956    :56 */
  double max_beta;     /* Max_beta  0.326086956    :60, FBP/physParamsTOMO.h:50 */
  double sid;          /* DIST_BTWN_SRC_AND_ISOCENT_CM 85.0            :25 */
  double det_radius;   /* DETECTOR_RADIUS_CURVATURE_CM 142.6           :27 */
  double det_src_iso;  /* DIST_BTWN_DETERCTORSRC_AND_ISOCENT_CM 85.0   :28 */
  int views;           /* projImgHeight (GantryRotationPeriod*DataSamplingRate) */
  int width;           /* projImgWidth: sinogram row stride */
  int recon_size;      /* N */
  double pixel_cm;     /* reconPixSize */
  int xfactor;         /* xfactor (txt field "Factor for output CT value") */
} orc_geom;

void orc_geom_default(orc_geom* g);

/* View angles and trig tables: MB/projectionDataTOMO.cpp:362-368,
 * MB/misc_TOMO.cpp:82-100 (FBP/projectionDataTOMO.cpp:201-208 is identical). */
void orc_trig_tables(int views, double start_view_deg, double* cos_t, double* sin_t);

/* Spectrum file + analytic mass attenuation: MB/prior_weight_production.cpp:180-297.
 * Z/A give the element table (the reference hard-codes H,C,N,O,P,Ca at :250-255).
 * mu is [M][NE] (bin fastest, stride NE).  Returns NE, or -1 on I/O error. */
int orc_spectrum(const char* path, int nthin, float* pdf, double* energy_mev, int cap);
void orc_attenuation(const double* energy_mev, int NE, const double* Z, const double* A, int M,
                     float* mu);

/* One ray walk (MB/reprojection_TOMO.cpp:53-283) for view cos/sin and channel
 * jj.  Writes segment lengths (cm), pixel indices and midpoint radii (cm);
 * returns the number of segments (0 when the ray misses the grid), or -1 when
 * cap is too small. */
int orc_walk(const orc_geom* g, double cosb, double sinb, int jj, double* seg_len, int* seg_pix,
             double* seg_r, int cap);

/* Forward projection, reference order: for every bin, transp is accumulated
 * over segments and materials exactly as MB/reprojection_TOMO.cpp:152-157,
 * the bin value is (float)(pdf*exp(-transp/xfactor)) (:196-197) and bins are
 * summed in float in bin order (MB/main.cpp:492-506).
 * rho: float densities [M][N][N] (int16/1000, MB/main.cpp:93-109).
 * full_out: [views][width] (rows >= views/2*2 and channels outside
 * [start,end) are left 0, as the reference leaves them).  nseg_out optional.
 * nthreads <= 0 uses OpenMP's default. */
void orc_forward_exact(const orc_geom* g, const double* cos_t, const double* sin_t, const float* rho,
                       int M, const float* mu, const float* pdf, int NE, float* full_out,
                       int* nseg_out, int nthreads);

/* Same geometry, evaluated in FP64 throughout: L_m = sum rho_m*len,
 * transp = sum_m mu_m*L_m, I = sum_E pdf*exp(-transp/xfactor), in double.
 * Optionally returns the per-ray line integrals L [views][width][M] (g/cm^2). */
void orc_forward_fp64(const orc_geom* g, const double* cos_t, const double* sin_t, const float* rho,
                      int M, const float* mu, const float* pdf, int NE, double* full_out,
                      double* lint_out, int nthreads);

/* As orc_forward_fp64, but densities are the stored integers divided by 1000
 * exactly (s/1000 in double) instead of the reference's float rounding of
 * (float)s/1000; the FP64 reference for a device path that carries s/1000
 * exactly.  maps: int16 [M][N][N]; negative entries contribute nothing. */
void orc_forward_fp64_maps(const orc_geom* g, const double* cos_t, const double* sin_t,
                           const short* maps, int M, const float* mu, const float* pdf, int NE,
                           double* full_out, double* lint_out, int nthreads);

/* ---- Adjoint support (no counterpart in the reference; FP64, test-only) ----
 * Exact intersection of the reference's ray (view cos/sin, channel jj; source
 * and detector as MB/reprojection_TOMO.cpp:53-74) with the N x N grid: every
 * pixel the line crosses with its true chord length (cm), in walk order.
 * Pixel index convention as the reference: col = floor(x/s + N/2),
 * row = floor(N/2 - y/s).  Returns the count, -1 if cap is too small. */
int orc_siddon(const orc_geom* g, double cosb, double sinb, int jj, double* seg_len, int* seg_pix, int cap);

/* Exact-Siddon forward projection of per-material images x (double [M][N][N])
 * to per-ray line integrals out (double [views][width][M]). */
void orc_siddon_project(const orc_geom* g, const double* cos_t, const double* sin_t, const double* x, int M,
                        double* out, int nthreads);

/* The reference walk as a linear operator A on FP64 densities (no counterpart
 * in the reference, which only walks int16 maps):
 *   orc_walk_project:     out[j][jj][m] = sum_seg rho_m(pix) * len   (A rho)
 *   orc_walk_backproject: out[m][pix]  = sum_rays w[j][jj][m] * len  (A^T w)
 * Segments whose midpoint radius reaches rmax are dropped, as in the walk. */
void orc_walk_project(const orc_geom* g, const double* cos_t, const double* sin_t, const double* rho, int M,
                      double* out, int nthreads);
/* A rho for a list of rays only (ray = view * width + channel); out [nrays][M]. */
void orc_walk_project_rays(const orc_geom* g, const double* cos_t, const double* sin_t, const double* rho, int M,
                           const int* rays, int nrays, double* out, int nthreads);
void orc_walk_backproject(const orc_geom* g, const double* cos_t, const double* sin_t, const double* w, int M,
                          double* out, int nthreads);

/* lengthproj_TOMO (MB/lengthproj_TOMO.cpp:14-185) for one slice: for every
 * mask pixel, npf = sum over the views used of (float)(lerp(proj, dj) * rr),
 * rr the pixel-width chord of the source-to-pixel-centre line, dj its hit on
 * the curved detector in channels, accumulated in float in view order.
 * proj: [views used][width] (row = view index from the first view used).
 * The first view follows the reference's z / pitch formula; with
 * couch_speed == 0 (pitch 0, where the reference divides 0/0 and reads its
 * trig tables out of range) the views start at 0. */
void orc_lengthproj(const orc_geom* g, const double* cos_t, const double* sin_t, const float* proj, double z,
                    double couch_speed, float* npf);

/* Beam-hardening correction, MB/beam_hardening_correction.cpp:49-56, in place
 * (mins: the minima before and after, may be NULL). */
void orc_beam_hardening(float* p, long long n, double alpha, double beta, double* mins);

/* lengthproj_TOMO_2 (MB/lengthproj_TOMO.cpp:188-276): orc_lengthproj over the
 * rows (ite-1)%thinout + k*thinout, k < (views/2*2)/thinout, with the chord
 * and channel rounded to float as the reference's side tables hold them. */
void orc_lengthproj2(const orc_geom* g, const double* cos_t, const double* sin_t, const float* proj, double z,
                     double couch_speed, int ite, int thinout, float* npf);
/* IR_ImageTOMO (MB/IR_ImageTOMO.cpp:19-72) on one N x N map (prior may be
 * NULL); `after` keeps its values outside the mask. */
void orc_ir_update(int N, const float* before, const float* prior, const float* npf, const float* npf_re,
                   double wbefore, double w_tv, double w_prior, int ite, int thinout, float* after);

/* Max-normalisation (MB/main.cpp:511-522) followed by gaussiannoise0
 * (MB/main.cpp:42-76) with glibc rand() after srand(seed) (the reference
 * never seeds: seed 1).  order selects which Uniform0() call in rand_gauss0
 * is evaluated first (the C++ expression leaves it unspecified); the shipped
 * golden fixes it.  sigma <= 0 normalises only.  Returns the noise-free
 * normalised minimum (projection_min). */
double orc_normalize_noise(float* sino, int nn, double sigma, unsigned seed, int order);

/* FBP: prepareConstMap (FBP/filterSinogramTOMO.cpp:9-138) -> h[C][C];
 * filterSinogram (:205-275); reconstructImage (FBP/reconstructImageTOMO.cpp:11-105). */
void orc_fbp_constmap(const orc_geom* g, int filter, double* h);
void orc_fbp_filter(const orc_geom* g, const float* sino, const double* h, int in_mode,
                    float* fltd);
/* Transpose of the FBP's linear part (in_mode 0) as a map from lam = -ln p
 * [views][width] to the image, in FP64 (no counterpart in the reference):
 * out = W^T F^T B^T u for u [N][N]; h is prepareConstMap's [C][C] matrix.
 * B^T follows orc_fbp_backproject's formula (FBP/reconstructImageTOMO.cpp:
 * 57-93), F^T the filter of FBP/filterSinogramTOMO.cpp:233-243. */
void orc_fbp_fp64(const orc_geom* g, const float* sino, const double* h, const double* cos_t,
                  const double* sin_t, double* img);
void orc_fbp_transpose(const orc_geom* g, const double* h, const double* cos_t, const double* sin_t,
                       const double* u, double* out);
void orc_fbp_backproject(const orc_geom* g, const float* fltd, const double* cos_t,
                         const double* sin_t, float* img);

/* Measured-data ingestion, MB/projectionDataTOMO.cpp:324-508.  The raw
 * layout constants of MB/physParamsTOMO.h: ch = NumberOfChannels (609),
 * skip = NumberOfSkips (27), air_rows = AirScn_Sinogram_Height (800),
 * air_blocks = AirScn_Sinogram_Number (5), [start_ch, end_ch) =
 * [Start_Channel, End_Channel).  views is projImgHeight after the sino_fact
 * thinning (nskip); rows_per_view 5 when DataSamplingRateOrig >= 200, else 1.
 * Files are read with fread into buffers that persist between reads, as the
 * reference reads them.  Returns -1 when either file is missing, -2 when an
 * IN-mode value in the channel window exceeds 1 (*maxv = that value: the
 * reference stops there), -3 when the sizes would take the reference outside
 * its buffers, else the rotations read (*maxv = IN-mode maximum, 0 for PR).
 * vol and mask are [rotations][views][width]. */
int orc_load_measured(const char* proj_file, const char* air_file, int in_mode, int width, int views, int nskip,
                      int rotations, int rows_per_view, int ch, int skip, int air_rows, int air_blocks,
                      int start_ch, int end_ch, float* vol, unsigned char* mask, double* maxv);
/* Helical z-interpolation of MB/main.cpp:347-371 (start_angle_num 0,
 * UsedReconAngle 2): out [views][width] from vol [rotations][views][width];
 * rows from views/2*2 on are left as they are. */
void orc_helical(const float* vol, int rotations, int views, int width, float* out);

/* Inscribed-circle mask: MB/misc_TOMO.cpp:10-39, FBP/misc.cpp:9-37. */
void orc_mask(int N, unsigned char* mask);

#ifdef __cplusplus
}
#endif
#endif
