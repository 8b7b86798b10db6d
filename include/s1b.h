/*
 * s1b -- B200-native (sm_100a) kernels for the s1proc per-burst
 * interferogram chain: TOPS deramp, FP64 zero-Doppler geocoding with
 * bilinear resampling and reramp (geo2rdr), crossmul with multilooking and
 * coherence, and the Goldstein filter.
 *
 * C ABI: plain pointers and sizes, no C++ or torch types.  Every function
 * returns an int status (S1B_OK = 0) and never exits the process.  Device
 * pointers are caller-owned CUDA device memory; `stream` is a cudaStream_t
 * passed as void* (NULL = the legacy default stream).  Calls are
 * asynchronous with respect to the host unless stated otherwise; errors
 * detected on the device are reported through the status words the
 * functions document.
 *
 * The reference project exposes this path as standalone executables
 * (geo2rdr, crossmul_daemon, crossmul, goldstein) that exchange binary files.
 * Each entry point below names the reference code it replaces.
 */
#ifndef S1B_H
#define S1B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define S1B_OK 0
#define S1B_ERR_INVALID_ARGUMENT 1
#define S1B_ERR_CUDA 2
#define S1B_ERR_TOO_LARGE 3
#define S1B_ERR_EMPTY 4          /* empty DEM window / empty overlap: nothing to do */
#define S1B_ERR_NO_DEVICE 5
#define S1B_ERR_UNSUPPORTED 6

/* Human-readable status text (static storage). */
const char *s1b_status_string(int status);
/* Library version, major*10000 + minor*100 + patch. */
int s1b_version(void);
/* Last CUDA error text recorded by this thread's most recent failing call. */
const char *s1b_last_error(void);
/* sizeof(s1b_burst_plan_t) and sizeof(s1b_orbit_poly_t) as compiled into the
 * library, for bindings that mirror the structs (ctypes, cgo). */
size_t s1b_sizeof_burst_plan(void);
size_t s1b_sizeof_orbit_poly(void);

/* ---------------------------------------------------------- input records */
#define S1B_MAX_STATE_VECTORS 64
#define S1B_MAX_ORBIT_WINDOWS (S1B_MAX_STATE_VECTORS - 3)

/* Orbit state vectors (host arrays), the content of the reference's orbit
 * text file: read_orbit_ascii, csrc/src/orbit.cu:147-168.  x, v: [n*3]. */
typedef struct s1b_orbit_t {
  int32_t n;
  const double *t;
  const double *x;
  const double *v;
} s1b_orbit_t;

/* FM-rate or Doppler-centroid polynomial records (host arrays):
 * read_polynomials, csrc/src/sario.cu:80-103.  Each record holds the
 * azimuth time, the reference range time t0 and c0 + c1 dt + c2 dt^2. */
typedef struct s1b_poly_table_t {
  int32_t n;
  const double *time;
  const double *t0;
  const double *c0;
  const double *c1;
  const double *c2;
} s1b_poly_table_t;

/* Subswath radar parameters: the DB keys geo2rdr reads,
 * csrc/src/geo2rdr.cu:333-349. */
typedef struct s1b_radar_t {
  int32_t samples_per_burst;
  int32_t lines_per_burst;
  double prf;
  double wvl;
  double hmin;
  double hmax;
  double range_sampling_rate;
  double slant_range_time;
  double azimuth_steering_rate; /* degrees / s */
  double azimuth_time_interval;
  double radar_frequency;
} s1b_radar_t;

/* One burst: azimuthTimeSeconds<i>, first/lastValidLine<i>,
 * first/lastValidSample<i> (csrc/src/geo2rdr.cu:365-376). */
typedef struct s1b_burst_t {
  double azimuth_time;
  int32_t first_valid_line;
  int32_t last_valid_line;
  int32_t first_valid_sample;
  int32_t last_valid_sample;
} s1b_burst_t;

/* Lat/lon grid of the DEM: readrsc, csrc/src/sario.cu:12-60. */
typedef struct s1b_rsc_t {
  int32_t nlat;
  int32_t nlon;
  double latmax; /* Y_FIRST */
  double lonmin; /* X_FIRST */
  double dlat;   /* Y_STEP (negative) */
  double dlon;   /* X_STEP */
} s1b_rsc_t;

/* Orbit as piecewise polynomials: one degree-7 polynomial per 4-vector
 * window (the same interpolant as the reference's 4-point Hermite,
 * csrc/src/orbit.cu:170-245), expanded around the window centre. */
typedef struct s1b_orbit_poly_t {
  int32_t n_state;
  int32_t n_win; /* n_state - 3; window w (1..n_win) uses vectors w-1..w+2 */
  double t0;     /* time of state vector 0 */
  double inv_dt; /* 1 / (t[1] - t[0]), the window selector of orbit.cu:229 */
  double tc[S1B_MAX_ORBIT_WINDOWS];
  double c[S1B_MAX_ORBIT_WINDOWS][3][8];
} s1b_orbit_poly_t;

/* Everything the reference computes on the host for one burst before its
 * kernels run (csrc/src/geo2rdr.cu:387-400, 469-542, 569-600), plus the
 * orbit polynomials.  Produced by s1b_burst_plan(); passed to the kernels
 * by value.  The DEM window is on the RSC grid, [top, bottom) x [left, right). */
typedef struct s1b_burst_plan_t {
  s1b_orbit_poly_t orbit;
  int32_t lines, samples;
  int32_t first_valid_line, last_valid_line, first_valid_sample, last_valid_sample;
  int32_t win_left, win_top, win_right, win_bottom;
  int32_t rsc_nlat, rsc_nlon;
  double tstart, dtaz, ati;
  double rngstart, dmrg;
  double slant_range_time, range_sampling_rate;
  double wvl, k4pi_wvl; /* 4 pi / wvl */
  double tmid, xmid[3], vmid[3], amid[3];
  double ks, etac0;
  double fm[4]; /* interpolated FM-rate t0, c0, c1, c2 at the burst centre */
  double dc[4]; /* interpolated Doppler-centroid t0, c0, c1, c2 */
  double lat0, lon0, dlat, dlon; /* lat of window row 0, lon of window column 0 */
  double latlon_box[4];          /* latmin, latmax, lonmin, lonmax */
} s1b_burst_plan_t;

/* Host only.  Fill `plan` for one burst.  Returns S1B_ERR_EMPTY (plan still
 * filled) when the burst's DEM window is empty, as geo2rdr skips it
 * (csrc/src/geo2rdr.cu:583-584).  `rsc` may be NULL (no DEM window). */
int s1b_burst_plan(const s1b_radar_t *radar, const s1b_orbit_t *orbit,
                   const s1b_poly_table_t *fm, const s1b_poly_table_t *dc,
                   const s1b_burst_t *burst, const s1b_rsc_t *rsc,
                   s1b_burst_plan_t *plan);

/* Host only.  Orbit polynomials from state vectors. */
int s1b_orbit_poly(const s1b_orbit_t *orbit, s1b_orbit_poly_t *poly);

/* Host only.  Burst footprint [latmin, latmax, lonmin, lonmax] at heights
 * hmin..hmax: replaces bounds(), csrc/src/bounds.cu:288-317. */
int s1b_bounds(const s1b_orbit_poly_t *orbit, double start_time, double end_time,
               double start_rng, double end_rng, double hmin, double hmax,
               double latlons[4]);

/* Host only.  Orbit position/velocity at n times: replaces intp_orbit,
 * csrc/src/orbit.cu:224-245 (and s1proc.orbit.interp_orbit). */
int s1b_orbit_eval_host(const s1b_orbit_poly_t *orbit, const double *t, int64_t n,
                        double *satx, double *satv);

/* One burst for s1b_burst_geometry (device record): what the reference's
 * geo2rdr reads from its DB for the burst (csrc/src/geo2rdr.cu:333-376). */
typedef struct s1b_burst_geometry_in_t {
  int32_t orbit;              /* index into the orbit-polynomial array */
  int32_t fm_table, dc_table; /* indices into the packed FM-rate / Doppler tables */
  int32_t lines, samples;
  double tstart;              /* azimuthTimeSeconds<i> */
  double prf, azimuth_time_interval, slant_range_time, range_sampling_rate;
  double radar_frequency, azimuth_steering_rate; /* Hz, degrees / s */
  double hmin, hmax;
} s1b_burst_geometry_in_t;

/* Result of s1b_burst_geometry for one burst (device record). */
typedef struct s1b_burst_geometry_t {
  double latlon_box[4]; /* footprint latmin, latmax, lonmin, lonmax at hmin..hmax */
  double ks, etac0;     /* TOPS steering rate term and etac at the first range sample */
  double fm[4], dc[4];  /* FM-rate / Doppler t0, c0, c1, c2 at the burst centre */
  int32_t win[4];       /* DEM window left, top, right, bottom on `rsc` (0 without rsc) */
  int32_t status;       /* 0 ok; 1 a bad index or radar parameter (record zeroed) */
} s1b_burst_geometry_t;

/* Burst geometry prep of n bursts on the GPU in one launch, FP64: the
 * footprint at hmin..hmax (bounds/rah2ll, csrc/src/bounds.cu:237-317, as
 * geo2rdr.cu:387-400 calls it), the DEM window on `rsc` (569-586) and the
 * FM-rate / Doppler interpolation and TOPS steering term at the burst
 * centre (469-542) -- the host planner's functions (s1b_burst_plan) on the
 * device.  orbits: device [n_orbits] (s1b_orbit_poly); tables: device
 * [n_tables * max_records * 5] records (time, t0, c0, c1, c2), table_records:
 * device [n_tables] record counts; bursts, out: device [n]; rsc: host
 * pointer or NULL. */
int s1b_burst_geometry(const s1b_orbit_poly_t *orbits, int32_t n_orbits, const double *tables,
                       const int32_t *table_records, int32_t n_tables, int32_t max_records,
                       const s1b_burst_geometry_in_t *bursts, int32_t n, const s1b_rsc_t *rsc,
                       s1b_burst_geometry_t *out, void *stream);

/* ------------------------------------------------------------- geo2rdr */

/* TOPS deramp of one burst: out = in * exp(-i pi kt (eta - etaref)^2).
 * Replaces deramp_burst, csrc/src/geo2rdr.cu:138-158 (+ the host
 * coefficients at 469-542).  in/out: complex64 [lines * samples] device
 * (in == out allowed).  Phase in FP64, reduced mod 2 pi, FP32 rotation. */
int s1b_deramp(const s1b_burst_plan_t *plan, const void *in, void *out, void *stream);

/* Sample types of SLC input: complex64 (what the reference's geo2rdr reads
 * from its stdin pipe) or complex int16 (re, im int16 pairs: the sample type
 * of the Sentinel-1 measurement TIFF, which the reference widens to complex64
 * on the host with GDAL before piping it, s1proc/sentinel_scene.py:164-207). */
#define S1B_SAMPLES_C64 0
#define S1B_SAMPLES_CI16 1

/* s1b_deramp on complex int16 input: in int16 [lines * samples * 2] device
 * (re, im), out complex64 [lines * samples] device.  The widening to float is
 * exact, so the result equals s1b_deramp on the widened complex64 burst bit
 * for bit.  Ingest boundary: replaces the host-side widening and the 8-byte
 * samples of the stdin pipe (s1proc/sentinel_scene.py:164-207,
 * geo2rdr.cu:545-557) with 4-byte samples widened on the device. */
int s1b_deramp_ci16(const s1b_burst_plan_t *plan, const void *in, void *out, void *stream);

/* Geocode a deramped burst onto the plan's DEM window: per DEM pixel FP64
 * llh->ECEF, zero-Doppler Newton, validity window, bilinear interpolation,
 * reramp and range phase.  Replaces reproject + find_nonzero_rows,
 * csrc/src/geo2rdr.cu:86-128, 170-248, 273-299.
 *   dem:       int16 device pointer to the window's first pixel (row `win_top`,
 *              column `win_left` of the RSC grid); `dem_pitch` elements per row.
 *   deramped:  complex64 [lines * samples] device.
 *   out:       complex64 [(win_bottom-win_top) * (win_right-win_left)] device.
 *   rows:      int32[2] device, or NULL: first and one-past-last window row
 *              holding a non-zero output pixel (first = nrow, last = -1 when
 *              none), like the reference's d_first/d_last. */
int s1b_geo2rdr(const s1b_burst_plan_t *plan, const int16_t *dem, int64_t dem_pitch,
                const void *deramped, void *out, int32_t *rows, void *stream);

/* Sample coordinates of every pixel of the plan's DEM window as the
 * geocoding solves them (per-warp orbit patch, line-model seeds, chord
 * Newton, in the frame's 128-row tiles, every pixel solved): az = line,
 * rg = sample of the burst, float64 [(win_bottom-win_top) * (win_right-
 * win_left)] device.  The reference computes them in-register and never
 * writes them (azoff/rgoff of reproject, csrc/src/geo2rdr.cu:197-207); here
 * they state the geocoding's offset error against an FP64 restatement. */
int s1b_geo2rdr_grid_offsets(const s1b_burst_plan_t *plan, const int16_t *dem, int64_t dem_pitch,
                             double *az, double *rg, void *stream);

/* Culling of geocoding work outside the burst's valid lines, on by default,
 * for every later s1b_geo2rdr and frame launch in the process (a frame's
 * captured graph keeps the setting it was captured with).  Blocks of 32
 * window rows whose azimuth lines lie outside [first_valid_line + 5,
 * last_valid_line - 5) at every int16 height are written as zeros without
 * their zero-Doppler solves; the products are identical either way.  No
 * reference counterpart (an execution choice).  Returns the previous setting. */
int s1b_set_geocode_culling(int32_t on);

/* Zero-Doppler solve for arbitrary ECEF points (device arrays, n points):
 * replaces orbitrangetime / orbitrangetime_vec (csrc/src/orbit.cu:247-280,
 * s1proc/orbit.py:118-188).  Seeds every point with (tline0, orbit(tline0)).
 * xyz: [n*3] f64; tline: [n] f64; dr: [n*3] f64 (or NULL). */
int s1b_zero_doppler(const s1b_orbit_poly_t *orbit, const double *xyz, int64_t n,
                     double tline0, double *tline, double *dr, void *stream);

/* Geodetic -> ECEF (device arrays [n*3], degrees/metres): replaces llh2xyz,
 * csrc/src/orbit.cu:15-35 and s1proc/geometry.py:150-162, 204-216. */
int s1b_llh2xyz(const double *llh, double *xyz, int64_t n, void *stream);

/* ------------------------------------------------- crossmul + multilook */

/* One interferogram: conj(ref) * sec over the aligned box, averaged over
 * rowlook x collook, together with the power looks of both SLCs and the
 * coherence.  Replaces conj_mul + cpx_col_look + cpx_row_look (+ point_angle)
 * of crossmul_daemon (csrc/src/sario.cu:199-286, crossmul_daemon.cu:921-975)
 * and the amplitude/coherence NumPy code (s1proc/coherence.py:14-147).
 *   ref/sec: complex64 device rasters of ref_height x ref_width (sec_...);
 *            pixel (r, c) of the global grid is at
 *            ref[(r - ref_top) * ref_width + (c - ref_left)].
 *   box:     full-resolution [top, top + nrow_ml*rowlook) x
 *            [left, left + ncol_ml*collook), inside both rasters.
 *   outputs  (each may be NULL), [nrow_ml * ncol_ml]:
 *     ifg   complex64  mean conj(ref)*sec
 *     amp1  float32    sqrt(mean |ref|^2)
 *     amp2  float32    sqrt(mean |sec|^2)
 *     coh   float32    |ifg| / (amp1 + 1e-12) / (amp2 + 1e-12); values > 1
 *                      replaced by a uniform [0,1) value hashed from
 *                      (fill_seed, output index)
 *     phase float32    atan2(ifg)  (--out-float) */
int s1b_crossmul_looks(const void *ref, int32_t ref_left, int32_t ref_top, int32_t ref_width,
                       int32_t ref_height, const void *sec, int32_t sec_left, int32_t sec_top,
                       int32_t sec_width, int32_t sec_height,
                       int32_t left, int32_t top, int32_t nrow_ml, int32_t ncol_ml,
                       int32_t rowlook, int32_t collook, void *ifg, float *amp1, float *amp2,
                       float *coh, float *phase, uint64_t fill_seed, void *stream);

/* Host only.  Intersection box of two cropped rasters aligned to the looks and
 * the output header, as crossmul_daemon.cu:612-666 (union = 0) or the legacy
 * crossmul.cu:191-213 (union = 1).  hdr1/hdr2: the 6 leading header words
 * [nrow0, ncol0, left, top, right, bottom].  box_out: [left, top, right,
 * bottom]; hdr_out: 6 words.  Returns S1B_ERR_EMPTY for an empty box. */
int s1b_crossmul_box(const int32_t *hdr1, const int32_t *hdr2, int32_t rowlook,
                     int32_t collook, int32_t use_union, int32_t *box_out,
                     int32_t *hdr_out);

/* ------------------------------------------------- radar-grid coregistration
 * (no reference counterpart: the reference geocodes every SLC onto a lat/lon
 * grid instead; these resample the secondary onto the reference radar grid
 * with the reference's geometry and TOPS formulas). */

#define S1B_INTERP_BILINEAR 0
#define S1B_INTERP_SINC8 1

/* Secondary sample coordinates of every pixel of the reference radar grid:
 * for float64 lat/lon/height rasters [lines * samples] of the reference
 * grid, the zero-Doppler time and range on the secondary orbit of `plan`
 * (the formulas of csrc/src/geo2rdr.cu:197-207), stored as float32 offsets
 * relative to the pixel index: az_off = az - row, rg_off = rg - column. */
int s1b_geo2rdr_offsets(const s1b_burst_plan_t *plan, const double *lat, const double *lon,
                        const double *hgt, int32_t lines, int32_t samples, float *az_off,
                        float *rg_off, void *stream);

/* s1b_geo2rdr_offsets plus the offsets' height sensitivities daz_dh, drg_dh
 * (samples per metre, float32 [lines * samples]).  A height error moves the
 * ground point of a reference pixel along the reference's zero-Doppler
 * iso-range circle (dp = (rhat_r x V_r) / (up . (rhat_r x V_r)), the
 * reference pixel being the reference sample (row, col) of ref_plan); the
 * secondary's zero-Doppler time moves by (V.dp) / (|V|^2 - dr.A) and its
 * range by rhat.(dp - V dt/dh).  Carries a DEM-error field into the offsets. */
int s1b_geo2rdr_offsets_dh(const s1b_burst_plan_t *plan, const s1b_burst_plan_t *ref_plan,
                           const double *lat, const double *lon, const double *hgt, int32_t lines,
                           int32_t samples, float *az_off, float *rg_off, float *daz_dh, float *drg_dh,
                           void *stream);

/* Resample the secondary burst of `plan` (complex64 [plan->lines *
 * plan->samples], as acquired, TOPS-modulated) onto the reference grid:
 * deramp (geo2rdr.cu:138-158), interpolate at (row + az_off, col + rg_off)
 * with an 8-tap windowed sinc (S1B_INTERP_SINC8: weights sinc(k-f) *
 * (0.5 + 0.5 cos(pi (k-f)/4)), k = -3..4, normalised) or bilinear, reramp with
 * the secondary's TOPS phase at the fractional position.  Pixels whose kernel
 * support leaves the burst are 0.  out: complex64 [lines * samples];
 * status: int32 device word, set to 1 if a tile's shared-memory staging did
 * not complete (not expected).  When the rasters allow tensor maps (16-byte
 * aligned bases, samples % 4 == 0, plan->samples even) tiles are staged by
 * TMA in a persistent kernel; otherwise by plain loads. */
int s1b_resample(const s1b_burst_plan_t *plan, const void *sec, const float *az_off,
                 const float *rg_off, int32_t lines, int32_t samples, int32_t interp, void *out,
                 int32_t *status, void *stream);

/* Polls each shared-memory staging wait of the TMA resampler makes before it
 * gives up, for later s1b_resample calls of the process (default 2^22).  A
 * wait that gives up sets the call's status word to 1, waits (with the
 * default limit) for the block's copies in flight and ends the block.  A
 * test hook for that error path: with 0 every wait gives up at once.  No
 * reference counterpart.  Returns the previous limit (pass it back to
 * restore). */
uint32_t s1b_set_staging_poll_limit(uint32_t polls);

/* Coherence |sum conj(ref) sec| / sqrt(sum |ref|^2 sum |sec|^2) over win x win
 * boxes at full resolution (win odd, <= 9; windows clipped at the raster
 * border), sums compensated in float32.  ref/sec: complex64 [lines *
 * samples]; coh: float32 [lines * samples]; status: int32 device word, set
 * to 1 if a tile's shared-memory staging did not complete (not expected). */
int s1b_box_coherence(const void *ref, const void *sec, int32_t lines, int32_t samples, int32_t win,
                      float *coh, int32_t *status, void *stream);

/* ------------------------------------------------------------ Goldstein */

/* Scratch bytes s1b_goldstein needs for an nrow x ncol image. */
size_t s1b_goldstein_scratch_bytes(int32_t nrow, int32_t ncol, int32_t n_win);

/* Goldstein filter of a complex64 image: n_win x n_win patches at step
 * n_win/4, FFT, 7x7 circular smoothing of |F|, patch-mean normalisation,
 * ^alpha weighting, inverse FFT, triangular-weight overlap-add.  Replaces
 * goldstein_filter_cuda_host and its kernels, csrc/src/goldstein.cu:87-408.
 * n_win must be 32 (the value s1proc uses) and nrow, ncol >= n_win.
 * in/out: complex64 [nrow * ncol] device (must not alias);
 * scratch: device buffer of s1b_goldstein_scratch_bytes(). */
int s1b_goldstein(const void *in, void *out, int32_t nrow, int32_t ncol, int32_t n_win,
                  float alpha, void *scratch, size_t scratch_bytes, void *stream);

/* Largest image of s1b_goldstein_noalloc, in 32x32 patches (32 MiB of
 * scratch; ceil(nrow/8)-3 times ceil(ncol/8)-3 patches, about 512 x 512 px). */
#define S1B_GOLDSTEIN_NOALLOC_MAX_PATCHES 4096

/* The Goldstein filter of s1b_goldstein for callers that cannot allocate
 * device memory while they filter -- for example a plugin inside a host
 * application whose own pool allocator already holds the GPU's memory, or a
 * pipeline that forbids allocation after start-up.  It allocates nothing:
 * its patch scratch is a fixed device array compiled into this library,
 * which every GPU that loads the library keeps (32 MiB) until the process
 * exits.  No counterpart in the reference.
 *   - Images needing more than S1B_GOLDSTEIN_NOALLOC_MAX_PATCHES patches
 *     return S1B_ERR_TOO_LARGE (use s1b_goldstein then).
 *   - The array's device address belongs to a CUDA context: the first call
 *     in each context (the device's primary context, or a context the host
 *     application made current) looks it up with cudaGetSymbolAddress and
 *     caches it under that context; make that first call before any stream
 *     capture.
 *   - All calls share the one array: calls that can run at the same time on
 *     the GPU (different streams, or threads without ordering) race and
 *     corrupt each other's results; serialise them.
 *   - in/out: complex64 [nrow * ncol] device, n_win must be 32.  in and out
 *     may be the same buffer: every read of `in` (the patch kernel) is
 *     ordered on the stream before the first write of `out` (the gather). */
int s1b_goldstein_noalloc(const void *in, void *out, int32_t nrow, int32_t ncol, int32_t n_win,
                          float alpha, void *stream);

/* ------------------------------------------------ amplitude / coherence files */

/* Amplitude looks of one cropped geocoded SLC (complex64 [height x width],
 * top-left pixel (left, top) of an nrow0 x ncol0 frame) into the full-frame
 * float32 amplitude grid amp [nrow0/rowlook x ncol0/collook]: the
 * look-aligned part of the crop, sqrt(mean |s|^2) (sqrt|s| for 1 x 1 looks,
 * as s1proc's powlooks), written everywhere when `first`, else only where
 * amp is 0 and the new value is not (s1proc/coherence.py:14-55). */
int s1b_amp_looks(const void *slc, int32_t width, int32_t height, int32_t left, int32_t top, int32_t nrow0,
                  int32_t ncol0, int32_t rowlook, int32_t collook, int32_t first, float *amp, void *stream);

/* .cc raster of an interferogram: rows [amp1*amp2 | coherence], coherence =
 * |ifg| / (amp1 + 1e-12) / (amp2 + 1e-12) with values above 1 replaced by a
 * uniform [0,1) value of (fill_seed, pixel index) (s1proc/coherence.py:136-147).
 * ifg complex64, amp1/amp2 float32 [nrow x ncol]; cc float32 [nrow x 2 ncol]. */
int s1b_coherence_cc(const void *ifg, const float *amp1, const float *amp2, int32_t nrow, int32_t ncol,
                     uint64_t fill_seed, float *cc, void *stream);

/* ECEF -> geodetic (deg, deg, m), one-step Bowring (s1proc/geometry.py:166-193). */
int s1b_xyz2llh(const double *xyz, double *llh, int64_t n, void *stream);

/* Line-of-sight unit vectors and look angles of every pixel of an RSC grid,
 * replacing s1proc/utils.py:240-292 (_los, via orbitrangetime_vec,
 * s1proc/orbit.py:168-188).  Pixel (row, col) is at latitude lat0 + row *
 * lat_step and longitude lon0 + col * lon_step (degrees; a separate multiply
 * and add, as numpy.mgrid forms rsc.grid()) and height dem[row * dem_pitch +
 * col] (int16, metres).  Its zero-Doppler time is solved by Newton from t0
 * (the middle state vector's time); los: float32 [nrow * ncol * 3], the unit
 * vector satellite -> point; theta: float32 [nrow * ncol], the look angle
 * acos(clip(los . -(cos lat cos lon, cos lat sin lon, sin lat), -1, 1)) in
 * degrees, formed from the float32 vector as the reference does.  Device
 * pointers; ncol <= 65535 * 128. */
int s1b_los_grid(const s1b_orbit_poly_t *orbit, double t0, double lat0, double lat_step, double lon0,
                 double lon_step, const int16_t *dem, int64_t dem_pitch, int32_t nrow, int32_t ncol, float *los,
                 float *theta, void *stream);

/* ------------------------------------------------------------ burst stitching */

/* One burst interferogram of a frame: `offset` = first element in the data
 * buffer (bursts back to back, row-major [bottom - top x right - left]);
 * left/top/right/bottom in frame pixels; subswath 1..3; `group` identifies
 * the pair of burst ids (the overlap phase offset is estimated when it
 * changes from the previous burst, s1proc/interfere.py:92-118). */
typedef struct {
  int64_t offset;
  int32_t left, top, right, bottom;
  int32_t subswath, group;
} s1b_stitch_burst_t;

/* Device workspace of s1b_stitch (subswath mosaics and tables). */
size_t s1b_stitch_workspace_bytes(const s1b_stitch_burst_t *bursts, int32_t n, int32_t out_float);

/* Stitch burst interferograms (complex64, or float32 phase with out_float)
 * into the frame [nrow0 x ncol0] (s1proc/interfere.py:81-180): per subswath,
 * bursts in order of top + bottom, overlap phase offset angle(mean(conj(old)
 * new)) plus the median residual angle, removed from the new burst, which
 * fills the mosaic where it is empty; subswaths 1..3 written in order where
 * non-zero.  bursts: host array; offsets_host (optional, double [n]): the
 * offset applied to each burst (synchronises the stream when given).  The
 * union box of a subswath is that of its first and last burst, as the
 * reference computes it; parts of middle bursts outside it are dropped. */
int s1b_stitch(const s1b_stitch_burst_t *bursts, int32_t n, const void *data, int32_t out_float, int32_t nrow0,
               int32_t ncol0, void *frame, double *offsets_host, void *workspace, size_t workspace_bytes,
               void *stream);

/* ------------------------------------------------------------ batched frame
 * All burst pairs of a frame (e.g. 3 subswaths x 9 bursts of uneven size)
 * processed with one launch per stage over a per-burst descriptor table.  By
 * default the deramp runs inside the geocoding's gathers and the geocoding
 * of both bursts of each pair forms the crossmul's look-row sums (one CTA
 * per tile of a pair's DEM windows); otherwise deramp and geocoding run one
 * CTA per tile over (tile x, tile y, burst) grids, or as persistent kernels
 * over the flat tile space of every burst (the autotuner picks).  The
 * crossmul box of each pair is formed on the device from the crop rows, so a
 * run has no host synchronisation and can be captured in a CUDA graph.  Replaces running geo2rdr per burst, crossmul_daemon and
 * goldstein per pair (csrc/src/geo2rdr.cu:316-651, crossmul_daemon.cu:566-975,
 * goldstein.cu:328-408); the per-pair results are those of s1b_deramp,
 * s1b_geo2rdr, s1b_crossmul_box, s1b_crossmul_looks and s1b_goldstein. */

typedef struct s1b_frame s1b_frame_t;

/* Per-pair result of a frame run, written on the device. */
typedef struct {
  int32_t ok;           /* 1: products valid; 0: a burst geocoded empty or the overlap is empty */
  int32_t nrow_ml, ncol_ml;
  int32_t filtered;     /* 1: Goldstein ran; 0: image smaller than n_win, filt = ifg */
  int32_t header[6];    /* interferogram header words (crossmul_daemon.cu:660-666) */
  int32_t box[4];       /* full-resolution box: left, top, right, bottom (DEM grid) */
  int32_t gslc_rows[4]; /* crop rows of ref and sec: first, last (exclusive), window rows */
} s1b_frame_pair_t;

typedef struct {
  size_t workspace_bytes;   /* device scratch: deramped bursts (or column tables), geocoded windows,
                               crossmul look-row sums, Goldstein patches */
  int64_t slc_elems;        /* samples of the SLC buffer: bursts back to back */
  int64_t product_elems;    /* elements of each product array (all pairs' slots) */
  int32_t max_nrow_ml, max_ncol_ml;
} s1b_frame_sizes_t;

/* Host only (uploads the descriptor tables; allocates them on the current
 * device).  plans: n_bursts burst plans on one DEM grid (s1b_burst_plan with
 * the same RSC); pair_ref/pair_sec: burst indices of each pair; n_win must
 * be 32.  Bursts whose DEM window is empty return S1B_ERR_EMPTY. */
int s1b_frame_create(const s1b_burst_plan_t *plans, int32_t n_bursts, const int32_t *pair_ref,
                     const int32_t *pair_sec, int32_t n_pairs, int32_t rowlook, int32_t collook,
                     int32_t n_win, float alpha, uint64_t fill_seed, s1b_frame_t **frame);
void s1b_frame_destroy(s1b_frame_t *frame);
int s1b_frame_sizes(const s1b_frame_t *frame, s1b_frame_sizes_t *sizes);
/* Element offset of burst b in the SLC buffer (lines * samples of the bursts before it). */
int s1b_frame_burst_offset(const s1b_frame_t *frame, int32_t burst, int64_t *slc_off);
/* Sample type of the SLC buffer later runs read: S1B_SAMPLES_C64 (the
 * default; 8 bytes per element) or S1B_SAMPLES_CI16 (4 bytes per element,
 * widened in the deramp stage).  Offsets and slc_elems count samples either
 * way.  Products are identical for the same integer-valued samples. */
int s1b_frame_set_sample_format(s1b_frame_t *frame, int32_t format);
/* Deramp stage of later runs (no reference counterpart; the reference
 * deramps a burst in its own kernel, csrc/src/geo2rdr.cu:138-158):
 * 1 (the default): the geocoding deramps the four samples of each bilinear
 * gather where it reads them, from the burst's raw samples and a per-column
 * table of (-kt, etaref) (no deramped copy of any burst is written; one
 * phasor per gathered line carries its deramp and the pixel's reramp); 0: a
 * deramp kernel writes every burst's deramped copy and the geocoding reads
 * it.  The products agree to float rounding (below 1e-6 rad of phase). */
int s1b_frame_set_deramp_fusion(s1b_frame_t *frame, int32_t fused);
/* Crossmul stage of later runs (no reference counterpart; the reference's
 * crossmul_daemon reads the geocoded .gslc files, crossmul_daemon.cu:520-528,
 * 921-975): 1 (the default when rowlook <= 128): the geocoding kernel
 * geocodes both bursts of a pair at each DEM pixel and sums conj(ref) sec and
 * both powers over each column's look rows; a second kernel adds the look
 * columns of the overlap box.  No geocoded window is written.  0: the
 * geocoding writes every burst's window and the crossmul kernel reads them.
 * The products agree to float rounding (the sums are formed in the same
 * order; the geocoding tiles differ).  S1B_ERR_UNSUPPORTED for rowlook > 128. */
int s1b_frame_set_crossmul_fusion(s1b_frame_t *frame, int32_t fused);
/* Slot of pair k in the product arrays: first element and capacity. */
int s1b_frame_pair_slot(const s1b_frame_t *frame, int32_t pair, int64_t *ml_off, int32_t *max_nrow_ml,
                        int32_t *max_ncol_ml);

/* Enqueue one frame run on `stream` (no host synchronisation).
 * slc: [slc_elems] samples of the frame's sample format (complex64 unless
 * set otherwise) device; dem: int16 RSC grid, row pitch in
 * elements; workspace: workspace_bytes, 16-byte aligned; ifg/filt complex64
 * and amp1/amp2/coh float32 [product_elems] (amp1/amp2/coh may be NULL);
 * pairs: s1b_frame_pair_t [n_pairs] device.  Pair k's products are row-major
 * [nrow_ml x ncol_ml] at its slot. */
int s1b_frame_run(s1b_frame_t *frame, const void *slc, const int16_t *dem, int64_t dem_pitch,
                  void *workspace, void *ifg, float *amp1, float *amp2, float *coh, void *filt,
                  s1b_frame_pair_t *pairs, void *stream);

/* Autotuner: times the candidate tile shapes and grids (one CTA per tile, or
 * persistent grids of 1..n CTAs per SM) of
 * the deramp and geocoding stages on these buffers (`reps` runs each, CUDA
 * events on `stream`), keeps the fastest in the frame for later runs and
 * synchronises the stream.  Not capturable.  Every candidate produces the
 * same results.  Stages with a single form are not timed: the deramp fused
 * into the gathers, the geocoding with the crossmul sums. */
int s1b_frame_autotune(s1b_frame_t *frame, const void *slc, const int16_t *dem, int64_t dem_pitch,
                       void *workspace, void *ifg, float *amp1, float *amp2, float *coh, void *filt,
                       s1b_frame_pair_t *pairs, int32_t reps, void *stream);

/* One run with CUDA events between its stages (synchronises the stream):
 * stage_ms[5] = deramp (or the column tables), geocoding (with the crossmul
 * look-row sums when fused), box, crossmul (the look columns when fused),
 * Goldstein (patches and overlap-add), in milliseconds.  For measurement; not
 * capturable. */
int s1b_frame_profile(s1b_frame_t *frame, const void *slc, const int16_t *dem, int64_t dem_pitch,
                      void *workspace, void *ifg, float *amp1, float *amp2, float *coh, void *filt,
                      s1b_frame_pair_t *pairs, float *stage_ms, void *stream);

/* Current tuning: [deramp rows per tile, deramp CTAs, geocoding columns per
 * tile, geocoding CTAs] (CTAs 0 = one CTA per tile, else a persistent grid). */
int s1b_frame_tuning(const s1b_frame_t *frame, int32_t tuning[4]);
/* Set the tuning by hand (validated; S1B_ERR_UNSUPPORTED for a shape not built). */
int s1b_frame_set_tuning(s1b_frame_t *frame, const int32_t tuning[4]);

/* ------------------------------------------- coregistration refinement
 * Coherence objective of radar-grid coregistration and its hand-written
 * adjoint (no reference counterpart).  For n_bursts reference/secondary
 * bursts of one size [lines x samples] (stacked back to back):
 *   az = row + az0 + p0 + p1 xa + p2 xr + daz_dh dh,
 *   rg = col + rg0 + p3 + p4 xa + p5 xr + drg_dh dh,
 *   xa = (row - lines/2) / lines, xr = (col - samples/2) / samples;
 * the secondary is resampled there (8-tap windowed sinc with TOPS deramp /
 * reramp, as s1b_resample) and crossed with the reference; over the rowlook x
 * collook windows of the multilook grid gamma = |sum conj(r) s| /
 * sqrt(sum |r|^2 sum |s|^2); the objective is J = -mean gamma over every
 * window of every burst.  params: float32 [n_bursts x 6] (p0..p5, samples);
 * dh: float32 height error [n_bursts x lines x samples] (metres);
 * daz_dh/drg_dh from s1b_geo2rdr_offsets_dh. */

typedef struct s1b_adjoint s1b_adjoint_t;

/* Host only.  sec_plans: the secondary burst plans (one size); rowlook must
 * divide 16, collook <= 64. */
int s1b_adjoint_create(const s1b_burst_plan_t *sec_plans, int32_t n_bursts, int32_t lines, int32_t samples,
                       int32_t rowlook, int32_t collook, s1b_adjoint_t **adjoint);
void s1b_adjoint_destroy(s1b_adjoint_t *adjoint);
/* Device workspace bytes of s1b_adjoint_run (per-tile partial sums). */
size_t s1b_adjoint_workspace_bytes(const s1b_adjoint_t *adjoint);

/* J into objective (double, device).  With grad_params (float32 [n_bursts x
 * 6]) and grad_dh (float32 like dh) also dJ/dparams and dJ/ddh, from one
 * fused pass that recomputes the window sums.  Deterministic (fixed
 * reduction order).  No host synchronisation. */
int s1b_adjoint_run(s1b_adjoint_t *adjoint, const void *ref, const void *sec, const float *az0,
                    const float *rg0, const float *daz_dh, const float *drg_dh, const float *params,
                    const float *dh, double *objective, float *grad_params, float *grad_dh, void *workspace,
                    size_t workspace_bytes, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* S1B_H */
