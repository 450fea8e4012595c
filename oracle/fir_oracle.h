/* Test infrastructure only: CPU oracle for the FIR projection and
 * reconstruction path.  A plain-C restatement of FIR's algorithms (double
 * geometry, float data, no FMA contraction, serial loops in FIR's own order),
 * used by tests/ and by the CPU-baseline leg of bench.py to check the CUDA
 * path.  The product (fir_b200/) never links or loads it.
 *
 * Parity is pinned in tests/test_oracle_pins.py against the known-answer
 * cases of FIR's unit tests (src_test/SiddonUnitTest.cc,
 * src_test/ProjHeaderUnitTest.cc) and against the compiled FIR sources
 * (oracle/_ref/libfirref.so) on identical inputs.
 */
#ifndef FIR_ORACLE_H
#define FIR_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define FO_MAX_SEGMENTS 1024

typedef struct
{
  int nx, ny, nz;
  double vx, vy, vz; /* voxel extents in mm */
  double ox, oy, oz; /* x,y: centre of first voxel; z: offset of volume centre */
} fo_vol;

typedef struct
{
  /* header (ProjHeader.h:15-40) */
  int n_rings, n_crystals_per_ring, segment_span, n_segments, n_tang_coords;
  /* derived (ProjHeader.h:42-80) */
  long long n_bins;
  int seg_offset, tang_offset, n_views, half_span, max_ring_diff;
  int n_axial[FO_MAX_SEGMENTS];
} fo_proj;

typedef struct
{
  /* ScannerHeader.h:7-46; zero means "use the default / minimum" */
  double crystal_dims[3];
  int crystal_repeat[2];
  double inter_crystal[2];
  double module_dims[3];
  int module_repeat[2];
  double inter_module[2];
  double rsector_dims[3];
  int rsector_repeat;
  double rsector_inner_radius;
} fo_scanner_params;

typedef struct
{
  int nx, ny, nz;
  double ext[3];  /* step sizes used by the traversal */
  double low[3];  /* volume border planes */
  double high[3];
} fo_grid;

/* Returns 0 or a negative error code; fills the derived fields. */
int fo_proj_fill(fo_proj* p);
/* Number of crystals per ring / rings implied by the scanner params after
 * defaults; returns 0 or a negative error code. */
int fo_scanner_check(fo_scanner_params* s, int* n_rings, int* n_crystals_per_ring);
/* xy: 2*n_crystals_per_ring doubles; z: 2*n_rings-1 doubles */
int fo_scanner_tables(const fo_scanner_params* s, double* xy, double* z);

void fo_crystal_axial(const fo_proj* p, int seg, int axial, int* a1, int* a2);
void fo_crystal_ang(const fo_proj* p, int view, int tang, int* c1, int* c2);

/* truncate != 0 reproduces FIR's integer voxel extents (Siddon.h:113). */
void fo_grid_init(fo_grid* g, const fo_vol* v, int truncate);
/* Returns 1 if the segment crosses the volume.  Writes at most cap elements,
 * *count = number of elements of the path. */
int fo_siddon(const fo_grid* g, double x1, double y1, double z1, double x2,
              double y2, double z2, int* coords, double* lengths, int cap,
              int* count);

/* Flat sinogram layout: segments -so..+so concatenated, each [view][axial][tang]. */
void fo_forward(const fo_vol* v, int truncate, const float* img, const fo_proj* p,
                const double* xy, const double* z, float* sino);
/* out: n_subsets frames of nx*ny*nz; sino may be NULL for the all-ones
 * sinogram of computeSensitivityVol. */
void fo_backward(const fo_proj* p, const float* sino, const fo_vol* v, int truncate,
                 const double* xy, const double* z, int n_subsets, float* out);

typedef struct
{
  int n_iterations, n_subsets, convolution_interval;
  float cut_radius;
  float fwhm[3];
} fo_osem_params;

/* One full reconstructAlgos::OSEM run; img holds the initial estimate.
 * sens: n_subsets frames.  bias may be NULL. */
void fo_osem(const fo_proj* p, const float* sino, const float* bias, const fo_vol* v,
             int truncate, const double* xy, const double* z, float* img,
             const float* sens, const fo_osem_params* prm);

/* Resolution-modelling OSEM with the Gaussian PSF inside the system model
 * (the corrected OSEM_ResoReco, reconAlgos.cc:203-367); with any FWHM <= 0
 * it is fo_osem. */
void fo_osem_psf(const fo_proj* p, const float* sino, const float* bias, const fo_vol* v,
                 int truncate, const double* xy, const double* z, float* img,
                 const float* sens, const fo_osem_params* prm);

/* reconAlgos::OSEM_ResoReco exactly as FIR runs it (reconAlgos.cc:203-367):
 * every frame of sens (n_sens_frames >= n_subsets) filtered in place once,
 * the unfiltered image projected, img /= sens[subset], img *= the filtered
 * backprojection. */
void fo_osem_reso_reco(const fo_proj* p, const float* sino, const float* bias, const fo_vol* v,
                       int truncate, const double* xy, const double* z, float* img, float* sens,
                       int n_sens_frames, const fo_osem_params* prm);

void fo_em_update(long long n, float* img, float* bp, const float* sens);

/* Precision study of the traversal (not FIR code): FIR's double traversal
 * against a float loop after FIR's double set-up (precision 1) or a float
 * set-up and loop (precision 2), over n bins of sinogram p.  out[5]: LORs
 * crossing, LORs with a different voxel list, largest relative length
 * difference on equal lists, largest and RMS relative difference of the
 * line integral of img. */
void fo_precision_study(const fo_proj* p, const double* xy, const double* z, const fo_vol* v, int truncate,
                        const float* img, const long long* bins, long long n, int precision, double* out);

/* OSEM with per-bin multiplicative factors m (ordinary-Poisson model):
 * estimate m * (A x) + bias; the backprojected value is m * y / estimate. */
void fo_osem_weighted(const fo_proj* p, const float* sino, const float* mult, const float* bias,
                      const fo_vol* v, int truncate, const double* xy, const double* z, float* img,
                      const float* sens, const fo_osem_params* prm);

/* ProjData::getBinCoordinates: 1 and the bin of the crystal pair, or 0. */
int fo_bin_coordinates(const fo_proj* p, int r1, int c1, int r2, int c2, int* seg, int* view, int* axial,
                       int* tang);
/* ProjData::rebinWeight on a flat sinogram (no-op for span 1). */
void fo_rebin_weight(const fo_proj* p, float* sino);
void fo_convolve(const fo_vol* v, float* img, const float* fwhm, float cut_radius);
void fo_cut_circle(const fo_vol* v, float* img, float cut_radius);
void fo_apply_mask(long long n, float* img, const float* mask);
void fo_hu_to_mu(long long n, float* img);
void fo_exponential(long long n, float* sino);
void fo_proj_multiply(long long n, float* a, const float* b);

#ifdef __cplusplus
}
#endif
#endif
