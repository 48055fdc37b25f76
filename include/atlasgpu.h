/*
 * atlasgpu.h -- C ABI of the B200 (sm_100a) hot path of ATLAS12 / SYNTHE.
 *
 * The reference (cconroy20/atlas12, Fortran 90) keeps these loops inside its
 * drivers; this library replaces them.  Each entry point names the reference
 * code it stands in for (file:line inside the reference tree).  The Fortran
 * side binds them with BIND(C) interfaces; Python binds
 * them with ctypes (atlas12_b200/_lib.py).
 *
 * Conventions
 *   - Every call returns 0 or a negative ATLASGPU_E* status; it never aborts.
 *     atlasgpu_last_error() describes the last failure on a context.
 *   - Arrays are the reference's column-major arrays seen from C: a Fortran
 *     A(n1, n2) is a C array [n2][n1].  Indices stored in arrays (nbuff,
 *     nelion, NU) keep the reference's 1-based meaning.
 *   - Host pointers are read or written only during the call.  Entry points
 *     whose name ends in _dev take device pointers instead and do no host
 *     transfer; they run on the context's stream and return without waiting.
 *   - One context per host thread; calls on one context serialise on its
 *     stream.  No global mutable state.
 */
#ifndef ATLASGPU_H
#define ATLASGPU_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ATLASGPU_OK 0
#define ATLASGPU_EINVAL -1     /* bad shape, index or argument */
#define ATLASGPU_ENOMEM -2     /* device allocation failed */
#define ATLASGPU_ECUDA -3      /* CUDA runtime error */
#define ATLASGPU_ETIMEOUT -4   /* a bounded device wait gave up */
#define ATLASGPU_ENONFINITE -5 /* non-finite value in an input table */
#define ATLASGPU_ESTATE -6     /* call order (e.g. operators not set) */

#define ATLASGPU_PREC_FP64 0  /* every quantity in FP64 (the plain FP64 GPU path) */
#define ATLASGPU_PREC_MIXED 1 /* FP32 Voigt/profile terms, FP64 sums and decisions, FP64 transfer */

#define ATLASGPU_NXTAU 51

typedef struct atlasgpu_ctx atlasgpu_ctx;

typedef struct {
  int device;    /* CUDA ordinal */
  int precision; /* ATLASGPU_PREC_* */
  void *stream;  /* cudaStream_t to run on, or NULL for a private stream */
} atlasgpu_opts;

/* BIND(C) twin of SYNTHE's lte_line_t (mod_mklinelist.f90:30-41), 32 bytes. */
typedef struct {
  int32_t nbuff;  /* grid index, 1-based, offset from ixwlbeg */
  float cgf;      /* line-strength factor */
  int32_t nelion; /* species index (nelem-1)*6 + ion stage, 1-based */
  float elo;      /* lower level energy, cm^-1 */
  float gamrf, gamsf, gamwf; /* damping / (4 pi nu) */
  float code;     /* species code (carried, unused by the kernels) */
} atlasgpu_lte_line;

/* SYNTHE log-lambda grid, synthe.f90:316-324 */
typedef struct {
  double ratio, ratiolg, wbegin;
  int32_t length, ixwlbeg;
} atlasgpu_grid;

/* Frequency-integral accumulators of TCORR/RADIAP/ROSS mode 2, each [nrhox]
 * (atlas12_modules.f90:2457-2522, 5072-5097, 5178-5190). */
typedef struct {
  double *rjmins, *rdabh, *rdiagj, *flxrad;
  double *raden, *h_total, *accrad, *abross;
  double pradk0;
} atlasgpu_accum;

/* ---- context ------------------------------------------------------- */
/* Number of visible CUDA devices (0 when none); never fails. */
int atlasgpu_device_count(void);
int atlasgpu_create(atlasgpu_ctx **out, const atlasgpu_opts *opts);
int atlasgpu_destroy(atlasgpu_ctx *ctx);
const char *atlasgpu_last_error(atlasgpu_ctx *ctx);
int atlasgpu_set_precision(atlasgpu_ctx *ctx, int precision);
int atlasgpu_set_stream(atlasgpu_ctx *ctx, void *stream);
int atlasgpu_synchronize(atlasgpu_ctx *ctx);
/* Kernel launches issued by this context since creation (all entry points). */
int64_t atlasgpu_launch_count(atlasgpu_ctx *ctx);
/* Device time (ms, CUDA events on the context stream) of the last launch of
 * the named kernel family ("synthe_core", "synthe_farwing", "josh_spectrum",
 * "atlas_linop", "atlas_rt", ...), or -1 if never timed.  Timing is recorded
 * only while enabled. */
int atlasgpu_enable_timing(atlasgpu_ctx *ctx, int on);
double atlasgpu_kernel_ms(atlasgpu_ctx *ctx, const char *name);

/* JOSH operator set: BLOCKJ/BLOCKH matrices (atlas12_modules.f90:18792-18860)
 * plus JOSH's fixed 51-point tau grid XTAU8 and surface weights CH_J, CK_J
 * (:18409-18451).  coefj/coefh column-major 51x51 (COEF(L,M) at [(M-1)*51+L-1]).
 * Replaces CALL BLOCKJ / CALL BLOCKH (synthe.f90:463-464, atlas12c.f90:242-243). */
int atlasgpu_set_operators(atlasgpu_ctx *ctx, const double *xtau8, const double *coefj,
                           const double *coefh, const double *ch_j, const double *ck_j);

/* ---- SYNTHE ----------------------------------------------------------- */
/* Grid scalars, synthe.f90:316-324 (host arithmetic, no device work). */
int atlasgpu_synthe_grid(double wlbeg, double wlend, double resolu, atlasgpu_grid *out);

/* Line -> bin index, bit-exact with the readers' INT(LOG(wlvac)/ratiolg+0.5)
 * - ixwlbeg + 1 (mod_mklinelist.f90:898-899; same rule :1313, :1472, :2134).
 * Computed on the device; quotients within 1e-8 of a rounding boundary are
 * re-evaluated on the host with the C library log the reference links. */
int atlasgpu_synthe_bin(atlasgpu_ctx *ctx, const double *wlvac, int64_t n, double ratiolg,
                        int32_t ixwlbeg, int32_t *nbuff_out);
int atlasgpu_synthe_bin_dev(atlasgpu_ctx *ctx, const double *d_wlvac, int64_t n, double ratiolg,
                            int32_t ixwlbeg, int32_t *d_nbuff, int64_t *n_flagged);

/* Continuum per depth on the grid: quadratic log10 interpolation across the
 * edges, floor at -15, 10**x (synthe.f90:483-516).  continall [nrhox][ncont_stride]
 * holds (left, mid, right) log10 kappa per edge interval (continall_m).
 * continuum_out [nrhox][length] float. */
int atlasgpu_synthe_continuum(atlasgpu_ctx *ctx, const double *wledge, int nedge,
                              const double *continall, int ncont_stride, int nrhox, double wbegin,
                              double ratio, int length, float *continuum_out);

/* LTE line opacity: the SYNTHE depth loop's line loop (synthe.f90:559-683 with
 * voigt_profile, synthe_module.f90:463-537).  Replaces the per-depth BUFFER
 * accumulation; writes opacity_matrix(length, nrhox) as [nrhox][length].
 *   lines     n records
 *   continuum [nrhox][length] (from atlasgpu_synthe_continuum)
 *   xnfdop, dopple [nrhox][nspec] (nspec = mw6 = 834 in the reference)
 *   xne, txnxn, hckt [nrhox]
 *   maxprof   profile cap (MAXPROF = 1000000, synthe_module.f90:219) */
int atlasgpu_synthe_line_opacity(atlasgpu_ctx *ctx, const atlasgpu_lte_line *lines, int64_t n,
                                 int length, int nrhox, double resolu, const float *continuum,
                                 const double *xnfdop, const double *dopple, int nspec,
                                 const double *xne, const double *txnxn, const double *hckt,
                                 int maxprof, float *opacity_out);
int atlasgpu_synthe_line_opacity_dev(atlasgpu_ctx *ctx, const atlasgpu_lte_line *d_lines, int64_t n,
                                     int length, int nrhox, double resolu, const float *d_continuum,
                                     const double *d_xnfdop, const double *d_dopple, int nspec,
                                     const double *d_xne, const double *d_txnxn,
                                     const double *d_hckt, int maxprof, float *d_opacity);

/* Spectrum: the SYNTHE wavelength loop (synthe.f90:698-718) with
 * setup_opacity_sv and process_wavelength_point (:797-902): per lambda two
 * JOSH(1,1) solves, continuum-only and continuum+line.  contabs/contscat
 * [nrhox][ncont_stride] log10 tables; opacity [nrhox][length].  flux/cont [length]. */
int atlasgpu_synthe_spectrum(atlasgpu_ctx *ctx, const double *wledge, int nedge,
                             const double *contabs, const double *contscat, int ncont_stride,
                             int nrhox, const double *rhox, const double *hkt, double wbegin,
                             double ratio, int length, const float *opacity, double *flux,
                             double *cont);
int atlasgpu_synthe_spectrum_dev(atlasgpu_ctx *ctx, const double *d_wledge, int nedge,
                                 const double *d_contabs, const double *d_contscat,
                                 int ncont_stride, int nrhox, const double *d_rhox,
                                 const double *d_hkt, double wbegin, double ratio, int length,
                                 const float *d_opacity, double *d_flux, double *d_cont);

#ifdef __cplusplus
}
#endif
#endif
