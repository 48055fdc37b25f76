/*
 * atlasgpu.h -- C ABI of the B200 (sm_100a) hot path of ATLAS12 / SYNTHE.
 *
 * The reference (cconroy20/atlas12, Fortran 90) keeps these loops inside its
 * drivers; this library replaces them.  Each entry point names the reference
 * code it stands in for (file:line inside the reference tree).  The Fortran
 * side binds them with BIND(C) interfaces; Python binds them with ctypes
 * (atlas12_b200/_lib.py).
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
 *     stream.  All state lives in contexts and the objects made on them,
 *     with one exception: atlasgpu_atlas_rt_pass_noalloc keeps its scratch
 *     in one fixed device array shared by every call in the process (its
 *     declaration says how calls must be serialised).
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

/* BIND(C) twin of the NLTE / complex-profile line record read from unit 19
 * (nlte_line_t, mod_mklinelist.f90:43-63; read at atlas12_modules.f90:19992),
 * padded to 64 bytes.  nbuff carries IWL (the integer log wavelength). */
typedef struct {
  double wlvac;            /* vacuum wavelength, nm */
  float elo, gf;           /* lower level energy (cm^-1), CGF */
  int32_t nblo, nbup;      /* NLTE level indices */
  int32_t nelion, itype;   /* species index; line type (0, 3 normal; 2 skipped) */
  int32_t ncon, nelionx;   /* continuum-edge index into CONTX, its species column */
  float gammar, gammas, gammaw; /* damping / (4 pi nu) */
  int32_t nbuff, lim;      /* IWL; wing extent index */
  int32_t pad;
} atlasgpu_nlte_line;

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
/* Algorithmic work units counted by the last timed launch of a kernel
 * family while timing is enabled, or -1: "synthe_voigt_evals" (SYNTHE core
 * Voigt evaluations), "synthe_farwing_updates" (far-wing bin updates),
 * "atlas_linop_points" (LINOP1 wing points added into XLINES), the batched
 * iteration's "batch_linop_points" and "batch_linop_atomics" (the atomics
 * its exact sums issue, counted by a pass that walks without adding), the batched
 * RT solve stage's "batch_rt_eliminated", "batch_rt_series" (systems solved
 * each way) and "batch_rt_series_steps".  No reference counterpart: these
 * are the numerators of the kernels' rooflines. */
double atlasgpu_kernel_work(atlasgpu_ctx *ctx, const char *name);

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

/* One Stehle MMM Stark-profile series (INIT_STARK_TABLES,
 * atlas12_modules.f90:17682-17746: Lyman, Balmer, Paschen, Brackett); n_dens
 * 0 marks a series that is not loaded.  max_dens_idx [n_trans] (1-based),
 * k_alpha [n_trans], profiles PROFILES(IA, IT, ID, ITRANS) at
 * [ITRANS-1][ID-1][IT-1][IA-1] ([n_trans][n_dens][10][60]), n_trans =
 * n_upper_max - n_upper_min + 1. */
typedef struct atlasgpu_stehle_series {
  int32_t n_lower, n_upper_min, n_upper_max, n_dens;
  double density_grid[20], temp_grid[10], log_dalpha_grid[60];
  const int32_t *max_dens_idx;
  const double *k_alpha;
  const double *profiles;
} atlasgpu_stehle_series;

/* the depth vectors SYNTHE's hydrogen lines read: T, XNFPH(J,1), XNFPH(J,2),
 * XNFHE(J,1), XNFH2(J) [nrhox] */
typedef struct atlasgpu_synthe_hydrogen {
  const double *t, *xnfph1, *xnfph2, *xnfhe1, *xnfh2;
} atlasgpu_synthe_hydrogen;

struct atlasgpu_hydrogen_tables; /* defined with XLINOP's entry points below */

/* Keeps SYNTHE's hydrogen_line_profile tables (its own values, in the layout
 * of atlasgpu_hydrogen_tables; eh = EHYD(1..10), elim = ELIM_HI) and the four
 * Stehle series (NULL: none loaded, the analytic profile throughout) on the
 * context, for atlasgpu_synthe_nlte_opacity. */
int atlasgpu_synthe_set_hydrogen_tables(atlasgpu_ctx *ctx, const struct atlasgpu_hydrogen_tables *tables,
                                        const atlasgpu_stehle_series *stehle);

/* The NLTE / complex-profile list's normal-metal lines (TYPE 0, 3 and the He I
 * fallthrough TYPE <= -3) of compute_line_opacity (synthe_module.f90:3167-3458,
 * called per depth at synthe.f90:554): wings walked from the record's grid
 * index nbuff, red wing tested before the add, blue wing after it, stop at
 * continuum(i)*LINE_CUTOFF; blue of the continuum edge WCON = 1e7 /
 * (CONTX(NCON,NELIONX) - EMERGE(J)) nothing is added, WCON..WTAIL (500 cm^-1
 * redder) tapers linearly; lambdas shifted by (1 + velshift/c).  FP64 sums,
 * added into opacity_inout [nrhox][length] (the LTE opacity matrix).
 *   recs [n] (nbuff = grid index); continuum [nrhox][length];
 *   xnfdop, dopple [nrhox][nspec]; xne, txnxn, hckt [nrhox];
 *   contx [17][26]: CONTX(26,17) column-major.
 * With xnfpel [nrhox][nspec] (XNFPEL = populations / RHO, synthe.f90:533-542)
 * also the autoionizing (Shore) lines, TYPE 1 (:3609-3650): the Fano profile
 * with GAMMAS, GAMMAW as the Shore parameters, each wing point added and then
 * tested; and the merged-continuum edges, TYPE = NLAST >= 4 (:3652-3696, vacuum
 * wavelengths): flat from the line to WMERGE, tapering to zero at WTAIL, the
 * grid indices computed on the host with the C library.  xnfpel NULL skips
 * both.  With h (and the tables of atlasgpu_synthe_set_hydrogen_tables) also
 * the hydrogen and deuterium lines, TYPE -1/-2 (:3460-3606): KAPPA0 = GF *
 * XNFDOP(J,1) * exp(-ELO*HCKT) gated by the continuum, wings of
 * hydrogen_line_profile(NBLO, NBUP, J, WAVE - WL) (:1032-1980: the Stehle
 * tables convolved with a Voigt kernel where a loaded series covers the line
 * and XNE, else the Peterson/Kurucz analytic profile) for the alpha/isolated
 * lines (NCON 0 or NBUP = NBLO+1), the beta lines (red wing stopping at
 * ALPHAHYD(NBLO)) and the higher members (tapered between WCON and WTAIL of
 * the series limit CONTH(NCON), vacuum wavelengths).  NBLO 1..99, NBUP
 * NBLO+1..100 and NCON 0..15 (the reference aborts or reads outside EHYD,
 * ALPHAHYD and CONTH otherwise).  h NULL skips them. */
int atlasgpu_synthe_nlte_opacity(atlasgpu_ctx *ctx, const atlasgpu_nlte_line *recs, int64_t n, int length,
                                 int nrhox, double wbegin, double ratio, double wlend, double velshift_kms,
                                 const float *continuum, const double *xnfdop, const double *dopple,
                                 const double *xnfpel, int nspec, const double *xne, const double *txnxn,
                                 const double *hckt, const double *contx, const atlasgpu_synthe_hydrogen *h,
                                 float *opacity_inout);

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


/* ---- ATLAS12 ---------------------------------------------------------- */
/* TABVOIGT (atlas12_modules.f90:19796-19851) on the host: H0 = exp(-v^2),
 * H1 = MAP1 of the tabulated H1 (tabvi, tabh1 [ntab], the reference's TABVI
 * and TABH1 data, :19805-19835) onto v = (i-1)/vsteps, H2 = H0 - 2 v^2 H0,
 * each [n].  No device work; needs no context. */
int atlasgpu_atlas_tabvoigt(double vsteps, int n, const double *tabvi, const double *tabh1, int ntab,
                            double *h0, double *h1, double *h2);

/* Voigt tables of TABVOIGT(200, 2001) (atlas12_modules.f90:19796-19851), as
 * the driver computes them at start-up (atlas12c.f90:236).  n = 2001.  Also
 * builds TABLOG (:2083-2086) on the host with the C library pow. */
int atlasgpu_atlas_set_voigt_tables(atlasgpu_ctx *ctx, const double *h0tab, const double *h1tab,
                                    const double *h2tab, int n);

/* LINOP1 (atlas12_modules.f90:18132-18374): line opacity XLINES(J,NU) from
 * the stored LINEDATA records.
 *   linedata [n][4] int32 (LINEREC, :1950-1977)
 *   xnfdop, dopple [nspec][kw] (XNFDOP(J,NELION), DOPPLE(J,NELION))
 *   xne, txnxn, hckt [nrhox]; tabcont [nwave+1][kw]; iwavetab [nwave+1]
 *   waveset [numnu]; xlines_out [numnu][kw]
 * lines_used (may be NULL) receives LINEUSED (lines above TABCONT at some
 * coarse depth).  Lines redward of WAVESET(NUMNU-1) take NU = NUMNU (the
 * reference's walk runs past the grid there). */
int atlasgpu_atlas_linop(atlasgpu_ctx *ctx, const int32_t *linedata, int64_t n, int nrhox, int kw,
                         const double *xnfdop, const double *dopple, int nspec, const double *xne,
                         const double *txnxn, const double *hckt, const double *tabcont,
                         const int32_t *iwavetab, int nwave, const double *waveset, int numnu,
                         double *xlines_out, int64_t *lines_used);

/* The hydrogen line profile's tables: HPROF4's (atlas12_modules.f90:
 * 20553-20700), STARK_PROFILE's (:20376-20450 and data/stark_profile.dat)
 * and XLINOP's level energies EH(1..10) with ELIM_HI (:19964-19975, :385).
 * Two-index tables at [first index - 1][second index - 1]; PROPBM(IP, J, K)
 * at [K-1][J-1][IP-1], C and D (IP, K) at [K-1][IP-1]. */
typedef struct atlasgpu_hydrogen_tables {
  double xknmtb[4][3]; /* XKNMTB(N, M-N) */
  double y1wtm[2][2];  /* Y1WTM(N, M-N) */
  double stalph[34], stwtal[34];
  int32_t istal[4], lnghal[4];
  double stcomp[5][4], stcpwt[5][4]; /* STCOMP(I, N) */
  int32_t lncomp[4];
  double cutoffh2plus[111], cutoffh2[91];
  double asum[100], asumlyman[100];
  double betagrid[15], pp[5];
  double propbm[7][15][5];
  double c[7][5], d[7][5];
  double eh[10], elim;
} atlasgpu_hydrogen_tables;

/* the depth vectors HPROF4 reads besides XNE, XNFP and DOPPLE: T(J),
 * XNF(J,1) (H I), XNF(J,2) (H II), XNH2(J), each [nrhox] */
typedef struct atlasgpu_xlinop_hydrogen {
  const double *t, *xnf1, *xnf2, *xnh2;
} atlasgpu_xlinop_hydrogen;

/* Keeps the hydrogen tables on the context for XLINOP's hydrogen lines. */
int atlasgpu_atlas_set_hydrogen_tables(atlasgpu_ctx *ctx, const atlasgpu_hydrogen_tables *tables);

/* XLINOP (atlas12_modules.f90:19873-20250).  The normal-line branch (TYPE 0 and 3, :20040-20174):
 * the LINOP1 walk on unit-19 records with MAX_WING = 2000, LORENTZ_PREFAC =
 * 0.5642 and the blue-wing cutoff at the continuum edge WCON = 1e7 /
 * (CONTX(NCON,NELIONX) - EMERGE(J)), EMERGE(J) = RYDBERG_INF / NMERGE(J)**2,
 * NMERGE = 1600 / XNE(J)**(2/15) (:19964-19977).  Adds into xlines_inout
 * [numnu][kw] (RUN_RT_PASS calls it after LINOP1, :3893-3894).
 *   recs [n], sorted by wavelength (the reference advances NU and NUCONT
 *   monotonically and stops at the first line with NU >= NUMNU)
 *   contx [16][25]: CONTX(25,16) column-major (XLINOP's edge table)
 * With xnfp [nspec][kw] (XNFP(J,NELION)) and rho [kw] (RHO(J)) also the
 * autoionizing lines (TYPE 1, Fano profile over MAX_WING = 2000 points,
 * :20201-20226) and the merged-continuum records (every other TYPE but -1,
 * NLAST = TYPE, flat up to the dissolution limit, at most 1001 points,
 * :20228-20245); both NULL: those are skipped and counted in n_other.
 * With h (and xnfp, and the tables of atlasgpu_atlas_set_hydrogen_tables)
 * also the hydrogen lines (TYPE -1, :20177-20199): CENTER = GF *
 * exp(-EH(NBLO)*HCKT) * XNFDOP(J,1), wings of HPROF4(NBLO, NBUP, J, WAVESET -
 * WLVAC) over MAX_WING points, the red one skipping and the blue one
 * stopping blueward of WCON = 1e7 / (CONTX(NCON,1) - EMERGE(J)).  TYPE 2
 * records are skipped as in the reference; the types not handled are
 * counted in n_other (may be NULL). */
int atlasgpu_atlas_xlinop(atlasgpu_ctx *ctx, const atlasgpu_nlte_line *recs, int64_t n, int nrhox, int kw,
                          const double *xnfdop, const double *dopple, int nspec, const double *xne,
                          const double *txnxn, const double *hckt, const double *tabcont,
                          const int32_t *iwavetab, int nwave, const double *waveset, int numnu,
                          const double *contx, const double *xnfp, const double *rho,
                          const atlasgpu_xlinop_hydrogen *h, double *xlines_inout, int64_t *n_other);

/* KAPP's hydrogen continuum tables, as the reference reads them from its data
 * files and DATA statements (Fortran arrays column-major):
 *   XKARZAS (atlas12_modules.f90:11635-11804): data/karzas_freqn.dat,
 *     karzas_xn.dat, karzas_xl.dat, karzas_ekarzas.dat (REAL(4));
 *   COULFF (:11995-12196): data/gauntff_vanhoof.dat, the 146 rows of 81
 *     thermally averaged g_ff (the library takes log10 as the reader does);
 *   holtsmark_Q (:425-464): Q_HOLTSMARK;
 *   HOP (:11359-11608): the level energies E_n of n = 1..15 (cm^-1; E_1 = 0);
 *   HMINOP (:12360-12558): WBF, BF, THETAFF, WAVEK, FF (FF holds REAL(4)
 *     literals, so its values are single-precision roundings);
 *   H2PLOP (:12224-12252): the FR and ES fit coefficients, signed, lowest
 *     order first;
 *   HRAYOP (:12740-12906): GAVRILAM, GAVRILAMAB, GAVRILAMBC, GAVRILAMCD,
 *     GAVRILALYMANCONT, FGAVRILALYMANCONT;
 * and the helium ones:
 *   HE1OP (:12939-13143): CHI, HEFREQ, G of its ten resolved levels;
 *   CROSSHE (:13160-13236): X505, X50, X20, X10 (1e-18 cm^2);
 *   HE12S1S, HE12S3S, HE12P1P, HE12P3P (:13299-13545): log10 frequency and
 *     log10 cross-section knots (FREQ1S/X1S, FREQ3S/X3S, FREQ1P/X1P,
 *     FREQ3P/X3P);
 *   HEMIOP (:13716-13833): WHEM (nm), THEM (K), KHEM(17,12) (cm^4/dyn; the
 *     library takes the logs as the reference's first call does);
 * and HLINOP's: hydrogen_f_value's (:17760-17829) GF_LYMAN, GF_BALMER,
 *   GF_PASCHEN, GF_BRACKETT; STARK's (:17528-17659) KNMTAB(5,4), FSTARK(10,4). */
typedef struct atlasgpu_kapp_tables {
  float freqn[15][29], xn[15][29], xl[6][6][29], ekarzas[29];
  double gff[146][81];
  double q_holtsmark[150];
  double hop_elev[15];
  double hmin_wbf[116], hmin_bf[116], hmin_thetaff[11], hmin_wavek[22], hmin_ff[22][11];
  double h2p_fr[5], h2p_es[6];
  double ray_m[74], ray_ab[27], ray_bc[24], ray_cd[22], ray_ly[64], ray_fly[64];
  double he1_chi[10], he1_freq[10], he1_g[10];
  double he_x505[92], he_x50[16], he_x20[11], he_x10[21];
  double he2s1s_f[16], he2s1s_x[16], he2s3s_f[16], he2s3s_x[16];
  double he2p1p_f[16], he2p1p_x[16], he2p3p_f[16], he2p3p_x[16];
  double hem_w[17], hem_t[12], hem_k[12][17];
  double gf_lyman[29], gf_balmer[28], gf_paschen[27], gf_brackett[3];
  double stark_knm[4][5], stark_f[4][10];
} atlasgpu_kapp_tables;

/* Keeps KAPP's hydrogen tables on the context for atlasgpu_atlas_kapp_hydrogen
 * (COULFF's log10 of g_ff and HMINOP's log tables are taken here, once, as the
 * reference's first calls do). */
int atlasgpu_atlas_set_kapp_tables(atlasgpu_ctx *ctx, const atlasgpu_kapp_tables *tables);

/* KAPP (atlas12_modules.f90:11202-11324) with its hydrogen, H-, H2+ and
 * scattering sources, per frequency and depth: HOP (:11359-11608: bound-free
 * from n = 1..15 with Karzas-Latter cross-sections and the occupation
 * probabilities of Hummer & Mihalas, n = 16..80, the dissolved-level
 * pseudo-continuum, free-free with COULFF), H2PLOP, HMINOP (McLaughlin
 * bound-free, Bell & Berrington free-free), HRAYOP (Gavrila), ELECOP; the
 * totals ACONT, SCONT, SIGMAC as KAPP forms them with the helium, metal, H2
 * and line sources zero.  WAVESET (nm) [numnu]; depth vectors [nrhox]: T, XNE,
 * RHO, XNFP(J,1) (H I number density over its partition function), XNFP(J,2)
 * (H II); bhyd BHYD(J,1..6) as [6][kw] and bmin BMIN(J) [kw], or NULL for LTE
 * (1).  Outputs [numnu][kw]; parts, if not NULL, [numnu][7][kw]: AHYD, SHYD,
 * AH2P, AHMIN, SHMIN, SIGH, SIGEL. */
int atlasgpu_atlas_kapp_hydrogen(atlasgpu_ctx *ctx, int numnu, const double *waveset, int nrhox, int kw,
                                 const double *t, const double *xne, const double *rho, const double *xnfp1,
                                 const double *xnfp2, const double *bhyd, const double *bmin, double *acont,
                                 double *sigmac, double *scont, double *parts);

/* Depth vectors [nrhox] for atlasgpu_atlas_kapp: the hydrogen ones as for
 * atlasgpu_atlas_kapp_hydrogen, and the helium populations the helium
 * sources read: XNFP(J,3) (He I over its partition function), XNFP(J,4)
 * (He II), XNFP(J,5) (He III) and XNF(J,4) (the He II number density, which
 * HE1OP's free-free term takes). */
typedef struct atlasgpu_kapp_pops {
  const double *t, *xne, *rho;
  const double *xnfp_h1, *xnfp_h2;
  const double *xnfp_he1, *xnfp_he2, *xnfp_he3, *xnf_he2;
  const double *bhyd, *bmin; /* NULL for LTE, as for atlasgpu_atlas_kapp_hydrogen */
  const double *xnf_he1;     /* XNF(J,3), the He I number density: non-NULL adds the H2 sources */
} atlasgpu_kapp_pops;

/* KAPP's H2 tables, as the reference reads them:
 *   H2MINOP (atlas12_modules.f90:12611-12708): WH2M (nm), TH2M (K),
 *     KH2M(10,7) (cm^4/dyn; the library takes the logs);
 *   PARTFNH2 (:22324-22418): data/partfnh2.dat, Q(H2) at pf_tstart +
 *     (n-1) pf_tstep, n = 1..pf_n (the library forms the cubic spline's
 *     second derivatives as the reader does);
 *   H2COLLOP (:16371-16527): data/h2collop.dat, log10 of the CIA
 *     coefficients of the pairs H2-H2, H2-He, H2-H, H-He on the wavenumber
 *     grid cia_nu0 + (i-1) cia_dnu, i = 1..cia_nnu: cia_temp [4][cia_ntmax]
 *     (cia_nt[p] used), cia_tab [4][cia_ntmax][cia_nnu]; use_pair =
 *     USE_CIA_PAIR. */
typedef struct atlasgpu_kapp_h2_tables {
  double h2m_w[10], h2m_t[7], h2m_k[7][10];
  int32_t pf_n;
  double pf_tstart, pf_tstep;
  const double *pf;
  int32_t cia_nnu, cia_ntmax, cia_nt[4], use_pair[4];
  double cia_nu0, cia_dnu;
  const double *cia_temp, *cia_tab;
} atlasgpu_kapp_h2_tables;

/* Keeps the H2 tables on the context for atlasgpu_atlas_kapp (pops->xnf_he1
 * non-NULL). */
int atlasgpu_atlas_set_kapp_h2_tables(atlasgpu_ctx *ctx, const atlasgpu_kapp_h2_tables *tables);

/* KAPP (atlas12_modules.f90:11202-11324) with the hydrogen sources of
 * atlasgpu_atlas_kapp_hydrogen and the helium ones: HE1OP (:12939-13143: the
 * ten resolved levels with CROSSHE, the 2s/2p fits and XKARZAS for the n = 3
 * levels, the inner-shell thresholds to He II n = 2 and 3, n = 4..27, the
 * dissolved-level term, free-free), HE2OP (:13569-13674), HEMIOP
 * (:13716-13833), HERAOP (:13918-13941); with pops->xnf_he1 also the H2
 * sources H2MINOP (:12611-12708), H2COLLOP (:16371-16527) and H2RAOP
 * (:17289-17338) with EQUILH2 (:22437-22469); ACONT, SCONT and SIGMAC as KAPP
 * forms them with the metal and line sources (and without xnf_he1 the H2
 * ones) zero.  Outputs as for atlasgpu_atlas_kapp_hydrogen; parts, if not
 * NULL, [numnu][11][kw] (or [numnu][14][kw] with H2): AHYD, SHYD, AH2P,
 * AHMIN, SHMIN, SIGH, SIGEL, AHE1, AHE2, AHEMIN, SIGHE (, AH2MIN, AH2COLL,
 * SIGH2). */
int atlasgpu_atlas_kapp(atlasgpu_ctx *ctx, int numnu, const double *waveset, int nrhox, int kw,
                        const atlasgpu_kapp_pops *pops, double *acont, double *sigmac, double *scont,
                        double *parts);

/* Keeps the four Stehle series (Lyman, Balmer, Paschen, Brackett) that
 * STARK_MMM (atlas12_modules.f90:17854-18106) reads on the context for
 * atlasgpu_atlas_hlinop; NULL (or a series with n_dens 0): STARK's analytic
 * profile throughout, as when the reference finds no table file. */
int atlasgpu_atlas_set_stehle_tables(atlasgpu_ctx *ctx, const atlasgpu_stehle_series *stehle);

/* HLINOP (atlas12_modules.f90:17381-17503): the hydrogen line
 * pseudo-continuum of KAPP, per frequency and depth -- the lines of the
 * series whose lower level n = int(sqrt(nu_Lyman / nu)) (n <= 4; Lyman only
 * above 2e15 Hz, Balmer above 4.44e14 Hz) nearest the frequency, their Stark
 * profiles from STARK_MMM (Stehle tables where loaded, else STARK
 * :17528-17659) with the occupation probabilities and departure
 * coefficients.  Depth vectors [nrhox] T, XNE, RHO, XNFP(J,1), each positive
 * but XNFP (STARK divides by XNE); bhyd BHYD(J,1..6) as [6][kw], positive, or
 * NULL (LTE).  Outputs AHLINE, SHLINE
 * [numnu][kw] (frequencies outside the four series: 0 and 0, as KAPP's
 * zeroed arrays; depths past the dissolved-level cut: 0 and BNU).  The
 * tables of atlasgpu_atlas_set_kapp_tables must be set. */
int atlasgpu_atlas_hlinop(atlasgpu_ctx *ctx, int numnu, const double *waveset, int nrhox, int kw, const double *t,
                          const double *xne, const double *rho, const double *xnfp1, const double *bhyd,
                          double *ahline, double *shline);

/* RUN_RT_PASS frequency loop (atlas12_modules.f90:3880-3951): per NU the
 * Planck terms, ALINE = XLINES*STIM, JOSH(1,0) (:18398-18776), the negative
 * floor and the TCORR/RADIAP/ROSS mode-2 sums.  acont/sigmac [numnu][kw]
 * from KAPP, scont [numnu][kw] or NULL for SCONT = BNU; xlines [numnu][kw].
 * out: sums over all frequencies (zeroed by the call, i.e. mode 1 included);
 * hsurf_out [numnu] = HNU(1) per frequency (the .flux record). */
int atlasgpu_atlas_rt_pass(atlasgpu_ctx *ctx, int numnu, const double *waveset, const double *rcoset,
                           const double *acont, const double *sigmac, const double *scont, int kw,
                           const double *xlines, int nrhox, const double *rhox, const double *t,
                           const double *hkt, double teff, atlasgpu_accum *out, double *hsurf_out);

/* Model arrays for the end of an iteration, [nrhox] each, updated in place. */
typedef struct {
  int nrhox, iter;
  double teff, grav, pradk0;
  double *t, *rhox, *p, *xne, *abross, *prad, *vturb, *pturb, *tauros, *accrad, *raden, *oldt1;
  double *flxerr, *dtflux, *dtlamb, *dtsurf, *t1; /* outputs: the .iter columns */
  /* ROSSTAB store (atlas12_modules.f90:5937-6228), in/out: ross_n points of
   * normalised (log T, log P, log10 kappa_R) in ross_t/p/k [ross_max], with
   * the normalisation fixed by the first store (ross_n = 0 on iteration 1) */
  int ross_n, ross_max;
  double ross_zerot, ross_slopet, ross_zerop, ross_slopep;
  double *ross_t, *ross_p, *ross_k;
} atlasgpu_finish_state;

/* ROSS(3), the ROSSTAB store, RADIAP(3) and TCORR(3) (atlas12_modules.f90:
 * 5193-5198, 5937-6228, 5108-5135, 2528-2977) with TTAUP (:6303-6523),
 * radiative branch, on the device.  acc = the mode-2 sums from atlasgpu_atlas_rt_pass.  max_flxerr
 * receives max |FLXERR| in percent (the convergence metric). */
int atlasgpu_atlas_finish(atlasgpu_ctx *ctx, atlasgpu_finish_state *s, const atlasgpu_accum *acc,
                          double *max_flxerr);

/* ---- SELECTLINES: the line databases -> LINEDATA ----------------------
 * SELECTLINES (atlas12_modules.f90:19171-19781) keeps the lines whose
 * centre opacity can reach the continuum cutoff: per record, the NU advance
 * over IWAVETAB (DO WHILE (IWL >= IWAVETAB(NU)), which sets FREQ), then
 * CENRATIO = CEN_PREFAC * TABLOG(IGFLOG) * XNFDOPMAX(NELION, NU) / FREQ >= 1
 * and CENRATIO * exp(-E * HCKT(NRHOX)) >= 1, and the record packed as
 * LINEDATA (PACK_LINEDATA, :1964-1977).  One call runs one database loop;
 * the driver order (:19262-19767) is the caller's. */
#define ATLASGPU_SEL_LOWPRED 1  /* gfpred LINEREC [4] int32, unit 11 (:19262-19312) */
#define ATLASGPU_SEL_LOWOBS 2   /* lowobsat12 LINEREC, unit 111 (:19314-19357) */
#define ATLASGPU_SEL_HI 3       /* hilines LINEREC, unit 21 (:19359-19402) */
#define ATLASGPU_SEL_DIATOMIC 4 /* LINEREC as the diatomic reader packs them, sorted by IWL,
                                   IGFLOG before the isotopologue correction (:19403-19529) */
#define ATLASGPU_SEL_TIO 5      /* MOL2 records, 32 bytes, after the header (:19531-19648) */
#define ATLASGPU_SEL_H2O 6      /* {int32 IWL; int16 IELO, IGFLOG}, 8 bytes (:19650-19720) */
#define ATLASGPU_SEL_H3PLUS 7   /* h3plus LINEREC, unit 61 (:19722-19767) */

/* the module variables a database loop reads at entry and leaves behind:
 * NU (1-based bin of IWAVETAB), FREQ (Hz) and IGR (INTEGER(2)) */
typedef struct atlasgpu_select_state {
  int32_t nu;
  int32_t igr;
  double freq;
} atlasgpu_select_state;

/* The tables every database loop reads, kept on the context: XNFDOPMAX
 * (:19248-19256, computed on the device from xnfdop [nspec][kw] and tabcont
 * [nwave+1][kw] over nrhox depths), HCKT(NRHOX) from hckt [nrhox], IWAVETAB
 * [nwave+1] (nondecreasing, the 2**30 sentinel last) and WAVETAB [nwave]
 * (nm, for FREQ = CLIGHT_NMS / WAVETAB(NU)).  nwave + 1 <= 1024. */
int atlasgpu_atlas_select_tables(atlasgpu_ctx *ctx, int nrhox, int kw, const double *xnfdop, int nspec,
                                 const double *hckt, const double *tabcont, const int32_t *iwavetab,
                                 const double *wavetab, int nwave);

/* One database loop over n records of kind's format, in file order (host
 * buffers).  state: in at entry, out as the loop leaves it.  The selected
 * records go to linedata_out [cap][4] in file order; *n_out their count.
 * The reference's fatal cases return ATLASGPU_EINVAL with the record index
 * in atlasgpu_last_error: an unknown diatomic MOLCODE; NELION outside
 * 1..nspec where the reference indexes XNFDOPMAX with it (every kind but
 * LOWPRED, which skips such records); IWL at or past the IWAVETAB sentinel;
 * more than cap selected records (LINEDATA overflow).  Records can be given
 * in chunks: the state carries the loop from one call to the next. */
int atlasgpu_atlas_selectlines(atlasgpu_ctx *ctx, int kind, const void *recs, int64_t n,
                               atlasgpu_select_state *state, int32_t *linedata_out, int64_t cap,
                               int64_t *n_out);

/* The same with device buffers: d_recs aligned to 16 bytes (8 for H2O),
 * d_linedata_out [cap][4] aligned to 16 bytes. */
int atlasgpu_atlas_selectlines_dev(atlasgpu_ctx *ctx, int kind, const void *d_recs, int64_t n,
                                   atlasgpu_select_state *state, int32_t *d_linedata_out, int64_t cap,
                                   int64_t *n_out);

/* ---- device-resident ATLAS12 model ----------------------------------
 * One atmosphere kept on the device for the whole iteration (atlas12c.f90
 * :496-606): hydrostatics, populations and continuum from the documented
 * synthetic surrogate (they stand in for the off-path EOS and KAPP),
 * KAPCONT once, then per iteration LINOP1, the RT pass, the reduction and
 * the finish, as one captured CUDA graph. */
typedef struct atlasgpu_model atlasgpu_model;
typedef struct {
  double teff, logg, vturb_kms;
  int nrhox;                               /* <= 100 */
  const double *t, *p, *rhox, *tauros;     /* starting model [nrhox] */
  const double *waveset, *rcoset;          /* [numnu] */
  int numnu;
  const double *cutoff_wave;               /* KAPCONT grid [nwave] (nm) */
  int nwave;
  const int32_t *linedata;                 /* [nlines][4] */
  int64_t nlines;
  const double *h0tab, *h1tab, *h2tab;     /* TABVOIGT tables, 2001 */
  double mh;                               /* [M/H]: metal abundances scaled by 10**mh */
} atlasgpu_model_desc;

int atlasgpu_model_create(atlasgpu_ctx *ctx, const atlasgpu_model_desc *desc, atlasgpu_model **out);
/* Run up to max_iter iterations; stop after the first whose max |FLXERR| <=
 * tol_percent (tol <= 0: run all).  iters_done and maxerr_hist[max_iter]
 * (may be NULL) receive the count and the per-iteration metric.
 * use_graph != 0 replays one captured graph per iteration. */
int atlasgpu_model_iterate(atlasgpu_ctx *ctx, atlasgpu_model *m, int max_iter, double tol_percent,
                           int use_graph, int *iters_done, double *maxerr_hist);
/* Copy the current structure (each [nrhox], any may be NULL) and the last
 * iteration's HNU(1) per frequency ([numnu], may be NULL). */
int atlasgpu_model_get(atlasgpu_ctx *ctx, atlasgpu_model *m, double *t, double *rhox, double *p,
                       double *xne, double *flxerr, double *hsurf);
/* Copy the model's tables of the last iteration: TABCONT [nwave+1][kw]
 * (KAPCONT's line-cutoff table, atlas12_modules.f90:19072-19138, built on
 * the model's first iteration), XLINES [numnu][kw] (LINOP1's output,
 * :18132-18374) and the continuum ACONT, SIGMAC [numnu][kw] of the RT pass
 * (any may be NULL; depths j >= nrhox are padding).  What the Fortran
 * driver holds in the module arrays TABCONT and XLINES after RUN_RT_PASS. */
int atlasgpu_model_get_tables(atlasgpu_ctx *ctx, atlasgpu_model *m, double *tabcont, double *xlines,
                              double *acont, double *sigmac);
/* Start the model again from a structure (T, P, RHOX [nrhox]), a warm
 * start: every other state vector (except VTURB), the ROSSTAB history, the
 * iteration count and KAPCONT's table start afresh, as after
 * atlasgpu_model_create, so nothing of the previous model carries over. */
int atlasgpu_model_set_structure(atlasgpu_ctx *ctx, atlasgpu_model *m, const double *t,
                                 const double *p, const double *rhox);
/* New stellar parameters for the next model on the same line list and grid
 * (call atlasgpu_model_set_structure after it); no reference counterpart:
 * the reference runs one model per process. */
int atlasgpu_model_set_params(atlasgpu_ctx *ctx, atlasgpu_model *m, double teff, double logg,
                              double vturb_kms, double mh);
/* Frequency sharding of one model over several GPUs.  The reference's
 * frequency loop (RUN_RT_PASS, atlas12_modules.f90:3905-3949) only adds into
 * the TCORR/RADIAP/ROSS mode-2 accumulators, so it splits into contiguous
 * ranges whose sums add; ROSS(3)/RADIAP(3)/TCORR(3) (atlas12c.f90:585-590)
 * then run on the total.  set_shard restricts LINOP1 (XLINES) and the RT pass
 * to NU_FIRST..NU_LAST (1-based, inclusive); set_sums_buffer makes the model
 * write its sums [8*kw + 1] to, and finish from, a caller-owned device buffer
 * (NULL: the model's own); iterate_begin enqueues one iteration up to the
 * sums, iterate_end enqueues the finish, waits and returns max |FLXERR|.
 * Between the two the caller adds the shards' sums (an all-reduce on the
 * context stream). */
int atlasgpu_model_set_shard(atlasgpu_ctx *ctx, atlasgpu_model *m, int nu_first, int nu_last);
int atlasgpu_model_set_sums_buffer(atlasgpu_ctx *ctx, atlasgpu_model *m, double *d_sums);
int atlasgpu_model_iterate_begin(atlasgpu_ctx *ctx, atlasgpu_model *m);
int atlasgpu_model_iterate_end(atlasgpu_ctx *ctx, atlasgpu_model *m, double *maxerr);
int atlasgpu_model_destroy(atlasgpu_ctx *ctx, atlasgpu_model *m);

/* The RT-pass frequency loop for callers that cannot allocate device memory.
 * No counterpart in the reference (it is a second entry to the work of
 * atlasgpu_atlas_rt_pass).  Every input and output is a device pointer owned
 * by the caller: d_waveset, d_rcoset [numnu]; d_acont, d_sigmac, d_scont
 * [numnu][kw] (d_scont may be NULL: SCONT = BNU); d_xlines_t = XLINES
 * transposed, [kw][numnu] (the layout the device LINOP1 writes); d_rhox,
 * d_t, d_hkt [nrhox]; d_sums [8*kw + 1] receives RJMINS, RDABH, RDIAGJ,
 * FLXRAD, RADEN, H_TOTAL, ACCRAD, ABROSS ([q*kw + j], zero for depths
 * nrhox <= j < kw) and PRADK0 ([8*kw]); d_hsurf [numnu] receives HNU(1) per
 * frequency.
 * The call allocates nothing: its scratch is a fixed device array of
 * 1024 x 801 doubles (6.6 MB) in the library image, held by every GPU that
 * loads the library until the process exits.  kw above 100 is rejected.
 * The first call on a device looks the array's address up once (make that
 * first call before any stream capture); that lookup is safe from several
 * host threads at once.  All calls share the array, so calls that overlap on
 * the GPU race: serialise them.  Runs on the context stream and returns
 * without waiting. */
int atlasgpu_atlas_rt_pass_noalloc(atlasgpu_ctx *ctx, int numnu, const double *d_waveset,
                                   const double *d_rcoset, const double *d_acont,
                                   const double *d_sigmac, const double *d_scont, int kw,
                                   const double *d_xlines_t, int nrhox, const double *d_rhox,
                                   const double *d_t, const double *d_hkt, double teff,
                                   double *d_sums, double *d_hsurf);

/* ---- batched ATLAS12 models ----------------------------------------
 * Replaces the reference's grid runs, which start one atlas12c process per
 * model (scripts/runat12_grid.slurm:1-16, scripts/atlas12.sh:231), each
 * running the iteration loop of atlas12c.f90:496-606.  A batch holds
 * `nslots` atmospheres that share the frequency grid, the line list and the
 * Voigt tables of the descriptor (its starting model and stellar parameters
 * are not used); every slot has its own parameters, structure and ROSSTAB
 * history.  One captured CUDA graph runs one iteration of every RUNNING
 * slot; a slot leaves the iteration by itself (status word on the device)
 * when max |FLXERR| <= its tolerance (CONVERGED), when it is not finite
 * (NONFINITE) or at its iteration cap (CAPPED), so a finished slot can be
 * loaded with the next model while the others run. */
#define ATLASGPU_BATCH_MAX_SLOTS 1024
#define ATLASGPU_BATCH_MAX_ITER 256
#define ATLASGPU_SLOT_IDLE 0
#define ATLASGPU_SLOT_RUNNING 1
#define ATLASGPU_SLOT_CONVERGED 2
#define ATLASGPU_SLOT_NONFINITE 3
#define ATLASGPU_SLOT_CAPPED 4
typedef struct atlasgpu_batch atlasgpu_batch;
int atlasgpu_batch_create(atlasgpu_ctx *ctx, const atlasgpu_model_desc *shared, int nslots,
                          atlasgpu_batch **out);
/* Start a model in `slot` (status RUNNING, iteration count 0) from the
 * structure T, P, RHOX [nrhox] on TAUSTD (READIN's starting model,
 * atlas12c.f90:256), with at most max_iter (<= ATLASGPU_BATCH_MAX_ITER)
 * iterations and convergence at max |FLXERR| <= tol_percent (<= 0: run
 * max_iter).  Waits for the context stream. */
int atlasgpu_batch_load(atlasgpu_ctx *ctx, atlasgpu_batch *b, int slot, double teff, double logg,
                        double vturb_kms, double mh, const double *t, const double *p,
                        const double *rhox, int max_iter, double tol_percent);
/* Enqueue n iterations of every RUNNING slot (graph replays; per-launch
 * timed launches when timing is enabled); returns without waiting. */
int atlasgpu_batch_step(atlasgpu_ctx *ctx, atlasgpu_batch *b, int n);
/* Wait, then read every slot's status, iterations done and last max
 * |FLXERR| (arrays [nslots], any may be NULL) and the number still running. */
int atlasgpu_batch_poll(atlasgpu_ctx *ctx, atlasgpu_batch *b, int *status, int *iters,
                        double *maxerr, int *nrunning);
/* Step and poll (every poll_every iterations) until no slot is RUNNING. */
int atlasgpu_batch_run(atlasgpu_ctx *ctx, atlasgpu_batch *b, int poll_every, int *status, int *iters,
                       double *maxerr);
/* A slot's structure (each [nrhox]), HNU(1) per frequency [numnu] of its last
 * iteration and its max |FLXERR| history [iterations done]; any may be NULL. */
int atlasgpu_batch_get(atlasgpu_ctx *ctx, atlasgpu_batch *b, int slot, double *t, double *rhox,
                       double *p, double *xne, double *flxerr, double *hsurf, double *maxerr_hist);
int atlasgpu_batch_nslots(atlasgpu_batch *b);
/* Launch shape of the batched kernels (no reference counterpart): LINOP1 CTAs
 * per SM over the whole batch (1..64, default 16) and the RT pass's frequency
 * groups sized for about rt_waves resident waves over the batch (1..256,
 * default 32).  Results do not depend on the shape beyond the grouping of the
 * frequency sums.  The next step captures a new graph. */
int atlasgpu_batch_set_shape(atlasgpu_ctx *ctx, atlasgpu_batch *b, int linop_ctas_per_sm, int rt_waves);
int atlasgpu_batch_get_shape(atlasgpu_ctx *ctx, atlasgpu_batch *b, int *linop_ctas_per_sm, int *rt_waves);
int atlasgpu_batch_destroy(atlasgpu_ctx *ctx, atlasgpu_batch *b);

/* ---- learned warm start ----------------------------------------------
 * A dense tanh MLP nin -> nh1 -> nh2 -> nout (FP32) that maps stellar
 * parameters to a starting structure; trained on the device on converged
 * models of this library's own ATLAS12 iteration.  No reference counterpart
 * (the reference starts from a tabulated model).  Parameters are one flat
 * vector [W1 (nh1 x nin), b1, W2 (nh2 x nh1), b2, W3 (nout x nh2), b3], W
 * row-major [out][in]; x [n][nin], targets/outputs [n][nout] (host).
 * Loss: mean squared error over samples and outputs. */
typedef struct atlasgpu_mlp atlasgpu_mlp;
int atlasgpu_mlp_create(atlasgpu_ctx *ctx, int nin, int nh1, int nh2, int nout, uint64_t seed,
                        atlasgpu_mlp **out);
int atlasgpu_mlp_destroy(atlasgpu_ctx *ctx, atlasgpu_mlp *p);
int64_t atlasgpu_mlp_nparam(atlasgpu_mlp *p);
int atlasgpu_mlp_get_params(atlasgpu_ctx *ctx, atlasgpu_mlp *p, float *out);
int atlasgpu_mlp_set_params(atlasgpu_ctx *ctx, atlasgpu_mlp *p, const float *in);
int atlasgpu_mlp_forward(atlasgpu_ctx *ctx, atlasgpu_mlp *p, const float *x, int n, float *y);
/* Loss and its gradient over the n samples (grad [nparam], may be NULL). */
int atlasgpu_mlp_loss_grad(atlasgpu_ctx *ctx, atlasgpu_mlp *p, const float *x, const float *t, int n,
                           float *grad, float *loss);
/* Adam (lr, beta 0.9/0.999, eps 1e-8) over `epochs` shuffled passes in
 * minibatches of `batch`; loss_hist [epochs] (may be NULL) receives each
 * epoch's last minibatch loss. */
int atlasgpu_mlp_train(atlasgpu_ctx *ctx, atlasgpu_mlp *p, const float *x, const float *t, int n,
                       int epochs, int batch, float lr, uint64_t seed, float *loss_hist);

/* Measured FP64 FMA throughput of the device (TFLOP/s, 2 flops per FMA):
 * the denominator of the FP64-pipe roofline of the transfer kernels.  No
 * reference counterpart.  Returns a negative value on failure. */
double atlasgpu_fp64_peak_tflops(atlasgpu_ctx *ctx);

/* Measured rate of 64-bit integer atomic adds at L2 (billions per second),
 * warps adding to 32 consecutive words at scattered places of a 64 MB
 * region, the access pattern of LINOP1's exact XLINES sums: the denominator
 * of LINOP1's roofline.  No reference counterpart.  Negative on failure. */
double atlasgpu_u64_atomic_peak(atlasgpu_ctx *ctx);

/* The surrogate physics on the device for given T, P [nrhox]: continuum
 * absorption and scattering kabs, sigma [nw][nrhox] at wave [nw] (nm),
 * electron density xne [nrhox] and XNFDOP [270][nrhox] (may be NULL).  No
 * reference counterpart: it exposes the stand-in for KAPP / the EOS that the
 * device-resident model uses, so that it can be checked. */
int atlasgpu_surrogate_eval(atlasgpu_ctx *ctx, int nrhox, const double *t, const double *p,
                            double vturb_kms, int nw, const double *wave, double *kabs, double *sigma,
                            double *xne, double *xnfdop);

#ifdef __cplusplus
}
#endif
#endif
