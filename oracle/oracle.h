/*
 * oracle.h -- CPU restatement of the ATLAS12 / SYNTHE hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * path in atlas12_b200/csrc: only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it.  The product never links it.
 *
 * Parity status: pinned.  The reference (Fortran 90) cannot be compiled in
 * this image (no Fortran compiler), so every routine below is a line-level
 * restatement of the cited reference source, pinned against the reference's
 * own data constants (operator matrices, quadrature weights, Voigt tables)
 * extracted by tests/golden/make_golden.py and against independent
 * known-answer tests (scipy wofz / expn / numpy.linalg.solve, analytic
 * transfer solutions).  Citations are file:line inside cconroy20/atlas12.
 *
 * Two arithmetic modes for the SYNTHE line loop:
 *   ORC_REF32 : the reference's REAL(4) semantics, lines summed sequentially
 *               in line order (synthe.f90:559-683);
 *   ORC_FP64  : every quantity in double (the all-FP64 accuracy oracle).
 */
#ifndef ATLAS12_ORACLE_H
#define ATLAS12_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NXTAU 51
#define ORC_REF32 0
#define ORC_FP64 1

/* ---- numerics (atlas12_modules.f90) ---------------------------------- */
void orc_parcoe(const double *f, const double *x, double *a, double *b,
                double *c, int n);                              /* :5358-5434 */
void orc_integ(const double *x, const double *f, double *fint, int n,
               double start);                                   /* :5293-5324 */
void orc_deriv(const double *x, const double *f, double *dfdx, int n); /* :5228 */
int orc_map1(const double *xold, const double *fold, int nold,
             const double *xnew, double *fnew, int nnew);       /* :5570-5692 */
void orc_solvit(double *a, int n, double *b, int *ipivot);      /* :5739-5847 */
double orc_expi(int n, double x);                               /* :21103-21225 */
double orc_powi(double x, int m);      /* gfortran REAL(8)**INTEGER */

/* ---- Voigt functions ------------------------------------------------- */
double orc_voigt_weideman(double v, double a); /* synthe_module.f90:463-537, FP64 */
float orc_voigt_profile(float v, float a);     /* same, REAL(4) interface */
void orc_tabvoigt(double vsteps, int n, const double *tabvi,
                  const double *tabh1, int ntab, double *h0tab,
                  double *h1tab, double *h2tab);      /* :19796-19851 */
double orc_voigt_kurucz(double v, double a, const double *h0tab,
                        const double *h1tab, const double *h2tab); /* :21033 */

/* ---- SYNTHE grid + binning (synthe.f90:316-324, mod_mklinelist:898) -- */
typedef struct {
  double ratio, ratiolg, wbegin;
  int32_t length, ixwlbeg;
} orc_grid_t;
void orc_synthe_grid(double wlbeg, double wlend, double resolu, orc_grid_t *g);
int32_t orc_synthe_nbuff(double wlvac, double ratiolg, int32_t ixwlbeg);

/* ---- SYNTHE continuum per depth (synthe.f90:483-516) ------------------
 * continall: [nrhox][3*(nedge-1)] log10 kappa (row = depth)
 * out      : [nrhox][length]  (float for REF32, double for FP64) */
void orc_synthe_continuum(int mode, const double *wledge, int nedge,
                          const double *continall, int ncont_stride,
                          int nrhox, double wbegin, double ratio,
                          int length, void *out);

/* ---- SYNTHE LTE line opacity (synthe.f90:559-683) --------------------
 * Lines are SoA; nelion is 1-based into the per-depth xnfdop/dopple rows
 * of width nspec.  continuum is the REAL(4) array of orc_synthe_continuum
 * (mode REF32) for both modes: the modes differ in the arithmetic of this
 * stage, not in its inputs.
 * opacity_out: [nrhox][length] float (both modes round the final sum). */
typedef struct {
  const int32_t *nbuff;
  const float *cgf;
  const int32_t *nelion;
  const float *elo, *gamrf, *gamsf, *gamwf;
  int64_t n;
} orc_lines_t;
void orc_synthe_line_opacity(int mode, const orc_lines_t *L, int length,
                             int nrhox, double resolu, const void *continuum,
                             const double *xnfdop, const double *dopple,
                             int nspec, const double *xne,
                             const double *txnxn, const double *hckt,
                             int maxprof, double *opacity_f64_out,
                             float *opacity_out);

/* ---- JOSH (atlas12_modules.f90:18398-18776) ------------------------- */
typedef struct {
  double xtau[ORC_NXTAU];
  double coefj[ORC_NXTAU * ORC_NXTAU]; /* column-major, COEFJ(L,M) at [(M-1)*51+L-1] */
  double coefh[ORC_NXTAU * ORC_NXTAU];
  double ch[ORC_NXTAU], ck[ORC_NXTAU];
} orc_ops_t;

typedef struct {
  /* inputs (nrhox) */
  const double *rhox, *acont, *aline, *sigmac, *sigmal, *scont, *sline, *bnu;
  int nrhox;
  /* outputs (nrhox) */
  double *abtot, *alpha, *taunu, *snu, *jnu, *hnu, *jmins;
  double knu1;
  int maxj, edd_iters;
} orc_josh_t;
void orc_josh(const orc_ops_t *ops, int ifscat, int ifsurf, orc_josh_t *s);

/* ---- SYNTHE spectrum (synthe.f90:698-718, 797-902) -------------------
 * contabs/contscat: [nrhox][3*(nedge-1)] log10 tables (contabs_sv layout
 * flattened as (k, iedge) per depth).  opacity: [nrhox][length] float.
 * Writes flux[length], cont[length]. */
void orc_synthe_spectrum(const orc_ops_t *ops, const double *wledge,
                         int nedge, const double *contabs,
                         const double *contscat, int ncont_stride, int nrhox,
                         const double *rhox, const double *hkt,
                         double wbegin, double ratio, int length,
                         const float *opacity, int iw0, int iw1,
                         double *flux, double *cont);

/* ---- ATLAS LINOP1 (atlas12_modules.f90:18132-18374) ------------------
 * linedata: [n][4] int32 (LINEREC); xnfdop, dopple: [nspec][kw] column-major
 * (index (nelion-1)*kw + j-1, i.e. XNFDOP(J,NELION)); tabcont [nwave+1][kw];
 * tablog[65536] indexed by (uint16)I; xlines_out [numnu][kw] (XLINES(J,NU)). */
typedef struct {
  const double *h0tab, *h1tab, *h2tab; /* 2001 */
  const double *tablog;                /* 65536, index = int16 + 32768 */
} orc_atlas_tables_t;
void orc_build_tablog(double *out65536);
int64_t orc_atlas_linop1(const orc_atlas_tables_t *tb, const int32_t *linedata,
                         int64_t nlines, int nrhox, int kw, const double *xnfdop,
                         const double *dopple, int nspec, const double *xne,
                         const double *txnxn, const double *hckt,
                         const double *tabcont, const int32_t *iwavetab,
                         int nwave, const double *waveset, int numnu,
                         double *xlines);

/* ---- XLINOP normal-line branch (atlas12_modules.f90:19873-20174) ------ */
typedef struct {
  double wlvac;
  float elo, gf;
  int32_t nblo, nbup, nelion, itype, ncon, nelionx;
  float gammar, gammas, gammaw;
  int32_t nbuff, lim, pad;
} orc_nlte_line_t;
/* HPROF4's tables (atlas12_modules.f90:20553-20700) and STARK_PROFILE's
 * (:20376-20450, data/stark_profile.dat), and XLINOP's hydrogen level
 * energies (:19964-19975), as the fixture extracted from the source holds
 * them.  Two-index tables are [first index - 1][second index - 1]. */
typedef struct {
  double xknmtb[4][3];  /* XKNMTB(N, M-N) */
  double y1wtm[2][2];   /* Y1WTM(N, M-N) */
  double stalph[34], stwtal[34];
  int32_t istal[4], lnghal[4];
  double stcomp[5][4], stcpwt[5][4]; /* STCOMP(I, N) */
  int32_t lncomp[4];
  double cutoffh2plus[111], cutoffh2[91];
  double asum[100], asumlyman[100];
  double betagrid[15], pp[5];
  double propbm[7][15][5]; /* PROPBM(IP, J, K) at [K-1][J-1][IP-1] */
  double c[7][5], d[7][5]; /* C(IP, K) at [K-1][IP-1] */
  double eh[10], elim;
} orc_htab_t;
/* the depth vectors HPROF4 reads besides XNE and the XNFP/DOPPLE rows of
 * species 1 and 3: T(J), XNF(J,1), XNF(J,2), XNH2(J) */
typedef struct {
  const double *t, *xnf1, *xnf2, *xnh2;
} orc_hatm_t;
double orc_stark_profile(const orc_htab_t *h, double b, double p, int n, int m); /* :20376-20514 */
double orc_hfnm(int n, int m);                                                  /* :20263-20305 */

/* Adds the TYPE 0/3 records' wings into xlines [numnu][kw]; contx is
 * CONTX(25,16) column-major.  With xnfp [nspec][kw] (XNFP(J,NELION)) and rho
 * [kw] also the autoionizing (TYPE 1) and merged-continuum (other TYPEs)
 * records (:20201-20245); NULL skips them.  With htab and hatm (and xnfp)
 * also the hydrogen lines (TYPE -1, HPROF4, :20177-20199).  Returns the
 * number of records read. */
int64_t orc_atlas_xlinop(const orc_atlas_tables_t *tb, const orc_nlte_line_t *recs, int64_t nrec,
                         int nrhox, int kw, const double *xnfdop, const double *dopple, int nspec,
                         const double *xne, const double *txnxn, const double *hckt,
                         const double *tabcont, const int32_t *iwavetab, int nwave,
                         const double *waveset, int numnu, const double *contx, const double *xnfp,
                         const double *rho, const orc_htab_t *htab, const orc_hatm_t *hatm,
                         double *xlines);

/* ---- SYNTHE compute_line_opacity, normal-metal branch
 *      (synthe_module.f90:3167-3458) and, with xnfpel [nrhox][nspec]
 *      (XNFPEL = populations / RHO, synthe.f90:533-542), the autoionizing
 *      (Shore) lines (:3609-3650) and the merged-continuum edges (TYPE >= 4,
 *      :3652-3696, vacuum wavelengths); FP64 restatement ----------------
 * Adds the TYPE 0/3 (and He I, TYPE <= -3) records' opacity at every depth
 * into out [nrhox][length] (double).  recs use nbuff as the grid index;
 * continuum [nrhox][length] (float, the REAL(4) continuum); xnfdop, dopple
 * [nrhox][nspec]; contx CONTX(26,17) column-major. */
void orc_synthe_nlte_opacity(const orc_nlte_line_t *recs, int64_t n, int length, int nrhox,
                             double wbegin, double ratio, double wlend, double velshift_kms,
                             const float *continuum, const double *xnfdop, const double *dopple,
                             const double *xnfpel, int nspec, const double *xne, const double *txnxn,
                             const double *hckt, const double *contx, double *out);

/* ---- ATLAS RT pass, mode-2 integrals (atlas12_modules.f90:3880-3951) --- */
typedef struct {
  double *rjmins, *rdabh, *rdiagj, *flxrad;  /* TCORR mode 2 */
  double *raden, *h_total, *accrad;           /* RADIAP mode 2 */
  double *abross;                             /* ROSS mode 2 */
  double pradk0;
} orc_accum_t;
void orc_atlas_rt_pass(const orc_ops_t *ops, int numnu, const double *waveset,
                       const double *rcoset, const double *acont,
                       const double *sigmac, const double *scont, int kw,
                       const double *xlines, int nrhox, const double *rhox,
                       const double *t, const double *hkt, double teff,
                       int nu0, int nu1, orc_accum_t *acc, double *hsurf);


/* ---- ATLAS12 iteration finish: ROSS(3), RADIAP(3), TCORR(3) ----------
 * Radiative branch (IFCONV = 0: CONVEC not called, CNVFLX = 0, CZ_CONSTRUCT
 * returns at once, no smoothing; USE_DTGRAD = .FALSE.).  ROSSTAB keeps the
 * model's own kappa_R history (stored after ROSS(3), looked up by TTAUP).
 * Arrays [nrhox] are updated in place as the Fortran module arrays are.
 * Returns max |FLXERR| (percent). */
typedef struct {
  int nrhox, iter;
  double teff, grav, pradk0;
  double *t, *rhox, *p, *xne, *abross, *prad, *vturb, *pturb, *tauros, *accrad, *raden, *oldt1;
  double *rjmins, *rdabh, *rdiagj, *flxrad, *h_total; /* mode-2 sums (rdabh modified) */
  double *flxerr, *dtflux, *dtlamb, *dtsurf, *t1;     /* outputs */
  /* ROSSTAB store (atlas12_modules.f90:5937-6228, IROSSTAB = 1): points
   * (normalised log T, log P, log10 kappa_R) appended after every ROSS(3) */
  int nross, maxtab;
  double zerot, slopet, zerop, slopep;
  double *tabt, *tabp, *tabk; /* [maxtab] */
} orc_tcorr_t;
void orc_rosstab_store(orc_tcorr_t *s);
double orc_rosstab(const orc_tcorr_t *s, double t, double p);
void orc_ttaup(const orc_tcorr_t *s, const double *tin, const double *tau, double *abstd,
               double *ptotal, double *pout, const double *prad, int n);
double orc_atlas_finish(orc_tcorr_t *s);

/* ---- SELECTLINES (atlas12_modules.f90:19171-19781) -------------------
 * One database loop of SELECTLINES: the records of one line list, filtered
 * by the line-centre ratio against XNFDOPMAX and the Boltzmann factor at the
 * deepest layer, and packed as LINEDATA records (:1964-1977).
 * kinds and their record formats:
 *   ORC_SEL_LOWPRED  int32[4] LINEREC, gfpred (unit 11)          :19262-19312
 *   ORC_SEL_LOWOBS   int32[4] LINEREC, lowobsat12 (unit 111)     :19314-19357
 *   ORC_SEL_HI       int32[4] LINEREC, hilines (unit 21)         :19359-19402
 *   ORC_SEL_DIATOMIC int32[4] LINEREC as the diatomic reader packs it, sorted
 *                    by IWL, IGFLOG before the isotopologue correction
 *                                                                  :19403-19529
 *   ORC_SEL_TIO      32-byte MOL2 records after the header        :19531-19648
 *   ORC_SEL_H2O      8-byte records {int32 IWL; int16 IELO, IGFLOG} :19650-19720
 *   ORC_SEL_H3PLUS   int32[4] LINEREC, h3plus (unit 61)          :19722-19767
 * st: the module variables the loop reads and leaves behind (NU, 1-based;
 * FREQ; IGR).  xmax [nwave+1][nspec] = XNFDOPMAX (orc_xnfdopmax).
 * Returns the number of records written to out [cap][4], or a negative
 * code (ORC_SEL_E*) with the offending record index in *bad. */
#define ORC_SEL_LOWPRED 1
#define ORC_SEL_LOWOBS 2
#define ORC_SEL_HI 3
#define ORC_SEL_DIATOMIC 4
#define ORC_SEL_TIO 5
#define ORC_SEL_H2O 6
#define ORC_SEL_H3PLUS 7
#define ORC_SEL_ENELION -1   /* NELION outside 1..nspec where the reference indexes with it */
#define ORC_SEL_EMOLCODE -2  /* diatomic MOLCODE not in MOLCODES (the reference stops) */
#define ORC_SEL_ESENTINEL -3 /* IWL at or past the IWAVETAB sentinel */
#define ORC_SEL_EOVERFLOW -4 /* more selected records than cap (LINEDATA overflow) */
typedef struct {
  int32_t nu;
  int32_t igr;
  double freq;
} orc_select_state_t;
/* SELECTLINES's constant tables (:19182-19207), passed in from the fixture
 * extracted out of the reference source */
typedef struct {
  const int32_t *molcodes, *isox; /* MOLCODES(NMOL), ISOX(NMOL) */
  int nmol;
  const int32_t *tio_isocorr;     /* TIO_ISOCORR(5) */
  const int32_t *h2o_isocorr;     /* H2O_ISOCORR(4) */
} orc_select_tables_t;
void orc_xnfdopmax(int nrhox, int kw, const double *xnfdop, int nspec, const double *tabcont,
                   int nwave, double *xmax);                        /* :19248-19256 */
int64_t orc_atlas_selectlines(const orc_select_tables_t *tb, int kind, const void *recs, int64_t n,
                              orc_select_state_t *st, const double *xmax, int nspec, double hckt_last,
                              const int32_t *iwavetab, const double *wavetab, int nwave,
                              int32_t *out, int64_t cap, int64_t *bad);

/* ---- SYNTHE's hydrogen and deuterium lines (compute_line_opacity TYPE -1/-2,
 *      synthe_module.f90:3460-3606) with hydrogen_line_profile (:1032-1980):
 *      the Peterson/Kurucz analytic profile and the Stehle MMM tables
 *      convolved with a Voigt kernel; FP64 restatement, the REAL(4) tables
 *      and threshold literals rounded to single precision as declared ------
 * One Stehle series (INIT_STARK_TABLES, atlas12_modules.f90:17682-17746):
 * n_dens = 0 marks a series that is not loaded.  profiles holds
 * PROFILES(IA, IT, ID, ITRANS) at [ITRANS-1][ID-1][IT-1][IA-1]. */
typedef struct {
  int32_t n_lower, n_upper_min, n_upper_max, n_dens;
  double density_grid[20], temp_grid[10], log_dalpha_grid[60];
  const int32_t *max_dens_idx; /* [n_trans] */
  const double *k_alpha;       /* [n_trans] */
  const double *profiles;      /* [n_trans][n_dens][10][60] */
} orc_stehle_t;
/* the depth vectors hydrogen_line_profile reads: T, XNFPH(J,1), XNFPH(J,2),
 * XNFHE(J,1), XNFH2(J) [nrhox] */
typedef struct {
  const double *t, *xnfph1, *xnfph2, *xnfhe1, *xnfh2;
} orc_shatm_t;
/* hydrogen_line_profile(N, M, J, DELW) at one depth, K-P path (no Stehle
 * tables); dopph is DOPPH(J).  For tests of the profile alone. */
double orc_synthe_hprof_kp(const orc_htab_t *h, int n, int m, double xne, double t, double xnfph1,
                           double xnfph2, double xnfhe1, double xnfh2, double dopph, double delw);
/* hydrogen_line_profile(N, M, J, DELW) on the Stehle path at one depth: the
 * convolution built with Doppler width dopph_conv (the line that built it),
 * evaluated with dopph (this line's); stehle [4].  For tests of the profile
 * alone. */
double orc_synthe_hprof_stehle(const orc_htab_t *h, const orc_stehle_t *stehle, int n, int m, double xne,
                               double t, double xnfph1, double xnfph2, double xnfhe1, double xnfh2,
                               double dopph_conv, double dopph, double delw);
/* Adds the TYPE -1/-2 records' opacity at every depth into out
 * [nrhox][length] (double), the other records skipped; stehle [4] (Lyman,
 * Balmer, Paschen, Brackett) or NULL for the K-P path throughout; tab holds
 * SYNTHE's own tables (eh: EHYD(1..10)).  Returns 0, or -1 when a record's
 * NBLO/NBUP/NCON is outside EHYD/ALPHAHYD/CONTH (the reference aborts). */
int orc_synthe_hydrogen_opacity(const orc_nlte_line_t *recs, int64_t n, int length, int nrhox,
                                double wbegin, double ratio, double wlend, double velshift_kms,
                                const float *continuum, const double *xnfdop, const double *dopple,
                                int nspec, const double *xne, const double *hckt, const orc_htab_t *tab,
                                const orc_stehle_t *stehle, const orc_shatm_t *atm, double *out);

/* ---- KAPP's hydrogen continuum sources (oracle/kapp.c) ---- */
/* Tables of HOP/XKARZAS/COULFF/occupation_prob, HMINOP, H2PLOP and HRAYOP,
 * as the reference reads them from its data files and DATA statements.
 * Fortran arrays column-major. */
typedef struct {
  const float *freqn, *xn, *xl, *ekarzas; /* FREQN(29,15), XN(29,15), XL(29,6,6), EKARZAS(29): REAL(4) */
  const double *gff_logtab;               /* GFF_LOGTAB(81,146): log10 of van Hoof's g_ff */
  const double *q_holtsmark;              /* Q_HOLTSMARK(150) */
  const double *hop_elev;                 /* HOP's level energies E_n (cm^-1), n = 1..15 */
  const double *hmin_wbf, *hmin_bf;       /* HMINOP WBF(116), BF(116) */
  const double *hmin_thetaff;             /* THETAFF(11) */
  const double *hmin_wavek;               /* WAVEK(22) */
  const double *hmin_ff;                  /* FF(11,22) (REAL(4) literals) */
  const double *h2p_fr, *h2p_es;          /* H2PLOP's fits: FR coefficients [5], ES [6], signed */
  const double *ray_m, *ray_ab, *ray_bc, *ray_cd; /* GAVRILAM(74), AB(27), BC(24), CD(22) */
  const double *ray_ly, *ray_fly;         /* GAVRILALYMANCONT(64), FGAVRILALYMANCONT(64) */
  /* helium */
  const double *he1_chi, *he1_freq, *he1_g;                 /* HE1OP CHI(10), HEFREQ(10), G(10) */
  const double *he_x505, *he_x50, *he_x20, *he_x10;         /* CROSSHE X505(92), X50(16), X20(11), X10(21) */
  const double *he2s1s_f, *he2s1s_x, *he2s3s_f, *he2s3s_x;  /* HE12S1S, HE12S3S knots (16 each) */
  const double *he2p1p_f, *he2p1p_x, *he2p3p_f, *he2p3p_x;  /* HE12P1P, HE12P3P knots (16 each) */
  const double *hem_w, *hem_t, *hem_k;                      /* HEMIOP WHEM(17), THEM(12), KHEM(17,12) */
  /* HLINOP: hydrogen_f_value's GF_LYMAN(29), GF_BALMER(28), GF_PASCHEN(27), GF_BRACKETT(3);
   * STARK's KNMTAB(5,4), FSTARK(10,4) */
  const double *gf_lyman, *gf_balmer, *gf_paschen, *gf_brackett, *stark_knm, *stark_f;
} orc_kapp_tables;

enum {
  ORC_KAPP_AHYD, ORC_KAPP_SHYD, ORC_KAPP_AH2P, ORC_KAPP_AHMIN, ORC_KAPP_SHMIN, ORC_KAPP_SIGH, ORC_KAPP_SIGEL,
  ORC_KAPP_ACONT, ORC_KAPP_SCONT, ORC_KAPP_SIGMAC, ORC_KAPP_NOUT,
  /* orc_kapp's helium rows after the ten above */
  ORC_KAPP_AHE1 = ORC_KAPP_NOUT, ORC_KAPP_AHE2, ORC_KAPP_AHEMIN, ORC_KAPP_SIGHE, ORC_KAPP_NOUT_HE
};

double orc_occupation_prob(const orc_kapp_tables *tb, int n, double xne);
void orc_log10_array(const double *in, double *out, int n);
double orc_xkarzas(const orc_kapp_tables *tb, double freq, double zeff2, int n, int l);
/* out[q * nrhox + j], q = ORC_KAPP_*; bhyd BHYD(J,n) at [(n-1)*nrhox + j] or NULL (1); bmin or NULL (1) */
void orc_kapp_hydrogen(const orc_kapp_tables *tb, double wave, int nrhox, const double *t, const double *xne,
                       const double *rho, const double *xnfp1, const double *xnfp2, const double *bhyd,
                       const double *bmin, double *out);
/* orc_kapp_hydrogen with the helium sources (HE1OP, HE2OP, HEMIOP, HERAOP):
 * xnfp3..5 = XNFP(J,3..5), xnf4 = XNF(J,4); out[q * nrhox + j] for
 * q < ORC_KAPP_NOUT_HE */
void orc_kapp(const orc_kapp_tables *tb, double wave, int nrhox, const double *t, const double *xne,
              const double *rho, const double *xnfp1, const double *xnfp2, const double *xnfp3,
              const double *xnfp4, const double *xnfp5, const double *xnf4, const double *bhyd, const double *bmin,
              double *out);
double orc_crosshe(const orc_kapp_tables *tb, double freq);

/* KAPP's H2 tables: H2MINOP's WH2M(10), TH2M(7), KH2M(10,7); PARTFNH2's
 * partfnh2.dat (Q at pf_tstart + (n-1) pf_tstep); H2COLLOP's h2collop.dat
 * (cia_temp [4][cia_ntmax], cia_tab [4][cia_ntmax][cia_nnu] log10) */
typedef struct {
  const double *h2m_w, *h2m_t, *h2m_k;
  int pf_n;
  double pf_tstart, pf_tstep;
  const double *pf;
  int cia_nnu, cia_ntmax;
  const int *cia_nt, *use_pair;
  double cia_nu0, cia_dnu;
  const double *cia_temp, *cia_tab;
} orc_kapp_h2_tables;

enum { ORC_KAPP_AH2MIN = ORC_KAPP_NOUT_HE, ORC_KAPP_AH2COLL, ORC_KAPP_SIGH2, ORC_KAPP_NOUT_H2 };

/* HLINOP (atlas12_modules.f90:17381-17503) at one wavelength (nm), all
 * depths: ahline[j], shline[j]; bhyd BHYD(J,n) at [(n-1)*nrhox + j] or NULL;
 * stehle [4] or NULL (STARK throughout) */
void orc_hlinop(const orc_kapp_tables *tb, const orc_stehle_t *stehle, double wave, int nrhox, const double *t,
                const double *xne, const double *rho, const double *xnfp1, const double *bhyd, double *ahline,
                double *shline);
double orc_stark_mmm(const orc_kapp_tables *tb, const orc_stehle_t *stehle, int n, int m, double freq, double t,
                     double xne);

double orc_partfnh2(const orc_kapp_h2_tables *h2, double t);
double orc_equilh2(const orc_kapp_h2_tables *h2, double t);
/* orc_kapp with the H2 sources (H2MINOP, H2COLLOP, H2RAOP): xnf3 = XNF(J,3);
 * out[q * nrhox + j] for q < ORC_KAPP_NOUT_H2 */
void orc_kapp_h2(const orc_kapp_tables *tb, const orc_kapp_h2_tables *h2, double wave, int nrhox, const double *t,
                 const double *xne, const double *rho, const double *xnfp1, const double *xnfp2, const double *xnfp3,
                 const double *xnfp4, const double *xnfp5, const double *xnf4, const double *xnf3, const double *bhyd,
                 const double *bmin, double *out);

#ifdef __cplusplus
}
#endif
#endif
