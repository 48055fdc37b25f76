"""Extract the reference's own data constants into a test fixture.

Run in a container where the reference checkout is mounted (it is read, never
modified).  Writes tests/golden/reference_tables.npz with:

  coefj, coefh   51x51 J and H operators, from data/blockj.dat, blockh.dat
                 (BLOCKJ/BLOCKH, atlas12_modules.f90:18792-18860: 2601 REAL*4
                 values after a 3-line header, column-major, promoted to
                 REAL*8) -- stored as coef[L-1, M-1] = COEF(L, M)
  xtau8, ch_j, ck_j   JOSH's fixed 51-point tau grid and surface H / K
                 quadrature weights (atlas12_modules.f90:18409-18451)
  tabvi, tabh1   TABVOIGT's 81-point H1(v) table (atlas12_modules.f90:19805-19835)
  awei, lwei     Weideman N=32 coefficients (synthe_module.f90:91-126), kept
                 only to pin the product's own derivation of them
  wavetab        KAPCONT's 361-point continuum-cutoff grid (atlas12_modules.f90:1811-1857)
  molcodes, isox SELECTLINES's diatomic species codes and isotopologue log gf
                 corrections in millidex (atlas12_modules.f90:19182-19202)
  tio_isocorr, h2o_isocorr   the TiO and H2O isotope corrections (:19204, :19207)
  stehle_dims    the four Stehle Stark-profile files' dimensions (stehle_dims)
  s_*            SYNTHE's hydrogen_line_profile tables, laid out like h_* (synthe_hydrogen_tables)
  h_*            the hydrogen line profile's tables (HPROF4, atlas12_modules.f90:20553-21002):
                 h_xknmtb XKNMTB(4,3) and h_y1wtm Y1WTM(2,2) as [n-1, m-n-1]; the fine
                 structure h_stalph, h_stwtal (34), h_istal, h_lnghal (4), h_stcomp,
                 h_stcpwt STCOMP/STCPWT(5,4) as [i-1, n-1], h_lncomp (4); the Lyman alpha
                 satellite cutoffs h_cutoffh2plus (111), h_cutoffh2 (91); the radiative
                 damping sums h_asum, h_asumlyman (100); STARK_PROFILE's grids
                 h_betagrid (15), h_pp (5) (:20376-20514) and its tables from
                 data/stark_profile.dat: h_propbm [7, 15, 5] (profile, beta, P), h_c,
                 h_d [7, 5]; XLINOP's hydrogen level energies h_eh (10) and ELIM_HI
                 h_elim (:19964-19975, :385)
  k_*            KAPP's continuum tables (kapp_tables, kapp_helium_tables, kapp_h2_tables):
                 the Karzas-Latter files, van Hoof's g_ff, Q_HOLTSMARK, HOP's level energies,
                 HMINOP's, H2PLOP's and HRAYOP's DATA statements; HE1OP's levels, CROSSHE,
                 the He I 2s/2p knots, HEMIOP's table; H2MINOP's table, data/partfnh2.dat
                 and data/h2collop.dat
  deck           the reference's converged solar model (workdir/ap00t5777g4.44at12.dat,
                 Teff 5777 K, log g 4.44, 72 depths, iteration 45): READ DECK6
                 columns RHOX, T, P, XNE, ABROSS, ACCRAD, VTURB as printed, [72, 7],
                 plus deck_pradk = PRADK -- output of the reference itself, used
                 to pin INTEG / ROSSTAB / TTAUP

It also writes atlas12_b200/data/operators.npz: the subset that a caller
passes to the library as its operator data (the JOSH operators and grids,
TABVOIGT's table, WAVETAB, the SELECTLINES tables, both programs'
hydrogen tables and KAPP's tables), the way a Fortran driver passes what BLOCKJ/BLOCKH and its
DATA statements hold.  Test-only entries (the Weideman coefficients, the
converged deck) stay in the fixture.

Usage:  python tests/golden/make_golden.py <reference_root>
        (or set ATLAS12_REFERENCE to the reference checkout)
"""
import ctypes
import os
import re
import sys

import numpy as np

ROOT = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ATLAS12_REFERENCE")
HERE = os.path.dirname(os.path.abspath(__file__))
PACKAGE_DATA = os.path.join(HERE, "..", "..", "atlas12_b200", "data", "operators.npz")
TEST_ONLY = ("awei", "lwei", "deck", "deck_pradk", "stehle_dims")

_libc = ctypes.CDLL(None)
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]


def read_real4_block(path):
    """List-directed READ of REAL*4 after 3 header lines (strtof = correctly rounded)."""
    with open(path) as f:
        lines = f.read().splitlines()[3:]
    toks = " ".join(lines).replace(",", " ").split()
    vals = np.array([_libc.strtof(t.encode(), None) for t in toks[:2601]], dtype=np.float32)
    assert vals.size == 2601, path
    # COEF = reshape(dble(C), (/51,51/)): column-major
    return vals.astype(np.float64).reshape(51, 51, order="F")


def fortran_array(src, name, count):
    i = src.index(name)
    j = src.index("/)", i) if "(/" in src[i:i + 200] else src.index("]", i)
    body = src[i:j]
    body = body[body.index("(/") + 2:] if "(/" in body else body[body.index("[") + 1:]
    body = re.sub(r"!.*", "", body)
    nums = re.findall(r"[-+]?\d*\.\d+(?:[DdEe][-+]?\d+)?|[-+]?\d+\.(?:[DdEe][-+]?\d+)?", body)
    vals = np.array([float(x.replace("D", "e").replace("d", "e")) for x in nums])
    assert vals.size == count, (name, vals.size)
    return vals


def fortran_int_array(src, name, count):
    """INTEGER array constructor (/ ... /) or [ ... ] following name, comments dropped."""
    i = src.index(name)
    if "(/" in src[i:i + 60]:
        body = src[src.index("(/", i) + 2:src.index("/)", i)]
    else:
        body = src[src.index("[", i) + 1:src.index("]", i)]
    body = re.sub(r"!.*", "", body).replace("&", " ")
    vals = np.array([int(x) for x in re.findall(r"[-+]?\d+", body)], dtype=np.int32)
    assert vals.size == count, (name, vals.size)
    return vals


def read_stark(path):
    """data/stark_profile.dat: per profile K = 1..7 the PROPBM block (15 rows of
    5), then C (5) and D (5), '#' lines between (STARK_PROFILE's list-directed
    reads, atlas12_modules.f90:20420-20450)."""
    vals = []
    for line in open(path):
        if line.startswith("#") or not line.strip():
            continue
        vals += [float(x.replace("D", "e").replace("d", "e")) for x in line.split()]
    vals = np.array(vals)
    assert vals.size == 7 * 85, vals.size
    v = vals.reshape(7, 85)
    return v[:, :75].reshape(7, 15, 5), v[:, 75:80], v[:, 80:85]


def read_deck(path):
    """READ DECK6 block and PRADK of an ATLAS12 model file."""
    lines = open(path).read().splitlines()
    i = next(k for k, l in enumerate(lines) if l.startswith("READ DECK6"))
    n = int(lines[i].split()[2].rstrip(","))
    rows = np.array([[float(x) for x in lines[i + 1 + j].split()[:7]] for j in range(n)])
    pradk = float(next(l for l in lines if l.startswith("PRADK")).split()[1])
    return rows, np.array([pradk])


def synthe_hydrogen_tables(syn, mod):
    """SYNTHE's own hydrogen_line_profile tables (synthe_module.f90:1047-1160),
    stark_quasistatic_profile's (:776-869) and compute_line_opacity's EHYD
    (:3299-3310), as s_* arrays laid out like the h_* ones.  They are REAL(4)
    PARAMETERs, so each value is rounded to single precision.  Y1WHT's four
    tabulated values are IF branches in the source (:1290-1299), at
    [N-1, M-N-1]; EHYD(9..10) follow ELIM_HI - RYDBERG_H / N**2."""
    hp = syn[syn.index("FUNCTION hydrogen_line_profile"):]
    sq = syn[syn.index("FUNCTION stark_quasistatic_profile"):]
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    const = lambda name: float(re.search(name + r"\s*=\s*([0-9.D+-]+)", mod).group(1).replace("D", "e"))
    elim, rydh = const(r"ELIM_HI"), const(r"RYDBERG_H  ")
    ehyd = [float(re.search(r"ehyd\(%d\) = ([0-9.D+-]+)" % k, syn).group(1).replace("D", "e")) for k in range(1, 9)]
    ehyd += [elim - rydh / float(k) ** 2 for k in (9, 10)]
    prob = np.stack([fortran_array(sq, "PROB%d(75) =" % k, 75).reshape(15, 5) for k in range(1, 8)])
    return dict(
        s_xknmtb=f32(fortran_array(hp, "XKNMTB(4,3) =", 12).reshape(4, 3, order="F")),
        s_y1wtm=np.array([[1.0e18, 1.0e17], [1.0e16, 1.0e14]]),
        s_stalph=f32(fortran_array(hp, "STALPH(34) =", 34)),
        s_stwtal=f32(fortran_array(hp, "STWTAL(34) =", 34)),
        s_istal=fortran_int_array(hp, "ISTAL(4) =", 4),
        s_lnghal=fortran_int_array(hp, "LNGHAL(4) =", 4),
        s_stcomp=f32(fortran_array(hp, "STCOMP(5,4) =", 20).reshape(5, 4, order="F")),
        s_stcpwt=f32(fortran_array(hp, "STCPWT(5,4) =", 20).reshape(5, 4, order="F")),
        s_lncomp=fortran_int_array(hp, "LNCOMP(4) =", 4),
        s_cutoffh2plus=f32(fortran_array(hp, "CUTOFFH2PLUS(111) =", 111)),
        s_cutoffh2=f32(fortran_array(hp, "CUTOFFH2(91) =", 91)),
        s_asum=f32(fortran_array(hp, "ASUM(100) =", 100)),
        s_asumlyman=f32(fortran_array(hp, "ASUMLYMAN(100) =", 100)),
        s_betagrid=f32(fortran_array(sq, "BETA(15) =", 15)),
        s_pp=f32(fortran_array(sq, "PP(5)   =", 5)),
        s_propbm=f32(prob),
        s_c=f32(fortran_array(sq, "CC(5,7) =", 35).reshape(5, 7, order="F").T),
        s_d=f32(fortran_array(sq, "DD(5,7) =", 35).reshape(5, 7, order="F").T),
        s_eh=np.array(ehyd),
        s_elim=np.array([elim]),
    )


def stehle_dims(datadir):
    """Per Stehle series (data/stehle_*.bin, read as INIT_STARK_TABLES does):
    n_lower, n_upper_min, n_upper_max, n_dens, and the number of profile
    values; the synthetic tables used by the tests have these shapes."""
    sys.path.insert(0, os.path.join(HERE, "..", ".."))
    from atlas12_b200 import linelists
    rows = []
    for s in linelists.read_stehle_dir(datadir):
        rows.append([s["n_lower"], s["n_upper_min"], s["n_upper_max"], len(s["density_grid"]), s["profiles"].size])
    return np.array(rows, dtype=np.int64)


def read_real4_lines(path, skip, count):
    """One REAL(4) per list-directed READ after `skip` header lines (XKARZAS's
    read_karzas_tables, atlas12_modules.f90:11730-11802)."""
    lines = open(path).read().splitlines()[skip:skip + count]
    vals = np.array([_libc.strtof(l.split()[0].encode(), None) for l in lines], dtype=np.float32)
    assert vals.size == count, path
    return vals


def read_gauntff(path):
    """data/gauntff_vanhoof.dat as COULFF's reader takes it (:12098-12194):
    five header values after the '#' comments, then 146 rows of 81 g_ff
    (read into REAL(8)); returned as GFF(81,146) column-major, the raw values
    (the library and the oracle take log10 themselves)."""
    rows = []
    for line in open(path):
        line = line.split("#", 1)[0].strip()
        if line:
            rows.append(line)
    head, data = rows[:5], rows[5:5 + 146]  # (the uncertainty table after it is not read)
    assert int(head[0]) == 20140210 and head[1].split() == ["81", "146"], head
    vals = np.array([[float(x.replace("D", "e").replace("d", "e")) for x in r.split()] for r in data])
    assert vals.shape == (146, 81), vals.shape
    return vals.reshape(-1)  # [J][I]: GFF(I, J) at J * 81 + I


def kapp_tables(mod, datadir):
    """KAPP's hydrogen continuum tables: XKARZAS's Karzas-Latter files,
    COULFF's van Hoof table, Q_HOLTSMARK, HOP's level energies, HMINOP's
    bound-free and Bell & Berrington free-free tables (FF is written with
    REAL(4) literals, so each value is rounded to single precision), H2PLOP's
    fits and HRAYOP's Gavrila factors (atlas12_modules.f90:425-464,
    :11359-11608, :12224-12252, :12360-12558, :12740-12906)."""
    hop = mod[mod.index("SUBROUTINE HOP"):mod.index("END SUBROUTINE HOP")]
    elev = [float(x) for x in re.findall(r"EXP\(-([0-9.]+)D0 \* HCKT\(J\)\)", hop)]
    assert len(elev) == 14, len(elev)  # n = 15 .. 2
    hmin = mod[mod.index("SUBROUTINE HMINOP"):mod.index("END SUBROUTINE HMINOP")]
    h2p = mod[mod.index("SUBROUTINE H2PLOP"):mod.index("END SUBROUTINE H2PLOP")]
    ray = mod[mod.index("SUBROUTINE HRAYOP"):mod.index("END SUBROUTINE HRAYOP")]
    num = r"([-+]?[0-9.]+D[-+]?[0-9]+)"
    f = lambda x: float(x.replace("D", "e"))
    fr = re.search(r"FR = " + num + r" \+ \(" + num + r" \+ \(" + num + r" &\s*\+ \(" + num + r" - " + num +
                   r" \* FREQLG\)", h2p)
    es = re.search(r"ES = " + num + r" \+ \(" + num + r" \+ \(" + num + r" &\s*\+ \(" + num + r" \+ \(" + num +
                   r" - " + num + r" \* FREQ\)", h2p)
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    return dict(
        k_freqn=read_real4_lines(os.path.join(datadir, "karzas_freqn.dat"), 2, 29 * 15),
        k_xn=read_real4_lines(os.path.join(datadir, "karzas_xn.dat"), 3, 29 * 15),
        k_xl=read_real4_lines(os.path.join(datadir, "karzas_xl.dat"), 3, 29 * 36),
        k_ekarzas=read_real4_lines(os.path.join(datadir, "karzas_ekarzas.dat"), 2, 29),
        k_gff=read_gauntff(os.path.join(datadir, "gauntff_vanhoof.dat")),
        k_q_holtsmark=fortran_array(mod, "Q_HOLTSMARK(150) =", 150),
        k_hop_elev=np.array([0.0] + elev[::-1]),
        k_hmin_wbf=fortran_array(hmin, ":: WBF(116) =", 116),
        k_hmin_bf=fortran_array(hmin, ":: BF(116) =", 116),
        k_hmin_thetaff=fortran_array(hmin, ":: THETAFF(11) =", 11),
        k_hmin_wavek=fortran_array(hmin, ":: WAVEK(22) =", 22),
        k_hmin_ff=f32(fortran_array(hmin, ":: FF(11, 22) =", 242)),
        k_h2p_fr=np.array([f(fr.group(1)), f(fr.group(2)), f(fr.group(3)), f(fr.group(4)), -f(fr.group(5))]),
        k_h2p_es=np.array([f(es.group(k)) for k in range(1, 6)] + [-f(es.group(6))]),
        k_ray_m=fortran_array(ray, ":: GAVRILAM(74) =", 74),
        k_ray_ab=fortran_array(ray, ":: GAVRILAMAB(27) =", 27),
        k_ray_bc=fortran_array(ray, ":: GAVRILAMBC(24) =", 24),
        k_ray_cd=fortran_array(ray, ":: GAVRILAMCD(22) =", 22),
        k_ray_ly=fortran_array(ray, ":: GAVRILALYMANCONT(64) =", 64),
        k_ray_fly=fortran_array(ray, ":: FGAVRILALYMANCONT(64) =", 64),
    )


def kapp_helium_tables(mod):
    """KAPP's helium tables: HE1OP's level energies, threshold frequencies and
    statistical weights, CROSSHE's Marr & West cross-sections, the 2s/2p fits
    of HE12S1S, HE12S3S, HE12P1P, HE12P3P and HEMIOP's John (1994) free-free
    table (atlas12_modules.f90:12939-13143, :13160-13236, :13299-13545,
    :13716-13833)."""
    def body(name):
        return mod[mod.index(name):mod.index("END " + name)]
    he1 = body("SUBROUTINE HE1OP")
    cross = body("FUNCTION CROSSHE")
    hem = body("SUBROUTINE HEMIOP")
    out = dict(
        k_he1_chi=fortran_array(he1, ":: CHI(10) =", 10),
        k_he1_freq=fortran_array(he1, ":: HEFREQ(10) =", 10),
        k_he1_g=fortran_array(he1, ":: G(10) =", 10),
        k_he_x505=fortran_array(cross, ":: X505(92) =", 92),
        k_he_x50=fortran_array(cross, ":: X50(16) =", 16),
        k_he_x20=fortran_array(cross, ":: X20(11) =", 11),
        k_he_x10=fortran_array(cross, ":: X10(21) =", 21),
        k_hem_w=fortran_array(hem, ":: WHEM(NWHEM) =", 17),
        k_hem_t=fortran_array(hem, ":: THEM(NTHEM) =", 12),
        k_hem_k=fortran_array(hem, ":: KHEM(NWHEM, NTHEM) =", 17 * 12),  # [it][iw]
    )
    # HLINOP's oscillator strengths and Stark parameters (hydrogen_f_value
    # :17760-17829, STARK :17528-17659; KNMTAB(5,4), FSTARK(10,4) column-major)
    hfv = body("FUNCTION hydrogen_f_value")
    stark = mod[mod.index("\nFUNCTION STARK(N, M, J)") + 1:mod.index("END FUNCTION STARK\n")]
    out.update(k_gf_lyman=fortran_array(hfv, ":: GF_LYMAN(29) =", 29),
               k_gf_balmer=fortran_array(hfv, ":: GF_BALMER(28) =", 28),
               k_gf_paschen=fortran_array(hfv, ":: GF_PASCHEN(27) =", 27),
               k_gf_brackett=fortran_array(hfv, ":: GF_BRACKETT(3) =", 3),
               k_stark_knm=fortran_array(stark, ":: KNMTAB(5,4) =", 20),
               k_stark_f=fortran_array(stark, ":: FSTARK(10,4) =", 40))
    for fn, f, x in (("HE12S1S", "FREQ1S", "X1S"), ("HE12S3S", "FREQ3S", "X3S"),
                     ("HE12P1P", "FREQ1P", "X1P"), ("HE12P3P", "FREQ3P", "X3P")):
        src = body("FUNCTION " + fn)
        key = fn[3:].lower()
        out["k_he%s_f" % key] = fortran_array(src, ":: %s(16) =" % f, 16)
        out["k_he%s_x" % key] = fortran_array(src, ":: %s(16) =" % x, 16)
    return out


def kapp_h2_tables(mod, datadir):
    """KAPP's H2 tables: H2MINOP's H2- free-free table (WH2M, TH2M, KH2M),
    PARTFNH2's data/partfnh2.dat (T, Q pairs; the reader skips '#' and blank
    lines) and H2COLLOP's data/h2collop.dat (log10 CIA coefficients of the
    H2-H2, H2-He, H2-H and H-He pairs on a uniform wavenumber grid), read as
    the reference reads them (atlas12_modules.f90:12611-12708, :22324-22418,
    :16371-16527).  CIATAB is returned [pair][temperature][wavenumber] with
    -99 past a pair's own temperature count, as the reader initialises it."""
    h2m = mod[mod.index("SUBROUTINE H2MINOP"):mod.index("END SUBROUTINE H2MINOP")]
    pf = []
    for line in open(os.path.join(datadir, "partfnh2.dat")):
        line = line.strip()
        if not line or line.startswith("#"):
            continue
        t, q = line.split()[:2]
        pf.append((float(t), float(q)))
    pf = np.array(pf)
    assert np.all(np.diff(pf[:, 0]) == pf[1, 0] - pf[0, 0]), "partfnh2.dat: T not uniform"
    toks, names = [], []
    lines = [l for l in open(os.path.join(datadir, "h2collop.dat")) if not l.startswith("#")]
    npair, ntmax = (int(x) for x in lines[0].split()[:2])
    ncianu, nu0, dnu = lines[1].split()[:3]
    ncianu, nu0, dnu = int(ncianu), float(nu0), float(dnu)
    temps = np.zeros((npair, ntmax))
    tab = np.full((npair, ntmax, ncianu), -99.0)
    nciat = np.zeros(npair, np.int32)
    body = lines[2:]
    ip = -1
    for line in body:
        if line[:1].isalpha():
            ip += 1
            name, n = line.split()[:2]
            names.append(name)
            nciat[ip] = int(n)
            toks.append([])
        else:
            toks[ip].extend(float(x.replace("D", "e").replace("d", "e")) for x in line.split())
    assert ip + 1 == npair == 4, (ip, npair)
    for ip in range(npair):
        n = nciat[ip]
        v = np.array(toks[ip])
        assert v.size == n + n * ncianu, (names[ip], v.size)
        temps[ip, :n] = v[:n]
        tab[ip, :n] = v[n:].reshape(n, ncianu)
    return dict(
        k_h2m_w=fortran_array(h2m, ":: WH2M(NWH2M) =", 10),
        k_h2m_t=fortran_array(h2m, ":: TH2M(NTH2M) =", 7),
        k_h2m_k=fortran_array(h2m, ":: KH2M(NWH2M, NTH2M) =", 70),  # [it][iw]
        k_pf_h2=pf[:, 1], k_pf_h2_t=pf[:, 0],
        k_cia_grid=np.array([ncianu, nu0, dnu]), k_cia_nt=nciat, k_cia_temp=temps, k_cia_tab=tab,
    )


def main():
    if not ROOT or not os.path.isdir(ROOT):
        sys.exit("usage: make_golden.py <reference_root>  (or ATLAS12_REFERENCE=<reference_root>)")
    mod = open(os.path.join(ROOT, "src", "atlas12_modules.f90")).read()
    syn = open(os.path.join(ROOT, "src", "synthe_module.f90")).read()
    out = dict(
        coefj=read_real4_block(os.path.join(ROOT, "data", "blockj.dat")),
        coefh=read_real4_block(os.path.join(ROOT, "data", "blockh.dat")),
        ch_j=fortran_array(mod, "CH_J(NXTAU) =", 51),
        ck_j=fortran_array(mod, "CK_J(NXTAU) =", 51),
        xtau8=fortran_array(mod, "XTAU8(NXTAU) =", 51),
        tabvi=fortran_array(mod, "TABVI(81) =", 81),
        tabh1=fortran_array(mod, "TABH1(81) =", 81),
        awei=fortran_array(syn, "AWEI(32) =", 32),
        lwei=np.array([float(re.search(r"LWEI = ([0-9.D+-]+)", syn).group(1).replace("D", "e"))]),
        wavetab=fortran_array(mod, "WAVETAB(NWAVE) =", 361),
        molcodes=fortran_int_array(mod, "MOLCODES(NMOL) =", 46),
        isox=fortran_int_array(mod, "ISOX(NMOL) =", 46),
        tio_isocorr=fortran_int_array(mod, "TIO_ISOCORR(5) =", 5),
        h2o_isocorr=fortran_int_array(mod, "H2O_ISOCORR(4) =", 4),
        h_xknmtb=fortran_array(mod, "XKNMTB(4,3) =", 12).reshape(4, 3, order="F"),
        h_y1wtm=fortran_array(mod, "Y1WTM(2,2) =", 4).reshape(2, 2, order="F"),
        h_stalph=fortran_array(mod, "STALPH(34) =", 34),
        h_stwtal=fortran_array(mod, "STWTAL(34) =", 34),
        h_istal=fortran_int_array(mod, "ISTAL(4) =", 4),
        h_lnghal=fortran_int_array(mod, "LNGHAL(4) =", 4),
        h_stcomp=fortran_array(mod, "STCOMP(5,4) =", 20).reshape(5, 4, order="F"),
        h_stcpwt=fortran_array(mod, "STCPWT(5,4) =", 20).reshape(5, 4, order="F"),
        h_lncomp=fortran_int_array(mod, "LNCOMP(4) =", 4),
        h_cutoffh2plus=fortran_array(mod, "CUTOFFH2PLUS(111) =", 111),
        h_cutoffh2=fortran_array(mod, "CUTOFFH2(91) =", 91),
        h_asum=fortran_array(mod, "ASUM(100) =", 100),
        h_asumlyman=fortran_array(mod, "ASUMLYMAN(100) =", 100),
        h_betagrid=fortran_array(mod, "BETAGRID(15) =", 15),
        h_pp=fortran_array(mod, "PP(5) =", 5),
        h_eh=np.array([float(re.search(r"EH\(%d\) = ([0-9.D+-]+)" % k, mod).group(1).replace("D", "e"))
                       for k in range(1, 11)]),
        h_elim=np.array([float(re.search(r"ELIM_HI = ([0-9.D+-]+)", mod).group(1).replace("D", "e"))]),
    )
    out["h_propbm"], out["h_c"], out["h_d"] = read_stark(os.path.join(ROOT, "data", "stark_profile.dat"))
    out.update(synthe_hydrogen_tables(syn, mod))
    out["stehle_dims"] = stehle_dims(os.path.join(ROOT, "data"))
    out.update(kapp_tables(mod, os.path.join(ROOT, "data")))
    out.update(kapp_helium_tables(mod))
    out.update(kapp_h2_tables(mod, os.path.join(ROOT, "data")))
    out["deck"], out["deck_pradk"] = read_deck(os.path.join(ROOT, "workdir", "ap00t5777g4.44at12.dat"))
    np.savez_compressed(os.path.join(HERE, "reference_tables.npz"), **out)
    np.savez_compressed(PACKAGE_DATA, **{k: v for k, v in out.items() if k not in TEST_ONLY})
    for k, v in out.items():
        print(k, v.shape)


if __name__ == "__main__":
    main()
