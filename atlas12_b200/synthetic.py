"""Seeded synthetic workloads with the shapes of the named configurations.

There is no network and the reference's line lists are not distributed with
it, so every workload is synthetic (numpy.random.default_rng(seed)):

* SYNTHE (one atmosphere): 72-depth Eddington grey model (Teff, log g), lines
  with lambda uniform in a window, log gf ~ N(-2, 1.5) and E_low ~ U(0, 8) eV
  for atoms, log gf ~ N(-4, 1) and E_low ~ U(0, 3) eV for molecules,
  log gamma_rad / Stark / vdW ~ N(8, 0.3) / N(-5.5, 0.5) / N(-7.5, 0.3)
  normalised by 4 pi nu as the gfall reader does (mod_mklinelist.f90:996-1006).
* ATLAS12 opacity sampling: LINEDATA records with int16 fields
  NINT(log10(x)*1000 + 16384) (atlas12_modules.f90:19497-19501).

Populations and continuum come from atlas12_b200.surrogate.
"""
import numpy as np

from . import surrogate as sg

C_NM = 2.99792458e17
EV_CM = 8065.543937


def synthe_edges(wlbeg, wlend):
    """Continuum edge list covering [wlbeg, wlend] with the H I edges that fall
    inside, ~2 nm apart, padded on both sides (wledge_m analogue)."""
    lo, hi = wlbeg * 0.98, wlend * 1.02
    n = max(int((hi - lo) / 2.0), 4)
    e = list(np.linspace(lo, hi, n + 1))
    for h in (91.175, 364.70, 820.6):
        if lo < h < hi:
            e.append(h)
    return np.unique(np.array(e))


def synthe_continuum_tables(wledge, t, p, e=None):
    """log10 kappa tables on (left edge, mid, right edge) of every interval,
    [nrhox, 3*(nedge-1)]: continall (abs+scat), contabs, contscat."""
    ne = wledge.size
    pts = []
    for i in range(ne - 1):
        a, b = wledge[i], wledge[i + 1]
        eps = (b - a) * 1e-9
        pts += [a + eps, 0.5 * (a + b), b - eps]
    ka, sgm = sg.continuum_opacity(np.array(pts), t, p, e)
    return (np.log10(ka + sgm).T.copy(), np.log10(ka).T.copy(), np.log10(sgm).T.copy())


def synthe_atmosphere(teff=5777.0, logg=4.44, vturb=1.5, nrhox=72, ross=None, mh=0.0):
    m = sg.grey_model(teff, logg, nrhox=nrhox, ross=ross)
    pop = sg.populations(m["t"], m["p"], vturb, mh=mh)
    t = m["t"]
    hkt = sg.HPLANCK / (sg.KBOL * t)
    hckt = hkt * sg.CLIGHT
    # SYNTHE keeps these as REAL(4) values (synthe.f90:374-392)
    xne32 = pop["xne"].astype(np.float32).astype(np.float64)
    nh = pop["xnfp"][:, 0] * 2.0
    txnxn = ((nh + 0.42 * 0.085 * nh) * (t.astype(np.float32) / 10000.0) ** 0.3).astype(np.float32)
    xnfdop = np.where(pop["dopple"] > 0, pop["xnfp"] / pop["rho"][:, None] / np.maximum(pop["dopple"], 1e-300), 0.0)
    return dict(model=m, t=t, p=m["p"], rhox=m["rhox"], rho=pop["rho"], hkt=hkt, hckt=hckt,
                xne=xne32, txnxn=txnxn.astype(np.float64), xnfdop=xnfdop, dopple=pop["dopple"],
                eos=pop, teff=teff, logg=logg)


def synthe_lines(n, wlbeg, wlend, seed=1, mol_frac=0.0):
    """Raw line parameters (vacuum nm, gf, elo cm^-1, damping) before binning."""
    rng = np.random.default_rng(seed)
    wl = np.sort(rng.uniform(wlbeg, wlend, n))
    is_mol = rng.uniform(size=n) < mol_frac
    loggf = np.where(is_mol, rng.normal(-4.0, 1.0, n), rng.normal(-2.0, 1.5, n))
    elo_ev = np.where(is_mol, rng.uniform(0.0, 3.0, n), rng.uniform(0.0, 8.0, n))
    lgr = rng.normal(8.0, 0.3, n)
    lgs = rng.normal(-5.5, 0.5, n)
    lgw = rng.normal(-7.5, 0.3, n)
    atoms = [sg.nelion(z, s) for z in sg.METALS[:, 0] for s in (1, 2)]
    mols = [sg.mol_nelion(s) for s in sg.MOLECULES[:, 0]]
    nel = np.where(is_mol, rng.choice(mols, n), rng.choice(atoms, n)).astype(np.int32)
    # reader conversions (mod_mklinelist.f90:996-1006)
    frelin = 2.99792458e17 / wl
    gf = (10.0 ** loggf.astype(np.float32)).astype(np.float32)
    cgf = (0.026538 / 1.77245 * gf.astype(np.float64) / frelin).astype(np.float32)
    frq4pi = 12.5664 * frelin
    return dict(wlvac=wl, cgf=cgf, nelion=nel, elo=(elo_ev * EV_CM).astype(np.float32),
                gamrf=(10.0 ** lgr / frq4pi).astype(np.float32),
                gamsf=(10.0 ** lgs / frq4pi).astype(np.float32),
                gamwf=(10.0 ** lgw / frq4pi).astype(np.float32))


def synthe_case(nlines=20000, wlbeg=400.0, wlend=410.0, resolu=500000.0, seed=1, teff=5777.0,
                logg=4.44, vturb=1.5, mol_frac=0.0, nrhox=72, ross=None, mh=0.0):
    """Complete SYNTHE input set (the small CPU-runnable case by default)."""
    atm = synthe_atmosphere(teff, logg, vturb, nrhox, ross=ross, mh=mh)
    wledge = synthe_edges(wlbeg, wlend)
    cont_all, cont_abs, cont_scat = synthe_continuum_tables(wledge, atm["t"], atm["p"], atm["eos"])
    lines = synthe_lines(nlines, wlbeg, wlend, seed=seed, mol_frac=mol_frac)
    return dict(atm=atm, wledge=wledge, continall=cont_all, contabs=cont_abs, contscat=cont_scat,
                lines=lines, wlbeg=wlbeg, wlend=wlend, resolu=resolu)


def grid_cases(n, seed=4, line_scale=1.0, lo=300.0, hi=1000.0):
    """The batched-grid workload: n atmospheres with Teff U(3500, 8000) K,
    log g U(1, 5), [M/H] U(-2, 0.5), each with its own window of U(5, 100) nm
    inside lo..hi at R = 500,000 and U(0.2, 5)M lines (times line_scale),
    30 % molecular.  Returns synthe_case dicts (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        teff, logg, mh = rng.uniform(3500.0, 8000.0), rng.uniform(1.0, 5.0), rng.uniform(-2.0, 0.5)
        width = rng.uniform(5.0, 100.0)
        wlbeg = rng.uniform(lo, hi - width)
        nl = int(rng.uniform(0.2e6, 5.0e6) * line_scale)
        c = synthe_case(nlines=nl, wlbeg=wlbeg, wlend=wlbeg + width, seed=seed * 1000 + k, teff=teff, logg=logg,
                        mol_frac=0.3, mh=mh)
        c["params"] = (teff, logg, mh)
        out.append(c)
    return out


# ---------------------------------------------------------------- ATLAS12
def encode_i16(x):
    """NINT(log10(x)*1000 + 16384) clipped to INTEGER(2) (atlas12_modules.f90:19497-19501)."""
    v = np.rint(np.log10(x) * 1000.0 + 16384.0)
    return np.clip(v, -32768, 32767).astype(np.int16)


def pack_linedata(iwl, ielion, ielo, igflog, igr, igs, igw):
    """LINEREC = [IWL | IELION,IELO | IGFLOG,IGR | IGS,IGW] (atlas12_modules.f90:1950-1977)."""
    def pair(lo, hi):
        return (lo.astype(np.int16).view(np.uint16).astype(np.uint32) |
                (hi.astype(np.int16).view(np.uint16).astype(np.uint32) << 16)).view(np.int32)
    return np.stack([iwl.astype(np.int32), pair(ielion, ielo), pair(igflog, igr), pair(igs, igw)], axis=1)


def atlas_lines(n, wl_lo, wl_hi, seed=2, mol_frac=0.0):
    """LINEDATA for the opacity-sampling line loop, lambda log-uniform."""
    rng = np.random.default_rng(seed)
    ratiolg = np.log(1.0 + 1.0 / 2000000.0)
    wl = np.sort(np.exp(rng.uniform(np.log(wl_lo), np.log(wl_hi), n)))
    iwl = np.floor(np.log(wl) / ratiolg + 0.5).astype(np.int64)
    is_mol = rng.uniform(size=n) < mol_frac
    loggf = np.where(is_mol, rng.normal(-4.0, 1.0, n), rng.normal(-2.0, 1.5, n))
    elo_ev = np.where(is_mol, rng.uniform(0.0, 3.0, n), rng.uniform(0.0, 8.0, n))
    atoms = [sg.nelion(z, s) for z in sg.METALS[:, 0] for s in (1, 2)]
    mols = [sg.mol_nelion(s) for s in sg.MOLECULES[:, 0]]
    nel = np.where(is_mol, rng.choice(mols, n), rng.choice(atoms, n))
    # IELION = 10*NELION (+ isotope digit 0); gammas are per-unit-frequency
    # widths times 4 pi c / lambda -> GAMMA = TABLOG(IG)*WLVAC*(1/(4 pi c)).
    gr = 10.0 ** rng.normal(8.0, 0.3, n)
    gs = 10.0 ** rng.normal(-5.5, 0.5, n)
    gw = 10.0 ** rng.normal(-7.5, 0.3, n)
    return pack_linedata(iwl, (nel * 10).astype(np.int16), encode_i16(elo_ev * EV_CM),
                         encode_i16(10.0 ** loggf), encode_i16(gr), encode_i16(gs), encode_i16(gw))


def nlte_records(n, wl_lo, wl_hi, seed=6, strong=0.05, ncon_frac=0.3, types=(0, 3, 2, 1), type_p=(.7, .15, .1, .05)):
    """Unit-19 records (the NLTE / complex-profile list XLINOP reads), sorted
    by wavelength, with the ATLAS line distributions plus: a fraction `strong`
    of lines 4 dex stronger (wings beyond LINOP1's 100 points), a fraction
    `ncon_frac` with a continuum-edge cutoff (NCON 1..10, NELIONX 1..16), and
    the line types in `types` with probabilities `type_p`."""
    from . import _lib
    rng = np.random.default_rng(seed)
    ratiolg = np.log(1.0 + 1.0 / 2000000.0)
    wl = np.sort(np.exp(rng.uniform(np.log(wl_lo), np.log(wl_hi), n)))
    atoms = [sg.nelion(z, s) for z in sg.METALS[:, 0] for s in (1, 2)]
    loggf = rng.normal(-2.0, 1.5, n) + np.where(rng.uniform(size=n) < strong, 4.0, 0.0)
    four_pi_c = 4.0 * np.pi * C_NM
    r = np.zeros(n, _lib.NLTE_LINE)
    r["wlvac"] = wl
    r["elo"] = rng.uniform(0.0, 8.0, n) * EV_CM
    r["gf"] = 0.026538 / np.sqrt(np.pi) / C_NM * wl * 10.0 ** loggf  # CGF
    r["nelion"] = rng.choice(atoms, n)
    r["itype"] = rng.choice(np.array(types), n, p=np.array(type_p) / np.sum(type_p))
    has = rng.uniform(size=n) < ncon_frac
    r["ncon"] = np.where(has, rng.integers(1, 11, n), 0)
    r["nelionx"] = np.where(has, rng.integers(1, 17, n), 0)
    r["gammar"] = 10.0 ** rng.normal(8.0, 0.3, n) * wl / four_pi_c
    r["gammas"] = 10.0 ** rng.normal(-5.5, 0.5, n) * wl / four_pi_c
    r["gammaw"] = 10.0 ** rng.normal(-7.5, 0.3, n) * wl / four_pi_c
    r["nbuff"] = np.floor(np.log(wl) / ratiolg + 0.5).astype(np.int32)  # IWL
    return r


def contx_table(seed=7):
    """A CONTX(25,16) edge table [16, 25] (cm^-1) placing continuum edges
    across the optical and near-UV: for tests of XLINOP's blue-wing cutoff."""
    rng = np.random.default_rng(seed)
    t = np.zeros((16, 25))
    t[:, :10] = rng.uniform(1.0e4, 1.0e5, (16, 10))
    return t


def atlas_waveset(nustart=9599, numnu=30000):
    """WAVESET(NU) = 10**(1 + 1e-4*(NU+NUSTART-1)) and RCOSET trapezoid weights
    (atlas12c.f90:451-491)."""
    nu = np.arange(1, numnu + 1)
    ws = 10.0 ** (1.0 + 0.0001 * (nu + nustart - 1))
    f = C_NM / ws
    rc = np.zeros(numnu)
    rc[0] = (f[0] - f[1]) * 1.5
    rc[1:-1] = (f[:-2] - f[2:]) * 0.5
    rc[-1] = (f[-2] + f[-1]) * 0.25
    return ws, rc


def geometric_waveset(wl_lo=9.0, wl_hi=160000.0, numnu=30000):
    """log-spaced grid over the stated span with the same trapezoid weights."""
    ws = np.geomspace(wl_lo, wl_hi, numnu)
    f = C_NM / ws
    rc = np.zeros(numnu)
    rc[0] = (f[0] - f[1]) * 1.5
    rc[1:-1] = (f[:-2] - f[2:]) * 0.5
    rc[-1] = (f[-2] + f[-1]) * 0.25
    return ws, rc


# ------------------------------------------------------------ SELECTLINES
def selectlines_tables(wavetab, nspec=1006, kw=80, nrhox=72, seed=11, dead_frac=0.15, faint_frac=0.03):
    """XNFDOP [nspec, kw], HCKT [nrhox], TABCONT [nwave+1, kw] for SELECTLINES.

    XNFDOPMAX(e, nu) comes out near FREQ(nu) * 10**(3.8 + N(0, 1)), so lines of
    log gf ~ -2 straddle the CENRATIO = 1 cut; a fraction of the species have
    no population (XNFDOPMAX = 0) and a few a vanishing one (<= 1e-37).
    Depths past nrhox hold values that would dominate the maximum if read."""
    rng = np.random.default_rng(seed)
    wavetab = np.asarray(wavetab, np.float64)
    nwave = wavetab.size
    freq = 2.99792458e17 / np.append(wavetab, wavetab[-1])
    j = np.arange(kw)
    h = 0.3 * np.sin(0.37 * j)
    d = -0.2 * np.cos(0.21 * j)
    c = -np.log10(freq) + rng.normal(0.0, 0.3, nwave + 1)
    tabcont = 10.0 ** (c[:, None] + d[None, :])
    s = 3.8 + rng.normal(0.0, 1.0, nspec) - np.max((h - d)[:nrhox])
    s[[894, 939]] = 5.6  # TiO and H2O (log gf ~ -4)
    xnfdop = 10.0 ** (s[:, None] + h[None, :])
    dead = rng.uniform(size=nspec) < dead_frac
    dead[[894, 939]] = False
    xnfdop[dead] = 0.0
    faint = (rng.uniform(size=nspec) < faint_frac) & ~dead
    faint[[894, 939]] = False
    xnfdop[faint] = 1.0e-60
    xnfdop[:, nrhox:] = 1.0e300
    tabcont[:, nrhox:] = 1.0e-300
    t = np.linspace(4000.0, 12000.0, nrhox)
    hckt = 1.4387773538277204 / t
    return xnfdop, hckt, tabcont


def _wl_iwl(rng, n, lo, hi, sort=True):
    ratiolg = np.log(1.0 + 1.0 / 2000000.0)
    wl = np.exp(rng.uniform(np.log(lo), np.log(hi), n))
    if sort:
        wl = np.sort(wl)
    return (np.log(wl) / ratiolg + 0.5).astype(np.int64)


def selectlines_records(kind, n, wavetab, seed=12, shuffle_frac=0.0, nspec=1006, bad_frac=0.0):
    """Seeded records of one SELECTLINES database kind (atlas12_b200._lib.SEL_*).

    LINEREC kinds span WAVETAB (a few below its first bin and past its last),
    with log gf ~ N(-2, 1.5), E ~ U(0, 64500) cm-1 and random species; MOL2 and
    H2O records mimic the TiO and H2O lists.  shuffle_frac swaps that fraction
    of records with a random other one (the NU advance then sees IWL go back);
    bad_frac plants NELION values outside 1..nspec (LINEREC kinds)."""
    from ._lib import SEL_DIATOMIC, SEL_TIO, SEL_H2O, SEL_H3PLUS, MOL2_REC, H2O_REC
    rng = np.random.default_rng(seed)
    lo, hi = float(wavetab[0]) * 0.97, float(wavetab[-1]) * 1.02
    if kind == SEL_TIO:
        r = np.zeros(n, MOL2_REC)
        r["wl"] = np.sort(np.exp(rng.uniform(np.log(300.0), np.log(5000.0), n))).astype(np.float32)
        r["gflog"] = rng.normal(-4.0, 1.2, n).astype(np.float32)
        r["e1"] = rng.uniform(0.0, 30000.0, n).astype(np.float32)
        r["e2"] = (r["e1"] + rng.normal(0.0, 3000.0, n)).astype(np.float32)
        r["code"] = np.where(rng.uniform(size=n) < 0.85, 822, rng.choice([606, 101, 823], n))
        r["iso"] = np.where(rng.uniform(size=n) < 0.9, rng.integers(46, 51, n), rng.choice([45, 51], n))
        r["gr"] = np.where(rng.uniform(size=n) < 0.5, 0, (100 * rng.normal(8.0, 0.4, n)).astype(np.int32))
        r["label"] = rng.integers(0, 2, n)
        bad = rng.uniform(size=n) < 0.002
        r["wl"][bad] = np.where(rng.uniform(size=bad.sum()) < 0.5, 0.0, -1.0).astype(np.float32)
        rec = r
    elif kind == SEL_H2O:
        r = np.zeros(n, H2O_REC)
        r["iwl"] = _wl_iwl(rng, n, 500.0, min(hi, 1.0e5))
        mag = rng.integers(1, 30000, n)
        r["ielo"] = np.where(rng.uniform(size=n) < 0.5, mag, -mag).astype(np.int16)
        g = np.clip(np.rint(16384 + 1000 * rng.normal(-4.0, 1.5, n)), 1, 32767).astype(np.int32)
        r["igflog"] = np.where(rng.uniform(size=n) < 0.5, g, -g).astype(np.int16)
        rec = r
    else:
        iwl = _wl_iwl(rng, n, lo, hi)
        if kind == SEL_DIATOMIC:
            # the diatomic species codes SELECTLINES knows (MOLCODES)
            codes = np.array([8410, 8411, 8460, 8461, 8470, 8471, 8480, 8481, 8482, 8510, 8511, 8512, 8530, 8531,
                              8532, 8580, 8581, 8582, 8583, 8584, 8620, 8621, 8622, 8623, 8640, 8641, 8642, 8643,
                              8680, 8681, 8682, 8690, 8691, 8692, 8693, 8700, 8701, 8702, 8703, 8704, 8705, 8890,
                              8891, 8892, 8896, 8960])
            ielion = rng.choice(codes, n)
            loggf = rng.normal(-3.0, 1.5, n)
        else:
            nel = rng.integers(1, nspec + 1, n)
            ielion = np.where(rng.uniform(size=n) < 0.5, 1, -1) * (10 * nel + rng.integers(0, 10, n))
            if bad_frac > 0:
                b = rng.uniform(size=n) < bad_frac
                ielion[b] = rng.choice([0, 5, -7, 10 * (nspec + 1), 10 * (nspec + 3) + 4], b.sum())
            loggf = rng.normal(-2.0, 1.5, n) if kind != SEL_H3PLUS else rng.normal(-1.0, 1.5, n)
        elo = rng.uniform(1.0, 64500.0, n)
        rec = pack_linedata(iwl, ielion.astype(np.int16), encode_i16(elo), encode_i16(10.0 ** loggf),
                            encode_i16(10.0 ** rng.normal(8.0, 0.3, n)), encode_i16(10.0 ** rng.normal(-5.5, 0.5, n)),
                            encode_i16(10.0 ** rng.normal(-7.5, 0.3, n)))
    if shuffle_frac > 0 and n > 1:
        k = int(n * shuffle_frac)
        a = rng.integers(0, n, k)
        b = rng.integers(0, n, k)
        tmp = rec[a].copy()
        rec[a] = rec[b]
        rec[b] = tmp
    return rec


def stehle_tables(seed=11, series=((1, 2, 30), (2, 3, 30), (3, 4, 30), (4, 5, 7))):
    """Stehle-format Stark profile tables with the shapes of the published
    ones (20 densities 1e10..3e19 per half dex, 10 temperatures 2500 K to
    1.26e6 K, 60 log Delta-alpha points -3.5..5.5) and Holtsmark-like values
    (flat core, Delta-alpha**-2.5 wings) that are zero above each transition's
    Inglis-Teller density, for tests of the Stark-convolution path.  Returns
    4 dicts in the layout the readers give (profiles [n_trans, n_dens, 10, 60])."""
    rng = np.random.default_rng(seed)
    out = []
    lg = np.linspace(-3.5, 5.5, 60)
    temps = np.array([2500., 5000., 10000., 19950., 39810., 79430., 158500., 316200., 631000., 1259600.])
    for n_lower, n_min, n_max in series:
        nd = 20 if n_lower < 4 else 18
        dens = 10.0 ** (10.0 + 0.5 * np.arange(nd))
        ntr = n_max - n_min + 1
        mdi = np.clip(nd - np.arange(ntr) // 2 - rng.integers(0, 3, ntr), 4, nd).astype(np.int32)
        kal = 10.0 ** rng.uniform(-5.0, 0.5, ntr)
        da = 10.0 ** lg
        prof = np.zeros((ntr, nd, 10, 60))
        for it in range(ntr):
            w = 0.3 * (1.0 + it) ** 1.5
            for idn in range(mdi[it]):
                for itp in range(10):
                    core = w * (1.0 + 0.05 * idn) * (1.0 + 0.02 * itp)
                    prof[it, idn, itp] = kal[it] / (core ** 2.5 + da ** 2.5) * (1.0 + 0.1 * np.sin(da + itp))
        prof[:, :, :, :2][rng.uniform(size=prof[:, :, :, :2].shape) < 0.02] = 0.0
        out.append(dict(n_lower=n_lower, n_upper_min=n_min, n_upper_max=n_max, density_grid=dens,
                        temp_grid=temps, log_dalpha_grid=lg, max_dens_idx=mdi, k_alpha=kal, profiles=prof))
    return out


def hydrogen_records(wl_lo, wl_hi, wbegin, ratio, series=((1, 2, 12), (2, 3, 25), (3, 4, 20), (4, 5, 12)),
                     deuterium=True, scale=1.0):
    """Unit-19 hydrogen (TYPE -1) and, with `deuterium`, deuterium (TYPE -2,
    0.027 % bluer, 1.5e-4 of the strength) records for the members n -> m of
    each (n, m_lo, m_hi) series that fall in [wl_lo, wl_hi] nm: NCON = n for
    the members past beta (the merged-continuum taper), 0 otherwise; ELO the
    lower level's energy; CGF from a Kramers-like oscillator strength; NBUFF
    the SYNTHE grid index of WLVAC on (wbegin, ratio).  Sorted by wavelength."""
    rh = 109677.583403
    elev = lambda n: 0.0 if n == 1 else 109678.764 - rh / float(n * n)
    out = []
    for n, m_lo, m_hi in series:
        for m in range(m_lo, m_hi):
            wl_h = 1e7 / (rh * (1.0 / n ** 2 - 1.0 / m ** 2))
            for it in ((-1, -2) if deuterium else (-1,)):
                wl = wl_h * (1.0 - 2.72e-4) if it == -2 else wl_h
                if not wl_lo <= wl <= wl_hi:
                    continue
                f = 1.96 * n * (m / ((m - n) * (m + n))) ** 3 * 0.7
                r = np.zeros((), _lib_nlte_dtype())
                r["wlvac"], r["nblo"], r["nbup"], r["itype"] = wl, n, m, it
                r["ncon"] = n if m > n + 2 else 0
                r["elo"] = elev(n)
                r["gf"] = scale * 0.026538 / np.sqrt(np.pi) / C_NM * wl * 2 * n * n * f * (1.5e-4 if it == -2 else 1.0)
                r["nbuff"] = int(np.floor(np.log(wl / wbegin) / np.log(ratio) + 1.5))
                out.append(r)
    recs = np.array(out, _lib_nlte_dtype())
    return recs[np.argsort(recs["wlvac"], kind="stable")]


def _lib_nlte_dtype():
    from . import _lib
    return _lib.NLTE_LINE


def hydrogen_atmosphere(teff=9500.0, logg=4.0, nspec=3):
    """A grey atmosphere's hydrogen inputs for SYNTHE's hydrogen lines:
    xnfdop, dopple [nrhox, nspec] (species 1 = H I), xne, hckt, and the
    depth vectors T, XNFPH(J,1..2), XNFHE(J,1), XNFH2 [nrhox]."""
    from . import surrogate as sg
    m = sg.grey_model(teff, logg)
    pop = sg.populations(m["t"], m["p"], 2.0)
    nr = m["t"].size
    nh1 = pop["nh"] * (1.0 - pop["xh"])
    xnfdop = np.zeros((nr, nspec))
    dopple = np.ones((nr, nspec))
    xnfdop[:, 0] = pop["xnfp"][:, 0] / pop["dopple"][:, 0] / pop["rho"]
    dopple[:, 0] = pop["dopple"][:, 0]
    hckt = sg.HPLANCK * sg.CLIGHT / (sg.KBOL * m["t"])
    return dict(xnfdop=xnfdop, dopple=dopple, xne=pop["xne"], txnxn=np.zeros(nr), hckt=hckt, t=m["t"],
                xnfph1=nh1, xnfph2=pop["nh"] * pop["xh"], xnfhe1=0.085 * pop["nh"],
                xnfh2=1e-5 * nh1 * np.exp(-m["t"] / 1500.0))
