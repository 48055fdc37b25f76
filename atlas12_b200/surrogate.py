"""Synthetic physics surrogate for the parts of ATLAS12/SYNTHE outside the hot path.

The hot path (line opacity, JOSH transfer, frequency integrals, T-correction)
consumes per-depth populations and per-frequency continuum opacities that the
reference computes with its EOS (NMOLEC / COMPUTE_ALL_POPS) and continuum
library (KAPP, ~40 sources).  Those are out of scope here; this module stands
in for them with a small, smooth, physically-shaped model:

* composition: hydrogen plus 18 metals (solar-like abundances) and 5 diatomic
  molecules; two ionisation stages per metal from a Saha balance with constant
  partition functions; molecules from a Guldberg-Waage-like T scaling;
* electron density: hydrogen + metal ionisation (Saha), ideal gas;
* continuum absorption: H- bound-free and free-free, H I bound-free from
  n = 1, 2, 3 (Lyman, Balmer, Paschen edges), metal bound-free from the
  neutral ground states (edges at 1239.84/chi nm), all with simple analytic
  cross-section shapes; scattering: Thomson + H I Rayleigh;
* Rosseland mean: tabulated from the same continuum on a (log T, log P) grid.

Every function is vectorised numpy and deterministic; the device kernels in
csrc/atlas_surrogate.cuh evaluate the same continuum formula.
"""
import numpy as np

KBOL = 1.380649e-16
HPLANCK = 6.62607015e-27
CLIGHT = 2.99792458e10
CLIGHT_NMS = 2.99792458e17
AMU = 1.66053906892e-24
EV_ERG = 1.602176634e-12
EV_CM = 8065.543937  # 1 eV in cm^-1
SIGMA_SB = 5.670374419e-5

# (Z, mass [amu], chi_I [eV], log eps, U_I, U_II)
METALS = np.array([
    (26, 55.845, 7.902, 7.50, 25.0, 40.0),
    (22, 47.867, 6.828, 4.95, 30.0, 50.0),
    (24, 51.996, 6.767, 5.64, 10.0, 7.0),
    (28, 58.693, 7.640, 6.22, 30.0, 10.0),
    (20, 40.078, 6.113, 6.34, 1.0, 2.0),
    (23, 50.942, 6.746, 3.93, 35.0, 30.0),
    (27, 58.933, 7.881, 4.99, 30.0, 25.0),
    (25, 54.938, 7.434, 5.43, 6.0, 7.0),
    (21, 44.956, 6.561, 3.15, 10.0, 20.0),
    (12, 24.305, 7.646, 7.60, 1.0, 2.0),
    (14, 28.086, 8.152, 7.51, 9.0, 6.0),
    (11, 22.990, 5.139, 6.24, 2.0, 1.0),
    (13, 26.982, 5.986, 6.45, 6.0, 1.0),
    (6, 12.011, 11.260, 8.43, 9.0, 6.0),
    (8, 15.999, 13.618, 8.69, 9.0, 4.0),
    (7, 14.007, 14.534, 7.83, 9.0, 9.0),
    (39, 88.906, 6.217, 2.21, 10.0, 15.0),
    (40, 91.224, 6.634, 2.58, 30.0, 40.0),
])
# (slot, mass, log abundance relative to H at 5000 K, T exponent)
MOLECULES = np.array([
    (41, 13.02, -7.0, 8.0),   # CH
    (42, 26.02, -8.0, 10.0),  # CN
    (43, 28.01, -4.5, 6.0),   # CO
    (44, 17.01, -7.5, 9.0),   # OH
    (45, 63.87, -9.0, 14.0),  # TiO
])
MW6 = 139 * 6  # SYNTHE's flattened species axis (mw*6)
MBF_SIGMA = 2.0e-17  # metal ground-state photo-ionisation cross-section at the edge (cm^2)
# Fraction of each metal / molecule population that the ATLAS12 synthetic line
# list draws on.  The ATLAS12 model here is purely radiative (the reference's
# convective flux, CONVEC, is outside the hot path), and a radiative solar
# model blanketed by 500,000 full-strength synthetic lines has no radiative-
# equilibrium solution reachable from the grey start: the deep layers heat
# without bound.  At 1/100 the grey start converges to max|FLXERR| <= 0.1 %
# in about 30 iterations.  SYNTHE's synthetic atmospheres use the full
# populations (line_pop = 1).
ATLAS_LINE_POP = 0.01


def nelion(z, ion_stage):
    """SYNTHE species index (nelem-1)*6 + ion stage (1 = neutral), 1-based."""
    return (int(z) - 1) * 6 + int(ion_stage)


def mol_nelion(slot):
    return (int(slot) - 1) * 6 + 1


def species_list():
    """All (nelion, mass) pairs the surrogate populates."""
    out = [(1, 1.008), (2, 1.008)]
    for z, m, *_ in METALS:
        out.append((nelion(z, 1), m))
        out.append((nelion(z, 2), m))
    for slot, m, *_ in MOLECULES:
        out.append((mol_nelion(slot), m))
    return out


def _saha(t, ne, chi, u1, u2):
    """n_II / n_I."""
    return 2.4147e15 * t ** 1.5 / np.maximum(ne, 1.0) * (2.0 * u2 / u1) * np.exp(-chi * EV_ERG / (KBOL * t))


def eos(t, p, mh=0.0):
    """Ideal-gas surrogate EOS -> dict(ntot, nh, xne, rho, xh) per depth.
    mh = [M/H]: every metal abundance scaled by 10**mh."""
    t = np.asarray(t, dtype=np.float64)
    p = np.asarray(p, dtype=np.float64)
    ntot = p / (KBOL * t)
    eps = 10.0 ** (METALS[:, 3] - 12.0 + mh)
    ne = np.maximum(ntot * 1e-4, 1.0)
    for _ in range(30):  # fixed-point on n_e
        nh = ntot / (1.1 + ne / ntot)
        rh = _saha(t, ne, 13.598, 2.0, 1.0)
        xh = rh / (1.0 + rh)
        rm = _saha(t[:, None], ne[:, None], METALS[None, :, 2], METALS[None, :, 4], METALS[None, :, 5])
        xm = rm / (1.0 + rm)
        ne_new = nh * xh + nh * np.sum(eps[None, :] * xm, axis=1) + 1.0
        ne = np.sqrt(ne * ne_new)
    nh = ntot / (1.1 + ne / ntot)
    rho = nh * 1.4 * AMU
    return dict(ntot=ntot, nh=nh, xne=ne, rho=rho, xh=xh, mh=mh)


def populations(t, p, vturb_kms, line_pop=1.0, mh=0.0):
    """Per-depth species number densities / partition function (XNFPEL analogue)
    and Doppler widths.  Returns dict of [nrhox, MW6] arrays plus eos fields.
    line_pop scales the metal and molecule entries (ATLAS_LINE_POP for the
    ATLAS12 model, 1 for SYNTHE); hydrogen and the EOS are unaffected."""
    t = np.asarray(t, dtype=np.float64)
    e = eos(t, p, mh)
    nr = t.size
    xnfp = np.zeros((nr, MW6))
    dop = np.zeros((nr, MW6))
    vt = np.broadcast_to(np.asarray(vturb_kms, dtype=np.float64) * 1e5, (nr,))

    def _dop(m):
        return np.sqrt(2.0 * KBOL * t / (m * AMU) + vt ** 2) / CLIGHT

    xnfp[:, 0] = e["nh"] * (1 - e["xh"]) / 2.0
    xnfp[:, 1] = e["nh"] * e["xh"]
    dop[:, 0] = dop[:, 1] = _dop(1.008)
    for z, m, chi, leps, u1, u2 in METALS:
        r = _saha(t, e["xne"], chi, u1, u2)
        n = e["nh"] * 10.0 ** (leps - 12.0 + mh)
        i1, i2 = nelion(z, 1) - 1, nelion(z, 2) - 1
        xnfp[:, i1] = n / (1.0 + r) / u1 * line_pop
        xnfp[:, i2] = n * r / (1.0 + r) / u2 * line_pop
        dop[:, i1] = dop[:, i2] = _dop(m)
    for slot, m, labund, texp in MOLECULES:
        i = mol_nelion(slot) - 1
        xnfp[:, i] = e["nh"] * 10.0 ** labund * np.minimum((5000.0 / t) ** texp, 1e6) / 1000.0 * line_pop
        dop[:, i] = _dop(m)
    e.update(xnfp=xnfp, dopple=dop)
    return e


def continuum_opacity(wave_nm, t, p, e=None, mh=0.0):
    """Surrogate continuum -> (kappa_abs, sigma) in cm^2/g, shape [nwave, nrhox].
    e: an eos()/populations() result (carries its [M/H]); else eos(t, p, mh)."""
    w = np.asarray(wave_nm, dtype=np.float64)[:, None]
    t = np.asarray(t, dtype=np.float64)[None, :]
    if e is None:
        e = eos(t[0], p, mh)
    mh = e.get("mh", 0.0)
    nh = e["nh"][None, :]
    ne = e["xne"][None, :]
    rho = e["rho"][None, :]
    xh = e["xh"][None, :]
    nh1 = nh * (1.0 - xh)
    theta = 5040.0 / t
    pe = ne * KBOL * t
    # H- bound-free: cross-section shape peaking near 850 nm, threshold 1642 nm
    x = np.clip(w / 1642.0, 0.0, 1.0)
    abf = 4.0e-17 * 6.0 * (x * np.sqrt(x)) * ((1.0 - x) * np.sqrt(1.0 - x)) * 4.0
    khm = 4.158e-10 * abf * pe * theta ** 2.5 * 10.0 ** (0.754 * theta) * nh1
    # H- free-free ~ lambda^2
    kff = 1.0e-26 * pe * nh1 * (w / 1000.0) ** 2 * (0.5 + 1.5 * theta)
    # H I bound-free from n = 1, 2, 3 (hydrogenic nu^-3 above each edge)
    kh = np.zeros(np.broadcast(w, t).shape)
    for n, edge in ((1, 91.175), (2, 364.70), (3, 820.6)):
        pop = nh1 * 2.0 * n * n * np.exp(-13.598 * (1.0 - 1.0 / (n * n)) * EV_ERG / (KBOL * t)) / 2.0
        sig = np.where(w <= edge, 7.9e-18 / n ** 5 * (w / edge) ** 3 * n ** 3 / 1.0, 0.0)
        kh = kh + pop * sig
    # metal bound-free from the neutral ground states, edges at 1239.84/chi nm
    kmet = np.zeros(np.broadcast(w, t).shape)
    for z, m, chi, leps, u1, u2 in METALS:
        r = _saha(t[0], e["xne"], chi, u1, u2)[None, :]
        n1 = nh * 10.0 ** (leps - 12.0 + mh) / (1.0 + r)
        edge = 1239.84198 / chi
        kmet = kmet + np.where(w <= edge, n1 * MBF_SIGMA * (w / edge) ** 3, 0.0)
    # Thomson + Rayleigh(H I)
    sray = 5.8e-24 * (121.6 / np.maximum(w, 125.0)) ** 4 * nh1
    sigma = (6.6524587051e-25 * ne + sray) / rho
    kabs = (khm + kff + kh + kmet) / rho + 1e-12
    return kabs, sigma


def planck_dbdt(wave_nm, t):
    """dB_nu/dT; 0 where h nu / kT overflows."""
    nu = CLIGHT_NMS / np.asarray(wave_nm)[:, None]
    x = HPLANCK * nu / (KBOL * np.asarray(t)[None, :])
    with np.errstate(over="ignore", invalid="ignore"):
        b = 2.0 * HPLANCK * nu ** 3 / CLIGHT ** 2 / np.expm1(x)
        d = b * x / np.asarray(t)[None, :] * np.exp(x) / np.expm1(x)
    return np.where(np.isfinite(d), d, 0.0)


class RossTable:
    """log kappa_Ross on a (log T, log P) grid from the surrogate continuum
    (the ROSSTAB analogue consumed by TTAUP)."""

    def __init__(self, lt0=np.log10(1000.0), lt1=np.log10(60000.0), lp0=-4.0, lp1=10.0, nt=104, np_=112,
                 mh=0.0, nwave=2400):
        self.lt = np.linspace(lt0, lt1, nt)
        self.lp = np.linspace(lp0, lp1, np_)
        wave = np.geomspace(9.0, 160000.0, nwave)
        nu = CLIGHT_NMS / wave
        dnu = np.abs(np.gradient(nu))
        tab = np.zeros((nt, np_))
        for i, lt in enumerate(self.lt):
            tt = np.full(np_, 10.0 ** lt)
            pp = 10.0 ** self.lp
            ka, sg = continuum_opacity(wave, tt, pp, mh=mh)
            d = planck_dbdt(wave, tt) * dnu[:, None]
            tab[i] = np.log10(np.sum(d, axis=0) / np.sum(d / (ka + sg), axis=0))
        self.table = tab

    def __call__(self, t, p):
        t = np.atleast_1d(np.asarray(t, dtype=np.float64))
        p = np.atleast_1d(np.asarray(p, dtype=np.float64))
        x = (np.log10(t) - self.lt[0]) / (self.lt[1] - self.lt[0])
        y = (np.log10(np.maximum(p, 1e-30)) - self.lp[0]) / (self.lp[1] - self.lp[0])
        x = np.clip(x, 0, self.lt.size - 1.000001)
        y = np.clip(y, 0, self.lp.size - 1.000001)
        i, j = x.astype(int), y.astype(int)
        fx, fy = x - i, y - j
        T = self.table
        v = (T[i, j] * (1 - fx) * (1 - fy) + T[i + 1, j] * fx * (1 - fy) + T[i, j + 1] * (1 - fx) * fy +
             T[i + 1, j + 1] * fx * fy)
        return 10.0 ** v


def grey_model(teff, logg, nrhox=72, tau1lg=-6.875, steplg=0.125, ross=None):
    """Eddington grey start: T^4 = 3/4 Teff^4 (tau + 2/3) on the standard
    Rosseland grid TAUSTD(J) = 10**(TAU1LG + (J-1)*STEPLG) (the reference's
    TAUSTD, atlas12_modules.f90:1792), P from dP/dtau = g / kappa_R
    integrated in ln tau (RK4) with the surrogate Rosseland table."""
    ross = ross or RossTable()
    g = 10.0 ** logg
    tau = 10.0 ** (tau1lg + steplg * np.arange(nrhox))
    t = (0.75 * teff ** 4 * (tau + 2.0 / 3.0)) ** 0.25

    def tfun(tt):
        return (0.75 * teff ** 4 * (tt + 2.0 / 3.0)) ** 0.25

    def f(lnt, lnp):
        tt = np.exp(lnt)
        pp = np.exp(lnp)
        return g * tt / (ross(tfun(tt), pp)[0] * pp)

    lnp = np.log(g * tau[0] / 0.01)
    for _ in range(50):  # self-consistent surface value
        lnp = np.log(g * tau[0] / ross(t[0], np.exp(lnp))[0])
    p = np.zeros(nrhox)
    p[0] = np.exp(lnp)
    for j in range(1, nrhox):
        h = np.log(tau[j] / tau[j - 1])
        x0 = np.log(tau[j - 1])
        sub = 4
        hh = h / sub
        for s in range(sub):
            xs = x0 + s * hh
            k1 = f(xs, lnp)
            k2 = f(xs + hh / 2, lnp + hh / 2 * k1)
            k3 = f(xs + hh / 2, lnp + hh / 2 * k2)
            k4 = f(xs + hh, lnp + hh * k3)
            lnp = lnp + hh / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        p[j] = np.exp(lnp)
    rhox = p / g
    return dict(teff=float(teff), logg=float(logg), grav=g, tauros=tau, t=t, p=p, rhox=rhox, ross=ross)
