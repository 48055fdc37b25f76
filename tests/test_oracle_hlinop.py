"""The oracle's HLINOP (oracle/kapp.c) against a second, plain-Python
restatement, on the CPU.

The restatement is written separately from the C oracle, line by line from
atlas12_modules.f90: HLINOP :17381-17503 (the series n = int(sqrt(nu_Lyman /
nu)), the members around the frequency, the dissolved-level cut, the
Paschen-alpha term of the Brackett series), STARK :17528-17659,
STARK_MMM :17854-18106 (on seeded Stehle-format tables of the published
shapes) and hydrogen_f_value :17760-17829.  Known answers: nothing outside
the four series or redward of the Lyman (2e15 Hz) and Balmer (4.44e14 Hz)
cuts; in LTE SHLINE is the Planck function; the Stark wings fall off as
Delta-nu^-2.5 past the tables.
"""
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import pyoracle as po  # noqa: E402
from atlas12_b200 import synthetic  # noqa: E402

TAB = dict(np.load(os.path.join(ROOT, "tests", "golden", "reference_tables.npz")))
KBOL, HPLANCK, CLIGHT = 1.380649e-16, 6.62607015e-27, 2.99792458e10
CLIGHT_ANGS = 2.99792458e18
RYDH = 109677.583403
NU_LYMAN = RYDH * CLIGHT
A0 = 0.0265384
STEHLE = synthetic.stehle_tables()
# wavelengths (nm): Lyman members and its 150 nm cut, the Balmer lines, limit and 675.6 nm cut,
# Paschen and Brackett lines and limits
WAVES = (91.5, 93.0, 97.0, 102.5, 121.6, 149.0, 151.0, 365.0, 366.0, 383.5, 397.0, 410.2, 434.0, 486.1, 656.3,
         675.0, 676.5, 821.0, 850.0, 954.6, 1005.0, 1094.0, 1282.0, 1459.0, 1500.0, 1875.0, 2166.0, 2280.0)


@pytest.fixture(scope="module")
def kt():
    return po.kapp_tables(TAB)


@pytest.fixture(scope="module")
def stehle():
    return po.stehle_structs(STEHLE)


def depths():
    rng = np.random.default_rng(3)
    n = 24
    t = np.geomspace(3000.0, 60000.0, n)
    xne = np.geomspace(1e9, 3e17, n)
    rho = np.geomspace(1e-11, 1e-5, n)
    x1 = rho / 1.67e-24 * rng.uniform(0.05, 0.5, n)
    return t, xne, rho, x1


# ---------------------------------------------------------------- restatement
def occ(n, xne):
    if n <= 1:
        return 1.0
    beta = 8.798905203085208e14 / (float(n) ** 5 * xne ** (2.0 / 3.0))
    if beta <= 0.01:
        return 0.0
    if beta >= 50.0:
        return 1.0
    idx_f = (math.log10(beta) + 2.0) / 2.4825302042523617e-02
    idx = max(0, min(148, int(idx_f)))
    q = TAB["k_q_holtsmark"]
    return q[idx] + (idx_f - idx) * (q[idx + 1] - q[idx])


def f_value(n, m):
    tabs = {1: "k_gf_lyman", 2: "k_gf_balmer", 3: "k_gf_paschen", 4: "k_gf_brackett"}
    g = TAB[tabs[n]]
    if m - n <= g.size:
        gf = g[m - n - 1]
    else:
        gf = 1.9603 * n ** 2 / (m ** 3 * (1.0 / n ** 2 - 1.0 / m ** 2) ** 3) * 0.80
    return gf / (2.0 * n ** 2)


def exint(x):
    return -math.log(x) - 0.57516 + (0.97996 + (-0.21654 + (0.033572 + (-0.0029222 + 1.05439e-4 * x) * x) * x) * x) * x


def stark(n, m, freq, t, xne):
    f0 = 1.25e-9 * xne ** (2.0 / 3.0)
    hkt = HPLANCK / (KBOL * t)
    x = n / m
    nn, mm = float(n * n), float(m * m)
    knm = TAB["k_stark_knm"].reshape(4, 5)[n - 1, m - n - 1] if m - n <= 5 else 5.5e-5 * (nn * mm) ** 2 / (mm - nn)
    fs = TAB["k_stark_f"].reshape(4, 10)[n - 1]
    fnm = fs[m - n - 1] if m - n <= 10 else fs[9] * ((20.0 * n + 100.0) / ((n + 10.0) * m * (1.0 - x * x))) ** 3
    freqnm = NU_LYMAN * (1.0 / nn - 1.0 / mm)
    de = abs(freq - freqnm)
    dbeta = CLIGHT_ANGS / freqnm ** 2 / f0 / knm
    beta = dbeta * de
    y1 = mm * de * hkt / 2.0
    y2 = math.pi ** 2 / 2.0 / A0 / CLIGHT * de ** 2 / xne
    qstat = 1.5 + 0.5 * (y1 ** 2 - 1.384) / (y1 ** 2 + 1.384)
    impact = 0.0
    if y1 < 8.0 and y1 < y2:
        impact = 1.438 * math.sqrt(y1 * (1.0 - x * x)) * (0.4 * math.exp(-y1) + exint(y1) -
                                                           0.5 * (exint(y2) if y2 <= 8.0 else 0.0))
    if beta <= 20.0:
        prof, ratio = 8.0 / (80.0 + beta ** 3), qstat + impact
    else:
        prof = 1.5 / beta / beta / math.sqrt(beta)
        dioi = 6.28 * 1.48e-25 * (2.0 * mm * NU_LYMAN / de) * xne * (
            math.sqrt(2.0 * mm * NU_LYMAN / de) * (1.3 * qstat + 0.30 * impact) - 3.9 * NU_LYMAN * hkt)
        ratio = qstat * min(1.0 + dioi, 1.25) + impact
    return A0 * fnm * prof * dbeta * ratio


def bracket(grid, v):
    """The first i (0-based) with v <= grid[i + 1], clamped to len - 2."""
    for i in range(len(grid) - 1):
        if v <= grid[i + 1]:
            return i
    return len(grid) - 2


def stark_mmm(n, m, freq, t, xne, use):
    if not use:
        return stark(n, m, freq, t, xne)
    s = STEHLE[n - 1]
    if not s["n_upper_min"] <= m <= s["n_upper_max"]:
        return stark(n, m, freq, t, xne)
    tr = m - s["n_upper_min"]
    dg, tg, ag = s["density_grid"], s["temp_grid"], s["log_dalpha_grid"]
    if xne > dg[-1] or t < tg[0] * 0.5 or t > tg[-1] * 2.0:
        return stark(n, m, freq, t, xne)
    ne = min(xne, dg[s["max_dens_idx"][tr] - 1])
    lam0 = 1e8 / RYDH * (n * m) ** 2 / ((m - n) * (m + n))
    f0 = 1.25e-9 * ne ** (2.0 / 3.0)
    dalpha = lam0 ** 2 / CLIGHT_ANGS * abs(freq - CLIGHT_ANGS / lam0) / f0
    norm = A0 * f_value(n, m) * lam0 ** 2 / (CLIGHT_ANGS * f0)
    i_d, i_t = bracket(dg, ne), bracket(tg, t)
    fd = min(1.0, max(0.0, (math.log10(ne) - math.log10(dg[i_d])) / (math.log10(dg[i_d + 1]) - math.log10(dg[i_d]))))
    ft = min(1.0, max(0.0, (math.log(t) - math.log(tg[i_t])) / (math.log(tg[i_t + 1]) - math.log(tg[i_t]))))
    ia, ib, fa = 0, 0, 0.0
    if dalpha > 0:
        lda = math.log10(dalpha)
        if lda >= ag[-1]:
            return norm * s["k_alpha"][tr] / dalpha ** 2.5
        if lda > ag[0]:
            ia = bracket(ag, lda)
            ib = ia + 1
            fa = min(1.0, max(0.0, (lda - ag[ia]) / (ag[ib] - ag[ia])))
    p = s["profiles"][tr]
    v = np.array([[[p[d, tt, ia], p[d, tt, ib]] for tt in (i_t, i_t + 1)] for d in (i_d, i_d + 1)])
    lg = bool(np.all(v > 0))
    if lg:
        v = np.log(v)
    va = v[..., 0] + fa * (v[..., 1] - v[..., 0])
    vt = va[:, 0] + ft * (va[:, 1] - va[:, 0])
    val = vt[0] + fd * (vt[1] - vt[0])
    return norm * max(math.exp(val) if lg else val, 0.0)


def hlinop_point(wave, t, xne, rho, x1, use):
    freq = 2.99792458e17 / wave
    n = int(math.sqrt(NU_LYMAN / freq))
    if n == 0 or n > 4 or (n == 1 and freq < 2.0e15) or (n == 2 and freq < 4.44e14):
        return 0.0, 0.0
    hkt = HPLANCK / (KBOL * t)
    ehvkt = math.exp(-freq * hkt)
    bnu = 2.0 * HPLANCK / CLIGHT ** 2 * 1e45 * (freq / 1e15) ** 3 * ehvkt / (1.0 - ehvkt)
    bolt = lambda k: math.exp(-(13.595 - 13.595 / k ** 2) / (KBOL / 1.602176634e-12 * t)) * 2.0 * k ** 2 * x1 / rho
    m1 = math.floor(math.sqrt(NU_LYMAN / (NU_LYMAN / n ** 2 - freq)) + 0.5)  # NINT
    m2 = m1 + 1
    m1 = max(m1, n + 1)
    h = 0.0
    if m1 > 6:
        if m1 > 80 or occ(m1, xne) < 1e-3:
            return 0.0, bnu
        m1, m2 = m1 - 1, m2 + 3
        if n >= 4 and m1 <= 8:
            h = stark_mmm(3, 4, freq, t, xne, use) * (1.0 - ehvkt) * bolt(3)
    for m in range(m1, m2 + 1):
        w = occ(m, xne) if m <= 80 else 0.0
        h += w * stark_mmm(n, m, freq, t, xne, use) * (1.0 - ehvkt) * bolt(n)
    return h, bnu


# ---------------------------------------------------------------- tests
def test_hlinop_tables_have_the_reference_shapes():
    assert TAB["k_gf_lyman"][0] == 0.8324 and TAB["k_gf_balmer"][0] == 5.126 and TAB["k_gf_brackett"][-1] == 2.092
    assert TAB["k_stark_knm"].reshape(4, 5)[0, 0] == 0.000356 and TAB["k_stark_knm"].reshape(4, 5)[3, 4] == 1.46
    assert TAB["k_stark_f"].reshape(4, 10)[0, 0] == 0.1387 and TAB["k_stark_f"].reshape(4, 10)[3, 9] == 0.003375


@pytest.mark.parametrize("use_stehle", [False, True])
@pytest.mark.parametrize("wave", WAVES)
def test_hlinop_matches_plain_restatement(kt, stehle, wave, use_stehle):
    t, xne, rho, x1 = depths()
    ah, sh = po.hlinop(kt, wave, t, xne, rho, x1, stehle=stehle[0] if use_stehle else None)
    for j in range(t.size):
        h, s = hlinop_point(wave, t[j], xne[j], rho[j], x1[j], use_stehle)
        assert ah[j] == pytest.approx(h, rel=1e-11, abs=1e-300), (wave, j)
        if ah[j] > 0 or s == 0.0:
            assert sh[j] == pytest.approx(s, rel=1e-11, abs=1e-300), (wave, j)


def test_hlinop_known_answers(kt, stehle):
    t, xne, rho, x1 = depths()
    for wave in (150.5, 680.0, 3000.0, 10000.0):  # past the Lyman and Balmer cuts, beyond Brackett
        ah, sh = po.hlinop(kt, wave, t, xne, rho, x1)
        assert not np.any(ah) and not np.any(sh)
    # LTE: SHLINE is the Planck function wherever there is line opacity
    ah, sh = po.hlinop(kt, 656.3, t, xne, rho, x1, stehle=stehle[0])
    freq = 2.99792458e17 / 656.3
    ehvkt = np.exp(-freq * HPLANCK / (KBOL * t))
    bnu = 2.0 * HPLANCK / CLIGHT ** 2 * 1e45 * (freq / 1e15) ** 3 * ehvkt / (1.0 - ehvkt)
    np.testing.assert_allclose(sh[ah > 0], bnu[ah > 0], rtol=1e-12)
    # past the tables the Stehle wing is k_alpha Delta-alpha^-2.5: 2.5 decades per decade of Delta-nu
    lam0 = 1e8 / RYDH * 36.0 / 5.0
    nu0 = CLIGHT_ANGS / lam0
    fa, fb = nu0 * 1.3, nu0 * 1.4  # Delta-alpha above 10^5.5 at Ne = 1e10
    ra = po.stark_mmm(kt, 2, 3, fa, 8000.0, 1e10, stehle[0]) / po.stark_mmm(kt, 2, 3, fb, 8000.0, 1e10, stehle[0])
    assert ra == pytest.approx(((fb - nu0) / (fa - nu0)) ** 2.5, rel=1e-9)
