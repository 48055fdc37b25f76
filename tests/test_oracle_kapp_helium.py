"""The oracle's KAPP helium sources (oracle/kapp.c) against the reference's
tables and a second, plain-Python restatement, on the CPU.

The restatement below is written separately from the C oracle, line by line
from atlas12_modules.f90: HE1OP :12939-13143 (with CROSSHE :13160-13236, the
2s/2p fits HE12S1S, HE12S3S, HE12P1P, HE12P3P :13299-13545, and XKARZAS
:11635-11804 in numpy float32 for its REAL(4) arithmetic), HE2OP
:13569-13674, HEMIOP :13716-13833, HERAOP :13918-13941, and KAPP's totals
:11300-11320.  The two must agree to rounding, at wavelengths either side of
every He I and He II threshold the sources test.  Known answers pin the
tables: CROSSHE returns its tabulated values at the grid wavelengths, He-
free-free reproduces John's coefficient at a tabulated (lambda, T) point,
HERAOP's cross-section goes as lambda^-4 in the red.
"""
import functools
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import pyoracle as po  # noqa: E402
from atlas12_b200 import surrogate as sg  # noqa: E402

TAB = dict(np.load(os.path.join(ROOT, "tests", "golden", "reference_tables.npz")))
KBOL, HPLANCK, CLIGHT = 1.380649e-16, 6.62607015e-27, 2.99792458e10
CLIGHT_ANGS = 2.99792458e18
RYDBERG_HE = 109722.277609
COEFF_FF = 3.69196e8
LN10 = 2.30258509299405
KBOL_EV = KBOL / 1.602176634e-12
FREQ_RYDH = 109677.583403 * CLIGHT
GFF_LOG = np.log10(TAB["k_gff"]).reshape(146, 81)
HEM_LOGK = np.log(TAB["k_hem_k"].reshape(12, 17))

# wavelengths (nm): the He II series limits n = 1..9 (22.78, 91.13, 205.06, 364.6, 569.6, 820.3, 1116.5, 1458.2,
# 1845.6 nm), the He I thresholds (50.43 nm and the excited levels), the inner-shell edges, the high-n (1.25408e16
# Hz) and 2.055e14 Hz switches, HERAOP's cap, HEMIOP's table ends (506.441, 210057.25 nm)
WAVES = (5.0, 12.0, 18.0, 22.7, 22.8, 23.9, 24.0, 30.0, 50.3, 50.5, 91.0, 91.2, 205.0, 205.2, 260.0, 312.0,
         331.0, 342.0, 364.5, 364.7, 500.0, 506.441, 569.5, 569.7, 663.0, 744.0, 820.2, 820.4, 1116.4, 1116.6,
         1458.1, 1458.3, 1845.5, 1845.7, 1460.0, 3000.0, 20000.0, 300000.0)


@pytest.fixture(scope="module")
def kt():
    return po.kapp_tables(TAB)


@functools.lru_cache(maxsize=None)
def atmosphere(teff=15000.0, logg=4.0):
    """A hot grey atmosphere with helium at 0.0851 of hydrogen by number, its
    ionisation split by smooth functions of T (any positive populations do for
    parity; these make He II and He III matter)."""
    m = sg.grey_model(teff, logg)
    e = sg.eos(m["t"], m["p"])
    t = m["t"]
    nhe = 0.0851 * e["nh"]
    f1 = 1.0 / (1.0 + np.exp(-(t - 12000.0) / 1500.0))  # He I -> He II
    f2 = 1.0 / (1.0 + np.exp(-(t - 22000.0) / 2500.0))  # He II -> He III
    xnf4 = nhe * f1 * (1.0 - f2)
    return dict(t=t, xne=e["xne"], rho=e["rho"], x1=e["nh"] * (1 - e["xh"]) / 2, x2=e["nh"] * e["xh"],
                x3=nhe * (1.0 - f1), x4=xnf4 / 2.0, x5=nhe * f1 * f2, xnf4=xnf4)


# ---------------------------------------------------------------- restatement
def xkarzas(freq, zeff2, n, l):
    """XKARZAS for n <= 6 (the l-resolved table when l < n)."""
    f32 = np.float32
    fl = f32(math.log10(freq / zeff2))
    fn = TAB["k_freqn"].reshape(15, 29)[n - 1]
    tab = TAB["k_xl"].reshape(6, 6, 29)[n - 1][l] if l < n else TAB["k_xn"].reshape(15, 29)[n - 1]
    if fl < fn[28]:
        return 0.0
    i = 2
    while i <= 29 and not fl > fn[i - 1]:
        i += 1
    i = min(i, 29)
    x = (fl - fn[i - 1]) / (fn[i - 2] - fn[i - 1]) * (tab[i - 2] - tab[i - 1]) + tab[i - 1]
    assert isinstance(x, np.float32)
    return math.exp(float(x) * LN10) / zeff2


def coulff(freq, t, z2log):
    hoverk = HPLANCK / KBOL
    lgam2 = z2log + math.log10(FREQ_RYDH * hoverk) - math.log(t) / LN10
    lu = (math.log(freq) - math.log(t)) / LN10 + math.log10(hoverk)
    xi, xj = (lgam2 + 6.0) / 0.2 + 1.0, (lu + 16.0) / 0.2 + 1.0
    i0, j0 = max(1, min(int(xi), 80)), max(1, min(int(xj), 145))
    fi, fj = max(0.0, min(xi - i0, 1.0)), max(0.0, min(xj - j0, 1.0))
    g = GFF_LOG
    lg = (1 - fi) * ((1 - fj) * g[j0 - 1, i0 - 1] + fj * g[j0, i0 - 1]) + fi * ((1 - fj) * g[j0 - 1, i0] + fj * g[j0, i0])
    return 10.0 ** lg


def crosshe(freq):
    if freq < 5.945209e15:
        return 0.0
    w = CLIGHT_ANGS / freq
    for lo, step, top, tab in ((50.0, 5.0, 92, "k_he_x505"), (20.0, 2.0, 16, "k_he_x50"), (10.0, 1.0, 11, "k_he_x20"),
                               (0.0, 0.5, 21, "k_he_x10")):
        if w > lo or lo == 0.0:
            x = TAB[tab]
            i = min(top, max(2, int(top + 1 - (w - lo) / step)))
            return ((w - (top - i) * step - lo) / step * (x[i - 2] - x[i - 1]) + x[i - 1]) * 1e-18


def knots(name, freq):
    f, x = TAB["k_he%s_f" % name], TAB["k_he%s_x" % name]
    fl = math.log10(freq)
    i = 2
    while i <= 16 and not fl > f[i - 1]:
        i += 1
    i = min(i, 16)
    return math.exp(((fl - f[i - 1]) / (f[i - 2] - f[i - 1]) * (x[i - 2] - x[i - 1]) + x[i - 1]) * LN10)


def fit2(freq, e0, ekc, width, a, ref, p, q):
    wavno = freq / CLIGHT
    eps = 2.0 * ((wavno - e0) / RYDBERG_HE - ekc) / width
    return a * (ref / wavno) ** p * 8.067e-18 * (eps + q) ** 2 / (1.0 + eps ** 2)


def trans_level(freq, n):
    above = freq > 2.4 * RYDBERG_HE * CLIGHT
    if n == 1:
        return crosshe(freq)
    if n == 2:
        if freq < 38454.691 * CLIGHT:
            return 0.0
        return fit2(freq, 38454.691, 2.47898, 0.000780, 0.01521, 470310.0, 3.12, -122.4) if above else knots("2s3s", freq)
    if n == 3:
        if freq < 32033.214 * CLIGHT:
            return 0.0
        return fit2(freq, 32033.214, 2.612316, 0.00322, 0.008175, 484940.0, 2.71, 76.21) if above else knots("2s1s", freq)
    if n == 4:
        return 0.0 if freq < 29223.753 * CLIGHT else knots("2p3p", freq)
    if n == 5:
        if freq < 27175.76 * CLIGHT:
            return 0.0
        if not above:
            return knots("2p1p", freq)
        wavno = freq / CLIGHT
        ek = (wavno - 27175.76) / RYDBERG_HE
        e1s, e1d = 2.0 * (ek - 2.446534) / 0.01037, 2.0 * (ek - 2.59427) / 0.00538
        return 0.0009487 * (466750.0 / wavno) ** 3.69 * 8.067e-18 * (
            (e1s - 29.30) ** 2 / (1.0 + e1s ** 2) + (e1d + 172.4) ** 2 / (1.0 + e1d ** 2))
    zl = {6: (1.236439, 0), 7: (1.102898, 0), 8: (1.045499, 1), 9: (1.001427, 2), 10: (0.9926, 1)}[n]
    return xkarzas(freq, zl[0], 3, zl[1])


def he1op(freq, t, xne, rho, x3, xnf4):
    tkev = KBOL_EV * t
    ehvkt = math.exp(-freq * HPLANCK / (KBOL * t))
    imin = next((n for n in range(1, 11) if TAB["k_he1_freq"][n - 1] <= freq), 0)
    trans = {n: trans_level(freq, n) if 0 < imin <= n else 0.0 for n in range(1, 11)}
    ryd = RYDBERG_HE * CLIGHT
    if imin >= 1:
        for elim, chain in ((527490.06, ((5, 171135.000), (4, 169087.0), (3, 166277.546), (2, 159856.069))),
                            (588451.59, ((10, 186209.471), (9, 186101.0), (8, 185564.0), (7, 184864.0),
                                         (6, 183236.0)))):
            for n, e in chain:
                fhe = (elim - e) * CLIGHT
                if not freq >= fhe:
                    break
                trans[n] = trans[n] + xkarzas(freq, fhe / ryd, 1, 0)
    xr = x3 * (4.0 / 2.0 / 13.595) * tkev / rho
    boltex, exlim = math.exp(-23.730 / tkev) * xr, math.exp(-24.587 / tkev) * xr
    ex = exlim / ehvkt if freq < 2.055e14 else boltex
    he1 = (ex - exlim) * (2.815e29 / freq ** 3)
    if imin > 0:
        for n in range(imin, 11):
            he1 += trans[n] * (math.exp(-TAB["k_he1_chi"][n - 1] / tkev) * TAB["k_he1_g"][n - 1] * x3 / rho)
    if freq >= 1.25408e16:
        for n in range(4, 28):
            bn = math.exp(-24.587 * (1.0 - 1.0 / n ** 2) / tkev) * 4.0 * n ** 2 * x3 / rho
            he1 += xkarzas(freq, 4.0 - 3.0 / n ** 2, 1, 0) * bn
    freet = xne * xnf4 / rho / math.sqrt(t)
    return (he1 + coulff(freq, t, 0.0) * freet * (COEFF_FF / freq ** 3)) * (1.0 - ehvkt)


HE2_LEVELS = (  # n = 9..1: threshold, n^5, g, E_n, Gaunt fit (a, b, c) or None
    (5418.390, 59049.0, 162.0, 433490.46, None), (6857.660, 32768.0, 128.0, 432051.19, None),
    (8956.950, 16807.0, 98.0, 429951.90, None), (12191.437, 7776.0, 72.0, 426717.413, (1.0986, -2.704e13, 1.229e27)),
    (17555.715, 3125.0, 50.0, 421353.135, (1.102, -3.909e13, 2.371e27)),
    (27430.925, 1024.0, 32.0, 411477.925, (1.101, -5.765e13, 4.593e27)),
    (48766.491, 243.0, 18.0, 390142.359, (1.101, -9.863e13, 1.035e28)),
    (109726.529, 32.0, 8.0, 329182.321, (1.105, -2.375e14, 4.077e28)),
    (438908.850, 1.0, 2.0, None, (0.9916, 2.719e13, -2.268e30)))


def he2op(freq, t, xne, rho, x4, x5):
    waveno = freq / CLIGHT
    hckt = HPLANCK * CLIGHT / (KBOL * t)
    stim = 1.0 - math.exp(-freq * HPLANCK / (KBOL * t))
    f3 = 2.815e29 / freq / freq / freq
    xr = x4 / rho
    h = f3 * 16.0 / (438889.068 * hckt) * (math.exp(-max(434519.959, 438908.85 - waveno) * hckt) -
                                          math.exp(-438908.85 * hckt)) * stim * xr
    for thr, n5, g, en, fit in HE2_LEVELS:
        if waveno < thr:
            break
        x = f3 * 16.0 / n5 * (1.0 if fit is None else fit[0] + (fit[1] + fit[2] / freq) / freq)
        h += x * g * (1.0 if en is None else math.exp(-en * hckt)) * stim * xr
    return h + COEFF_FF * 4.0 / math.sqrt(t) * coulff(freq, t, 0.60206) / freq * xne / freq * x5 / freq * stim / rho


def hemiop(wave, t, xne, rho, x3):
    w, tt = TAB["k_hem_w"], TAB["k_hem_t"]
    lk = HEM_LOGK
    wl = min(wave, w[16])
    iw = max([1] + [i for i in range(1, 17) if wl >= w[i - 1]])
    xw = (math.log(wl) - math.log(w[iw - 1])) / (math.log(w[iw]) - math.log(w[iw - 1]))
    kt = lk[:, iw - 1] * (1.0 - xw) + lk[:, iw] * xw
    it = max([1] + [i for i in range(1, 12) if t >= tt[i - 1]])
    xt = (math.log(max(t, 1.0)) - math.log(tt[it - 1])) / (math.log(tt[it]) - math.log(tt[it - 1]))
    xt = max(0.0, min(1.0, xt))
    return math.exp(kt[it - 1] * (1.0 - xt) + kt[it] * xt) * xne * KBOL * t * x3 / rho


def heraop(freq):
    w = CLIGHT_ANGS / min(freq, 5.15e15)
    ww = w * w
    return 5.484e-14 / ww / ww * (1.0 + (2.44e5 + 5.94e10 / (ww - 2.90e5)) / ww) ** 2


# ---------------------------------------------------------------- tests
def test_helium_tables_have_the_reference_shapes():
    assert TAB["k_he1_chi"][0] == 0.0 and TAB["k_he1_chi"][-1] == 23.086
    assert np.all(np.diff(TAB["k_he1_freq"]) < 0) and TAB["k_he1_freq"][0] == 5.945209e15
    assert list(TAB["k_he1_g"]) == [1, 3, 1, 9, 3, 3, 1, 9, 20, 3]
    assert TAB["k_he_x505"].size == 92 and TAB["k_he_x505"][-1] == TAB["k_he_x50"][0]
    assert TAB["k_he_x50"][-1] == TAB["k_he_x20"][0] and TAB["k_he_x20"][-1] == TAB["k_he_x10"][0]
    for k in ("2s1s", "2s3s", "2p1p", "2p3p"):
        assert np.all(np.diff(TAB["k_he%s_f" % k]) < 0)
    assert np.all(np.diff(TAB["k_hem_w"]) > 0) and np.all(np.diff(TAB["k_hem_t"]) > 0)
    assert TAB["k_hem_k"].size == 204 and np.all(TAB["k_hem_k"] > 0)
    # KHEM(IW, IT) at it*17 + iw: the first row is T = 1400 K
    assert TAB["k_hem_k"][0] == 1.21e-27 and TAB["k_hem_k"][16] == 1.3494e-22 and TAB["k_hem_k"][-1] == 2.901e-23


def test_crosshe_known_answers(kt):
    x505 = TAB["k_he_x505"]
    for i in (2, 10, 50, 92):  # WAVE = 50 + (92 - I) * 5 Angstrom lands on X505(I)
        w = 50.0 + (92 - i) * 5.0
        assert po.crosshe(kt, CLIGHT_ANGS / w) == pytest.approx(x505[i - 1] * 1e-18, rel=1e-13)
    assert po.crosshe(kt, 5.9e15) == 0.0  # below the 504 A threshold
    for f in (6.0e15, 1.0e16, 1.1e17, 2.0e17, 5.0e17):
        assert po.crosshe(kt, f) == pytest.approx(crosshe(f), rel=1e-14)


@pytest.mark.parametrize("wave", WAVES)
def test_helium_matches_plain_restatement(kt, wave):
    a = atmosphere()
    freq = 2.99792458e17 / wave
    got = po.kapp(kt, wave, a["t"], a["xne"], a["rho"], a["x1"], a["x2"], a["x3"], a["x4"], a["x5"], a["xnf4"])
    for j in range(0, a["t"].size, 7):
        args = (a["t"][j], a["xne"][j], a["rho"][j])
        want = dict(ahe1=he1op(freq, *args, a["x3"][j], a["xnf4"][j]), ahe2=he2op(freq, *args, a["x4"][j], a["x5"][j]),
                    ahemin=hemiop(wave, *args, a["x3"][j]), sighe=heraop(freq) * a["x3"][j] / a["rho"][j])
        for k, v in want.items():
            assert got[k][j] == pytest.approx(v, rel=1e-11, abs=1e-300), (k, wave, j)


def test_totals_take_the_helium_sources(kt):
    a = atmosphere()
    for wave in (22.0, 40.0, 300.0, 2000.0):
        h = po.kapp_hydrogen(kt, wave, a["t"], a["xne"], a["rho"], a["x1"], a["x2"])
        g = po.kapp(kt, wave, a["t"], a["xne"], a["rho"], a["x1"], a["x2"], a["x3"], a["x4"], a["x5"], a["xnf4"])
        for k in ("ahyd", "shyd", "ah2p", "ahmin", "shmin", "sigh", "sigel"):
            np.testing.assert_array_equal(g[k], h[k])
        av = g["ah2p"] + g["ahe1"] + g["ahe2"] + g["ahemin"]
        np.testing.assert_allclose(g["acont"], av + g["ahyd"] + g["ahmin"], rtol=1e-15)
        np.testing.assert_allclose(g["sigmac"], g["sigh"] + g["sighe"] + g["sigel"], rtol=1e-15)
        assert np.all(g["acont"] >= h["acont"])


def test_helium_physics(kt):
    a = atmosphere()
    j = 40
    one = lambda w: po.kapp(kt, w, a["t"][j:j + 1], a["xne"][j:j + 1], a["rho"][j:j + 1], a["x1"][j:j + 1],
                            a["x2"][j:j + 1], a["x3"][j:j + 1], a["x4"][j:j + 1], a["x5"][j:j + 1],
                            a["xnf4"][j:j + 1])
    # He I ground-state edge at 50.43 nm and He II Lyman edge at 22.78 nm
    assert one(50.3)["ahe1"][0] > 10.0 * one(50.6)["ahe1"][0]
    assert one(22.7)["ahe2"][0] > 10.0 * one(22.9)["ahe2"][0]
    # HERAOP goes as lambda^-4 in the red
    r = one(4000.0)["sighe"][0] / one(8000.0)["sighe"][0]
    assert r == pytest.approx(16.0, rel=2e-3)
    # He- free-free at a tabulated (lambda, T) point is John's coefficient * P_e * n(He I) / rho
    t0 = np.array([5040.0])
    g = po.kapp(kt, 911.55, t0, np.array([1e12]), np.array([1e-8]), np.array([1e15]), np.array([1e10]),
                np.array([1e14]), np.array([1e8]), np.array([1e4]), np.array([2e8]))
    assert g["ahemin"][0] == pytest.approx(TAB["k_hem_k"][7 * 17 + 4] * 1e12 * KBOL * 5040.0 * 1e14 / 1e-8, rel=1e-12)
