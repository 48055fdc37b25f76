"""The oracle's KAPP H2 sources (oracle/kapp.c) against the reference's tables
and a second, plain-Python restatement, on the CPU.

The restatement is written separately from the C oracle, from
atlas12_modules.f90: PARTFNH2 :22324-22418 (a natural cubic spline through
partfnh2.dat -- here scipy's CubicSpline with natural ends, a different
construction of the same interpolant), EQUILH2 :22437-22469, H2MINOP
:12611-12708, H2COLLOP :16371-16527 (per pair the wavenumber then the
temperature interpolation of log10 k), H2RAOP :17289-17338 and KAPP's totals
:11300-11320.  Known answers: the spline and the CIA table reproduce their
tabulated values at the nodes; H2- free-free is John's coefficient at a
tabulated (lambda, T); H2 Rayleigh goes as lambda^-4 in the red; no H2
density above 20,000 K.
"""
import functools
import math
import os
import sys

import numpy as np
import pytest
from scipy.interpolate import CubicSpline

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import pyoracle as po  # noqa: E402
from atlas12_b200 import surrogate as sg  # noqa: E402

TAB = dict(np.load(os.path.join(ROOT, "tests", "golden", "reference_tables.npz")))
KBOL, HPLANCK, CLIGHT, AMU = 1.380649e-16, 6.62607015e-27, 2.99792458e10, 1.66053906892e-24
CLIGHT_ANGS = 2.99792458e18
PAIRS = ("H2-H2", "H2-He", "H2-H", "H-He")
WAVES = (150.0, 300.0, 500.14, 800.0, 1000.274, 2000.0, 3999.0, 4000.0, 5001.363, 10000.0, 20000.0, 100000.0,
         210057.25, 300000.0, 399000.0, 410000.0)


@pytest.fixture(scope="module")
def kt():
    return po.kapp_tables(TAB)


@pytest.fixture(scope="module")
def h2():
    return po.kapp_h2_tables(TAB)


@functools.lru_cache(maxsize=None)
def atmosphere(teff=3500.0, logg=5.0):
    """A cool dwarf's grey atmosphere with helium at 0.0851 of hydrogen, all
    neutral (the H2 sources matter only where H2 forms)."""
    m = sg.grey_model(teff, logg)
    e = sg.eos(m["t"], m["p"])
    nhe = 0.0851 * e["nh"]
    z = np.zeros_like(nhe)
    return dict(t=m["t"], xne=e["xne"], rho=e["rho"], x1=e["nh"] * (1 - e["xh"]) / 2, x2=e["nh"] * e["xh"],
                x3=nhe, x4=z + 1e-30, x5=z, xnf4=z + 1e-30, xnf3=nhe)


# ---------------------------------------------------------------- restatement
PF_T, PF = TAB["k_pf_h2_t"], TAB["k_pf_h2"]
SPLINE = CubicSpline(PF_T, PF, bc_type="natural")


def partfnh2(t):
    return float(SPLINE(min(PF_T[-1], max(PF_T[0], t))))


def equilh2(t):
    m_h = 1.008 * AMU
    pref = 2.0 ** 1.5 / 4.0 / (2.0 * math.pi * m_h * KBOL / HPLANCK ** 2) ** 1.5
    return partfnh2(t) * pref / t ** 1.5 * math.exp(36118.11 * HPLANCK * CLIGHT / KBOL / t)


def h2minop(wave, t, xne, rho, xnh2m):
    w, tt = TAB["k_h2m_w"], TAB["k_h2m_t"]
    lk = np.log(TAB["k_h2m_k"].reshape(7, 10))
    wl = min(wave, w[-1])
    iw = max([1] + [i for i in range(1, 10) if wl >= w[i - 1]])
    xw = (math.log(wl) - math.log(w[iw - 1])) / (math.log(w[iw]) - math.log(w[iw - 1]))
    kt = lk[:, iw - 1] * (1 - xw) + lk[:, iw] * xw
    it = max([1] + [i for i in range(1, 7) if t >= tt[i - 1]])
    xt = min(1.0, max(0.0, (math.log(t) - math.log(tt[it - 1])) / (math.log(tt[it]) - math.log(tt[it - 1]))))
    return math.exp(kt[it - 1] * (1 - xt) + kt[it] * xt) * xne * KBOL * t * xnh2m / rho


def cia(waveno, t, dens, rho):
    nnu, nu0, dnu = TAB["k_cia_grid"]
    nnu = int(nnu)
    if waveno > nu0 + dnu * (nnu - 1) or waveno <= 0:
        return 0.0
    if waveno <= nu0:
        inu, delnu, dlow = 1, 0.0, 2.0 * math.log10(waveno / nu0)
    else:
        inu = min(int((waveno - nu0) / dnu) + 1, nnu - 1)
        delnu, dlow = (waveno - nu0 - dnu * (inu - 1)) / dnu, 0.0
    s = 0.0
    for ip in range(4):
        nt = TAB["k_cia_nt"][ip]
        temp, tab = TAB["k_cia_temp"][ip, :nt], TAB["k_cia_tab"][ip, :nt]
        if dens[ip] <= 0:
            continue
        tc = max(temp[0], min(temp[-1], t))
        it = max([1] + [i for i in range(1, nt) if tc >= temp[i - 1]])
        wt = (tc - temp[it - 1]) / (temp[it] - temp[it - 1])
        cnu = tab[:, inu - 1] * (1 - delnu) + tab[:, inu] * delnu + dlow
        s += 10.0 ** (cnu[it - 1] * (1 - wt) + cnu[it] * wt) * dens[ip] / rho
    return s


def h2raop(freq):
    w = CLIGHT_ANGS / min(freq, 2.922e15)
    ww = w * w
    return (8.14e-13 + 1.28e-6 / ww + 1.61 / (ww * ww)) / (ww * ww)


# ---------------------------------------------------------------- tests
def test_h2_tables_have_the_reference_shapes():
    assert TAB["k_pf_h2"].size == 200 and TAB["k_pf_h2_t"][0] == 100.0 and TAB["k_pf_h2_t"][-1] == 20000.0
    assert np.all(np.diff(TAB["k_pf_h2_t"]) == 100.0)
    assert list(TAB["k_cia_grid"]) == [800.0, 25.0, 25.0] and list(TAB["k_cia_nt"]) == [39, 55, 4, 10]
    for ip in range(4):
        nt = TAB["k_cia_nt"][ip]
        assert np.all(np.diff(TAB["k_cia_temp"][ip, :nt]) > 0)
        assert np.all(TAB["k_cia_tab"][ip, nt:] == -99.0) and np.all(TAB["k_cia_tab"][ip, :nt] > -99.0)
    assert TAB["k_h2m_k"].size == 70 and TAB["k_h2m_k"][9] == 2.994e-22 and TAB["k_h2m_k"][-1] == 9.217e-23


def test_partition_function_and_equilibrium(h2):
    for t, q in zip(PF_T[::17], PF[::17]):  # the spline passes through its nodes
        assert po.partfnh2(h2, t) == pytest.approx(q, rel=1e-14)
    for t in (50.0, 150.0, 777.0, 2345.6, 5000.0, 9999.0, 19950.0, 30000.0):
        assert po.partfnh2(h2, t) == pytest.approx(partfnh2(t), rel=1e-12), t
        if t >= 150.0:  # below, exp(D0/kT) leaves the double range
            assert po.equilh2(h2, t) == pytest.approx(equilh2(t), rel=1e-12), t


@pytest.mark.parametrize("wave", WAVES)
def test_h2_matches_plain_restatement(kt, h2, wave):
    a = atmosphere()
    freq = 2.99792458e17 / wave
    got = po.kapp_h2(kt, h2, wave, a["t"], a["xne"], a["rho"], a["x1"], a["x2"], a["x3"], a["x4"], a["x5"],
                     a["xnf4"], a["xnf3"])
    for j in range(0, a["t"].size, 5):
        t, xne, rho = a["t"][j], a["xne"][j], a["rho"][j]
        xnhi = a["x1"][j] * 2.0
        eq = equilh2(t)
        xnh2 = xnhi ** 2 * eq if t <= 20000.0 else 0.0
        dens = (xnh2 * xnh2, xnh2 * a["xnf3"][j], xnh2 * xnhi, xnhi * a["xnf3"][j])
        want = dict(ah2min=h2minop(wave, t, xne, rho, xnhi ** 2 * eq), ah2coll=cia(1e7 / wave, t, dens, rho),
                    sigh2=h2raop(freq) * xnh2 / rho)
        for k, v in want.items():
            assert got[k][j] == pytest.approx(v, rel=1e-11, abs=1e-300), (k, wave, j)
    av = got["ah2p"] + got["ahe1"] + got["ahe2"] + got["ahemin"] + got["ah2min"] + got["ah2coll"]
    np.testing.assert_allclose(got["acont"], av + got["ahyd"] + got["ahmin"], rtol=1e-15)
    np.testing.assert_allclose(got["sigmac"], got["sigh"] + got["sighe"] + got["sigel"] + got["sigh2"], rtol=1e-15)


def test_h2_known_answers(kt, h2):
    one = lambda w, t: po.kapp_h2(kt, h2, w, np.array([t]), np.array([1e12]), np.array([1e-6]), np.array([1e16]),
                                  np.array([1e8]), np.array([1e15]), np.array([1e-30]), np.array([0.0]),
                                  np.array([1e-30]), np.array([1e15]))
    # CIA at a grid wavenumber and a tabulated temperature of every pair is the table's value
    t = TAB["k_cia_temp"][0, 5]
    g = one(1e7 / (25.0 + 25.0 * 40), t)
    xnhi = 2e16
    xnh2 = xnhi ** 2 * po.equilh2(h2, t)
    want = 0.0
    for ip, den in enumerate((xnh2 * xnh2, xnh2 * 1e15, xnh2 * xnhi, xnhi * 1e15)):
        nt = TAB["k_cia_nt"][ip]
        temp = TAB["k_cia_temp"][ip, :nt]
        tc = max(temp[0], min(temp[-1], t))
        it = max([0] + [i for i in range(nt - 1) if tc >= temp[i]])
        wt = (tc - temp[it]) / (temp[it + 1] - temp[it])
        v = TAB["k_cia_tab"][ip, it, 40] * (1 - wt) + TAB["k_cia_tab"][ip, it + 1, 40] * wt
        want += 10.0 ** v * den / 1e-6
    assert g["ah2coll"][0] == pytest.approx(want, rel=1e-12)
    # H2- free-free at (5001.363 nm, 5000 K) is KH2M * P_e * n(H2) / rho
    g = one(5001.363, 5000.0)
    xnh2m = xnhi ** 2 * po.equilh2(h2, 5000.0)
    assert g["ah2min"][0] == pytest.approx(TAB["k_h2m_k"][2 * 10 + 5] * 1e12 * KBOL * 5000.0 * xnh2m / 1e-6, rel=1e-12)
    # H2 Rayleigh goes as lambda^-4 in the red; no H2 above 20,000 K
    assert one(4000.0, 3000.0)["sigh2"][0] / one(8000.0, 3000.0)["sigh2"][0] == pytest.approx(16.0, rel=2e-3)
    hot = one(4000.0, 21000.0)
    assert hot["sigh2"][0] == 0.0 and hot["ah2min"][0] > 0.0
    # beyond the CIA grid (25 + 25 x 799 cm^-1) there is no collision-induced absorption
    assert one(1e7 / 20100.0, 3000.0)["ah2coll"][0] == 0.0
