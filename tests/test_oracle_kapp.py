"""The oracle's KAPP hydrogen sources (oracle/kapp.c) against the reference's
tables and a second, plain-Python restatement, on the CPU.

The restatement below is written separately from the C oracle, loop for loop
from atlas12_modules.f90 (HOP :11359-11608, XKARZAS :11635-11804, COULFF
:11995-12196, H2PLOP :12224-12252, HMINOP :12360-12558, HRAYOP :12740-12906,
ELECOP :17212-17222, occupation_prob :22549-22567, KAPP :11202-11324), with
numpy float32 for XKARZAS's REAL(4) arithmetic; the two must agree to
rounding (the H- photodetachment edge at 1643.9 nm is among the cases).
Known answers pin the physics: the 1s photoionization cross-section at
threshold, the Lyman, Balmer and Paschen jumps at their series limits,
Rayleigh scattering going as lambda^-4 in the red, Thomson scattering.
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
from atlas12_b200 import surrogate as sg  # noqa: E402

TAB = dict(np.load(os.path.join(ROOT, "tests", "golden", "reference_tables.npz")))
KBOL, HPLANCK, CLIGHT = 1.380649e-16, 6.62607015e-27, 2.99792458e10
FREQ_RYDH = 109677.583403 * CLIGHT
LIMITS = [109678.764, 27419.659, 12186.462, 6854.871, 4387.113, 3046.604, 2238.320, 1713.713, 1354.044, 1096.776,
          906.426, 761.650, 648.980, 559.579, 487.456]


@pytest.fixture(scope="module")
def kt():
    return po.kapp_tables(TAB)


def atmosphere(teff=5777.0, logg=4.44):
    m = sg.grey_model(teff, logg)
    e = sg.eos(m["t"], m["p"])
    return dict(t=m["t"], xne=e["xne"], rho=e["rho"], x1=e["nh"] * (1 - e["xh"]) / 2, x2=e["nh"] * e["xh"])


# ---------------------------------------------------------------- restatement
def occ(n, xne):
    if n <= 1 or xne <= 0:
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


def xkarzas(freq, n):
    f32 = np.float32
    fl = f32(math.log10(freq))
    if n > 15:
        rn2 = f32(n) * f32(n)
        fq = [None] * 30
        fq[29] = f32(math.log10(FREQ_RYDH / float(rn2)))
        if fl < fq[29]:
            return 0.0
        ek = TAB["k_ekarzas"]
        i = 2
        while i <= 28:
            fq[i] = f32(math.log10(float(f32(ek[i - 1]) + f32(1.0) / rn2) * FREQ_RYDH))
            if fl > fq[i]:
                break
            i += 1
        if i > 28:
            i = 29
        if i == 2:
            fq[1] = f32(math.log10(float(f32(ek[0]) + f32(1.0) / rn2) * FREQ_RYDH))
        xn = TAB["k_xn"].reshape(15, 29)[14]
        x = (fl - fq[i]) / (fq[i - 1] - fq[i]) * (xn[i - 2] - xn[i - 1]) + xn[i - 1]
    else:
        fn = TAB["k_freqn"].reshape(15, 29)[n - 1]
        xn = TAB["k_xn"].reshape(15, 29)[n - 1]
        if fl < fn[28]:
            return 0.0
        i = 2
        while i <= 29 and not fl > fn[i - 1]:
            i += 1
        i = min(i, 29)
        x = (fl - fn[i - 1]) / (fn[i - 2] - fn[i - 1]) * (xn[i - 2] - xn[i - 1]) + xn[i - 1]
    assert isinstance(x, np.float32)
    return math.exp(float(x) * 2.30258509299405)


def linter(xo, yo, x):
    i = 2
    while i <= len(xo) and not x < xo[i - 1]:
        i += 1
    i = min(i, len(xo))
    return yo[i - 2] + (yo[i - 1] - yo[i - 2]) / (xo[i - 1] - xo[i - 2]) * (x - xo[i - 2])


def kapp_point(wave, t, xne, rho, x1, x2):
    """KAPP's hydrogen sources at one (wavelength, depth) in LTE."""
    freq = 2.99792458e17 / wave
    waveno = 1.0e7 / wave
    hkt = HPLANCK / (KBOL * t)
    hckt = hkt * CLIGHT
    tkev = KBOL / 1.602176634e-12 * t
    ehvkt = math.exp(-freq * hkt)
    stim = 1.0 - ehvkt
    bnu = 2.0 * HPLANCK / CLIGHT ** 2 * 1e45 * (freq / 1e15) ** 3 * ehvkt / stim
    elev = TAB["k_hop_elev"]
    H = S = 0.0
    for n in range(15, 0, -1):
        if waveno < LIMITS[n - 1]:
            break
        w = occ(n, xne) if n >= 7 else 1.0
        if n >= 7:
            a = w * xkarzas(freq, n) * 2 * n * n * math.exp(-elev[n - 1] * hckt) * stim
            H, S = H + a, S + a * bnu
        else:
            a = xkarzas(freq, n) * 2 * n * n * math.exp(-elev[n - 1] * hckt) * (1.0 - ehvkt)
            H, S = H + a, S + a * bnu * stim / (1.0 - ehvkt)
    for n in range(16, 81):
        if waveno < 109678.764 / n ** 2:
            continue
        w = occ(n, xne)
        if w < 1e-6:
            continue
        a = w * xkarzas(freq, n) * 2.0 * n ** 2 * math.exp(-(109678.764 - 109677.583403 / n ** 2) * hckt) * stim
        H, S = H + a, S + a * bnu
    for n in range(7, 81):
        w = occ(n, xne)
        if 1.0 - w < 1e-6:
            continue
        a = (1.0 - w) * 2.815e29 / freq ** 3 * 2.0 / n ** 3 * math.exp(-(109678.764 - 109677.583403 / n ** 2) * hckt) * stim
        H, S = H + a, S + a * bnu
    H, S = H * x1 / rho, S * x1 / rho
    # COULFF
    tlog = math.log(t)
    lgam2 = math.log10(FREQ_RYDH * HPLANCK / KBOL) - tlog / 2.30258509299405
    lu = (math.log(freq) - tlog) / 2.30258509299405 + math.log10(HPLANCK / KBOL)
    xi, xj = (lgam2 + 6.0) / 0.2 + 1.0, (lu + 16.0) / 0.2 + 1.0
    i0, j0 = max(1, min(int(xi), 80)), max(1, min(int(xj), 145))
    fi, fj = min(max(xi - i0, 0.0), 1.0), min(max(xj - j0, 0.0), 1.0)
    g = np.log10(TAB["k_gff"]).reshape(146, 81)
    lg = (1 - fi) * ((1 - fj) * g[j0 - 1, i0 - 1] + fj * g[j0, i0 - 1]) + fi * ((1 - fj) * g[j0 - 1, i0] + fj * g[j0, i0])
    a = 3.69196e8 / math.sqrt(t) * 10.0 ** lg / freq * xne / freq * x2 / freq * stim / rho
    ahyd = H + a
    # H2PLOP
    fr, es = TAB["k_h2p_fr"], TAB["k_h2p_es"]
    fl = math.log(freq)
    frp = fr[0] + (fr[1] + (fr[2] + (fr[3] + fr[4] * fl) * fl) * fl) * fl  # Horner, as written
    esp = es[0] + (es[1] + (es[2] + (es[3] + (es[4] + es[5] * freq) * freq) * freq) * freq) * freq
    ah2p = 0.0 if freq > FREQ_RYDH else math.exp(-esp / tkev + frp) * x1 * 2.0 * x2 / rho * stim
    # HMINOP
    ff = TAB["k_hmin_ff"].reshape(22, 11)
    wfflog = np.log(91.134 / TAB["k_hmin_wavek"])
    fftt = [math.exp(linter(wfflog, np.log(ff[:, it] * 1e-26), math.log(wave))) / TAB["k_hmin_thetaff"][it]
            * (0.4342944819032518 / (KBOL / 1.602176634e-12)) * KBOL for it in range(11)]
    theta = 0.4342944819032518 / (KBOL / 1.602176634e-12) / t
    hminff = linter(TAB["k_hmin_thetaff"], fftt, theta) * x1 * 2.0 * xne / rho
    saha = 2.0 * (2.0 * math.pi * 9.1093837139e-28 * KBOL / HPLANCK ** 2) ** 1.5
    xhmin = math.exp(0.75419 / tkev) / (saha * t * math.sqrt(t)) * x1 * xne
    bf = po.map1(TAB["k_hmin_wbf"], TAB["k_hmin_bf"], np.array([wave]))[0] if freq > 1.82365e14 else 0.0
    ahmin = bf * 1e-18 * (1.0 - ehvkt) * xhmin / rho + hminff
    sigel = 6.6524587051e-25 * xne / rho
    return dict(ahyd=ahyd, ah2p=ah2p, ahmin=ahmin, sigel=sigel, acont=ah2p + ahyd + ahmin)


# ---------------------------------------------------------------- tests
def test_tables_have_the_reference_shapes():
    assert TAB["k_freqn"].shape == (435,) and TAB["k_xn"].shape == (435,) and TAB["k_xl"].shape == (1044,)
    assert TAB["k_gff"].shape == (146 * 81,) and np.all(TAB["k_gff"] > 0)
    assert TAB["k_hop_elev"][0] == 0.0 and TAB["k_hop_elev"][1] == 82259.105 and TAB["k_hop_elev"][14] == 109191.313
    # FF is written with REAL(4) literals: every value is a single-precision rounding
    ff = TAB["k_hmin_ff"]
    assert np.array_equal(ff, ff.astype(np.float32).astype(np.float64))
    assert TAB["k_hmin_wbf"][-1] == 1643.908 and TAB["k_hmin_bf"][-1] == 0.0
    q = TAB["k_q_holtsmark"]
    assert q.shape == (150,) and np.all(np.diff(q) > 0) and q[-1] < 1.0


def test_occupation_probability(kt):
    L = po._lib_kapp()
    assert L.orc_occupation_prob(kt, 1, 1e16) == 1.0
    w = [L.orc_occupation_prob(kt, n, 1e14) for n in range(2, 81)]
    assert all(a >= b for a, b in zip(w, w[1:]))  # higher levels dissolve first
    assert L.orc_occupation_prob(kt, 3, 1e8) == 1.0  # low density: bound
    for n in (2, 10, 30):
        for xne in (1e10, 1e13, 1e15):
            assert L.orc_occupation_prob(kt, n, xne) == pytest.approx(occ(n, xne), rel=1e-15, abs=1e-300)


def test_xkarzas_known_answers(kt):
    L = po._lib_kapp()
    nu1 = FREQ_RYDH * 1.0001
    # hydrogen 1s photoionization at threshold: 6.3e-18 cm^2
    assert L.orc_xkarzas(kt, nu1, 1.0, 1, 1) == pytest.approx(6.3e-18, rel=0.01)
    assert L.orc_xkarzas(kt, FREQ_RYDH * 0.999, 1.0, 1, 1) == 0.0  # below the edge
    for n in (1, 2, 5, 15, 16, 40, 80):
        for f in (FREQ_RYDH / n ** 2 * 1.01, 3e15, 1e16):
            assert L.orc_xkarzas(kt, f, 1.0, n, n) == xkarzas(f, n)


@pytest.mark.parametrize("wave", [30.0, 91.0, 91.4, 120.0, 364.0, 365.0, 500.0, 820.0, 822.0, 1600.0, 1700.0,
                                  12000.0, 150000.0])
def test_kapp_matches_plain_restatement(kt, wave):
    at = atmosphere()
    out = po.kapp_hydrogen(kt, wave, at["t"], at["xne"], at["rho"], at["x1"], at["x2"])
    for j in (0, 20, 45, 71):
        ref = kapp_point(wave, at["t"][j], at["xne"][j], at["rho"][j], at["x1"][j], at["x2"][j])
        for k in ("ahyd", "ah2p", "ahmin", "sigel", "acont"):
            assert out[k][j] == pytest.approx(ref[k], rel=1e-12, abs=1e-300), (k, j)


def test_series_jumps_and_thresholds(kt):
    at = atmosphere()
    args = (at["t"], at["xne"], at["rho"], at["x1"], at["x2"])
    j = 50
    for limit in (109678.764, 27419.659, 12186.462):  # Lyman, Balmer, Paschen edges
        blue = po.kapp_hydrogen(kt, 1e7 / limit * (1 - 1e-4), *args)["ahyd"][j]
        red = po.kapp_hydrogen(kt, 1e7 / limit * (1 + 1e-4), *args)["ahyd"][j]
        assert blue > 3 * red
    # H- photodetachment peaks near 850 nm, ten times the free-free part there
    o = po.kapp_hydrogen(kt, 850.0, *args)
    assert o["ahmin"][j] > 10 * po.kapp_hydrogen(kt, 1700.0, *args)["ahmin"][j] * (850.0 / 1700.0) ** 2
    # Rayleigh scattering goes as lambda^-4 far to the red of Lyman alpha
    s1 = po.kapp_hydrogen(kt, 2000.0, *args)["sigh"][j]
    s2 = po.kapp_hydrogen(kt, 4000.0, *args)["sigh"][j]
    assert s1 / s2 == pytest.approx(16.0, rel=0.05)
    # Thomson scattering
    o = po.kapp_hydrogen(kt, 500.0, *args)
    assert np.allclose(o["sigel"], 6.6524587051e-25 * at["xne"] / at["rho"], rtol=1e-15)
    # KAPP's totals: SIGMAC = SIGH + SIGEL, SCONT = BNU where only LTE sources act
    assert np.allclose(o["sigmac"], o["sigh"] + o["sigel"], rtol=1e-15)
