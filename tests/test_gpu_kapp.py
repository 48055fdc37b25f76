"""KAPP's hydrogen continuum sources on the GPU (atlasgpu_atlas_kapp_hydrogen,
through the C ABI) against the CPU oracle (oracle/kapp.c), which restates
HOP, XKARZAS, COULFF, H2PLOP, HMINOP, HRAYOP, ELECOP and KAPP's totals
(atlas12_modules.f90:11202-12906, :17212-17222).

Tolerance: relative 1e-10 per element of every source and total.  Both sides
are FP64 (XKARZAS's REAL(4) interpolation in single precision, rounded as
written); they differ by FMA contraction and the last bit of the device's
exp/log/pow, and by the occupation probabilities and Boltzmann factors being
formed once per depth on the device (the same functions of the same inputs).
Three of the reference's formulas amplify those roundings: H2PLOP's fit is a
polynomial in ln(nu) whose terms (~3e3) cancel to ~-30 before the exp, MAP1
evaluates HMINOP's bound-free parabola in absolute wavelength (terms ~1e6
cancelling to ~30), and the non-LTE source functions divide by BMIN - EHVKT.
Measured: up to 5.4e-12 (H2+), 3.4e-12 (H-), 1.3e-11 (SHMIN with departure
coefficients), 1e-14 elsewhere; the reference's own build (-O3
-march=native, which contracts a*b+c into FMAs) differs from the uncontracted
oracle by the same order.
"""
import ctypes

import numpy as np
import pytest

from atlas12_b200 import _lib, atlas, surrogate, synthetic

pytestmark = pytest.mark.gpu

RTOL = 1e-10
NAMES = ("ahyd", "shyd", "ah2p", "ahmin", "shmin", "sigh", "sigel")


def atmosphere(teff, logg):
    m = surrogate.grey_model(teff, logg)
    e = surrogate.eos(m["t"], m["p"])
    return dict(t=m["t"], xne=e["xne"], rho=e["rho"], x1=e["nh"] * (1 - e["xh"]) / 2, x2=e["nh"] * e["xh"])


@pytest.fixture(scope="module")
def kapp(gpu_ctx, tables):
    a = atlas.Atlas(gpu_ctx, tables)
    a.set_kapp_tables(tables)
    return a


def rel_err(got, ref):
    return float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)))


@pytest.mark.parametrize("teff,logg,nlte", [(5777.0, 4.44, False), (4000.0, 2.0, True), (8000.0, 4.0, False)])
def test_kapp_hydrogen_matches_oracle(po, tables, kapp, teff, logg, nlte):
    at = atmosphere(teff, logg)
    nr, kw = at["t"].size, 80
    # 600 frequencies over the opacity-sampling range, plus points just either side of
    # the Lyman, Balmer and Paschen limits, Lyman alpha's Rayleigh resonance and the H- edge
    ws, _ = synthetic.geometric_waveset(9.0, 160000.0, 600)
    edges = np.array([1e7 / 109678.764, 1e7 / 27419.659, 1e7 / 12186.462, 121.567, 102.57, 1643.908])
    ws = np.sort(np.concatenate([ws, edges * (1 - 1e-6), edges * (1 + 1e-6)]))
    bhyd = bmin = None
    if nlte:
        rng = np.random.default_rng(5)
        bhyd = np.zeros((6, kw))
        bhyd[:, :nr] = rng.uniform(0.7, 1.4, (6, nr))
        bmin = np.zeros(kw)
        bmin[:nr] = rng.uniform(0.8, 1.2, nr)
    ac, sg, sc, parts = kapp.kapp_hydrogen(ws, at["t"], at["xne"], at["rho"], at["x1"], at["x2"], bhyd=bhyd,
                                           bmin=bmin, kw=kw, parts=True)
    kt = po.kapp_tables(tables)
    worst = {}
    for i, w in enumerate(ws):
        ref = po.kapp_hydrogen(kt, w, at["t"], at["xne"], at["rho"], at["x1"], at["x2"],
                               None if bhyd is None else bhyd[:, :nr], None if bmin is None else bmin[:nr])
        got = dict(acont=ac[i, :nr], sigmac=sg[i, :nr], scont=sc[i, :nr], **{k: parts[i, q, :nr] for q, k in
                                                                                 enumerate(NAMES)})
        for k, v in got.items():
            worst[k] = max(worst.get(k, 0.0), rel_err(v, ref[k]))
    print("max relative error", worst)
    assert max(worst.values()) <= RTOL, worst
    # the padding depths nrhox..kw-1 are zero
    assert not np.any(ac[:, nr:]) and not np.any(sg[:, nr:]) and not np.any(sc[:, nr:])
    assert np.all(ac[:, :nr] > 0) and np.all(np.isfinite(sc[:, :nr]))


def test_kapp_hydrogen_rejects_bad_input(gpu_ctx, tables):
    fresh = _lib.Context(0, _lib.PREC_MIXED)
    try:
        a = atlas.Atlas(fresh, tables)
        at = atmosphere(5777.0, 4.44)
        ws = np.array([500.0, 600.0])
        args = (at["t"], at["xne"], at["rho"], at["x1"], at["x2"])
        with pytest.raises(RuntimeError):  # tables not set
            a.kapp_hydrogen(ws, *args)
        a.set_kapp_tables(tables)
        bad = dict(at)
        bad["xne"] = at["xne"].copy()
        bad["xne"][10] = np.nan
        with pytest.raises(RuntimeError, match="non-finite"):
            a.kapp_hydrogen(ws, bad["t"], bad["xne"], bad["rho"], bad["x1"], bad["x2"])
        neg = at["t"].copy()
        neg[3] = -1.0
        with pytest.raises(RuntimeError, match="not positive"):
            a.kapp_hydrogen(ws, neg, *args[1:])
        with pytest.raises(RuntimeError, match="WAVESET"):
            a.kapp_hydrogen(np.array([500.0, 0.0]), *args)
        t = dict(tables)
        t["k_gff"] = tables["k_gff"].copy()
        t["k_gff"][7] = np.inf
        with pytest.raises(RuntimeError, match="non-finite"):
            a.set_kapp_tables(t)
        # the call after the refused ones still works
        ac, sg, sc = a.kapp_hydrogen(ws, *args)
        assert np.all(ac > 0)
    finally:
        fresh.close()
