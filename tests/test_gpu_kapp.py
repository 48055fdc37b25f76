"""KAPP's hydrogen, helium and H2 continuum sources on the GPU
(atlasgpu_atlas_kapp_hydrogen and atlasgpu_atlas_kapp, through the C ABI)
against the CPU oracle (oracle/kapp.c), which restates HOP, XKARZAS, COULFF,
H2PLOP, HMINOP, HRAYOP, ELECOP, HE1OP, HE2OP, HEMIOP, HERAOP, H2MINOP,
H2COLLOP, H2RAOP with PARTFNH2 and EQUILH2, and KAPP's totals
(atlas12_modules.f90:11202-17338, :22324-22469).

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
NAMES_HE = NAMES + ("ahe1", "ahe2", "ahemin", "sighe")
NAMES_H2 = NAMES_HE + ("ah2min", "ah2coll", "sigh2")


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


def helium_atmosphere(teff, logg):
    """atmosphere() with helium at 0.0851 of hydrogen by number, its
    ionisation split by smooth functions of T."""
    at = atmosphere(teff, logg)
    t = at["t"]
    e = surrogate.eos(t, surrogate.grey_model(teff, logg)["p"])
    nhe = 0.0851 * e["nh"]
    f1 = 1.0 / (1.0 + np.exp(-(t - 12000.0) / 1500.0))
    f2 = 1.0 / (1.0 + np.exp(-(t - 22000.0) / 2500.0))
    xnf4 = nhe * f1 * (1.0 - f2)
    return dict(at, x3=nhe * (1.0 - f1), x4=xnf4 / 2.0, x5=nhe * f1 * f2, xnf4=xnf4)


HE_EDGES = np.array([22.78, 50.43, 91.13, 205.06, 260.0, 312.1, 331.2, 342.2, 364.6, 569.6, 820.3, 1116.5, 1458.2,
                     1845.6, 23.905, 1458.8, 506.441, 58.21])


@pytest.mark.parametrize("teff,logg,nlte", [(15000.0, 4.0, False), (25000.0, 4.5, True), (6000.0, 4.0, False)])
def test_kapp_helium_matches_oracle(po, tables, kapp, teff, logg, nlte):
    at = helium_atmosphere(teff, logg)
    nr, kw = at["t"].size, 80
    ws, _ = synthetic.geometric_waveset(5.0, 300000.0, 600)
    ws = np.sort(np.concatenate([ws, HE_EDGES * (1 - 1e-6), HE_EDGES * (1 + 1e-6)]))
    bhyd = bmin = None
    if nlte:
        rng = np.random.default_rng(7)
        bhyd = np.zeros((6, kw))
        bhyd[:, :nr] = rng.uniform(0.7, 1.4, (6, nr))
        bmin = np.zeros(kw)
        bmin[:nr] = rng.uniform(0.8, 1.2, nr)
    pops = (at["t"], at["xne"], at["rho"], at["x1"], at["x2"], at["x3"], at["x4"], at["x5"], at["xnf4"])
    ac, sg, sc, parts = kapp.kapp(ws, *pops, bhyd=bhyd, bmin=bmin, kw=kw, parts=True)
    kt = po.kapp_tables(tables)
    worst = {}
    for i, w in enumerate(ws):
        ref = po.kapp(kt, w, *pops, None if bhyd is None else bhyd[:, :nr], None if bmin is None else bmin[:nr])
        got = dict(acont=ac[i, :nr], sigmac=sg[i, :nr], scont=sc[i, :nr],
                   **{k: parts[i, q, :nr] for q, k in enumerate(NAMES_HE)})
        for k, v in got.items():
            worst[k] = max(worst.get(k, 0.0), rel_err(v, ref[k]))
    print("max relative error", worst)
    assert max(worst.values()) <= RTOL, worst
    assert not np.any(ac[:, nr:]) and not np.any(sg[:, nr:]) and not np.any(parts[:, :, nr:])
    # the hydrogen sources are those of kapp_hydrogen, bit for bit; helium only adds
    ach, sgh, sch, ph = kapp.kapp_hydrogen(ws, *pops[:5], bhyd=bhyd, bmin=bmin, kw=kw, parts=True)
    np.testing.assert_array_equal(parts[:, :7], ph)
    assert np.all(ac >= ach) and np.all(sg >= sgh)
    if teff >= 15000.0:
        assert np.max(parts[:, 7:11, :nr]) > 0 and np.max(ac - ach) > 0


@pytest.mark.parametrize("teff,logg,nlte", [(3500.0, 5.0, False), (4500.0, 4.5, True), (9000.0, 4.0, False)])
def test_kapp_h2_matches_oracle(po, tables, kapp, teff, logg, nlte):
    kapp.set_kapp_h2_tables(tables)
    at = helium_atmosphere(teff, logg)
    nr, kw = at["t"].size, 80
    xnf3 = at["x3"] * 1.0  # He I partition function 1
    # 600 frequencies over 9 nm - 400 um (the CIA grid ends at 20,000 cm^-1 = 500 nm), plus points either side
    # of H2MINOP's and the CIA grid's ends and H2RAOP's cap
    ws, _ = synthetic.geometric_waveset(9.0, 400000.0, 600)
    edges = np.array([500.14, 210057.25, 1e7 / 20000.0, 1e7 / 25.0, 102.6, 1e7 / 1012.5])
    ws = np.sort(np.concatenate([ws, edges * (1 - 1e-6), edges * (1 + 1e-6)]))
    bhyd = bmin = None
    if nlte:
        rng = np.random.default_rng(9)
        bhyd = np.zeros((6, kw))
        bhyd[:, :nr] = rng.uniform(0.7, 1.4, (6, nr))
        bmin = np.zeros(kw)
        bmin[:nr] = rng.uniform(0.8, 1.2, nr)
    pops = (at["t"], at["xne"], at["rho"], at["x1"], at["x2"], at["x3"], at["x4"], at["x5"], at["xnf4"])
    ac, sg, sc, parts = kapp.kapp(ws, *pops, bhyd=bhyd, bmin=bmin, kw=kw, parts=True, xnf3=xnf3)
    kt, h2 = po.kapp_tables(tables), po.kapp_h2_tables(tables)
    worst = {}
    for i, w in enumerate(ws):
        ref = po.kapp_h2(kt, h2, w, *pops, xnf3, None if bhyd is None else bhyd[:, :nr],
                         None if bmin is None else bmin[:nr])
        got = dict(acont=ac[i, :nr], sigmac=sg[i, :nr], scont=sc[i, :nr],
                   **{k: parts[i, q, :nr] for q, k in enumerate(NAMES_H2)})
        for k, v in got.items():
            worst[k] = max(worst.get(k, 0.0), rel_err(v, ref[k]))
    print("max relative error", worst)
    assert max(worst.values()) <= RTOL, worst
    assert not np.any(ac[:, nr:]) and not np.any(parts[:, :, nr:])
    if teff < 5000.0:
        assert np.max(parts[:, 11:14, :nr]) > 0


def test_kapp_h2_requires_its_tables(gpu_ctx, tables):
    fresh = _lib.Context(0, _lib.PREC_MIXED)
    try:
        a = atlas.Atlas(fresh, tables)
        a.set_kapp_tables(tables)
        at = helium_atmosphere(3500.0, 5.0)
        pops = [at[k] for k in ("t", "xne", "rho", "x1", "x2", "x3", "x4", "x5", "xnf4")]
        ws = np.array([1000.0, 5000.0])
        with pytest.raises(RuntimeError, match="H2 tables not set"):
            a.kapp(ws, *pops, xnf3=at["x3"])
        t = dict(tables)
        t["k_cia_tab"] = tables["k_cia_tab"].copy()
        t["k_cia_tab"][1, 3, 17] = np.nan
        with pytest.raises(RuntimeError, match="non-finite"):
            a.set_kapp_h2_tables(t)
        a.set_kapp_h2_tables(tables)
        ac, sg, sc = a.kapp(ws, *pops, xnf3=at["x3"])
        ac0, sg0, sc0 = a.kapp(ws, *pops)
        # the H2 sources only add (to rounding: the two calls run different kernel instantiations)
        assert np.all(ac >= ac0 * (1 - 1e-13)) and np.all(sg >= sg0 * (1 - 1e-13)) and np.any(ac > ac0 * (1 + 1e-6))
    finally:
        fresh.close()


@pytest.mark.parametrize("use_stehle,nlte", [(False, False), (True, False), (True, True)])
def test_hlinop_matches_oracle(po, tables, kapp, use_stehle, nlte):
    """HLINOP (atlasgpu_atlas_hlinop) against orc_hlinop: AHLINE and SHLINE at
    every (frequency, depth) over 80-2300 nm with the Lyman, Balmer, Paschen
    and Brackett members and limits, on seeded Stehle tables or STARK alone,
    LTE and with departure coefficients (which make SHLINE differ from BNU)."""
    rng = np.random.default_rng(4)
    nr, kw = 40, 48
    t = np.geomspace(3000.0, 60000.0, nr)
    xne = np.geomspace(1e9, 3e17, nr)
    rho = np.geomspace(1e-11, 1e-5, nr)
    x1 = rho / 1.67e-24 * rng.uniform(0.05, 0.5, nr)
    ws, _ = synthetic.geometric_waveset(80.0, 2300.0, 700)
    lines = np.array([97.25, 102.57, 121.57, 364.6, 383.54, 410.17, 486.13, 656.28, 820.4, 1005.2, 1875.1, 1458.2,
                      2166.1])
    ws = np.sort(np.concatenate([ws, lines * (1 - 1e-5), lines * (1 + 1e-5)]))
    st_dicts = synthetic.stehle_tables() if use_stehle else None
    kapp.set_stehle_tables(st_dicts)
    bhyd = None
    if nlte:
        bhyd = np.ones((6, kw))
        bhyd[:, :nr] = rng.uniform(0.6, 1.5, (6, nr))
    ah, sh = kapp.hlinop(ws, t, xne, rho, x1, bhyd=bhyd, kw=kw)
    st = po.stehle_structs(st_dicts)[0] if use_stehle else None
    worst = {"ahline": 0.0, "shline": 0.0}
    kt = po.kapp_tables(tables)
    for i, w in enumerate(ws):
        ra, rs = po.hlinop(kt, w, t, xne, rho, x1, None if bhyd is None else np.ascontiguousarray(bhyd[:, :nr]), st)
        worst["ahline"] = max(worst["ahline"], rel_err(ah[i, :nr], ra))
        worst["shline"] = max(worst["shline"], rel_err(sh[i, :nr], rs))
    print("max relative error", worst)
    assert max(worst.values()) <= RTOL, worst
    assert np.count_nonzero(ah[:, :nr]) > 0.3 * ah[:, :nr].size and not np.any(ah[:, nr:])
    kapp.set_stehle_tables(None)


def test_kapp_helium_rejects_bad_input(gpu_ctx, tables, kapp):
    at = helium_atmosphere(15000.0, 4.0)
    ws = np.array([50.0, 500.0])
    pops = [at[k] for k in ("t", "xne", "rho", "x1", "x2", "x3", "x4", "x5", "xnf4")]
    bad = [p.copy() for p in pops]
    bad[5][4] = np.inf
    with pytest.raises(RuntimeError, match="non-finite"):
        kapp.kapp(ws, *bad)
    pp = _lib.KappPops(*[p.ctypes.data for p in pops[:5]], None, None, None, None, None, None)
    out = [np.zeros((2, pops[0].size)) for _ in range(3)]
    with pytest.raises(RuntimeError, match="bad argument"):
        gpu_ctx.call("atlasgpu_atlas_kapp", 2, ws.ctypes.data, pops[0].size, pops[0].size, ctypes.byref(pp),
                     *[o.ctypes.data for o in out], None)
    ac, sg, sc = kapp.kapp(ws, *pops)
    assert np.all(ac > 0)


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
