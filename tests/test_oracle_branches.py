"""The oracle's XLINOP autoionizing / merged-continuum records
(atlas12_modules.f90:20201-20245) and SYNTHE compute_line_opacity's Shore
and merged-continuum branches (synthe_module.f90:3609-3696) against a second
restatement in plain Python loops, on small seeded inputs (no GPU).  Both
use the C library's exp, log, pow and (for SYNTHE's REAL(4) edge test) expf
in the same operation order, so they agree bit for bit.
"""
import ctypes
import math

import numpy as np
import pytest

from atlas12_b200 import atlas, synthetic

CLIGHT_NMS = 2.99792458e17
RYDBERG_INF = 109737.31568157
RYDBERG_H = 109677.583403
_libm = ctypes.CDLL("libm.so.6")
_libm.expf.restype = ctypes.c_float
_libm.expf.argtypes = [ctypes.c_float]


def py_xlinop_other(recs, nrhox, kw, nspec, xne, hckt, tabcont, iwt, waveset, xnfp, rho):
    """XLINOP's record loop for TYPE 1 and the merged-continuum TYPEs only
    (the inputs hold no TYPE 0/3 records)."""
    numnu, nwave = waveset.size, iwt.size - 1
    xl = np.zeros((numnu, kw))
    emerge = [RYDBERG_INF / ((1600.0 / math.pow(xne[j], 2.0 / 15.0)) * (1600.0 / math.pow(xne[j], 2.0 / 15.0)))
              for j in range(nrhox)]
    nucont, nu = 1, 1
    for r in recs:
        wl = float(r["wlvac"])
        if wl > waveset[-1]:
            return xl
        iwl = int(r["nbuff"])
        while iwl >= iwt[nucont - 1]:
            nucont += 1
            if nucont > nwave + 1:
                nucont = nwave + 1
                break
        while wl >= waveset[nu - 1]:
            nu += 1
            if nu >= numnu:
                return xl
        t, nel = int(r["itype"]), int(r["nelion"])
        if t in (2, -1, 0, 3) or nel < 1 or nel > nspec:
            continue
        elo = float(r["elo"])
        for j in range(nrhox):
            xp = xnfp[nel - 1, j]
            if t == 1:
                tc = tabcont[nucont - 1, j]
                g, ash, bsh, gr = float(r["gf"]), float(r["gammas"]), float(r["gammaw"]), float(r["gammar"])
                frelin = CLIGHT_NMS / wl
                center = bsh * g * xp / rho[j]
                if center < tc:
                    continue
                center = center * math.exp(-(elo * hckt[j]))
                if center < tc:
                    continue
                for iw in range(nu, min(nu + 2000, numnu) + 1):
                    eps = 2.0 * (CLIGHT_NMS / waveset[iw - 1] - frelin) / gr
                    cv = center * (ash * eps + bsh) / (eps * eps + 1.0) / bsh
                    xl[iw - 1, j] += cv
                    if cv < tc:
                        break
                for i in range(1, 2001):
                    iw = nu - i
                    if iw <= 0:
                        break
                    eps = 2.0 * (CLIGHT_NMS / waveset[iw - 1] - frelin) / gr
                    cv = center * (ash * eps + bsh) / (eps * eps + 1.0) / bsh
                    xl[iw - 1, j] += cv
                    if cv < tc:
                        break
            else:
                z = 2.0 if nel == 4 else 1.0
                wshift = 1.0e7 / (1.0e7 / wl - RYDBERG_INF * (z * z) / (float(t) * float(t)))
                wmerge = 1.0e7 / (1.0e7 / wl - emerge[j] * (z * z))
                wmax = wmerge if wmerge > wshift else wshift
                con = float(r["gf"]) * xp * math.exp(-(elo * hckt[j])) / rho[j]
                for iw in range(nu, min(nu + 1000, numnu) + 1):
                    if wmax < waveset[iw - 1]:
                        break
                    xl[iw - 1, j] += con
    return xl


def py_synthe_other(recs, length, nrhox, wbegin, ratio, wlend, cont, xnfpel, xne, hckt):
    """compute_line_opacity's Shore and merged-continuum branches (vacuum), FP64."""
    out = np.zeros((nrhox, length))
    ratiolg = math.log(ratio)
    ixwlbeg = int(round(math.log(wbegin) / ratiolg))
    nspec = xnfpel.shape[1]
    for j in range(nrhox):
        inglis = np.float32(1600.0 / math.pow(xne[j], 2.0 / 15.0))
        nmerge = np.float32(inglis - np.float32(1.5))
        for r in recs:
            t, nel = int(r["itype"]), int(r["nelion"])
            if nel < 1 or nel > nspec:
                continue
            wl = float(r["wlvac"])
            nbuff = int(r["nbuff"])
            if t == 1:
                gr, gs, gw = float(r["gammar"]), float(r["gammas"]), float(r["gammaw"])
                kappa0 = gw * float(r["gf"]) * xnfpel[j, nel - 1]
                ic = min(max(nbuff, 1), length)
                kapmin = float(cont[j, ic - 1]) * 1e-3
                if kappa0 < kapmin:
                    continue
                kappa0 = kappa0 * math.exp(-float(r["elo"]) * hckt[j])
                if kappa0 < kapmin:
                    continue
                frelin = CLIGHT_NMS / wl
                if wl <= wlend:
                    minred = max(nbuff, 1)
                    freq = CLIGHT_NMS / (wbegin * atlas_powi(ratio, minred - 1))
                    for ib in range(minred, length + 1):
                        eps = 2.0 * (freq - frelin) / gr
                        kap = kappa0 * (gs * eps + gw) / (eps * eps + 1.0) / gw
                        out[j, ib - 1] += kap
                        if kap < float(cont[j, ib - 1]) * 1e-3:
                            break
                        freq = freq / ratio
                    if nbuff == 1 or wl < wbegin:
                        continue
                ib = min(length + 1, nbuff)
                maxblue = ib - 1
                freq = CLIGHT_NMS / (wbegin * atlas_powi(ratio, ib - 1))
                for _ in range(maxblue):
                    ib -= 1
                    freq = freq * ratio
                    eps = 2.0 * (freq - frelin) / gr
                    kap = kappa0 * (gs * eps + gw) / (eps * eps + 1.0) / gw
                    out[j, ib - 1] += kap
                    if kap < float(cont[j, ib - 1]) * 1e-3:
                        break
            elif t >= 4:
                ryd = RYDBERG_H if nel == 1 else RYDBERG_INF
                em = ryd / (float(nmerge) * float(nmerge))
                wshift = 1.0e7 / (1.0e7 / wl - ryd / (float(t) * float(t)))
                wmerge = 1.0e7 / (1.0e7 / wl - em)
                if wmerge < 0.0:
                    wmerge = wshift + wshift
                wmerge = max(wmerge, wshift)
                wmerge = min(wshift + wshift, wmerge)
                wtail = 1.0e7 / (1.0e7 / wmerge - 500.0)
                if wtail < 0.0:
                    wtail = wmerge + wmerge
                wtail = min(wmerge + wmerge, wtail)
                ixwl = int(math.log(wl) / ratiolg)
                edgeblue = _libm.expf(float(np.float32(ixwl) * np.float32(ratiolg)))
                if np.float32(edgeblue) > np.float32(wl):
                    ixwl -= 1
                n1 = ixwl + 1 - ixwlbeg + 1
                n2 = int(math.log(wmerge) / ratiolg + 0.5) - ixwlbeg + 1
                n3 = int(math.log(wtail) / ratiolg + 0.5) - ixwlbeg + 1
                if n1 > length or n3 < 1:
                    continue
                n1 = max(n1, 1)
                kappa = float(r["gf"]) * xnfpel[j, nel - 1] * math.exp(-float(r["elo"]) * hckt[j])
                dn = float(n3 - n2)
                tail = 1.0
                for ib in range(n1, min(n3, length) + 1):
                    if ib > n2:
                        tail = float(n3 - ib) / dn
                    out[j, ib - 1] += kappa * tail
    return out


def atlas_powi(x, m):
    """gfortran's REAL(8)**INTEGER by binary exponentiation (as the oracle's orc_powi)."""
    n = abs(m)
    y = x if n % 2 else 1.0
    n >>= 1
    while n:
        x = x * x
        if n % 2:
            y = y * x
        n >>= 1
    return 1.0 / y if m < 0 else y


@pytest.fixture(scope="module")
def small_atm():
    rng = np.random.default_rng(3)
    nrhox, kw, nspec = 10, 12, 30
    xne = 10.0 ** np.linspace(10.0, 16.0, nrhox)
    hckt = 1.4388 / np.linspace(4000.0, 12000.0, nrhox)
    xnfp = 10.0 ** rng.uniform(8.0, 12.0, (nspec, kw))
    rho = 10.0 ** np.linspace(-10.0, -6.0, kw)
    return dict(nrhox=nrhox, kw=kw, nspec=nspec, xne=xne, hckt=hckt, xnfp=xnfp, rho=rho)


def test_xlinop_branches_match_plain_loops(po, tables, small_atm):
    a = small_atm
    ws = np.geomspace(400.0, 440.0, 600)
    cut = atlas.cutoff_grid()
    iwt = atlas.iwavetab(cut)
    tabcont = np.full((cut.size + 1, a["kw"]), 1.0e-14)
    recs = synthetic.nlte_records(60, 400.5, 439.5, seed=4, types=(1, 2, -1, 7, 12, -3), type_p=(.4, .1, .1, .15,
                                                                                                      .15, .1))
    rng = np.random.default_rng(5)
    recs["nelion"] = rng.integers(1, 35, recs.size)  # a few outside 1..nspec
    recs["nelion"][::9] = 4
    f = recs["itype"] == 1
    recs["gammaw"][f] = 10.0 ** rng.uniform(-2.0, 0.0, f.sum())
    recs["gammas"][f] = recs["gammaw"][f] * rng.uniform(-2.0, 2.0, f.sum())
    recs["gammar"][f] = 10.0 ** rng.uniform(11.0, 13.0, f.sum())
    recs["gf"] = 10.0 ** rng.uniform(-22.0, -18.0, recs.size)
    h = po.tabvoigt(tables["tabvi"], tables["tabh1"])
    atm = dict(xnfdop=np.zeros((a["nspec"], a["kw"])), dopple=np.ones((a["nspec"], a["kw"])), xne=a["xne"],
               txnxn=np.zeros(a["kw"]), hckt=a["hckt"], nrhox=a["nrhox"], xnfp=a["xnfp"], rho=a["rho"])
    got, _ = po.atlas_xlinop(*h, po.build_tablog(), recs, atm, tabcont, iwt, ws, synthetic.contx_table())
    want = py_xlinop_other(recs, a["nrhox"], a["kw"], a["nspec"], a["xne"], a["hckt"], tabcont, iwt, ws, a["xnfp"],
                           a["rho"])
    assert np.count_nonzero(want) > 1000
    np.testing.assert_array_equal(got, want)


def test_synthe_branches_match_plain_loops(po, small_atm):
    a = small_atm
    g = po.synthe_grid(400.0, 400.8, 500000.0)
    length = g["length"]
    rng = np.random.default_rng(6)
    n = 40
    recs = np.zeros(n, po.NLTE_LINE)
    recs["wlvac"] = np.sort(rng.uniform(399.9, 400.9, n))
    recs["nbuff"] = [po.nbuff(w, g["ratiolg"], g["ixwlbeg"]) for w in recs["wlvac"]]
    recs["itype"] = rng.choice([1, 4, 9, 30, 100], n)
    recs["nelion"] = rng.integers(1, 8, n)
    recs["gf"] = 10.0 ** rng.uniform(-24.0, -21.0, n)
    recs["elo"] = rng.uniform(0.0, 3.0e4, n)
    recs["gammaw"] = 10.0 ** rng.uniform(0.0, 2.0, n)
    recs["gammas"] = recs["gammaw"] * rng.uniform(-2.0, 2.0, n)
    recs["gammar"] = 10.0 ** rng.uniform(9.0, 11.0, n)
    nrhox, nspec = a["nrhox"], 8
    cont = (10.0 ** rng.uniform(-12.0, -10.0, (nrhox, length))).astype(np.float32)
    xnfpel = 10.0 ** rng.uniform(9.0, 11.0, (nrhox, nspec))
    atm = dict(xnfdop=np.zeros((nrhox, nspec)), dopple=np.ones((nrhox, nspec)), xne=a["xne"],
               txnxn=np.zeros(nrhox), hckt=a["hckt"], xnfpel=xnfpel)
    got = po.synthe_nlte_opacity(recs, length, g["wbegin"], g["ratio"], 400.8, 0.0, cont, atm,
                                 np.zeros((17, 26)))
    want = py_synthe_other(recs, length, nrhox, g["wbegin"], g["ratio"], 400.8, cont, xnfpel, a["xne"], a["hckt"])
    assert np.count_nonzero(want) > 0.5 * want.size
    np.testing.assert_array_equal(got, want)
