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
        inglis = np.float32(1600.0 / math.pow(xne[j], float(np.float32(2.0) / np.float32(15.0))))
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


# ------------------------------------------------------------- hydrogen
def _powi(x, m):
    return atlas_powi(x, m)


def py_stark(h, b, p, n, m):
    """STARK_PROFILE (atlas12_modules.f90:20376-20514) in plain Python."""
    indx = 2 * (n - 1) + (m - n) if (n <= 3 and m - n <= 2) else 7
    b2, sb = b * b, math.sqrt(b)
    if b > 500.0:
        return (1.5 / sb + 27.0 / b2) / b2
    im = min(int(5.0 * p) + 1, 4)
    ip = im + 1
    wtpp = 5.0 * (p - h["h_pp"][im - 1])
    wtpm = 1.0 - wtpp
    if b > 25.12:
        cc = h["h_c"][indx - 1, ip - 1] * wtpp + h["h_c"][indx - 1, im - 1] * wtpm
        dd = h["h_d"][indx - 1, ip - 1] * wtpp + h["h_d"][indx - 1, im - 1] * wtpm
        return (1.5 / sb + 27.0 / b2) / b2 * (1.0 + dd / (cc + b * sb))
    jm = 1
    for j in range(2, 16):
        if b <= h["h_betagrid"][j - 1]:
            jm = j - 1
            break
    jp = jm + 1
    g = h["h_betagrid"]
    wtbp = (b - g[jm - 1]) / (g[jp - 1] - g[jm - 1])
    pb = h["h_propbm"][indx - 1]
    cbp = pb[jp - 1, ip - 1] * wtpp + pb[jp - 1, im - 1] * wtpm
    cbm = pb[jm - 1, ip - 1] * wtpp + pb[jm - 1, im - 1] * wtpm
    corr = 1.0 + cbp * wtbp + cbm * (1.0 - wtbp)
    wt = max(min(0.5 * (10.0 - b), 1.0), 0.0)
    pr1 = 8.0 / (83.0 + (2.0 + 0.95 * b2) * b) if b <= 10.0 else 0.0
    pr2 = (1.5 / sb + 27.0 / b2) / b2 if b >= 8.0 else 0.0
    return (pr1 * wt + pr2 * (1.0 - wt)) * corr


def py_hfnm(n, m):
    if m <= n:
        return 0.0
    xn, xm, xmn = float(n), float(m), float(m - n)
    ginf, gca, fkn = 0.2027 / math.pow(xn, 0.71), 0.124 / xn, xn * 1.9603
    wtc = 0.45 - 2.4 / _powi(xn, 3) * (xn - 1.0)
    fk = fkn * _powi(xm / (xmn * (xm + float(n))), 3)
    x12 = math.pow(xmn, 1.2)
    wt = (x12 - 1.0) / (x12 + wtc)
    return fk * (1.0 - wt * ginf - (0.222 + gca / xm) * (1.0 - wt))


def py_hprof4(h, n, m, xne, t, xnfp3, xnh2, xnf1, xnf2, xnfp1, dop1, delw, expi):
    """HPROF4 (atlas12_modules.f90:20553-21002) in plain Python."""
    c, ca, pi, spi = 2.99792458e10, 2.99792458e18, 3.141592653589793, 1.7724538509055159
    x16 = math.pow(xne, 1.0 / 6.0)
    pp, fo = x16 * 0.08989 / math.sqrt(t), _powi(x16, 4) * 1.25e-9
    y1b = 2.0 / (1.0 + 0.012 / t * math.sqrt(xne / t))
    t43 = math.pow(t / 10000.0, 0.3)
    y1s, t3nhe, t3nh2 = t43 / x16, t43 * xnfp3, t43 * xnh2
    c1d, c2d = fo * 78940.0 / t, _powi(fo, 2) / 5.96e-23 / xne
    gcon1 = 0.2 + 0.09 * math.sqrt(t / 10000.0) / (1.0 + xne / 1.0e13)
    gcon2 = 0.2 / (1.0 + xne / 1.0e15)
    mmn, xn, xm = m - n, float(n), float(m)
    xn2, xm2 = xn * xn, xm * xm
    xmn2, xm2mn2 = xm2 * xn2, xm2 - xn2
    gnm = xm2mn2 / xmn2
    xknm = h["h_xknmtb"][n - 1, mmn - 1] if (mmn <= 3 and n <= 4) else 5.5e-5 / gnm * xmn2 / (1.0 + 0.13 / mmn)
    y1num = 550.0 if m == 2 else 380.0 if m == 3 else 320.0
    y1wht = 1.0e13
    if mmn <= 3:
        y1wht = 1.0e14
    if mmn <= 2 and n <= 2:
        y1wht = h["h_y1wtm"][n - 1, mmn - 1]
    freqnm = 109677.583403 * 2.99792458e10 * gnm
    dbeta = ca / _powi(freqnm, 2) / xknm
    wavenm = ca / freqnm
    c1con, c2con = xknm / wavenm * gnm * xm2mn2, _powi(xknm / wavenm, 2)
    radamp = h["h_asumlyman"][m - 1] if n == 1 else h["h_asum"][n - 1] + h["h_asum"][m - 1]
    radamp = radamp / (4.0 * pi) / freqnm
    resont = py_hfnm(1, m) / xm / (1.0 - 1.0 / xm2)
    if n != 1:
        resont = resont + py_hfnm(1, n) / xn / (1.0 - 1.0 / xn2)
    resont = resont * 3.92e-24 / gnm
    vdw = 4.45e-26 / gnm * math.pow(xm2 * (7.0 * xm2 + 5.0), 0.4)
    starkc = 1.6678e-18 * freqnm * xknm
    if n > 4 or m > 10:
        fs = [(0.0, 1.0)]
    elif mmn != 1:
        fs = [(h["h_stcomp"][i, n - 1] * 1.0e7, h["h_stcpwt"][i, n - 1] / xn2) for i in range(h["h_lncomp"][n - 1])]
    else:
        k0 = h["h_istal"][n - 1] - 1
        fs = [(h["h_stalph"][k0 + i] * 1.0e7, h["h_stwtal"][k0 + i] / xn2 / 3.0) for i in range(h["h_lnghal"][n - 1])]
    dst = -10.0 * delw / wavenm * freqnm
    freq4 = ca / (wavenm + delw * 10.0)
    de = abs(freq4 - freqnm)
    hwstk, hwvdw, hwrad = starkc * fo, vdw * t3nhe + 2.0 * vdw * t3nh2, radamp
    hwres = resont * xnf1
    hwlor = hwres + hwvdw + hwrad
    nwid = 1 if (dop1 >= hwstk and dop1 >= hwlor) else (2 if hwlor >= hwstk else 3)
    core = abs(de) <= freqnm * max(dop1, hwlor, hwstk)
    dop = freqnm * dop1
    hp = 0.0
    if not core or nwid == 1:
        for f, w in fs:
            d = abs(freq4 - freqnm - f) / dop
            if d <= 7.0:
                hp = hp + math.exp(-d * d) * w
        if core:
            return hp
    if not core or nwid == 2:
        if n == 1 and m == 2:
            hwres = hwres * 4.0
            hwlor = hwres + hwvdw + hwrad
            hhw = freqnm * hwlor
            if freq4 > (82259.105 - 4000.0) * c:
                res = hwres * freqnm / pi / (de * de + hhw * hhw) * spi * dop
            else:
                cut = 0.0
                if freq4 >= 50000.0 * c:
                    sp, f0 = 200.0 * c, (82259.105 - 22000.0) * c
                    tb = h["h_cutoffh2"]
                    if freq4 < f0:
                        cut = (tb[1] - tb[0]) / sp * (freq4 - f0) + tb[0]
                    else:
                        ic = min(int((freq4 - f0) / sp), 89)
                        cut = (tb[ic + 1] - tb[ic]) / sp * (freq4 - (ic * sp + f0)) + tb[ic]
                    cut = math.pow(10.0, cut - 14.0) * xnfp1 * 2.0 / c
                res = cut * spi * dop
            rad = 0.0 if freq4 <= 2.463e15 else hwrad * freqnm / pi / (de * de + hhw * hhw) * spi * dop
            vd = 0.0 if freq4 < 1.8e15 else hwvdw * freqnm / pi / (de * de + hhw * hhw) * spi * dop
            hp = hp + (res + rad + vd)
        else:
            hhw = freqnm * hwlor
            hp = hp + hhw / pi / (de * de + hhw * hhw) * spi * dop
        if core:
            return hp
    wty1 = 1.0 / (1.0 + xne / y1wht)
    y1scal = y1num * y1s * wty1 + y1b * (1.0 - wty1)
    c1, c2 = c1d * c1con * y1scal, c2d * c2con
    g1 = 6.77 * math.sqrt(c1)
    gnot = g1 * max(0.0, 0.2114 + math.log(math.sqrt(c2) / c1)) * (1.0 - gcon1 - gcon2)
    beta = abs(dst) / fo * dbeta
    y1, y2 = c1 * beta, c2 * beta * beta
    gam = gnot
    if not (y2 <= 1.0e-4 and y1 <= 1.0e-5):
        gam = g1 * (0.5 * math.exp(-min(80.0, y1)) + expi(1, y1) - 0.5 * expi(1, y2)) * \
            (1.0 - gcon1 / (1.0 + _powi(90.0 * y1, 3)) - gcon2 / (1.0 + 2000.0 * y1))
        if gam <= 1.0e-20:
            gam = 0.0
    prqs = py_stark(h, beta, pp, n, m)
    if m <= 2:
        prqs = prqs * 0.5
        if freq4 >= (82259.105 - 20000.0) * c:
            if freq4 > (82259.105 - 4000.0) * c:
                b4 = 4000.0 * c / fo * dbeta
                p4 = py_stark(h, b4, pp, n, m) * 0.5 / fo * dbeta
                c4 = math.pow(10.0, -11.07 - 14.0) / c * xnf2
                hp = hp + c4 / p4 * prqs / fo * dbeta * spi * dop
            else:
                f0, sp = (82259.105 - 15000.0) * c, 100.0 * c
                tb = h["h_cutoffh2plus"]
                if freq4 < f0:
                    cut = (tb[1] - tb[0]) / sp * (freq4 - f0) + tb[0]
                else:
                    ic = min(int((freq4 - f0) / sp), 109)
                    cut = (tb[ic + 1] - tb[ic]) / sp * (freq4 - (ic * sp + f0)) + tb[ic]
                hp = hp + math.pow(10.0, cut - 14.0) / c * xnf2 * spi * dop
    f = gam / pi / (gam * gam + beta * beta) if gam > 0.0 else 0.0
    p1 = _powi(0.9 * y1, 2)
    fns = (p1 + 0.03 * math.sqrt(y1)) / (p1 + 1.0)
    return hp + (prqs * (1.0 + fns) + f) / fo * dbeta * spi * dop


def test_stark_profile_and_hfnm_match_plain_loops(po, tables):
    h = po.HTab.from_tables(tables)
    rng = np.random.default_rng(8)
    for _ in range(400):
        b = float(10.0 ** rng.uniform(-1.0, 3.0))
        p = float(rng.uniform(0.0, 1.0))
        n = int(rng.integers(1, 5))
        m = n + int(rng.integers(1, 8))
        assert po.stark_profile(h, b, p, n, m) == py_stark(tables, b, p, n, m)
    for n in range(1, 8):
        for m in range(1, 30):
            assert po.hfnm(n, m) == py_hfnm(n, m)


@pytest.mark.parametrize("n,m", [(1, 2), (1, 3), (2, 3), (2, 4), (2, 9), (3, 4), (3, 7), (4, 12), (5, 20)])
def test_hprof4_matches_plain_loops(po, tables, n, m):
    """HPROF4 over depths of a cool dwarf to a hot giant and both wings: the C
    oracle and the plain-loop restatement agree bit for bit."""
    h = po.HTab.from_tables(tables)
    rng = np.random.default_rng(n * 100 + m)
    delws = np.concatenate([-np.geomspace(1e-4, 50.0, 40), [0.0], np.geomspace(1e-4, 50.0, 40)])
    if (n, m) == (1, 2):  # Lyman alpha: far red wing through the H2 and H2+ satellite tables
        delws = np.concatenate([delws, np.linspace(1.0, 100.0, 60)])
    for _ in range(6):
        st = dict(xne=10.0 ** rng.uniform(10.0, 16.0), t=rng.uniform(3500.0, 20000.0),
                  xnfp3=10.0 ** rng.uniform(10.0, 16.0), xnh2=10.0 ** rng.uniform(0.0, 14.0),
                  xnf1=10.0 ** rng.uniform(12.0, 17.0), xnf2=10.0 ** rng.uniform(10.0, 15.0),
                  xnfp1=10.0 ** rng.uniform(10.0, 16.0), dop1=rng.uniform(1e-5, 5e-5))
        for dw in delws:
            a = po.hprof4(h, n, m, *st.values(), float(dw))
            b = py_hprof4(tables, n, m, *st.values(), float(dw), po.expi)
            assert a == b, (n, m, dw, a, b)


def py_xlinop_hydrogen(po, h, recs, nrhox, kw, xnfdop1, dopple1, xnfp, xne, hckt, tabcont, iwt, waveset, contx, hatm):
    """XLINOP's record loop for the hydrogen lines (atlas12_modules.f90:
    20177-20199) in plain Python, HPROF4 from the oracle's point function."""
    numnu, nwave = waveset.size, iwt.size - 1
    xl = np.zeros((numnu, kw))
    emerge = [RYDBERG_INF / ((1600.0 / math.pow(xne[j], 2.0 / 15.0)) * (1600.0 / math.pow(xne[j], 2.0 / 15.0)))
              for j in range(nrhox)]
    nucont, nu = 1, 1
    for r in recs:
        wl = float(r["wlvac"])
        while int(r["nbuff"]) >= iwt[nucont - 1]:
            nucont += 1
            if nucont > nwave + 1:
                nucont = nwave + 1
                break
        while wl >= waveset[nu - 1]:
            nu += 1
            if nu >= numnu:
                return xl
        n, m, ncon = int(r["nblo"]), int(r["nbup"]), int(r["ncon"])
        if int(r["itype"]) != -1 or n < 1 or m <= n or m > 100 or ncon < 1 or ncon > 25:
            continue
        eh = h.eh[n - 1] if n <= 10 else h.elim - 109677.583403 / (n * n)
        for j in range(nrhox):
            tc = tabcont[nucont - 1, j]
            center = float(r["gf"]) * (math.exp(-eh * hckt[j]) * xnfdop1[j])
            if center < tc:
                continue
            wcon = 1.0e7 / (contx.ravel()[ncon - 1] - emerge[j])

            def cv_at(iw):
                return center * po.hprof4(h, n, m, xne[j], hatm["t"][j], xnfp[2, j], hatm["xnh2"][j],
                                          hatm["xnf1"][j], hatm["xnf2"][j], xnfp[0, j], dopple1[j],
                                          waveset[iw - 1] - wl)
            for iw in range(nu, min(nu + 2000, numnu) + 1):
                if waveset[iw - 1] < wcon:
                    continue
                cv = cv_at(iw)
                xl[iw - 1, j] += cv
                if cv < tc:
                    break
            for i in range(1, 2001):
                iw = nu - i
                if iw <= 0 or waveset[iw - 1] < wcon:
                    break
                cv = cv_at(iw)
                xl[iw - 1, j] += cv
                if cv < tc:
                    break
    return xl


def test_xlinop_hydrogen_walk_matches_plain_loops(po, tables, small_atm):
    """The oracle's hydrogen-line walk (CENTER, the Lyman/Balmer continuum-edge
    stop of the blue wing, MAX_WING, test after add) against plain loops: bit
    for bit, Balmer lines on both sides of the Balmer edge at 364.7 nm."""
    a = small_atm
    nrhox, kw, nspec = a["nrhox"], a["kw"], a["nspec"]
    h = po.HTab.from_tables(tables)
    ws = np.geomspace(350.0, 420.0, 500)
    cut = atlas.cutoff_grid()
    iwt = atlas.iwavetab(cut)
    tabcont = np.full((cut.size + 1, kw), 1.0e-12)
    rh = 109677.583403
    series = [(2, m) for m in range(6, 26)] + [(3, 40), (1, 2), (12, 90), (2, 2), (2, 101)]
    recs = np.zeros(len(series), po.NLTE_LINE)
    for i, (n, m) in enumerate(series):
        wl = 1e7 / (rh * (1.0 / n ** 2 - 1.0 / m ** 2)) if m > n else 400.0
        recs[i]["wlvac"] = wl if 351.0 < wl < 419.0 else 351.0 + i
        recs[i]["nblo"], recs[i]["nbup"], recs[i]["itype"], recs[i]["ncon"] = n, m, -1, min(n, 25)
        recs[i]["gf"] = 1.0e-12 * (i + 1)
        recs[i]["nbuff"] = int(np.floor(np.log(recs[i]["wlvac"]) / np.log(1.0 + 1.0 / 2000000.0) + 0.5))
    recs = recs[np.argsort(recs["wlvac"], kind="stable")]
    contx = np.zeros((16, 25))
    contx[0, :10] = rh / np.arange(1, 11) ** 2
    rng = np.random.default_rng(21)
    t = np.linspace(4500.0, 12000.0, kw)
    hatm = dict(t=t, xnf1=10.0 ** rng.uniform(14.0, 17.0, kw), xnf2=10.0 ** rng.uniform(11.0, 15.0, kw),
                xnh2=10.0 ** rng.uniform(4.0, 12.0, kw))
    xnfdop = np.zeros((nspec, kw))
    xnfdop[0] = 10.0 ** rng.uniform(13.0, 15.0, kw)
    dopple = np.full((nspec, kw), 1.0)
    dopple[0] = rng.uniform(1.5e-5, 4e-5, kw)
    atm = dict(xnfdop=xnfdop, dopple=dopple, xne=a["xne"], txnxn=np.zeros(kw), hckt=a["hckt"], nrhox=nrhox,
               xnfp=a["xnfp"], rho=a["rho"], htab=h, **hatm)
    got, _ = po.atlas_xlinop(*po.tabvoigt(tables["tabvi"], tables["tabh1"]), po.build_tablog(), recs, atm, tabcont,
                             iwt, ws, contx)
    want = py_xlinop_hydrogen(po, h, recs, nrhox, kw, xnfdop[0], dopple[0], a["xnfp"], a["xne"], a["hckt"], tabcont,
                              iwt, ws, contx, hatm)
    assert np.count_nonzero(want) > 1000
    blue = ws < 1e7 / (rh / 4.0 - 50.0)
    assert np.count_nonzero(want[blue]) < np.count_nonzero(want[~blue])
    np.testing.assert_array_equal(got, want)
