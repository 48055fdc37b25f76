"""SYNTHE's hydrogen lines on the CPU: the Stehle table reader, the synthetic
tables' shapes against the published files' (recorded in the fixture), and
the oracle's restatement of compute_line_opacity's TYPE -1/-2 branch
(synthe_module.f90:3460-3606) with hydrogen_line_profile (:1032-1980)."""
import numpy as np
import pytest

from atlas12_b200 import linelists, synthetic


def _write_fortran(path, arrays):
    with open(path, "wb") as f:
        for a in arrays:
            b = np.ascontiguousarray(a).tobytes()
            f.write(np.int32(len(b)).tobytes() + b + np.int32(len(b)).tobytes())


def test_read_stehle_round_trip(tmp_path):
    """INIT_STARK_TABLES's seven records, PROFILES column-major, back as
    [n_trans, n_dens, n_temps, n_dalpha]; a missing series is None."""
    s = synthetic.stehle_tables()[3]
    nt = s["n_upper_max"] - s["n_upper_min"] + 1
    nd = len(s["density_grid"])
    hdr = np.array([s["n_lower"], s["n_upper_min"], s["n_upper_max"], nd, 10, 60], np.int32)
    prof_f = np.transpose(s["profiles"], (3, 2, 1, 0)).ravel(order="F")  # PROFILES(IA, IT, ID, ITRANS)
    _write_fortran(tmp_path / "stehle_brackett.bin",
                   [hdr, s["density_grid"], s["temp_grid"], s["log_dalpha_grid"], s["max_dens_idx"].astype(np.int32),
                    s["k_alpha"], prof_f])
    got = linelists.read_stehle_dir(str(tmp_path))
    assert got[:3] == [None, None, None]
    g = got[3]
    assert g["profiles"].shape == (nt, nd, 10, 60)
    np.testing.assert_array_equal(g["profiles"], s["profiles"])
    np.testing.assert_array_equal(g["max_dens_idx"], s["max_dens_idx"])
    np.testing.assert_array_equal(g["density_grid"], s["density_grid"])
    (tmp_path / "bad.bin").write_bytes(np.int32(8).tobytes() + b"\0" * 8 + np.int32(4).tobytes())
    with pytest.raises(ValueError, match="markers"):
        linelists.read_stehle(str(tmp_path / "bad.bin"))


def test_synthetic_stehle_tables_have_the_published_shapes(tables):
    dims = tables["stehle_dims"]
    for row, s in zip(dims, synthetic.stehle_tables()):
        assert [s["n_lower"], s["n_upper_min"], s["n_upper_max"], len(s["density_grid"]), s["profiles"].size] == \
            row.tolist()


@pytest.fixture(scope="module")
def balmer(po, tables):
    g = po.synthe_grid(355.0, 700.0, 20000.0)
    atm = synthetic.hydrogen_atmosphere()
    cont = np.full((atm["t"].size, g["length"]), 0.5, np.float32)
    return g, atm, cont, po.HTab.from_tables(tables, "s_")


def test_deuterium_line_reuses_the_hydrogen_convolution(po, balmer):
    """The reference keeps one Stark (x) Voigt convolution between calls and
    rebuilds it only when N, M or the depth change: a hydrogen line right
    after the deuterium line of the same transition is convolved with the
    deuterium line's Doppler width.  With the analytic profile (no tables)
    the two lines add independently."""
    g, atm, cont, hs = balmer
    recs = synthetic.hydrogen_records(640.0, 670.0, g["wbegin"], g["ratio"], series=((2, 3, 4),))
    assert list(recs["itype"]) == [-2, -1]
    st = synthetic.stehle_tables()
    run = lambda r, s: po.synthe_hydrogen_opacity(r, g["length"], g["wbegin"], g["ratio"], 700.0, 0.0, cont, atm,
                                                  hs, s)
    for s, additive in ((None, True), (st, False)):
        both, d_only, h_only = run(recs, s), run(recs[:1], s), run(recs[1:], s)
        assert np.count_nonzero(h_only) > 1000
        err = np.max(np.abs(both - d_only - h_only) / (np.abs(h_only) + 1e-300))
        assert (err < 1e-9) == additive, (s is None, err)


def test_variants_and_tables_change_the_result(po, balmer):
    """Alpha, beta and the tapered higher members all contribute, the Stehle
    path differs from the analytic one, and a record outside EHYD/CONTH is
    refused (the reference aborts)."""
    g, atm, cont, hs = balmer
    recs = synthetic.hydrogen_records(355.0, 700.0, g["wbegin"], g["ratio"], series=((2, 3, 12),), deuterium=False)
    assert set(recs["nbup"]) >= {3, 4, 5, 6}
    kp = po.synthe_hydrogen_opacity(recs, g["length"], g["wbegin"], g["ratio"], 700.0, 0.0, cont, atm, hs)
    stk = po.synthe_hydrogen_opacity(recs, g["length"], g["wbegin"], g["ratio"], 700.0, 0.0, cont, atm, hs,
                                     synthetic.stehle_tables())
    wav = g["wbegin"] * g["ratio"] ** np.arange(g["length"])
    for wl in recs["wlvac"]:
        i = int(np.argmin(np.abs(wav - wl)))
        assert kp[:, i].max() > 0 and stk[:, i].max() > 0
    assert np.max(np.abs(stk - kp)) > 0
    # the higher members stop blueward of WCON >= WSHIFT = 1e7 / (CONTH(2) - RYDBERG_H / 81**2)
    high = recs[recs["nbup"] >= 5]
    kph = po.synthe_hydrogen_opacity(high, g["length"], g["wbegin"], g["ratio"], 700.0, 0.0, cont, atm, hs)
    wshift = 1e7 / (27419.659 - 109677.583403 / 81.0 ** 2)
    assert np.count_nonzero(kph[:, wav < wshift]) == 0 and np.count_nonzero(kph[:, wav < 370.0]) > 0
    bad = recs[:1].copy()
    bad["nbup"] = bad["nblo"]
    with pytest.raises(ValueError):
        po.synthe_hydrogen_opacity(bad, g["length"], g["wbegin"], g["ratio"], 700.0, 0.0, cont, atm, hs)


# ------------------------------------------------------------- the analytic profile in plain Python
def _f32(x):
    return np.float32(x)


def _lya_freq(dw):
    return float(_f32(_f32(82259.10) - _f32(dw)) * _f32(2.99792458e10))


def _lya_cut(tb, freq, x, spacing, start, lo_edge=None):
    c4 = _f32(2.99792458e10)
    spc = _f32(spacing) * c4
    f0 = _f32(_f32(82259.10) - _f32(start)) * c4
    if lo_edge is not None and freq < float(_f32(lo_edge) * c4):
        return None
    if freq < float(f0):
        return (tb[1] - tb[0]) / float(spc) * (freq - float(f0)) + tb[0]
    ic = min(int((freq - float(f0)) / float(spc)), tb.size - 2)
    cf = float(_f32(_f32(ic) * spc) + f0)
    return (tb[ic + 1] - tb[ic]) / float(spc) * (freq - cf) + tb[ic]


def py_synthe_kp(h, n, m, xne, t, xnfph1, xnfph2, xnfhe1, xnfh2, hwdop, delw):
    """hydrogen_line_profile's Peterson/Kurucz path (synthe_module.f90:
    1203-1358, :1698-1892) in plain Python on SYNTHE's tables (s_*)."""
    import math
    from test_oracle_branches import py_hfnm, py_stark
    c4 = float(_f32(2.99792458e10))
    freq_rydh = 109677.583403 * 2.99792458e10
    sqrtpi, pi = 1.7724538509055159, 3.141592653589793
    hh = {k.replace("s_", "h_"): v for k, v in h.items() if k.startswith("s_")}
    xne16 = math.pow(xne, 1.0 / 6.0)
    pp = xne16 * 0.08989 / math.sqrt(t)
    fo = (xne16 * xne16) * (xne16 * xne16) * 1.25e-9
    y1b = 2.0 / (1.0 + 0.012 / t * math.sqrt(xne / t))
    t4 = t / 10000.0
    t43 = math.pow(t4, 0.3)
    y1s, t3nhe, t3nh2 = t43 / xne16, t43 * xnfhe1, t43 * xnfh2
    c1d, c2d = fo * 78940.0 / t, fo * fo / 5.96e-23 / xne
    gcon1, gcon2 = 0.2 + 0.09 * math.sqrt(t4) / (1.0 + xne / 1.0e13), 0.2 / (1.0 + xne / 1.0e15)
    mmn = m - n
    xn, xm = float(n), float(m)
    xn2, xm2 = xn * xn, xm * xm
    xmn2, xm2mn2 = xm2 * xn2, xm2 - xn2
    gnm = xm2mn2 / xmn2
    xknm = h["s_xknmtb"][n - 1, mmn - 1] if (mmn <= 3 and n <= 4) else 5.5e-5 / gnm * xmn2 / (1.0 + 0.13 / mmn)
    y1num = 550.0 if m == 2 else (380.0 if m == 3 else 320.0)
    y1wht = 1.0e14 if mmn <= 3 else 1.0e13
    if mmn <= 2 and n <= 2:
        y1wht = h["s_y1wtm"][n - 1, mmn - 1]
    freqnm = 109677.583403 * 2.99792458e10 * gnm
    dbeta = 2.99792458e18 / (freqnm * freqnm) / xknm
    wavenm = 2.99792458e18 / freqnm
    c1con = xknm / wavenm * gnm * xm2mn2
    c2con = (xknm / wavenm) * (xknm / wavenm)
    radamp = h["s_asumlyman"][m - 1] if n == 1 else h["s_asum"][n - 1] + h["s_asum"][m - 1]
    radamp = radamp / (4.0 * pi) / freqnm
    resont = py_hfnm(1, m) / xm / (1.0 - 1.0 / xm2)
    if n != 1:
        resont = resont + py_hfnm(1, n) / xn / (1.0 - 1.0 / xn2)
    resont = resont * 3.579e-24 / gnm
    vdw = 4.45e-26 / gnm * math.pow(xm2 * (7.0 * xm2 + 5.0), 0.4)
    stark = 1.6678e-18 * freqnm * xknm
    if n > 4 or m > 10:
        fs = [(0.0, 1.0)]
    elif mmn == 1:
        k0 = h["s_istal"][n - 1] - 1
        fs = [(h["s_stalph"][k0 + i] * 1.0e7, h["s_stwtal"][k0 + i] / xn2 / 3.0) for i in range(h["s_lnghal"][n - 1])]
    else:
        fs = [(h["s_stcomp"][i, n - 1] * 1.0e7, h["s_stcpwt"][i, n - 1] / xn2) for i in range(h["s_lncomp"][n - 1])]
    freq = 2.99792458e18 / (wavenm + delw * 10.0)
    dl = abs(freq - freqnm)
    hwstk = stark * fo
    hwvdw = vdw * t3nhe + 2.0 * vdw * t3nh2
    hwres = resont * xnfph1 * 2.0
    hwlor = hwres + hwvdw + radamp
    dop = freqnm * hwdop
    nwid = 1
    if hwdop < hwstk or hwdop < hwlor:
        nwid = 3 if hwlor < hwstk else 2
    core = dl <= freqnm * max(hwdop, hwlor, hwstk)
    hp = 0.0
    if not core or nwid == 1:
        for fe, fw in fs:
            d = abs(freq - freqnm - fe) / dop
            if d <= 7.0:
                hp = hp + math.exp(-d * d) * fw
        if core:
            return hp
    if not core or nwid == 2:
        if n == 1 and m == 2:
            hw4 = hwres * 4.0
            hhw = freqnm * (hw4 + hwvdw + radamp)
            if freq > _lya_freq(4000.0):
                pres = hw4 * freqnm / pi / (dl * dl + hhw * hhw) * sqrtpi * dop
            else:
                cv = _lya_cut(h["s_cutoffh2"], freq, None, 200.0, 22000.0, lo_edge=50000.0)
                pres = 0.0 if cv is None else math.pow(10.0, cv - 14.0) * float(_f32(xnfph1)) * 2.0 / c4 * sqrtpi * dop
            prad = 0.0
            if freq > float(_f32(2.4190611e15)) and freq < float(_f32(0.77)) * freq_rydh:
                prad = radamp * freqnm / pi / (dl * dl + hhw * hhw) * sqrtpi * dop
            pvdw = hwvdw * freqnm / pi / (dl * dl + hhw * hhw) * sqrtpi * dop
            if freq < float(_f32(1.8e15)):
                pvdw = 0.0
            hp = hp + pres + prad + pvdw
        else:
            hhw = freqnm * hwlor
            top = hhw
            for mm, a, b in ((3, 0.885, 0.890), (4, 0.936, 0.938), (5, 0.959, 0.961)):
                if n == 1 and m == mm and float(_f32(a)) * freq_rydh < freq < float(_f32(b)) * freq_rydh:
                    top = hhw - freqnm * radamp
            hp = hp + top / pi / (dl * dl + hhw * hhw) * sqrtpi * dop
        if core:
            return hp
    wty1 = 1.0 / (1.0 + xne / y1wht)
    y1scal = y1num * y1s * wty1 + y1b * (1.0 - wty1)
    c1, c2 = c1d * c1con * y1scal, c2d * c2con
    g1 = 6.77 * math.sqrt(c1)
    gnot = g1 * max(0.0, 0.2114 + math.log(math.sqrt(c2) / c1)) * (1.0 - gcon1 - gcon2)
    beta = abs(dl) / fo * dbeta
    y1, y2 = c1 * beta, c2 * (beta * beta)

    def e1(x):
        if x <= 0.0:
            return 0.0
        if x <= 1.0:
            return -math.log(x) - 0.57721566 + x * (0.99999193 + x * (-0.24991055 + x * (0.05519968 + x * (
                -0.00976004 + x * 0.00107857))))
        if x <= 30.0:
            return (x * (x + 2.334733) + 0.25062) / (x * (x + 3.330657) + 1.681534) / x * math.exp(-x)
        return 0.0
    gam = gnot
    if not (y2 <= 1.0e-4 and y1 <= 1.0e-5):
        q = 90.0 * y1
        gam = g1 * (0.5 * math.exp(-min(80.0, y1)) + e1(y1) - 0.5 * e1(y2)) * \
            (1.0 - gcon1 / (1.0 + (q * q) * q) - gcon2 / (1.0 + 2000.0 * y1))
        if gam <= 1.0e-20:
            gam = 0.0
    prqs = py_stark(hh, beta, pp, n, m)
    if m == 2:
        prqs = prqs * 0.5
        if _lya_freq(20000.0) <= freq <= _lya_freq(4000.0):
            cv = _lya_cut(h["s_cutoffh2plus"], freq, None, 100.0, 15000.0)
            hp = hp + math.pow(10.0, cv - 14.0) / c4 * float(_f32(xnfph2)) * sqrtpi * dop
        elif freq > _lya_freq(4000.0):
            b4 = 4000.0 * c4 / fo * dbeta
            p4 = py_stark(hh, b4, pp, n, m) * 0.5 / fo * dbeta
            c4000 = math.pow(10.0, -11.07 - 14.0) / c4 * xnfph2
            hp = hp + c4000 / p4 * prqs / fo * dbeta * sqrtpi * dop
    f = gam / pi / (gam * gam + beta * beta) if gam > 0.0 else 0.0
    p1 = (0.9 * y1) * (0.9 * y1)
    fns = (p1 + 0.03 * math.sqrt(y1)) / (p1 + 1.0)
    return hp + (prqs * (1.0 + fns) + f) / fo * dbeta * sqrtpi * dop


@pytest.mark.parametrize("n,m", [(1, 2), (1, 3), (1, 4), (1, 5), (2, 3), (2, 4), (2, 9), (3, 4), (3, 12), (4, 7),
                                 (5, 9)])
def test_synthe_analytic_profile_matches_plain_loops(po, tables, n, m):
    """The oracle's K-P profile against the plain-Python restatement, bit for
    bit, over a cool dwarf to a hot giant, the core to 50 nm and, for the
    Lyman lines, the satellite windows and the radiative-damping notches."""
    h = po.HTab.from_tables(tables, "s_")
    rng = np.random.default_rng(100 * n + m)
    dws = np.concatenate([-np.geomspace(1e-4, 50.0, 30), [0.0], np.geomspace(1e-4, 50.0, 30)])
    if n == 1:
        dws = np.concatenate([dws, np.linspace(-15.0, 90.0, 80)])
    for _ in range(5):
        st = (10.0 ** rng.uniform(10.0, 16.0), rng.uniform(3500.0, 20000.0), 10.0 ** rng.uniform(12.0, 17.0),
              10.0 ** rng.uniform(10.0, 15.0), 10.0 ** rng.uniform(11.0, 16.0), 10.0 ** rng.uniform(0.0, 12.0),
              rng.uniform(1e-5, 5e-5))
        for dw in dws:
            a = po.synthe_hprof_kp(h, n, m, *st, float(dw))
            b = py_synthe_kp(tables, n, m, *st, float(dw))
            assert a == b, (n, m, dw, a, b)


def py_synthe_hydrogen_walk(po, h, recs, length, wbegin, ratio, wlend, cont, atm):
    """compute_line_opacity's TYPE -1/-2 walks (synthe_module.f90:3460-3606)
    in plain Python with the oracle's analytic profile point function."""
    import math
    rydh, cutoff = 109677.583403, 1.0e-3
    conth = [109678.764, 27419.659, 12186.462, 6854.871, 4387.113, 3046.604, 2238.320, 1713.713, 1354.044,
             1096.776, 906.426, 761.650, 648.980, 559.579, 487.456]
    eh = [h.eh[k] for k in range(10)] + [h.elim - rydh / (float(k) * float(k)) for k in range(11, 101)]
    alphahyd = [1.0e7 / (eh[k + 1] - eh[k]) for k in range(99)]
    nrhox = atm["xne"].size
    out = np.zeros((nrhox, length))
    from test_oracle_branches import atlas_powi
    for j in range(nrhox):
        inglis = np.float32(1600.0 / math.pow(atm["xne"][j], float(np.float32(2.0) / np.float32(15.0))))
        nmerge = np.float32(inglis - np.float32(1.5))
        emergeh = rydh / (float(nmerge) * float(nmerge))
        c = cont[j].astype(np.float64)
        for r in recs:
            n, m, ncon, nbuff = int(r["nblo"]), int(r["nbup"]), int(r["ncon"]), int(r["nbuff"])
            wl = float(r["wlvac"])
            kappa0 = float(r["gf"]) * atm["xnfdop"][j, 0]
            kapmin = c[(length if m == 2 else min(max(nbuff, 1), length)) - 1] * cutoff
            if kappa0 < kapmin:
                continue
            dopph = np.float32(atm["dopple"][j, 0])
            if r["itype"] == -2:
                dopph = np.float32(dopph / np.float32(1.4142))
            kappa0 = kappa0 * math.exp(-float(r["elo"]) * atm["hckt"][j])
            if kappa0 < kapmin:
                continue

            def K(wave):
                return kappa0 * po.synthe_hprof_kp(h, n, m, atm["xne"][j], atm["t"][j], atm["xnfph1"][j],
                                                   atm["xnfph2"][j], atm["xnfhe1"][j], atm["xnfh2"][j], float(dopph),
                                                   wave - wl)
            minred = max(1, nbuff)
            general = not (ncon == 0 or m == n + 1) and m != n + 2
            wcon = wtail = 0.0
            blue = True
            if ncon == 0 or m == n + 1:
                if wl <= wlend:
                    wave = wbegin * atlas_powi(ratio, minred - 1)
                    for ib in range(minred, length + 1):
                        k = K(wave)
                        out[j, ib - 1] += k
                        if k < c[ib - 1] * cutoff:
                            break
                        wave = wave * ratio
                    blue = not (minred == 1 or wl < wbegin)
            elif m == n + 2:
                if wl <= wlend:
                    wave = wbegin * atlas_powi(ratio, minred - 1)
                    exited = False
                    for ib in range(minred, length + 1):
                        if wave > alphahyd[n - 1]:
                            exited = True
                            break
                        k = K(wave)
                        out[j, ib - 1] += k
                        if k < c[ib - 1] * cutoff:
                            exited = True
                            break
                        wave = wave * ratio
                    if not exited and (minred == 1 or wl < wbegin or nbuff < 1):
                        blue = False
                elif nbuff < 1:
                    blue = False
            else:
                wshift = 1.0e7 / (conth[ncon - 1] - rydh / (81.0 * 81.0))
                wmerge = 1.0e7 / (conth[ncon - 1] - emergeh)
                if wmerge < 0.0:
                    wmerge = wshift + wshift
                wcon = max(wshift, wmerge)
                wtail = 1.0e7 / (1.0e7 / wcon - 500.0)
                wcon = min(wshift + wshift, wcon)
                if wtail < 0.0:
                    wtail = wcon + wcon
                wtail = min(wcon + wcon, wtail)
                if wl <= wlend:
                    if wcon > wlend:
                        continue
                    if wbegin <= alphahyd[n - 1]:
                        wave = wbegin * atlas_powi(ratio, minred - 1)
                        if wave >= wcon:
                            k = K(wave)
                            if k >= c[min(minred, length) - 1] * cutoff:
                                if wave < wtail:
                                    k = k * ((wave - wcon) / (wtail - wcon))
                                if minred <= length:
                                    out[j, minred - 1] += k
                                wave = wave * ratio
                                for ib in range(minred + 1, length + 1):
                                    if wave >= wcon:
                                        k = K(wave)
                                        if wave < wtail:
                                            k = k * ((wave - wcon) / (wtail - wcon))
                                        out[j, ib - 1] += k
                                        if k < c[ib - 1] * cutoff:
                                            break
                                    wave = wave * ratio
                        if minred == 1:
                            continue
                    if wl < wbegin:
                        continue
            if not blue:
                continue
            ib = min(length + 1, nbuff)
            wave = wbegin * atlas_powi(ratio, ib - 1)
            for _ in range(ib - 1):
                ib -= 1
                wave = wave / ratio
                if general and wave < wcon:
                    break
                k = K(wave)
                if general and wave < wtail:
                    k = k * ((wave - wcon) / (wtail - wcon))
                out[j, ib - 1] += k
                if k < c[ib - 1] * cutoff:
                    break
    return out


def test_synthe_hydrogen_walks_match_plain_loops(po, tables):
    """The oracle's alpha, beta and tapered walks (the analytic profile)
    against plain loops, bit for bit: Balmer lines with deuterium partners on
    a window cut through the series limit and H alpha's red wing."""
    g = po.synthe_grid(362.0, 420.0, 8000.0)
    atm = synthetic.hydrogen_atmosphere()
    atm = {k: (v[::6] if np.ndim(v) else v) for k, v in atm.items()}
    nr = atm["xne"].size
    rng = np.random.default_rng(4)
    cont = (10.0 ** rng.uniform(-1.0, 0.5, (nr, g["length"]))).astype(np.float32)
    recs = synthetic.hydrogen_records(300.0, 700.0, g["wbegin"], g["ratio"], series=((2, 3, 14),))
    h = po.HTab.from_tables(tables, "s_")
    got = po.synthe_hydrogen_opacity(recs, g["length"], g["wbegin"], g["ratio"], 420.0, 0.0, cont, atm, h)
    want = py_synthe_hydrogen_walk(po, h, recs, g["length"], g["wbegin"], g["ratio"], 420.0, cont, atm)
    assert np.count_nonzero(want) > 0.2 * want.size
    np.testing.assert_array_equal(got, want)


def py_synthe_stehle(po, h, stl, n, m, xne, t, xnfph1, xnfph2, xnfhe1, xnfh2, dconv, dopph, delw):
    """hydrogen_line_profile's Stehle path (synthe_module.f90:1414-1696, with
    interp_stark_at :2007-2037) in plain Python: the table bilinear in
    (log Ne, T), the Stark (x) Voigt convolution on its two-zone grid built
    with Doppler width dconv, then the log-log evaluation with dopph.  The
    Voigt kernel is the oracle's (pinned on its own)."""
    import math
    from test_oracle_branches import py_hfnm
    rydh, cang, pi, sqrtpi = 109677.583403, 2.99792458e18, 3.141592653589793, 1.7724538509055159
    S = stl[n - 1]
    xn, xm = float(n), float(m)
    xn2, xm2 = xn * xn, xm * xm
    gnm = (xm2 - xn2) / (xm2 * xn2)
    freqnm = rydh * 2.99792458e10 * gnm
    wavenm = cang / freqnm
    radamp = (h["s_asumlyman"][m - 1] if n == 1 else h["s_asum"][n - 1] + h["s_asum"][m - 1]) / (4.0 * pi) / freqnm
    resont = py_hfnm(1, m) / xm / (1.0 - 1.0 / xm2)
    if n != 1:
        resont = resont + py_hfnm(1, n) / xn / (1.0 - 1.0 / xn2)
    resont = resont * 3.579e-24 / gnm
    vdw = 4.45e-26 / gnm * math.pow(xm2 * (7.0 * xm2 + 5.0), 0.4)
    t43 = math.pow(t / 10000.0, 0.3)
    hwvdw = vdw * (t43 * xnfhe1) + 2.0 * vdw * (t43 * xnfh2)
    hwres = resont * xnfph1 * 2.0
    hwlor_conv = hwres * 4.0 + hwvdw + radamp if (n == 1 and m == 2) else hwres + hwvdw + radamp
    lam0 = 1.0e8 / rydh * ((xn * xm) * (xn * xm)) / ((xm - xn) * (xm + xn))
    itr = m - S["n_upper_min"] + 1
    dg, tg, lg = S["density_grid"], S["temp_grid"], S["log_dalpha_grid"]
    nd = len(dg)
    dcap = dg[S["max_dens_idx"][itr - 1] - 1]
    ne = xne if xne < dcap else dcap
    F0 = 1.25e-9 * math.pow(ne, 2.0 / 3.0)
    dag = [math.pow(10.0, x) for x in lg]
    id1 = next((i for i in range(1, nd) if ne <= dg[i]), nd)
    id1 = max(1, min(nd - 1, id1))
    fd = (math.log10(ne) - math.log10(dg[id1 - 1])) / (math.log10(dg[id1]) - math.log10(dg[id1 - 1]))
    fd = min(max(fd, 0.0), 1.0)
    it1 = min(next((i for i in range(1, 10) if t <= tg[i]), 10), 9)
    ft = min(max((t - tg[it1 - 1]) / (tg[it1] - tg[it1 - 1]), 0.0), 1.0)
    P = S["profiles"][itr - 1]
    sp = []
    for ia in range(60):
        v00, v01, v10, v11 = P[id1 - 1, it1 - 1, ia], P[id1 - 1, it1, ia], P[id1, it1 - 1, ia], P[id1, it1, ia]
        if v00 > 0 and v01 > 0 and v10 > 0 and v11 > 0:
            sp.append(math.exp(math.log(v00) * (1 - fd) * (1 - ft) + math.log(v01) * (1 - fd) * ft +
                               math.log(v10) * fd * (1 - ft) + math.log(v11) * fd * ft))
        else:
            sp.append(v00 * (1 - fd) * (1 - ft) + v01 * (1 - fd) * ft + v10 * fd * (1 - ft) + v11 * fd * ft)

    def interp(da):
        if da >= math.pow(10.0, lg[59]):
            return sp[59]
        x = math.log10(da)
        i = min(next((k for k in range(1, 60) if x <= lg[k]), 60), 59)
        fr = (x - lg[i - 1]) / (lg[i] - lg[i - 1])
        if sp[i - 1] > 0.0 and sp[i] > 0.0:
            return math.exp(math.log(sp[i - 1]) * (1.0 - fr) + math.log(sp[i]) * fr)
        return sp[i - 1] * (1.0 - fr) + sp[i] * fr
    dopd = lam0 * lam0 / cang * freqnm * dconv / F0
    lord = lam0 * lam0 / cang * freqnm * hwlor_conv / F0
    va = float(np.float32(lord / dopd))
    dx = dopd / 3.0
    dlog = (lg[59] - lg[0]) / 59.0
    nlog = max(next((ia - 1 for ia in range(1, 61) if dag[ia - 1] * dlog * math.log(10.0) > dx), 60), 1)
    dtr = dag[nlog - 1]
    nw, dwm = 200, dtr + 200.0 * dx
    if dwm > dag[59]:
        dwm = dag[59]
        nw = max(int((dwm - dtr) / dx), 0)
    if 2 * nw + 2 * nlog + 1 > 600:
        nw = (600 - 2 * nlog - 1) // 2
        dwm = dtr + float(nw) * dx
    grid = [(-(dtr + float(iw) * dx), interp(dtr + float(iw) * dx)) for iw in range(nw, 0, -1)]
    grid += [(-dag[ia - 1], sp[ia - 1]) for ia in range(nlog, 0, -1)] + [(0.0, sp[0])]
    grid += [(dag[ia - 1], sp[ia - 1]) for ia in range(1, nlog + 1)]
    grid += [(dtr + float(iw) * dx, interp(dtr + float(iw) * dx)) for iw in range(1, nw + 1)]
    cda = [g[0] for g in grid]
    ic = len(cda)
    cst = [cda[1] - cda[0]] + [0.5 * (cda[k + 1] - cda[k - 1]) for k in range(1, ic - 1)] + [cda[-1] - cda[-2]]
    prof = []
    for ia in range(60):
        da = dag[ia]
        if da > dwm and dwm > 0.0:
            prof.append(sp[ia] + va * dopd / (pi * (da * da)))
        else:
            s = 0.0
            for (x, pv), w in zip(grid, cst):
                kern = float(np.float32(po.voigt_weideman(float(np.float32((da - x) / dopd)), va)))
                s = s + pv * kern * w
            prof.append(s / (dopd * sqrtpi))
    freq = cang / (wavenm + delw * 10.0)
    dac = lam0 * lam0 / cang * abs(freq - freqnm) / F0
    if dac <= math.pow(10.0, lg[0]):
        I = prof[0]
    elif dac >= math.pow(10.0, lg[59]):
        I = S["k_alpha"][m - S["n_upper_min"]] / math.pow(dac, 2.5) + va * dopd / (pi * (dac * dac))
    else:
        x = math.log10(dac)
        i = min(next((k for k in range(1, 60) if x <= lg[k]), 60), 59)
        fa = (x - lg[i - 1]) / (lg[i] - lg[i - 1])
        p1, p2 = prof[i - 1], prof[i]
        I = math.exp(math.log(p1) * (1.0 - fa) + math.log(p2) * fa) if (p1 > 0.0 and p2 > 0.0) else \
            p1 * (1.0 - fa) + p2 * fa
    return I * (lam0 * lam0) / (cang * F0) * sqrtpi * (freqnm * dopph)


@pytest.mark.parametrize("n,m", [(2, 3), (2, 7), (3, 5), (4, 6)])
def test_synthe_stehle_profile_matches_plain_loops(po, tables, n, m):
    """The oracle's Stehle path (tables, convolution grid, Voigt kernel sums,
    log-log evaluation) against the plain-Python restatement, bit for bit,
    with the convolution built from another line's Doppler width."""
    h = po.HTab.from_tables(tables, "s_")
    stl = synthetic.stehle_tables()
    rng = np.random.default_rng(10 * n + m)
    for _ in range(3):
        xne = 10.0 ** rng.uniform(10.5, 15.5)
        st = (xne, rng.uniform(4000.0, 30000.0), 10.0 ** rng.uniform(12.0, 17.0), 10.0 ** rng.uniform(10.0, 15.0),
              10.0 ** rng.uniform(11.0, 16.0), 10.0 ** rng.uniform(0.0, 12.0))
        dconv, dop = float(np.float32(rng.uniform(1e-5, 5e-5))), float(np.float32(rng.uniform(1e-5, 5e-5)))
        for dw in (0.0, 1e-4, 3e-3, 0.05, 0.4, 2.0, 12.0, -0.02, -1.5):
            a = po.synthe_hprof_stehle(h, stl, n, m, *st, dconv, dop, dw)
            b = py_synthe_stehle(po, tables, stl, n, m, *st, dconv, dop, dw)
            assert a == b, (n, m, dw, a, b)


def test_hydrogen_records_follow_the_rydberg_series(po):
    """The synthetic unit-19 hydrogen records: Rydberg wavelengths, deuterium
    just blueward, NCON set past beta, grid indices that bracket WLVAC."""
    g = po.synthe_grid(90.0, 2000.0, 5000.0)
    recs = synthetic.hydrogen_records(90.0, 2000.0, g["wbegin"], g["ratio"])
    h = recs[recs["itype"] == -1]
    n, m = h["nblo"].astype(float), h["nbup"].astype(float)
    np.testing.assert_allclose(h["wlvac"], 1e7 / (109677.583403 * (1 / n ** 2 - 1 / m ** 2)), rtol=1e-12)
    assert np.all(np.diff(recs["wlvac"]) >= 0)
    assert np.all((recs["ncon"] > 0) == (recs["nbup"] > recs["nblo"] + 2))
    d = recs[recs["itype"] == -2]
    assert len(d) == len(h) and np.all(d["gf"] < 1e-3 * np.max(h["gf"]))
    lo = g["wbegin"] * g["ratio"] ** (recs["nbuff"].astype(float) - 1.5)
    hi = g["wbegin"] * g["ratio"] ** (recs["nbuff"].astype(float) - 0.5)
    assert np.all((lo <= recs["wlvac"] * (1 + 1e-12)) & (recs["wlvac"] <= hi * (1 + 1e-12)))
