"""ATLAS12 hot path on the GPU (through the C ABI) against the CPU oracle.

Tolerances (all FP64 on both sides; differences come from FMA contraction and
the order of the FP64 atomic/partial sums):
  * XLINES: relative 1e-9 per element (a flipped wing-stop decision would be ~1e-3)
  * RT-pass sums: relative 1e-9; HNU(1) per frequency: relative 1e-6
  * finish (T, RHOX, P after TCORR(3) and the remap): relative 1e-9
"""
import numpy as np
import pytest

from atlas12_b200 import _lib, atlas, surrogate, synthetic

pytestmark = pytest.mark.gpu

NSPEC = 270


@pytest.fixture(scope="module")
def atlas_case():
    ross = surrogate.RossTable()
    m = surrogate.grey_model(5777.0, 4.44, ross=ross)
    pop = surrogate.populations(m["t"], m["p"], 1.5)
    nr = m["t"].size
    xnfdop = np.zeros((NSPEC, nr))
    dopple = np.ones((NSPEC, nr))
    nsp = min(NSPEC, pop["xnfp"].shape[1])
    xd = np.where(pop["dopple"] > 0, pop["xnfp"] / np.maximum(pop["dopple"], 1e-300) / pop["rho"][:, None], 0.0)
    xnfdop[:nsp] = xd[:, :nsp].T
    dopple[:nsp] = np.where(pop["dopple"][:, :nsp].T > 0, pop["dopple"][:, :nsp].T, 1.0)
    t = m["t"]
    hkt = surrogate.HPLANCK / (surrogate.KBOL * t)
    hckt = hkt * surrogate.CLIGHT
    txnxn = (pop["nh"] * (1 - pop["xh"]) + 0.42 * 0.085 * pop["nh"]) * (t / 1e4) ** 0.3
    ws, rc = synthetic.geometric_waveset(9.0, 160000.0, 3000)
    cut = atlas.cutoff_grid()
    iw = atlas.iwavetab(cut)
    ka, sg = surrogate.continuum_opacity(cut, t, m["p"], pop)
    stim_c = 1.0 - np.exp(-(surrogate.CLIGHT_NMS / cut)[:, None] * hkt[None, :])
    tab = (ka + sg) * atlas.LINE_CUTOFF / stim_c
    tab[cut <= ws[0]] = (1e10 + 0.0) * atlas.LINE_CUTOFF / stim_c[cut <= ws[0]]
    tabcont = np.vstack([tab, tab[-1:]])
    acont, sigmac = surrogate.continuum_opacity(ws, t, m["p"], pop)
    lines = synthetic.atlas_lines(20000, ws[2], ws[-3], seed=4)
    return dict(m=m, pop=pop, xnfdop=xnfdop, dopple=dopple, xne=pop["xne"], txnxn=txnxn, hkt=hkt, hckt=hckt,
                ws=ws, rc=rc, cut=cut, iw=iw, tabcont=tabcont, acont=acont, sigmac=sigmac, lines=lines, ross=ross)


@pytest.fixture(scope="module")
def h_tables(po, tables):
    return po.tabvoigt(tables["tabvi"], tables["tabh1"])


@pytest.fixture(scope="module")
def oracle_linop(po, atlas_case, h_tables):
    c = atlas_case
    atm = dict(xnfdop=c["xnfdop"], dopple=c["dopple"], xne=c["xne"], txnxn=c["txnxn"], hckt=c["hckt"])
    return po.atlas_linop1(*h_tables, po.build_tablog(), c["lines"], atm, c["tabcont"], c["iw"], c["ws"])


@pytest.mark.parametrize("prec,tol", [(_lib.PREC_FP64, 1e-9), (_lib.PREC_MIXED, 1e-6)])
def test_linop_matches_oracle(gpu_ctx, tables, atlas_case, h_tables, oracle_linop, prec, tol):
    """FP64: every element to 1e-9.  Mixed precision (FP32 profile values,
    FP64 index, regime and stop decisions, FP64 sums): the same wing points
    (identical nonzero pattern) and every element to 1e-6."""
    c = atlas_case
    A = atlas.Atlas(gpu_ctx, tables, *h_tables)
    gpu_ctx.set_precision(prec)
    try:
        xl, used = A.linop1(c["lines"], 72, c["xnfdop"], c["dopple"], c["xne"], c["txnxn"], c["hckt"],
                            c["tabcont"], c["iw"], c["ws"])
    finally:
        gpu_ctx.set_precision(_lib.PREC_MIXED)
    ref, ref_used = oracle_linop
    assert used == ref_used and used > 100
    assert np.count_nonzero(ref) > 1000
    np.testing.assert_array_equal(xl != 0, ref != 0)
    scale = np.maximum(np.abs(ref), 1e-300)
    assert np.max(np.abs(xl - ref) / scale) < tol


def test_linop_bit_identical_run_to_run(gpu_ctx, tables, atlas_case, h_tables):
    """XLINES is an exact fixed-point sum rounded once: the same inputs give
    the same bits however the GPU orders the adds (both precisions)."""
    c = atlas_case
    A = atlas.Atlas(gpu_ctx, tables, *h_tables)
    for prec in (_lib.PREC_FP64, _lib.PREC_MIXED):
        gpu_ctx.set_precision(prec)
        try:
            runs = [A.linop1(c["lines"], 72, c["xnfdop"], c["dopple"], c["xne"], c["txnxn"], c["hckt"],
                             c["tabcont"], c["iw"], c["ws"])[0] for _ in range(3)]
        finally:
            gpu_ctx.set_precision(_lib.PREC_MIXED)
        for r in runs[1:]:
            assert np.array_equal(r.view(np.uint64), runs[0].view(np.uint64))


def test_linop_empty_and_out_of_grid(gpu_ctx, tables, atlas_case, h_tables, po):
    c = atlas_case
    A = atlas.Atlas(gpu_ctx, tables, *h_tables)
    xl, used = A.linop1(np.zeros((0, 4), np.int32), 72, c["xnfdop"], c["dopple"], c["xne"], c["txnxn"], c["hckt"],
                        c["tabcont"], c["iw"], c["ws"])
    assert used == 0 and not xl.any()
    # lines outside START..STOP and with an out-of-range species are skipped
    ld = c["lines"][:50].copy()
    ld[:10, 0] = 1000                            # ~ 1.0005 nm, blue of the grid
    ld[10:20, 1] = (ld[10:20, 1] & ~0xffff) | 9999  # NELION = 999 > nspec
    atm = dict(xnfdop=c["xnfdop"], dopple=c["dopple"], xne=c["xne"], txnxn=c["txnxn"], hckt=c["hckt"])
    ref, ru = po.atlas_linop1(*h_tables, po.build_tablog(), ld, atm, c["tabcont"], c["iw"], c["ws"])
    got, gu = A.linop1(ld, 72, c["xnfdop"], c["dopple"], c["xne"], c["txnxn"], c["hckt"], c["tabcont"], c["iw"],
                       c["ws"])
    assert gu == ru
    np.testing.assert_allclose(got, ref, rtol=1e-6, atol=0)  # mixed precision (FP32 profile values)


def test_rt_pass_matches_oracle(po, ops, gpu_ctx, tables, atlas_case, oracle_linop):
    c = atlas_case
    xl = oracle_linop[0]
    m = c["m"]
    ref, rhs = po.atlas_rt_pass(ops, c["ws"], c["rc"], c["acont"], c["sigmac"], xl, m["rhox"], m["t"], c["hkt"],
                                5777.0)
    A = atlas.Atlas(gpu_ctx, tables)
    got, ghs = A.rt_pass(c["ws"], c["rc"], c["acont"], c["sigmac"], xl, m["rhox"], m["t"], c["hkt"], 5777.0)
    for k in atlas.ACC_NAMES:
        np.testing.assert_allclose(got[k], ref[k], rtol=1e-9, err_msg=k)
    assert abs(got["pradk0"] - ref["pradk0"]) <= 1e-9 * abs(ref["pradk0"])
    # per-frequency H(1): where the Eddington sweep runs, its stop test (summed
    # error < 1e-5) is summed in a different order, which can change the last
    # sweep and H(1) by up to ~1e-7
    np.testing.assert_allclose(ghs, rhs, rtol=1e-6)


def test_finish_matches_oracle(po, ops, gpu_ctx, tables, atlas_case, oracle_linop):
    c = atlas_case
    m = c["m"]
    acc, _ = po.atlas_rt_pass(ops, c["ws"], c["rc"], c["acont"], c["sigmac"], oracle_linop[0], m["rhox"], m["t"],
                              c["hkt"], 5777.0)
    nr = m["t"].size

    def state():
        return dict(t=m["t"].copy(), rhox=m["rhox"].copy(), p=m["p"].copy(), xne=c["xne"].copy(),
                    abross=np.zeros(nr), prad=np.zeros(nr), vturb=np.full(nr, 1.5e5), pturb=np.zeros(nr),
                    tauros=m["tauros"].copy(), accrad=np.zeros(nr), raden=np.zeros(nr), oldt1=np.zeros(nr),
                    teff=5777.0, grav=m["grav"])

    A = atlas.Atlas(gpu_ctx, tables)
    store_o, store_g = po.RossStore(), atlas.RossStore()
    for it in (1, 2, 3):
        so, sg = state(), state()
        so["oldt1"] = np.linspace(-20, 30, nr)  # OLDT1 is updated in place: one copy each
        sg["oldt1"] = np.linspace(-20, 30, nr)
        eo, oo = po.atlas_finish(so, acc, it, store_o)
        eg, og = A.finish(sg, acc, it, store_g)
        assert store_g.n == store_o.n == 72 * it
        np.testing.assert_allclose(store_g.k[:store_g.n], store_o.k[:store_o.n], rtol=1e-12)
        assert abs(eg - eo) <= 1e-9 * max(eo, 1e-3)
        for k in ("t", "rhox", "p", "xne", "prad", "tauros"):
            np.testing.assert_allclose(sg[k], so[k], rtol=1e-9, err_msg=k)
        for k in ("flxerr", "dtflux", "dtlamb", "t1"):
            np.testing.assert_allclose(og[k], oo[k], rtol=1e-8, atol=1e-9, err_msg=k)


def test_model_iteration_reduces_flux_error(gpu_ctx, tables):
    ws, rc = synthetic.geometric_waveset(9.0, 160000.0, 6000)
    lines = synthetic.atlas_lines(20000, ws[2], ws[-3], seed=4)
    model = atlas.AtlasModel(gpu_ctx, tables, teff=5777.0, logg=4.44, linedata=lines, waveset=ws, rcoset=rc)
    n, hist = model.iterate(max_iter=12, tol_percent=0.0, graph=True)
    s = model.structure()
    model.close()
    assert n == 12 and np.all(np.isfinite(hist))
    assert hist[-1] < 0.5 * hist[0], hist
    assert np.all(np.diff(s["t"]) > 0) and s["t"].min() >= 1200.0


@pytest.mark.parametrize("prec,tol", [(_lib.PREC_FP64, 1e-9), (_lib.PREC_MIXED, 1e-6)])
def test_xlinop_normal_branch_matches_oracle(po, gpu_ctx, tables, atlas_case, h_tables, prec, tol):
    """XLINOP's normal-line branch on unit-19 records over a grid fine enough
    that strong lines walk past LINOP1's 100 points (up to MAX_WING = 2000),
    with continuum-edge cutoffs, TYPE 2 skips and other types counted.
    Same tolerances and nonzero pattern as LINOP1."""
    c = atlas_case
    ws = np.geomspace(300.0, 600.0, 4000)
    recs = synthetic.nlte_records(5000, 300.5, 599.5, seed=6, strong=0.1)
    contx = synthetic.contx_table()
    atm = dict(xnfdop=c["xnfdop"], dopple=c["dopple"], xne=c["xne"], txnxn=c["txnxn"], hckt=c["hckt"])
    base = np.zeros((ws.size, 72))
    base[::7, 3] = 1e-3  # XLINOP adds into the LINOP1 result
    ref, nread = po.atlas_xlinop(*h_tables, po.build_tablog(), recs, atm, c["tabcont"], c["iw"], ws, contx, base)
    nocut, _ = po.atlas_xlinop(*h_tables, po.build_tablog(), recs, atm, c["tabcont"], c["iw"], ws,
                               np.zeros_like(contx), base)
    assert nread > 4000
    assert np.count_nonzero(ref != base) > 20000
    assert np.sum(nocut) > np.sum(ref)  # the continuum-edge cutoff removed blue wings
    # some walks are longer than LINOP1's 100 points
    rows = np.nonzero(np.any(ref != base, axis=1))[0]
    assert np.max(np.diff(rows)) < 50 and np.count_nonzero(np.any(ref != base, axis=1)) > 2000
    A = atlas.Atlas(gpu_ctx, tables, *h_tables)
    gpu_ctx.set_precision(prec)
    try:
        got, other = A.xlinop(recs, 72, c["xnfdop"], c["dopple"], c["xne"], c["txnxn"], c["hckt"], c["tabcont"],
                              c["iw"], ws, contx, base)
    finally:
        gpu_ctx.set_precision(_lib.PREC_MIXED)
    assert other == int(np.sum(recs["itype"] == 1))
    np.testing.assert_array_equal(got != base, ref != base)
    scale = np.maximum(np.abs(ref), 1e-300)
    assert np.max(np.abs(got - ref) / scale) < tol


@pytest.mark.parametrize("prec,tol", [(_lib.PREC_FP64, 1e-9), (_lib.PREC_MIXED, 1e-6)])
def test_xlinop_autoionizing_and_merged_continuum_match_oracle(po, gpu_ctx, tables, atlas_case, h_tables, prec,
                                                                tol):
    """XLINOP with populations: the autoionizing lines (TYPE 1, Fano profile
    with ASHORE = GAMMAS, BSHORE = GAMMAW) and the merged-continuum records
    (TYPE 7, 12, -3: NLAST = TYPE; NELION 4 takes Z = 2) on top of the normal
    lines; hydrogen (TYPE -1) is the only type left out and counted."""
    c = atlas_case
    ws = np.geomspace(300.0, 600.0, 4000)
    recs = synthetic.nlte_records(4000, 300.5, 599.5, seed=9, strong=0.1, types=(0, 3, 2, 1, -1, 7, 12, -3),
                                  type_p=(.45, .1, .05, .2, .05, .05, .05, .05))
    rng = np.random.default_rng(10)
    f = recs["itype"] == 1
    recs["gammaw"][f] = 10.0 ** rng.uniform(3.0, 6.0, f.sum())                # BSHORE
    recs["gammas"][f] = recs["gammaw"][f] * rng.uniform(-2.0, 2.0, f.sum())   # ASHORE
    recs["gammar"][f] = 10.0 ** rng.uniform(11.0, 13.0, f.sum())             # GAMMAR (Hz)
    m = np.isin(recs["itype"], (7, 12, -3))
    recs["nelion"][np.nonzero(m)[0][::4]] = 4
    pop = c["pop"]
    nsp = min(NSPEC, pop["xnfp"].shape[1])
    xnfp = np.zeros((NSPEC, 72))
    xnfp[:nsp] = pop["xnfp"][:, :nsp].T
    rho = pop["rho"]
    contx = synthetic.contx_table()
    atm = dict(xnfdop=c["xnfdop"], dopple=c["dopple"], xne=c["xne"], txnxn=c["txnxn"], hckt=c["hckt"])
    plain, _ = po.atlas_xlinop(*h_tables, po.build_tablog(), recs, atm, c["tabcont"], c["iw"], ws, contx)
    ref, nread = po.atlas_xlinop(*h_tables, po.build_tablog(), recs, dict(atm, xnfp=xnfp, rho=rho), c["tabcont"],
                                 c["iw"], ws, contx)
    assert nread > 3000
    assert np.count_nonzero(ref != plain) > 2000  # the two branches add where the normal lines do not
    A = atlas.Atlas(gpu_ctx, tables, *h_tables)
    gpu_ctx.set_precision(prec)
    try:
        got, other = A.xlinop(recs, 72, c["xnfdop"], c["dopple"], c["xne"], c["txnxn"], c["hckt"], c["tabcont"],
                              c["iw"], ws, contx, xnfp=xnfp, rho=rho)
    finally:
        gpu_ctx.set_precision(_lib.PREC_MIXED)
    assert other == int(np.sum(recs["itype"] == -1))
    np.testing.assert_array_equal(got != 0, ref != 0)
    scale = np.maximum(np.abs(ref), 1e-300)
    assert np.max(np.abs(got - ref) / scale) < tol


def hydrogen_case(po, atlas_case, n_other=2000, seed=12):
    """Lyman, Balmer, Paschen and Brackett series (TYPE -1, NCON = NBLO, CGF
    from 2 n^2 f(n, m)) among normal lines over 90-2000 nm, CONTX(N,1) at the
    hydrogen level edges, and the atmosphere's T, XNF(J,1), XNF(J,2), XNH2."""
    c = atlas_case
    rh = 109677.583403
    recs = synthetic.nlte_records(n_other, 92.0, 1990.0, seed=seed, strong=0.1)
    series = [(n, m) for n, hi in ((1, 12), (2, 25), (3, 16), (4, 12)) for m in range(n + 1, hi)]
    hr = np.zeros(len(series), recs.dtype)
    for i, (n, m) in enumerate(series):
        wl = 1e7 / (rh * (1.0 / n ** 2 - 1.0 / m ** 2))
        hr[i]["wlvac"], hr[i]["nblo"], hr[i]["nbup"], hr[i]["itype"], hr[i]["ncon"] = wl, n, m, -1, n
        hr[i]["nelion"] = 1
        hr[i]["gf"] = 0.026538 / np.sqrt(np.pi) / synthetic.C_NM * wl * 2 * n * n * po.hfnm(n, m)
        hr[i]["nbuff"] = int(np.floor(np.log(wl) / np.log(1.0 + 1.0 / 2000000.0) + 0.5))
    recs = np.concatenate([recs, hr])
    recs = recs[np.argsort(recs["wlvac"], kind="stable")]
    contx = synthetic.contx_table()
    contx[0, :10] = rh / np.arange(1, 11) ** 2
    pop, t = c["pop"], c["m"]["t"]
    nh1 = pop["nh"] * (1.0 - pop["xh"])
    hyd = dict(t=t, xnf1=nh1, xnf2=pop["nh"] * pop["xh"], xnh2=1e-4 * nh1 * np.exp(-t / 1000.0))
    nsp = min(NSPEC, pop["xnfp"].shape[1])
    xnfp = np.zeros((NSPEC, 72))
    xnfp[:nsp] = pop["xnfp"][:, :nsp].T
    return recs, contx, hyd, xnfp, pop["rho"]


@pytest.mark.parametrize("prec,tol", [(_lib.PREC_FP64, 1e-9), (_lib.PREC_MIXED, 1e-6)])
def test_xlinop_hydrogen_lines_match_oracle(po, gpu_ctx, tables, atlas_case, h_tables, prec, tol):
    """XLINOP's hydrogen lines (HPROF4 over up to MAX_WING points a side, the
    blue wing stopping at the level's continuum edge) on top of the other
    types: every record type handled, none counted."""
    c = atlas_case
    ws = np.geomspace(90.0, 2000.0, 6000)
    recs, contx, hyd, xnfp, rho = hydrogen_case(po, atlas_case)
    atm = dict(xnfdop=c["xnfdop"], dopple=c["dopple"], xne=c["xne"], txnxn=c["txnxn"], hckt=c["hckt"], xnfp=xnfp,
               rho=rho)
    plain, _ = po.atlas_xlinop(*h_tables, po.build_tablog(), recs, atm, c["tabcont"], c["iw"], ws, contx)
    ref, _ = po.atlas_xlinop(*h_tables, po.build_tablog(), recs, dict(atm, htab=po.HTab.from_tables(tables), **hyd),
                             c["tabcont"], c["iw"], ws, contx)
    assert np.count_nonzero(ref != plain) > 50000
    A = atlas.Atlas(gpu_ctx, tables, *h_tables)
    A.set_hydrogen_tables(tables)
    gpu_ctx.set_precision(prec)
    try:
        got, other = A.xlinop(recs, 72, c["xnfdop"], c["dopple"], c["xne"], c["txnxn"], c["hckt"], c["tabcont"],
                              c["iw"], ws, contx, xnfp=xnfp, rho=rho, hydrogen=hyd)
        plain_got, other_plain = A.xlinop(recs, 72, c["xnfdop"], c["dopple"], c["xne"], c["txnxn"], c["hckt"],
                                          c["tabcont"], c["iw"], ws, contx, xnfp=xnfp, rho=rho)
    finally:
        gpu_ctx.set_precision(_lib.PREC_MIXED)
    assert other == 0 and other_plain == int(np.sum(recs["itype"] == -1))
    np.testing.assert_array_equal(got != 0, ref != 0)
    scale = np.maximum(np.abs(ref), 1e-300)
    assert np.max(np.abs(got - ref) / scale) < tol
    np.testing.assert_array_equal(plain_got != 0, plain != 0)


def test_xlinop_rejects_unsorted_records(gpu_ctx, tables, atlas_case, h_tables):
    c = atlas_case
    recs = synthetic.nlte_records(100, 300.5, 599.5, seed=6)[::-1].copy()
    A = atlas.Atlas(gpu_ctx, tables, *h_tables)
    with pytest.raises(_lib.AtlasGPUError, match="not sorted"):
        A.xlinop(recs, 72, c["xnfdop"], c["dopple"], c["xne"], c["txnxn"], c["hckt"], c["tabcont"], c["iw"],
                 np.geomspace(300.0, 600.0, 400), synthetic.contx_table())
