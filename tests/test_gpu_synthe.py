"""SYNTHE hot path on the GPU (through the C ABI) against the CPU oracle.

Tolerances:
  * nbuff (binning): bit-exact.
  * continuum (REAL(4)): 2 ulp (device exp10 vs the C library powf).
  * kappa_line: |GPU - oracle_fp64| <= 1e-5 * (kappa_line + kappa_cont) per bin
    for both precisions (typically ~1e-7 mixed, ~1e-12 fp64).  Against the
    reference's REAL(4) sequential sums (oracle ref32): <= 1e-5 * (k + k_c)
    on the small case.  At the C1 size (20,000 lines) the reference's own
    REAL(4) accumulation is further than that from the exact sum: the FP64
    oracle itself differs from ref32 by 1.8e-5 there (the strongest line
    cores, where hundreds of REAL(4) additions land in one bin and
    kappa_line >> kappa_cont).  The C1 bound is therefore derived: the GPU's
    distance from ref32 may exceed the FP64 oracle's distance from ref32 by
    at most 1e-6 (the GPU adds nothing beyond the reference's rounding).
  * flux: relative 1e-4 against the oracle on the same opacity.
"""
import numpy as np
import pytest

from atlas12_b200 import _lib, synthetic
from atlas12_b200 import synthe as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_case():
    return synthetic.synthe_case(nlines=3000, wlbeg=400.0, wlend=402.0, seed=5)


@pytest.fixture(scope="module")
def prepared(po, small_case):
    case = small_case
    g = po.synthe_grid(case["wlbeg"], case["wlend"], case["resolu"])
    nb = np.array([po.nbuff(w, g["ratiolg"], g["ixwlbeg"]) for w in case["lines"]["wlvac"]], np.int32)
    lines = dict(case["lines"], nbuff=nb)
    cont = po.synthe_continuum(po.REF32, case["wledge"], case["continall"], g["wbegin"], g["ratio"], g["length"])
    o32, o32_64 = po.synthe_line_opacity(po.REF32, lines, g["length"], case["atm"], cont, case["resolu"])
    o64, o64_64 = po.synthe_line_opacity(po.FP64, lines, g["length"], case["atm"], cont, case["resolu"])
    return dict(case=case, grid=g, lines=lines, cont=cont, ref32=o32_64, fp64=o64_64)


def _rec(lines):
    return S.make_lte_lines(lines["nbuff"], lines["cgf"], lines["nelion"], lines["elo"], lines["gamrf"],
                            lines["gamsf"], lines["gamwf"])


def _kappa_err(got, ref, cont):
    return np.max(np.abs(got.astype(np.float64) - ref) / (ref + cont.astype(np.float64)))


def test_bin_bitexact_including_boundaries(po, gpu_ctx, tables):
    syn = S.Synthe(gpu_ctx, tables)
    g = S.synthe_grid(300.0, 1000.0, 500000.0)
    rng = np.random.default_rng(11)
    wl = np.sort(rng.uniform(300.0, 1000.0, 200000))
    k = rng.integers(g["ixwlbeg"], g["ixwlbeg"] + g["length"], 2000)
    edge = np.exp((k + 0.5) * g["ratiolg"])              # on the rounding boundary
    near = np.nextafter(edge, edge * (1 + rng.choice([-1, 1], edge.size)))
    onpt = g["wbegin"] * g["ratio"] ** rng.integers(0, g["length"], 2000)
    allw = np.concatenate([wl, edge, near, onpt])
    got = syn.bin_lines(allw, g)
    ref = np.array([po.nbuff(w, g["ratiolg"], g["ixwlbeg"]) for w in allw], np.int32)
    np.testing.assert_array_equal(got, ref)


def test_continuum_matches_oracle(prepared, gpu_ctx, tables):
    p = prepared
    syn = S.Synthe(gpu_ctx, tables)
    got = syn.continuum(p["case"]["wledge"], p["case"]["continall"], p["grid"])
    np.testing.assert_allclose(got, p["cont"], rtol=2.5e-7)


@pytest.mark.parametrize("prec", [_lib.PREC_FP64, _lib.PREC_MIXED])
def test_line_opacity_matches_fp64_oracle(prepared, gpu_ctx, tables, prec):
    p = prepared
    gpu_ctx.set_precision(prec)
    syn = S.Synthe(gpu_ctx, tables)
    atm = p["case"]["atm"]
    got = syn.line_opacity(_rec(p["lines"]), p["grid"], p["case"]["resolu"], p["cont"], atm["xnfdop"],
                           atm["dopple"], atm["xne"], atm["txnxn"], atm["hckt"])
    gpu_ctx.set_precision(_lib.PREC_MIXED)
    e64 = _kappa_err(got, p["fp64"], p["cont"])
    e32 = _kappa_err(got, p["ref32"], p["cont"])
    assert e64 <= 1e-5, e64
    assert e32 <= 1e-5, e32
    assert np.all(np.isfinite(got)) and got.max() > 0


def test_line_opacity_edge_cases(po, prepared, gpu_ctx, tables):
    p = prepared
    syn = S.Synthe(gpu_ctx, tables)
    atm = p["case"]["atm"]
    g = p["grid"]
    # empty line list
    empty = S.make_lte_lines(*[np.zeros(0)] * 7)
    out = syn.line_opacity(empty, g, p["case"]["resolu"], p["cont"], atm["xnfdop"], atm["dopple"], atm["xne"],
                           atm["txnxn"], atm["hckt"])
    assert out.shape == p["cont"].shape and not out.any()
    # lines off both ends of the grid (wings reach in) and a small profile cap
    L = dict(p["lines"])
    L = {k: v[:400].copy() for k, v in L.items()}
    L["nbuff"][:100] -= g["length"] + 50
    L["nbuff"][100:200] += g["length"] + 50
    for maxprof in (1000000, 60):
        ref = po.synthe_line_opacity(po.FP64, L, g["length"], atm, p["cont"], p["case"]["resolu"],
                                     maxprof=maxprof)[1]
        got = syn.line_opacity(_rec(L), g, p["case"]["resolu"], p["cont"], atm["xnfdop"], atm["dopple"],
                               atm["xne"], atm["txnxn"], atm["hckt"], maxprof=maxprof)
        assert _kappa_err(got, ref, p["cont"]) <= 1e-5


def test_spectrum_matches_oracle(po, ops, prepared, gpu_ctx, tables):
    p = prepared
    case, g = p["case"], p["grid"]
    syn = S.Synthe(gpu_ctx, tables)
    op = p["ref32"].astype(np.float32)
    atm = case["atm"]
    flux, cont = syn.spectrum(case["wledge"], case["contabs"], case["contscat"], atm["rhox"], atm["hkt"], g, op)
    sel = np.linspace(1, g["length"], 300).astype(int)
    rf = np.zeros(sel.size)
    rc = np.zeros(sel.size)
    for i, iw in enumerate(sel):
        f, c = po.synthe_spectrum(ops, case["wledge"], case["contabs"], case["contscat"], atm["rhox"], atm["hkt"],
                                  g["wbegin"], g["ratio"], op, iw0=int(iw), iw1=int(iw))
        rf[i], rc[i] = f[0], c[0]
    np.testing.assert_allclose(flux[sel - 1], rf, rtol=1e-4)
    np.testing.assert_allclose(cont[sel - 1], rc, rtol=1e-4)
    assert np.all(flux > 0) and np.all(flux <= cont * (1 + 1e-9))


def test_full_c1_pipeline(po, gpu_ctx, tables):
    """The CPU-runnable configuration end to end: 20k lines, 12,346 points."""
    case = synthetic.synthe_case()
    syn = S.Synthe(gpu_ctx, tables)
    wave, flux, cflux, op = syn.run(case)
    g = po.synthe_grid(case["wlbeg"], case["wlend"], case["resolu"])
    assert op.shape == (72, g["length"]) == (72, 12346)
    nb = np.array([po.nbuff(w, g["ratiolg"], g["ixwlbeg"]) for w in case["lines"]["wlvac"]], np.int32)
    lines = dict(case["lines"], nbuff=nb)
    cont = po.synthe_continuum(po.REF32, case["wledge"], case["continall"], g["wbegin"], g["ratio"], g["length"])
    ref = po.synthe_line_opacity(po.FP64, lines, g["length"], case["atm"], cont, case["resolu"])[1]
    assert _kappa_err(op, ref, cont) <= 1e-5
    assert np.all(np.isfinite(flux)) and np.all(flux > 0)
    # against the reference's REAL(4) sequential order: no further than the
    # exact (FP64) sums are from it, plus 1e-6
    r32 = po.synthe_line_opacity(po.REF32, lines, g["length"], case["atm"], cont, case["resolu"])[1]
    e_exact = _kappa_err(ref.astype(np.float32), r32, cont)
    e_gpu = _kappa_err(op, r32, cont)
    print(f"C1 kappa_line vs REAL(4) order: GPU {e_gpu:.3e}, FP64 oracle {e_exact:.3e}")
    assert e_exact <= 3e-5, e_exact
    assert e_gpu <= e_exact + 1e-6, (e_gpu, e_exact)


def _nlte_records(po, case, g, seed=8):
    """NLTE-list records from the case's lines: all line types, continuum edges,
    5 % of lines moved 0.3 nm blue and 5 % 0.3 nm red of the window."""
    rng = np.random.default_rng(seed)
    L = case["lines"]
    n = L["wlvac"].size
    wl = L["wlvac"] + np.where(rng.uniform(size=n) < 0.05, -0.3, 0.0) + np.where(rng.uniform(size=n) < 0.05, 0.3, 0.0)
    order = np.argsort(wl)
    r = np.zeros(n, _lib.NLTE_LINE)
    r["wlvac"] = wl[order]
    r["elo"] = L["elo"][order]
    r["gf"] = L["cgf"][order]
    r["nelion"] = L["nelion"][order]
    r["itype"] = rng.choice([0, 3, -3, 2, -1, 1], n, p=[.6, .1, .1, .1, .05, .05])
    has = rng.uniform(size=n) < 0.3
    r["ncon"] = np.where(has, rng.integers(1, 11, n), 0)
    r["nelionx"] = np.where(has, rng.integers(1, 18, n), 0)
    for a, b in (("gammar", "gamrf"), ("gammas", "gamsf"), ("gammaw", "gamwf")):
        r[a] = L[b][order]
    r["nbuff"] = [po.nbuff(w, g["ratiolg"], g["ixwlbeg"]) for w in r["wlvac"]]
    return r


def test_nlte_normal_lines_match_fp64_oracle(po, gpu_ctx, tables, prepared):
    """compute_line_opacity's normal-metal branch: GPU (FP64 sums, FP32
    output) against the FP64 restatement, relative to kappa + kappa_cont
    per bin (1e-6; the FP32 output rounding is ~6e-8)."""
    p = prepared
    case, g, cont = p["case"], p["grid"], p["cont"]
    recs = _nlte_records(po, case, g)
    assert (recs["nbuff"] < 1).any() and (recs["nbuff"] > g["length"]).any()
    rng = np.random.default_rng(9)
    contx = np.zeros((17, 26))
    # edges (cm^-1) whose WCON = 1e7 / (CONTX - EMERGE) lands inside the 400-402 nm window
    contx[:, :10] = 1.0e7 / rng.uniform(399.5, 402.5, (17, 10))
    atm = case["atm"]
    wlend = case["wlend"]
    ref = po.synthe_nlte_opacity(recs, g["length"], g["wbegin"], g["ratio"], wlend, 2.5, cont, atm, contx)
    nocut = po.synthe_nlte_opacity(recs, g["length"], g["wbegin"], g["ratio"], wlend, 2.5, cont, atm,
                                   np.zeros_like(contx))
    assert np.count_nonzero(ref) > 0.3 * ref.size and np.sum(nocut) > np.sum(ref)
    syn = S.Synthe(gpu_ctx, tables)
    got = syn.nlte_opacity(recs, g, wlend, cont, atm["xnfdop"], atm["dopple"], atm["xne"], atm["txnxn"], atm["hckt"],
                           contx, np.zeros((72, g["length"]), np.float32), velshift_kms=2.5)
    err = np.abs(got.astype(np.float64) - ref) / (ref + cont.astype(np.float64))
    assert err.max() <= 1e-6, err.max()
    # it adds into the LTE opacity it is given
    base = np.full((72, g["length"]), 1.0e-3, np.float32)
    got2 = syn.nlte_opacity(recs, g, wlend, cont, atm["xnfdop"], atm["dopple"], atm["xne"], atm["txnxn"],
                            atm["hckt"], contx, base, velshift_kms=2.5)
    np.testing.assert_allclose(got2.astype(np.float64) - 1.0e-3, ref, rtol=1e-5, atol=2e-10)


def test_nlte_shore_and_merged_lines_match_fp64_oracle(po, gpu_ctx, tables, prepared):
    """compute_line_opacity with XNFPEL given: the autoionizing (Shore) lines
    (Fano profile from GAMMAS, GAMMAW and GAMMAR, red wing added before its
    test) and the merged-continuum edges (TYPE = NLAST >= 4, flat to WMERGE,
    tapering to WTAIL; NELION 1 with RYDBERG_H), on top of the normal lines;
    GPU against the FP64 restatement (1e-6 of kappa + kappa_cont per bin)."""
    p = prepared
    case, g, cont = p["case"], p["grid"], p["cont"]
    recs = _nlte_records(po, case, g)
    rng = np.random.default_rng(21)
    u = rng.uniform(size=recs.size)
    f = u < 0.3
    recs["itype"][f] = 1
    recs["gammaw"][f] = 10.0 ** rng.uniform(4.0, 6.0, f.sum())               # BSHORE
    recs["gammas"][f] = recs["gammaw"][f] * rng.uniform(-2.0, 2.0, f.sum())  # ASHORE
    recs["gammar"][f] = 10.0 ** rng.uniform(10.0, 12.0, f.sum())            # GAMMAR (Hz)
    mrg = (u >= 0.3) & (u < 0.33)
    recs["itype"][mrg] = rng.choice([4, 9, 30, 100], mrg.sum())
    recs["nelion"][np.nonzero(mrg)[0][::3]] = 1
    contx = np.zeros((17, 26))
    atm = case["atm"]
    xnfpel = atm["xnfdop"] * atm["dopple"]
    wlend = case["wlend"]
    plain = po.synthe_nlte_opacity(recs, g["length"], g["wbegin"], g["ratio"], wlend, 0.0, cont, atm, contx)
    ref = po.synthe_nlte_opacity(recs, g["length"], g["wbegin"], g["ratio"], wlend, 0.0, cont,
                                 dict(atm, xnfpel=xnfpel), contx)
    assert np.count_nonzero(ref != plain) > 0.1 * ref.size
    syn = S.Synthe(gpu_ctx, tables)
    got = syn.nlte_opacity(recs, g, wlend, cont, atm["xnfdop"], atm["dopple"], atm["xne"], atm["txnxn"], atm["hckt"],
                           contx, np.zeros((72, g["length"]), np.float32), xnfpel=xnfpel)
    err = np.abs(got.astype(np.float64) - ref) / (ref + cont.astype(np.float64))
    assert err.max() <= 1e-6, err.max()


@pytest.mark.parametrize("stehle", [False, True], ids=["analytic", "stehle"])
@pytest.mark.parametrize("window", ["balmer", "lyman"])
def test_nlte_hydrogen_lines_match_fp64_oracle(po, gpu_ctx, tables, window, stehle):
    """compute_line_opacity's hydrogen and deuterium lines: the Lyman series
    (Lyman alpha with its H2 and H2+ satellites) over 92-130 nm and the Balmer
    series over 380-700 nm in a 9500 K atmosphere, alpha, beta and the
    tapered higher members, each deuterium line just before its hydrogen line
    (which then reuses its Stark convolution), with the analytic profile or
    Stehle-format tables.  Same tolerance as the other NLTE branches; without
    the hydrogen inputs the records are skipped."""
    from atlas12_b200 import surrogate as sg
    lo, hi, res = (380.0, 700.0, 30000.0) if window == "balmer" else (92.0, 130.0, 20000.0)
    g = po.synthe_grid(lo, hi, res)
    length = g["length"]
    wav = g["wbegin"] * g["ratio"] ** np.arange(length)
    m = sg.grey_model(9500.0, 4.0)
    ka, sgm = sg.continuum_opacity(wav, m["t"], m["p"], sg.populations(m["t"], m["p"], 2.0))
    cont = np.ascontiguousarray((ka + sgm).T, np.float32)
    atm = synthetic.hydrogen_atmosphere()
    recs = synthetic.hydrogen_records(lo, hi, g["wbegin"], g["ratio"])
    assert set(recs["itype"]) == {-1, -2} and len(recs) >= 14
    st = synthetic.stehle_tables() if stehle else None
    ref = po.synthe_hydrogen_opacity(recs, length, g["wbegin"], g["ratio"], hi, 0.0, cont, atm,
                                     po.HTab.from_tables(tables, "s_"), st)
    assert np.count_nonzero(ref) > 0.3 * ref.size
    syn = S.Synthe(gpu_ctx, tables)
    syn.set_hydrogen_tables(tables, st)
    args = (recs, g, hi, cont, atm["xnfdop"], atm["dopple"], atm["xne"], atm["txnxn"], atm["hckt"],
            np.zeros((17, 26)), np.zeros((atm["t"].size, length), np.float32))
    got = syn.nlte_opacity(*args, hydrogen=atm)
    assert _kappa_err(got, ref, cont) <= 1e-6
    assert not np.any(syn.nlte_opacity(*args))


def test_run_adds_the_unit19_lines(po, gpu_ctx, tables, small_case):
    """PROGRAM SYNTHE with hydrogen records: the opacity matrix is the LTE
    lines' plus compute_line_opacity's (here H delta's far blue wing, which
    reaches only the deep layers), and the flux does not rise."""
    case = dict(small_case)
    g = po.synthe_grid(case["wlbeg"], case["wlend"], case["resolu"])
    syn = S.Synthe(gpu_ctx, tables)
    syn.set_hydrogen_tables(tables)
    atm = case["atm"]
    nr = atm["xne"].size
    recs = synthetic.hydrogen_records(395.0, 415.0, g["wbegin"], g["ratio"], series=((2, 6, 7),))
    hy = synthetic.hydrogen_atmosphere()
    hyd = {k: hy[k][:nr] for k in ("t", "xnfph1", "xnfph2", "xnfhe1", "xnfh2")}
    _, flux0, _, op0 = syn.run(case)
    case.update(nlte=recs, contx=np.zeros((17, 26)), hydrogen=hyd)
    _, flux1, _, op1 = syn.run(case)
    cont = syn.continuum(case["wledge"], case["continall"], g)
    alone = syn.nlte_opacity(recs, g, case["wlend"], cont, atm["xnfdop"], atm["dopple"], atm["xne"], atm["txnxn"],
                             atm["hckt"], case["contx"], np.zeros_like(op0), hydrogen=hyd)
    assert np.count_nonzero(alone) > 0.1 * alone.size  # H delta's blue wing over the deeper layers
    np.testing.assert_allclose(op1, op0 + alone, rtol=1e-6)
    assert np.all(flux1 <= flux0 * (1 + 1e-6))


def test_concurrent_spectra_match_one_at_a_time(gpu_ctx, tables):
    """Spectra of atmospheres with their own windows and line lists on four
    concurrent contexts equal those computed one at a time (flux to 1e-6:
    only the order of the FP64 atomic sums differs)."""
    from atlas12_b200 import synthe_batch
    cases = synthetic.grid_cases(6, seed=5, line_scale=0.002, lo=400.0, hi=520.0)
    for c in cases:  # keep the windows short for the test
        c["wlend"] = c["wlbeg"] + min(c["wlend"] - c["wlbeg"], 2.0)
        keep = c["lines"]["wlvac"] < c["wlend"]
        c["lines"] = {k: v[keep] for k, v in c["lines"].items()}
    one = synthe_batch.SyntheBatch(0, tables, lanes=1)
    many = synthe_batch.SyntheBatch(0, tables, lanes=4)
    r1, r4 = one.run(cases), many.run(cases)
    one.close()
    many.close()
    for a, b in zip(r4, r1):
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_allclose(a[1], b[1], rtol=1e-6)
        np.testing.assert_allclose(a[2], b[2], rtol=1e-6)
