"""Failure detection with faults made on the host.

The reference stops with a message on bad input (CALL EXIT(1)) and keeps
iterating through its own guards (the JOSH negative-S reset,
atlas12_modules.f90:18596-18621; the RUN_RT_PASS floor, :3926-3937).  The
library instead returns ATLASGPU_ENONFINITE from every entry point whose
input tables must be finite, leaves the context usable, and takes a batched
model whose iteration stops being finite out of the batch (SLOT_NONFINITE)
while the other slots run on.

Every fault here is made on the host: a NaN or an infinity written into an
input array.  The kernels that a non-finite structure reaches index their
tables only through bounded searches or guarded conversions, so nothing
here reads outside a buffer, waits or traps.
"""
import numpy as np
import pytest

from atlas12_b200 import _lib, atlas, linelists, surrogate, synthe, synthetic

pytestmark = pytest.mark.gpu


def _expect_nonfinite(fn, *args):
    with pytest.raises(_lib.AtlasGPUError) as e:
        fn(*args)
    assert e.value.code == _lib.ENONFINITE, str(e.value)


def test_operators_and_voigt_tables_refuse_non_finite(gpu_ctx, tables):
    for key, idx, bad in (("coefj", (3, 7), np.nan), ("coefh", (50, 0), np.inf), ("xtau8", (10,), -np.inf),
                          ("ch_j", (0,), np.nan), ("ck_j", (50,), np.inf)):
        t = {k: np.array(tables[k], copy=True) for k in ("xtau8", "coefj", "coefh", "ch_j", "ck_j")}
        t[key][idx] = bad
        _expect_nonfinite(gpu_ctx.set_operators, t["xtau8"], t["coefj"], t["coefh"], t["ch_j"], t["ck_j"])
    h0, h1, h2 = atlas.tabvoigt(tables)
    bad = h1.copy()
    bad[1000] = np.inf
    with pytest.raises(_lib.AtlasGPUError) as e:
        atlas.Atlas(gpu_ctx, tables, h0, bad, h2)
    assert e.value.code == _lib.ENONFINITE
    # the context is still usable: a small RT pass after the refusals
    A = atlas.Atlas(gpu_ctx, tables)
    m = surrogate.grey_model(5777.0, 4.44)
    pop = surrogate.populations(m["t"], m["p"], 1.5)
    ws, rc = synthetic.geometric_waveset(9.0, 160000.0, 500)
    ac, sg = surrogate.continuum_opacity(ws, m["t"], m["p"], pop)
    hkt = surrogate.HPLANCK / (surrogate.KBOL * m["t"])
    acc, hs = A.rt_pass(ws, rc, ac, sg, np.zeros_like(ac), m["rhox"], m["t"], hkt, 5777.0)
    assert np.all(np.isfinite(hs)) and np.all(np.isfinite(acc["flxrad"]))


def test_selectlines_tables_refuse_non_finite(gpu_ctx, tables):
    wt = tables["wavetab"]
    xn, hckt, tc = synthetic.selectlines_tables(wt)
    iwt = atlas.iwavetab(wt)
    for which in ("xnfdop", "tabcont", "hckt", "wavetab"):
        a = dict(xnfdop=xn.copy(), tabcont=tc.copy(), hckt=hckt.copy(), wavetab=wt.copy())
        flat = a[which].reshape(-1)
        flat[flat.size // 2] = np.nan if which != "hckt" else np.inf
        _expect_nonfinite(linelists.SelectLines, gpu_ctx, 72, a["xnfdop"], a["hckt"], a["tabcont"], iwt,
                          a["wavetab"])


def test_synthe_continuum_and_spectrum_refuse_non_finite(gpu_ctx, tables):
    case = synthetic.synthe_case(nlines=200, wlbeg=400.0, wlend=400.2, seed=5)
    S = synthe.Synthe(gpu_ctx, tables)
    grid = synthe.synthe_grid(case["wlbeg"], case["wlend"], case["resolu"])
    ca = case["continall"].copy()
    ca[5, 3] = np.nan
    _expect_nonfinite(S.continuum, case["wledge"], ca, grid)
    cont = S.continuum(case["wledge"], case["continall"], grid)
    op = np.zeros_like(cont)
    atm = case["atm"]
    for which, bad in (("contabs", np.inf), ("contscat", np.nan), ("rhox", np.nan), ("hkt", np.inf)):
        a = dict(contabs=case["contabs"].copy(), contscat=case["contscat"].copy(), rhox=atm["rhox"].copy(),
                 hkt=atm["hkt"].copy())
        flat = a[which].reshape(-1)
        flat[flat.size // 3] = bad
        _expect_nonfinite(S.spectrum, case["wledge"], a["contabs"], a["contscat"], a["rhox"], a["hkt"], grid, op)
    # and the context still synthesises
    wave, flux, cflux, _ = S.run(case)
    assert np.all(np.isfinite(flux)) and np.all(flux > 0)


def test_model_iteration_reports_non_finite_structure(gpu_ctx, tables):
    """A starting structure with an infinite temperature at one depth: the
    iteration's FLXERR is not finite, and iterate says so instead of
    returning a number."""
    ws, rc = synthetic.geometric_waveset(9.0, 160000.0, 1000)
    lines = synthetic.atlas_lines(2000, ws[2], ws[-3], seed=3)
    m = atlas.AtlasModel(gpu_ctx, tables, linedata=lines, waveset=ws, rcoset=rc)
    s = surrogate.grey_model(5777.0, 4.44)
    t = s["t"].copy()
    t[40] = np.inf
    m.set_structure(t, s["p"], s["rhox"])
    with pytest.raises(_lib.AtlasGPUError) as e:
        m.iterate(max_iter=3, tol_percent=0.0, graph=False)
    assert e.value.code == _lib.ENONFINITE
    # the same model object runs a finite start afterwards
    m.set_structure(s["t"], s["p"], s["rhox"])
    n, hist = m.iterate(max_iter=2, tol_percent=0.0, graph=True)
    assert n == 2 and np.all(np.isfinite(hist))
    m.close()


PARAMS = [(5777.0, 4.44, 0.0, 1.5), (6000.0, 4.3, -0.3, 1.5), (5200.0, 4.5, 0.1, 1.0)]


def test_batch_slot_goes_nonfinite_and_the_others_finish(gpu_ctx, tables):
    """Three slots; the middle model starts with T = +inf at one depth (it
    passes batch_load, whose check is T > 0).  Its first finish writes
    SLOT_NONFINITE and the graph skips it from then on; the other two run
    their iterations and end exactly where they end in a batch whose middle
    model is finite (relative 1e-8, the batch parity tolerance: LINOP1's FP64
    atomics may add in another order)."""
    ws, rc = synthetic.geometric_waveset(9.0, 160000.0, 2000)
    lines = synthetic.atlas_lines(5000, ws[2], ws[-3], seed=3)
    starts = [surrogate.grey_model(te, lg, ross=surrogate.RossTable(mh=mh, nwave=600)) for te, lg, mh, _ in PARAMS]
    bad = dict(starts[1])
    bad["t"] = starts[1]["t"].copy()
    bad["t"][40] = np.inf
    nit = 4
    b = atlas.AtlasBatch(gpu_ctx, tables, nslots=3, linedata=lines, waveset=ws, rcoset=rc, shape=None)
    ref = b.run_queue(PARAMS, starts, max_iter=nit, tol_percent=0.0, poll_every=1)
    got = b.run_queue(PARAMS, [starts[0], bad, starts[2]], max_iter=nit, tol_percent=0.0, poll_every=1)
    b.close()
    assert got[1]["status"] == _lib.SLOT_NONFINITE and got[1]["iters"] == 1
    for i in (0, 2):
        assert got[i]["status"] == _lib.SLOT_CAPPED and got[i]["iters"] == nit
        for q in ("t", "p", "rhox"):
            np.testing.assert_allclose(got[i][q], ref[i][q], rtol=1e-8, err_msg=f"model {i} {q}")
        np.testing.assert_allclose(got[i]["hist"], ref[i]["hist"], rtol=1e-8)
