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
