"""Known-answer tests pinning the CPU oracle (no GPU)."""
import os
import re

import numpy as np
import pytest
from scipy.special import expn, wofz

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def weideman_coefficients(n=32):
    """Weideman (1994) construction of the N-term coefficients."""
    M = 2 * n
    k = np.arange(-M + 1, M)
    L = np.sqrt(n / np.sqrt(2))
    t = L * np.tan(k * np.pi / M / 2)
    f = np.concatenate([[0.0], np.exp(-t ** 2) * (L ** 2 + t ** 2)])
    a = np.real(np.fft.fft(np.fft.fftshift(f))) / (2 * M)
    return np.flipud(a[1:n + 1]), L


def _embedded(path, name):
    s = open(path).read()
    i = s.index(name)
    j = s.index("};", i)
    return np.array([float(x) for x in re.findall(r"[-+]?\d\.\d+e[-+]\d+", s[i:j])])


def test_weideman_coefficients_pinned(tables):
    a, L = weideman_coefficients()
    np.testing.assert_array_equal(a, tables["awei"])
    assert L == tables["lwei"][0]
    for path, name in ((os.path.join(ROOT, "oracle", "oracle.c"), "WEI_A[32]"),
                       (os.path.join(ROOT, "atlas12_b200", "csrc", "voigt.cuh"), "kWeiA[32]")):
        np.testing.assert_array_equal(_embedded(path, name), a)


def test_voigt_weideman_vs_wofz(po):
    rng = np.random.default_rng(0)
    v = rng.uniform(0, 14, 3000)
    a = 10 ** rng.uniform(-5, 0.5, 3000)
    core = (v + a) <= 15
    got = np.array([po.voigt_weideman(x, y) for x, y in zip(v, a)])
    ref = wofz(v + 1j * a).real
    # Weideman N=32 is accurate to ~1e-14 absolute (Weideman 1994, table 1)
    assert np.max(np.abs(got[core] - ref[core])) < 5e-14
    # Humlicek asymptote region: the reference's own approximation, ~1e-4
    v2 = rng.uniform(15, 60, 500)
    a2 = 10 ** rng.uniform(-4, 0, 500)
    got2 = np.array([po.voigt_weideman(x, y) for x, y in zip(v2, a2)])
    assert np.max(np.abs(got2 - wofz(v2 + 1j * a2).real) / wofz(v2 + 1j * a2).real) < 3e-3


def test_expi_e3_vs_scipy(po):
    for x in [1e-6, 1e-3, 0.01, 0.3, 1.0, 2.5, 4.0, 4.5, 9.9, 30.0]:
        assert abs(po.expi(3, x) - expn(3, x)) <= 2e-12 * max(expn(3, x), 1e-300) + 1e-300
    assert po.expi(1, 0.0) == 0.0


def test_integ_exact_on_lines_and_interior_quadratics(po):
    # PARCOE fits straight lines on the first three and the last two
    # intervals and blended parabolas inside, so INTEG is exact for linear
    # integrands everywhere and for quadratics on the interior intervals.
    x = np.linspace(0.3, 5.0, 40) ** 1.3
    f = 2.0 + 3.0 * x
    np.testing.assert_allclose(po.integ(x, f, 0.0), 2 * (x - x[0]) + 1.5 * (x ** 2 - x[0] ** 2),
                               rtol=1e-12, atol=1e-12)
    q = 2.0 + 3.0 * x - 0.5 * x ** 2
    F = po.integ(x, q, 0.0)
    prim = 2 * x + 1.5 * x ** 2 - x ** 3 / 6
    inc, exact = np.diff(F), np.diff(prim)
    np.testing.assert_allclose(inc[3:-2], exact[3:-2], rtol=1e-11)


def test_map1_reproduces_quadratics(po):
    xo = np.linspace(0.0, 10.0, 30) ** 1.5
    fo = 1.0 + xo - 0.01 * xo ** 2
    xn = np.linspace(0.5, 30.0, 77)
    fn, last = po.map1(xo, fo, xn)
    # brackets 2 and 3 use straight lines; parabolas (exact here) from bracket 4 on
    inner = (xn >= xo[2]) & (xn < xo[-1])
    np.testing.assert_allclose(fn[inner], (1.0 + xn - 0.01 * xn ** 2)[inner], rtol=1e-11)
    lin = 1.0 + 2.0 * xn
    np.testing.assert_allclose(po.map1(xo, 1.0 + 2.0 * xo, xn)[0], lin, rtol=1e-12)
    assert 1 <= last <= xo.size


def test_solvit_vs_numpy(po):
    rng = np.random.default_rng(3)
    for _ in range(5):
        A = rng.normal(size=(51, 51)) + 5 * np.eye(51)
        b = rng.normal(size=51)
        np.testing.assert_allclose(po.solvit(A, b), np.linalg.solve(A, b), rtol=1e-10, atol=1e-12)


def test_josh_linear_source_surface_flux(po, ops):
    # S = a + b tau, pure absorption: H(0) = (a + 2b/3) / 4
    nr = 72
    tau = 10 ** (-6.875 + 0.125 * np.arange(nr))
    k = np.ones(nr)
    for a, b in ((1.0, 2.0), (0.5, 10.0), (3.0, 0.0)):
        S = a + b * tau
        r = po.josh(ops, 1, 1, tau, k, 0 * k, 0 * k, 0 * k, S, S, S)
        assert abs(r["hnu"][0] - (a + 2 * b / 3) / 4) < 2e-9 * (a + b)
        full = po.josh(ops, 1, 0, tau, k, 0 * k, 0 * k, 0 * k, S, S, S)
        # COEFH row 1 and CH_J are separate tabulations of the same surface weights
        np.testing.assert_allclose(full["hnu"][0], r["hnu"][0], rtol=1e-6)  # REAL*4 operator data
        # deep layers: diffusion limit H = b/3
        np.testing.assert_allclose(full["hnu"][-1], b / 3, rtol=1e-6, atol=1e-12)


def test_josh_scattering_conserves_flux(po, ops):
    # conservative scattering: S = J, H constant with depth (grey, alpha -> 1 deep)
    nr = 72
    tau = 10 ** (-6.875 + 0.125 * np.arange(nr))
    z = np.zeros(nr)
    sig = np.ones(nr) * 0.999
    kap = np.ones(nr) * 0.001
    B = 1.0 + 1.5 * tau
    r = po.josh(ops, 1, 0, tau, kap, z, sig, z, B, B, B)
    assert r["maxj"] > 40
    assert np.all(r["hnu"] > 0) and np.all(np.isfinite(r["jnu"]))


def test_operator_fixture_row_sums(tables):
    cj = tables["coefj"]
    ch = tables["coefh"]
    assert abs(cj[0].sum() - 0.5) < 1e-6 and abs(cj[-1].sum() - 1.0) < 1e-6
    assert abs(ch[0].sum() - 0.25) < 1e-6
    assert abs(tables["ch_j"].sum() - 0.25) < 1e-8
    assert tables["xtau8"][0] == 0.0 and tables["xtau8"][-1] == 20.0


def test_tabvoigt_tables(po, tables):
    h0, h1, h2 = po.tabvoigt(tables["tabvi"], tables["tabh1"])
    v = np.arange(2001) / 200.0
    np.testing.assert_allclose(h0, np.exp(-v * v), rtol=1e-15)
    np.testing.assert_allclose(h2, (1 - 2 * v * v) * np.exp(-v * v), rtol=1e-12, atol=1e-300)
    assert h1[0] == tables["tabh1"][0]
    # Kurucz VOIGT against wofz where its quadratic-in-a expansion holds
    for vv, aa in ((0.5, 0.01), (2.0, 0.05), (5.0, 0.001), (12.0, 0.1)):
        got = po.voigt_kurucz(vv, aa, h0, h1, h2)
        assert abs(got - wofz(vv + 1j * aa).real) / wofz(vv + 1j * aa).real < 2e-2


def test_synthe_grid_and_binning(po):
    g = po.synthe_grid(400.0, 410.0, 500000.0)
    assert g["length"] == 12346
    assert g["wbegin"] >= 400.0
    # a line exactly on a grid point bins to that point
    for i in (1, 17, 12346):
        w = g["wbegin"] * g["ratio"] ** (i - 1)
        assert po.nbuff(w, g["ratiolg"], g["ixwlbeg"]) == i


# ---- pins against the reference's own converged solar model (READ DECK6 of
# workdir/ap00t5777g4.44at12.dat: Teff 5777 K, log g 4.44, 72 depths) ----

def test_integ_reproduces_reference_tau_grid(po, tables):
    """ROSS(3)'s TAUROS = INTEG(RHOX, ABROSS, ABROSS(1)*RHOX(1)) on the converged
    deck returns the standard grid log tau = -6.875 + 0.125 (j-1) that the
    reference remapped the model onto (TAU1LG/STEPLG, atlas12_modules.f90:1792),
    to the deck's print precision (4 digits of ABROSS)."""
    d = tables["deck"]
    rhox, ab = d[:, 0], d[:, 4]
    tau = po.integ(rhox, ab, ab[0] * rhox[0])
    std = -6.875 + 0.125 * np.arange(d.shape[0])
    assert np.max(np.abs(np.log10(tau) - std)) < 2e-4


def test_ttaup_reproduces_reference_deck(po, tables):
    """TTAUP (atlas12_modules.f90:6303-6523) with ROSSTAB holding the deck's
    own (T, P, ABROSS) integrates hydrostatic equilibrium on the standard tau
    grid back to the deck's P and RHOX (printed to 4 digits) and looks up its
    ABROSS."""
    d = tables["deck"]
    rhox, t, p, ab = d[:, 0], d[:, 1], d[:, 2], d[:, 4]
    g = 10.0 ** 4.44
    store = po.RossStore()
    po.rosstab_store(store, t, p, ab)
    assert store.n == d.shape[0]
    tau = 10.0 ** (-6.875 + 0.125 * np.arange(d.shape[0]))
    abstd, ptot, pout = po.ttaup(store, t, tau, g, np.zeros_like(t))
    assert np.max(np.abs(pout / p - 1.0)) < 3e-3
    assert np.max(np.abs(ptot / (g * rhox) - 1.0)) < 3e-3
    assert np.max(np.abs(abstd / ab - 1.0)) < 2e-3


def test_mlp_oracle_gradient_is_the_derivative():
    """The network restatement's analytic gradient against central differences."""
    import mlp_ref
    shape = (4, 6, 5, 7)
    rng = np.random.default_rng(0)
    n = sum(a * b + a for a, b in ((6, 4), (5, 6), (7, 5)))
    p = rng.normal(0, 0.5, n)
    x = rng.uniform(-1, 1, (9, 4))
    t = rng.normal(0, 1, (9, 7))
    _, g = mlp_ref.loss_grad(p, x, t, shape)
    h = 1e-6
    for i in rng.choice(n, 25, replace=False):
        e = np.zeros(n)
        e[i] = h
        fd = (mlp_ref.loss_grad(p + e, x, t, shape)[0] - mlp_ref.loss_grad(p - e, x, t, shape)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-6 * abs(g[i])
