"""Host-side mirror of SYNTHE's hot path (synthe.f90), on the CUDA C ABI.

Names and argument meaning follow the reference driver:

* ``synthe_grid``      -- the log-lambda grid (synthe.f90:316-324)
* ``bin_lines``        -- nbuff of every line (mod_mklinelist.f90:898-899)
* ``continuum``        -- continuum(nbuff) per depth (synthe.f90:483-516)
* ``line_opacity``     -- opacity_matrix(length, nrhox) (synthe.f90:559-686)
* ``spectrum``         -- the wavelength loop, two JOSH per point
                          (synthe.f90:698-718, 797-902)
* ``Synthe.run``       -- all of the above for one model, as PROGRAM SYNTHE

Arrays are numpy; ``opacity_matrix`` is returned as [nrhox, length] float32,
the memory layout of the reference's (length, nrhox) REAL(4) array.
Errors raise AtlasGPUError with the library's message (the reference prints
and calls EXIT(1)).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import LTE_LINE, Context, ptr

MAXPROF = 1000000  # synthe_module.f90:219
RESOLU_MIN = 300000.0  # synthe.f90 refuses coarser grids


def synthe_grid(wlbeg, wlend, resolu):
    if resolu < RESOLU_MIN:
        raise ValueError(f"resolu below the supported floor: {resolu} < {RESOLU_MIN}")
    g = _lib.Grid()
    rc = _lib.lib().atlasgpu_synthe_grid(float(wlbeg), float(wlend), float(resolu), g)
    if rc != 0:
        raise _lib.AtlasGPUError(rc, "require 0 < wlbeg < wlend")
    return dict(ratio=g.ratio, ratiolg=g.ratiolg, wbegin=g.wbegin, length=g.length, ixwlbeg=g.ixwlbeg)


def make_lte_lines(nbuff, cgf, nelion, elo, gamrf, gamsf, gamwf, code=None):
    """Pack SoA line parameters into the 32-byte BIND(C) lte_line records."""
    n = len(nbuff)
    rec = np.zeros(n, dtype=LTE_LINE)
    rec["nbuff"], rec["cgf"], rec["nelion"], rec["elo"] = nbuff, cgf, nelion, elo
    rec["gamrf"], rec["gamsf"], rec["gamwf"] = gamrf, gamsf, gamwf
    if code is not None:
        rec["code"] = code
    return rec


class Synthe:
    """One SYNTHE synthesis on one GPU context."""

    def __init__(self, ctx: Context, operators):
        self.ctx = ctx
        ctx.set_operators(operators["xtau8"], operators["coefj"], operators["coefh"],
                          operators["ch_j"], operators["ck_j"])

    def bin_lines(self, wlvac, grid):
        wl = np.ascontiguousarray(wlvac, np.float64)
        out = np.zeros(wl.size, np.int32)
        self.ctx.call("atlasgpu_synthe_bin", ptr(wl), wl.size, grid["ratiolg"], grid["ixwlbeg"], ptr(out))
        return out

    def continuum(self, wledge, continall, grid):
        we = np.ascontiguousarray(wledge, np.float64)
        ca = np.ascontiguousarray(continall, np.float64)
        nrhox, stride = ca.shape
        out = np.zeros((nrhox, grid["length"]), np.float32)
        self.ctx.call("atlasgpu_synthe_continuum", ptr(we), we.size, ptr(ca), stride, nrhox,
                      grid["wbegin"], grid["ratio"], grid["length"], ptr(out))
        return out

    def line_opacity(self, lines, grid, resolu, continuum, xnfdop, dopple, xne, txnxn, hckt, maxprof=MAXPROF):
        lines = np.ascontiguousarray(lines, dtype=LTE_LINE)
        cont = np.ascontiguousarray(continuum, np.float32)
        xd = np.ascontiguousarray(xnfdop, np.float64)
        dp = np.ascontiguousarray(dopple, np.float64)
        nrhox, nspec = xd.shape
        vecs = [np.ascontiguousarray(v, np.float64) for v in (xne, txnxn, hckt)]
        out = np.zeros((nrhox, grid["length"]), np.float32)
        self.ctx.call("atlasgpu_synthe_line_opacity", ptr(lines), lines.size, grid["length"], nrhox,
                      float(resolu), ptr(cont), ptr(xd), ptr(dp), nspec, *[ptr(v) for v in vecs],
                      int(maxprof), ptr(out))
        return out

    def spectrum(self, wledge, contabs, contscat, rhox, hkt, grid, opacity):
        we = np.ascontiguousarray(wledge, np.float64)
        ca = np.ascontiguousarray(contabs, np.float64)
        cs = np.ascontiguousarray(contscat, np.float64)
        nrhox, stride = ca.shape
        rx = np.ascontiguousarray(rhox, np.float64)
        hk = np.ascontiguousarray(hkt, np.float64)
        op = np.ascontiguousarray(opacity, np.float32)
        flux = np.zeros(grid["length"])
        cont = np.zeros(grid["length"])
        self.ctx.call("atlasgpu_synthe_spectrum", ptr(we), we.size, ptr(ca), ptr(cs), stride, nrhox, ptr(rx),
                      ptr(hk), grid["wbegin"], grid["ratio"], grid["length"], ptr(op), ptr(flux), ptr(cont))
        return flux, cont

    def set_hydrogen_tables(self, tables, stehle=None):
        """SYNTHE's hydrogen_line_profile tables (the s_* arrays extracted from
        the reference) and the Stehle series (4 dicts as read_stehle gives, None
        entries not loaded; None: the analytic profile throughout)."""
        self._shtab = _lib.HydrogenTables.from_tables(tables, "s_")
        st, self._stehle_keep = (None, []) if stehle is None else _lib.stehle_array(stehle)
        self.ctx.call("atlasgpu_synthe_set_hydrogen_tables", ctypes.byref(self._shtab),
                      None if st is None else st)

    def nlte_opacity(self, records, grid, wlend, continuum, xnfdop, dopple, xne, txnxn, hckt, contx, opacity,
                     velshift_kms=0.0, xnfpel=None, hydrogen=None):
        """compute_line_opacity's normal-metal lines (NLTE_LINE records, nbuff
        = grid index) added into a copy of opacity [nrhox, length] (float32);
        with xnfpel [nrhox, nspec] (populations / RHO) also the autoionizing
        (Shore) lines; with hydrogen = dict(t, xnfph1, xnfph2, xnfhe1, xnfh2)
        [nrhox] (and set_hydrogen_tables) also the hydrogen and deuterium
        lines.  contx: CONTX(26,17) as [17, 26]."""
        rec = np.ascontiguousarray(records, _lib.NLTE_LINE)
        cont = np.ascontiguousarray(continuum, np.float32)
        xd = np.ascontiguousarray(xnfdop, np.float64)
        dp = np.ascontiguousarray(dopple, np.float64)
        nrhox, nspec = xd.shape
        vec = [np.ascontiguousarray(v, np.float64) for v in (xne, txnxn, hckt)]
        out = np.array(opacity, np.float32, copy=True, order="C")
        xp = None if xnfpel is None else np.ascontiguousarray(xnfpel, np.float64)
        hy = None
        if hydrogen is not None:
            hv = [np.ascontiguousarray(hydrogen[k], np.float64) for k in ("t", "xnfph1", "xnfph2", "xnfhe1", "xnfh2")]
            hs = _lib.SyntheHydrogen(*[v.ctypes.data for v in hv])
            hy = ctypes.byref(hs)
        self.ctx.call("atlasgpu_synthe_nlte_opacity", ptr(rec), rec.shape[0], int(grid["length"]), nrhox,
                      float(grid["wbegin"]), float(grid["ratio"]), float(wlend), float(velshift_kms), ptr(cont),
                      ptr(xd), ptr(dp), ptr(xp), nspec, *[ptr(v) for v in vec],
                      ptr(np.ascontiguousarray(contx, np.float64)), hy, ptr(out))
        return out

    def run(self, case):
        """PROGRAM SYNTHE on a prepared case dict (see synthetic.synthe_case):
        returns (wavelength_angstrom, flux, continuum_flux, opacity_matrix).
        With case["nlte"] (NLTE_LINE records, nbuff the grid index) and
        case["contx"] ([17, 26]) also the unit-19 lines, and with
        case["xnfpel"] / case["hydrogen"] their Shore and merged-continuum /
        hydrogen branches (set_hydrogen_tables first for the latter)."""
        grid = synthe_grid(case["wlbeg"], case["wlend"], case["resolu"])
        L = case["lines"]
        nb = self.bin_lines(L["wlvac"], grid)
        lines = make_lte_lines(nb, L["cgf"], L["nelion"], L["elo"], L["gamrf"], L["gamsf"], L["gamwf"])
        atm = case["atm"]
        cont = self.continuum(case["wledge"], case["continall"], grid)
        op = self.line_opacity(lines, grid, case["resolu"], cont, atm["xnfdop"], atm["dopple"], atm["xne"],
                               atm["txnxn"], atm["hckt"])
        if case.get("nlte") is not None and len(case["nlte"]):
            # unit-19 lines (compute_line_opacity, called per depth before the LTE loop at synthe.f90:554)
            op = self.nlte_opacity(case["nlte"], grid, case["wlend"], cont, atm["xnfdop"], atm["dopple"], atm["xne"],
                                   atm["txnxn"], atm["hckt"], case["contx"], op, xnfpel=case.get("xnfpel"),
                                   hydrogen=case.get("hydrogen"))
        flux, cflux = self.spectrum(case["wledge"], case["contabs"], case["contscat"], atm["rhox"], atm["hkt"],
                                    grid, op)
        wave = grid["wbegin"] * grid["ratio"] ** np.arange(grid["length"]) * 10.0
        return wave, flux, cflux, op


def main(argv=None):
    """One synthesis of a synthetic case with the kernel times, e.g.

        python -m atlas12_b200.synthe --lines 20000 --wlbeg 400 --wlend 410

    (the 20,000-line window is the CPU-runnable configuration; 20M lines over
    300-1000 nm with --mol 0.3 the full-optical one)."""
    import argparse
    import json

    from . import operators, synthetic
    ap = argparse.ArgumentParser()
    ap.add_argument("--lines", type=int, default=20000)
    ap.add_argument("--wlbeg", type=float, default=400.0)
    ap.add_argument("--wlend", type=float, default=410.0)
    ap.add_argument("--mol", type=float, default=0.0, help="fraction of molecular lines")
    ap.add_argument("--fp64", action="store_true", help="all-FP64 line opacity")
    ap.add_argument("--reps", type=int, default=2)
    a = ap.parse_args(argv)
    case = synthetic.synthe_case(nlines=a.lines, wlbeg=a.wlbeg, wlend=a.wlend, seed=1, mol_frac=a.mol)
    ctx = Context(0, _lib.PREC_FP64 if a.fp64 else _lib.PREC_MIXED)
    S = Synthe(ctx, operators.load())
    for _ in range(max(a.reps, 1)):
        ctx.enable_timing(True)
        wave, flux, cflux, op = S.run(case)
        ms = {k: ctx.kernel_ms(k) for k in ("synthe_core", "synthe_farfill", "synthe_farwing", "josh_spectrum")}
        work = {k: ctx.kernel_work(k) for k in ("synthe_voigt_evals", "synthe_farwing_updates",
                                                "synthe_farwing_expansions", "synthe_farwing_direct_pairs")}
        ctx.enable_timing(False)
    print(json.dumps({"points": int(flux.size), "lines": a.lines, "kernel_ms": ms, "work": work,
                      "flux_sum": float(np.sum(flux)), "cflux_sum": float(np.sum(cflux))}))
    ctx.close()


if __name__ == "__main__":
    main()
