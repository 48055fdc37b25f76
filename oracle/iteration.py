"""One ATLAS12 iteration on the CPU oracle (test infrastructure).

The iteration of atlas12c.f90:496-606 for the surrogate models, in two
halves split at the frequency sums: begin() runs hydrostatics, the surrogate
populations, KAPCONT (first iteration), LINOP1 and the RT pass over the
frequencies nu0..nu1 (RUN_RT_PASS, atlas12_modules.f90:3880-3951) and
returns the mode-2 sums; end(acc) runs ROSS(3), RADIAP(3), TCORR(3) and the
remap on (possibly several shards') summed accumulators.  Used as the CPU
baseline by bench.py and as the checker of the frequency sharding.
"""
import numpy as np

ACC = ("rjmins", "rdabh", "rdiagj", "flxrad", "raden", "h_total", "accrad", "abross")


class OracleIteration:
    def __init__(self, po, atlas, tables, waveset, rcoset, lines, start, teff, vturb_kms, nu0=1, nu1=None, mh=0.0,
                 grav=None):
        from atlas12_b200 import surrogate as sg
        self.po, self.atlas, self.sg = po, atlas, sg
        self.ops = po.Ops.from_tables(tables)
        self.h = po.tabvoigt(tables["tabvi"], tables["tabh1"])
        self.tl = po.build_tablog()
        self.cut = atlas.cutoff_grid()
        self.iw = atlas.iwavetab(self.cut)
        self.ws, self.rc, self.lines = waveset, rcoset, lines
        self.teff, self.vturb, self.mh = teff, vturb_kms, mh
        self.nu0, self.nu1 = nu0, (waveset.size if nu1 is None else nu1)
        nr = start["t"].size
        self.st = dict(t=start["t"].copy(), rhox=start["rhox"].copy(), p=start["p"].copy(), xne=np.zeros(nr),
                       abross=np.zeros(nr), prad=np.zeros(nr), vturb=np.full(nr, vturb_kms * 1e5),
                       pturb=np.zeros(nr), tauros=start["tauros"].copy(), accrad=np.zeros(nr), raden=np.zeros(nr),
                       oldt1=np.zeros(nr), teff=teff, grav=start["grav"] if grav is None else grav)
        self.store = po.RossStore()
        self.it = 0
        self.tabcont = None

    def begin(self):
        """Iteration it+1 up to the frequency sums over nu0..nu1 (dict of [nrhox] and pradk0)."""
        sg, po, st = self.sg, self.po, self.st
        self.it += 1
        nr = st["t"].size
        if self.it > 1:
            p = st["grav"] * st["rhox"] - st["prad"]
            st["p"] = np.where(p <= 0, np.maximum(st["grav"] * st["rhox"] * 1e-4, 1e-10), p)
        pop = sg.populations(st["t"], st["p"], self.vturb, sg.ATLAS_LINE_POP, mh=self.mh)
        t = st["t"]
        xd = np.zeros((270, nr))
        dp = np.ones((270, nr))
        xx = np.where(pop["dopple"] > 0, pop["xnfp"] / np.maximum(pop["dopple"], 1e-300) / pop["rho"][:, None], 0.0)
        xd[:] = xx[:, :270].T
        dp[:] = np.where(pop["dopple"][:, :270].T > 0, pop["dopple"][:, :270].T, 1.0)
        hkt = sg.HPLANCK / (sg.KBOL * t)
        hckt = hkt * sg.CLIGHT
        txnxn = (pop["nh"] * (1 - pop["xh"]) + 0.42 * 0.085 * pop["nh"]) * (t / 1e4) ** 0.3
        st["xne"] = pop["xne"]
        if self.tabcont is None:
            # KAPCONT (atlas12_modules.f90:19072-19138): ACONT = 1e10 and no
            # KAPP call at cutoff wavelengths not redward of WAVESET(1)
            ka, sgm = sg.continuum_opacity(self.cut, t, st["p"], pop)
            below = self.cut <= self.ws[0]
            ka[below], sgm[below] = 1.0e10, 0.0
            stc = 1 - np.exp(-(sg.CLIGHT_NMS / self.cut)[:, None] * hkt[None, :])
            tab = (ka + sgm) * 1e-3 / stc
            self.tabcont = np.vstack([tab, tab[-1:]])
        atm = dict(xnfdop=xd, dopple=dp, xne=pop["xne"], txnxn=txnxn, hckt=hckt)
        xl, _ = po.atlas_linop1(*self.h, self.tl, self.lines, atm, self.tabcont, self.iw, self.ws)
        self.xlines = xl
        ac, sgm = sg.continuum_opacity(self.ws, t, st["p"], pop)
        acc, _ = po.atlas_rt_pass(self.ops, self.ws, self.rc, ac, sgm, xl, st["rhox"], t, hkt, self.teff,
                                  nu0=self.nu0, nu1=self.nu1)
        return acc

    def end(self, acc):
        """The finish of the current iteration on the summed accumulators; returns max |FLXERR|."""
        err, self.finish = self.po.atlas_finish(self.st, acc, self.it, self.store)
        return err

    def step(self):
        return self.end(self.begin())


def pack(acc, nrhox):
    """Accumulators as one vector [8*nrhox + 1] (the device sums layout)."""
    return np.concatenate([np.asarray(acc[k], np.float64) for k in ACC] + [np.array([acc["pradk0"]])])


def unpack(v, nrhox):
    d = {k: np.array(v[q * nrhox:(q + 1) * nrhox], np.float64) for q, k in enumerate(ACC)}
    d["pradk0"] = float(v[8 * nrhox])
    return d
