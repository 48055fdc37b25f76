"""The device surrogate (EOS / continuum stand-in) agrees with atlas12_b200.surrogate."""
import numpy as np
import pytest

from atlas12_b200 import _lib, surrogate
from atlas12_b200._lib import ptr

pytestmark = pytest.mark.gpu


def test_device_surrogate_matches_numpy(gpu_ctx):
    m = surrogate.grey_model(5777.0, 4.44)
    t, p = m["t"], m["p"]
    wave = np.geomspace(9.0, 160000.0, 777)
    nr, nw = t.size, wave.size
    ka, sg = np.zeros((nw, nr)), np.zeros((nw, nr))
    xne, xd = np.zeros(nr), np.zeros((270, nr))
    gpu_ctx.call("atlasgpu_surrogate_eval", nr, ptr(t), ptr(p), 1.5, nw, ptr(wave), ptr(ka), ptr(sg), ptr(xne), ptr(xd))
    rk, rs = surrogate.continuum_opacity(wave, t, p)
    pop = surrogate.populations(t, p, 1.5, surrogate.ATLAS_LINE_POP)
    np.testing.assert_allclose(xne, pop["xne"], rtol=1e-10)
    np.testing.assert_allclose(ka, rk, rtol=1e-9)
    np.testing.assert_allclose(sg, rs, rtol=1e-10)
    ref = np.where(pop["dopple"] > 0, pop["xnfp"] / np.maximum(pop["dopple"], 1e-300) / pop["rho"][:, None], 0.0)
    np.testing.assert_allclose(xd, ref[:, :270].T, rtol=1e-10, atol=1e-300)
