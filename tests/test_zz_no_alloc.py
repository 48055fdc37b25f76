"""The RT pass for callers that cannot allocate device memory.

A caller that manages all of its device memory itself (its own allocator or
pool, a fixed memory budget) passes every input and output as a device
pointer to atlasgpu_atlas_rt_pass_noalloc, which keeps its only scratch in a
fixed array inside the library.  Its results must equal those of the
ordinary entry point atlasgpu_atlas_rt_pass on the same inputs, call after
call (the shared scratch must not carry one call's state into the next), and
the padding depths of a kw > nrhox call must come back zero.
Tolerance: relative 1e-9 on the frequency sums, 1e-6 per frequency on H(1)
(the same bounds the RT-pass parity test uses).

This file is named to be collected last.
"""
import numpy as np
import pytest

from atlas12_b200 import _lib, atlas, surrogate, synthetic
from atlas12_b200._lib import ptr

pytestmark = pytest.mark.gpu


def _inputs(numnu, seed):
    m = surrogate.grey_model(5777.0, 4.44)
    pop = surrogate.populations(m["t"], m["p"], 1.5)
    ws, rc = synthetic.geometric_waveset(9.0, 160000.0, numnu)
    ac, sg = surrogate.continuum_opacity(ws, m["t"], m["p"], pop)
    rng = np.random.default_rng(seed)
    xl = ac * 10.0 ** rng.uniform(-3.0, 2.0, ac.shape)  # XLINES [numnu][kw]
    hkt = surrogate.HPLANCK / (surrogate.KBOL * m["t"])
    return dict(ws=ws, rc=rc, ac=ac, sg=sg, xl=xl, rhox=m["rhox"], t=m["t"], hkt=hkt)


def _pad(a, kw):
    """[numnu][nrhox] -> [numnu][kw], the padding depths filled with values the pass must not read."""
    out = np.full((a.shape[0], kw), 1.0e30)
    out[:, :a.shape[1]] = a
    return out


def test_noalloc_rt_pass_matches_rt_pass_call_after_call(tables):
    torch = pytest.importorskip("torch")
    if _lib.device_count() == 0:
        pytest.skip("no CUDA device")
    ctx = _lib.Context(0, _lib.PREC_MIXED)
    A = atlas.Atlas(ctx, tables)

    def dev(x):
        return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device="cuda")

    # three calls in a row sharing the fixed scratch: 72 depths in arrays of
    # kw = 72, then of kw = 80 (the reference's kw with 72 depths: the
    # depths 72..79 of every sum must come back zero, not left over from the
    # call before), then kw = 72 again
    for call, (seed, kw) in enumerate(((1, 72), (2, 80), (3, 72))):
        d = _inputs(2500 + 500 * call, seed)
        nr = d["rhox"].size
        ref, ref_hs = A.rt_pass(d["ws"], d["rc"], d["ac"], d["sg"], d["xl"], d["rhox"], d["t"], d["hkt"], 5777.0)
        numnu = d["ws"].size
        dws, drc = dev(d["ws"]), dev(d["rc"])
        dac, dsg = dev(_pad(d["ac"], kw)), dev(_pad(d["sg"], kw))
        dxt = dev(_pad(d["xl"], kw).T)  # [kw][numnu]
        drx, dt, dhk = dev(d["rhox"]), dev(d["t"]), dev(d["hkt"])
        sums = torch.full((8 * kw + 1,), np.nan, dtype=torch.float64, device="cuda")
        hs = torch.zeros(numnu, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        ctx.call("atlasgpu_atlas_rt_pass_noalloc", numnu, ptr(dws), ptr(drc), ptr(dac), ptr(dsg), None, kw,
                 ptr(dxt), nr, ptr(drx), ptr(dt), ptr(dhk), 5777.0, ptr(sums), ptr(hs))
        ctx.synchronize()
        got = sums.cpu().numpy()
        for q, k in enumerate(atlas.ACC_NAMES):
            np.testing.assert_allclose(got[q * kw:q * kw + nr], ref[k], rtol=1e-9, err_msg=f"call {call} {k}")
            np.testing.assert_array_equal(got[q * kw + nr:(q + 1) * kw], 0.0, err_msg=f"call {call} {k} padding")
        assert abs(got[8 * kw] - ref["pradk0"]) <= 1e-9 * abs(ref["pradk0"])
        np.testing.assert_allclose(hs.cpu().numpy(), ref_hs, rtol=1e-6)
    # sizes beyond the fixed scratch are refused with a clear error
    with pytest.raises(_lib.AtlasGPUError, match="exceeds the fixed scratch limit"):
        ctx.call("atlasgpu_atlas_rt_pass_noalloc", 10, ptr(dws), ptr(drc), ptr(dac), ptr(dsg), None, 101,
                 ptr(dxt), 72, ptr(drx), ptr(dt), ptr(dhk), 5777.0, ptr(sums), ptr(hs))
    ctx.close()
