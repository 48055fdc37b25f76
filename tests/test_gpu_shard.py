"""Frequency shards of one device-resident ATLAS12 model (atlasgpu_model_set_shard,
_set_sums_buffer, _iterate_begin/_end) on one GPU.

Two models each own half of the frequencies; per iteration both run up to
their sums, the sums are added (what the all-reduce does across GPUs) and both
finish on the total.  After 3 iterations each must hold the unsharded model's
structure and max |FLXERR| history (relative 1e-8: only the grouping of the
frequency sums differs).  The two shards run one after the other on one GPU;
no kernel waits on another.
"""
import numpy as np
import pytest

from atlas12_b200 import atlas, synthetic
from atlas12_b200.shard import shard_range

pytestmark = pytest.mark.gpu


def test_two_shards_match_unsharded_model(gpu_ctx, tables):
    import torch
    ws, rc = synthetic.geometric_waveset(9.0, 160000.0, 3000)
    lines = synthetic.atlas_lines(20000, ws[2], ws[-3], seed=4)
    ref = atlas.AtlasModel(gpu_ctx, tables, linedata=lines, waveset=ws, rcoset=rc)
    n, hist = ref.iterate(max_iter=3, tol_percent=0.0, graph=True)
    want = ref.structure()
    ref.close()
    shards = []
    for r in range(2):
        m = atlas.AtlasModel(gpu_ctx, tables, linedata=lines, waveset=ws, rcoset=rc)
        m.set_shard(*shard_range(ws.size, r, 2))
        s = torch.zeros(8 * m.nrhox + 1, dtype=torch.float64, device="cuda")
        m.set_sums_buffer(s)
        shards.append((m, s))
    got = []
    for _ in range(3):
        for m, _s in shards:
            m.iterate_begin()
        gpu_ctx.synchronize()
        total = shards[0][1] + shards[1][1]
        for _m, s in shards:
            s.copy_(total)
        torch.cuda.synchronize()
        got.append([m.iterate_end() for m, _s in shards])
    got = np.array(got)
    np.testing.assert_allclose(got[:, 0], hist, rtol=1e-8)
    np.testing.assert_array_equal(got[:, 0], got[:, 1])
    for m, _s in shards:
        st = m.structure()
        for k in ("t", "p", "rhox"):
            np.testing.assert_allclose(st[k], want[k], rtol=1e-8, err_msg=k)
        m.set_sums_buffer(None)
        m.close()
    # a shard outside the grid is refused
    m = atlas.AtlasModel(gpu_ctx, tables, linedata=lines[:10], waveset=ws, rcoset=rc)
    with pytest.raises(Exception, match="outside"):
        m.set_shard(2000, ws.size + 1)
    m.close()
