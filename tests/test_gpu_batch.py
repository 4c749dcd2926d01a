"""The batched form (one persistent launch over many (field, sun) items).

Item i of a batch traces the same Philox rays as a plain qmcrt_trace with
params.item = i, so its integer count map must equal that trace's exactly,
whatever the chunking, tile or graph replay; float flux maps agree to float
atomic-ordering tolerance.
"""
import ctypes as C

import numpy as np
import pytest

from onemirror_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from onemirror_b200.scene import Batch, SolarScene  # noqa: E402

RAYS = 1 << 20  # 4096 points per item: at least one per heliostat of the 4000-heliostat field


# every third sun position of the day (the first and last, at 5 deg, spread
# the spots widest) on all three fields
PICKS = list(range(0, 45, 3)) + [44]


@pytest.fixture(scope="module")
def setup():
    fields, suns, items, params = W.batched(rays_per_item=RAYS)
    assert [f.n for f in fields] == [300, 1000, 4000] and len(suns) == 45
    scenes = [SolarScene.from_workload(f) for f in fields]
    its = [(f, suns[k][3]) for f in range(3) for k in PICKS]
    b = Batch(scenes, its, params)
    yield scenes, its, params, b
    b.close()
    for s in scenes:
        s.close()


@pytest.fixture(scope="module")
def plains(setup):
    """Count maps of the plain traces of every item."""
    scenes, its, params, b = setup
    return [plain(scenes, its, params, i)[0] for i in range(len(its))]


def plain(scenes, its, params, i):
    si, sun = its[i]
    p = W.params(int(params.rays), params.rays_per_point, params.point_spacing, seed=params.seed)
    p.item = i
    r = scenes[si].trace(sun, p)
    torch.cuda.synchronize()
    return r["counts"].cpu().numpy().view(np.uint32), r["flux"].cpu().numpy(), r["stats"]


def test_items_equal_plain_traces(setup):
    scenes, its, params, b = setup
    b.run()
    torch.cuda.synchronize()
    for i in range(len(its)):
        c, f, st = b.read(i)
        pc, pf, pst = plain(scenes, its, params, i)
        assert np.array_equal(c, pc), i
        assert np.allclose(f, pf, rtol=1e-4, atol=1e-3 * pf.max())
        assert abs(st.intercept_ratio - pst.intercept_ratio) < 1e-5
        assert abs(st.total_power - pst.total_power) / pst.total_power < 1e-9


@pytest.mark.parametrize("chunk,ctas,tile", [(256, 1, 0), (4096, 3, 32), (65536, 4, 48), (1 << 20, 2, 0),
                                             (16384, 4, 48), (262144, 3, 32)])
def test_tunings_do_not_change_counts(setup, plains, chunk, ctas, tile):
    """Every tuning, the shared-memory tiles included (a tile is anchored on
    the chunk's first point; hits outside it go to the global maps), gives
    each item the counts of its plain trace."""
    scenes, its, params, b = setup
    b.set_tuning(chunk, ctas, tile)
    b.run()
    for i in range(len(its)):
        c, f, st = b.read(i)
        assert np.array_equal(c, plains[i]), (chunk, ctas, tile, i)


def test_graph_replay_matches_direct_run(setup):
    scenes, its, params, b = setup
    b.set_tuning(16384, 4, 32)
    b.run()
    ref = [b.read(i)[0] for i in range(len(its))]
    b.capture()
    for _ in range(2):
        b.launch()
        torch.cuda.synchronize()
        for i in range(len(its)):
            assert np.array_equal(b.read(i)[0], ref[i])


def test_autotune_picks_a_valid_tuning(setup):
    scenes, its, params, b = setup
    t = b.autotune()
    assert t.chunk_rays in (16384, 65536, 262144) and t.ctas_per_sm in (3, 4) and t.tile in (0, 32, 48)
    assert t.ms > 0
    b.run()
    assert np.array_equal(b.read(3)[0], plain(scenes, its, params, 3)[0])


def test_batch_argument_errors(setup):
    scenes, its, params, b = setup
    bad = W.params(RAYS, 256, 0.4, quirks=capi.QUIRK_SKIP_ORIGIN_CELL)
    with pytest.raises(capi.QmcrtError) as e:
        Batch(scenes, its, bad)
    assert e.value.status == capi.ERR_NOT_SUPPORTED
    with pytest.raises(capi.QmcrtError):
        Batch(scenes, [(5, its[0][1])], params)
    with pytest.raises(capi.QmcrtError):
        b.set_tuning(1000, 4, 0)
