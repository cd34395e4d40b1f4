"""Autotuner (hrdayapy_b200.autotune): re-bricking a prepared problem on the
CPU must give exactly what preparing it with that brick shape gives; on the
GPU the tuner times every candidate and its winner runs the same arithmetic
as the problem it came from."""
import numpy as np
import pytest

from tests import cases


def _prep(brick, T=2.0):
    from hrdayapy_b200 import monodomain as M
    args, fibre, kw = cases.ragged_aniso_case(T=T)
    nodes, el, act, S, phi = args
    prob, _ = M.prepare(nodes, el, act, S, S, phi, fibre_dir=fibre, anisotropic=True,
                        vm_save_dt=kw["dt"], act_threshold=-20.0, deact_threshold=-20.0,
                        brick=brick, **dict(kw, A_P=2.0 / kw["R_P"]))
    return prob


@pytest.mark.parametrize("brick", [(4, 8, 8), (2, 4, 16), (8, 8, 8)])
def test_relayout_equals_direct_preparation(brick):
    from hrdayapy_b200.autotune import relayout
    src = _prep((4, 4, 8))
    ref = _prep(brick)
    got = relayout(src, brick)
    assert got.layout.brick == ref.layout.brick and got.layout.n_bricks == ref.layout.n_bricks
    np.testing.assert_array_equal(got.layout.brick_nbr, ref.layout.brick_nbr)
    np.testing.assert_array_equal(got.layout.slot_of_node, ref.layout.slot_of_node)
    np.testing.assert_array_equal(got.tag, ref.tag)
    np.testing.assert_array_equal(np.ravel(got.wface), np.ravel(ref.wface))
    np.testing.assert_array_equal(np.ravel(got.doff), np.ravel(ref.doff))
    np.testing.assert_array_equal(got.pk_idx, ref.pk_idx)
    m = (np.asarray(ref.tag) & (1 << 28)) != 0        # junction rows are read where tagged
    np.testing.assert_array_equal(np.asarray(got.pmj_row)[m], np.asarray(ref.pmj_row)[m])


@pytest.mark.gpu
def test_tuner_picks_a_candidate_that_runs_identically(tmp_path):
    from hrdayapy_b200 import monodomain as M
    from hrdayapy_b200.autotune import tune
    prob = _prep((4, 4, 8), T=6.0)
    cache = tmp_path / "tune.json"
    best, table = tune(prob, steps=40, warmup=10, cache_path=str(cache))
    assert len([t for t in table if "voxel_steps_per_s" in t]) == 8
    assert table[0]["voxel_steps_per_s"] >= max(t.get("voxel_steps_per_s", 0) for t in table)
    again, table2 = tune(prob, cache_path=str(cache))        # cache hit
    assert tuple(again.layout.brick) == tuple(best.layout.brick) and again.kernel == best.kernel

    def vm(p):
        sim = M.MonoHandle(p)
        sim.run(p.n_steps, graph_chunk=50)
        out = sim.vm_frames()
        sim.close()
        return out

    np.testing.assert_array_equal(vm(best), vm(prob))
