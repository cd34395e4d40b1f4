"""Snapshot and activation-map files against the upstream writer's own
output (tests/golden/act_maps_iso.npz, made by running the upstream
compute_activation_maps / save_activation_maps)."""
import numpy as np
import pytest

from hrdayapy_b200.simulation import (ActivationMaps, VmSnapshots, compute_activation_maps,
                                      load_activation_maps, load_vm_snapshots,
                                      save_activation_maps)

KEYS = ("node_ids", "coords_mm", "vox_idx", "activation_times", "deactivation_times",
        "n_activations", "n_deactivations", "act_threshold", "deact_threshold", "grid_shape")


def _same_file(path, g, prefix):
    z = np.load(path)
    assert set(z.files) == set(KEYS) | {"source_vm_path"}
    for k in KEYS:
        ref = g[prefix + k]
        assert z[k].dtype == ref.dtype, k
        assert z[k].shape == ref.shape, k
        np.testing.assert_array_equal(z[k], ref, err_msg=k)


def test_debounced_chatter_vs_upstream(golden, tmp_path):
    g = golden("act_maps_iso.npz")
    vs = VmSnapshots(node_ids=np.arange(6, dtype=np.int32), coords_mm=g["chatter_in_coords"],
                     vox_idx=g["chatter_in_vox"], Vm=g["chatter_in_Vm"], time_vm=g["chatter_in_t"],
                     dt_solver=0.5, vm_save_dt=0.5)
    m = compute_activation_maps(vs, None, act_threshold=-40.0, deact_threshold=-45.0,
                                min_event_gap_ms=3.0, save_path=tmp_path / "chatter")
    _same_file(tmp_path / "chatter.npz", g, "chatter_")
    assert m.n_events == max(g["chatter_activation_times"].shape[1],
                             g["chatter_deactivation_times"].shape[1])


def test_slab_snapshots_to_maps_vs_upstream(golden, tmp_path):
    """Oracle run (FP64, the upstream method) -> this package's snapshot
    writer -> loader -> maps -> writer: the upstream file, array for array."""
    from hrdayapy_b200.monodomain import save_vm_snapshots
    from oracle import mono as orc
    from tests import cases
    g = golden("act_maps_iso.npz")
    args, kw = cases.iso_case()
    nodes, el, act, S, phi = args
    kw = dict(kw, T=float(g["T"]))
    r = orc.run(nodes, el, act, S, phi, vm_save_dt=float(g["vm_save_dt"]), **kw)
    vox = r["vox_idx"]
    coords = (vox[:, [1, 0, 2]] * np.float32(kw["voxel_size"])).astype(np.float32)
    save_vm_snapshots(tmp_path / "vm.npz", np.arange(len(vox), dtype=np.int32) + r["Np"], coords,
                      vox, r["Vm"], r["time_vm"], kw["dt"], float(g["vm_save_dt"]))
    snap = load_vm_snapshots(tmp_path / "vm")
    assert snap.n_frames == r["Vm"].shape[0] and snap.N_myo == len(vox)
    compute_activation_maps(snap, S, act_threshold=-20.0, deact_threshold=-60.0,
                            save_path=tmp_path / "maps.npz")
    _same_file(tmp_path / "maps.npz", g, "slab_")
    m = load_activation_maps(tmp_path / "maps")
    assert m.source_vm_path.endswith("vm.npz")
    apd = m.apd_map(1)
    assert np.isfinite(apd).all() and apd.min() > 100.0
    grid = m.activation_grid(1)
    assert grid.shape == S.shape and np.isfinite(grid).all()
    assert np.isnan(m.activation_map(2)).all()


def test_containers_and_errors(tmp_path):
    rng = np.random.default_rng(0)
    n, f = 5, 8
    vs = VmSnapshots(node_ids=np.arange(n, dtype=np.int32),
                     coords_mm=rng.uniform(0, 10, (n, 3)).astype(np.float32),
                     vox_idx=rng.integers(0, 4, (n, 3)).astype(np.int32),
                     Vm=rng.normal(-60, 30, (f, n)).astype(np.float32),
                     time_vm=np.arange(f, dtype=np.float32), dt_solver=1.0, vm_save_dt=1.0)
    k = vs.nearest_node(vs.coords_mm[3])
    assert k == 3 and vs.vm_at_node(3).shape == (f,)
    with pytest.raises(IndexError):
        vs.vm_at_node(n)
    fld, t = vs.field_at_time(2.4)
    assert t == 2.0 and fld.shape == (n,)
    assert 3 in vs.nodes_in_sphere(vs.coords_mm[3], 0.1)
    assert vs.mean_vm_in_sphere([1e6, 0, 0], 1.0).shape == (f,)
    with pytest.raises(ValueError):
        compute_activation_maps(VmSnapshots(vs.node_ids, vs.coords_mm, vs.vox_idx, vs.Vm[:1],
                                            vs.time_vm[:1], 1.0, 1.0))
    m = compute_activation_maps(vs)          # grid_shape from the bounding box
    assert tuple(m.grid_shape) == tuple(vs.vox_idx.max(axis=0) + 1)
    save_activation_maps(m, tmp_path / "m")
    assert isinstance(load_activation_maps(tmp_path / "m.npz"), ActivationMaps)
    with pytest.raises(FileNotFoundError):
        load_activation_maps(tmp_path / "absent")
    with pytest.raises(FileNotFoundError):
        load_vm_snapshots(tmp_path / "absent")
    np.savez(tmp_path / "bad.npz", node_ids=np.zeros(1))
    with pytest.raises(KeyError):
        load_activation_maps(tmp_path / "bad.npz")
    with pytest.raises(KeyError):
        load_vm_snapshots(tmp_path / "bad.npz")
    m.grid_shape = None
    with pytest.raises(ValueError):
        m.activation_grid()
