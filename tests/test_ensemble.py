"""Batched ensembles of heart variants (hrdayapy_b200.ensemble): host-side
concatenation on the CPU, and on the GPU one ensemble run against separate
runs of its variants -- every variant must evolve bit for bit as it does
alone."""
import numpy as np
import pytest

from tests import cases


def _variant(seed, shape, T, brick=(4, 4, 8)):
    from hrdayapy_b200 import monodomain as M
    args, fibre, kw = cases.ragged_aniso_case(seed=seed, shape=shape, T=T)
    nodes, el, act, S, phi = args
    kwx = dict(kw, A_P=2.0 / kw["R_P"])
    prob, _ = M.prepare(nodes, el, act, S, S, phi, fibre_dir=fibre, anisotropic=True,
                        vm_save_dt=kw["dt"], act_threshold=-20.0, deact_threshold=-20.0,
                        brick=brick, **kwx)
    return prob


def test_concatenation_keeps_variants_apart():
    from hrdayapy_b200.ensemble import build_ensemble
    pa = _variant(11, (28, 24, 18), 2.0)
    pb = _variant(12, (24, 20, 16), 2.0)
    ens = build_ensemble([pa, pb], gks=[1.0, 1.4], gkr=[1.0, 0.6])
    p = ens.problem
    na, nb_ = pa.layout.n_bricks, pb.layout.n_bricks
    assert p.layout.n_bricks == na + nb_ and p.n_myo == pa.n_myo + pb.n_myo
    assert p.n_pk == pa.n_pk + pb.n_pk
    nbr = p.layout.brick_nbr
    # neighbour tables never cross variants
    assert ((nbr[:na] < na) | (nbr[:na] < 0)).all()
    assert ((nbr[na:] >= na) | (nbr[na:] < 0)).all()
    assert (p.brick_variant[:na] == 0).all() and (p.brick_variant[na:] == 1).all()
    # Purkinje CSR of variant b points into b's nodes / slots
    idx = p.pk_idx[p.pk_ptr[pa.n_pk]:]
    pk = idx[idx >= 0]
    slots = -idx[idx < 0] - 1
    assert (pk >= pa.n_pk).all() and (slots >= pa.layout.n_slots).all()
    assert p.site_amp.shape[0] == 2 and p.site_on.shape == (2, pa.n_steps + 1)
    np.testing.assert_array_equal(p.site_on[1], pb.site_on)
    a_part, b_part = ens.split(np.arange(p.n_myo))
    assert len(a_part) == pa.n_myo and len(b_part) == pb.n_myo
    with pytest.raises(ValueError):
        build_ensemble([pa, _variant(12, (24, 20, 16), 2.0, brick=(4, 8, 8))])


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [0, 2])
def test_ensemble_matches_separate_runs(kernel):
    from hrdayapy_b200 import monodomain as M
    from hrdayapy_b200.ensemble import build_ensemble
    pa = _variant(11, (28, 24, 18), 20.0)
    pb = _variant(12, (24, 20, 16), 20.0)
    gks, gkr = [1.0, 1.4], [1.0, 0.6]
    ens = build_ensemble([pa, pb], gks=gks, gkr=gkr)

    def run(p):
        p.kernel = kernel
        sim = M.MonoHandle(p)
        sim.run(p.n_steps, graph_chunk=50)
        vm = sim.vm_frames()
        a, na, d, nd = sim.events()
        sim.close()
        return vm, a, na

    vm_e, act_e, n_e = run(ens.problem)
    for v, p in enumerate((pa, pb)):
        p.variant_gks = np.array([gks[v]])
        p.variant_gkr = np.array([gkr[v]])
        vm_s, act_s, n_s = run(p)
        np.testing.assert_array_equal(ens.split(vm_e)[v], vm_s)
        np.testing.assert_array_equal(ens.split(act_e)[v], act_s)
        np.testing.assert_array_equal(ens.split(n_e)[v], n_s)
    # the ionic scaling reaches the second variant: it differs from an unscaled run
    pb.variant_gks = None
    pb.variant_gkr = None
    vm_u, _, _ = run(pb)
    assert np.abs(ens.split(vm_e)[1] - vm_u).max() > 0.1


@pytest.mark.gpu
def test_theta_scheme_ensemble_matches_separate_runs():
    """At theta = 0.5 the ensemble's CG solves all variants together (one
    set of CG scalars), so variants are not bit-identical to separate runs,
    but every variant stays within the parity tolerances of its own run."""
    import dataclasses
    from hrdayapy_b200 import monodomain as M
    from hrdayapy_b200.ensemble import build_ensemble
    pa = _variant(11, (28, 24, 18), 20.0)
    pb = _variant(12, (24, 20, 16), 20.0)
    cn = dict(theta=0.5, cn_tol=1e-6, cn_max_iter=100)
    pa, pb = dataclasses.replace(pa, **cn), dataclasses.replace(pb, **cn)
    ens = build_ensemble([pa, pb])

    def run(p):
        sim = M.MonoHandle(p)
        sim.run(p.n_steps, graph_chunk=16)
        vm = sim.vm_frames()
        a, na, d, nd = sim.events()
        _, _, unconv, brk = sim.cn_stats()
        sim.close()
        assert unconv == 0 and brk == 0
        return vm, a[0]

    vm_e, act_e = run(ens.problem)
    for v, p in enumerate((pa, pb)):
        vm_s, act_s = run(p)
        ve = ens.split(vm_e)[v]
        assert np.sqrt(np.mean((ve.astype(np.float64) - vm_s) ** 2)) <= 0.5
        ae = ens.split(act_e)[v]
        ok = np.isfinite(act_s)
        assert (np.isfinite(ae) == ok).all()
        assert np.max(np.abs(ae[ok] - act_s[ok])) <= 0.1


@pytest.mark.gpu
def test_ensemble_variants_vs_fp64_oracle():
    """The batched ensemble's per-variant parameters (longitudinal
    conductivity, g_Ks and g_Kr multipliers, its own geometry and tree)
    against FP64 oracle runs of each variant with the same parameters: two
    variants of uneven size advanced in one launch per step, Vm RMS <= 0.5 mV
    over every frame and max activation-time error <= 0.1 ms at -20 mV."""
    from hrdayapy_b200 import monodomain as M
    from hrdayapy_b200.ensemble import build_ensemble
    from oracle import mono as orc
    spec = [dict(seed=11, shape=(28, 24, 18), sigma_l=0.25, gks=0.7, gkr=1.3),
            dict(seed=12, shape=(24, 20, 16), sigma_l=0.38, gks=1.4, gkr=0.6)]
    probs, inputs = [], []
    for sp in spec:
        args, fibre, kw = cases.ragged_aniso_case(seed=sp["seed"], shape=sp["shape"], T=25.0)
        kw = dict(kw, sigma_l=sp["sigma_l"])
        nodes, el, act, S, phi = args
        prob, _ = M.prepare(nodes, el, act, S, S, phi, fibre_dir=fibre, anisotropic=True,
                            vm_save_dt=kw["dt"], act_threshold=-20.0, deact_threshold=-20.0,
                            brick=(4, 4, 8), **dict(kw, A_P=2.0 / kw["R_P"]))
        probs.append(prob)
        inputs.append((args, fibre, kw))
    ens = build_ensemble(probs, gks=[s["gks"] for s in spec], gkr=[s["gkr"] for s in spec])
    sim = M.MonoHandle(ens.problem)
    sim.run(ens.problem.n_steps, graph_chunk=50)
    vm_e = sim.vm_frames()
    a_e, n_e, _, _ = sim.events()
    sim.close()
    for v, (sp, (args, fibre, kw)) in enumerate(zip(spec, inputs)):
        nodes, el, act, S, phi = args
        r = orc.run(nodes, el, act, S, phi, fibre_dir=fibre, anisotropic=True, vm_save_dt=kw["dt"],
                    gks_scale=sp["gks"], gkr_scale=sp["gkr"], **kw)
        vm = ens.split(vm_e)[v]
        assert vm.shape == r["Vm"].shape
        rms = float(np.sqrt(np.mean((vm.astype(np.float64) - r["Vm"]) ** 2)))
        ra = orc.activation_maps(r["Vm"], r["time_vm"], -20.0, -20.0)["activation_times"][:, 0]
        ok = np.isfinite(ra)
        ae, ne = ens.split(a_e[0])[v], ens.split(n_e)[v]
        assert ok.sum() > 0.5 * len(ok)
        assert (ne[ok] >= 1).all() and (ne[~ok] == 0).all()
        err = float(np.max(np.abs(ae[ok] - ra[ok])))
        print(f"ensemble variant {v} ({len(ok)} voxels, sigma_l {sp['sigma_l']}, g_Ks x{sp['gks']}, "
              f"g_Kr x{sp['gkr']}): Vm RMS {rms:.2e} mV, max |dLAT| {err:.2e} ms vs FP64")
        assert rms <= 0.5 and err <= 0.1
