"""Input builders shared by the tests (geometry of the golden fixtures,
restated from tests/golden/make_golden.py, plus larger seeded cases)."""
from __future__ import annotations

import numpy as np


def stub_tree(nx, ny, nz):
    nodes = np.array([[ny + 8.0, nx + 8.0, nz + 8.0], [ny + 8.0, nx + 8.0, nz + 12.0]])
    return nodes, np.array([[0, 1]]), np.array([0.0, 1.0])


def iso_case():
    nx, ny, nz = 16, 16, 4
    S = np.ones((nx, ny, nz), np.uint8)
    phi = np.ones(S.shape, np.float32)
    ect = np.zeros(S.shape, bool)
    ect[:4, :4, :] = True
    nodes, el, act = stub_tree(nx, ny, nz)
    kw = dict(voxel_size=0.25, dx_p=0.25, sigma_P=0.0, sigma_M=0.13, Cm=0.01, A_P=133.33,
              A_M=140.0, R_P=0.015, dt=0.02, T=20.0,
              stim_protocol=[dict(name="corner", target="ectopic", amp=0.52, dur=1.0, onset=0.0)],
              ectopic_region=ect, stim_len_mm=1.0, c_pmj=0.0, n_pmj=1)
    return (nodes, el, act, S, phi), kw


def aniso_case():
    nx, ny, nz = 12, 10, 6
    rng = np.random.default_rng(7)
    S = np.ones((nx, ny, nz), np.uint8)
    S[0, 0, :] = 0
    S[nx - 1, ny - 1, nz - 1] = 0
    ii, jj, kk = np.indices(S.shape)
    phi = (kk / (nz - 1)).astype(np.float32)
    phi[S == 0] = np.nan
    a = 0.4 * ii + 0.3 * jj + rng.uniform(0, 0.2, S.shape)
    b = 0.5 * kk / nz
    f = np.stack([np.cos(a) * np.cos(b), np.sin(a) * np.cos(b), np.sin(b)], -1)
    f /= np.linalg.norm(f, axis=-1, keepdims=True)
    fibre = f.astype(np.float32)
    nodes = np.array([[1.0, 1.0, -2.0], [4.0, 5.0, -1.0], [8.0, 3.0, -0.5],
                      [3.0, 9.0, -0.5], [7.0, 10.0, -0.6]])
    el = np.array([[0, 1], [1, 2], [1, 3], [3, 4]])
    act = np.array([0.0, 1.0, 2.0, 2.0, 3.0])
    ect = np.zeros(S.shape, bool)
    ect[8:12, 6:10, 3:6] = True
    prot = [dict(name="av_node", target="root", amp=12.0, dur=2.0, onset=0.0),
            dict(name="focus", target="ectopic", amp=1.0, dur=2.0, onset=1.0)]
    kw = dict(voxel_size=0.4, dx_p=0.2, sigma_P=0.45, sigma_l=0.34, sigma_t=0.06, Cm=0.01,
              A_M=140.0, R_P=0.015, dt=0.02, T=20.0, stim_protocol=prot, ectopic_region=ect,
              stim_len_mm=0.5, c_pmj=0.01, n_pmj=2, phi_endo_max=0.3, phi_epi_min=0.7)
    return (nodes, el, act, S, phi), fibre, kw


def ragged_aniso_case(seed=11, shape=(28, 24, 18), T=30.0):
    """Irregular mask (two overlapping ellipsoidal shells with jitter), smooth
    fibres, phenotype layers, Purkinje tree with several junctions."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    ii, jj, kk = np.indices(shape).astype(np.float64)
    r = np.sqrt(((ii - nx / 2) / (nx / 2.2)) ** 2 + ((jj - ny / 2) / (ny / 2.2)) ** 2 +
                ((kk - nz / 2) / (nz / 2.2)) ** 2)
    r += rng.uniform(-0.04, 0.04, shape)
    S = ((r > 0.55) & (r < 1.0)).astype(np.uint8)
    phi = np.clip((r - 0.55) / 0.45, 0, 1).astype(np.float32)
    phi[S == 0] = np.nan
    th = 0.3 * ii + 0.2 * kk
    f = np.stack([np.cos(th), np.sin(th) * 0.8, np.sin(th) * 0.6], -1)
    f /= np.linalg.norm(f, axis=-1, keepdims=True)
    nodes = np.array([[ny / 2, nx / 2, nz / 2], [ny / 2 + 3, nx / 2 + 2, nz / 2],
                      [ny / 2 + 6, nx / 2 + 3, nz / 2 + 2], [ny / 2 + 1, nx / 2 + 6, nz / 2 - 1],
                      [ny / 2 - 4, nx / 2 + 1, nz / 2 + 3]])
    el = np.array([[0, 1], [1, 2], [1, 3], [0, 4]])
    act = np.array([0.0, 1.0, 2.0, 2.0, 1.0])
    kw = dict(voxel_size=0.4, dx_p=0.2, sigma_P=0.45, sigma_l=0.34, sigma_t=0.06, Cm=0.01,
              A_M=140.0, R_P=0.015, dt=0.02, T=T,
              stim_protocol=[dict(name="av", target="root", amp=30.0, dur=2.0, onset=0.0),
                             dict(name="focus", target="ectopic", amp=1.0, dur=2.0, onset=0.5)],
              stim_len_mm=0.6, c_pmj=0.01, n_pmj=3, phi_endo_max=0.3, phi_epi_min=0.7)
    ect = np.zeros(shape, bool)
    ect[:, : ny // 3, :] = True
    kw["ectopic_region"] = ect & (S == 1) & (kk < nz / 2)
    return (nodes, el, act, S, phi), f.astype(np.float32), kw
