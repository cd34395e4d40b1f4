"""Torso test inputs: the golden fixture's case and larger seeded variants."""
import numpy as np


def golden_case(g):
    lab = g["labels"]
    sigma_map = {int(k): float(v) for k, v in zip(g["sigma_keys"], g["sigma_vals"])}
    vox = g["heart_vox"]
    coords = vox[:, [1, 0, 2]].astype(np.float64) * float(g["h_fine"])
    reg = dict(R=np.eye(3), t=g["reg_t"], scale=1.0, dice=1.0)
    return lab, sigma_map, float(g["dx"]), vox, coords, reg, float(g["h_fine"]), g["Vm"]


def random_case(seed=0, shape=(40, 34, 44), dx=1.5):
    rng = np.random.default_rng(seed)
    ni, nj, nk = shape
    ii, jj, kk = np.indices(shape).astype(np.float64)
    ci, cj = (ni - 1) / 2, (nj - 1) / 2
    lab = np.zeros(shape, np.int32)
    body = (((ii - ci) / (0.45 * ni)) ** 2 + ((jj - cj) / (0.45 * nj)) ** 2 <= 1) & (kk >= 1) & (kk <= nk - 2)
    lab[body] = 1
    for s in (-1, 1):
        lung = ((ii - ci - s * 0.22 * ni) / (0.15 * ni)) ** 2 + ((jj - cj) / (0.25 * nj)) ** 2 + \
               ((kk - nk / 2) / (0.3 * nk)) ** 2 <= 1
        lab[lung & body] = 2
    blood = ((ii - ci) / 3) ** 2 + ((jj - cj) / 3) ** 2 + ((kk - nk / 2 + 2) / 3) ** 2 <= 1
    lab[blood & body] = 3
    sigma_map = {1: 0.2, 2: 0.05, 3: 0.7}
    h = 0.5
    gi, gj, gk = np.indices((50, 44, 50))
    cen = np.array([24.5, 21.5, 24.5])
    r = np.sqrt(((gi - cen[0])) ** 2 + ((gj - cen[1])) ** 2 + ((gk - cen[2])) ** 2)
    vox = np.argwhere((r >= 12) & (r <= 19)).astype(np.int32)
    coords = vox[:, [1, 0, 2]].astype(np.float64) * h
    t = np.array([ci * dx - 11.0, cj * dx - 12.5, nk / 2 * dx - 12.5])
    reg = dict(R=np.eye(3), t=t, scale=1.0, dice=1.0)
    frames = []
    x = vox[:, 0].astype(np.float64)
    for f in range(4):
        front = 10.0 + 6.0 * f
        frames.append((-85.0 + 110.0 / (1.0 + np.exp(-(front - x) / 1.5)) +
                       rng.normal(0, 0.3, len(vox))).astype(np.float32))
    return lab, sigma_map, dx, vox, coords, reg, h, np.array(frames)
