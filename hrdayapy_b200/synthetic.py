"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference works on patient data (NRRD masks, UVC coordinates, rule-based
fibres, Berg-grown Purkinje trees) that is not available here; these
generators stand in for it with the sizes and value distributions the
benchmark configurations state:

* :func:`slab`       -- 64 x 64 x 16 slab at 0.25 mm, all epicardial cells,
                        isotropic 0.13 S/m, corner stimulus (the CPU-runnable
                        case).
* :func:`biv_shell`  -- biventricular shell in a 256^3 grid at 0.4 mm: two
                        truncated prolate ellipsoids (LV wall 10 mm, RV wall
                        4 mm) with a seeded +/-1-voxel boundary jitter, a
                        transmural Laplace coordinate, helical fibres from
                        +60 deg (endo) to -60 deg (epi), endo/M/epi layers at
                        0.3/0.7, and a fractal Purkinje tree grown on the
                        endocardium (LV 1200 + RV 600 terminals, 2 +/- 0.5 mm
                        segments, 30 +/- 10 deg branching).

All functions return the reference-API inputs (nodes, elements,
activation_times, S, Z, phi, fibre_dir, keyword arguments).
"""
from __future__ import annotations

import math

import numpy as np

_LAST = {}


def last_inputs():
    """Inputs of the most recent *_problem() call (for CPU baselines)."""
    return _LAST


def stub_tree(shape):
    nx, ny, nz = shape
    nodes = np.array([[ny + 8.0, nx + 8.0, nz + 8.0], [ny + 8.0, nx + 8.0, nz + 12.0]])
    return nodes, np.array([[0, 1]]), np.array([0.0, 1.0])


def slab(nx=64, ny=64, nz=16):
    S = np.ones((nx, ny, nz), np.uint8)
    phi = np.ones(S.shape, np.float32)
    ect = np.zeros(S.shape, bool)
    ect[:4, :4, :] = True
    nodes, el, act = stub_tree(S.shape)
    kw = dict(voxel_size=0.25, dx_p=0.25, sigma_P=0.0, sigma_M=0.13, Cm=0.01, A_P=133.33,
              A_M=140.0, R_P=0.015, dt=0.02, T=300.0,
              stim_protocol=[dict(name="corner", target="ectopic", amp=0.52, dur=1.0,
                                  onset=0.0)],
              ectopic_region=ect, stim_len_mm=1.0, c_pmj=0.0, n_pmj=1)
    return (nodes, el, act, S, phi), None, kw


# --------------------------------------------------------------------------
# biventricular shell
# --------------------------------------------------------------------------

def _ellipsoid_level(ii, jj, kk, c, a, b, cz):
    return np.sqrt(((ii - c[0]) / a) ** 2 + ((jj - c[1]) / b) ** 2 + ((kk - c[2]) / cz) ** 2)


def biv_geometry(n=256, h=0.4, seed=0, scale=1.05):
    """Mask, cavity masks and bounding info of the biventricular shell."""
    rng = np.random.default_rng(seed)
    ii, jj, kk = np.meshgrid(np.arange(n, dtype=np.float32) * h, np.arange(n, dtype=np.float32) * h,
                             np.arange(n, dtype=np.float32) * h, indexing="ij")
    L = n * h
    s = float(scale)
    c_lv = np.array([0.45 * L, 0.5 * L, 0.62 * L], np.float32)
    jit = rng.uniform(-h, h, ii.shape).astype(np.float32)
    # LV: endocardial cavity semi-axes (a, a, c); wall 10 mm
    a_en, c_en, w_lv = 26.0 * s, 50.0 * s, 10.0 * s
    r_en = _ellipsoid_level(ii, jj, kk, c_lv, a_en, a_en, c_en)
    r_ep = _ellipsoid_level(ii, jj, kk, c_lv, a_en + w_lv, a_en + w_lv, c_en + w_lv)
    # RV: cavity offset along +i, wall 4 mm, wrapping the LV's right side
    c_rv = c_lv + np.array([22.0 * s, 0.0, 4.0 * s], np.float32)
    ra, rb, rc, w_rv = 24.0 * s, 30.0 * s, 44.0 * s, 4.0 * s
    r_rv_en = _ellipsoid_level(ii, jj, kk, c_rv, ra, rb, rc)
    r_rv_ep = _ellipsoid_level(ii, jj, kk, c_rv, ra + w_rv, rb + w_rv, rc + w_rv)
    # jitter the boundaries by about +/- one voxel (level sets scaled to mm)
    lv_cav = (r_en - 1.0) * a_en + jit < 0
    lv_epi = (r_ep - 1.0) * (a_en + w_lv) + jit < 0
    rv_cav = ((r_rv_en - 1.0) * ra + jit < 0) & ~lv_epi
    rv_epi = (r_rv_ep - 1.0) * (ra + w_rv) + jit < 0
    base = kk <= c_lv[2] + 0.3 * c_en           # truncation plane (base)
    lv_wall = lv_epi & ~lv_cav & base
    rv_wall = rv_epi & ~rv_cav & ~lv_epi & base
    S = (lv_wall | rv_wall)
    del ii, jj, kk, r_en, r_ep, r_rv_en, r_rv_ep, jit
    return dict(S=S.astype(np.uint8), lv_cav=lv_cav & base, rv_cav=rv_cav & base,
                base=base, c_lv=c_lv, h=h, n=n)


def transmural_coordinate(geo, iters=200):
    """phi = 0 on the endocardium (faces touching a cavity), 1 on the
    epicardium (faces touching the exterior), Laplace in between (Neumann at
    the base plane); Jacobi-preconditioned CG from a distance-ratio guess."""
    import torch
    from scipy import ndimage as ndi
    S = geo["S"].astype(bool)
    cav = geo["lv_cav"] | geo["rv_cav"]
    ext = ~S & ~cav
    d_endo = ndi.distance_transform_edt(~cav).astype(np.float32)
    d_epi = ndi.distance_transform_edt(~ext).astype(np.float32)
    guess = d_endo / np.maximum(d_endo + d_epi, 1e-6)
    vox = np.argwhere(S)
    N = len(vox)
    shape = S.shape
    idx = -np.ones(shape, np.int64)
    idx[vox[:, 0], vox[:, 1], vox[:, 2]] = np.arange(N)
    nb_list, bc0, bc1 = [], np.zeros(N, np.float32), np.zeros(N, np.float32)
    base_plane_free = geo["base"]
    for d in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
        n_ = vox + np.array(d)
        inb = np.all((n_ >= 0) & (n_ < np.array(shape)), 1)
        nc = np.clip(n_, 0, np.array(shape) - 1)
        j = np.where(inb, idx[nc[:, 0], nc[:, 1], nc[:, 2]], -1)
        is_cav = inb & cav[nc[:, 0], nc[:, 1], nc[:, 2]]
        is_ext = inb & ext[nc[:, 0], nc[:, 1], nc[:, 2]] & base_plane_free[nc[:, 0], nc[:, 1], nc[:, 2]]
        bc0 += is_cav          # Dirichlet 0 faces
        bc1 += is_ext          # Dirichlet 1 faces
        nb_list.append(j)
    nb = np.stack(nb_list, 1)
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    nb_t = torch.as_tensor(nb, device=dev)
    has = nb_t >= 0
    nbc = nb_t.clamp(min=0)
    diag = has.sum(1).to(torch.float32) + torch.as_tensor(bc0 + bc1, device=dev)
    rhs = torch.as_tensor(bc1, device=dev)

    def A(x):
        return diag * x - (x[nbc] * has).sum(1)

    x = torch.as_tensor(guess[vox[:, 0], vox[:, 1], vox[:, 2]], device=dev)
    Minv = 1.0 / diag.clamp(min=1.0)
    r = rhs - A(x)
    z = Minv * r
    p = z.clone()
    rz = torch.dot(r.double(), z.double())
    for _ in range(iters):
        Ap = A(p)
        alpha = rz / torch.dot(p.double(), Ap.double())
        x = x + alpha.float() * p
        r = r - alpha.float() * Ap
        z = Minv * r
        rz_new = torch.dot(r.double(), z.double())
        p = z + (rz_new / rz).float() * p
        rz = rz_new
    phi_full = guess.copy()
    phi_full[vox[:, 0], vox[:, 1], vox[:, 2]] = x.clamp(0, 1).cpu().numpy()
    phi = np.full(shape, np.nan, np.float32)
    phi[vox[:, 0], vox[:, 1], vox[:, 2]] = phi_full[vox[:, 0], vox[:, 1], vox[:, 2]]
    return phi, phi_full


def helical_fibres(geo, phi_full, alpha_endo=60.0, alpha_epi=-60.0):
    """Unit fibre vectors (raw array-axis order): helix angle linear in phi
    from alpha_endo to alpha_epi, in the local frame (circumferential,
    longitudinal) orthogonal to grad(phi); long axis = array axis 2."""
    S = geo["S"].astype(bool)
    vox = np.argwhere(S)
    g = np.stack(np.gradient(phi_full.astype(np.float32)), -1)[vox[:, 0], vox[:, 1], vox[:, 2]]
    et = g / np.maximum(np.linalg.norm(g, axis=1, keepdims=True), 1e-9)
    ez = np.array([0.0, 0.0, 1.0], np.float32)
    ec = np.cross(np.broadcast_to(ez, et.shape), et)
    nrm = np.linalg.norm(ec, axis=1, keepdims=True)
    ec = np.where(nrm > 1e-6, ec / np.maximum(nrm, 1e-9), np.array([1.0, 0.0, 0.0], np.float32))
    el = np.cross(et, ec)
    ph = phi_full[vox[:, 0], vox[:, 1], vox[:, 2]]
    a = np.deg2rad(alpha_endo + (alpha_epi - alpha_endo) * ph)[:, None]
    f = np.cos(a) * ec + np.sin(a) * el
    f /= np.maximum(np.linalg.norm(f, axis=1, keepdims=True), 1e-9)
    fib = np.zeros(S.shape + (3,), np.float32)
    fib[vox[:, 0], vox[:, 1], vox[:, 2]] = f
    return fib


def _rotate(v, axis, ang):
    """Rodrigues rotation of vector v about unit axis by ang (radians)."""
    return (v * math.cos(ang) + np.cross(axis, v) * math.sin(ang) +
            axis * np.dot(axis, v) * (1 - math.cos(ang)))


def fractal_tree(surface_pts, normals, root, direction, n_terminals, rng, seg_mean=2.0,
                 seg_sd=0.5, ang_mean=30.0, ang_sd=10.0, min_dist=0.8, p_branch=0.35):
    """Grows a branching tree on a surface point cloud (mm).  Each tip
    advances by one segment (length seg_mean +/- seg_sd) projected onto the
    surface; a segment end bifurcates with probability p_branch (children at
    +/- angle about the local surface normal) and otherwise continues with a
    small random turn; a tip stops when it would come closer than min_dist
    to the existing tree or leaves the surface; growth stops once n_terminals
    tips exist.
    Returns node positions (mm) and parent-child edges (root = node 0)."""
    from scipy.spatial import cKDTree
    surf = cKDTree(surface_pts)
    nodes = [np.asarray(root, np.float64)]
    edges = []
    tips = [(0, np.asarray(direction, np.float64))]
    terminals = []
    tree = None
    tree_n = 0
    while tips:
        if len(tips) + len(terminals) >= n_terminals:
            terminals += [t[0] for t in tips]
            break
        new_tips = []
        if tree_n != len(nodes):
            tree = cKDTree(np.array(nodes))
            tree_n = len(nodes)
        for (ni, d) in tips:
            p = nodes[ni]
            seg = max(1.0, rng.normal(seg_mean, seg_sd))
            q = p + seg * d
            dist, k = surf.query(q)
            if dist > 2.0 * seg:
                terminals.append(ni)
                continue
            q = surface_pts[k].astype(np.float64)
            near = tree.query_ball_point(q, min_dist)
            if any(j != ni for j in near) or np.linalg.norm(q - p) < 0.5:
                terminals.append(ni)
                continue
            nodes.append(q)
            qi = len(nodes) - 1
            edges.append((ni, qi))
            nrm = normals[k]
            dn = q - p
            dn -= nrm * np.dot(nrm, dn)
            dn /= max(np.linalg.norm(dn), 1e-9)
            if ni == 0 or rng.uniform() < p_branch:
                for sgn in (1.0, -1.0):
                    ang = math.radians(max(5.0, rng.normal(ang_mean, ang_sd)))
                    new_tips.append((qi, _rotate(dn, nrm, sgn * ang)))
            else:
                new_tips.append((qi, _rotate(dn, nrm, math.radians(rng.normal(0.0, 8.0)))))
        tips = new_tips
        if len(terminals) + len(tips) >= n_terminals:
            # keep only as many tips as needed to reach the terminal count
            tips = tips[: max(0, n_terminals - len(terminals))]
    return np.array(nodes), np.array(edges, np.int64).reshape(-1, 2), terminals


def biv_shell(n=256, h=0.4, seed=0, scale=1.05, lv_terminals=1200, rv_terminals=600,
              phi_iters=200):
    geo = biv_geometry(n, h, seed, scale)
    phi, phi_full = transmural_coordinate(geo, iters=phi_iters)
    fib = helical_fibres(geo, phi_full)
    S = geo["S"]
    rng = np.random.default_rng(seed + 1)
    vox = np.argwhere(S == 1)
    from scipy import ndimage as ndi
    trees = []
    for cav, nterm, side in ((geo["lv_cav"], lv_terminals, -1.0), (geo["rv_cav"], rv_terminals, 1.0)):
        touch = ndi.binary_dilation(cav) & (S == 1)
        pts_v = np.argwhere(touch)
        pts = pts_v.astype(np.float64) * h
        # surface normals: gradient of the distance to the cavity
        dcav = ndi.distance_transform_edt(~cav).astype(np.float32)
        grad = np.stack(np.gradient(dcav), -1)
        nr = grad[pts_v[:, 0], pts_v[:, 1], pts_v[:, 2]].astype(np.float64)
        del dcav, grad
        nr /= np.maximum(np.linalg.norm(nr, axis=1, keepdims=True), 1e-9)
        # root: septal base of this cavity (closest to the other ventricle, high k)
        # septum: +i side of the LV cavity, -i side of the RV cavity
        score = pts[:, 2] - side * 0.5 * pts[:, 0]
        top = np.argsort(-score)[:1]
        r0 = pts[top[0]]
        d0 = np.array([0.0, 0.0, -1.0])       # grow towards the apex
        d0 -= nr[top[0]] * np.dot(nr[top[0]], d0)
        d0 /= max(np.linalg.norm(d0), 1e-9)
        nodes_mm, edges, _ = fractal_tree(pts, nr, r0, d0, nterm, rng)
        trees.append((nodes_mm, edges))
    # join: common root (AV node) above both sub-roots
    (n_lv, e_lv), (n_rv, e_rv) = trees
    av = 0.5 * (n_lv[0] + n_rv[0]) + np.array([0.0, 0.0, 2.0])
    nodes_mm = np.concatenate([av[None], n_lv, n_rv])
    off_lv, off_rv = 1, 1 + len(n_lv)
    edges = np.concatenate([[[0, off_lv], [0, off_rv]], e_lv + off_lv, e_rv + off_rv])
    # activation times: path length from the root at 2 mm/ms
    act = np.full(len(nodes_mm), np.inf)
    act[0] = 0.0
    for a, b in edges:             # edges are listed parent-first
        act[b] = act[a] + np.linalg.norm(nodes_mm[b] - nodes_mm[a]) / 2.0
    nodes_vox = nodes_mm[:, [1, 0, 2]] / h     # (x, y, z) = (col, row, depth)
    # S/m equals the reference's mS/mm: 0.34 / 0.06 S/m along / across the fibre
    kw = dict(voxel_size=h, dx_p=0.2, sigma_P=0.45, sigma_l=0.34, sigma_t=0.06, Cm=0.01,
              A_M=140.0, R_P=0.015, dt=0.02, T=400.0, stim_protocol=None, stim_len_mm=2.0,
              c_pmj=0.01, n_pmj=1, phi_endo_max=0.3, phi_epi_min=0.7)
    return (nodes_vox, edges, act, S, phi), fib, kw


def slab_problem():
    from . import monodomain as M
    args, _, kw = slab()
    nodes, el, act, S, phi = args
    _LAST.clear()
    _LAST.update(args=(nodes, el, act, S, phi), kw=dict(kw), anisotropic=False)
    prob, info = M.prepare(nodes, el, act, S, S, phi, vm_save_dt=None, save_every=None, **kw)
    prob.frame_steps = 50
    return prob, info


def junction_bands(nodes_vox, el, act, S, h, n_bands=7, amp=1.0, dur=2.0):
    """Stimulus sites on the myocardial voxels nearest to the tree's terminal
    nodes, grouped into n_bands onset bands by the terminals' activation
    time.  A 100 kOhm junction cannot depolarise a 0.4 mm voxel by itself
    (source-sink mismatch: the voxel's 18 neighbours load it ~30x more than
    the junction conductance), so the benchmark workload delivers the
    tree's activation sequence to the junction voxels as stimulus sites
    ("custom" targets of the reference's protocol)."""
    from scipy.spatial import cKDTree
    deg = np.bincount(np.asarray(el).ravel(), minlength=len(nodes_vox))
    term = np.where(deg == 1)[0]
    term = term[term != 0]
    vox = np.argwhere(np.asarray(S) == 1)
    xyz = vox[:, [1, 0, 2]].astype(np.float64) * h
    _, nn = cKDTree(xyz).query(np.asarray(nodes_vox)[term] * h)
    t = np.asarray(act)[term]
    edges = np.quantile(t, np.linspace(0, 1, n_bands + 1))
    sites = []
    for b in range(n_bands):
        sel = (t >= edges[b]) & ((t < edges[b + 1]) if b < n_bands - 1 else (t <= edges[b + 1]))
        if not sel.any():
            continue
        sites.append(dict(name=f"junction_band_{b}", target="custom", amp=amp, dur=dur,
                          onset=float(np.round(t[sel].min(), 2)), node_ids=nn[sel]))
    return sites


def biv_shell_problem(seed=0, scale=1.05, n=256, **kw_over):
    from . import monodomain as M
    args, fib, kw = biv_shell(n=n, seed=seed, scale=scale)
    kw.update(kw_over)
    nodes, el, act, S, phi = args
    if kw.get("stim_protocol") is None:
        # Purkinje root pulse (reference default) + junction-voxel bands;
        # custom node ids are global ids: Purkinje comp nodes come first
        comp, _, _ = M.discretise_tree(np.asarray(nodes, np.float32) * np.float32(kw["voxel_size"]),
                                       el, kw["dx_p"])
        bands = junction_bands(nodes, el, act, S, kw["voxel_size"])
        for b in bands:
            b["node_ids"] = np.asarray(b["node_ids"]) + len(comp)
        kw["stim_protocol"] = [dict(name="av_node", target="root", amp=12.0, dur=2.0,
                                    onset=0.0)] + bands
    kwp = dict(kw, A_P=2.0 / kw["R_P"])
    _LAST.clear()
    _LAST.update(args=(nodes, el, act, S, phi), kw=dict(kw, fibre_dir=fib, anisotropic=True),
                 anisotropic=True)
    prob, info = M.prepare(nodes, el, act, S, S, phi, fibre_dir=fib, anisotropic=True,
                           vm_save_dt=None, save_every=None, **kwp)
    prob.frame_steps = 50
    return prob, info


def ensemble_params(v, seed=0):
    """(scale s ~ U[0.7, 1.1], sigma_l ~ U[0.2, 0.4] S/m, g_Ks and g_Kr
    multipliers ~ U[0.5, 1.5]) of variant v of the seeded ensemble."""
    rng = np.random.default_rng([seed, v])
    s = rng.uniform(0.7, 1.1)
    sigma_l = rng.uniform(0.2, 0.4)
    gks, gkr = rng.uniform(0.5, 1.5, 2)
    return float(s), float(sigma_l), float(gks), float(gkr)


def ensemble_variant(v, seed=0):
    """Variant v of the seeded 16-heart ensemble: the biventricular shell
    scaled by s, longitudinal conductivity sigma_l, g_Ks / g_Kr multipliers
    (ensemble_params), its own tree / jitter seed.  Returns (prepared
    problem, g_Ks multiplier, g_Kr multiplier)."""
    s, sigma_l, gks, gkr = ensemble_params(v, seed)
    # the grid grows with the heart (h stays 0.4 mm) so no variant is clipped
    n = int(np.ceil(256 * max(1.0, s) / 8) * 8)
    prob, _ = biv_shell_problem(seed=1000 + v, scale=1.05 * s, n=n, sigma_l=sigma_l)
    return prob, float(gks), float(gkr)


# --------------------------------------------------------------------------
# torso (ECG forward problem)
# --------------------------------------------------------------------------

TORSO_SIGMA = {1: 0.2, 2: 0.05, 3: 0.7, 4: 0.2}   # bulk, lung, blood, heart (S/m)


def torso_for_heart(geo, shape=(192, 160, 256), dx=1.5, heart_center_mm=None):
    """Elliptic-cylinder torso with two ellipsoidal lungs and the heart of
    `geo` (a biv_geometry dict) embedded by nearest sampling at the torso
    voxel centres: myocardium -> label 4, LV/RV cavities -> blood (label 3).

    Heart node coordinates follow the solver convention (x, y, z) = (col,
    row, depth) * h; the registration {R = I, scale = 1, t} maps them to
    torso millimetres with the torso's own (axis0, axis1, axis2) order.
    Returns (labels int32, sigma_map, registration dict)."""
    ni, nj, nk = shape
    L0, L1, L2 = ni * dx, nj * dx, nk * dx
    c = ((np.arange(ni) + 0.5) * dx, (np.arange(nj) + 0.5) * dx, (np.arange(nk) + 0.5) * dx)
    A, B, Cz = np.meshgrid(*c, indexing="ij")
    lab = np.zeros(shape, np.int32)
    body = ((A - L0 / 2) / (0.49 * L0)) ** 2 + ((B - L1 / 2) / (0.49 * L1)) ** 2 <= 1.0
    body &= (Cz > 2 * dx) & (Cz < L2 - 2 * dx)
    lab[body] = 1
    for s in (-1.0, 1.0):
        lung = (((A - L0 / 2 - s * 0.27 * L0) / (0.17 * L0)) ** 2 +
                ((B - L1 / 2 - 0.03 * L1) / (0.3 * L1)) ** 2 +
                ((Cz - 0.6 * L2) / (0.28 * L2)) ** 2) <= 1.0
        lab[lung & body] = 2
    h = geo["h"]
    n = geo["n"]
    if heart_center_mm is None:
        heart_center_mm = np.array([L0 / 2 + 0.06 * L0, L1 / 2 - 0.12 * L1, 0.6 * L2])
    t = np.asarray(heart_center_mm, np.float64) - 0.5 * n * h
    # torso voxel centre -> heart (x, y, z) -> heart array (row=y, col=x, depth=z)
    x = A - t[0]; y = B - t[1]; z = Cz - t[2]
    hi = np.floor(y / h).astype(np.int64)
    hj = np.floor(x / h).astype(np.int64)
    hk = np.floor(z / h).astype(np.int64)
    inside = (hi >= 0) & (hi < n) & (hj >= 0) & (hj < n) & (hk >= 0) & (hk < n) & body
    ii, jj, kk = hi[inside], hj[inside], hk[inside]
    myo = geo["S"][ii, jj, kk] == 1
    cav = geo["lv_cav"][ii, jj, kk] | geo["rv_cav"][ii, jj, kk]
    sub = lab[inside]
    sub[cav] = 3
    sub[myo] = 4
    lab[inside] = sub
    reg = dict(R=np.eye(3), t=t, scale=1.0, dice=1.0)
    return lab, dict(TORSO_SIGMA), reg


def twelve_lead_electrodes(grid, reg, heart_n=256, heart_h=0.4):
    """Approximate standard electrode sites on the torso surface (mm):
    limb electrodes at the shoulders / lower flanks, V1-V6 on a chest arc at
    heart level.  Order: RA, LA, RL, LL, V1..V6."""
    surf = np.asarray(grid["surface_xyz"], np.float64)
    lo, hi = surf.min(0), surf.max(0)
    mid = 0.5 * (lo + hi)
    zc = float(reg["t"][2] + 0.5 * heart_n * heart_h)
    ext = hi - lo
    front = lo[1]                         # anterior = low axis-1
    pts = [(mid[0] - 0.4 * ext[0], mid[1], hi[2] - 0.12 * ext[2]),    # RA
           (mid[0] + 0.4 * ext[0], mid[1], hi[2] - 0.12 * ext[2]),    # LA
           (mid[0] - 0.4 * ext[0], mid[1], lo[2] + 0.12 * ext[2]),    # RL
           (mid[0] + 0.4 * ext[0], mid[1], lo[2] + 0.12 * ext[2])]    # LL
    for k, frac in enumerate((-0.08, 0.02, 0.1, 0.18, 0.28, 0.38)):  # V1..V6
        pts.append((mid[0] + frac * ext[0], front + (0.05 + 0.12 * max(frac, 0)) * ext[1], zc))
    return np.array(pts)


def body_surface_grid(grid, reg, n=16, heart_n=256, heart_h=0.4):
    """n x n electrode grid on the anterior torso surface around heart level."""
    surf = np.asarray(grid["surface_xyz"], np.float64)
    lo, hi = surf.min(0), surf.max(0)
    zc = float(reg["t"][2] + 0.5 * heart_n * heart_h)
    a = np.linspace(lo[0] + 0.15 * (hi[0] - lo[0]), hi[0] - 0.15 * (hi[0] - lo[0]), n)
    z = np.linspace(zc - 0.2 * (hi[2] - lo[2]), zc + 0.2 * (hi[2] - lo[2]), n)
    A, Z = np.meshgrid(a, z, indexing="ij")
    return np.stack([A.ravel(), np.full(A.size, lo[1]), Z.ravel()], 1)
