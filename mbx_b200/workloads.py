"""Seeded synthetic inputs for the 2-body/3-body path.

No public benchmark or dataset exists for this path; the workloads are built
from their stated recipes with numpy ``default_rng(seed)``:

* ``water_box(n_side, n_mol, L)``: rigid waters (O-H 0.9572 A, HOH 104.52 deg)
  with uniformly random orientations (uniform quaternions), oxygens on an
  ``n_side^3`` lattice of spacing L/n_side (``n_mol`` sites drawn without
  replacement), each oxygen jittered by U(-0.3, 0.3) A per component; cubic
  periodic box of edge L.  256 waters: n_side 7, L 19.72 A; 2048 waters:
  n_side 14, L 39.44 A (1.0 g/cm^3).
* ``beads(base, n, sigma)``: path-integral beads, every atom displaced by
  independent N(0, sigma^2) noise.
* ``water_cluster(n)``: gas-phase cluster of n random rigid waters at liquid
  density (0.0334 molecules/A^3) inside a sphere, O-O >= 2.5 A by rejection.
* ``gas_trimers / gas_dimers``: isolated n-mers with O-O distances uniform in
  a range and random orientations.
* ``methane_water_box``: 57 CH4 (C-H 1.09 A, tetrahedral) + 513 H2O, random
  centres with heavy-atom separation >= 2.6 A, box 24.6 x 24.6 x 31.0 A.

Coordinates are returned in the reference's input layout: a list of monomer
ids and the real atoms in input order (3 floats per atom).
"""
import numpy as np

R_OH = 0.9572
THETA_HOH = np.deg2rad(104.52)
R_CH = 1.09


def random_rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def water_body():
    h = THETA_HOH / 2
    return np.array([[0.0, 0.0, 0.0],
                     [R_OH * np.sin(h), 0.0, R_OH * np.cos(h)],
                     [-R_OH * np.sin(h), 0.0, R_OH * np.cos(h)]])


def methane_body():
    t = R_CH / np.sqrt(3.0)
    return np.array([[0, 0, 0], [t, t, t], [t, -t, -t], [-t, t, -t], [-t, -t, t]], float)


def ammonia_body(r_nh=1.012, theta=106.7):
    """N first, three H on a cone (H-N-H angle theta degrees)."""
    t = np.radians(theta)
    # half-angle of the cone from the H-N-H angle: cos t = 1 - 1.5 sin^2 a
    a = np.arcsin(np.sqrt((1.0 - np.cos(t)) / 1.5))
    phis = np.radians([0.0, 120.0, 240.0])
    h = [[r_nh * np.sin(a) * np.cos(f), r_nh * np.sin(a) * np.sin(f), r_nh * np.cos(a)] for f in phis]
    return np.array([[0.0, 0.0, 0.0]] + h)


def co2_body(r_co=1.16):
    return np.array([[0.0, 0.0, 0.0], [0.0, 0.0, r_co], [0.0, 0.0, -r_co]])


def h2_body(r_hh=0.741):
    return np.array([[0.0, 0.0, 0.0], [0.0, 0.0, r_hh]])


def n2o5_body(r_on=1.50, r_no=1.19, a_non=112.0, a_ono=134.0):
    """O2N-O-NO2: the bridging O first, the two N (N-O-N angle a_non), then
    each N's two terminal O (O-N-O angle a_ono) above and below the N-O-N
    plane, the bridging O - N bond bisecting them."""
    h = np.radians(a_non) / 2.0
    t = np.radians(a_ono) / 2.0
    atoms = [[0.0, 0.0, 0.0]]
    ns = []
    for sgn in (1.0, -1.0):
        u = np.array([sgn * np.sin(h), -np.cos(h), 0.0])
        ns.append((r_on * u, u))
        atoms.append(r_on * u)
    for n, u in ns:
        for z in (1.0, -1.0):
            atoms.append(n + r_no * (np.cos(t) * u + z * np.sin(t) * np.array([0.0, 0.0, 1.0])))
    return np.array(atoms)


BODIES = {"h2o": water_body, "mbpbe": water_body, "ch4": methane_body, "nh3": ammonia_body,
          "nh3pbe0d3bj": ammonia_body, "co2": co2_body, "co2_archive": co2_body, "h2": h2_body, "n2o5": n2o5_body}
BODIES.update({m: co2_body for m in ("co2cm5100", "co2cm595", "co2cm590", "co2cm585", "co2cm5875", "co2cm580")})


def molecule_box(ids, n_side=7, L=19.72, seed=0, jitter=0.3):
    """Molecules (ids in input order; one-atom ions and argon too) on the
    sites of an n_side^3 lattice in a cubic box of edge L, picked and
    jittered like water_box, each rigid body randomly rotated."""
    rng = np.random.default_rng(seed)
    s = L / n_side
    g = (np.arange(n_side) + 0.5) * s - L / 2
    lattice = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pick = rng.choice(len(lattice), size=len(ids), replace=False)
    centres = lattice[pick] + rng.uniform(-jitter, jitter, size=(len(ids), 3))
    parts = []
    for m, c in zip(ids, centres):
        body = BODIES[m]() if m in BODIES else np.zeros((1, 3))
        parts.append(place(rng, body, c[None, :])[0].reshape(-1))
    box = np.array([L, 0, 0, 0, L, 0, 0, 0, L], float)
    return list(ids), np.concatenate(parts), box


def dilute_box(solute, n_solute, n_water=220, dmin=6.5, n_side=7, L=19.72, seed=0):
    """molecule_box of n_solute one-atom solutes in water whose solute-solute
    distances (minimum image) are all at least dmin: the first seed from
    `seed` on that gives such a box."""
    for s in range(seed, seed + 1000):
        ids, xyz, box = molecule_box([solute] * n_solute + ["h2o"] * n_water, n_side, L, s)
        p = xyz[:3 * n_solute].reshape(-1, 3)
        d = p[:, None, :] - p[None, :, :]
        d -= L * np.round(d / L)
        r = np.linalg.norm(d, axis=2) + np.eye(n_solute) * 1e9
        if r.min() >= dmin:
            return ids, xyz, box
    raise ValueError("no dilute box found")


def place(rng, body, centres):
    rot = random_rotations(rng, len(centres))
    return centres[:, None, :] + np.einsum("nij,aj->nai", rot, body)


def water_box(n_side=14, n_mol=2048, L=39.44, seed=0, jitter=0.3):
    rng = np.random.default_rng(seed)
    s = L / n_side
    g = (np.arange(n_side) + 0.5) * s - L / 2
    lattice = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pick = rng.choice(len(lattice), size=n_mol, replace=False)
    centres = lattice[pick] + rng.uniform(-jitter, jitter, size=(n_mol, 3))
    xyz = place(rng, water_body(), centres)
    box = np.array([L, 0, 0, 0, L, 0, 0, 0, L], float)
    return ["h2o"] * n_mol, xyz.reshape(-1), box


def ion_water_box(ions, n_side=7, n_mol=256, L=19.72, seed=0, jitter=0.3):
    """Water box of the water_box recipe in which the first len(ions) of the
    picked lattice sites hold the given monomer ids (one-atom ions at the
    site centre) instead of waters.  Input order: the ions, then the waters."""
    rng = np.random.default_rng(seed)
    s = L / n_side
    g = (np.arange(n_side) + 0.5) * s - L / 2
    lattice = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pick = rng.choice(len(lattice), size=n_mol, replace=False)
    centres = lattice[pick] + rng.uniform(-jitter, jitter, size=(n_mol, 3))
    ni = len(ions)
    xyz = place(rng, water_body(), centres[ni:])
    out = np.concatenate([centres[:ni].reshape(-1), xyz.reshape(-1)])
    box = np.array([L, 0, 0, 0, L, 0, 0, 0, L], float)
    return list(ions) + ["h2o"] * (n_mol - ni), out, box


def water_256(seed=0):
    return water_box(7, 256, 19.72, seed)


def water_2048(seed=0):
    return water_box(14, 2048, 39.44, seed)


def beads(xyz, n, sigma=0.05, seed=0):
    rng = np.random.default_rng(seed)
    xyz = np.asarray(xyz, float).reshape(-1)
    return [xyz + rng.normal(0.0, sigma, size=xyz.shape) for _ in range(n)]


def water_256_bead(seed=0, sigma=0.05):
    """One path-integral bead of the 256-water box: every atom displaced by
    independent Gaussian noise (sigma in A), so that the waters are no longer
    rigid (the 1-body term sees stretched and bent molecules)."""
    ids, xyz, box = water_256(seed)
    return ids, beads(xyz, 1, sigma=sigma, seed=seed + 1)[0], box


def water_cluster(n, seed=0, density=0.0334, dmin=2.5):
    rng = np.random.default_rng(seed)
    radius = (3.0 * n / (4.0 * np.pi * density)) ** (1.0 / 3.0)
    centres = []
    tries = 0
    while len(centres) < n:
        tries += 1
        if tries > 2000 * n:
            radius *= 1.02
            tries = 0
        p = rng.uniform(-radius, radius, size=3)
        if np.dot(p, p) > radius * radius:
            continue
        if centres and np.min(np.linalg.norm(np.array(centres) - p, axis=1)) < dmin:
            continue
        centres.append(p)
    xyz = place(rng, water_body(), np.array(centres))
    return ["h2o"] * n, xyz.reshape(-1)


def _random_directions(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def gas_dimers(n=20000, rmin=2.2, rmax=9.0, seed=0):
    """[n, 18] AoS (O H H, O H H), O-O distance uniform in [rmin, rmax]."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(rmin, rmax, size=n)
    c2 = _random_directions(rng, n) * r[:, None]
    a = place(rng, water_body(), np.zeros((n, 3)))
    b = place(rng, water_body(), c2)
    return np.concatenate([a.reshape(n, 9), b.reshape(n, 9)], 1)


def gas_trimers(n=20000, rmin=2.4, rmax=6.5, seed=0):
    """[n, 27] AoS, the two O-O distances from molecule a uniform in [rmin, rmax]."""
    rng = np.random.default_rng(seed)
    rb = rng.uniform(rmin, rmax, size=n)
    rc = rng.uniform(rmin, rmax, size=n)
    cb = _random_directions(rng, n) * rb[:, None]
    cc = _random_directions(rng, n) * rc[:, None]
    a = place(rng, water_body(), np.zeros((n, 3)))
    b = place(rng, water_body(), cb)
    c = place(rng, water_body(), cc)
    return np.concatenate([a.reshape(n, 9), b.reshape(n, 9), c.reshape(n, 9)], 1)


def methane_water_box(n_ch4=57, n_h2o=513, box=(24.6, 24.6, 31.0), seed=0, dmin=2.6):
    rng = np.random.default_rng(seed)
    L = np.array(box, float)
    n = n_ch4 + n_h2o
    centres = np.zeros((0, 3))
    while len(centres) < n:
        p = (rng.uniform(size=3) - 0.5) * L
        if len(centres):
            d = centres - p
            d -= L * np.round(d / L)
            if np.min(np.einsum("ij,ij->i", d, d)) < dmin * dmin:
                continue
        centres = np.vstack([centres, p])
    ch4 = place(rng, methane_body(), centres[:n_ch4])
    h2o = place(rng, water_body(), centres[n_ch4:])
    ids = ["ch4"] * n_ch4 + ["h2o"] * n_h2o
    xyz = np.concatenate([ch4.reshape(-1), h2o.reshape(-1)])
    return ids, xyz, np.array([L[0], 0, 0, 0, L[1], 0, 0, 0, L[2]], float)


def batch_beads_clusters(n_beads=32, n_clusters=64, sigma=0.05, nmin=8, nmax=512, seed=0):
    """The batched workload: n_beads path-integral beads of the 2048-water box
    (every atom displaced by independent Gaussian noise of width sigma A per
    bead) plus n_clusters gas-phase water clusters of sizes drawn uniformly
    from nmin..nmax molecules at liquid density in a sphere.  Returns
    [(ids, input-order xyz, box or None)]."""
    ids, xyz, box = water_2048(seed)
    out = [(ids, b, box) for b in beads(xyz, n_beads, sigma, seed + 1)]
    rng = np.random.default_rng(seed + 2)
    sizes = rng.integers(nmin, nmax + 1, size=n_clusters)
    for k, n in enumerate(sizes):
        cid, cxyz = water_cluster(int(n), seed=seed + 1000 + k)
        out.append((cid, cxyz, None))
    return out
