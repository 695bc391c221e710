"""Seeded synthetic workloads for the XRF self-absorption benchmarks.

No measured data ships with the reference (its examples read external
``/data`` files), so every workload is generated here from a fixed seed with
the shapes, sizes and value ranges of the five benchmark configurations:

* ``ellipsoid_grains``  -- 8-20 random ellipsoids, concentration U(0.2, 1.0)
  over a 0.05 background (64^3, one element);
* ``voronoi_grains``    -- Voronoi grains with per-grain U(0, 1) concentration
  per element and 2-voxel grain-boundary shells at 3x (128^3, three elements);
* ``layered``           -- planar layers with random tilt plus spherical
  inclusions (256^3, four elements).

Cross sections are synthetic constants (xraylib is not used), chosen so the
optical depth mu*pix*N across a volume is of order 0.1-5.
"""
import math

import numpy as np

__all__ = ["ellipsoid_grains", "voronoi_grains", "layered", "xrf_params", "cone_mask_angle",
           "Workload", "make_workload", "make_batch_workloads"]


def cone_mask_angle(diameter_mm=7.0, distance_mm=30.0):
    """Full acceptance angle (degrees) of a round detector of the given
    diameter at the given distance: 2*atan(r/d)."""
    return 2.0 * math.degrees(math.atan(0.5 * diameter_mm / distance_mm))


def _grid(n):
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    return z.astype(np.float32), y.astype(np.float32), x.astype(np.float32)


def ellipsoid_grains(n, rng, n_min=8, n_max=20, lo=0.2, hi=1.0, background=0.05):
    """(n, n, n) float32 volume of random ellipsoidal grains."""
    vol = np.full((n, n, n), background, np.float32)
    z, y, x = _grid(n)
    for _ in range(int(rng.integers(n_min, n_max + 1))):
        c = rng.uniform(0.2 * n, 0.8 * n, 3)
        r = rng.uniform(0.05 * n, 0.18 * n, 3)
        q = ((z - c[0]) / r[0]) ** 2 + ((y - c[1]) / r[1]) ** 2 + ((x - c[2]) / r[2]) ** 2
        vol[q <= 1.0] = rng.uniform(lo, hi)
    return vol


def voronoi_grains(n, rng, n_elem, n_seeds=64, shell=2.0, shell_gain=3.0):
    """(n_elem, n, n, n) float32: per-grain U(0,1) per element, with voxels
    within `shell` voxels of a grain boundary scaled by `shell_gain`."""
    seeds = rng.uniform(0, n, (n_seeds, 3)).astype(np.float32)
    conc = rng.uniform(0.0, 1.0, (n_seeds, n_elem)).astype(np.float32)
    pts = np.stack(_grid(n), -1).reshape(-1, 3)
    best = np.full(pts.shape[0], np.inf, np.float32)
    second = np.full(pts.shape[0], np.inf, np.float32)
    label = np.zeros(pts.shape[0], np.int64)
    for k in range(n_seeds):
        d = np.sqrt(((pts - seeds[k]) ** 2).sum(-1))
        closer = d < best
        second = np.where(closer, best, np.minimum(second, d))
        label = np.where(closer, k, label)
        best = np.where(closer, d, best)
    # distance to the bisector plane of the two nearest seeds ~ (d2 - d1)/2
    boundary = (second - best) * 0.5 < 0.5 * shell
    out = conc[label].T.reshape(n_elem, n, n, n).copy()
    out[:, boundary.reshape(n, n, n)] *= shell_gain
    return out


def layered(n, rng, n_elem, n_layers=5, n_incl=200, r_min=2, r_max=6):
    """(n_elem, n, n, n) float32: tilted planar layers plus spherical inclusions."""
    z, y, x = _grid(n)
    normal = np.array([1.0, 0.0, 0.0]) + rng.normal(0, 0.15, 3)
    normal /= np.linalg.norm(normal)
    depth = (z * normal[0] + y * normal[1] + x * normal[2])
    edges = np.linspace(depth.min(), depth.max() + 1e-3, n_layers + 1)
    layer = np.clip(np.searchsorted(edges, depth, side="right") - 1, 0, n_layers - 1)
    conc = rng.uniform(0.0, 1.0, (n_layers, n_elem)).astype(np.float32)
    out = np.moveaxis(conc[layer], -1, 0).astype(np.float32)
    for _ in range(n_incl):
        c = rng.uniform(0, n, 3)
        r = rng.uniform(r_min, r_max)
        lo = np.maximum(np.floor(c - r).astype(int), 0)
        hi = np.minimum(np.ceil(c + r).astype(int) + 1, n)
        zz, yy, xx = np.meshgrid(*[np.arange(l, h) for l, h in zip(lo, hi)], indexing="ij")
        m = (zz - c[0]) ** 2 + (yy - c[1]) ** 2 + (xx - c[2]) ** 2 <= r * r
        val = rng.uniform(0.0, 1.0, n_elem).astype(np.float32)
        for e in range(n_elem):
            sub = out[e, lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
            sub[m] = val[e]
    return out


# Synthetic cross sections (cm^2/g) and densities (g/cm^3) per element; the
# products cs*rho set the attenuation per unit mass fraction.
_ELEMENTS = {
    "Ca": dict(rho=2.7, cs_in=95.0, cs_line=48.0, em=40.0),
    "Fe": dict(rho=5.2, cs_in=30.0, cs_line=36.0, em=35.0),
    "Ni": dict(rho=6.7, cs_in=28.0, cs_line=41.0, em=38.0),
    "Cu": dict(rho=6.3, cs_in=31.0, cs_line=46.0, em=42.0),
    "Zn": dict(rho=5.6, cs_in=27.0, cs_line=39.0, em=36.0),
}
MATRIX_MU = 5.0   # cm^-1, uniform matrix attenuation


def xrf_params(elements, n_angle, energy_kev, pix_cm, rng=None):
    """A param dict in the reference's layout (FL/core.py:213-341 produces the
    same keys): elements 'E' with compounds 'E_c', plus a matrix compound
    'matrix' with cs*rho = MATRIX_MU at every energy and no emission line."""
    rng = rng or np.random.default_rng(0)
    comps = [f"{e}_c" for e in elements]
    cs = {"elem_type": list(elements), "elem_compound": comps + ["matrix"]}
    rho = {}
    em_cs = {}
    scale_in = (14.0 / energy_kev) ** 2.6
    for e, c in zip(elements, comps):
        p = _ELEMENTS[e]
        rho[c] = p["rho"]
        cs[f"{c}-x"] = np.full(n_angle, p["cs_in"] * scale_in)
        for e2 in elements:
            # absorption of compound c at the line of element e2 (higher above
            # the absorbing element's edge)
            boost = 2.0 if _ELEMENTS[e2]["cs_line"] > p["cs_line"] else 1.0
            cs[f"{c}-{e2}"] = p["cs_line"] * boost * float(rng.uniform(0.9, 1.1))
        em_cs[e] = np.full(n_angle, p["em"])
    rho["matrix"] = 1.0
    cs["matrix-x"] = np.full(n_angle, MATRIX_MU)
    for e2 in elements:
        cs[f"matrix-{e2}"] = MATRIX_MU
    return {"cs": cs, "rho": rho, "pix": pix_cm, "elem_type": list(elements),
            "elem_compound": comps + ["matrix"], "em_cs": em_cs}


class Workload:
    """Truth volumes, parameters, angles and cone mask of one configuration."""

    def __init__(self, name, conc, elements, angles_deg, energy_kev, pix_cm, mask_angle_deg,
                 n_iter, recompute_every, noise_max_counts, seed):
        self.name = name
        # the concentrations are mass fractions: every voxel's total over the
        # elements is scaled to at most 0.9 (grain values and the 3x shells
        # keep their ratios)
        tot = float(conc.sum(axis=0).max())
        if tot > 0.9:
            conc = (conc * np.float32(0.9 / tot)).astype(np.float32)
        self.conc = conc                      # (L, N, N, N) float32 truth
        self.elements = list(elements)
        self.angles = np.asarray(angles_deg, np.float64)
        self.energy = energy_kev
        self.pix = pix_cm
        self.mask_angle = mask_angle_deg
        self.n_iter = n_iter
        self.recompute_every = recompute_every
        self.noise_max_counts = noise_max_counts
        self.seed = seed
        self.param = xrf_params(self.elements, len(self.angles), energy_kev, pix_cm,
                                np.random.default_rng(seed + 1))

    @property
    def N(self):
        return self.conc.shape[-1]

    def frac(self):
        """(L+1, N, N, N) fractions: the element concentrations plus the matrix (1)."""
        L, N = self.conc.shape[0], self.N
        return np.concatenate([self.conc, np.ones((1, N, N, N), np.float32)], 0)


def make_batch_workloads(n_volumes=16, seed=20240611, sizes=(64, 96, 128, 160, 192),
                         n_iter=20, recompute_every=5):
    """The uneven batch of configuration 3: n_volumes seeded Voronoi volumes
    with side lengths drawn from `sizes`, 1-3 elements, 60-180 angles over
    [0, 180), incident energy U(10, 16) keV and detector distance U(20, 40)
    mm (a 7 mm detector, so the cone angle is 2 atan(3.5 / d)).  Every volume
    images the same 128 um sample (pixel 1.28e-2 / N cm), so the optical depth
    across it stays in the range of the 128^3 workload whatever N is."""
    rng = np.random.default_rng(seed + 3)
    names = ["Fe", "Ni", "Cu"]
    out = []
    for i in range(n_volumes):
        n = int(rng.choice(sizes))
        L = int(rng.integers(1, 4))
        A = int(rng.integers(60, 181))
        energy = float(rng.uniform(10.0, 16.0))
        dist = float(rng.uniform(20.0, 40.0))
        conc = voronoi_grains(n, rng, L, n_seeds=32)
        out.append(Workload("cfg3-v%02d-%dc-%delem-%dang" % (i, n, L, A), conc, names[:L],
                            np.linspace(0, 180, A, endpoint=False), energy, 1.28e-2 / n,
                            cone_mask_angle(7.0, dist), n_iter, recompute_every, 0, seed + 17 * i))
    return out


def make_workload(cfg, seed=20240611):
    """Workload for configuration index cfg (0, 1, 2 or 4; see module doc)."""
    rng = np.random.default_rng(seed + cfg)
    ang = cone_mask_angle(7.0, 30.0)
    if cfg == 0:
        conc = ellipsoid_grains(64, rng)[None]
        return Workload("cfg0-64c-1elem-60ang", conc, ["Fe"], np.linspace(0, 180, 60, endpoint=False),
                        12.0, 1e-4, ang, 20, 5, 1e4, seed)
    if cfg == 1:
        conc = voronoi_grains(128, rng, 3)
        return Workload("cfg1-128c-3elem-120ang", conc, ["Fe", "Ni", "Cu"],
                        np.linspace(0, 180, 120, endpoint=False), 14.0, 1e-4, ang, 50, 5, 1e4, seed)
    if cfg == 2:
        conc = voronoi_grains(96, rng, 3)
        return Workload("cfg2-96c-3elem-90ang", conc, ["Fe", "Ni", "Cu"],
                        np.linspace(0, 180, 90, endpoint=False), 14.0, 1e-4, ang, 200, 1, 0, seed)
    if cfg == 4:
        conc = layered(256, rng, 4)
        return Workload("cfg4-256c-4elem-180ang", conc, ["Ca", "Fe", "Ni", "Zn"],
                        np.linspace(0, 180, 180, endpoint=False), 15.0, 1e-4, ang, 0, 1, 0, seed)
    raise ValueError("unknown configuration %r" % cfg)
