"""Seeded particle distributions with the shapes of the workloads beside the uniform headline case.

* ``ellipsoid_surface``: area-uniform points on the surface of an ellipsoid with semi-axes (0.5, 0.3, 0.2)
  centred in the unit cube (very uneven leaf occupancy, most leaves empty).  Points uniform on the unit
  sphere are mapped to the ellipsoid and kept with probability proportional to the surface element
  sqrt((b c u_x)^2 + (a c u_y)^2 + (a b u_z)^2), which makes them uniform in area.  (The reference's
  own generator, FGenerateDistribution.hpp:108-175, is neither area-uniform nor axis-aligned.)
* ``plummer``: Plummer sphere of scale radius 0.1 centred in the unit cube, r = a / sqrt(U^(-2/3) - 1),
  isotropic directions, points outside the unit cube rejected.
Charges come from the caller.
"""
import numpy as np


def ellipsoid_surface(n, seed, axes=(0.5, 0.3, 0.2), center=(0.5, 0.5, 0.5)):
    a, b, c = axes
    rng = np.random.default_rng(seed)
    gmax = max(b * c, a * c, a * b)
    out = []
    have = 0
    while have < n:
        u = rng.standard_normal((3, 2 * n))
        u /= np.linalg.norm(u, axis=0)
        g = np.sqrt((b * c * u[0]) ** 2 + (a * c * u[1]) ** 2 + (a * b * u[2]) ** 2)
        keep = rng.random(2 * n) * gmax < g
        p = np.array([a * u[0], b * u[1], c * u[2]])[:, keep]
        out.append(p)
        have += p.shape[1]
    p = np.concatenate(out, axis=1)[:, :n]
    # the x semi-axis touches the box faces: keep the points strictly inside [0, 1)
    p = np.clip(p + np.array(center)[:, None], 0.0, np.nextafter(1.0, 0.0))
    return p[0].copy(), p[1].copy(), p[2].copy()


def plummer(n, seed, scale=0.1, center=(0.5, 0.5, 0.5)):
    rng = np.random.default_rng(seed)
    out = []
    have = 0
    while have < n:
        m = 2 * n
        r = scale / np.sqrt(rng.random(m) ** (-2.0 / 3.0) - 1.0)
        d = rng.standard_normal((3, m))
        d /= np.linalg.norm(d, axis=0)
        p = d * r + np.array(center)[:, None]
        keep = np.all((p >= 0.0) & (p < 1.0), axis=0)
        out.append(p[:, keep])
        have += int(keep.sum())
    p = np.concatenate(out, axis=1)[:, :n]
    return p[0].copy(), p[1].copy(), p[2].copy()
