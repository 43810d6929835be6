"""Seeded synthetic phantoms (stand-ins for measured data; no dataset is used).

Images are float32 [z][y][x] on the ImageGeometry grid (mm coordinates of voxel centres:
z = min_z + index * vz + origin, y,x centred on 0).
"""
from __future__ import annotations

import numpy as np

from .geometry import ImageGeometry


def _grid(img: ImageGeometry):
    vz, vy, vx = img.voxel_size
    z = (np.arange(img.nz) + img.min_z) * vz + img.origin[0]
    y = (np.arange(img.ny) + img.min_y) * vy + img.origin[1]
    x = (np.arange(img.nx) + img.min_x) * vx + img.origin[2]
    zc = z - z.mean()
    return np.meshgrid(zc, y, x, indexing="ij")


def cylinder_with_spheres(img: ImageGeometry, radius_mm=100.0, n_spheres=2, sphere_radius=(10.0, 10.0),
                          contrast=4.0, seed=1, ellipse_axes=None) -> np.ndarray:
    """Water cylinder (or elliptical body with `ellipse_axes`=(a_x, a_y) semi-axes in mm) of activity 1
    with `n_spheres` hot spheres of activity `contrast` at seeded positions inside it."""
    Z, Y, X = _grid(img)
    if ellipse_axes is None:
        body = (X ** 2 + Y ** 2) <= radius_mm ** 2
        ax, ay = radius_mm, radius_mm
    else:
        ax, ay = ellipse_axes
        body = (X / ax) ** 2 + (Y / ay) ** 2 <= 1.0
    out = body.astype(np.float32)
    rng = np.random.default_rng(seed)
    zext = (img.nz * img.voxel_size[0]) / 2
    for _ in range(n_spheres):
        r = rng.uniform(*sphere_radius)
        cx = rng.uniform(-0.5, 0.5) * ax
        cy = rng.uniform(-0.5, 0.5) * ay
        cz = rng.uniform(-0.5, 0.5) * max(zext - r, 0.0)
        s = (X - cx) ** 2 + (Y - cy) ** 2 + (Z - cz) ** 2 <= r ** 2
        out[s] = contrast
    return out


def attenuation_cylinder(img: ImageGeometry, radius_mm=100.0, mu_per_mm=0.0096, ellipse_axes=None) -> np.ndarray:
    Z, Y, X = _grid(img)
    if ellipse_axes is None:
        body = (X ** 2 + Y ** 2) <= radius_mm ** 2
    else:
        ax, ay = ellipse_axes
        body = (X / ax) ** 2 + (Y / ay) ** 2 <= 1.0
    return (body * mu_per_mm).astype(np.float32)


def smooth_random_field(img: ImageGeometry, sigma_vox=3.0, seed=10) -> np.ndarray:
    """Gaussian noise blurred with sigma `sigma_vox` voxels, clipped >= 0."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(img.shape).astype(np.float32)
    for axis in range(3):
        r = int(3 * sigma_vox)
        k = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma_vox) ** 2)
        k /= k.sum()
        a = np.apply_along_axis(lambda v: np.convolve(v, k, mode="same"), axis, a)
    a = a / a.std()
    return np.clip(a + 1.0, 0.0, None).astype(np.float32)


def dynamic_regions(img: ImageGeometry, ellipse_axes=(150.0, 100.0), seed=3):
    """Three tissue regions of a kinetic phantom as float32 masks [3][z][y][x]: 0 = blood pool (a sphere of
    radius 20 mm), 1 = background tissue (the elliptical body minus the other regions), 2 = three lesions
    (spheres of radius 8-15 mm) at seeded positions."""
    Z, Y, X = _grid(img)
    ax, ay = ellipse_axes
    body = (X / ax) ** 2 + (Y / ay) ** 2 <= 1.0
    rng = np.random.default_rng(seed)
    blood = (X + 0.4 * ax) ** 2 + Y ** 2 + Z ** 2 <= 20.0 ** 2
    lesion = np.zeros_like(body)
    zext = (img.nz * img.voxel_size[0]) / 2
    for _ in range(3):
        r = rng.uniform(8.0, 15.0)
        cx, cy = rng.uniform(0.0, 0.5) * ax, rng.uniform(-0.5, 0.5) * ay
        cz = rng.uniform(-0.5, 0.5) * max(zext - r, 0.0)
        lesion |= (X - cx) ** 2 + (Y - cy) ** 2 + (Z - cz) ** 2 <= r ** 2
    lesion &= ~blood
    tissue = body & ~blood & ~lesion
    return np.stack([blood, tissue, lesion]).astype(np.float32)


def time_activity(t_min):
    """Activity of the three regions at time t (minutes): a blood input function (gamma-variate peak
    falling to a slow exponential tail), a tissue curve rising to a plateau and a lesion curve that
    keeps accumulating.  Arbitrary units."""
    t = np.asarray(t_min, np.float64)
    blood = 40.0 * t * np.exp(-t / 0.6) + 2.0 * np.exp(-t / 40.0) * (1.0 - np.exp(-t / 0.3))
    tissue = 1.0 - np.exp(-t / 2.0)
    lesion = 0.06 * t + 2.0 * (1.0 - np.exp(-t / 4.0))
    return np.stack([blood, tissue, lesion], axis=-1)
