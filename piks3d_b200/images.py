"""Seeded synthetic voxel images (uint8, 1 = solid, x fastest as PIKS3D reads them).

These stand in for the porous-media images of the benchmark configurations:
  centred_sphere   — one solid sphere in a periodic box (the 32^3, r = 12 case)
  sphere_pack      — Boolean overlapping spheres, centres uniform, radii uniform, added
                     until the porosity reaches a target (isolated pores kept)
  gaussian_field   — Gaussian-correlated random field thresholded at a porosity, keeping
                     only the pore cluster that percolates along x
All return a C-contiguous (Nz, Ny, Nx) uint8 array; .tobytes() is the raw image stream.
"""
import numpy as np


def centred_sphere(n=32, radius=12.0):
    """Solid sphere centred in an n^3 box, voxel (i,j,k) 1-based solid if its distance to
    ((n+1)/2, (n+1)/2, (n+1)/2) is below `radius`."""
    c = (n + 1) / 2.0
    idx = np.arange(1, n + 1, dtype=np.float64)
    z, y, x = np.meshgrid(idx, idx, idx, indexing="ij")
    solid = (x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2 < radius * radius
    return np.ascontiguousarray(solid.astype(np.uint8))


def quarter_sphere(n=100, porosity=0.75):
    """The tutorial geometry of PIKS3D's conf/createSphere.F90: a solid sphere of radius
    floor((n-1)*((1-porosity)*3/(4*pi))^(1/3)) centred at ((n+1)/2, 1, 1), so that the
    box holds a quarter sphere; voxel (i,j,k) 1-based is solid if its squared distance
    to the centre is below radius^2."""
    import math
    r = math.floor((n - 1) * ((1.0 - porosity) * 3.0 / 4.0 / (math.atan(1.0) * 4.0)) ** (1.0 / 3.0))
    idx = np.arange(1, n + 1, dtype=np.float64)
    z, y, x = np.meshgrid(idx, idx, idx, indexing="ij")
    d2 = (z - 1.0) ** 2 + (y - 1.0) ** 2 + (x - (n + 1) / 2.0) ** 2
    return np.ascontiguousarray((d2 < r * r).astype(np.uint8))


def sphere_pack(n, porosity, rmin=4.0, rmax=8.0, seed=12345):
    """Boolean overlapping spheres in an n^3 box, added until porosity <= `porosity`.
    Centres uniform in the box, radii uniform in [rmin, rmax] (numpy PCG64, `seed`)."""
    rng = np.random.default_rng(seed)
    solid = np.zeros((n, n, n), dtype=bool)
    coords = np.arange(n, dtype=np.float64) + 0.5
    target_solid = (1.0 - porosity) * n ** 3
    nsolid = 0
    while nsolid < target_solid:
        c = rng.uniform(0.0, n, size=3)
        r = rng.uniform(rmin, rmax)
        lo = np.maximum(np.floor(c - r).astype(int), 0)
        hi = np.minimum(np.ceil(c + r).astype(int) + 1, n)
        zz = coords[lo[2]:hi[2], None, None] - c[2]
        yy = coords[None, lo[1]:hi[1], None] - c[1]
        xx = coords[None, None, lo[0]:hi[0]] - c[0]
        ball = (xx * xx + yy * yy + zz * zz) < r * r
        block = solid[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
        nsolid += int(np.count_nonzero(ball & ~block))
        block |= ball
    return np.ascontiguousarray(solid.astype(np.uint8))


def gaussian_field(n, porosity, corr=6.0, seed=2024):
    """Threshold a Gaussian-correlated field (white noise * Gaussian kernel of length
    `corr`, via FFT) so that a fraction `porosity` is pore; keep the pore cluster
    (6-connected) that touches both x = 1 and x = n."""
    from scipy import ndimage

    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((n, n, n))
    k = np.fft.fftfreq(n)
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    filt = np.exp(-2.0 * (np.pi * corr) ** 2 * (kx * kx + ky * ky + kz * kz))
    field = np.real(np.fft.ifftn(np.fft.fftn(noise) * filt))
    thr = np.quantile(field, porosity)
    pore = field < thr
    lab, nlab = ndimage.label(pore)
    left = set(np.unique(lab[:, :, 0])) - {0}
    right = set(np.unique(lab[:, :, -1])) - {0}
    keep = sorted(left & right)
    pore = np.isin(lab, keep) if keep else np.zeros_like(pore)
    return np.ascontiguousarray((~pore).astype(np.uint8))


def porosity(img):
    return float((img == 0).mean())
