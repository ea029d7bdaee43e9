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


def sphere_pack(n, porosity, rmin=4.0, rmax=8.0, seed=12345, batch=64):
    """Boolean overlapping spheres in an n^3 box until porosity <= `porosity`."""
    rng = np.random.default_rng(seed)
    solid = np.zeros((n, n, n), dtype=bool)
    coords = np.arange(n, dtype=np.float64) + 0.5
    target_solid = (1.0 - porosity) * n ** 3
    count = 0
    while solid.sum() < target_solid:
        for _ in range(batch):
            c = rng.uniform(0.0, n, size=3)
            r = rng.uniform(rmin, rmax)
            lo = np.maximum(np.floor(c - r).astype(int), 0)
            hi = np.minimum(np.ceil(c + r).astype(int) + 1, n)
            zz = coords[lo[2]:hi[2], None, None] - c[2]
            yy = coords[None, lo[1]:hi[1], None] - c[1]
            xx = coords[None, None, lo[0]:hi[0]] - c[0]
            solid[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] |= (xx * xx + yy * yy + zz * zz) < r * r
            count += 1
            if solid.sum() >= target_solid:
                break
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
