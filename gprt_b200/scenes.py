"""Seeded synthetic scenes with the shapes of the benchmark workloads.

There is no public dataset here: every scene is generated from a seed.
  * soup(n):     n triangles, centroids uniform in a unit cube, each vertex =
                 centroid + N(0, sigma^2) per axis (sigma 0.002), indices
                 (3i, 3i+1, 3i+2).
  * mixture(n):  n triangles from a k-cluster Gaussian mixture: cluster
                 centres uniform in [0,1]^3, sigma_c uniform in [0.005, 0.05],
                 triangle edges N(0, 0.001^2).
  * rays(m):     origins uniform on the sphere of radius 2 about the cube
                 centre, directions normalised towards uniform points in the
                 cube; tmin = 0, tmax = +inf.
  * mesh sizes:  log-uniform integer sizes in [lo, hi].
Host-side numpy generation; the arrays are then copied to the device.
"""
import numpy as np


def soup(n, seed=0, sigma=0.002, offset=(0.0, 0.0, 0.0)):
    rng = np.random.default_rng(seed)
    c = rng.random((n, 3), dtype=np.float32) + np.asarray(offset, np.float32)
    pos = (np.repeat(c, 3, axis=0) + rng.normal(0.0, sigma, (3 * n, 3)).astype(np.float32)).astype(np.float32)
    tri = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return pos, tri


def mixture(n, clusters=64, seed=0, edge_sigma=0.001):
    rng = np.random.default_rng(seed)
    centres = rng.random((clusters, 3))
    sig = rng.uniform(0.005, 0.05, size=clusters)
    k = rng.integers(0, clusters, size=n)
    c = (centres[k] + rng.normal(0.0, 1.0, (n, 3)) * sig[k, None]).astype(np.float32)
    pos = (np.repeat(c, 3, axis=0) + rng.normal(0.0, edge_sigma, (3 * n, 3)).astype(np.float32)).astype(np.float32)
    tri = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return pos, tri


def rays(m, seed=1, lo=(0.0, 0.0, 0.0), size=1.0, radius=2.0):
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    centre = lo + 0.5 * size
    u = rng.normal(size=(m, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    org = centre + radius * size * u
    tgt = lo + size * rng.random((m, 3))
    d = tgt - org
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((m, 8), np.float32)
    r[:, 0:3] = org
    r[:, 3] = 0.0
    r[:, 4:7] = d
    r[:, 7] = np.inf
    return r


def mesh_sizes(count, lo=64, hi=65536, seed=2):
    rng = np.random.default_rng(seed)
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))).astype(np.int64)


def batch(sizes, seed=0, sigma=0.002, rays_per_tri=0, spacing=2.0):
    """Meshes of the given triangle counts, mesh m a soup inside its own unit
    cube at a grid offset (m mod 16, m // 16 mod 16, m // 256) * spacing.
    Returns pos [V,3], tri [N,3] (global vertex indices), tri_off [M+1] and,
    when rays_per_tri > 0, rays [R,8] with ray_off [M+1] (rays of mesh m aimed
    at its cube from the radius-2 sphere around it)."""
    sizes = np.asarray(sizes, np.int64)
    off = np.zeros(sizes.size + 1, np.int64)
    off[1:] = np.cumsum(sizes)
    pos = np.empty((3 * int(off[-1]), 3), np.float32)
    rays_l, ray_off = [], np.zeros(sizes.size + 1, np.int64)
    for m, n in enumerate(sizes):
        o = np.array([m % 16, (m // 16) % 16, m // 256], np.float32) * spacing
        p, _ = soup(int(n), seed=seed * 1000003 + m, sigma=sigma, offset=o)
        pos[3 * off[m]:3 * off[m + 1]] = p
        if rays_per_tri:
            r = rays(int(n) * rays_per_tri, seed=seed * 7919 + m + 17, lo=o)
            rays_l.append(r)
            ray_off[m + 1] = ray_off[m] + r.shape[0]
    tri = np.arange(3 * int(off[-1]), dtype=np.uint32).reshape(-1, 3)
    if rays_per_tri:
        return pos, tri, off, np.concatenate(rays_l), ray_off
    return pos, tri, off
