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
  * solid_grid(g): a volume mesh of g^3 jittered grid cubes, each cube
                 filled with one seeded choice of linear cells: a hexahedron,
                 two wedges, six pyramids on the cube's centre, six
                 tetrahedra around its main diagonal, or a tetrahedral pair;
                 per-vertex densities N(0, 1).
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


# ---------------------------------------------------------------------------
# Host restatement of the device generators (gprt_b200/csrc/gen.cu): the same
# counter-based SplitMix64 streams and formulas evaluated with numpy, so a CPU
# process can rebuild any index range of a device-generated scene (the values
# agree up to the rounding of the device's log/sin/cos/rsqrt).
# ---------------------------------------------------------------------------
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_STREAM = np.uint64(0x632BE59BD9B4E019)


def _splitmix64(x):
    x = (x + _GOLDEN).astype(np.uint64)
    x = (x ^ (x >> np.uint64(30))) * _M1
    x = (x ^ (x >> np.uint64(27))) * _M2
    return x ^ (x >> np.uint64(31))


def _u01(seed, stream, i):
    with np.errstate(over="ignore"):
        h = _splitmix64(np.uint64(seed) ^ _splitmix64(np.uint64(stream) * _STREAM + np.asarray(i, np.uint64)))
    return (h >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0)


def _normal2(seed, stream, i):
    i = np.asarray(i, np.uint64)
    u = np.maximum(_u01(seed, stream, 2 * i), 1e-7)
    v = _u01(seed, stream, 2 * i + 1)
    r = np.sqrt(-2.0 * np.log(u))
    return r * np.cos(2.0 * np.pi * v), r * np.sin(2.0 * np.pi * v)


def device_mixture_range(n, clusters, seed, lo, hi, edge_sigma=0.001):
    """Triangles [lo, hi) of gprtcuGenMixture(n, clusters, seed, edge_sigma):
    positions [3*(hi-lo), 3] and local indices."""
    i = np.arange(lo, hi, dtype=np.uint64)
    k = (i * np.uint64(clusters)) // np.uint64(n)
    centre = np.stack([_u01(seed, 10, 3 * k + a) for a in range(3)], axis=1)
    sg = 0.005 + 0.045 * _u01(seed, 11, k)
    g = np.empty((i.size, 12))
    for j in range(6):
        a, b = _normal2(seed, 12, 6 * i + j)
        g[:, 2 * j], g[:, 2 * j + 1] = a, b
    c = centre + sg[:, None] * g[:, 0:3]
    pos = np.empty((i.size, 3, 3), np.float64)
    for v in range(3):
        pos[:, v, :] = c + edge_sigma * g[:, 3 + 3 * v:6 + 3 * v]
    pos = pos.reshape(-1, 3).astype(np.float32)
    tri = np.arange(3 * i.size, dtype=np.uint32).reshape(-1, 3)
    return pos, tri


def device_rays_range(seed, lo, hi, box_lo, box_hi):
    """Rays [lo, hi) of gprtcuGenRays aimed at one box: [hi-lo, 8] float32."""
    r = np.arange(lo, hi, dtype=np.uint64)
    box_lo = np.asarray(box_lo, np.float64)
    box_hi = np.asarray(box_hi, np.float64)
    ext = float(np.max(box_hi - box_lo))
    ux, uy = _normal2(seed, 20, 2 * r)
    uz, _ = _normal2(seed, 20, 2 * r + 1)
    inv = 1.0 / np.sqrt(np.maximum(ux * ux + uy * uy + uz * uz, 1e-20))
    centre = 0.5 * (box_lo + box_hi)
    o = centre + 2.0 * ext * np.stack([ux, uy, uz], axis=1) * inv[:, None]
    t = box_lo + (box_hi - box_lo) * np.stack([_u01(seed, 21, 3 * r + a) for a in range(3)], axis=1)
    d = t - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out = np.zeros((r.size, 8), np.float32)
    out[:, 0:3] = o
    out[:, 4:7] = d
    out[:, 7] = np.inf
    return out


# Corners of a unit cube by (x, y, z) bits, and the cells one cube is split
# into, as node lists of corner numbers (8 = the cube's centre vertex).  Node
# orders follow the shape functions of the reference's cells
# (gprt/gprt_fallbacks.slang:370-406): hexahedron 000 100 110 010 001 101 111
# 011; wedge = a triangle at t = 0 then the same triangle at t = 1; pyramid =
# a bilinear base quad, then the apex.
def _c(x, y, z):
    return x | (y << 1) | (z << 2)


_HEX = [_c(0, 0, 0), _c(1, 0, 0), _c(1, 1, 0), _c(0, 1, 0), _c(0, 0, 1), _c(1, 0, 1), _c(1, 1, 1), _c(0, 1, 1)]
_WEDGES = [[_c(0, 0, 0), _c(1, 0, 0), _c(0, 1, 0), _c(0, 0, 1), _c(1, 0, 1), _c(0, 1, 1)],
           [_c(1, 1, 0), _c(0, 1, 0), _c(1, 0, 0), _c(1, 1, 1), _c(0, 1, 1), _c(1, 0, 1)]]
_FACES = [[_c(0, 0, 0), _c(1, 0, 0), _c(1, 1, 0), _c(0, 1, 0)], [_c(0, 0, 1), _c(0, 1, 1), _c(1, 1, 1), _c(1, 0, 1)],
          [_c(0, 0, 0), _c(0, 0, 1), _c(1, 0, 1), _c(1, 0, 0)], [_c(0, 1, 0), _c(1, 1, 0), _c(1, 1, 1), _c(0, 1, 1)],
          [_c(0, 0, 0), _c(0, 1, 0), _c(0, 1, 1), _c(0, 0, 1)], [_c(1, 0, 0), _c(1, 0, 1), _c(1, 1, 1), _c(1, 1, 0)]]
_PYRAMIDS = [f + [8] for f in _FACES]
_TETS = []
for _a, _b in ((0, 1), (0, 2), (1, 0), (1, 2), (2, 0), (2, 1)):
    _e = [0, 0, 0]
    _e[_a] = 1
    _p1 = _c(*_e)
    _e[_b] = 1
    _TETS.append([_c(0, 0, 0), _p1, _c(*_e), _c(1, 1, 1)])
SOLID_FILLS = [(12, [_HEX]), (13, _WEDGES), (14, _PYRAMIDS), (10, _TETS), (23, [_HEX])]


def solid_grid(g, seed=0, jitter=0.15, fills=None):
    """(vertices float32 [V, 4], indices uint32 [C, 8], types uint8 [C]) of a
    g^3-cube volume mesh over [0, 1]^3: grid vertices jittered by up to
    `jitter` of the spacing, one extra centre vertex per cube; each cube
    filled by a seeded choice among SOLID_FILLS (or the given fill indices);
    unused index slots are 0xFFFFFFFF."""
    rng = np.random.default_rng(seed)
    h = 1.0 / g
    gv = np.stack(np.meshgrid(np.arange(g + 1), np.arange(g + 1), np.arange(g + 1), indexing="ij"), -1)
    gv = gv.reshape(-1, 3).astype(np.float64) * h + rng.uniform(-jitter, jitter, ((g + 1) ** 3, 3)) * h
    cc = np.stack(np.meshgrid(np.arange(g), np.arange(g), np.arange(g), indexing="ij"), -1).reshape(-1, 3)
    centre = (cc + 0.5) * h + rng.uniform(-jitter / 2, jitter / 2, (g ** 3, 3)) * h
    verts = np.zeros(((g + 1) ** 3 + g ** 3, 4), np.float32)
    verts[:, :3] = np.concatenate([gv, centre])
    verts[:, 3] = rng.normal(0.0, 1.0, verts.shape[0])
    # vertex numbers of each cube's 8 corners and its centre: [g^3, 9]
    stride = np.array([(g + 1) ** 2, g + 1, 1])
    corner = np.array([[(k >> 0) & 1, (k >> 1) & 1, (k >> 2) & 1] for k in range(8)])
    cv = np.concatenate([((cc[:, None, :] + corner[None]) * stride).sum(-1),
                         ((g + 1) ** 3 + np.arange(g ** 3))[:, None]], axis=1)
    fill = rng.integers(0, len(SOLID_FILLS), g ** 3) if fills is None else np.resize(np.asarray(fills), g ** 3)
    idx_parts, type_parts, order = [], [], []
    for f, (ctype, cells) in enumerate(SOLID_FILLS):
        cubes = np.nonzero(fill == f)[0]
        for j, nodes in enumerate(cells):
            ix = np.full((cubes.size, 8), 0xFFFFFFFF, np.uint32)
            ix[:, :len(nodes)] = cv[cubes][:, nodes]
            idx_parts.append(ix)
            type_parts.append(np.full(cubes.size, ctype, np.uint8))
            order.append(cubes * 8 + j)
    # cells numbered cube by cube (a cube's cells consecutive)
    o = np.argsort(np.concatenate(order), kind="stable")
    return verts, np.concatenate(idx_parts)[o], np.concatenate(type_parts)[o]
