"""The benchmark workloads as device-resident scenes with their timed steps.

  PlainScene  plain LBVH build + closest-hit trace: 262,144 soup triangles
              (centroids uniform in the unit cube, vertices N(0, 0.002^2)
              about them), 1,048,576 rays from the radius-2 sphere aimed at
              uniform points in the cube.
  WideScene   quantised wide BVH: 16,777,216 triangles of a 64-cluster
              Gaussian mixture, 16,777,216 rays; plain (binary build + binary
              trace) against quantised (binary build + collapse + wide
              trace), closest and any hit.
  LargeScene  large combined: 67,108,864 mixture triangles (256 clusters)
              split into 16,384 meshes of log-uniform size, 134,217,728 rays
              (2 per triangle, each mesh's rays aimed at that mesh's box):
                plain     the single-mesh entry points once per mesh (build,
                          then trace): what a caller of the plain API issues;
                batched   one batched build + one batched binary trace;
                batched+q one batched build + collapse + wide trace, captured
                          once in a CUDA graph and replayed.
Every time is device time from CUDA events on the launching stream.
"""
import ctypes

import numpy as np
import torch

from . import api, lib, scenes


def _ev():
    return torch.cuda.Event(enable_timing=True)


def time_steps(fn, steps, warmup, flush=None):
    """Per-step device times (ms) of fn() after `warmup` untimed calls; the L2
    is flushed (a write larger than it) before every call when flush is given."""
    for _ in range(warmup):
        if flush is not None:
            flush.zero_()
        fn()
    ts = []
    for _ in range(steps):
        if flush is not None:
            flush.zero_()
        a, b = _ev(), _ev()
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return ts


class PlainScene:
    def __init__(self, n=262_144, nrays=1_048_576, seed=0, device="cuda"):
        dev = torch.device(device)
        self.n, self.nrays = n, nrays
        self.pos_h, self.tri_h = scenes.soup(n, seed=seed)
        self.rays_h = scenes.rays(nrays, seed=1000 + seed)
        self.pos = torch.from_numpy(self.pos_h).to(dev)
        self.tri = torch.from_numpy(self.tri_h.view(np.int32)).to(dev)
        self.rays = torch.from_numpy(self.rays_h).to(dev)
        self.bvh = api.Lbvh(n, dev)
        self.hits = torch.empty((nrays, 2), dtype=torch.int32, device=dev)
        self.tscr = api.scratch(lib().gprtcuTraceScratchSize(), dev)

    def build(self):
        api.lbvh_build_triangles(self.pos, self.tri, self.bvh)

    def trace(self):
        api.trace(self.bvh, self.rays, self.hits, scr=self.tscr)

    def step(self):
        self.build()
        self.trace()

    # the same scene through the 8-wide quantised BVH (collapse of the binary
    # LBVH just built, then the wide traversal)
    def wide_setup(self):
        self.wide = api.WideBvh(self.n, 1, self.rays.device)
        self.hw = torch.empty_like(self.hits)

    def collapse(self):
        api.wide_build(self.bvh, wide=self.wide)

    def wide_trace(self):
        api.wide_trace(self.wide, self.rays, hits=self.hw, scr=self.tscr)


class WideScene:
    def __init__(self, n=16_777_216, nrays=16_777_216, clusters=64, device="cuda"):
        dev = torch.device(device)
        self.n, self.nrays, self.clusters = n, nrays, clusters
        self.pos, self.tri = api.gen_mixture(n, clusters=clusters, seed=3, device=dev)
        self.rays = api.gen_rays(nrays, seed=4, device=dev)
        self.bvh = api.Lbvh(n, dev, with_aabbs=False)
        self.wide = api.WideBvh(n, 1, dev)
        self.hb = torch.empty((nrays, 2), dtype=torch.int32, device=dev)
        self.hw = torch.empty_like(self.hb)
        self.tscr = api.scratch(lib().gprtcuTraceScratchSize(), dev)

    def run(self, steps=2, warmup=1, flush=None):
        mean = lambda ts: float(np.mean(ts))
        out = {"triangles": self.n, "rays": self.nrays, "clusters": self.clusters}
        t_build = mean(time_steps(lambda: api.lbvh_build_triangles(self.pos, self.tri, self.bvh), steps, warmup, flush))
        t_collapse = mean(time_steps(lambda: api.wide_build(self.bvh, wide=self.wide), steps, warmup, flush))
        for anyhit in (False, True):
            t_bin = mean(time_steps(lambda: api.trace(self.bvh, self.rays, self.hb, anyhit=anyhit, scr=self.tscr),
                                    steps, warmup, flush))
            t_wide = mean(time_steps(lambda: api.wide_trace(self.wide, self.rays, hits=self.hw, anyhit=anyhit,
                                                            scr=self.tscr), steps, warmup, flush))
            if anyhit:
                same = bool(torch.equal(self.hb[:, 0] == -1, self.hw[:, 0] == -1))
            else:
                same = bool(torch.equal(self.hb, self.hw))
            out["any" if anyhit else "closest"] = {
                "plain_trace_ms": t_bin, "quantised_trace_ms": t_wide,
                "plain_mrays_s": self.nrays / (t_build + t_bin) / 1e3,
                "quantised_mrays_s": self.nrays / (t_build + t_collapse + t_wide) / 1e3,
                "trace_only_speedup": t_bin / t_wide, "hits_identical": same,
                "hit_fraction": float((self.hw[:, 0] != -1).float().mean().item())}
        out["build_ms"] = t_build
        out["collapse_ms"] = t_collapse
        out["build_mprims_s"] = self.n / t_build / 1e3
        torch.cuda.synchronize()
        out["wide_nodes"] = int(self.wide.count.item())
        return out


def large_sizes(meshes=16_384, total=67_108_864, seed=2):
    """Log-uniform mesh sizes in [64, 65536], scaled to sum to `total`."""
    rng = np.random.default_rng(seed)
    s = np.exp(rng.uniform(np.log(64), np.log(65536), size=meshes))
    s = np.maximum(np.floor(s * (total / s.sum())), 2).astype(np.int64)
    s[-1] += total - s.sum()
    return s


class LargeScene:
    TRI_SEED, RAY_SEED, CLUSTERS = 5, 6, 256

    def __init__(self, meshes=16_384, n=67_108_864, rays_per_tri=2, device="cuda", seed_offset=0):
        dev = torch.device(device)
        self.dev = dev
        self.meshes, self.n = meshes, n
        self.tri_seed = self.TRI_SEED + 1000 * seed_offset
        self.ray_seed = self.RAY_SEED + 1000 * seed_offset
        self.sizes = large_sizes(meshes, n)
        self.off = np.zeros(meshes + 1, np.int64)
        self.off[1:] = np.cumsum(self.sizes)
        self.roff = self.off * rays_per_tri
        self.nrays = int(self.roff[-1])
        self.pos, self.tri = api.gen_mixture(n, clusters=self.CLUSTERS, seed=self.tri_seed, device=dev)
        self.batch = api.BatchLbvh(self.off, dev, with_aabbs=False)
        self.ray_off = torch.from_numpy(self.roff.astype(np.uint32).view(np.int32)).to(dev)
        api.batch_build_triangles(self.pos, self.tri, self.batch)  # per-mesh boxes to aim the rays at
        self.rays = api.gen_rays(self.nrays, seed=self.ray_seed, ray_off=self.ray_off, meshes=meshes,
                                 boxes=self.batch.scene, device=dev)
        self.wide = api.WideBvh(n, meshes, dev)
        self.tscr = api.scratch(lib().gprtcuTraceScratchSize(), dev)
        self.h_plain = torch.empty((self.nrays, 2), dtype=torch.int32, device=dev)
        self.h_bat = torch.empty_like(self.h_plain)
        self.h_q = torch.empty_like(self.h_plain)
        self._plain_ready = False
        self.graph = None

    # ---- plain: one build + one trace per mesh through the single-mesh API
    def _plain_setup(self):
        L = lib()
        maxn = int(self.sizes.max())
        self.local_tri = torch.arange(3 * maxn, dtype=torch.int32, device=self.dev)
        self.pscr = api.scratch(L.gprtcuLbvhScratchSize(maxn), self.dev)
        b = self.batch
        self.descs = []
        for m in range(self.meshes):
            o = int(self.off[m])
            self.descs.append(api.LbvhDesc(0, b.codes.data_ptr() + 4 * o, b.ids.data_ptr() + 4 * o,
                                           b.nodes.data_ptr() + 16 * (2 * o - m), None, None, None,
                                           b.bvh2.data_ptr() + 64 * (o - m), b.leaf.data_ptr() + 48 * o))
        self._plain_ready = True

    def plain_mesh(self, m, stream):
        L = lib()
        o, cnt = int(self.off[m]), int(self.sizes[m])
        st = L.gprtcuLbvhBuildTriangles(self.pos.data_ptr() + 36 * o, self.local_tri.data_ptr(), cnt, 0,
                                        ctypes.byref(self.descs[m]), self.pscr.data_ptr(), self.pscr.numel(), stream)
        if st:
            raise RuntimeError("plain build failed: %d" % st)
        r0, rc = int(self.roff[m]), int(self.roff[m + 1] - self.roff[m])
        st = L.gprtcuTraceClosest(ctypes.byref(self.descs[m]), self.rays.data_ptr() + 32 * r0, rc,
                                  self.h_plain.data_ptr() + 8 * r0, self.tscr.data_ptr(), self.tscr.numel(), stream)
        if st:
            raise RuntimeError("plain trace failed: %d" % st)

    def plain(self):
        if not self._plain_ready:
            self._plain_setup()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        for m in range(self.meshes):
            self.plain_mesh(m, stream)

    # ---- batched binary
    def batched(self):
        api.batch_build_triangles(self.pos, self.tri, self.batch)
        api.batch_trace(self.batch, self.rays, self.ray_off, hits=self.h_bat, scr=self.tscr)

    # ---- batched + quantised
    def build_quantised(self):
        api.batch_build_triangles(self.pos, self.tri, self.batch)
        api.wide_build(self.batch, wide=self.wide)

    def trace_quantised(self):
        api.wide_trace(self.wide, self.rays, self.ray_off, hits=self.h_q, scr=self.tscr)

    def quantised(self):
        self.build_quantised()
        self.trace_quantised()

    def capture(self):
        """Capture the batched + quantised step once into a CUDA graph."""
        self.quantised()
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph(keep_graph=True)
        with torch.cuda.graph(self.graph):
            self.quantised()
        self.graph.replay()
        torch.cuda.synchronize()
        return self.graph

    # ---- end to end from pinned host buffers, pipelined over mesh chunks
    def e2e_setup(self, host, hits_host, chunks=8):
        """Split the meshes into `chunks` runs of about equal triangle count.
        Each run is its own batch (its triangles' vertex indices still point
        into the whole position array), collapsed and traced on its own, so
        the run's host-to-device copies, its build + trace and its hits' copy
        back overlap those of the other runs on three streams.  host: dict of
        pinned tensors "pos", "tri", "rays" (the scene's shapes)."""
        self.e2e_host, self.e2e_hits_host = host, hits_host
        cum = self.off[1:]
        cuts = [0] + [int(np.searchsorted(cum, self.n * k / chunks, side="left")) + 1 for k in range(1, chunks)]
        cuts = sorted(set(min(max(c, 1), self.meshes) for c in cuts[1:]) | {0, self.meshes})
        self.e2e_runs = []
        for m0, m1 in zip(cuts[:-1], cuts[1:]):
            t0, t1 = int(self.off[m0]), int(self.off[m1])
            r0, r1 = int(self.roff[m0]), int(self.roff[m1])
            off = self.off[m0:m1 + 1] - t0
            roff = self.roff[m0:m1 + 1] - r0
            b = api.BatchLbvh(off, self.dev, with_aabbs=False)
            w = api.WideBvh(t1 - t0, m1 - m0, self.dev)
            ro = torch.from_numpy(roff.astype(np.uint32).view(np.int32)).to(self.dev)
            # the run's mesh and ray offsets are inputs too: copied every step
            ho = (torch.from_numpy(off.astype(np.uint32).view(np.int32)).pin_memory(),
                  torch.from_numpy(roff.astype(np.uint32).view(np.int32)).pin_memory())
            self.e2e_runs.append((t0, t1, r0, r1, b, w, ro, ho))
        self.e2e_hits = torch.empty_like(self.h_q)
        self.s_in, self.s_run, self.s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()

    def e2e_step(self):
        """One pipelined end-to-end step; the caller's stream waits for all of it."""
        h = self.e2e_host
        start = torch.cuda.Event()
        start.record()
        for s in (self.s_in, self.s_run, self.s_out):
            s.wait_event(start)
        ev_in, ev_run = [], []
        with torch.cuda.stream(self.s_in):
            for t0, t1, r0, r1, b, _, ro, ho in self.e2e_runs:
                b.tri_off.copy_(ho[0], non_blocking=True)
                ro.copy_(ho[1], non_blocking=True)
                self.pos[3 * t0:3 * t1].copy_(h["pos"][3 * t0:3 * t1], non_blocking=True)
                self.tri[t0:t1].copy_(h["tri"][t0:t1], non_blocking=True)
                self.rays[r0:r1].copy_(h["rays"][r0:r1], non_blocking=True)
                e = torch.cuda.Event()
                e.record()
                ev_in.append(e)
        with torch.cuda.stream(self.s_run):
            for (t0, t1, r0, r1, b, w, ro, _), e in zip(self.e2e_runs, ev_in):
                self.s_run.wait_event(e)
                api.batch_build_triangles(self.pos, self.tri[t0:t1], b)
                api.wide_build(b, wide=w)
                api.wide_trace(w, self.rays[r0:r1], ro, hits=self.e2e_hits[r0:r1], scr=self.tscr)
                e2 = torch.cuda.Event()
                e2.record()
                ev_run.append(e2)
        with torch.cuda.stream(self.s_out):
            for (t0, t1, r0, r1, _, _, _, _), e in zip(self.e2e_runs, ev_run):
                self.s_out.wait_event(e)
                self.e2e_hits_host[r0:r1].copy_(self.e2e_hits[r0:r1], non_blocking=True)
            done = torch.cuda.Event()
            done.record()
        torch.cuda.current_stream().wait_event(done)

    def host_sample(self, min_tris, hits=None):
        """The first meshes up to `min_tris` triangles, copied from the device
        exactly as they were built and traced: a list of (pos, tri, rays,
        hits) per mesh, with each mesh's triangles local ([k, 3] indices into
        its own [3k, 3] positions) and its hits mesh-local (by default those
        of the batched + quantised step, `h_q`)."""
        m_end = min(max(int(np.searchsorted(self.off, min_tris)) + 1, 1), self.meshes)
        t1, r1 = int(self.off[m_end]), int(self.roff[m_end])
        tri = self.tri[:t1].to(torch.int64).reshape(-1)
        pos = self.pos.view(-1, 3)[tri].cpu().numpy()
        rays = self.rays[:r1].cpu().numpy()
        h = (self.h_q if hits is None else hits)[:r1].cpu().numpy()
        out = []
        for m in range(m_end):
            lo, hi = int(self.off[m]), int(self.off[m + 1])
            rlo, rhi = int(self.roff[m]), int(self.roff[m + 1])
            lt = np.arange(3 * (hi - lo), dtype=np.uint32).reshape(-1, 3)
            out.append((np.ascontiguousarray(pos[3 * lo:3 * hi]), lt, rays[rlo:rhi], h[rlo:rhi]))
        return out

    def release(self):
        self.graph = None
        for k in ("pos", "tri", "batch", "rays", "wide", "h_plain", "h_bat", "h_q", "pscr", "local_tri", "descs",
                  "tscr", "ray_off", "e2e_runs", "e2e_hits", "e2e_host", "e2e_hits_host"):
            if hasattr(self, k):
                delattr(self, k)
        torch.cuda.empty_cache()


def large_cpu_sample(min_tris=1 << 21, meshes=16_384, n=67_108_864, rays_per_tri=2, seed_offset=0):
    """The large workload's first meshes up to `min_tris` triangles, generated
    on the host only (no device): list of (pos, tri, rays) per mesh."""
    sizes = large_sizes(meshes, n)
    off = np.zeros(meshes + 1, np.int64)
    off[1:] = np.cumsum(sizes)
    m_end = int(np.searchsorted(off, min_tris)) + 1
    m_end = min(max(m_end, 1), meshes)
    tri_seed = LargeScene.TRI_SEED + 1000 * seed_offset
    ray_seed = LargeScene.RAY_SEED + 1000 * seed_offset
    out = []
    for m in range(m_end):
        lo, hi = int(off[m]), int(off[m + 1])
        pos, tri = scenes.device_mixture_range(n, LargeScene.CLUSTERS, tri_seed, lo, hi)
        box = pos.min(axis=0), pos.max(axis=0)
        rays = scenes.device_rays_range(ray_seed, lo * rays_per_tri, hi * rays_per_tri, *box)
        out.append((pos, tri, rays))
    return out


class UserScene:
    """Spheres (radius uniform in [0.0005, 0.002], centres uniform in the unit
    cube) or swept-sphere hair strands (random walks of 16 segments, radius
    tapering from [0.0005, 0.0015] to half), n primitives, nrays rays as in
    PlainScene; bounds + box LBVH + closest-hit trace."""

    def __init__(self, kind="spheres", n=4_194_304, nrays=4_194_304, seed=7, device="cuda"):
        dev = torch.device(device)
        rng = np.random.default_rng(seed)
        self.kind, self.n, self.nrays = kind, n, nrays
        if kind == "spheres":
            s = np.empty((n, 4), np.float32)
            s[:, :3] = rng.random((n, 3), dtype=np.float32)
            s[:, 3] = rng.uniform(0.0005, 0.002, n).astype(np.float32)
            self.prims = torch.from_numpy(s).to(dev)
            self.idx = None
        else:
            segs = 16
            strands = n // segs
            start = rng.random((strands, 1, 3))
            steps = rng.normal(0.0, 0.004, (strands, segs, 3))
            p = np.concatenate([start, start + np.cumsum(steps, axis=1)], axis=1)
            r0 = rng.uniform(0.0005, 0.0015, (strands, 1))
            r = r0 * (1.0 - 0.5 * np.arange(segs + 1)[None, :] / segs)
            v = np.concatenate([p, r[:, :, None]], axis=2).reshape(-1, 4).astype(np.float32)
            base = (np.arange(strands) * (segs + 1))[:, None] + np.arange(segs)[None, :]
            idx = np.stack([base, base + 1], axis=2).reshape(-1, 2).astype(np.int32)
            self.prims = torch.from_numpy(v).to(dev)
            self.idx = torch.from_numpy(idx).to(dev)
            self.n = idx.shape[0]
        self.rays = api.gen_rays(nrays, seed=seed + 1, device=dev)
        self.boxes = torch.empty((self.n, 6), dtype=torch.float32, device=dev)
        self.bvh = api.Lbvh(self.n, dev)
        self.hits = torch.empty((nrays, 2), dtype=torch.int32, device=dev)
        self.u = torch.empty(nrays, dtype=torch.float32, device=dev)
        self.tscr = api.scratch(lib().gprtcuTraceScratchSize(), dev)

    def build(self):
        if self.idx is None:
            api.sphere_bounds(self.prims, out=self.boxes)
        else:
            api.lss_bounds(self.prims, self.idx, out=self.boxes)
        api.lbvh_build_boxes(self.boxes, self.bvh)

    def trace(self):
        if self.idx is None:
            api.trace_spheres(self.bvh, self.prims, self.rays, self.hits, self.u, scr=self.tscr)
        else:
            api.trace_lss(self.bvh, self.prims, self.idx, self.rays, hits=self.hits, u=self.u, scr=self.tscr)

    def run(self, steps=3, warmup=1, flush=None):
        tb = float(np.mean(time_steps(self.build, steps, warmup, flush)))
        tt = float(np.mean(time_steps(self.trace, steps, warmup, flush)))
        return {"primitives": self.n, "rays": self.nrays, "build_ms": tb, "trace_ms": tt,
                "build_mprims_s": self.n / tb / 1e3, "trace_mrays_s": self.nrays / tt / 1e3,
                "step_mrays_s": self.nrays / (tb + tt) / 1e3,
                "hit_fraction": float((self.hits[:, 0] != -1).float().mean().item())}


class SolidScene:
    """A volume mesh of g^3 jittered grid cubes filled with linear cells
    (hexahedra, wedge pairs, six pyramids, six tetrahedra or a tetrahedral
    pair per cube; scenes.solid_grid), per-vertex densities N(0, 1); point
    location of `npts` points uniform in [0, 1]^3: cell bounds + box LBVH
    build, then the query."""

    def __init__(self, g=96, npts=16_777_216, seed=13, device="cuda"):
        dev = torch.device(device)
        self.g, self.npts = g, npts
        self.verts_h, self.idx_h, self.types_h = scenes.solid_grid(g, seed=seed)
        self.n = int(self.types_h.size)
        self.solids = api.Solids(torch.from_numpy(self.verts_h).to(dev),
                                 torch.from_numpy(self.idx_h.view(np.int32)).to(dev),
                                 torch.from_numpy(self.types_h).to(dev))
        gen = torch.Generator(device=dev).manual_seed(seed + 1)
        self.points = torch.zeros((npts, 4), dtype=torch.float32, device=dev)
        self.points[:, :3] = torch.rand((npts, 3), generator=gen, device=dev)
        self.aabbs = torch.empty((self.n, 8), dtype=torch.float32, device=dev)
        self.boxes = torch.empty((self.n, 6), dtype=torch.float32, device=dev)
        self.bvh = api.Lbvh(self.n, dev)
        self.hits = torch.empty((npts, 2), dtype=torch.int32, device=dev)
        self.rstw = torch.empty((npts, 4), dtype=torch.float32, device=dev)
        self.tscr = api.scratch(lib().gprtcuTraceScratchSize(), dev)

    def build(self):
        api.solid_bounds(self.solids, self.aabbs, self.boxes)
        api.lbvh_build_boxes(self.boxes, self.bvh)

    def locate(self):
        api.locate_solid_points(self.bvh, self.solids, self.points, self.hits, self.rstw, scr=self.tscr)

    def run(self, steps=3, warmup=1, flush=None):
        tb = float(np.mean(time_steps(self.build, steps, warmup, flush)))
        tq = float(np.mean(time_steps(self.locate, steps, warmup, flush)))
        return {"grid": self.g, "cells": self.n, "vertices": int(self.verts_h.shape[0]),
                "cell_types": {str(int(t)): int(c) for t, c in zip(*np.unique(self.types_h, return_counts=True))},
                "points": self.npts, "build_ms": tb, "locate_ms": tq,
                "build_mcells_s": self.n / tb / 1e3, "locate_mqueries_s": self.npts / tq / 1e3,
                "found_fraction": float((self.hits[:, 0] != -1).float().mean().item())}

    def host_sample(self, k, seed=0):
        """k of the query points and the GPU's answers for them (numpy)."""
        idx = np.sort(np.random.default_rng(seed).choice(self.npts, size=k, replace=False))
        ti = torch.from_numpy(idx).to(self.points.device)
        return (self.points[ti].cpu().numpy(), self.hits[ti].cpu().numpy().view(np.uint32),
                self.rstw[ti].cpu().numpy())


class InstanceScene:
    """Two-level scene: a batch of `meshes` bottom-level meshes (Gaussian
    mixture triangles, log-uniform sizes summing to `n`), `instances` placements
    of them (mesh i mod meshes; random rotation, uniform scale in [0.5, 2],
    translation uniform in [0, 24]^3; masks cycling 0x01, 0x02, 0x04, 0x08) and
    nrays rays aimed at the world box as in PlainScene.  A step re-prepares the
    instances, rebuilds the top-level LBVH and traces every ray (mask 0xFF)."""

    def __init__(self, meshes=64, n=4_194_304, instances=16_384, nrays=16_777_216, seed=11, device="cuda"):
        dev = torch.device(device)
        rng = np.random.default_rng(seed)
        self.meshes, self.n, self.ninst, self.nrays = meshes, n, instances, nrays
        self.off = np.zeros(meshes + 1, np.int64)
        self.off[1:] = np.cumsum(large_sizes(meshes, n, seed=seed))
        self.pos, self.tri = api.gen_mixture(n, clusters=meshes, seed=seed, edge_sigma=0.002, device=dev)
        self.blas = api.BatchLbvh(self.off, dev, with_aabbs=False)
        rec = np.zeros(instances, np.dtype(api.INSTANCE_DTYPE))
        q, _ = np.linalg.qr(rng.normal(size=(instances, 3, 3)))
        m = np.zeros((instances, 3, 4))
        m[:, :, :3] = q * rng.uniform(0.5, 2.0, (instances, 1, 1))
        m[:, :, 3] = rng.uniform(0.0, 24.0, (instances, 3))
        rec["transform"] = m.reshape(instances, 12)
        rec["custom_mask"] = ((1 << (np.arange(instances) % 4)) << 24) | np.arange(instances)
        rec["blas"] = np.arange(instances) % meshes
        self.records = rec
        self.instances = api.instances_tensor(rec, dev)
        self.blas_ms = float(np.mean(time_steps(self.build_blas, 3, 1)))
        self.tlas = api.Tlas(self.instances, self.blas.root, meshes)
        b = self.tlas.boxes
        world = torch.cat([b[:, :3].min(0).values, b[:, 3:].max(0).values]).contiguous()
        self.rays = api.gen_rays(nrays, seed=seed + 1, boxes=world, device=dev)
        self.hits = torch.empty((nrays, 2), dtype=torch.int32, device=dev)
        self.hit_inst = torch.empty(nrays, dtype=torch.int32, device=dev)
        self.tscr = api.scratch(lib().gprtcuTraceScratchSize(), dev)

    def build_blas(self):
        api.batch_build_triangles(self.pos, self.tri, self.blas)

    def build_tlas(self):
        self.tlas.build()

    def trace(self):
        api.trace_instances(self.tlas, self.blas, self.rays, self.blas.tri_off, self.meshes, 0xFF, self.hits,
                            self.hit_inst, scr=self.tscr)

    def run(self, steps=3, warmup=1, flush=None):
        tb = float(np.mean(time_steps(self.build_tlas, steps, warmup, flush)))
        tt = float(np.mean(time_steps(self.trace, steps, warmup, flush)))
        return {"meshes": self.meshes, "triangles": self.n, "instances": self.ninst, "rays": self.nrays,
                "blas_build_ms": self.blas_ms, "tlas_build_ms": tb, "trace_ms": tt,
                "trace_mrays_s": self.nrays / tt / 1e3, "step_mrays_s": self.nrays / (tb + tt) / 1e3,
                "hit_fraction": float((self.hits[:, 0] != -1).float().mean().item())}


class BatchedScene:
    """Batched build configuration: 4,096 meshes of log-uniform size in [64,
    65,536] (about 40M triangles), each mesh of the small-LBVH distribution
    in its own unit cube; 64 rays per triangle aimed at the mesh's box (about
    2.5G rays), generated on the device and traced in chunks of meshes so
    that no more than `chunk_rays` rays are resident at once.  Timed: the
    batched build, the collapse, and the wide trace of every chunk (ray
    generation is outside the timed events)."""

    def __init__(self, meshes=4096, rays_per_tri=64, chunk_rays=1 << 27, seed=2024, device="cuda"):
        dev = torch.device(device)
        rng = np.random.default_rng(seed)
        self.sizes = np.floor(np.exp(rng.uniform(np.log(64), np.log(65536), size=meshes))).astype(np.int64)
        self.meshes = meshes
        self.off = np.zeros(meshes + 1, np.int64)
        self.off[1:] = np.cumsum(self.sizes)
        self.n = int(self.off[-1])
        self.roff = self.off * rays_per_tri
        self.nrays = int(self.roff[-1])
        toff = torch.from_numpy(self.off.astype(np.uint32).view(np.int32)).to(dev)
        self.pos, self.tri = api.gen_soup(self.n, seed=seed + 1, sigma=0.002, tri_off=toff, meshes=meshes,
                                          spacing=2.0, device=dev)
        self.batch = api.BatchLbvh(self.off, dev, with_aabbs=False)
        self.wide = api.WideBvh(self.n, meshes, dev)
        # chunks of whole meshes, each at most chunk_rays rays (a mesh alone may exceed it)
        self.chunks = []
        m0 = 0
        while m0 < meshes:
            m1 = int(np.searchsorted(self.roff, self.roff[m0] + chunk_rays, side="right")) - 1
            m1 = max(m1, m0 + 1)
            self.chunks.append((m0, min(m1, meshes)))
            m0 = min(m1, meshes)
        biggest = max(int(self.roff[b] - self.roff[a]) for a, b in self.chunks)
        self.hits = torch.empty((biggest, 2), dtype=torch.int32, device=dev)
        self.tscr = api.scratch(lib().gprtcuTraceScratchSize(), dev)
        self.seed = seed

    def _chunk_offsets(self, a, b):
        """Ray offsets over all meshes for chunk [a, b): meshes outside it get no rays."""
        r0, r1 = self.roff[a], self.roff[b]
        ro = np.clip(self.roff - r0, 0, r1 - r0)
        return torch.from_numpy(ro.astype(np.uint32).view(np.int32)).to(self.hits.device), int(r1 - r0)

    def run(self, steps=2, warmup=1, flush=None):
        tb = float(np.mean(time_steps(lambda: api.batch_build_triangles(self.pos, self.tri, self.batch), steps, warmup,
                                      flush)))
        tc = float(np.mean(time_steps(lambda: api.wide_build(self.batch, wide=self.wide), steps, warmup, flush)))
        tt, hits, same = 0.0, 0, None
        for k, (a, b) in enumerate(self.chunks):
            ro, nr = self._chunk_offsets(a, b)
            rays = api.gen_rays(nr, seed=self.seed + 7 + k, ray_off=ro, meshes=self.meshes, boxes=self.batch.scene,
                                device=self.hits.device)
            h = self.hits[:nr]
            tt += float(np.mean(time_steps(lambda: api.wide_trace(self.wide, rays, ro, hits=h, scr=self.tscr), 1,
                                           1 if k == 0 else 0, flush)))
            hits += int((h[:, 0] != -1).sum().item())
            if k == 0:
                hb = api.batch_trace(self.batch, rays, ro, scr=self.tscr)
                same = bool(torch.equal(hb, h))
                del hb
            del rays
        return {"meshes": self.meshes, "triangles": self.n, "rays": self.nrays, "ray_chunks": len(self.chunks),
                "build_ms": tb, "collapse_ms": tc, "build_mprims_s": self.n / (tb + tc) / 1e3,
                "trace_ms": tt, "trace_mrays_s": self.nrays / tt / 1e3,
                "hit_fraction": hits / self.nrays, "hits_identical_binary_first_chunk": same}
