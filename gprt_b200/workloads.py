"""Timed workloads beyond the headline step (used by bench.py).

  c3  quantised wide BVH: 16,777,216 triangles of a 64-cluster Gaussian
      mixture, 16,777,216 rays; plain (binary build + binary trace) against
      quantised (binary build + collapse + wide trace), closest and any hit.
  c4  large combined: 67,108,864 mixture triangles (256 clusters) split into
      16,384 meshes of log-uniform size, 134,217,728 rays (2 per triangle,
      each mesh's rays aimed at that mesh's box):
        plain     the plain entry points once per mesh (build, then trace):
                  what a caller of the single-mesh API issues;
        batched   one batched build + one batched binary trace;
        batched+q one batched build + collapse + wide trace, captured once in
                  a CUDA graph and replayed.
      Hits of all three are compared on every ray (must be identical).
Every time is device time from CUDA events on the launching stream.
"""
import ctypes

import numpy as np
import torch

from . import api, lib


def _ev():
    return torch.cuda.Event(enable_timing=True)


def _time(fn, steps, warmup, flush=None):
    for _ in range(warmup):
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
    return float(np.mean(ts)), ts


def c3(steps=2, warmup=1, n=16_777_216, nrays=16_777_216, flush=None):
    dev = torch.device("cuda")
    pos, tri = api.gen_mixture(n, clusters=64, seed=3)
    rays = api.gen_rays(nrays, seed=4)
    bvh = api.Lbvh(n, dev, with_aabbs=False)
    wide = api.WideBvh(n, 1, dev)
    hb = torch.empty((nrays, 2), dtype=torch.int32, device=dev)
    hw = torch.empty_like(hb)
    tscr = api.scratch(lib().gprtcuTraceScratchSize(), dev)
    out = {"triangles": n, "rays": nrays, "clusters": 64}
    t_build, _ = _time(lambda: api.lbvh_build_triangles(pos, tri, bvh), steps, warmup, flush)
    t_collapse, _ = _time(lambda: api.wide_build(bvh, wide=wide), steps, warmup, flush)
    for anyhit in (False, True):
        key = "any" if anyhit else "closest"
        t_bin, _ = _time(lambda: api.trace(bvh, rays, hb, anyhit=anyhit, scr=tscr), steps, warmup, flush)
        t_wide, _ = _time(lambda: api.wide_trace(wide, rays, hits=hw, anyhit=anyhit, scr=tscr), steps, warmup, flush)
        if anyhit:
            same = bool(torch.equal(hb[:, 0] == -1, hw[:, 0] == -1))
        else:
            same = bool(torch.equal(hb, hw))
        out[key] = {"plain_trace_ms": t_bin, "quantised_trace_ms": t_wide,
                    "plain_mrays_s": nrays / (t_build + t_bin) / 1e3,
                    "quantised_mrays_s": nrays / (t_build + t_collapse + t_wide) / 1e3,
                    "trace_only_speedup": t_bin / t_wide, "hits_identical": same,
                    "hit_fraction": float((hw[:, 0] != -1).float().mean().item())}
    out["build_ms"] = t_build
    out["collapse_ms"] = t_collapse
    out["build_mprims_s"] = n / t_build / 1e3
    torch.cuda.synchronize()
    out["wide_nodes"] = int(wide.count.item())
    del pos, tri, rays, bvh, wide, hb, hw
    torch.cuda.empty_cache()
    return out


def c4_sizes(meshes=16_384, total=67_108_864, seed=2):
    rng = np.random.default_rng(seed)
    s = np.exp(rng.uniform(np.log(64), np.log(65536), size=meshes))
    s = np.maximum(np.floor(s * (total / s.sum())), 2).astype(np.int64)
    s[-1] += total - s.sum()
    return s


def c4(steps=2, warmup=1, meshes=16_384, n=67_108_864, rays_per_tri=2, flush=None):
    dev = torch.device("cuda")
    sizes = c4_sizes(meshes, n)
    off = np.zeros(meshes + 1, np.int64)
    off[1:] = np.cumsum(sizes)
    roff = off * rays_per_tri
    nrays = int(roff[-1])
    pos, tri = api.gen_mixture(n, clusters=256, seed=5)
    batch = api.BatchLbvh(off, dev, with_aabbs=False)
    ray_off = torch.from_numpy(roff.astype(np.uint32).view(np.int32)).to(dev)
    # per-mesh boxes for aiming the rays: from one batched build
    api.batch_build_triangles(pos, tri, batch)
    rays = api.gen_rays(nrays, seed=6, ray_off=ray_off, meshes=meshes, boxes=batch.scene)
    wide = api.WideBvh(n, meshes, dev)
    tscr = api.scratch(lib().gprtcuTraceScratchSize(), dev)
    h_plain = torch.empty((nrays, 2), dtype=torch.int32, device=dev)
    h_bat = torch.empty_like(h_plain)
    h_q = torch.empty_like(h_plain)
    out = {"triangles": n, "meshes": meshes, "rays": nrays, "mesh_sizes": "log-uniform in [64, 65536] scaled to the total",
           "clusters": 256}

    # ---- plain: one build + one trace per mesh through the single-mesh API
    L = lib()
    maxn = int(sizes.max())
    local_tri = torch.arange(3 * maxn, dtype=torch.int32, device=dev)
    pscr = api.scratch(L.gprtcuLbvhScratchSize(maxn), dev)
    descs = []
    for m in range(meshes):
        b = int(off[m])
        d = api.LbvhDesc(0, batch.codes.data_ptr() + 4 * b, batch.ids.data_ptr() + 4 * b,
                         batch.nodes.data_ptr() + 16 * (2 * b - m), None, None, None,
                         batch.bvh2.data_ptr() + 64 * (b - m), batch.leaf.data_ptr() + 48 * b)
        descs.append(d)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    pos_p, hits_p, rays_p = pos.data_ptr(), h_plain.data_ptr(), rays.data_ptr()
    build, trace = L.gprtcuLbvhBuildTriangles, L.gprtcuTraceClosest
    lt, sp, sn, tp, tn = local_tri.data_ptr(), pscr.data_ptr(), pscr.numel(), tscr.data_ptr(), tscr.numel()

    def plain():
        for m in range(meshes):
            b, cnt = int(off[m]), int(sizes[m])
            st = build(pos_p + 36 * b, lt, cnt, 0, ctypes.byref(descs[m]), sp, sn, stream)
            if st:
                raise RuntimeError("plain build failed: %d" % st)
            r0, rc = int(roff[m]), int(roff[m + 1] - roff[m])
            st = trace(ctypes.byref(descs[m]), rays_p + 32 * r0, rc, hits_p + 8 * r0, tp, tn, stream)
            if st:
                raise RuntimeError("plain trace failed: %d" % st)

    t_plain, _ = _time(plain, steps, warmup, flush)

    # ---- batched binary
    def batched():
        api.batch_build_triangles(pos, tri, batch)
        api.batch_trace(batch, rays, ray_off, hits=h_bat, scr=tscr)

    t_bat, _ = _time(batched, steps, warmup, flush)

    # ---- batched + quantised, captured in a CUDA graph
    def bq():
        api.batch_build_triangles(pos, tri, batch)
        api.wide_build(batch, wide=wide)
        api.wide_trace(wide, rays, ray_off, hits=h_q, scr=tscr)

    bq()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        bq()
    t_q, _ = _time(g.replay, steps, warmup, flush)
    torch.cuda.synchronize()
    same_bat = bool(torch.equal(h_plain, h_bat))
    same_q = bool(torch.equal(h_plain, h_q))
    out.update({
        "plain_ms": t_plain, "batched_ms": t_bat, "batched_quantised_graph_ms": t_q,
        "plain_mrays_s": nrays / t_plain / 1e3, "batched_mrays_s": nrays / t_bat / 1e3,
        "batched_quantised_mrays_s": nrays / t_q / 1e3,
        "speedup_batched_quantised_vs_plain": t_plain / t_q,
        "speedup_batched_quantised_vs_batched": t_bat / t_q,
        "hits_identical_plain_batched": same_bat, "hits_identical_plain_quantised": same_q,
        "hit_fraction": float((h_q[:, 0] != -1).float().mean().item()),
        "plain_launches_per_step": meshes * 11,
    })
    del g
    del pos, tri, batch, rays, wide, h_plain, h_bat, h_q, pscr, local_tri
    torch.cuda.empty_cache()
    return out
