"""Benchmark of the B200 acceleration-structure path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
    python bench.py --only sortscan [--steps K] [--warmup W] [--sort-n N] [--scan-n N]
                    (those extras alone; the sizes default to the full workload)

One step = the large combined workload's batched + quantised pass, replayed
from one CUDA graph: a batched LBVH build over 67,108,864 fp32 triangles in
16,384 meshes (bounds, Morton30 codes, segmented 64-bit (mesh, code) radix
sort, Karras topology, refit), the collapse into 8-wide BVHs with uint8
outward-rounded child boxes, and the closest-hit trace of 134,217,728 rays
(2 per triangle, each mesh's rays aimed at its own box).  Triangles: a
256-cluster Gaussian mixture (centres uniform in [0,1]^3, sigma uniform in
[0.005, 0.05], edges N(0, 0.001^2)); mesh sizes log-uniform in [64, 65536]
scaled to the total.  Synthetic, seeded data generated on the device; inputs
resident in HBM when a step starts; L2 (126 MB) flushed by a 256 MB write
between steps, outside the timed events.

The JSON line's value is whole-job Mrays/s of that step.  It also carries:
  roofline      the wide trace kernel (the largest share of the step) against
                the measured HBM copy bandwidth, at 40 algorithmic bytes per ray
  plain         the same scene through the single-mesh entry points, one build
                and one trace per mesh, and the batched binary path; hits of
                all three compared on every ray
  t_check       hit distances of a seeded 1% subsample of the hits against an
                FP64 plane-equation distance
  cpu_baseline  the CPU oracle on this host's cores, on the first meshes of
                the same workload (their triangles and rays copied from the
                device); oracle_match: the oracle's hits for those meshes
                against the batched + quantised step's, ids and t bits, every
                ray (a mismatch fails the run after the line is printed)
  e2e           the same work from pinned host buffers: triangles, indices,
                offsets and rays copied in and the hits copied out inside the
                timed region, pipelined over 16 runs of meshes on three streams
                (copies in, build + collapse + trace, copies out); the serial
                version (copy all, replay the graph, copy back) is reported
                beside it; h2d_roofline: the bytes copied in per step over
                the step's time against one pinned copy of the rays timed
                alone
  gpu_launches  this library's kernels in the timed region, counted from the
                captured graph's kernel nodes
  small_lbvh    plain LBVH build + trace, 262,144 triangles, 1,048,576 rays
  wide_bvh      binary against quantised wide BVH, 16,777,216 triangles and
                rays, closest and any hit
  spheres, lss  4,194,304 spheres / swept-sphere segments (hair strands):
                bounds + box LBVH build and closest-hit trace of 4,194,304 rays
  solids        a volume mesh of 96^3 jittered cubes filled with tetrahedra,
                pyramids, wedges, hexahedra and tetrahedral pairs (~2.8M
                cells): cell bounds + box LBVH build, and point location of
                16,777,216 points; a sample checked against the oracle
  batched_build 4,096 meshes of log-uniform size in [64, 65,536] (~40M
                triangles, each mesh in its own unit cube): batched build,
                collapse, and the wide trace of 64 rays per triangle (~2.5G
                rays, generated on the device in chunks of meshes)
  instances     two-level scene: 16,384 instances of 64 meshes (4,194,304
                triangles), top-level rebuild and closest-hit trace of
                16,777,216 rays
  c0            the small plain case: 1,048,576 uniform uint32 keys (seed 0)
                with payload = index, and inclusive and exclusive sums of
                1,048,576 uint32 values uniform in [0, 255]; bit-exact against
                std::stable_sort and the serial sum beside them
  sort, scan    268,435,456 Zipf(1.1) uint32 key/payload pairs and a
                1,073,741,824-element uint32 exclusive sum, GB/s of
                algorithmic traffic against the measured HBM bandwidth; beside
                each, the CPU oracle (std::stable_sort, serial exclusive sum,
                one thread) on a bounded sample of the same data
  partition, select
                stable split of 1,073,741,824 uniform int32 by sign (items
                >= 0 first, the rest reversed behind them) and the selection of
                the items >= 0 alone; GB/s of algorithmic traffic, with the
                serial CPU oracle beside each
  clocks        SM clock samples taken during the timed region
Multi-GPU (torchrun): every rank builds and traces its own scene (weak
scaling, no data-path collective); time = max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LBVH build Mprims/s + closest-hit Mrays/s, batched+quantised vs plain; sort GB/s"
TRACE_BYTES_PER_RAY = 40
BUILD_BYTES_PER_PRIM = 300
SORT_N = 268_435_456
SCAN_N = 1_073_741_824
WORKLOAD = ("large combined, batched + quantised: {tris:,} fp32 triangles in {meshes:,} meshes, {rays:,} "
            "closest-hit rays; batched LBVH build + 8-wide uint8-quantised collapse + wide trace in one CUDA graph")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def zipf_keys(n, seed, s=1.1):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    u = torch.rand(n, generator=g, device="cuda", dtype=torch.float64)
    r = torch.floor((1.0 - u) ** (-1.0 / (s - 1.0))).clamp_(1, 2 ** 32 - 1)
    return (r - 1).to(torch.int64).to(torch.int32)  # wraps to the uint32 bit pattern


def c0_small(args, dev, peak, cpu=False):
    """The small plain case: 2^20 uniform uint32 keys from seed 0 with payload
    = index, and inclusive / exclusive sums of 2^20 uint32 values uniform in
    [0, 255].  Device-resident, L2 flushed between calls; with cpu, the
    oracle's std::stable_sort and serial sums (the reference tests' own host
    oracles) are timed beside them and the GPU results compared bit for bit."""
    import torch

    from gprt_b200 import api
    n = 1 << 20
    rng = np.random.default_rng(0)
    kh = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    vh = np.arange(n, dtype=np.uint32)
    xh = rng.integers(0, 256, size=n, dtype=np.uint64).astype(np.uint32)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    k0 = torch.from_numpy(kh.view(np.int32)).to(dev)
    v0 = torch.from_numpy(vh.view(np.int32)).to(dev)
    k, v = torch.empty_like(k0), torch.empty_like(v0)
    sscr = api.scratch(api.sort_scratch_size(n, 4, 4), dev)
    x = torch.from_numpy(xh.view(np.int32)).to(dev)
    oe, oi = torch.empty_like(x), torch.empty_like(x)
    tot = torch.empty(1, dtype=torch.int32, device=dev)
    cscr = api.scratch(api.scan_scratch_size(n), dev)

    def timed(fn, prep=None):
        ts = []
        for i in range(args.warmup + args.steps):
            if prep:
                prep()
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            if i >= args.warmup:
                ts.append(a.elapsed_time(b))
        return float(np.mean(ts))

    sort_ms = timed(lambda: api.sort(k, v, 0, 32, sscr), lambda: (k.copy_(k0), v.copy_(v0)))
    excl_ms = timed(lambda: api.exclusive_sum(x, oe, tot, cscr))
    incl_ms = timed(lambda: api.inclusive_sum(x, oi, tot, cscr))
    out = {"n": n, "note": "L2-resident sizes: fractions reported, not graded",
           "sort": {"ms": sort_ms, "mkeys_s": n / sort_ms / 1e3, "gbs": 68 * n / sort_ms / 1e6,
                    "frac_of_hbm": 68 * n / sort_ms / 1e6 / peak},
           "exclusive_sum": {"ms": excl_ms, "gbs": 8 * n / excl_ms / 1e6, "frac_of_hbm": 8 * n / excl_ms / 1e6 / peak},
           "inclusive_sum": {"ms": incl_ms, "gbs": 8 * n / incl_ms / 1e6, "frac_of_hbm": 8 * n / incl_ms / 1e6 / peak}}
    if cpu:
        import oracle
        ck, cv = kh.copy(), vh.copy()
        t0 = time.perf_counter()
        oracle.lib().orc_sort(ck.ctypes.data, 4, cv.ctypes.data, 4, n)
        t_sort = time.perf_counter() - t0
        ce, ci = np.empty_like(xh), np.empty_like(xh)
        t0 = time.perf_counter()
        oracle.lib().orc_scan_u32(xh.ctypes.data, ce.ctypes.data, n, 0)
        t_excl = time.perf_counter() - t0
        t0 = time.perf_counter()
        oracle.lib().orc_scan_u32(xh.ctypes.data, ci.ctypes.data, n, 1)
        t_incl = time.perf_counter() - t0
        out["bit_exact"] = {
            "sort": bool(np.array_equal(k.cpu().numpy().view(np.uint32), ck)
                         and np.array_equal(v.cpu().numpy().view(np.uint32), cv)),
            "exclusive_sum": bool(np.array_equal(oe.cpu().numpy().view(np.uint32), ce)),
            "inclusive_sum": bool(np.array_equal(oi.cpu().numpy().view(np.uint32), ci))}
        out["cpu_baseline"] = {
            "kind": "port", "cores": 1,
            "sample": "the same 2^20 keys and values: std::stable_sort of (key, payload) and the serial "
                      "exclusive / inclusive sum loops, one thread",
            "sort_mkeys_s": n / t_sort / 1e6, "exclusive_sum_gbs": 8 * n / t_excl / 1e9,
            "inclusive_sum_gbs": 8 * n / t_incl / 1e9}
    del flush
    return out


def sortscan(args, dev, peak, rank, cpu=False):
    """Sort and scan extras; with cpu, the oracle's single-thread C++ sort
    (std::stable_sort on (key, payload), the reference test's own oracle) and
    serial exclusive sum timed beside them on bounded samples of the same data."""
    import torch

    from gprt_b200 import api
    sort_n, scan_n = args.sort_n, args.scan_n
    out = {"c0": c0_small(args, dev, peak, cpu)}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    # sort: Zipf(1.1) uint32 keys, payload = index
    k0 = zipf_keys(sort_n, 7 + rank)
    v0 = torch.arange(sort_n, dtype=torch.int32, device=dev)
    k = torch.empty_like(k0)
    v = torch.empty_like(v0)
    scr = api.scratch(api.sort_scratch_size(sort_n, 4, 4), dev)
    ts = []
    for i in range(args.warmup + args.steps):
        k.copy_(k0)
        v.copy_(v0)
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        api.sort(k, v, 0, 32, scr)
        b.record()
        b.synchronize()
        if i >= args.warmup:
            ts.append(a.elapsed_time(b))
    ok = bool(torch.all(k[1:].to(torch.int64) & 0xFFFFFFFF >= k[:-1].to(torch.int64) & 0xFFFFFFFF).item())
    t = sum(ts) / len(ts)
    alg = 4 + 4 * 2 * 8  # 68 B per pair at 8-bit digits
    out["sort"] = {"n": sort_n, "keys": "Zipf(1.1) uint32 + uint32 payload", "ms": t,
                   "mkeys_s": sort_n / (t * 1e-3) / 1e6, "gbs": alg * sort_n / (t * 1e-3) / 1e9,
                   "frac_of_hbm": alg * sort_n / (t * 1e-3) / 1e9 / peak, "sorted": ok,
                   "gpu_launches_per_call": 6}
    if cpu:
        import oracle
        m = min(1 << 24, sort_n)
        kh = k0[:m].cpu().numpy().view(np.uint32).copy()
        vh = np.arange(m, dtype=np.uint32)
        t0 = time.perf_counter()
        oracle.lib().orc_sort(kh.ctypes.data, 4, vh.ctypes.data, 4, m)
        dt = time.perf_counter() - t0
        out["sort"]["cpu_baseline"] = {"value": m / dt / 1e6, "unit": "Mkeys/s", "cores": 1, "kind": "port",
                                       "sample": "first %d of the same Zipf pairs: std::stable_sort of (key, payload)"
                                                 % m, "ms": dt * 1e3}
    del k0, v0, k, v, scr
    torch.cuda.empty_cache()
    x = torch.randint(0, 256, (scan_n,), dtype=torch.int32, device=dev)
    o = torch.empty_like(x)
    tot = torch.empty(1, dtype=torch.int32, device=dev)
    scr = api.scratch(api.scan_scratch_size(scan_n), dev)
    ts = []
    for i in range(args.warmup + args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        api.exclusive_sum(x, o, tot, scr)
        b.record()
        b.synchronize()
        if i >= args.warmup:
            ts.append(a.elapsed_time(b))
    t = sum(ts) / len(ts)
    out["scan"] = {"n": scan_n, "values": "uniform [0,255] uint32", "ms": t, "gbs": 8 * scan_n / (t * 1e-3) / 1e9,
                   "frac_of_hbm": 8 * scan_n / (t * 1e-3) / 1e9 / peak,
                   "total_ok": int(tot.item()) & 0xFFFFFFFF == int(x.sum().item()) & 0xFFFFFFFF}
    if cpu:
        import oracle
        m = min(1 << 28, scan_n)
        xh = x[:m].cpu().numpy().view(np.uint32).copy()
        oh = np.empty_like(xh)
        t0 = time.perf_counter()
        oracle.lib().orc_scan_u32(xh.ctypes.data, oh.ctypes.data, m, 0)
        dt = time.perf_counter() - t0
        out["scan"]["cpu_baseline"] = {"value": 8 * m / dt / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
                                       "sample": "first %d of the same values: serial exclusive sum" % m,
                                       "ms": dt * 1e3}
        del xh, oh
    del x, o
    torch.cuda.empty_cache()
    # partition / select by sign: uniform int32, items >= 0 selected
    g = torch.Generator(device=dev).manual_seed(11 + rank)
    x = torch.randint(-(1 << 31), (1 << 31) - 1, (scan_n,), dtype=torch.int32, device=dev, generator=g)
    o = torch.empty_like(x)
    cnt = torch.empty(1, dtype=torch.int32, device=dev)
    want = int((x >= 0).sum().item())
    xsum = int(x.sum(dtype=torch.int64).item())
    for name, sel in (("partition", False), ("select", True)):
        ts = []
        for i in range(args.warmup + args.steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            api.partition(x, True, o, cnt, scr, select_only=sel)
            b.record()
            b.synchronize()
            if i >= args.warmup:
                ts.append(a.elapsed_time(b))
        t = sum(ts) / len(ts)
        c = int(cnt.item())
        ok = c == want and bool((o[:c] >= 0).all().item())
        if not sel:
            ok = ok and bool((o[c:] < 0).all().item()) and int(o.sum(dtype=torch.int64).item()) == xsum
        alg = 4 * scan_n + 4 * (c if sel else scan_n)
        out[name] = {"n": scan_n, "values": "uniform int32, items >= 0 selected", "ms": t,
                     "gbs": alg / (t * 1e-3) / 1e9, "frac_of_hbm": alg / (t * 1e-3) / 1e9 / peak, "ok": ok}
        if cpu:
            import oracle
            m = min(1 << 28, scan_n)
            xh = x[:m].cpu().numpy()
            t0 = time.perf_counter()
            _, hc = oracle.partition(xh, True, partition=not sel)
            dt = time.perf_counter() - t0
            out[name]["cpu_baseline"] = {"value": (4 * m + 4 * (hc if sel else m)) / dt / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
                                         "sample": "first %d of the same values: serial stable %s" % (m, name),
                                         "ms": dt * 1e3}
            del xh
    del x, o, scr, flush
    torch.cuda.empty_cache()
    return out




def max_over_ranks(x, device, world):
    """The largest x over all ranks (the slowest rank's time); every rank
    calls it at the same point."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, ms_per_step, world):
    """Millions of units per second for all ranks together, each rank having
    processed units_per_rank in the slowest rank's ms_per_step."""
    return world * units_per_rank / (ms_per_step * 1e-3) / 1e6


def cpu_sample_run(sample, match=None):
    """The CPU oracle (test infrastructure) over a list of (pos, tri, rays[,
    gpu_hits]) meshes: a full build and a closest-hit trace of every mesh.
    Returns (seconds building, seconds tracing, triangles, rays).  With a
    `match` dict and GPU hits in the sample, the oracle's hits are compared
    with them (ids on every ray, t bits on every hit) and the counts added to
    `match`; the comparison is outside the timed parts."""
    import oracle
    tb = tt = 0.0
    ntri = nray = 0
    for item in sample:
        pos, tri, rays = item[:3]
        t0 = time.perf_counter()
        e = oracle.lbvh_build_tri(pos, tri)
        t1 = time.perf_counter()
        exp = oracle.trace_lbvh(pos, tri, e, rays)
        t2 = time.perf_counter()
        tb += t1 - t0
        tt += t2 - t1
        ntri += tri.shape[0]
        nray += rays.shape[0]
        if match is not None and len(item) > 3:
            got = item[3]
            gp = np.ascontiguousarray(got[:, 0]).view(np.uint32)
            hit = exp["prim"] != 0xFFFFFFFF
            bad_id = int((gp != exp["prim"]).sum())
            bad_t = int((np.ascontiguousarray(got[hit, 1]).view(np.uint32)
                         != np.ascontiguousarray(exp["t"][hit]).view(np.uint32)).sum())
            match["meshes"] += 1
            match["rays"] += int(rays.shape[0])
            match["hits"] += int(hit.sum())
            match["id_mismatches"] += bad_id
            match["t_mismatches"] += bad_t
            # diagnostic: the FP64 closest id through the same tree
            d = oracle.fp64_id_diagnostic(pos, tri, e, rays, gp)
            f = match.setdefault("fp64_ids", {})
            for k, v in d.items():
                f[k] = f.get(k, 0) + v
    return tb, tt, ntri, nray


def cpu_baseline(sample, meshes):
    """The oracle timed on the first meshes of the headline workload (copied
    from the device), and its hits compared with the GPU's for those meshes."""
    import oracle
    oracle.lib()
    cpu_sample_run(sample[:1])  # warm-up
    match = {"meshes": 0, "rays": 0, "hits": 0, "id_mismatches": 0, "t_mismatches": 0}
    tb, tt, ntri, nray = cpu_sample_run(sample, match)
    match["match"] = match["id_mismatches"] == 0 and match["t_mismatches"] == 0 and match["rays"] > 0
    match["compared"] = ("the oracle's FP32 LBVH build + closest-hit traversal of each mesh against the "
                         "batched + quantised step's hits: primitive id of every ray, t bits of every hit")
    if "fp64_ids" in match:
        match["fp64_ids"]["compared"] = (
            "diagnostic: the GPU's closest id against the FP64 closest id through the same tree (watertight test "
            "in double precision); fp32_edge / fp64_edge: one precision's test hits a triangle the other's "
            "misses (rays through shared edges and vertices); near_ties: both hit both triangles and their FP64 "
            "distances agree within 1e-6 relative")
    return {"value": nray / (tb + tt) / 1e6, "unit": "Mrays/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": "first %d of %d meshes of the same workload (%d triangles, %d rays), copied from the "
                      "device; per mesh a full LBVH build and a closest-hit trace of its rays"
                      % (len(sample), meshes, ntri, nray),
            "build_mprims_s": ntri / tb / 1e6, "trace_mrays_s": nray / tt / 1e6}, match


def run_reference(args, world, rank):
    if rank != 0:
        return
    import oracle
    from gprt_b200 import workloads
    oracle.lib()
    sample = workloads.large_cpu_sample(args.ref_tris, meshes=args.meshes, n=args.triangles)
    for _ in range(args.warmup):
        cpu_sample_run(sample)
    vals, ms = [], []
    for _ in range(args.steps):
        tb, tt, ntri, nray = cpu_sample_run(sample)
        vals.append(nray / (tb + tt) / 1e6)
        ms.append((tb + tt) * 1e3)
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.median(ms)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD.format(tris=args.triangles, meshes=args.meshes, rays=2 * args.triangles),
                       "triangles_per_gpu": args.triangles, "meshes_per_gpu": args.meshes,
                       "rays_per_gpu": 2 * args.triangles},
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": oracle.num_threads(), "kind": "port",
                             "sample": "first %d of %d meshes (%d triangles, %d rays) per step, regenerated on "
                                       "the host; per mesh a full LBVH build and a closest-hit trace"
                                       % (len(sample), args.meshes, ntri, nray)},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's GPU path needs Vulkan + slangc (unavailable on this box); this arm is the CPU "
                    "restatement of its LBVH build with the watertight traversal, on all host threads"}
    print(json.dumps(line), flush=True)


def t_check(sc, frac=0.01, seed=0):
    """FP64 plane-equation distance against the reported t on a seeded
    subsample of the hits (prim ids of a batch are mesh-local)."""
    import torch
    h = sc.h_q.cpu().numpy()
    hit = np.nonzero(h[:, 0] != -1)[0]
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(hit, size=max(1, int(frac * hit.size)), replace=False))
    mesh = np.searchsorted(sc.roff, idx, side="right") - 1
    prim = sc.off[mesh] + h[idx, 0].astype(np.int64)
    rays = sc.rays[torch.from_numpy(idx).to(sc.rays.device)].double().cpu().numpy()
    tri_ix = torch.from_numpy(prim).to(sc.pos.device)
    v = sc.pos.view(-1, 3, 3)[tri_ix].double().cpu().numpy()
    o, d = rays[:, 0:3], rays[:, 4:7]
    n = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    t64 = np.einsum("ij,ij->i", v[:, 0] - o, n) / np.einsum("ij,ij->i", d, n)
    t32 = h[idx, 1].view(np.float32).astype(np.float64)
    rel = np.abs(t32 - t64) / np.abs(t64)
    return {"rays_checked": int(idx.size), "max_rel_err": float(rel.max()), "tolerance": 1e-6,
            "within_tolerance": bool(rel.max() <= 1e-6)}


def run_b200(args, world, rank, local):
    import torch
    import torch.distributed as dist

    import gprt_b200
    from gprt_b200 import launches, workloads

    torch.cuda.set_device(local)
    gprt_b200.lib()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    peak, peak_kind = measured_peaks()
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def slowest(x):
        return max_over_ranks(x, dev, world)

    if args.only == "sortscan":
        # the sort, scan, partition and select extras alone (their own JSON
        # object, no headline line): a short command to profile those kernels
        out = sortscan(args, dev, peak, rank, cpu=rank == 0 and world == 1 and not args.skip_cpu)
        barrier()
        if rank == 0:
            print(json.dumps({"only": "sortscan", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                              "peak_gbs": peak, "peak_kind": peak_kind, **out}))
        if world > 1:
            dist.destroy_process_group()
        return

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    sc = workloads.LargeScene(meshes=args.meshes, n=args.triangles, seed_offset=rank, device=dev)
    g = sc.capture()
    names = launches.graph_kernels(g)
    launches_per_step = sum(c for n, c in names.items() if launches.PREFIX in n)
    other_kernels = sum(c for n, c in names.items() if launches.PREFIX not in n)

    for _ in range(args.warmup):
        flush.zero_()
        g.replay()
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with Clocks(local) as clk:
        barrier()
        for e0, e1 in ev:
            flush.zero_()
            e0.record(stream)
            g.replay()
            e1.record(stream)
        barrier()
    clocks = clk.summary()
    step_ms = slowest(sum(a.elapsed_time(b) for a, b in ev)) / args.steps
    value = whole_job_rate(sc.nrays, step_ms, world)

    # the step's parts, eager, for the roofline and the build rate
    trace_ms = float(np.mean(workloads.time_steps(sc.trace_quantised, args.steps, 1, flush)))
    build_ms = float(np.mean(workloads.time_steps(sc.build_quantised, args.steps, 1, flush)))
    # the plain and batched binary paths on the same scene
    bat_ms = float(np.mean(workloads.time_steps(sc.batched, args.steps, 1, flush)))
    plain_steps = min(args.steps, args.plain_steps)
    plain_ms = None
    if plain_steps > 0:
        plain_ms = slowest(np.mean(workloads.time_steps(sc.plain, plain_steps, 1, flush)))
    g.replay()
    torch.cuda.synchronize()
    same_bat = bool(torch.equal(sc.h_plain, sc.h_bat)) if plain_ms is not None else None
    same_q = bool(torch.equal(sc.h_plain, sc.h_q)) if plain_ms is not None else bool(torch.equal(sc.h_bat, sc.h_q))
    hit_fraction = float((sc.h_q[:, 0] != -1).float().mean().item())
    tchk = t_check(sc)
    # the first meshes exactly as built and traced, for the CPU oracle (its
    # timing and its hit comparison) once the GPU work is done
    cpu_sample = sc.host_sample(args.cpu_tris) if rank == 0 and world == 1 and not args.skip_cpu else None
    plain_launches = None
    if plain_ms is not None:
        plain_launches, _ = launches.count_kernels(lambda: sc.plain_mesh(0, torch.cuda.current_stream().cuda_stream))

    # ---- end to end from pinned host buffers through the same graph
    host = {}
    for name, t in (("pos", sc.pos), ("tri", sc.tri), ("rays", sc.rays), ("ray_off", sc.ray_off),
                    ("tri_off", sc.batch.tri_off)):
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t)
        host[name] = (h, t)
    hits_p = torch.empty(sc.h_q.shape, dtype=sc.h_q.dtype).pin_memory()
    h2d = sum(h.numel() * h.element_size() for h, _ in host.values())
    d2h = hits_p.numel() * hits_p.element_size()

    def e2e_serial():
        for h, d in host.values():
            d.copy_(h, non_blocking=True)
        g.replay()
        hits_p.copy_(sc.h_q, non_blocking=True)

    serial_ms = slowest(np.sum(workloads.time_steps(e2e_serial, args.steps, max(1, args.warmup), flush))) / args.steps
    serial_ok = bool(torch.equal(hits_p, sc.h_q.cpu()))
    # the timed e2e step: copies in, build + collapse + trace, and hits out
    # pipelined over 16 runs of meshes on three streams
    hits_p.zero_()
    sc.e2e_setup({k: host[k][0] for k in ("pos", "tri", "rays")}, hits_p, chunks=16)
    e2e_ms = slowest(np.sum(workloads.time_steps(sc.e2e_step, args.steps, max(1, args.warmup), flush))) / args.steps
    e2e_v = whole_job_rate(sc.nrays, e2e_ms, world)
    e2e_ok = bool(torch.equal(hits_p, sc.h_q.cpu())) and serial_ok
    h2d = sum(host[k][0].numel() * host[k][0].element_size() for k in ("pos", "tri", "rays")) + \
        sum(ho[0].numel() * 4 + ho[1].numel() * 4 for *_, ho in sc.e2e_runs)
    # the host-to-device link alone, the bound of the e2e step: one pinned
    # copy of the rays (the step's largest input) timed by itself
    hr, dr = host["rays"]
    link_ms = slowest(float(np.median(workloads.time_steps(lambda: dr.copy_(hr, non_blocking=True), 3, 1))))
    link_bytes = hr.numel() * hr.element_size()
    link_gbs = link_bytes / (link_ms * 1e-3) / 1e9
    del hr, dr
    nrays, ntri, meshes = sc.nrays, sc.n, sc.meshes
    del host, hits_p, g
    sc.release()
    del sc
    torch.cuda.empty_cache()

    extra = {}
    if not args.skip_extra:
        ps = workloads.PlainScene(seed=rank, device=dev)
        pb = workloads.time_steps(ps.build, args.steps, args.warmup, flush)
        pt = workloads.time_steps(ps.trace, args.steps, args.warmup, flush)
        extra["small_lbvh"] = {
            "triangles": ps.n, "rays": ps.nrays, "build_ms": float(np.mean(pb)), "trace_ms": float(np.mean(pt)),
            "build_mprims_s": ps.n / np.mean(pb) / 1e3, "trace_mrays_s": ps.nrays / np.mean(pt) / 1e3,
            "step_mrays_s": ps.nrays / (np.mean(pb) + np.mean(pt)) / 1e3}
        # the same scene through the quantised wide BVH, beside the plain path
        ps.wide_setup()
        ps.build()
        wc = workloads.time_steps(ps.collapse, args.steps, args.warmup, flush)
        wt = workloads.time_steps(ps.wide_trace, args.steps, args.warmup, flush)
        ps.trace()
        torch.cuda.synchronize()
        extra["small_lbvh"]["quantised"] = {
            "collapse_ms": float(np.mean(wc)), "trace_ms": float(np.mean(wt)),
            "trace_mrays_s": ps.nrays / np.mean(wt) / 1e3,
            "step_mrays_s": ps.nrays / (np.mean(pb) + np.mean(wc) + np.mean(wt)) / 1e3,
            "hits_identical": bool(torch.equal(ps.hits, ps.hw))}
        del ps
        ws = workloads.WideScene(device=dev)
        extra["wide_bvh"] = ws.run(steps=2, warmup=1, flush=flush)
        del ws
        for kind in ("spheres", "lss"):
            us = workloads.UserScene(kind, device=dev)
            extra[kind] = us.run(steps=3, warmup=1, flush=flush)
            del us
        ss = workloads.SolidScene(device=dev)
        sol = ss.run(steps=3, warmup=1, flush=flush)
        qms = sol["locate_ms"]
        sol["roofline"] = {"kernel": "k_locate_solids", "bound": "hbm",
                           "limiter": "instruction issue (Newton inversion of every candidate cell)",
                           "achieved": 40 * ss.npts / (qms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                           "frac": 40 * ss.npts / (qms * 1e-3) / 1e9 / peak,
                           "algorithmic_bytes": "40 B/query (16 B point in, 8 B hit + 16 B rstw out)"}
        if rank == 0 and world == 1 and not args.skip_cpu:
            import oracle
            k = 2000
            pts, gh, gr = ss.host_sample(k)
            t0 = time.perf_counter()
            ec, ek, er = oracle.solid_locate_brute(ss.verts_h, ss.idx_h, ss.types_h, pts)
            dt = time.perf_counter() - t0
            sol["oracle_match"] = {"points": k, "cells_equal": bool(np.array_equal(gh[:, 0], ec)),
                                   "kinds_equal": bool(np.array_equal(gh[:, 1], ek)),
                                   "rstw_bits_equal": bool(np.array_equal(gr.view(np.uint32), er.view(np.uint32)))}
            sol["cpu_baseline"] = {"value": k / dt / 1e6, "unit": "Mqueries/s", "cores": oracle.num_threads(),
                                   "kind": "port", "sample": "%d of the points: every cell's box, then the Newton "
                                                             "inversion of each cell whose box holds the point" % k}
        extra["solids"] = sol
        del ss
        isc = workloads.InstanceScene(device=dev)
        extra["instances"] = isc.run(steps=3, warmup=1, flush=flush)
        del isc
        torch.cuda.empty_cache()
        bsc = workloads.BatchedScene(device=dev)
        extra["batched_build"] = bsc.run(steps=2, warmup=1, flush=flush)
        del bsc
        torch.cuda.empty_cache()
        torch.cuda.empty_cache()
        del flush
        torch.cuda.empty_cache()
        extra.update(sortscan(args, dev, peak, rank, cpu=rank == 0 and world == 1 and not args.skip_cpu))
    barrier()

    if rank == 0:
        cb = om = None
        if cpu_sample is not None:
            cb, om = cpu_baseline(cpu_sample, meshes)
            del cpu_sample
        achieved = TRACE_BYTES_PER_RAY * nrays / (trace_ms * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD.format(tris=ntri, meshes=meshes, rays=nrays),
                       "triangles_per_gpu": ntri, "meshes_per_gpu": meshes,
                       "rays_per_gpu": nrays, "l2": "flushed (256 MB write) between timed steps",
                       "parallelism": "independent scene per GPU" if world > 1 else "single GPU"},
            "roofline": {"kernel": "k_trace_wide_closest + k_wide_refine (closest hit, batched: the two kernels "
                                   "of one gprtcuWideTrace call, timed together)", "bound": "hbm",
                         "limiter": "instruction issue (divergent per-ray traversal), not DRAM bandwidth: the HBM "
                                    "roofline is the denominator of frac, not what limits the kernel",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind + " hbm_gbs (copy)",
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None,
                         "traffic_source": "not measured by this run (CUDA events give time, not DRAM bytes); "
                                           "taken from ncu captures of this kernel",
                         "algorithmic_bytes": "40 B/ray (32 B ray in + 8 B hit out) x %d rays per launch" % nrays,
                         "launch_ms": trace_ms},
            "build": {"value": ntri / (build_ms * 1e-3) / 1e6, "unit": "Mprims/s", "ms": build_ms,
                      "includes": "batched build + wide collapse",
                      "algorithmic_gbs": BUILD_BYTES_PER_PRIM * ntri / (build_ms * 1e-3) / 1e9},
            "plain": {"plain_ms": plain_ms,
                      "plain_mrays_s": world * nrays / (plain_ms * 1e-3) / 1e6 if plain_ms else None,
                      "plain_steps": plain_steps, "plain_launches_per_mesh": plain_launches,
                      "batched_binary_ms": bat_ms, "batched_binary_mrays_s": nrays / (bat_ms * 1e-3) / 1e6,
                      "speedup_batched_quantised_vs_plain": plain_ms / step_ms if plain_ms else None,
                      "speedup_batched_quantised_vs_batched_binary": bat_ms / step_ms,
                      "hits_identical_plain_batched": same_bat,
                      "hits_identical_plain_quantised" if plain_ms else "hits_identical_batched_quantised": same_q,
                      "hit_fraction": hit_fraction},
            "t_check": tchk,
            "e2e": {"value": e2e_v, "unit": "Mrays/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "ms_per_step": e2e_ms, "hits_match_device": e2e_ok,
                    "h2d_roofline": {"achieved_gbs": h2d / (e2e_ms * 1e-3) / 1e9, "link_gbs": link_gbs,
                                     "frac": h2d / (e2e_ms * 1e-3) / 1e9 / link_gbs,
                                     "link": "one pinned host-to-device copy of the %.2f GB of rays, timed alone"
                                             % (link_bytes / 1e9)},
                    "pipeline": "16 runs of meshes; host-to-device copies, build + collapse + trace and the hits' "
                                "copy back overlap on three streams",
                    "serial_ms_per_step": serial_ms},
            "gpu_launches": launches_per_step * args.steps,
            "gpu_launches_detail": {"per_step": launches_per_step, "other_kernels_in_graph": other_kernels,
                                    "source": "kernel nodes of the replayed CUDA graph"},
            "clocks": clocks,
            "cpu_baseline": cb,
            "oracle_match": om,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
        if om is not None and not om["match"]:
            sys.stderr.write("bench: the GPU hits differ from the oracle's on the CPU sample: %s\n" % json.dumps(om))
            sys.exit(3)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--meshes", type=int, default=16_384, help="meshes of the large workload")
    ap.add_argument("--triangles", type=int, default=67_108_864, help="triangles of the large workload")
    ap.add_argument("--plain-steps", type=int, default=2,
                    help="timed steps of the per-mesh plain comparison (0: no plain comparison)")
    ap.add_argument("--cpu-tris", type=int, default=1 << 23, help="triangles in the CPU baseline sample")
    ap.add_argument("--ref-tris", type=int, default=1 << 20, help="triangles per step of the reference arm")
    ap.add_argument("--skip-extra", action="store_true", help="only the headline workload")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--sort-n", type=int, default=SORT_N, help="pairs of the sort extra")
    ap.add_argument("--scan-n", type=int, default=SCAN_N, help="elements of the scan, partition and select extras")
    ap.add_argument("--only", choices=["sortscan"],
                    help="run only the named extras and print them as one JSON object (no headline line)")
    args = ap.parse_args()
    world, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_b200(args, world, rank, local)


if __name__ == "__main__":
    main()
