"""Benchmark of the B200 acceleration-structure path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one LBVH build over 262,144 fp32 triangles (bounds, Morton30
codes, stable code/id radix sort, Karras topology, refit) followed by one
closest-hit trace of 1,048,576 rays -- the plain LBVH build + trace workload
(soup of triangles with centroids uniform in the unit cube and vertices
N(0, 0.002^2) about them; ray origins uniform on the radius-2 sphere, aimed
at uniform points in the cube).  Synthetic, seeded data; inputs resident in
HBM when a step starts; L2 (126 MB) flushed by a 256 MB write between steps,
outside the timed events.

The JSON line's value is whole-job Mrays/s over build + trace.  It also
carries:
  roofline      the trace kernel (the largest share of the step) against the
                measured HBM copy bandwidth, at 40 algorithmic bytes per ray
  cpu_baseline  the CPU oracle on this host's cores, bounded ray sample
  e2e           the same step through the C ABI from pinned host buffers
                (host->device copies of triangles and rays, device->host
                copy of the hits inside the timed region)
  build, trace  the two halves separately (Mprims/s, Mrays/s)
  sort, scan    268,435,456 Zipf(1.1) uint32 key/payload pairs and a
                1,073,741,824-element uint32 exclusive sum, GB/s of
                algorithmic traffic against the measured HBM bandwidth
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
N_TRI = 262_144
N_RAYS = 1_048_576
TRACE_BYTES_PER_RAY = 40
BUILD_BYTES_PER_PRIM = 300
SORT_N = 268_435_456
SCAN_N = 1_073_741_824
WORKLOAD = "plain LBVH build + closest-hit trace: 262,144 fp32 triangles, 1,048,576 rays"


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


def cpu_baseline(pos, tri, rays, sample_rays):
    """The CPU oracle (test infrastructure) timed on this host: full build,
    bounded ray sample, scaled to the whole step."""
    import oracle
    oracle.lib()
    rs = rays[:sample_rays]
    oracle.lbvh_build_tri(pos, tri)  # warm-up
    t0 = time.perf_counter()
    e = oracle.lbvh_build_tri(pos, tri)
    t1 = time.perf_counter()
    oracle.trace_lbvh(pos, tri, e, rs)
    t2 = time.perf_counter()
    build_s = t1 - t0
    trace_s = (t2 - t1) * (rays.shape[0] / rs.shape[0])
    return {"value": rays.shape[0] / (build_s + trace_s) / 1e6, "unit": "Mrays/s", "cores": oracle.num_threads(),
            "kind": "port",
            "sample": "full %d-triangle build + closest-hit trace of the first %d of %d rays, trace time scaled "
                      "to all rays" % (pos.shape[0] // 3 if tri is None else tri.shape[0], rs.shape[0], rays.shape[0]),
            "build_mprims_s": tri.shape[0] / build_s / 1e6, "trace_mrays_s": rays.shape[0] / trace_s / 1e6}


def zipf_keys(n, seed, s=1.1):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    u = torch.rand(n, generator=g, device="cuda", dtype=torch.float64)
    r = torch.floor((1.0 - u) ** (-1.0 / (s - 1.0))).clamp_(1, 2 ** 32 - 1)
    return (r - 1).to(torch.int64).to(torch.int32)  # wraps to the uint32 bit pattern


def run_reference(args, world, rank):
    if rank != 0:
        return
    from gprt_b200 import scenes
    pos, tri = scenes.soup(N_TRI, seed=0)
    rays = scenes.rays(N_RAYS, seed=1)
    sample = 65536
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(pos, tri, rays, sample)
    for _ in range(args.steps):
        vals.append(cpu_baseline(pos, tri, rays, sample))
    v = float(np.median([x["value"] for x in vals]))
    cb = dict(vals[0])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": N_RAYS / v / 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "triangles": N_TRI, "rays": N_RAYS},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's GPU path needs Vulkan + slangc (unavailable on this box); this arm is the "
                    "CPU restatement of its LBVH build with the watertight traversal, all host threads"}
    print(json.dumps(line), flush=True)


def run_b200(args, world, rank, local):
    import torch
    import torch.distributed as dist

    import gprt_b200
    from gprt_b200 import api, scenes

    torch.cuda.set_device(local)
    gprt_b200.lib()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    peak, peak_kind = measured_peaks()

    pos_h, tri_h = scenes.soup(N_TRI, seed=rank)
    rays_h = scenes.rays(N_RAYS, seed=1000 + rank)
    pos = torch.from_numpy(pos_h).to(dev)
    tri = torch.from_numpy(tri_h.view(np.int32)).to(dev)
    rays = torch.from_numpy(rays_h).to(dev)
    bvh = api.Lbvh(N_TRI, dev)
    hits = torch.empty((N_RAYS, 2), dtype=torch.int32, device=dev)
    tscr = api.scratch(gprt_b200.lib().gprtcuTraceScratchSize(), dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    def step():
        api.lbvh_build_triangles(pos, tri, bvh)
        api.trace(bvh, rays, hits, scr=tscr)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        flush.zero_()
        step()
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with Clocks(local) as clk:
        barrier()
        for e0, e1, e2 in ev:
            flush.zero_()
            e0.record(stream)
            api.lbvh_build_triangles(pos, tri, bvh)
            e1.record(stream)
            api.trace(bvh, rays, hits, scr=tscr)
            e2.record(stream)
        barrier()
    clocks = clk.summary()
    build_ms = [a.elapsed_time(b) for a, b, _ in ev]
    trace_ms = [b.elapsed_time(c) for _, b, c in ev]
    step_ms = sum(build_ms) / len(ev) + sum(trace_ms) / len(ev)
    total = torch.tensor([step_ms * args.steps], device=dev)
    if world > 1:
        dist.all_reduce(total, op=dist.ReduceOp.MAX)
    step_ms = float(total.item()) / args.steps
    value = world * N_RAYS / (step_ms * 1e-3) / 1e6
    trace_avg = sum(trace_ms) / len(trace_ms)
    build_avg = sum(build_ms) / len(build_ms)
    launches_per_step = 11  # bounds, codes, sort (hist + 4 passes + final copy), karras, refit, trace

    # ---- end to end through the C ABI from pinned host memory
    pos_p = torch.from_numpy(pos_h).pin_memory()
    tri_p = torch.from_numpy(tri_h.view(np.int32)).pin_memory()
    rays_p = torch.from_numpy(rays_h).pin_memory()
    hits_p = torch.empty((N_RAYS, 2), dtype=torch.int32).pin_memory()
    h2d = pos_p.numel() * 4 + tri_p.numel() * 4 + rays_p.numel() * 4
    d2h = hits_p.numel() * 4

    def e2e_step():
        pos.copy_(pos_p, non_blocking=True)
        tri.copy_(tri_p, non_blocking=True)
        rays.copy_(rays_p, non_blocking=True)
        step()
        hits_p.copy_(hits, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e2e_step()
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    e2e_t = torch.tensor([sum(e2e_ms)], device=dev)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_v = world * N_RAYS / (float(e2e_t.item()) / args.steps * 1e-3) / 1e6

    # ---- parity spot check of this run's output against the oracle (sample)
    got = api.hits_numpy(hits)

    # ---- sort and scan at the large sizes (rank-local)
    extra = {}
    if not args.skip_sortscan:
        del flush
        torch.cuda.empty_cache()
        extra = sortscan(args, dev, peak, rank)
        flush = None

    if world > 1:
        dist.barrier()
    if rank == 0:
        cb = None
        if world == 1 and not args.skip_cpu:
            cb = cpu_baseline(pos_h, tri_h, rays_h, args.cpu_rays)
        achieved = TRACE_BYTES_PER_RAY * N_RAYS / (trace_avg * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "triangles_per_gpu": N_TRI, "rays_per_gpu": N_RAYS,
                       "l2": "flushed (256 MB write) between timed steps", "code": "morton30",
                       "parallelism": "independent scene per GPU" if world > 1 else "single GPU"},
            "roofline": {"kernel": "k_trace_bin (closest hit)", "bound": "hbm", "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind + " hbm_gbs", "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "algorithmic_bytes": "40 B/ray (32 B ray in + 8 B hit out) x 1,048,576 rays per launch",
                         "launch_ms": trace_avg},
            "build": {"value": N_TRI / (build_avg * 1e-3) / 1e6, "unit": "Mprims/s", "ms": build_avg,
                      "algorithmic_gbs": BUILD_BYTES_PER_PRIM * N_TRI / (build_avg * 1e-3) / 1e9},
            "trace": {"value": N_RAYS / (trace_avg * 1e-3) / 1e6, "unit": "Mrays/s", "ms": trace_avg,
                      "hit_fraction": float((got["prim"] != 0xFFFFFFFF).mean())},
            "e2e": {"value": e2e_v, "unit": "Mrays/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
            "cpu_baseline": cb,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def sortscan(args, dev, peak, rank):
    import torch

    from gprt_b200 import api
    out = {}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    # sort: Zipf(1.1) uint32 keys, payload = index
    k0 = zipf_keys(SORT_N, 7 + rank)
    v0 = torch.arange(SORT_N, dtype=torch.int32, device=dev)
    k = torch.empty_like(k0)
    v = torch.empty_like(v0)
    scr = api.scratch(api.sort_scratch_size(SORT_N, 4, 4), dev)
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
    out["sort"] = {"n": SORT_N, "keys": "Zipf(1.1) uint32 + uint32 payload", "ms": t,
                   "mkeys_s": SORT_N / (t * 1e-3) / 1e6, "gbs": alg * SORT_N / (t * 1e-3) / 1e9,
                   "frac_of_hbm": alg * SORT_N / (t * 1e-3) / 1e9 / peak, "sorted": ok,
                   "gpu_launches_per_call": 6}
    del k0, v0, k, v, scr
    torch.cuda.empty_cache()
    x = torch.randint(0, 256, (SCAN_N,), dtype=torch.int32, device=dev)
    o = torch.empty_like(x)
    tot = torch.empty(1, dtype=torch.int32, device=dev)
    scr = api.scratch(api.scan_scratch_size(SCAN_N), dev)
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
    out["scan"] = {"n": SCAN_N, "values": "uniform [0,255] uint32", "ms": t, "gbs": 8 * SCAN_N / (t * 1e-3) / 1e9,
                   "frac_of_hbm": 8 * SCAN_N / (t * 1e-3) / 1e9 / peak,
                   "total_ok": int(tot.item()) & 0xFFFFFFFF == int(x.sum().item()) & 0xFFFFFFFF}
    del x, o, scr, flush
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-rays", type=int, default=131072)
    ap.add_argument("--skip-sortscan", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_b200(args, world, rank, local)


if __name__ == "__main__":
    main()
