"""Device scene generators and the benchmark workloads at small sizes: the
plain per-mesh, batched and batched+quantised (CUDA graph) paths return
identical hits; the quantised single-mesh path matches the binary one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_generators_are_seeded_and_in_range(cuda):
    import torch
    from gprt_b200 import api
    p1, t1 = api.gen_soup(10000, seed=3)
    p2, _ = api.gen_soup(10000, seed=3)
    p3, _ = api.gen_soup(10000, seed=4)
    assert torch.equal(p1, p2) and not torch.equal(p1, p3)
    assert torch.equal(t1.flatten(), torch.arange(30000, dtype=torch.int32, device="cuda"))
    c = p1.view(-1, 3, 3).mean(dim=1)
    assert float(c.min()) > -0.05 and float(c.max()) < 1.05
    pm, _ = api.gen_mixture(100000, clusters=8, seed=1)
    assert torch.isfinite(pm).all()
    r = api.gen_rays(5000, seed=2)
    d = r[:, 4:7]
    assert torch.allclose(d.norm(dim=1), torch.ones(5000, device="cuda"), atol=1e-5)
    o = r[:, 0:3] - 0.5
    assert torch.allclose(o.norm(dim=1), torch.full((5000,), 2.0, device="cuda"), atol=1e-4)
    assert torch.isinf(r[:, 7]).all() and (r[:, 3] == 0).all()


def test_wide_scene_small_quantised_matches_plain(cuda):
    from gprt_b200 import workloads
    out = workloads.WideScene(n=200_000, nrays=100_000).run(steps=1, warmup=1)
    assert out["closest"]["hits_identical"] and out["any"]["hits_identical"]
    assert out["closest"]["hit_fraction"] > 0.05


def test_large_scene_small_all_paths_identical(cuda):
    import torch
    from gprt_b200 import launches, workloads
    sc = workloads.LargeScene(meshes=64, n=300_000)
    sc.plain()
    sc.batched()
    sc.capture()
    torch.cuda.synchronize()
    assert torch.equal(sc.h_plain, sc.h_bat) and torch.equal(sc.h_plain, sc.h_q)
    assert float((sc.h_q[:, 0] != -1).float().mean()) > 0.0
    # launch counts: the captured batched+quantised step holds only this
    # library's kernels; one plain mesh is one build and one trace
    names = launches.graph_kernels(sc.graph)
    assert names and all("gprtcu" in n for n in names)
    ours, others = launches.count_kernels(sc.batched)
    assert ours >= 9 and not others
    sc.release()


def test_host_generator_restatement_tracks_device(cuda):
    # the CPU baseline regenerates mesh ranges with numpy: same streams and
    # formulas as the device kernels, equal up to the device's transcendental
    # rounding
    import torch
    from gprt_b200 import api, scenes
    n, k, seed = 1_000_000, 256, 5
    pos, _ = api.gen_mixture(n, clusters=k, seed=seed)
    lo, hi = 123_457, 125_000
    hp, _ = scenes.device_mixture_range(n, k, seed, lo, hi)
    dp = pos[3 * lo:3 * hi].cpu().numpy()
    assert np.abs(hp - dp).max() < 1e-5
    box_lo, box_hi = dp.min(axis=0), dp.max(axis=0)
    boxes = torch.from_numpy(np.concatenate([box_lo, box_hi]).astype(np.float32)[None]).cuda()
    off = torch.tensor([0, 4096], dtype=torch.int32, device="cuda")
    r = api.gen_rays(4096, seed=6, ray_off=off, meshes=1, boxes=boxes).cpu().numpy()
    hr = scenes.device_rays_range(6, 0, 4096, box_lo, box_hi)
    fin = np.isfinite(hr)
    assert np.abs(hr[fin] - r[fin]).max() < 1e-4 and np.array_equal(np.isinf(hr), np.isinf(r))


def test_bench_sortscan_extras_small(cuda):
    # The bench's sort / scan / partition / select section on small sizes, as
    # a user runs it: one JSON object whose own checks all hold.
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--only", "sortscan", "--sort-n", "1048583",
                          "--scan-n", "4194311", "--steps", "1", "--warmup", "1", "--skip-cpu"],
                         cwd=root, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [l for l in out.stdout.splitlines() if l.startswith("{")][-1]
    d = json.loads(line)
    assert d["only"] == "sortscan" and d["sort"]["n"] == 1048583 and d["scan"]["n"] == 4194311
    assert d["sort"]["sorted"] and d["scan"]["total_ok"] and d["partition"]["ok"] and d["select"]["ok"]
