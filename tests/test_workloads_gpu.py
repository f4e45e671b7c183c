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


def test_c3_small_quantised_matches_plain(cuda):
    from gprt_b200 import workloads
    out = workloads.c3(steps=1, warmup=1, n=200_000, nrays=100_000)
    assert out["closest"]["hits_identical"] and out["any"]["hits_identical"]
    assert out["closest"]["hit_fraction"] > 0.05


def test_c4_small_all_paths_identical(cuda):
    from gprt_b200 import workloads
    out = workloads.c4(steps=1, warmup=1, meshes=64, n=300_000)
    assert out["hits_identical_plain_batched"] and out["hits_identical_plain_quantised"]
    assert out["hit_fraction"] > 0.0
