"""Event-sharded evaluation (multi-GPU decomposition), checked on the CPU.

Two gloo ranks each take one event block of the same workload, compute their
per-sample sums with the CPU oracle, all-reduce them and finalize; the result
must equal the unsharded evaluation. The GPU engine's shard sums use the same
layout (tests/test_gpu_parity.py checks them against these)."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from ctpwa_b200 import workloads
from oracle.binding import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, cfg, p, port, q):
    import sys

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from oracle.binding import Oracle as Orc

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        o = Orc(cfg, shard=(rank, world))
        sums = torch.from_numpy(o.shard_sums(p, nthreads=2))
        dist.all_reduce(sums)
        nll, g = o.finalize_sums(p, sums.numpy())
        q.put((rank, nll, g, o.nev))
    finally:
        dist.destroy_process_group()


def _rank_hessian(rank, world, cfg, p, port, q):
    import sys

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from ctpwa_b200 import shards
    from oracle.binding import Oracle as Orc

    class OracleShard:
        """CPU stand-in for a sharded analysis handle: value sums from the
        oracle; tangent sums and the finalize by differentiating the oracle's."""

        def __init__(self):
            self.o = Orc(cfg, shard=(rank, world))

        def getShardSums(self, params, precision=None):
            return torch.from_numpy(self.o.shard_sums(params.numpy(), nthreads=2))

        def getShardHvpSums(self, params, dirs):
            return torch.from_numpy(self.o.hvp_sums_fd(params.numpy(), dirs.numpy()).ravel())

        def finalizeShardHvp(self, params, dirs, sums, tsums):
            return torch.from_numpy(self.o.finalize_hvp_fd(params.numpy(), dirs.numpy(), sums.numpy(), tsums.numpy()))

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        H = shards.hessian(OracleShard(), torch.from_numpy(p))
        q.put((rank, H.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def workload(tmp_path_factory):
    d = tmp_path_factory.mktemp("shards")
    cfg = workloads.make("kkpi", d, n_phsp=6_001, n_data=1_503, n_bkg=301, bkg_weight=0.3, accept_reject=False,
                         seed=9, gpu_generator=False)
    o = Oracle(cfg)
    p = workloads.true_params(o.nV, o.theta_init()[0])
    p[2 * o.nV:] *= 1.003
    return cfg, p, o


def test_shard_blocks_partition_the_samples(workload):
    cfg, p, full = workload
    counts = np.array([Oracle(cfg, shard=(r, 3)).nev for r in range(3)])
    assert tuple(counts.sum(axis=0)) == full.nev


def test_single_process_sum_of_shards_equals_full(workload):
    cfg, p, full = workload
    sums = sum(Oracle(cfg, shard=(r, 3)).shard_sums(p) for r in range(3))
    nll, g = full.finalize_sums(p, sums)
    onll, og, _ = full.nll_grad(p)
    assert abs(nll - onll) <= 1e-10 * abs(onll)
    assert np.max(np.abs(g - og)) <= 1e-9 * np.max(np.abs(og))


def test_two_gloo_ranks_equal_unsharded(workload):
    cfg, p, full = workload
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, cfg, p, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=300) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    onll, og, _ = full.nll_grad(p)
    for rank, nll, g, nev in res:
        assert abs(nll - onll) <= 1e-10 * abs(onll), (rank, nll, onll)
        assert np.max(np.abs(g - og)) <= 1e-9 * np.max(np.abs(og))
    assert sum(np.array(r[3]) for r in res).tolist() == list(full.nev)


def test_two_gloo_ranks_hessian_equals_unsharded(workload):
    """shards.hessian: value sums and tangent sums each all-reduced once; the
    Hessian of the union equals the unsharded oracle Hessian."""
    cfg, p, full = workload
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank_hessian, args=(r, 2, cfg, p, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=600) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    Ho = full.hessian_fd(p)
    scale = np.max(np.abs(Ho))
    for rank, H in res:
        assert np.array_equal(H, H.T)
        assert np.max(np.abs(H - Ho)) <= 1e-8 * scale, (rank, np.max(np.abs(H - Ho)) / scale)
    assert np.array_equal(res[0][1], res[1][1])


def _rank_device(rank, world, cfg, p, port, q):
    """One rank of the product's sharded path: its event block on the GPU,
    shards.nll_grad / shards.hessian with a gloo process group."""
    import sys

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import ctpwa_b200
    from ctpwa_b200 import shards

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ana = ctpwa_b200.analysis(cfg, device=0, shard=(rank, world))
        pt = torch.tensor(p, dtype=torch.float64, device="cuda:0")
        out = {}
        for prec in ("fp64", "mixed"):
            nll, g = shards.nll_grad(ana, pt, precision=prec)
            out[prec] = (float(nll), g.cpu().numpy())
        out["hessian"] = shards.hessian(ana, pt).cpu().numpy()
        out["nev"] = ana.getNEvents()
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_product_shards_over_gloo_equal_unsharded(tmp_path):
    """The product's multi-process glue (ctpwa_b200.shards) on the device: two
    processes, each holding one event block on the GPU, exchange their
    per-sample sums over a gloo group; NLL, gradient and exact Hessian of the
    union equal the unsharded handle's (FP64 1e-10 / 1e-9 / 1e-9; mixed form
    within its 1e-3 bar)."""
    import torch
    import ctpwa_b200

    cfg = workloads.make("kkpi", tmp_path, n_phsp=60_011, n_data=10_007, n_bkg=2_003, accept_reject=False, seed=13)
    full = ctpwa_b200.analysis(cfg, device=0)
    p = workloads.true_params(full.getNVector(), full.getFreeResParams()[0].numpy())
    p[2 * full.getNVector():] *= 1.002
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 31500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank_device, args=(r, 2, cfg, p, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=600) for _ in procs]
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    pt = torch.tensor(p, dtype=torch.float64, device="cuda:0")
    n64, g64 = full.getNLLAndGrad(pt, "fp64")
    n64, g64 = float(n64), g64.cpu().numpy()
    H = full.getHessian(pt).cpu().numpy()
    for rank, out in res:
        nll, g = out["fp64"]
        assert abs(nll - n64) <= 1e-10 * abs(n64), (rank, nll, n64)
        assert np.max(np.abs(g - g64)) <= 1e-9 * np.max(np.abs(g64))
        assert abs(out["mixed"][0] - n64) < 1e-3
        assert np.max(np.abs(out["hessian"] - H)) <= 1e-9 * np.max(np.abs(H))
    assert sum(np.array(r[1]["nev"]) for r in res).tolist() == list(full.getNEvents())
