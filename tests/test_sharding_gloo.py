"""View-sharded MLEM with world_size 2 over gloo on CPU.

recon_b200.sharding.sharded_mlem_iteration -- the function bench.py runs at
N > 1 -- drives a CPU stand-in of the plan with the same three methods
(mlem_forward / mlem_backward / mlem_update over a view range, backed by the
FP64 oracle).  The sharded iteration equals the single-process one, the
cross-rank sum is taken in rank order, and every rank ends with the same
bits."""
import os
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import small_cfg


def _setup():
    from oracle import oracle as O
    from recon_b200.configs import geom_dict

    cfg = small_cfg(Xdim=12, Ydim=12, Zdim=8, AxPixels=20, TAxPixels=16, AxPixDim=2.5, TAxPixDim=2.5, NumProj=10)
    g = O.Geom.from_dict(geom_dict(cfg))
    rng = np.random.default_rng(0)
    meas = rng.random(10 * g.npix) * 2.0
    return O, cfg, g, meas


def _projector(O, g, nproj, dang):
    npix = g.npix

    def fp(f, first, count):
        out = np.zeros(count * npix)
        for k in range(count):
            img = np.zeros(npix)
            O.lib().orc_x_fp_view(g, float(np.float32(first + k) * dang), f, img)
            out[k * npix:(k + 1) * npix] = img
        return out

    def bp(sino, first, count):
        vol = np.zeros(g.nvox)
        for k in range(count):
            # back project one view through the FP64 ray walk (views are independent)
            one = np.zeros(nproj * npix)
            one[(first + k) * npix:(first + k + 1) * npix] = sino[k * npix:(k + 1) * npix]
            vol += O.x_bp_all(g, nproj, dang, one, threads=1)
        return vol

    return fp, bp


class _OraclePlan:
    """The split-iteration methods of recon_b200.Plan (recon_mlem_forward,
    recon_mlem_backward, recon_mlem_update), restated on the FP64 oracle: the
    ratios of views [first, first + count) kept inside, their back projection
    into ht, and f = (sens != 0) ? f * ht / sens : 0."""

    def __init__(self, O, g, nproj, dang):
        self.nproj = nproj
        self.fp, self.bp = _projector(O, g, nproj, dang)
        self.npix = g.npix
        self.sens = O.x_bp_all(g, nproj, dang, np.ones(nproj * g.npix), threads=1)
        self.ratio = None

    def mlem_forward(self, g, f, first, count):
        hf = self.fp(f.numpy(), first, count)
        gm = g.numpy()[first * self.npix:(first + count) * self.npix]
        self.ratio = np.where(hf != 0, gm / np.where(hf != 0, hf, 1), 0.0)

    def mlem_backward(self, ht, first, count):
        ht.copy_(torch.from_numpy(self.bp(self.ratio, first, count)))

    def mlem_update(self, f, ht):
        fv, h, s = f.numpy(), ht.numpy(), self.sens
        fv[:] = np.where(s != 0, fv * h / np.where(s != 0, s, 1), 0.0)


def _worker(rank, world, init_file, out_dir):
    dist.init_process_group("gloo", init_method=f"file://{init_file}", rank=rank, world_size=world)
    from recon_b200.sharding import ordered_sum_, sharded_mlem_iteration, view_range

    O, cfg, g, meas = _setup()
    nproj, dang = 10, np.float32(36.0)
    P = _OraclePlan(O, g, nproj, dang)
    f = torch.ones(g.nvox, dtype=torch.float64)
    gt = torch.from_numpy(meas)
    ht = torch.zeros(g.nvox, dtype=torch.float64)
    for _ in range(2):
        sharded_mlem_iteration(P, gt, f, ht)
    np.save(os.path.join(out_dir, f"f{rank}.npy"), f.numpy())
    # the rank-ordered sum itself, twice (its exchange buffers are reused)
    for rep in range(2):
        x = torch.full((7,), float(rank + 1), dtype=torch.float64) * torch.arange(7, dtype=torch.float64)
        ordered_sum_(x)
        np.save(os.path.join(out_dir, f"s{rank}_{rep}.npy"), x.numpy())
    assert view_range(10, rank, world)[1] == 5
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_mlem_two_ranks():
    out_dir = tempfile.mkdtemp()
    init_file = os.path.join(out_dir, "init")
    mp.start_processes(_worker, args=(2, init_file, out_dir), nprocs=2, start_method="spawn")
    f0 = np.load(os.path.join(out_dir, "f0.npy"))
    f1 = np.load(os.path.join(out_dir, "f1.npy"))
    assert np.array_equal(f0, f1)
    for rep in range(2):
        s = np.load(os.path.join(out_dir, f"s0_{rep}.npy"))
        assert np.array_equal(s, 3.0 * np.arange(7))
        assert np.array_equal(s, np.load(os.path.join(out_dir, f"s1_{rep}.npy")))
    # single-process reference
    O, cfg, g, meas = _setup()
    nproj, dang = 10, np.float32(36.0)
    fp, bp = _projector(O, g, nproj, dang)
    sens = O.x_bp_all(g, nproj, dang, np.ones(nproj * g.npix), threads=1)
    f = np.ones(g.nvox)
    for _ in range(2):
        hf = fp(f, 0, nproj)
        ratio = np.where(hf != 0, meas / np.where(hf != 0, hf, 1), 0.0)
        ht = bp(ratio, 0, nproj)
        f = np.where(sens != 0, f * ht / np.where(sens != 0, sens, 1), 0.0)
    assert np.max(np.abs(f - f0)) <= 1e-12 * np.max(np.abs(f))


def test_view_range_partition():
    from recon_b200.sharding import view_range

    for n in (1, 7, 360, 361):
        for w in (1, 2, 3, 8):
            ranges = [view_range(n, r, w) for r in range(w)]
            assert sum(c for _, c in ranges) == n
            assert all(ranges[r][0] + ranges[r][1] == ranges[r + 1][0] for r in range(w - 1))


def test_batched_problems_shard_by_rank():
    # the batched workload over several GPUs: every problem on exactly one rank,
    # largest first to the least-loaded rank, the same split on every rank
    import bench
    from recon_b200.configs import batched_problems

    cfgs = batched_problems(48)
    work = [float(c["NumProj"]) * c["AxPixels"] * c["TAxPixels"] * (c["Xdim"] + c["Ydim"] + c["Zdim"]) for c in cfgs]
    for world in (1, 2, 4, 8):
        parts = bench.shard_problems(work, world)
        assert sorted(p for part in parts for p in part) == list(range(48))
        assert parts == bench.shard_problems(work, world)
        loads = [sum(work[p] for p in part) for part in parts]
        assert max(loads) - min(loads) <= max(work)


class _OracleQuarterPlan(_OraclePlan):
    """_OraclePlan with the quarter-set halves (recon_mlem_forward_quarters /
    recon_mlem_backward_quarters): base views first .. first+count-1 of each of
    the four quarters."""

    quarter_sets = True

    def _ranges(self, first, count):
        q = self.nproj // 4
        return [(first + r * q, count) for r in range(4)]

    def mlem_forward_quarters(self, g, f, first, count):
        self.ratios = []
        for a, c in self._ranges(first, count):
            self.mlem_forward(g, f, a, c)
            self.ratios.append(self.ratio)

    def mlem_backward_quarters(self, ht, first, count):
        total = np.zeros(ht.numel())
        for (a, c), ratio in zip(self._ranges(first, count), self.ratios):
            total += self.bp(ratio, a, c)
        ht.copy_(torch.from_numpy(total))


def _quarter_worker(rank, world, init_file, out_dir):
    dist.init_process_group("gloo", init_method=f"file://{init_file}", rank=rank, world_size=world)
    from recon_b200.sharding import sharded_mlem_iteration

    O, cfg, g, _ = _setup()
    nproj, dang = 12, np.float32(30.0)
    meas = np.random.default_rng(5).random(nproj * g.npix) * 2.0
    P = _OracleQuarterPlan(O, g, nproj, dang)
    f = torch.ones(g.nvox, dtype=torch.float64)
    ht = torch.zeros(g.nvox, dtype=torch.float64)
    for _ in range(2):
        sharded_mlem_iteration(P, torch.from_numpy(meas), f, ht)
    np.save(os.path.join(out_dir, f"q{rank}.npy"), f.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_mlem_quarter_sets_two_ranks():
    """Plans whose back projection takes quarter sets are split by quarter sets
    (rank 0: base views 0, 1 of each quarter; rank 1: base view 2); the result
    is the single-process iteration's."""
    out_dir = tempfile.mkdtemp()
    init_file = os.path.join(out_dir, "init")
    mp.start_processes(_quarter_worker, args=(2, init_file, out_dir), nprocs=2, start_method="spawn")
    f0 = np.load(os.path.join(out_dir, "q0.npy"))
    assert np.array_equal(f0, np.load(os.path.join(out_dir, "q1.npy")))
    O, cfg, g, _ = _setup()
    nproj, dang = 12, np.float32(30.0)
    meas = np.random.default_rng(5).random(nproj * g.npix) * 2.0
    fp, bp = _projector(O, g, nproj, dang)
    sens = O.x_bp_all(g, nproj, dang, np.ones(nproj * g.npix), threads=1)
    f = np.ones(g.nvox)
    for _ in range(2):
        hf = fp(f, 0, nproj)
        ratio = np.where(hf != 0, meas / np.where(hf != 0, hf, 1), 0.0)
        f = np.where(sens != 0, f * bp(ratio, 0, nproj) / np.where(sens != 0, sens, 1), 0.0)
    assert np.max(np.abs(f - f0)) <= 1e-12 * np.max(np.abs(f))


def test_quarter_sets_partition():
    """The ranks' quarter sets cover every view exactly once."""
    from recon_b200.sharding import view_range

    for n in (4, 12, 360, 720):
        for w in (1, 2, 3, 8):
            q = n // 4
            views = []
            for r in range(w):
                a, c = view_range(q, r, w)
                views += [a + k + s * q for s in range(4) for k in range(c)]
            assert sorted(views) == list(range(n))
