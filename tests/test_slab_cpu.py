"""x-slab decomposition, host side: the partition (nsf_slab_plan), the refusal of immersed bodies, and the
exchange protocol of a slab group run by two gloo ranks on the CPU -- the same plane transfers as the device
group (each slab's last interior plane to the next slab's first halo plane and back, the periodic x faces
between the end slabs) and the same reductions (maximum of the dt terms, sum of the change norms), on a
model update, must give the single-process result bit for bit."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import nsfsi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_partition_covers_the_interior_planes():
    cfg = nsfsi.config_load(nsfsi.case_path("tgv256"))
    for n in (2, 3, 4, 8):
        plan = nsfsi.slab_plan(cfg, n)
        assert plan[0][0] == 1 and plan[-1][1] == cfg.NI - 2
        for (a, b), (c, _) in zip(plan, plan[1:]):
            assert c == b + 1 and b - a + 1 >= 2
        sizes = [b - a + 1 for a, b in plan]
        assert max(sizes) - min(sizes) <= 1


def test_partition_refuses_too_thin_slabs():
    cfg = nsfsi.config_load(os.path.join(ROOT, "tests", "golden", "cases", "tgv_small.cfg"))
    with pytest.raises(nsfsi.NsfError):
        nsfsi.slab_plan(cfg, int(cfg.NI))


def test_slab_group_refuses_immersed_bodies():
    with pytest.raises(nsfsi.NsfError) as e:
        nsfsi.SlabGroup(nsfsi.case_path("sphere48"), 2)
    assert e.value.code == 6  # NSF_ERR_ARG, before any device work


# ----------------------------------------------------------------------------- exchange protocol, 2 ranks
NI, M, STEPS = 18, 7, 6  # planes (2 faces + 16 interior), values per plane, steps


def model_step(u, lo, hi):
    """A 3-point update of planes lo..hi (periodic x faces copied separately), four stages like RK4."""
    new = u.copy()
    new[lo:hi + 1] = 0.5 * u[lo:hi + 1] + 0.25 * (u[lo - 1:hi] + u[lo + 1:hi + 2]) + 0.01 * np.sin(u[lo:hi + 1])
    return new


def single(u0):
    u = u0.copy()
    terms = []
    for _ in range(STEPS):
        for _stage in range(4):
            u = model_step(u, 1, NI - 2)
            u[0], u[NI - 1] = u[NI - 2], u[1]  # periodic x faces
        terms.append((np.abs(u[1:NI - 1]).max(), (u[1:NI - 1] ** 2).sum()))
    return u, terms


def rank_main(rank, world, port, u0, plan, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    a, b = plan[rank]
    u = u0[a - 1:b + 2].copy()  # local planes: [a-1, b+1]
    n = u.shape[0]
    terms = []

    def send(arr, to):
        dist.send(torch.from_numpy(np.ascontiguousarray(arr)), to)

    def recv(frm):
        t = torch.empty(M, dtype=torch.float64)
        dist.recv(t, frm)
        return t.numpy()

    for _ in range(STEPS):
        for _stage in range(4):
            u = model_step(u, 1, n - 2)
            # periodic x faces between the end slabs (after the stage, before the boundary work)
            if rank == world - 1:
                send(u[n - 2], 0)
            if rank == 0:
                u[0] = recv(world - 1)
                send(u[1], world - 1)
            if rank == world - 1:
                u[n - 1] = recv(0)
            # halos: last interior plane -> next slab's plane 0, first interior plane -> previous slab's last
            if rank + 1 < world:
                send(u[n - 2], rank + 1)
                u[n - 1] = recv(rank + 1)
            if rank > 0:
                u[0] = recv(rank - 1)
                send(u[1], rank - 1)
        mx = torch.tensor([np.abs(u[1:n - 1]).max()], dtype=torch.float64)
        sq = torch.tensor([(u[1:n - 1] ** 2).sum()], dtype=torch.float64)
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sq, op=dist.ReduceOp.SUM)
        terms.append((float(mx.item()), float(sq.item())))
    out[rank] = (a, b, u, terms)
    dist.destroy_process_group()


def test_two_gloo_ranks_follow_the_slab_exchange():
    rng = np.random.default_rng(5)
    u0 = rng.standard_normal((NI, M))
    u0[0], u0[NI - 1] = u0[NI - 2], u0[1]
    cfg = nsfsi.config_load(os.path.join(ROOT, "tests", "golden", "cases", "tgv_small.cfg"))
    cfg.NI = NI
    plan = nsfsi.slab_plan(cfg, 2)
    ref, ref_terms = single(u0)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = 29500 + os.getpid() % 1000
        mp.start_processes(rank_main, args=(2, port, u0, plan, out), nprocs=2, start_method="spawn")
        got = np.zeros_like(ref)
        for r in range(2):
            a, b, u, terms = out[r]
            got[a:b + 1] = u[1:b - a + 2]
            if r == 0:
                got[0] = u[0]
            if r == 1:
                got[NI - 1] = u[-1]
            for (m1, s1), (m2, s2) in zip(terms, ref_terms):
                assert m1 == m2 and abs(s1 - s2) <= 1e-12 * s2
    assert np.array_equal(got, ref)
