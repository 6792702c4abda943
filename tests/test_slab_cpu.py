"""x-slab decomposition, host side: the partition (nsf_slab_plan), the refusal of immersed bodies, the
schedule of a group over several processes (nsf_slab_schedule: which process holds which slab, the plane
transfers in issue order), and that schedule run by two gloo ranks on the CPU -- the transfers the library
lists (each slab's last interior plane to the next slab's halo plane and back, the periodic x faces between
the end slabs; within a process a copy, across processes a send / receive) and the same reductions
(per-slab partials gathered and combined in slab order), on a model update, must give the single-process
result bit for bit."""
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


def model_cfg():
    cfg = nsfsi.config_load(os.path.join(ROOT, "tests", "golden", "cases", "tgv_small.cfg"))
    cfg.NI = NI
    return cfg


def rank_main(rank, world, port, u0, nslabs, out):
    """This process's slabs of the model grid, exchanged exactly as the library's schedule says: after every
    stage the periodic x faces (list 1), then the halos (list 0), each list's sends and receives posted
    together (as one NCCL group) in the schedule's order; then the two reductions over all slabs."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    cfg = model_cfg()
    plan = nsfsi.slab_plan(cfg, nslabs)
    owner, xfers = nsfsi.slab_schedule(cfg, nslabs, world)
    mine = [p for p in range(nslabs) if owner[p] == rank]
    # slab p: global planes a-1 .. b+1
    u = {p: u0[plan[p][0] - 1:plan[p][1] + 2].copy() for p in mine}

    def at(p, g):  # slab p's local index of global plane g
        return g - (plan[p][0] - 1)

    def exchange(lst):
        reqs, landing = [], []
        for (l, a, ga, b, gb) in xfers:
            if l != lst:
                continue
            if owner[a] == rank and owner[b] == rank:
                landing.append((b, gb, u[a][at(a, ga)].copy()))
                continue
            if owner[a] == rank:
                reqs.append(dist.isend(torch.from_numpy(u[a][at(a, ga)].copy()), owner[b]))
            if owner[b] == rank:
                t = torch.empty(M, dtype=torch.float64)
                reqs.append(dist.irecv(t, owner[a]))
                landing.append((b, gb, t))
        for r in reqs:
            r.wait()
        for (b, gb, v) in landing:
            u[b][at(b, gb)] = np.asarray(v)

    terms = []
    for _ in range(STEPS):
        for _stage in range(4):
            for p in mine:
                n = u[p].shape[0]
                u[p] = model_step(u[p], 1, n - 2)
            exchange(1)
            exchange(0)
        parts = torch.zeros(nslabs, 2, dtype=torch.float64)  # per slab: maximum, sum of squares
        for p in mine:
            n = u[p].shape[0]
            parts[p, 0] = float(np.abs(u[p][1:n - 1]).max())
            parts[p, 1] = float((u[p][1:n - 1] ** 2).sum())
        dist.all_reduce(parts)  # every entry has one contributor: the gather of the slabs' partials
        mx, sq = 0.0, 0.0
        for p in range(nslabs):  # combined in slab order, as k_slab_combine
            mx = max(mx, float(parts[p, 0]))
            sq += float(parts[p, 1])
        terms.append((mx, sq))
    out[rank] = ({p: (plan[p], u[p]) for p in mine}, terms)
    dist.destroy_process_group()


def test_schedule_owners_and_transfers():
    cfg = model_cfg()
    owner, xfers = nsfsi.slab_schedule(cfg, 4, 2)
    assert owner == [0, 0, 1, 1]
    plan = nsfsi.slab_plan(cfg, 4)
    halos = [x for x in xfers if x[0] == 0]
    assert len(halos) == 2 * 3 and len([x for x in xfers if x[0] == 2]) == 2 * 3
    for p in range(3):  # slab p's last interior plane to p+1's low halo, p+1's first to p's high halo
        assert (0, p, plan[p][1], p + 1, plan[p + 1][0] - 1) in halos
        assert (0, p + 1, plan[p + 1][0], p, plan[p][1] + 1) in halos
    wraps = [x for x in xfers if x[0] == 1]  # periodic x faces (tgv_small is periodic in x)
    assert wraps == [(1, 3, NI - 2, 0, 0), (1, 0, 1, 3, NI - 1)]
    assert nsfsi.slab_schedule(cfg, 3, 3)[0] == [0, 1, 2]
    with pytest.raises(nsfsi.NsfError):
        nsfsi.slab_schedule(cfg, 2, 3)  # more processes than slabs


@pytest.mark.parametrize("nslabs", [2, 4])
def test_two_gloo_ranks_follow_the_slab_schedule(nslabs):
    rng = np.random.default_rng(5)
    u0 = rng.standard_normal((NI, M))
    u0[0], u0[NI - 1] = u0[NI - 2], u0[1]
    ref, ref_terms = single(u0)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = 29500 + (os.getpid() + nslabs) % 1000
        mp.start_processes(rank_main, args=(2, port, u0, nslabs, out), nprocs=2, start_method="spawn")
        got = np.full_like(ref, np.nan)
        for r in range(2):
            slabs, terms = out[r]
            for p, ((a, b), up) in slabs.items():
                got[a:b + 1] = up[1:-1]
                if p == 0:
                    got[0] = up[0]
                if p == nslabs - 1:
                    got[NI - 1] = up[-1]
            for (m1, s1), (m2, s2) in zip(terms, ref_terms):
                assert m1 == m2 and abs(s1 - s2) <= 1e-12 * s2
    assert np.array_equal(got, ref)


def test_multi_process_group_checks_its_arguments_before_any_device_work():
    cfg = nsfsi.config_load(nsfsi.case_path("tgv256"))
    for rank, world in ((0, 5), (2, 2), (-1, 2)):  # more processes than slabs, rank outside the group
        with pytest.raises(nsfsi.NsfError) as e:
            nsfsi.SlabGroup(cfg, 4, 0, rank=rank, world=world, nccl_id=bytes(nsfsi.NCCL_ID_BYTES))
        assert e.value.code == 6  # NSF_ERR_ARG
    with pytest.raises(nsfsi.NsfError) as e:  # immersed bodies stay refused across processes too
        nsfsi.SlabGroup(nsfsi.case_path("sphere48"), 2, 0, rank=0, world=2, nccl_id=bytes(nsfsi.NCCL_ID_BYTES))
    assert e.value.code == 6
