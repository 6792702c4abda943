"""Regenerates the long-horizon golden fixtures: the benchmark workloads at their stated step counts.

Run in a container that has the reference sources, after building the reference (oracle/Makefile.ref,
REF_SRC=<the reference's src directory>) and the oracle (__graft_entry__.build()):

    python tests/golden/make_long_golden.py [tgv256_200] [ensemble64_200] [spheres16_150]

tgv256_200      the 256^3 Taylor-Green workload, 200 RK4 steps of the unmodified reference (about 40 CPU
                minutes on one core).
ensemble64_200  the 64 members of the batched-ensemble workload, 200 RK4 steps each in the reference (run
                in parallel, one process per member). A member whose flow becomes non-finite in the
                reference is run again to the last step before that, and its fields are stored there.
spheres16_150   the 16-sphere 256x128x128 workload for 150 RK4 steps (its flow stays finite until step
                168) in the oracle's extended-precision image-point mode, at steps 10, 50, 100 and 150,
                plus the per-field distance between the reference's own raw double-precision solve and
                that oracle at the same steps (how the ill-conditioned image-point systems' rounding grows).

Each fixture stores a fixed seeded node subsample of all twelve fields (rho, rho_u, rho_v, rho_w, rho_E,
u, v, w, p, T, mu, kappa), per-field checks over every node (sum |f|, sqrt(sum f^2), max |f|), t and the
per-step history (t after the step, dt used, dt next, five change norms).
"""
import multiprocessing as mp
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "3d-ns-fsi_b200"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)
from oracle import pyoracle as po  # noqa: E402

TGV_SAMPLE = 8192       # nodes sampled from the 16.8 M of the 256^3 grid
MEMBER_SAMPLE = 256     # nodes sampled per ensemble member
SPHERES16_LEVELS = [10, 50, 100, 150]


def checks(f):
    """Per-field (sum |f|, sqrt(sum f^2), max |f|) over every node; f has shape (fields, nodes)."""
    return np.stack([np.abs(f).sum(axis=1), np.sqrt((f * f).sum(axis=1)), np.abs(f).max(axis=1)], axis=1)


def sample_idx(n, count, seed):
    return np.sort(np.random.default_rng(seed).choice(n, size=min(count, n), replace=False))


def tgv256_200():
    cfg = os.path.join(ROOT, "3d-ns-fsi_b200", "cases", "tgv256.cfg")
    with tempfile.TemporaryDirectory(prefix="nsf_tgv256_") as out:
        po.run_reference(cfg, [200], outdir=out)
        fl = po.read_ref_fields(out, 200)
        hist = po.read_ref_history(out)
        f = fl["fields"]
        idx = sample_idx(f.shape[1], TGV_SAMPLE, 256200)
        rec = dict(level=np.array(200), t=np.array(fl["t"]), dt_next=np.array(fl["dt"]), sample_idx=idx,
                   fields=f[:, idx].copy(), checks=checks(f), history=hist)
    np.savez_compressed(os.path.join(HERE, "tgv256_200.npz"), **rec)
    print("tgv256_200 ok", os.path.getsize(os.path.join(HERE, "tgv256_200.npz")))


def _member(args):
    """One ensemble member in the reference: fields at step 200, or at the last step before the first
    step whose change norms are not finite."""
    m, text, steps = args
    with tempfile.TemporaryDirectory(prefix="nsf_ens_") as tmp:
        cfg = os.path.join(tmp, "member.cfg")
        with open(cfg, "w") as fh:
            fh.write(text)
        out = os.path.join(tmp, "a")
        os.makedirs(out)
        po.run_reference(cfg, [steps], outdir=out)
        hist = po.read_ref_history(out)
        bad = np.flatnonzero(~np.isfinite(hist[:, 3:]).all(axis=1))
        nonfinite = int(bad[0]) + 1 if len(bad) else -1  # the step after which the norms are not finite
        level = steps if nonfinite < 0 else nonfinite - 1
        if level != steps:
            out = os.path.join(tmp, "b")
            os.makedirs(out)
            po.run_reference(cfg, [level], outdir=out)
        fl = po.read_ref_fields(out, level)
        f = fl["fields"]
        assert np.isfinite(f).all(), m
        idx = sample_idx(f.shape[1], MEMBER_SAMPLE, 640000 + m)
        return dict(level=level, t=fl["t"], nonfinite=nonfinite, idx=idx, fields=f[:, idx].copy(), checks=checks(f),
                    history=hist)


def ensemble64_200(steps=200):
    import nsfsi
    from sweep_cases import ensemble_member_text
    cfgs = nsfsi.ensemble_configs(n=64, steps=steps)
    jobs = [(m, ensemble_member_text(c, steps), steps) for m, c in enumerate(cfgs)]
    # largest members first so the pool finishes together
    jobs.sort(key=lambda j: -int(cfgs[j[0]].NI * cfgs[j[0]].NJ * cfgs[j[0]].NK))
    with mp.get_context("spawn").Pool(max(1, (os.cpu_count() or 2) - 1)) as pool:
        res = dict(zip([j[0] for j in jobs], pool.map(_member, jobs, chunksize=1)))
    rec = dict(steps=np.array(steps), members=np.array(len(cfgs)))
    for m in range(len(cfgs)):
        r = res[m]
        for k in ("level", "t", "nonfinite"):
            rec["%s_%d" % (k, m)] = np.array(r[k])
        for k in ("idx", "fields", "checks", "history"):
            rec["%s_%d" % (k, m)] = r[k]
    np.savez_compressed(os.path.join(HERE, "ensemble64_200.npz"), **rec)
    print("ensemble64_200 ok", os.path.getsize(os.path.join(HERE, "ensemble64_200.npz")),
          "non-finite members:", sorted((m, res[m]["nonfinite"]) for m in res if res[m]["nonfinite"] > 0))


def spheres16_150():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_parity_gpu import field_errors  # the parity tests' per-field measure
    cfg = os.path.join(ROOT, "3d-ns-fsi_b200", "cases", "spheres16.cfg")
    g = np.load(os.path.join(HERE, "spheres16.npz"))
    idx = g["sample_idx"]
    rec = dict(levels=np.array(SPHERES16_LEVELS), sample_idx=idx)
    with tempfile.TemporaryDirectory(prefix="nsf_s16_") as out:
        po.run_reference(cfg, SPHERES16_LEVELS, outdir=out)
        rec["ref_history"] = po.read_ref_history(out)
        o = po.Oracle(open(cfg).read(), exact_image_solve=True)
        done = 0
        for lv in SPHERES16_LEVELS:
            o.march(lv - done)
            done = lv
            f = o.fields()
            raw = po.read_ref_fields(out, lv)["fields"]
            rec["fields_%d" % lv] = f[:, idx].copy()
            rec["checks_%d" % lv] = checks(f)
            rec["t_%d" % lv] = np.array(o.t)
            rec["raw_vs_exact_%d" % lv] = field_errors(raw, f)
            print("spheres16 level", lv, "reference raw solve vs exact-image oracle:",
                  " ".join("%.2e" % x for x in rec["raw_vs_exact_%d" % lv]), flush=True)
        rec["history"] = o.history()
        o.close()
    np.savez_compressed(os.path.join(HERE, "spheres16_150.npz"), **rec)
    print("spheres16_150 ok", os.path.getsize(os.path.join(HERE, "spheres16_150.npz")))


TARGETS = {"tgv256_200": tgv256_200, "ensemble64_200": ensemble64_200, "spheres16_150": spheres16_150}

if __name__ == "__main__":
    if not po.ref_available():
        sys.exit("oracle/_ref/ref_runner is not built; run make -f oracle/Makefile.ref REF_SRC=... first")
    for n in sys.argv[1:] or list(TARGETS):
        TARGETS[n]()
