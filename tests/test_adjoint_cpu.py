"""The term table of the discrete adjoint (3d-ns-fsi_b200/csrc/gen_rhs_adjoint.py) on the CPU:

* its forward polynomial reproduces the reference's right-hand side (the oracle's, Solver.cpp:181-418)
  on a flow state, and
* its gather-form adjoint is the transpose of that polynomial's Jacobian (dot-product test against
  central finite differences of the forward polynomial).
"""
import importlib.util
import os

import numpy as np
import pytest

from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
spec = importlib.util.spec_from_file_location("gen", os.path.join(ROOT, "3d-ns-fsi_b200", "csrc", "gen_rhs_adjoint.py"))
gen = importlib.util.module_from_spec(spec)
spec.loader.exec_module(gen)

CNAMES = ["ax", "ay", "az", "h0", "xm_xx", "xm_yy", "xm_zz", "xm_yx", "xm_xy", "xm_zx", "xm_xz", "ym_xx", "ym_yy",
          "ym_zz", "ym_xy", "ym_yx", "ym_zy", "ym_yz", "zm_xx", "zm_yy", "zm_zz", "zm_zx", "zm_xz", "zm_zy", "zm_yz",
          "e_xx23", "e_xx12", "e_yx6", "e_zx6", "e_yx4", "e_zx4", "e_yy12", "e_yy23", "e_zy6", "e_zy4", "e_zz12",
          "e_zz23"]


def consts(dx, dy, dz, gamma):
    C = dict(ax=-1 / (2 * dx), ay=-1 / (2 * dy), az=-1 / (2 * dz), h0=1 / (gamma - 1),
             xm_xx=2 / (3 * dx * dx), xm_yy=1 / (2 * dy * dy), xm_zz=1 / (2 * dz * dz), xm_yx=-1 / (6 * dy * dx),
             xm_xy=1 / (4 * dx * dy), xm_zx=-1 / (6 * dz * dx), xm_xz=1 / (4 * dx * dz),
             ym_xx=1 / (2 * dx * dx), ym_yy=2 / (3 * dy * dy), ym_zz=1 / (2 * dz * dz), ym_xy=-1 / (6 * dx * dy),
             ym_yx=1 / (4 * dy * dx), ym_zy=-1 / (6 * dz * dy), ym_yz=1 / (4 * dy * dz),
             zm_xx=1 / (2 * dx * dx), zm_yy=1 / (2 * dy * dy), zm_zz=2 / (3 * dz * dz), zm_zx=1 / (4 * dz * dx),
             zm_xz=-1 / (6 * dx * dz), zm_zy=1 / (4 * dz * dy), zm_yz=-1 / (6 * dy * dz),
             e_xx23=2 / (3 * dx * dx), e_xx12=1 / (2 * dx * dx), e_yx6=-1 / (6 * dy * dx), e_zx6=-1 / (6 * dz * dx),
             e_yx4=1 / (4 * dy * dx), e_zx4=1 / (4 * dz * dx), e_yy12=1 / (2 * dy * dy), e_yy23=2 / (3 * dy * dy),
             e_zy6=-1 / (6 * dz * dy), e_zy4=1 / (4 * dz * dy), e_zz12=1 / (2 * dz * dz), e_zz23=2 / (3 * dz * dz))
    assert set(C) == set(CNAMES)
    return C


def test_term_table_reproduces_the_reference_rhs():
    o = po.Oracle(open(os.path.join(ROOT, "tests/golden/cases/sphere_small.cfg")).read())
    o.march(5)
    f = o.fields()
    shape = tuple(int(x) for x in np.load(os.path.join(ROOT, "tests/golden/sphere_small.npz"))["shape"])
    g = o.geometry()
    C = consts(g[0], g[1], g[2], 1.4)
    fields = {q: f[i].reshape(shape) for q, i in zip(gen.VARS, [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11])}
    mine = gen.forward(gen.rhs_polys(), fields, C)
    ref = o.rhs()
    interior = o.node_types() == 0
    for e in range(5):
        a, b = mine[e].reshape(-1)[interior], ref[e][interior]
        assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-12), e


def test_adjoint_gather_is_the_transpose():
    rng = np.random.default_rng(7)
    shape = (9, 8, 7)
    fields = {q: rng.uniform(0.5, 1.5, shape) for q in gen.VARS}
    C = consts(0.11, 0.13, 0.17, 1.4)
    eqs = gen.rhs_polys()
    inner = np.zeros(shape, bool)
    inner[1:-1, 1:-1, 1:-1] = True
    lam = [rng.standard_normal(shape) * inner for _ in range(5)]
    bar = gen.adjoint(gen.adjoint_terms(eqs), fields, lam, C)
    for q in gen.VARS:
        d = rng.standard_normal(shape)
        h = 1e-6
        fp = dict(fields)
        fm = dict(fields)
        fp[q] = fields[q] + h * d
        fm[q] = fields[q] - h * d
        rp, rm = gen.forward(eqs, fp, C), gen.forward(eqs, fm, C)
        jvp = sum(((rp[e] - rm[e]) / (2 * h) * lam[e]).sum() for e in range(5))
        vjp = (bar[q] * d).sum()
        assert abs(jvp - vjp) <= 1e-7 * max(abs(vjp), 1.0), (q, jvp, vjp)


def test_generated_gather_is_up_to_date():
    """The committed CUDA gather (nsf_rhs_adjoint.cuh) is what the generator emits from the term table."""
    text = gen.emit_cuda(gen.adjoint_terms(gen.rhs_polys()))
    with open(os.path.join(ROOT, "3d-ns-fsi_b200", "csrc", "nsf_rhs_adjoint.cuh")) as f:
        assert f.read() == text


def test_dual_number_oracle_matches_its_finite_differences():
    """The oracle's dual-number run (nsfo_dual_objective) gives the directional derivative of the adjoint's
    objective: on the small sphere case (12 steps, J over the last 4) it matches the oracle's own central
    difference at h = 1e-5 to 1e-7, along a joint perturbation of the level-0 field and the inflow profile."""
    cfg = open(os.path.join(ROOT, "tests/golden/cases/sphere_small.cfg")).read()
    o = po.Oracle(cfg)
    u0 = o.fields()[:5].copy()
    o.march(12)
    dts = o.history()[:, 1].copy()
    o.close()
    rng = np.random.default_rng(3)
    du = rng.standard_normal(u0.shape) * np.maximum(np.abs(u0).max(axis=1), 1e-3)[:, None]
    di = rng.standard_normal((16, 16))
    J, dJ = po.dual_objective(cfg, dts, 4, u0=u0, du0=du, inflow=np.ones((16, 16)), dinflow=di)
    assert J == po.dual_objective(cfg, dts, 4)[0]  # the case's own initial condition, factor 1
    h = 1e-5
    Jp = po.dual_objective(cfg, dts, 4, u0=u0 + h * du, inflow=1 + h * di)[0]
    Jm = po.dual_objective(cfg, dts, 4, u0=u0 - h * du, inflow=1 - h * di)[0]
    assert abs((Jp - Jm) / (2 * h) - dJ) <= 1e-7 * abs(dJ), (dJ, (Jp - Jm) / (2 * h))


def _gather_in_python(text):
    """The generated CUDA gather as a Python function gather(C, lam, val, inner) -> bar[11] (a line-by-line
    translation of its few statement forms)."""
    import re
    body = ["def gather(C, lam, val, inner):", "    bar = [0.0] * 11"]
    indent = 1
    for raw in text.split("\n"):
        line = raw.split("//")[0].strip()
        if not line or line.startswith(("#", "namespace", "template", "__device__", "const Lam", "const Inner",
                                        "}  //", "for (int q")) or "asm volatile" in line:
            continue
        if line.startswith("if (inner("):
            body.append("    " * indent + "if " + line[4:-3] + ":")
            indent += 1
            body.append("    " * indent + "pass")
        elif line == "}":
            indent = max(1, indent - 1)
        elif line.startswith("const double"):
            body.append("    " * indent + line[len("const double "):].rstrip(";"))
        elif line.startswith("bar["):
            body.append("    " * indent + line.rstrip(";"))
    body.append("    return bar")
    src = "\n".join(body)
    src = re.sub(r"C\.(\w+)", r"C['\1']", src)
    ns = {}
    exec(src, ns)
    return ns["gather"]


def test_generated_gather_matches_the_numpy_adjoint():
    """The emitted CUDA expressions (grouped and factored) give the numpy transposed stencil's values at an
    inner node and at nodes next to the faces."""
    rng = np.random.default_rng(11)
    shape = (7, 7, 7)
    fields = {q: rng.uniform(0.5, 1.5, shape) for q in gen.VARS}
    C = consts(0.11, 0.13, 0.17, 1.4)
    inner = np.zeros(shape, bool)
    inner[1:-1, 1:-1, 1:-1] = True
    lam = [rng.standard_normal(shape) * inner for _ in range(5)]
    ref = gen.adjoint(gen.adjoint_terms(gen.rhs_polys()), fields, lam, C)
    with open(os.path.join(ROOT, "3d-ns-fsi_b200", "csrc", "nsf_rhs_adjoint.cuh")) as f:
        gather = _gather_in_python(f.read())
    for X in [(3, 3, 3), (1, 3, 2), (0, 0, 0), (6, 5, 1), (2, 6, 6)]:
        def ok(di, dj, dk):
            return all(0 <= X[a] + d < shape[a] for a, d in enumerate((di, dj, dk)))
        lamf = lambda e, di, dj, dk: lam[e][X[0] + di, X[1] + dj, X[2] + dk] if ok(di, dj, dk) else 0.0  # noqa: E731
        valf = lambda q, di, dj, dk: fields[gen.VARS[q]][X[0] + di, X[1] + dj, X[2] + dk] if ok(di, dj, dk) else 0.0  # noqa: E731
        innerf = lambda di, dj, dk: bool(ok(-di, -dj, -dk) and inner[X[0] - di, X[1] - dj, X[2] - dk])  # noqa: E731
        bar = gather(C, lamf, valf, innerf)
        for q, name in enumerate(gen.VARS):
            r = ref[name][X]
            assert abs(bar[q] - r) <= 1e-12 * max(1.0, abs(r)), (X, name, bar[q], r)
