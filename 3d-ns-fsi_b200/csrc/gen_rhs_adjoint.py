"""Generator of the transposed right-hand-side stencil (discrete adjoint of the RHS, gather form).

The right-hand side of the five flux loops (Solver.cpp:181-418; the stage kernel evaluates it as x_node,
x_face and yz_part in nsf_physics.cuh) is written below once, as a polynomial in nodal quantities at stencil offsets
(RU, RV, RW, RE: conserved momenta and energy; u, v, w, p, T, mu, ka: primitive and transport values)
with the reference's stencil coefficients. From it this script emits

  * nsf_rhs_adjoint.cuh: a device function that, for one node m, gathers the adjoint of every input
    quantity at m from the RHS adjoints lambda_e of the interior nodes whose stencil contains m:
        qbar(m) = sum_e sum_terms lambda_e(m - o) * d(term at m - o)/d(q at m)
    (no scatter, no atomics: every node writes only its own adjoint);
  * numpy versions of the forward RHS and of the same gather (forward() and adjoint() below), used by
    the tests as an independent check of the emitted code and of the term table against the oracle.

    python 3d-ns-fsi_b200/csrc/gen_rhs_adjoint.py      (rewrites nsf_rhs_adjoint.cuh)
"""
import itertools
import os

import numpy as np

VARS = ["RU", "RV", "RW", "RE", "u", "v", "w", "p", "T", "mu", "ka"]
VIDX = {v: q for q, v in enumerate(VARS)}
OFF = {"P": (0, 0, 0), "E": (1, 0, 0), "W": (-1, 0, 0), "N": (0, 1, 0), "S": (0, -1, 0), "U": (0, 0, 1),
       "D": (0, 0, -1)}


def off(name):
    o = [0, 0, 0]
    for ch in name:
        d = OFF[ch]
        o = [a + b for a, b in zip(o, d)]
    return tuple(o)


class Poly:
    """Polynomial in nodal quantities: {monomial: {constant-name tuple: float}}; a monomial is a sorted
    tuple of (variable, offset) factors."""

    def __init__(self, terms=None):
        self.t = terms or {}

    @staticmethod
    def var(v, o):
        return Poly({((v, off(o)),): {(): 1.0}})

    @staticmethod
    def const(name):
        return Poly({(): {(name,): 1.0}})

    @staticmethod
    def num(x):
        return Poly({(): {(): float(x)}})

    def __add__(self, other):
        out = {m: dict(c) for m, c in self.t.items()}
        for m, c in other.t.items():
            d = out.setdefault(m, {})
            for k, x in c.items():
                d[k] = d.get(k, 0.0) + x
        return Poly({m: {k: x for k, x in c.items() if x != 0.0} for m, c in out.items()})

    def __neg__(self):
        return Poly({m: {k: -x for k, x in c.items()} for m, c in self.t.items()})

    def __sub__(self, other):
        return self + (-other)

    def __mul__(self, other):
        out = Poly()
        for (m1, c1), (m2, c2) in itertools.product(self.t.items(), other.t.items()):
            m = tuple(sorted(m1 + m2))
            c = {}
            for (k1, x1), (k2, x2) in itertools.product(c1.items(), c2.items()):
                k = tuple(sorted(k1 + k2))
                c[k] = c.get(k, 0.0) + x1 * x2
            out = out + Poly({m: c})
        return out


def rhs_polys():
    """The five RHS equations (continuity, x/y/z momentum, energy), term by term in the reference's order."""
    V, K = Poly.var, Poly.const
    ax, ay, az = K("ax"), K("ay"), K("az")

    def visc_norm(c, q, a, b):  # c*((mu_a+mu_P)(q_a-q_P) - (mu_b+mu_P)(q_P-q_b))
        return K(c) * ((V("mu", a) + V("mu", "P")) * (V(q, a) - V(q, "P")) -
                       (V("mu", b) + V("mu", "P")) * (V(q, "P") - V(q, b)))

    def cross(c, m1, q, a1, b1, m2, a2, b2):  # c*(mu_m1 (q_a1 - q_b1) - mu_m2 (q_a2 - q_b2))
        return K(c) * (V("mu", m1) * (V(q, a1) - V(q, b1)) - V("mu", m2) * (V(q, a2) - V(q, b2)))

    eq = []
    eq.append(ax * (V("RU", "E") - V("RU", "W")) + ay * (V("RV", "N") - V("RV", "S")) +
              az * (V("RW", "U") - V("RW", "D")))
    # x momentum
    eq.append(ax * (V("RU", "E") * V("u", "E") + V("p", "E") - V("RU", "W") * V("u", "W") - V("p", "W")) +
              ay * (V("RU", "N") * V("v", "N") - V("RU", "S") * V("v", "S")) +
              az * (V("RU", "U") * V("w", "U") - V("RU", "D") * V("w", "D")) +
              visc_norm("xm_xx", "u", "E", "W") + visc_norm("xm_yy", "u", "N", "S") + visc_norm("xm_zz", "u", "U", "D") +
              cross("xm_xy", "N", "v", "EN", "WN", "S", "ES", "WS") + cross("xm_yx", "E", "v", "EN", "ES", "W", "WN", "WS") +
              cross("xm_xz", "U", "w", "EU", "WU", "D", "ED", "WD") + cross("xm_zx", "E", "w", "EU", "ED", "W", "WU", "WD"))
    # y momentum
    eq.append(ax * (V("RV", "E") * V("u", "E") - V("RV", "W") * V("u", "W")) +
              ay * (V("RV", "N") * V("v", "N") + V("p", "N") - V("RV", "S") * V("v", "S") - V("p", "S")) +
              az * (V("RV", "U") * V("w", "U") - V("RV", "D") * V("w", "D")) +
              visc_norm("ym_xx", "v", "E", "W") + visc_norm("ym_yy", "v", "N", "S") + visc_norm("ym_zz", "v", "U", "D") +
              cross("ym_yx", "E", "u", "EN", "ES", "W", "WN", "WS") + cross("ym_xy", "N", "u", "EN", "WN", "S", "ES", "WS") +
              cross("ym_yz", "U", "w", "NU", "SU", "D", "ND", "SD") + cross("ym_zy", "N", "w", "NU", "ND", "S", "SU", "SD"))
    # z momentum
    eq.append(ax * (V("RW", "E") * V("u", "E") - V("RW", "W") * V("u", "W")) +
              ay * (V("RW", "N") * V("v", "N") - V("RW", "S") * V("v", "S")) +
              az * (V("RW", "U") * V("w", "U") + V("p", "U") - V("RW", "D") * V("w", "D") - V("p", "D")) +
              visc_norm("zm_xx", "w", "E", "W") + visc_norm("zm_yy", "w", "N", "S") + visc_norm("zm_zz", "w", "U", "D") +
              cross("zm_zx", "E", "u", "EU", "ED", "W", "WU", "WD") + cross("zm_xz", "U", "u", "EU", "WU", "D", "ED", "WD") +
              cross("zm_zy", "N", "v", "NU", "ND", "S", "SU", "SD") + cross("zm_yz", "U", "v", "NU", "SU", "D", "ND", "SD"))
    # energy
    h0 = K("h0")

    def inv(c, vel, a, b):
        return K(c) * ((h0 + V("RE", a) + V("p", a)) * V(vel, a) - (h0 + V("RE", b) + V("p", b)) * V(vel, b))

    def vf(c, q, a, b):  # c*((mu_a q_a + mu_P q_P)(q_a - q_P) - (mu_b q_b + mu_P q_P)(q_P - q_b))
        return K(c) * ((V("mu", a) * V(q, a) + V("mu", "P") * V(q, "P")) * (V(q, a) - V(q, "P")) -
                       (V("mu", b) * V(q, b) + V("mu", "P") * V(q, "P")) * (V(q, "P") - V(q, b)))

    def vc(c, m1, f1, q, a1, b1, m2, f2, a2, b2):  # c*(mu_m1 f_m1 (q_a1-q_b1) - mu_m2 f_m2 (q_a2-q_b2))
        return K(c) * (V("mu", m1) * V(f1, m1) * (V(q, a1) - V(q, b1)) -
                       V("mu", m2) * V(f2, m2) * (V(q, a2) - V(q, b2)))

    def hf(c, a, b):
        return K(c) * ((V("ka", a) + V("ka", "P")) * (V("T", a) - V("T", "P")) -
                       (V("ka", b) + V("ka", "P")) * (V("T", "P") - V("T", b)))

    e = (inv("ax", "u", "E", "W") + inv("ay", "v", "N", "S") + inv("az", "w", "U", "D") +
         vf("e_xx23", "u", "E", "W") + vf("e_xx12", "v", "E", "W") + vf("e_xx12", "w", "E", "W") +
         vc("e_yx6", "E", "u", "v", "EN", "ES", "W", "u", "WN", "WS") +
         vc("e_zx6", "E", "u", "w", "EU", "ED", "W", "u", "WU", "WD") +
         vc("e_yx4", "E", "v", "u", "EN", "ES", "W", "v", "WN", "WS") +
         vc("e_zx4", "E", "w", "u", "EU", "ED", "W", "w", "WU", "WD") +
         vf("e_yy12", "u", "N", "S") + vf("e_yy23", "v", "N", "S") + vf("e_yy12", "w", "N", "S") +
         vc("e_yx6", "N", "v", "u", "EN", "WN", "S", "v", "ES", "WS") +
         vc("e_zy6", "N", "v", "w", "NU", "ND", "S", "v", "SU", "SD") +
         vc("e_yx4", "N", "u", "v", "EN", "WN", "S", "u", "ES", "WS") +
         vc("e_zy4", "N", "w", "v", "NU", "ND", "S", "w", "SU", "SD") +
         vf("e_zz12", "u", "U", "D") + vf("e_zz12", "v", "U", "D") + vf("e_zz23", "w", "U", "D") +
         vc("e_zx6", "U", "w", "u", "EU", "WU", "D", "w", "ED", "WD") +
         vc("e_zy6", "U", "w", "v", "NU", "SU", "D", "w", "ND", "SD") +
         vc("e_zx4", "U", "u", "w", "EU", "WU", "D", "u", "ED", "WD") +
         vc("e_zy4", "U", "v", "w", "NU", "SU", "D", "v", "ND", "SD") +
         hf("e_xx12", "E", "W") + hf("e_yy12", "N", "S") + hf("e_zz12", "U", "D"))
    eq.append(e)
    return eq


def adjoint_terms(eqs):
    """[(e, o, q, coef, others)]: lambda_e(m - o) * coef * prod(others at m - o + o') adds to qbar(m)."""
    out = []
    for e, poly in enumerate(eqs):
        for mono, coef in poly.t.items():
            if not mono or not coef:
                continue
            for f, (q, o) in enumerate(mono):
                others = mono[:f] + mono[f + 1:]
                out.append((e, o, q, coef, others))
    return out


# ------------------------------------------------------------------------------------------ numpy
def _shift(a, o):
    """b[X] = a[X + o] (zero outside the grid)."""
    b = np.zeros_like(a)
    src = tuple(slice(max(0, d), a.shape[ax] + min(0, d)) for ax, d in enumerate(o))
    dst = tuple(slice(max(0, -d), a.shape[ax] + min(0, -d)) for ax, d in enumerate(o))
    b[dst] = a[src]
    return b


def _coef_value(coef, C):
    return sum(x * np.prod([C[n] for n in k]) if k else x for k, x in coef.items())


def forward(eqs, fields, C):
    """RHS of every node from the term table (fields: dict var -> (NI, NJ, NK) array); valid where the
    whole stencil lies inside the grid."""
    out = []
    for poly in eqs:
        r = 0.0
        for mono, coef in poly.t.items():
            t = _coef_value(coef, C)
            for q, o in mono:
                t = t * _shift(fields[q], o)
            r = r + t
        out.append(r)
    return out


def adjoint(terms, fields, lam, C):
    """Gather of the input adjoints (dict var -> array) from lam[e] (zero where no RHS is taken)."""
    bar = {q: np.zeros_like(fields["u"]) for q in VARS}
    for e, o, q, coef, others in terms:
        mo = tuple(-x for x in o)
        t = _coef_value(coef, C) * _shift(lam[e], mo)
        for q2, o2 in others:
            t = t * _shift(fields[q2], tuple(a + b for a, b in zip(mo, o2)))
        bar[q] = bar[q] + t
    return bar


# ------------------------------------------------------------------------------------------- CUDA
def _coef_expr(coef):
    cs = []
    for k, x in sorted(coef.items()):
        c = " * ".join(["C.%s" % n for n in k]) if k else ""
        if x == 1.0:
            cs.append(c or "1.0")
        elif x == -1.0:
            cs.append("-" + (c or "1.0"))
        else:
            cs.append(("%r * " % x) + c if c else "%r" % x)
    return "(" + " + ".join(cs) + ")" if len(cs) > 1 else cs[0]


SUB_VALUES = 64  # most input values one block reads (64: one block per RHS node, which measured fastest)


def emit_cuda(terms):
    lines = []
    w = lines.append
    w("// Generated by gen_rhs_adjoint.py from the RHS term table: do not edit. The transposed stencil of the")
    w("// right-hand side (Solver.cpp:181-418) in gather form: rhs_adjoint_gather(...) returns, for node")
    w("// X = (i, j, k), the adjoint of each input quantity (RU, RV, RW, RE, u, v, w, p, T, mu, ka) summed over")
    w("// every interior node whose RHS reads it. lam(e, di, dj, dk): RHS adjoint of equation e at node")
    w("// (i+di, j+dj, k+dk) (zero where no RHS is taken); val(q, di, dj, dk): input quantity q there (offsets")
    w("// within one node of X: the 7-point stencil for u, v, w, T, mu, ka, X itself for the others);")
    w("// inner(di, dj, dk): the node (i-di, j-dj, k-dk) is one whose RHS was taken (its whole stencil then")
    w("// lies inside the grid). All offsets are literals, so a caller's index arithmetic folds. The terms of")
    w("// one RHS node are grouped by equation and, within an equation, by coefficient.")
    w("#ifndef NSF_RHS_ADJOINT_CUH")
    w("#define NSF_RHS_ADJOINT_CUH")
    w("")
    w("namespace nsf {")
    w("")
    w("template <class Lam, class Val, class Inner>")
    w("__device__ __forceinline__ void rhs_adjoint_gather(const Consts& C, const Lam& lam, const Val& val,")
    w("                                                   const Inner& inner, double bar[%d]) {" % len(VARS))
    w("  for (int q = 0; q < %d; ++q) bar[q] = 0.0;" % len(VARS))
    rel = sorted({(q, tuple(o2[a] - t[1][a] for a in range(3))) for t in terms for (q, o2) in t[4]},
                 key=lambda x: (x[1], VIDX[x[0]]))
    names = {x: "w%d" % n for n, x in enumerate(rel)}
    by_o = {}
    for t in terms:
        by_o.setdefault(t[1], []).append(t)
    for o in sorted(by_o, key=lambda o: (sum(map(abs, o)), o)):
        def rel_of(others):
            return {(q2, tuple(o2[a] - o[a] for a in range(3))) for q2, o2 in others}

        # outputs grouped so that no group reads more than SUB_VALUES input values: each group is a block
        # of its own (the RHS node's values are then never all live at once)
        used = {}
        for _, _, q, _, others in by_o[o]:
            used.setdefault(q, set()).update(rel_of(others))
        groups = []
        for q in sorted(used, key=lambda q: -len(used[q])):
            for g in groups:
                if len(g[1] | used[q]) <= SUB_VALUES:
                    g[0].append(q)
                    g[1] |= used[q]
                    break
            else:
                groups.append([[q], set(used[q])])
        for outs, vals in groups:
            # a compiler fence per block: each block loads its own values (a value shared by several blocks
            # would otherwise stay in a register from its first to its last use, and with all of them live
            # the kernel runs out of registers)
            w("  asm volatile(\"\" ::: \"memory\");")
            w("  if (inner(%d, %d, %d)) {" % o)
            for e in sorted({t[0] for t in by_o[o] if t[2] in outs}):
                w("    const double l%d = lam(%d, %d, %d, %d);" % (e, e, -o[0], -o[1], -o[2]))
            for q, a in sorted(vals, key=lambda x: (x[1], VIDX[x[0]])):
                w("    const double %s = val(%d, %d, %d, %d);  // %s %s" % (names[(q, a)], VIDX[q], *a, q, a))
            for q in VARS:
                if q not in outs:
                    continue
                # per equation, the terms grouped by coefficient (one multiplication by it per group), and
                # within a group a value shared by every product factored out
                by_e = {}
                for e, _, qq, coef, others in by_o[o]:
                    if qq != q:
                        continue
                    factors = [names[(q2, tuple(o2[a] - o[a] for a in range(3)))] for q2, o2 in others]
                    by_e.setdefault(e, {}).setdefault(tuple(sorted(coef.items())), []).append(factors)
                parts = []
                for e, by_c in sorted(by_e.items()):
                    sums = []
                    for ckey, prods in sorted(by_c.items()):
                        cexpr = _coef_expr(dict(ckey))
                        common = set(prods[0])
                        for f in prods[1:]:
                            common &= set(f)
                        shared = sorted(common)[0] if common and len(prods) > 1 else None
                        if shared:
                            rest = []
                            for f in prods:
                                g = list(f)
                                g.remove(shared)
                                rest.append(" * ".join(g) if g else "1.0")
                            inner = " + ".join(rest)
                            sums.append("%s * %s * (%s)" % (cexpr, shared, inner))
                        else:
                            inner = " + ".join(" * ".join(f) if f else "1.0" for f in prods)
                            sums.append("%s * (%s)" % (cexpr, inner) if len(prods) > 1 or prods[0] else cexpr)
                    sums = [s.replace(" * (1.0)", "") for s in sums]
                    parts.append("l%d * (%s)" % (e, " + ".join(sums)) if len(sums) > 1 else "l%d * %s" % (e, sums[0]))
                w("    bar[%d] += %s;  // %s" % (VIDX[q], " + ".join(parts), q))
            w("  }")
    w("}")
    w("")
    w("}  // namespace nsf")
    w("#endif")
    return "\n".join(lines) + "\n"


def main():
    eqs = rhs_polys()
    terms = adjoint_terms(eqs)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "nsf_rhs_adjoint.cuh")
    with open(path, "w") as f:
        f.write(emit_cuda(terms))
    nmono = sum(len(p.t) for p in eqs)
    print("%s: %d monomials, %d adjoint terms, %d lambda offsets" % (path, nmono, len(terms),
                                                                     len({t[1] for t in terms})))


if __name__ == "__main__":
    main()
