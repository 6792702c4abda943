"""Seeded random cases for the sweep tests (tests/test_oracle_sweep_cpu.py, tests/test_parity_sweep_gpu.py).

random_case(seed) draws a grid, one boundary type per axis (inlet/outlet, periodic, symmetry or outlet
pairs in x; periodic, symmetry or outlet in y; periodic or symmetry in z), 0-2 spheres or a z-cylinder kept
clear of the faces, Mach and Reynolds numbers, a filter interval and an initial condition (every sixth
case a fully periodic Taylor-Green box), and returns the case file's text.
"""
import numpy as np

N_CASES = 32  # cases each sweep runs
STEPS = 8

COMMON = """stopCriterion = "timesteps"
t_end = 200.
convStabilityLimit = 0.5
viscStabilityLimit = -0.68
filterIntervalChangeTimes = []
statusReportInterval = 2.
saveDensity = true
saveMomentum = false
saveEnergy = false
saveVelocity = true
savePressure = true
saveTemperature = true
saveViscosity = false
saveThermalCond = false
saveIC = false
saveFinal = false
saveIntervals = false
savePeriod = 5.
saveIntervalsStartTime = 0.
saveIntervalsEndTime = 0.
saveConvergenceHistory = "all"
Gamma = 1.4
Pr = 0.71
R = 287.
sutherlands_C1 = 1.458E-6
sutherlands_C2 = 110.4
T_0 = 300.
"""


def spacing(bc, n, L):
    """Grid spacing of one axis from its min-face boundary type (Mesh.cpp:44-49)."""
    return L / (n - 2) if bc == "periodic" else L / (n - 3) if bc == "symmetry" else L / (n - 1)


def random_case(seed):
    """The text of one seeded case file."""
    rng = np.random.default_rng(seed)
    bx = [("inlet", "outlet"), ("periodic", "periodic"), ("symmetry", "symmetry"), ("outlet", "outlet")][rng.integers(4)]
    by = [("periodic", "periodic"), ("symmetry", "symmetry"), ("outlet", "outlet")][rng.integers(3)]
    bz = [("periodic", "periodic"), ("symmetry", "symmetry")][rng.integers(2)]
    tgv = seed % 6 == 5  # every sixth case: a fully periodic box with the Taylor-Green initial condition
    if tgv:
        bx = by = bz = ("periodic", "periodic")
    L = [float(rng.uniform(1.2, 2.0)), float(rng.uniform(0.8, 1.2)), float(rng.uniform(0.8, 1.2))]
    bodies = int(rng.integers(4))  # 0: none, 1-2: spheres, 3: a z-cylinder
    if bodies:
        n = [int(rng.integers(22, 30)), int(rng.integers(16, 22)), int(rng.integers(14, 20))]
    else:
        n = [int(rng.integers(10, 22)), int(rng.integers(8, 16)), int(rng.integers(5, 14))]
    d = [spacing(b[0], nn, LL) for b, nn, LL in zip((bx, by, bz), n, L)]
    shapes = ""
    if bodies in (1, 2):
        spheres = []
        for _ in range(200):
            if len(spheres) == bodies:
                break
            r = float(rng.uniform(2.5, 3.5)) * max(d)
            if min(L[a] - 2 * (r + 4 * d[a]) for a in (1, 2)) <= 0:
                continue
            c = [float(rng.uniform(0.3, 0.7)) * L[0]] + [float(rng.uniform(r + 4 * d[a], L[a] - r - 4 * d[a]))
                                                          for a in (1, 2)]
            if all(np.linalg.norm(np.subtract(c, s[:3])) > r + s[3] + 4 * max(d) for s in spheres):
                spheres.append(c + [r])
        shapes = "  spheres = ( %s );\n" % ", ".join("(%.6f, %.6f, %.6f, %.6f)" % tuple(s) for s in spheres)
    elif bodies == 3:
        r = min(float(rng.uniform(2.5, 3.5)) * max(d[0], d[1]), 0.5 * L[1] - 4.5 * d[1])
        c = [float(rng.uniform(0.35, 0.6)) * L[0], float(rng.uniform(r + 4 * d[1], L[1] - r - 4 * d[1])), 0.5 * L[2]]
        shapes = '  cylinders = ( ("z", %.6f, %.6f, %.6f, %.6f) );\n' % (c[0], c[1], c[2], r)
    M0 = float(rng.uniform(0.1, 0.4))
    ic = "tgv" if tgv else "freestream_noise"
    text = "NI = %d\nNJ = %d\nNK = %d\nstopTimeLevel = %d\nfilterIntervals = [%d]\n" % (
        n[0], n[1], n[2], STEPS, int(rng.integers(3, 7)))
    text += COMMON
    text += "Re = %.6f\nM_0 = %.6f\nL_x = %.6f\nL_y = %.6f\nL_z = %.6f\n" % (
        float(rng.uniform(200, 2000)), M0, L[0], L[1], L[2])
    text += "case = {\n  kind = \"custom\";\n"
    for ax, b in zip("xyz", (bx, by, bz)):
        text += '  bc_%s_min = "%s";\n  bc_%s_max = "%s";\n' % (ax, b[0], ax, b[1])
    text += shapes
    text += '  ic = "%s";\n  noise_amp = 1e-3;\n  seed = %dL;\n};\n' % (ic, 1000 + seed)
    return text


def wide_case(seed, dt0=None):
    """A second family (oracle against the reference only): cylinders along any periodic axis, a stagnation
    start behind an inlet, up to three filter intervals with change times, and every other case stopped by
    end_time, whose last step the reference shortens to land on t_end. Change times and t_end are set in
    units of the case's first dt: call once with dt0=None (placeholders) to read dt0, then with it."""
    rng = np.random.default_rng(10_000 + seed)
    bx = [("inlet", "outlet"), ("periodic", "periodic"), ("symmetry", "symmetry"), ("inlet", "outlet")][rng.integers(4)]
    by = [("periodic", "periodic"), ("symmetry", "symmetry"), ("outlet", "outlet")][rng.integers(3)]
    bz = [("periodic", "periodic"), ("symmetry", "symmetry")][rng.integers(2)]
    L = [float(rng.uniform(1.2, 2.0)), float(rng.uniform(0.8, 1.2)), float(rng.uniform(0.8, 1.2))]
    n = [int(rng.integers(22, 30)), int(rng.integers(16, 22)), int(rng.integers(14, 20))]
    d = [spacing(b[0], nn, LL) for b, nn, LL in zip((bx, by, bz), n, L)]
    shapes = ""
    periodic = [a for a, b in enumerate((bx, by, bz)) if b[0] == "periodic"]
    if periodic and rng.integers(2):
        ax = int(periodic[rng.integers(len(periodic))])
        o1, o2 = [a for a in range(3) if a != ax]
        r = float(rng.uniform(2.5, 3.5)) * max(d[o1], d[o2])
        r = min(r, 0.5 * L[o1] - 4.5 * d[o1], 0.5 * L[o2] - 4.5 * d[o2])
        c = [0.5 * L[0], 0.5 * L[1], 0.5 * L[2]]
        for a in (o1, o2):
            lo, hi = (0.35 * L[0], 0.6 * L[0]) if a == 0 else (r + 4 * d[a], L[a] - r - 4 * d[a])
            c[a] = float(rng.uniform(lo, hi))
        shapes = '  cylinders = ( ("%s", %.6f, %.6f, %.6f, %.6f) );\n' % ("xyz"[ax], c[0], c[1], c[2], r)
    elif rng.integers(2):
        r = min(float(rng.uniform(2.5, 3.5)) * max(d), min(0.5 * L[a] - 4.5 * d[a] for a in (1, 2)))
        c = [float(rng.uniform(0.35, 0.6)) * L[0]] + [float(rng.uniform(r + 4 * d[a], L[a] - r - 4 * d[a])) for a in (1, 2)]
        shapes = "  spheres = ( (%.6f, %.6f, %.6f, %.6f) );\n" % (c[0], c[1], c[2], r)
    ic = "stagnation" if bx[0] == "inlet" and rng.integers(2) else "freestream_noise"
    nf = int(rng.integers(1, 4))
    intervals = [int(rng.integers(2, 6)) for _ in range(nf)]
    end_time = seed % 2 == 1
    unit = dt0 if dt0 else 1.0
    changes = ", ".join(repr((2.5 + 2 * q) * unit) for q in range(nf - 1))  # floats in the config grammar
    text = "NI = %d\nNJ = %d\nNK = %d\nstopTimeLevel = %d\nfilterIntervals = [%s]\n" % (
        n[0], n[1], n[2], STEPS, ", ".join(map(str, intervals)))
    common = COMMON.replace("filterIntervalChangeTimes = []", "filterIntervalChangeTimes = [%s]" % changes)
    if end_time:
        common = common.replace('stopCriterion = "timesteps"', 'stopCriterion = "end_time"')
        common = common.replace("t_end = 200.", "t_end = " + repr(5.5 * unit if dt0 else 200.0))
    text += common
    text += "Re = %.6f\nM_0 = %.6f\nL_x = %.6f\nL_y = %.6f\nL_z = %.6f\n" % (
        float(rng.uniform(200, 2000)), float(rng.uniform(0.1, 0.4)), L[0], L[1], L[2])
    text += "case = {\n  kind = \"custom\";\n"
    for ax, b in zip("xyz", (bx, by, bz)):
        text += '  bc_%s_min = "%s";\n  bc_%s_max = "%s";\n' % (ax, b[0], ax, b[1])
    text += shapes
    text += '  ic = "%s";\n  noise_amp = 1e-3;\n  seed = %dL;\n};\n' % (ic, 2000 + seed)
    return text


def shipped_case(seed, dt0=None):
    """The reference's own default case (kind "shipped": Solver::initialize unchanged — inlet/outlet x,
    symmetry y, periodic z, its cylinder, stagnation start, end_time stop) with seeded grid, box, flow
    and filter settings. t_end and the filter change times are in units of the first dt (see wide_case)."""
    rng = np.random.default_rng(20_000 + seed)
    unit = dt0 if dt0 else 1.0
    nf = int(rng.integers(1, 4))
    text = "NI = %d\nNJ = %d\nNK = %d\n" % (int(rng.integers(30, 60)), int(rng.integers(16, 32)),
                                            int(rng.integers(3, 7)))
    text += 'stopCriterion = "end_time"\nstopTimeLevel = 20\nt_end = %s\n' % repr(7.5 * unit if dt0 else 200.0)
    text += "convStabilityLimit = %s\nviscStabilityLimit = -0.68\n" % repr(float(rng.uniform(0.5, 0.9)))
    text += "filterIntervals = [%s]\nfilterIntervalChangeTimes = [%s]\n" % (
        ", ".join(str(int(rng.integers(2, 6))) for _ in range(nf)),
        ", ".join(repr((2.5 + 2 * q) * unit) for q in range(nf - 1)))
    text += COMMON[COMMON.index("statusReportInterval"):].replace("Pr = 0.71", "Pr = %s" % repr(
        float(rng.uniform(0.65, 0.75))))
    text += "Re = %s\nM_0 = %s\nL_x = %s\nL_y = %s\nL_z = %s\n" % (
        repr(float(rng.uniform(100, 1000))), repr(float(rng.uniform(0.1, 0.4))), repr(float(rng.uniform(1.5, 3.0))),
        repr(float(rng.uniform(0.8, 1.5))), repr(float(rng.uniform(0.03, 0.1))))
    text += 'case = {\n  kind = "shipped";\n};\n'
    return text


def ensemble_member_text(c, steps):
    """The case file of one member of the batched-ensemble workload (nsfsi.ensemble_configs, built there from
    the 48^3 sphere case) with `steps` RK4 steps."""
    import re
    import nsfsi
    text = open(nsfsi.case_path("sphere48")).read()
    sp = c.spheres[0]
    for key, val in (("NI", str(c.NI)), ("NJ", str(c.NJ)), ("NK", str(c.NK)), ("stopTimeLevel", str(steps)),
                     ("L_x", repr(c.lx)), ("L_y", repr(c.ly)), ("L_z", repr(c.lz)), ("M_0", repr(c.m0)),
                     ("Re", repr(c.re))):
        text, n = re.subn(r"^%s = .*$" % key, "%s = %s" % (key, val), text, flags=re.M)
        assert n == 1, key
    text, n = re.subn(r"spheres = .*;", "spheres = ( (%r, %r, %r, %r) );" % (sp.cx, sp.cy, sp.cz, sp.r), text)
    assert n == 1
    text, n = re.subn(r"seed = .*;", "seed = %dL;" % c.seed, text)
    assert n == 1
    return text
