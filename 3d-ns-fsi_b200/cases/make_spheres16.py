"""Writes cases/spheres16.cfg: the ghost-node-heavy workload (256 x 128 x 128 nodes on [0,2]x[0,1]x[0,1],
16 static spheres, inflow/outflow in x, periodic in y and z, freestream Mach 0.3 with +-1e-4 noise).

Radii are drawn from U[0.03, 0.06] and centres by seeded rejection sampling with x in [0.3, 1.5] and y, z
kept at least r + 5 dy from the faces (the reference's sphere bounding box is never clamped, so a body must
not reach a face). Two spheres keep a surface gap of at least 6 grid spacings, so their ghost, filter and
image-point cells never meet. Re = 200 on the mean diameter, converted to the reference's Re per unit length
at the stagnation state: Re_ref = Re_D / (M0 * D_mean).

    python 3d-ns-fsi_b200/cases/make_spheres16.py
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SEED = 20240216
NI, NJ, NK = 256, 128, 128
LX, LY, LZ = 2.0, 1.0, 1.0
M0, RE_D = 0.3, 200.0


def draw():
    rng = np.random.default_rng(SEED)
    dx, dy, dz = LX / (NI - 1), LY / (NJ - 2), LZ / (NK - 2)
    dmax = max(dx, dy, dz)
    spheres = []
    while len(spheres) < 16:
        r = rng.uniform(0.03, 0.06)
        c = np.array([rng.uniform(0.3, 1.5), rng.uniform(r + 5 * dy, LY - r - 5 * dy),
                      rng.uniform(r + 5 * dz, LZ - r - 5 * dz)])
        if all(np.linalg.norm(c - np.array(s[:3])) >= r + s[3] + 6 * dmax for s in spheres):
            spheres.append((float(c[0]), float(c[1]), float(c[2]), float(r)))
    return spheres


def main():
    spheres = draw()
    d_mean = 2 * np.mean([s[3] for s in spheres])
    re_ref = RE_D / (M0 * d_mean)
    base = open(os.path.join(HERE, "sphere48.cfg")).read().split("case = {")[0]
    repl = {"NI = 48": "NI = %d" % NI, "NJ = 48": "NJ = %d" % NJ, "NK = 48": "NK = %d" % NK,
            "stopTimeLevel = 100": "stopTimeLevel = 500", "Re = 1666.6666666666667": "Re = %r" % float(re_ref),
            "L_x = 1.": "L_x = 2."}
    for a, b in repl.items():
        assert a in base, a
        base = base.replace(a, b)
    body = ",\n              ".join("(%r, %r, %r, %r)" % s for s in spheres)
    text = base + """case = {
  kind = "custom";
  bc_x_min = "inlet";
  bc_x_max = "outlet";
  bc_y_min = "periodic";
  bc_y_max = "periodic";
  bc_z_min = "periodic";
  bc_z_max = "periodic";
  spheres = ( %s );
  ic = "freestream_noise";
  noise_amp = 1e-4;
  seed = %dL;
};
""" % (body, SEED)
    with open(os.path.join(HERE, "spheres16.cfg"), "w") as f:
        f.write(text)
    print("spheres16.cfg: Re_ref = %.6f, mean D = %.6f" % (re_ref, d_mean))


if __name__ == "__main__":
    main()
