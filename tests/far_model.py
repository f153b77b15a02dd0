"""Restatement, in numpy (FP64), of the fast walk's far-cell expansion
(FarExp in pot_b200/csrc/pot_walk_fast.cu): the field of monopoles far from
a target group, expanded once about the group's centre c and evaluated at
each target's offset delta from c.  Test infrastructure: it pins the
expansion's components and the error bound the walk relies on, not the CUDA
code.

For a monopole of charge q at s and d = c - s, r = |d|, w = q / r^3:
  E_a   = w d_a
  J_ab  = w (delta_ab - 3 d_a d_b / r^2)
  H_abc = w / r^2 (15 d_a d_b d_c / r^2 - 3 (delta_ab d_c + delta_ac d_b + delta_bc d_a))
J keeps 5 components and H 7; the others follow from tracelessness.  The
field at c + delta is E + J delta + H delta delta / 2."""
import numpy as np

COMPONENTS = ("ex", "ey", "ez", "jxx", "jyy", "jxy", "jxz", "jyz",
              "hxxx", "hyyy", "hxxy", "hxxz", "hxyy", "hyyz", "hxyz")


def expansion(c, sources):
    """The 15 accumulated components for monopoles sources[k] = (x, y, z, q)
    about c, in the kernel's expressions (FarExp::add)."""
    acc = dict.fromkeys(COMPONENTS, 0.0)
    for sx, sy, sz, q in sources:
        dx, dy, dz = c[0] - sx, c[1] - sy, c[2] - sz
        r2 = dx * dx + dy * dy + dz * dz
        ri = 1.0 / np.sqrt(r2)
        ri2 = ri * ri
        w = q * ri2 * ri
        acc["ex"] += w * dx
        acc["ey"] += w * dy
        acc["ez"] += w * dz
        w3 = -3.0 * w * ri2
        acc["jxx"] += w3 * dx * dx + w
        acc["jyy"] += w3 * dy * dy + w
        acc["jxy"] += w3 * dx * dy
        acc["jxz"] += w3 * dx * dz
        acc["jyz"] += w3 * dy * dz
        v3 = w3
        v15 = -5.0 * w3 * ri2
        acc["hxxx"] += dx * (v15 * dx * dx + 3.0 * v3)
        acc["hyyy"] += dy * (v15 * dy * dy + 3.0 * v3)
        acc["hxxy"] += dy * (v15 * dx * dx + v3)
        acc["hxxz"] += dz * (v15 * dx * dx + v3)
        acc["hxyy"] += dx * (v15 * dy * dy + v3)
        acc["hyyz"] += dz * (v15 * dy * dy + v3)
        acc["hxyz"] += v15 * dx * dy * dz
    return acc


def evaluate(acc, delta):
    """The expansion's field at c + delta (FarExp::at)."""
    x, y, z = delta
    jzz = -acc["jxx"] - acc["jyy"]
    hxzz = -acc["hxxx"] - acc["hxyy"]
    hyzz = -acc["hxxy"] - acc["hyyy"]
    hzzz = -acc["hxxz"] - acc["hyyz"]
    xx, yy, zz, xy, xz, yz = 0.5 * x * x, 0.5 * y * y, 0.5 * z * z, x * y, x * z, y * z
    a = acc
    ex = (a["ex"] + a["jxx"] * x + a["jxy"] * y + a["jxz"] * z + a["hxxx"] * xx + a["hxyy"] * yy + hxzz * zz
          + a["hxxy"] * xy + a["hxxz"] * xz + a["hxyz"] * yz)
    ey = (a["ey"] + a["jxy"] * x + a["jyy"] * y + a["jyz"] * z + a["hxxy"] * xx + a["hyyy"] * yy + hyzz * zz
          + a["hxyy"] * xy + a["hxyz"] * xz + a["hyyz"] * yz)
    ez = (a["ez"] + a["jxz"] * x + a["jyz"] * y + jzz * z + a["hxxz"] * xx + a["hyyz"] * yy + hzzz * zz
          + a["hxyz"] * xy + hxzz * xz + hyzz * yz)
    return np.array([ex, ey, ez])


def direct(target, sources):
    """The exact field q (t - s) / |t - s|^3 summed over the sources."""
    e = np.zeros(3)
    for sx, sy, sz, q in sources:
        d = np.array([target[0] - sx, target[1] - sy, target[2] - sz])
        e += q * d / np.linalg.norm(d) ** 3
    return e
