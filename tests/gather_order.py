"""Pure-Python restatement of the CUDA serial-order gather
(k_force_serial / k_theta_serial in peridyn_b200/csrc/pd_exact.cu).

Used on the CPU to show that replaying, per particle, the order in which
the reference's serial scatter loop (general_material.jl:330-368) touches
f_p reproduces its result bit for bit:
    A. neighbours q < p, ascending   (terms added from q's loop)
    B. all neighbours, descending    (p's own loop)
    C. neighbours q > p, ascending   (terms from q's loop)
Python floats are IEEE doubles with unfused arithmetic, like the kernel
compiled with -fmad=false.
"""
import math

import numpy as np


def _mag(a, b, c):
    return math.sqrt(a * a + b * b + c * c)


def gather_force(kind, x, y, family, intact, type_rel, cs, density, vol, c, m=None, theta=None, K=None, G=None):
    """Returns (f 3xn, intact_after) for one block, f starting at zero."""
    M, n = family.shape
    f = np.zeros((3, n), order="F")
    new_intact = intact.copy()
    c11 = float(c.reshape(-1, order="F")[0]) if kind == 0 else 0.0

    def term(p, q):
        X = (x[0, q] - x[0, p], x[1, q] - x[1, p], x[2, q] - x[2, p])
        Y = (y[0, q] - y[0, p], y[1, q] - y[1, p], y[2, q] - y[2, p])
        yij = _mag(*Y)
        xij = _mag(*X)
        ext = yij - xij
        s = ext / xij
        tp, tq = type_rel[p] - 1, type_rel[q] - 1
        if not (s < cs[tp, tq]):
            return None
        if kind == 0:
            t = s * c11
        else:
            k35 = 3 * K[tp, tq] - 5 * G[tp, tq]
            g15 = 15 * G[tp, tq]
            w = 1.0 / xij
            a = w / m[p]
            b = w / m[q]
            t = k35 * (theta[p] * xij * a + theta[q] * xij * b) + g15 * ext * (a + b)
        xx = 0.5 * t / yij
        rho = density[tp]
        return (xx * Y[0] * vol[q] / rho, xx * Y[1] * vol[q] / rho, xx * Y[2] * vol[q] / rho)

    for p in range(n):
        nb = [(k, family[k, p] - 1) for k in range(M) if family[k, p] > 0]
        fx = fy = fz = 0.0
        # A
        kc = len(nb) - 1
        while kc >= 0 and nb[kc][1] < p:
            k, q = nb[kc]
            if intact[k, p]:
                t = term(p, q)
                if t is not None:
                    fx, fy, fz = fx + t[0], fy + t[1], fz + t[2]
            kc -= 1
        # B
        for k, q in nb:
            if intact[k, p]:
                t = term(p, q)
                if t is not None:
                    fx, fy, fz = fx + t[0], fy + t[1], fz + t[2]
                else:
                    new_intact[k, p] = False
        # C
        for idx in range(kc, -1, -1):
            k, q = nb[idx]
            if intact[k, p]:
                t = term(p, q)
                if t is not None:
                    fx, fy, fz = fx + t[0], fy + t[1], fz + t[2]
        f[0, p], f[1, p], f[2, p] = fx, fy, fz
    return f, new_intact


def gather_theta(x, y, family, intact, vol, m):
    """k_theta_serial: theta_p over p's own family, stored order."""
    M, n = family.shape
    th = np.zeros(n)
    for p in range(n):
        c_i = 3.0 / m[p]
        acc = 0.0
        for k in range(M):
            if family[k, p] > 0 and intact[k, p]:
                q = family[k, p] - 1
                xij = _mag(x[0, q] - x[0, p], x[1, q] - x[1, p], x[2, q] - x[2, p])
                yij = _mag(y[0, q] - y[0, p], y[1, q] - y[1, p], y[2, q] - y[2, p])
                e = yij - xij
                w = 1.0 / xij
                acc = acc + c_i * w * xij * e * vol[q]
        th[p] = acc
    return th
