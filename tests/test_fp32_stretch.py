"""Why the FP32-compensated mode computes the bond stretch the way it does,
checked on the CPU in numpy float32.

The throughput walk (pd_fast.cu, Kin<float>) forms the reference bond
xi = x_q - x_p and the displacement difference eta = u_q - u_p in FP32 (from
records holding x relative to the block centre and u, the displacement,
whose FP64 copy is the position accumulator) and the stretch as

    s = eta . (xi + Y) / ((|Y| + |xi|) |xi|),   Y = xi + eta,

whose numerator is |Y|^2 - |xi|^2 without the subtraction of two nearly
equal squares.  The reference's own expression, s = (|Y| - |xi|) / |xi|
(general_material.jl:340-341), evaluated in FP32 on absolute positions,
loses the stretch to cancellation at the small strains a bond carries
before it breaks (critical stretches 0.002-0.01).
"""
import numpy as np


def _bonds(rng, n, strain):
    xi = rng.normal(size=(n, 3))
    xi *= (rng.uniform(1.0e-3, 3.015e-3, size=n) / np.linalg.norm(xi, axis=1))[:, None]
    eta = rng.normal(size=(n, 3)) * (strain * np.linalg.norm(xi, axis=1))[:, None]
    return xi, eta


def _stretch64(xi, eta):
    lx = np.linalg.norm(xi, axis=1)
    num = (eta * (2.0 * xi + eta)).sum(axis=1)
    return num / ((np.linalg.norm(xi + eta, axis=1) + lx) * lx)


def _stretch32_compensated(xi, eta):
    d, e = xi.astype(np.float32), eta.astype(np.float32)
    Y = d + e
    num = (e * (d + Y)).sum(axis=1, dtype=np.float32)
    xx2 = (d * d).sum(axis=1, dtype=np.float32)
    lx = np.sqrt(xx2)
    ly = np.sqrt(xx2 + num)
    return num / ((ly + lx) * lx)


def _stretch32_positions(x_p, xi, eta, u_p):
    # the reference's form on FP32 absolute positions y = x + u
    yp = (x_p + u_p).astype(np.float32)
    yq = (x_p + xi + u_p + eta).astype(np.float32)
    xp32, xq32 = x_p.astype(np.float32), (x_p + xi).astype(np.float32)
    lx = np.linalg.norm(xq32 - xp32, axis=1).astype(np.float32)
    ly = np.linalg.norm(yq - yp, axis=1).astype(np.float32)
    return (ly - lx) / lx


def _strain_scale(xi, eta):
    # |eta| / |xi|: the size of the strain a bond carries; the stretch error
    # is measured against it (the stretch itself passes through zero when
    # eta is nearly perpendicular to xi)
    return np.linalg.norm(eta, axis=1) / np.linalg.norm(xi, axis=1)


def test_compensated_stretch_keeps_fp32_precision_at_small_strains():
    rng = np.random.default_rng(11)
    for strain in (1e-6, 1e-4, 1e-3, 1e-2):
        xi, eta = _bonds(rng, 20000, strain)
        err = np.abs(_stretch32_compensated(xi, eta).astype(np.float64) - _stretch64(xi, eta))
        err /= _strain_scale(xi, eta)
        # a few FP32 ulps of the strain, whatever its size (measured: median
        # 3e-8, largest 4e-7 of the strain)
        assert err.max() < 1e-6, (strain, err.max())


def test_reference_form_in_fp32_loses_small_strains():
    rng = np.random.default_rng(12)
    # a particle 2.5 cm from the block centre, displaced by 10 um: the
    # magnitudes a 50 mm specimen reaches
    xi, eta = _bonds(rng, 20000, 1e-4)
    x_p = np.tile([2.5e-2, -1.0e-2, 5.0e-3], (xi.shape[0], 1))
    u_p = np.tile([1.0e-5, 0.0, -1.0e-5], (xi.shape[0], 1))
    ref, scale = _stretch64(xi, eta), _strain_scale(xi, eta)
    naive = np.median(np.abs(_stretch32_positions(x_p, xi, eta, u_p).astype(np.float64) - ref) / scale)
    comp = np.median(np.abs(_stretch32_compensated(xi, eta).astype(np.float64) - ref) / scale)
    # measured: 1.2e-3 of the strain for the reference's form (the FP32
    # rounding of positions 2.5 cm from the origin), 3e-8 compensated
    assert naive > 1e-4 and comp < 1e-7 and naive > 1000 * comp, (naive, comp)
