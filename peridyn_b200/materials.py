"""Material types mirroring src/materials/*.jl of the reference.

These classes hold the host-side description of a material block.  The
family, intact flags and weighted volume are built on the GPU when the block
enters an environment (:func:`peridyn_b200.Env`); afterwards the
``family``/``intact``/``weighted_volume`` attributes read them back in the
reference's layout (M' x N column-major, 1-based, descending, 0 padding).
"""
import itertools
import math
from decimal import Decimal, localcontext

import numpy as np

from . import _abi

_block_counter = itertools.count(1)  # const_macros.jl:9 PDBlockID


# ---------------------------------------------------------------------------
# Julia scalar arithmetic used by the reference constructors
# ---------------------------------------------------------------------------
def _fma(a, b, c):
    """Correctly rounded a*b + c (Python 3.12 has no math.fma)."""
    if not (math.isfinite(a) and math.isfinite(b) and math.isfinite(c)):
        return a * b + c
    with localcontext() as ctx:
        ctx.prec = 2200
        return float(Decimal(a) * Decimal(b) + Decimal(c))


def julia_pow_int(x, n):
    """Julia 1.10 ``^(x::Float64, n::Integer)`` (base/math.jl pow_body): a
    compensated repeated squaring whose muladd is fused."""
    x = float(x)
    if n == 0:
        return 1.0
    if n == 3:
        return x * x * x
    y, xnlo, ynlo = 1.0, 0.0, 0.0
    if n < 0:
        rx = 1.0 / x
        if n == -2:
            return rx * rx
        if math.isfinite(x):
            xnlo = -_fma(x, rx, -1.0) * rx
        x, n = rx, -n
    while n > 1:
        if n & 1:
            err = _fma(y, xnlo, x * ynlo)
            p = x * y
            ynlo = _fma(x, y, -p)
            y = p
            ynlo += err
        err = x * 2 * xnlo
        p = x * x
        xnlo = _fma(x, x, -p)
        x = p
        xnlo += err
        n >>= 1
    err = _fma(y, xnlo, x * ynlo)
    return _fma(x, y, err) if (math.isfinite(x) and math.isfinite(err)) else x * y


def make_matrix(S):
    """utils.jl:12-25: vector of the upper triangle (row by row) -> symmetric
    matrix; a matrix is returned as is (utils.jl:35-37)."""
    S = np.asarray(S, dtype=np.float64)
    if S.ndim == 2:
        return np.asfortranarray(S)
    n = S.size
    N = int(math.sqrt(2 * n + 0.5 ** 2) - 0.5)
    bs = np.zeros((N, N), dtype=np.float64, order="F")
    a = 0
    for i in range(N):
        for j in range(i, N):
            bs[i, j] = S[a]
            bs[j, i] = S[a]
            a += 1
    return bs


def _as_vec(v):
    return np.atleast_1d(np.asarray(v, dtype=np.float64))


# ---------------------------------------------------------------------------
# GeneralMaterial (general_material.jl:43-98)
# ---------------------------------------------------------------------------
class GeneralMaterial:
    """``GeneralMaterial(y0, v0, x, volume, type, horizon; max_neigh=100,
    particle_size=0, skip_bb=false)``.  Arrays are 3xN (numpy shape (3, N),
    stored column-major like Julia)."""

    def __init__(self, y0, v0, x, volume, type, horizon, max_neigh=100, particle_size=0, skip_bb=False):
        self.x = np.asfortranarray(np.asarray(x, dtype=np.float64).reshape(3, -1))
        self.y = np.asfortranarray(np.asarray(y0, dtype=np.float64).reshape(3, -1))
        self.velocity = np.asfortranarray(np.asarray(v0, dtype=np.float64).reshape(3, -1))
        self.volume = np.ascontiguousarray(np.asarray(volume, dtype=np.float64).reshape(-1))
        self.type = np.ascontiguousarray(np.asarray(type, dtype=np.int64).reshape(-1))
        n = self.x.shape[1]
        if not (self.y.shape[1] == n and self.velocity.shape[1] == n and self.volume.size == n
                and self.type.size == n):
            raise ValueError("x, y0, v0, volume and type must describe the same particles")
        if particle_size == 0:
            particle_size = float(self.volume[0]) ** (1 / 3)  # general_material.jl:82-84
        self.particle_size = float(particle_size)
        self.horizon = float(horizon)
        self.max_neigh = int(max_neigh)
        self.skip_bb = bool(skip_bb)
        self.deformed = [not np.array_equal(self.y, self.x)]  # general_material.jl:92-96
        self._env = None
        self._block = None

    @property
    def n(self):
        return self.x.shape[1]

    # device-backed attributes, available once the block is in an Env
    def _need_env(self):
        if self._env is None:
            raise RuntimeError("family data is built on the GPU when the material enters an Env")
        return self._env

    @property
    def family(self):
        return self._need_env()._family(self._block)[0]

    @property
    def intact(self):
        return self._need_env()._family(self._block)[1]

    @property
    def weighted_volume(self):
        env = self._need_env()
        m = np.zeros(self.n)
        _abi.check(_abi.lib().pd_env_get_weighted_volume(env._h, self._block, _abi.dptr(m)))
        return m


# ---------------------------------------------------------------------------
# Specific materials
# ---------------------------------------------------------------------------
class SpecificMaterial:
    kind = None


class BondBasedSpecific(SpecificMaterial):
    """bond_based.jl:21-122.  ``bond_stiffness = 18K/pi/horizon^4`` once the
    horizon is known (``init`` with the general material)."""

    kind = _abi.PD_MAT_BOND_BASED

    def __init__(self, K, critical_stretch, density, horizon=None, func=None):
        K = make_matrix(_as_vec(K)) if np.ndim(K) < 2 else make_matrix(K)
        cs = make_matrix(_as_vec(critical_stretch)) if np.ndim(critical_stretch) < 2 else make_matrix(critical_stretch)
        self.bulk_modulus = K
        self.critical_stretch = cs
        self.density = _as_vec(density)
        self.func = func
        if horizon is None:
            self.bond_stiffness = np.zeros_like(K)
        else:
            h4 = julia_pow_int(float(horizon), 4)
            self.bond_stiffness = np.asfortranarray(18 * K / math.pi / h4)

    def init(self, gen):
        return BondBasedSpecific(self.bulk_modulus, self.critical_stretch, self.density, horizon=gen.horizon,
                                 func=self.func)


class OrdinaryStateBasedSpecific(SpecificMaterial):
    """ordinary_state_based.jl:18-63 (linear peridynamic solid)."""

    kind = _abi.PD_MAT_ORDINARY_STATE_BASED

    def __init__(self, bulk_modulus, shear_modulus, critical_stretch, density):
        self.bulk_modulus = make_matrix(bulk_modulus) if np.ndim(bulk_modulus) == 2 else make_matrix(_as_vec(bulk_modulus))
        self.shear_modulus = make_matrix(shear_modulus) if np.ndim(shear_modulus) == 2 else make_matrix(_as_vec(shear_modulus))
        self.critical_stretch = (make_matrix(critical_stretch) if np.ndim(critical_stretch) == 2
                                 else make_matrix(_as_vec(critical_stretch)))
        self.density = _as_vec(density)
        self.theta = np.zeros(0)

    def init(self, gen):
        self.theta = np.zeros(gen.n)
        return self


class VonMises:
    """elasto_plastic.jl:453-479 Von Mises criterion."""

    @staticmethod
    def effective_stress2(s1, s2, s3):
        # ((s1 - s2)^2 + (s2 - s3)^2 + (s1 - s3)^2) / 2, element-wise
        a, b, c = s1 - s2, s2 - s3, s1 - s3
        return (a * a + b * b + c * c) / 2


class ElastoPlasticSolidSpecific(SpecificMaterial):
    """elasto_plastic.jl:31-116: ``ElastoPlasticSolidSpecific(K, G, cs,
    density, sigma_y; criteria=VonMises())``.  ``init`` sets the yield value
    psi = 75/(8 pi) * sigma_e^2 / horizon^5 per type pair, the plastic
    deviatoric strain edp (per bond) and td_norm2 to zero (:60-68)."""

    kind = _abi.PD_MAT_ELASTO_PLASTIC

    def __init__(self, bulk_modulus, shear_modulus, critical_stretch, density, yield_stress, criteria=None):
        self.bulk_modulus = make_matrix(bulk_modulus) if np.ndim(bulk_modulus) == 2 else make_matrix(_as_vec(bulk_modulus))
        self.shear_modulus = make_matrix(shear_modulus) if np.ndim(shear_modulus) == 2 else make_matrix(_as_vec(shear_modulus))
        self.critical_stretch = (make_matrix(critical_stretch) if np.ndim(critical_stretch) == 2
                                 else make_matrix(_as_vec(critical_stretch)))
        self.density = _as_vec(density)
        self.yield_stress = (make_matrix(yield_stress) if np.ndim(yield_stress) == 2
                             else make_matrix(_as_vec(yield_stress)))
        self.criteria = VonMises() if criteria is None else criteria
        if not hasattr(self.criteria, "effective_stress2"):
            raise NotImplementedError(f"effective_stress not implemented for {type(self.criteria).__name__}")
        self.psi = np.zeros_like(self.yield_stress)
        self.theta = np.zeros(0)

    def init(self, gen):
        d = gen.horizon
        # sigma = [1, 0, 0] * sigma_y (elasto_plastic.jl:62-65)
        sy = self.yield_stress
        se2 = self.criteria.effective_stress2(sy * 1.0, sy * 0.0, sy * 0.0)
        self.psi = np.asfortranarray((75 / (8 * math.pi)) * se2 / julia_pow_int(d, 5))
        self.theta = np.zeros(gen.n)
        return self


class SkipSpecific(SpecificMaterial):
    """skip_specific.jl:39-49: no material forces (rigid/passive block)."""

    kind = _abi.PD_MAT_SKIP

    def __init__(self, density=(1.0,)):
        self.density = _as_vec(density)
        n = self.density.size
        self.critical_stretch = np.full((n, n), np.inf, order="F")

    def init(self, gen):
        return self


class PeridynamicsMaterial:
    """``PeridynamicsMaterial(gen, spc; name)`` (general_material.jl:175-222):
    a material block.  ``type`` is the type range minimum:maximum of the
    general material's particle types."""

    def __init__(self, gen, spc, name="PeridynamicsMaterial", blockid=None):
        self.name = name
        self.general = gen
        self.specific = spc.init(gen)
        self.blockid = next(_block_counter) if blockid is None else int(blockid)
        self.type = range(int(gen.type.min()), int(gen.type.max()) + 1)

    @property
    def kind(self):
        return self.specific.kind

    def descriptor(self):
        """The C-ABI pd_material_desc for this block (arrays kept alive on
        the returned object)."""
        spc = self.specific
        nt = len(self.type)
        keep = []

        def mat(a):
            a = np.asfortranarray(np.asarray(a, dtype=np.float64))
            if a.shape != (nt, nt):
                raise ValueError(f"{self.name}: parameter matrix must be {nt}x{nt}")
            keep.append(a)
            return _abi.dptr(a)

        d = _abi.MaterialDesc()
        d.kind = spc.kind
        d.ntypes = nt
        d.type_start = self.type.start
        dens = np.ascontiguousarray(np.asarray(spc.density, dtype=np.float64).reshape(-1)[:nt])
        if dens.size != nt:
            raise ValueError(f"{self.name}: density needs {nt} entries")
        keep.append(dens)
        d.density = _abi.dptr(dens)
        if spc.kind != _abi.PD_MAT_SKIP:
            d.critical_stretch = mat(spc.critical_stretch)
        if spc.kind == _abi.PD_MAT_BOND_BASED:
            d.bond_stiffness = mat(spc.bond_stiffness)
        if spc.kind in (_abi.PD_MAT_ORDINARY_STATE_BASED, _abi.PD_MAT_ELASTO_PLASTIC):
            d.bulk_modulus = mat(spc.bulk_modulus)
            d.shear_modulus = mat(spc.shear_modulus)
        if spc.kind == _abi.PD_MAT_ELASTO_PLASTIC:
            d.plastic_psi = mat(spc.psi)
        d.horizon = self.general.horizon
        d.particle_size = self.general.particle_size
        d.max_neigh = self.general.max_neigh
        d._keep = keep
        return d


def BondBasedMaterial(gen, spc, name="BondBasedMaterial"):
    return PeridynamicsMaterial(gen, spc, name=name)


def OrdinaryStateBasedMaterial(gen, spc, name="OrdinaryStateBasedMaterial"):
    return PeridynamicsMaterial(gen, spc, name=name)


def SkipMaterial(gen, spc, name="SkipMaterial"):
    return PeridynamicsMaterial(gen, spc, name=name)
