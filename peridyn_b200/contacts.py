"""Contact models mirroring src/contacts/*.jl of the reference.

Only the parameters live here; neighbour search and forces run on the GPU.
"""
import math

from . import _abi
from .materials import julia_pow_int


class ContactModel:
    pass


class NonLinearSpringContactModel12(ContactModel):
    """nonlinearspring.jl:15-25 with ContactModel12_gcal (contacts.jl:76-91)."""

    kind = _abi.PD_CONTACT_12

    def __init__(self, exponent, stifness, mat1, mat2, distanceD=1.0, distanceX=3.0, max_neighs=50):
        self.exponent = float(exponent)
        self.stifness = float(stifness)
        self.pair = (mat1.type, mat2.type)
        self.mat1, self.mat2 = mat1, mat2
        self.name = f"{mat1.name}-{mat2.name}"
        self.equi_dist = (mat1.general.particle_size + mat2.general.particle_size) / 2 * distanceD
        self.distance = distanceX * self.equi_dist
        n2 = mat2.general.n
        self.max_neighs = min(int(max_neighs), n2)


class NonLinearSpringContactModel11(ContactModel):
    """nonlinearspring.jl:32-44 with ContactModel11_gcal (contacts.jl:105-124).

    ``ordered=False`` keeps the reference's neighbour search
    (contacts.jl:539-573), whose merge walk assumes ascending families and so
    finds at most the first family member.  ``ordered=True`` (an extension)
    lists every family member whose bond is broken, in a search cell adjacent
    to the particle's and within ``equi_dist``, in family order, up to
    ``max_neighs`` of them.
    """

    def __init__(self, exponent, stifness, mat1, distanceD=1.0, distanceX=5, max_neighs=50, ordered=False):
        self.ordered = bool(ordered)
        self.kind = _abi.PD_CONTACT_11_ORDERED if self.ordered else _abi.PD_CONTACT_11
        self.exponent = float(exponent)
        self.stifness = float(stifness)
        self.type = mat1.type
        self.bid = mat1.blockid
        self.mat1 = mat1
        self.material = mat1.general
        self.name = f"{mat1.name}-{mat1.name}"
        self.equi_dist = mat1.general.particle_size * distanceD
        self.distance = distanceX * self.equi_dist
        self.rows = int(max_neighs)  # neighs = zeros(max_neighs, N)
        self.max_neighs = min(int(max_neighs), mat1.general.n)


def NonLinearSpringContactModel(exponent, stifness, mat1, mat2=None, distanceD=1.0, distanceX=None, max_neighs=50,
                                ordered=False):
    """nonlinearspring.jl:63-111: two blocks -> 12 (distanceX=3.0),
    one block -> 11 (distanceX=5); ``ordered`` selects the ordered
    self-contact search (one block only)."""
    if mat2 is not None:
        if ordered:
            raise ValueError("ordered neighbour search applies to self contact (one block) only")
        return NonLinearSpringContactModel12(exponent, stifness, mat1, mat2, distanceD=distanceD,
                                             distanceX=3.0 if distanceX is None else distanceX,
                                             max_neighs=max_neighs)
    return NonLinearSpringContactModel11(exponent, stifness, mat1, distanceD=distanceD,
                                         distanceX=5 if distanceX is None else distanceX, max_neighs=max_neighs,
                                         ordered=ordered)


def LinearSpringContactModel(stifness, mat1, mat2=None, **kwargs):
    """linearspring.jl:175-196: exponent 1."""
    return NonLinearSpringContactModel(1, stifness, mat1, mat2, **kwargs)


def ShortRangeContactModel(K, horizon, mat1, mat2=None, mfactor=1.0, **kwargs):
    """shortrange.jl:219-246: stiffness 18K/(pi*horizon^4) * mfactor."""
    stifness = 18 * K / (math.pi * julia_pow_int(float(horizon), 4)) * mfactor
    return LinearSpringContactModel(stifness, mat1, mat2, **kwargs)
