"""Materials of the hot path (drop-in names of ``gfem.materials``).

  * ``LinearElastic(E, nu)`` — small-strain isotropic elasticity
    (gfem/materials.py:56-68);
  * ``J2Plasticity(E, nu, table, Hk=0)`` — small-strain von Mises plasticity with
    tabulated isotropic hardening and linear kinematic hardening, radial return
    with a fixed 25-iteration local Newton (gfem/materials.py:228-302).  The table
    is extended exactly as the reference does: a single row means perfect
    plasticity, and a last point at eps_p = 1e6 continues the final slope.
  * ``from_props`` — the property-dictionary constructor for these two models
    (gfem/materials.py:335-391: ``E``, ``nu``, ``plastic`` table or ``yield`` +
    ``tangent`` bilinear, ``Hk``).

The constitutive arithmetic runs in the CUDA kernels; these objects carry the
parameters and produce the ``exfem_material`` struct of the C ABI.
"""
import numpy as np

from . import _lib


def lame(E, nu):                                                       # gfem/materials.py:18-19
    return E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))


class Material:
    nstate = 1
    small_strain = True
    linear = False
    name = "material"

    def modulus(self):
        return float(self.mu * (3 * self.lam + 2 * self.mu) / (self.lam + self.mu))

    def describe(self):
        return f"{type(self).__name__}({self.name})"


class LinearElastic(Material):
    linear = True

    def __init__(self, E, nu, density=1.0, name=None, alpha=0.0, tref=0.0, **kw):
        self.E, self.nu = float(E), float(nu)
        self.mu, self.lam = lame(self.E, self.nu)
        self.density = float(density)
        # thermal expansion (gfem/materials.py:28-30); a temperature field that would
        # strain the material is refused by the model (the kernels have no thermal strain)
        self.alpha, self.tref = float(alpha), float(tref)
        if name:
            self.name = name

    def to_c(self):
        m = _lib.Material()
        m.kind, m.E, m.nu, m.Hk, m.ntab = _lib.LINEAR_ELASTIC, self.E, self.nu, 0.0, 0
        return m


class J2Plasticity(Material):
    nstate = 19

    def __init__(self, E, nu, table, Hk=0.0, density=1.0, name=None, alpha=0.0, tref=0.0, **kw):
        self.E, self.nu = float(E), float(nu)
        self.mu, self.lam = lame(self.E, self.nu)
        self.K = self.lam + 2 * self.mu / 3
        self.Hk = float(Hk)
        self.density = float(density)
        self.alpha, self.tref = float(alpha), float(tref)
        if name:
            self.name = name
        t = np.asarray(table, dtype=np.float64).reshape(-1, 2)
        if t.shape[0] == 1:                                            # perfect plasticity
            t = np.array([[t[0, 0], 0.0], [t[0, 0], 1e3]])
        sy_tab, ep_tab = t[:, 0], t[:, 1]
        slope = (sy_tab[-1] - sy_tab[-2]) / max(ep_tab[-1] - ep_tab[-2], 1e-30)
        self.ep_tab = np.append(ep_tab, 1e6)
        self.sy_tab = np.append(sy_tab, sy_tab[-1] + slope * (1e6 - ep_tab[-1]))
        if len(self.ep_tab) > _lib.MAX_TABLE:
            raise ValueError(f"hardening table longer than {_lib.MAX_TABLE - 1} rows")
        self.table = t
        self.sy0 = float(t[0, 0])

    def to_c(self):
        m = _lib.Material()
        m.kind, m.E, m.nu, m.Hk = _lib.J2, self.E, self.nu, self.Hk
        m.ntab = len(self.ep_tab)
        for i, (s, e) in enumerate(zip(self.sy_tab, self.ep_tab)):
            m.sy_tab[i], m.ep_tab[i] = float(s), float(e)
        return m


def from_props(p, name=None):
    """Material from a property dictionary (the keys of gfem/materials.py:335-391)
    for the two small-strain models covered.  A plastic material takes a hardening
    table, or a yield stress with an optional elastic-plastic tangent modulus Et:
    the plastic modulus of that straight line is H = E Et / (E - Et), giving the
    two-row table (sy, 0), (sy + H, 1)."""
    common = dict(density=p.get("density", 1.0), alpha=p.get("alpha", 0.0), tref=p.get("tref", 0.0), name=name)
    if not ("plastic" in p or "yield" in p or p.get("model") == "plastic"):
        return LinearElastic(p["E"], p["nu"], **common)
    table = p.get("plastic")
    if table is None:
        E, Et, sy = float(p["E"]), float(p.get("tangent", 0.0)), float(p["yield"])
        H = E * Et / (E - Et) if Et > 0.0 else 0.0
        table = [[sy, 0.0], [sy + H, 1.0]]
    return J2Plasticity(p["E"], p["nu"], table, Hk=p.get("Hk", 0.0), **common)
