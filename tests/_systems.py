"""Small seeded systems shared by the tests (host setup + oracle assembly)."""

from __future__ import annotations

from functools import lru_cache

import numpy as np
import scipy.sparse as sp

from cutcell_b200.aggregation import build_extension
from cutcell_b200.cutgeom import PlaneLevelSet, SphereExteriorLevelSet
from cutcell_b200.problem import build_problem, manufactured_sine
from oracle.aggregation import restrict_spd
from oracle.assembly import assemble_full


def plane5(offset=0.23):
    a = np.deg2rad(5.0)
    return PlaneLevelSet((np.cos(a), np.sin(a), 0.0), offset)


def sphere(r=0.31):
    return SphereExteriorLevelSet((0.5, 0.5, 0.5), r)


@lru_cache(maxsize=None)
def system(kind: str, n: int, p: int, a_mass: float = 0.0, nitsche: bool = True):
    phi = {"sphere": sphere(), "plane": plane5(), "sphere_small": sphere(0.2)}[kind]
    u, f = manufactured_sine()
    prob = build_problem(phi, n, p, a_mass=a_mass, a_stiff=1.0, nitsche=nitsche, forcing=f, dirichlet=u)
    ext = build_extension(prob.gamma, prob.basis, p)
    A_full = assemble_full(prob)
    A_red = restrict_spd(A_full, ext.E)
    b = np.asarray(ext.E.T @ prob.load)
    return prob, ext, A_full, sp.csr_matrix(A_red), b
