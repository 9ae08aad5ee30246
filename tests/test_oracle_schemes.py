"""Time schemes of the Divergence operators in the CPU oracle.

Equations/TimeDiscretizationSchemes.h:29-76 gives the weights w[0..T];
Grid/Cartesian/Divergence_Cartesian.inl:186-205 scales the implicit
coefficients by w[0] and adds, for every explicit level t >= 1, w[t] * A *
(rhs_E - rhs_W + ...) of that level's face stencil, each level being a copy
of the level-0 stencil (:61-62).  The reference has no test that exercises a
scheme other than EULER_BACKWARD, so these properties pin the restatement:
coefficients = w[0] x the EULER_BACKWARD ones (exact: w[0] scales a sum of
products it does not enter), rhs = (1 + sum_{t>=1} w[t]) x the
EULER_BACKWARD deferred-correction rhs (up to rounding: the level-0 rhs is
assigned after the w[0] scaling, so it enters unweighted), DDT untouched.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import oracle_assembly, oracle_grid

WEIGHTS = {
    "EULER_BACKWARD": (1.0,),
    "EULER_FORWARD": (0.0, 1.0),
    "CRANK_NICHOLSON": (0.5, 0.5),
    "ADAMS_BASHFORTH": (0.0, 1.5, -0.5),
    "ADAMS_MOULTON": (5.0 / 12.0, 8.0 / 12.0, -1.0 / 12.0),
}


def _case(scheme, dt=0.0, diffusion=False, convection=True, seed=3):
    rng = np.random.default_rng(seed)
    n = (7, 6, 9)
    phi = rng.random(tuple(x + 4 for x in n))
    # periodic: a Dirichlet face would add 2 bc X to the rhs, X scaling with w[0]
    c = {"n": n, "size": (1.0, 0.8, 1.3), "periodic": (1, 1, 1), "dt": dt, "phi0": phi,
         "limiter": "VANLEER", "scheme": scheme}
    if convection:
        c["face_vel"] = [rng.normal(size=tuple(x + (1 if e == d else 0) for e, x in enumerate(n)))
                         for d in range(3)]
    if diffusion:
        c["D"] = 3e-3
    return c


def _assemble(case):
    og = oracle_grid(case)
    desc = oracle_assembly(og, case)
    phi = np.ascontiguousarray(case["phi0"].reshape(-1))
    return O.assemble(desc, phi, phi)


@pytest.mark.parametrize("scheme", list(WEIGHTS))
def test_convection_scales_with_scheme_weights(scheme):
    w = WEIGHTS[scheme]
    d0, r0, m0 = _assemble(_case("EULER_BACKWARD"))
    d1, r1, m1 = _assemble(_case(scheme))
    np.testing.assert_array_equal(m0, m1)
    # w[0] = 0 leaves signed zeros, compared by value
    np.testing.assert_array_equal(d1, w[0] * d0)
    # the level-0 rhs enters unweighted (it is set after s_c *= w[0])
    np.testing.assert_allclose(r1, (1.0 + sum(w[1:])) * r0, rtol=1e-12, atol=1e-15 * np.abs(r0).max())


@pytest.mark.parametrize("scheme", list(WEIGHTS))
def test_diffusion_and_ddt(scheme):
    w = WEIGHTS[scheme]
    dt = 0.02
    base = _assemble(_case("EULER_BACKWARD", dt=dt, diffusion=True, convection=False))
    got = _assemble(_case(scheme, dt=dt, diffusion=True, convection=False))
    ddt = _assemble(_case("EULER_BACKWARD", dt=dt, convection=False))
    # the gradient stencil carries no rhs: only DDT's old-level term remains
    np.testing.assert_array_equal(got[1], base[1])
    off = [1, 2, 3, 4, 5, 6]
    np.testing.assert_array_equal(got[0][off], w[0] * base[0][off])
    # centre = DDT weight + w[0] x the diffusion centre
    np.testing.assert_allclose(got[0][0] - ddt[0][0], w[0] * (base[0][0] - ddt[0][0]), rtol=1e-12, atol=1e-300)


def test_unknown_scheme_rejected():
    case = _case("EULER_BACKWARD")
    og = oracle_grid(case)
    desc = oracle_assembly(og, case)
    desc.scheme = 17
    with pytest.raises(ValueError):
        O.assemble(desc, np.ascontiguousarray(case["phi0"].reshape(-1)))
