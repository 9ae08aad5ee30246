"""Generate tests/golden/operators.json: known answers from hpc-dave/dare's own tests.

The reference's operator tests compute their expected values from closed
formulas (its GTest code, read as text).  This script re-evaluates those same
formulas in IEEE double precision, in the same order of operations, and writes
the results as fixtures.  Python floats are IEEE binary64, so the values are
what the reference's tests compare against.

Sources (paths inside the hpc-dave/dare tree):
  - Laplacian  ``mb = -1 * div(grad(mb))``: Grid/test/test_Cartesian_Operators.cpp:713-965
  - TVD face matrix stencils (CDS, UPWIND, MINMOD, VANALBADA; velocity +-1):
    Grid/test/test_Cartesian_Operators.cpp:1064-1110, 1126-1168, 1250-1333, 1420-1501
  - DDT implicit Euler: Equations/test/test_DDT.cpp:73-110

Run: python tests/golden/make_golden.py  (writes operators.json beside itself)
"""
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))
NUM_GHOST = 2


def geometry(res, size):
    """Cartesian ctor: CartesianMesh.inl:75-83."""
    dx = [s / n for s, n in zip(size, res)]
    vol = 1.0
    for d in dx:
        vol *= d
    area = [vol / d for d in dx]
    dn_r = [1.0 / d for d in dx]
    return dx, vol, area, dn_r


def laplacian_cases():
    cases = []
    for dim in (1, 2, 3):
        res = [10 + n for n in range(dim)]          # GetResolutionTestCartesianOperators
        size = [1.0 + n for n in range(dim)]        # GetSizeTestCartesianOperators
        _, _, A, dn = geometry(res, size)
        exp = {"W": -A[0] * dn[0], "E": -A[0] * dn[0]}
        c = 2.0 * A[0] * dn[0]
        if dim > 1:
            exp["S"] = -A[1] * dn[1]
            exp["N"] = -A[1] * dn[1]
            c = c + 2.0 * A[1] * dn[1]
        if dim > 2:
            exp["B"] = -A[2] * dn[2]
            exp["T"] = -A[2] * dn[2]
            c = c + 2.0 * A[2] * dn[2]
        exp["C"] = c
        cases.append({"dim": dim, "n": res, "size": size, "ordinal": 0, "expected": exp,
                      "exact": True})
    return cases


def _std_min(a, b):
    return b if b < a else a


def _std_max(a, b):
    return b if a < b else a


def _minmod(r):
    if math.isnan(r):
        r = 0.0
    return _std_max(0.0, _std_min(r, 1.0))


def _vanalbada(r):
    if math.isnan(r):
        r = 0.0
    return (r + r * r) / (1.0 + r * r)


def _div(a, b):
    if b == 0.0:
        if a == 0.0 or math.isnan(a):
            return math.nan
        return math.copysign(math.inf, a) * math.copysign(1.0, b)
    return a / b


def tvd_cases():
    """1D grid, 10 cells, size 1, ghost 2; internal ordinal 0 -> local index 2."""
    cases = []
    ind = NUM_GHOST
    for limiter, field_kind in (("CDS", "linear"), ("UPWIND", "linear"),
                                ("MINMOD", "quadratic"), ("VANALBADA", "quadratic")):
        for vel in (1.0, -1.0):
            for comp in (0, 1, 2):                 # N = 3 components in the test fixture
                if field_kind == "linear":
                    f = lambda i, c=comp: float(i * c)
                else:
                    f = lambda i, c=comp: float(i * i * c)
                pc, pw, pww, pe, pee = f(ind), f(ind - 1), f(ind - 2), f(ind + 1), f(ind + 2)
                if vel > 0:
                    face = {"W": {"nb": vel, "c": 0.0}, "E": {"nb": 0.0, "c": vel}}
                else:
                    face = {"W": {"nb": 0.0, "c": vel}, "E": {"nb": vel, "c": 0.0}}
                exact = limiter in ("UPWIND", "MINMOD", "VANALBADA")
                if limiter == "CDS":                   # :1086-1109 (rhs NEAR, 1e3 eps)
                    if vel > 0:
                        rw = -0.5 * (pc - pw) * vel
                        re = -0.5 * (pe - pc) * vel
                    else:
                        rw = -0.5 * (pw - pc) * vel
                        re = -0.5 * (pc - pe) * vel
                elif limiter == "UPWIND":              # :1147-1167 (rhs == 0)
                    rw = re = 0.0
                else:
                    lim = _minmod if limiter == "MINMOD" else _vanalbada
                    if vel > 0:                        # :1278-1298, :1448-1468
                        r_w = lim(_div(pw - pww, pc - pw))
                        rw = -0.5 * r_w * (pc - pw) * vel
                        r_e = lim(_div(pc - pw, pe - pc))
                        re = -0.5 * r_e * (pe - pc) * vel
                    else:                              # :1313-1333, :1483-1501
                        r_w = lim(_div(pe - pc, pc - pw))
                        rw = -0.5 * r_w * (pw - pc) * vel
                        r_e = lim(_div(pee - pe, pe - pc))
                        re = -0.5 * r_e * (pc - pe) * vel
                face["W"]["rhs"] = rw
                face["E"]["rhs"] = re
                cases.append({"limiter": limiter, "vel": vel, "component": comp,
                              "field": field_kind, "n": [10], "size": [1.0], "ordinal": 0,
                              "expected_face": face, "rhs_exact": exact, "rhs_eps_tol": 1e3})
    return cases


def ddt_cases():
    """test_DDT.cpp:73-110 (EulerBackward, single field): 3D grid (10,11,12),
    size (1,2,3), ordinal 0, dt = 0.1, phi level t = (t+1)*0.3."""
    res, size = [10, 11, 12], [1.0, 2.0, 3.0]
    _, vol, _, _ = geometry(res, size)
    dt = 0.1
    phi_base = 0.3
    dv_dt = vol / dt
    return [{"n": res, "size": size, "dt": dt, "phi_new": 1.0 * phi_base, "phi_old": 2.0 * phi_base,
             "expected": {"C": dv_dt, "rhs": dv_dt * 2.0 * phi_base},
             "abs_tol": 2.220446049250313e-16}]


def main():
    out = {"laplacian": laplacian_cases(), "tvd": tvd_cases(), "ddt": ddt_cases()}
    path = os.path.join(HERE, "operators.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1, allow_nan=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
