"""The fused end of a time step's solve, checked on the CPU.

k_solution_to_field (dare_b200/csrc/dare_core.cu) does in one pass what
k_scale, k_scatter_to_field and k_halo_fill did one after the other: x =
invd .* x (the right preconditioner's x = M^-1 y at the exit of
BiCGStab2.inl:571-574), CopyTo into the field (Trilinos.inl:166-177) and
the periodic face ghosts of ExchangeHaloCells (HaloBuffer.inl:194-208; only
ghosts outside the internal range in exactly one dimension), each ghost
written by the internal cell it images.  This restates the kernel's thread
and block arithmetic and checks, for 1-D / 2-D / 3-D grids, periodic and
bounded, ghost widths 2 and 3 and sizes down to n = ng, that every access
stays inside x and the ghosted field, that no cell is written twice, and
that x and the field end up equal, cell for cell, to the three kernels'
results and to the oracle's CopyTo + ExchangeHaloCells -- before the kernel
ever runs.
"""
import itertools

import numpy as np
import pytest

from oracle import oracle as O


def grid_dev(dim, n, ng, periodic):
    n3 = list(n) + [1] * (3 - dim)
    og = [ng if d < dim else 0 for d in range(3)]
    per = list(periodic) + [0] * (3 - dim)
    gn = [n3[d] + 2 * og[d] for d in range(3)]
    return {"dim": dim, "ng": ng, "n": n3, "og": og, "gn": gn, "periodic": per}


def fused_ok(g):
    return all(not g["periodic"][d] or (g["og"][d] == g["ng"] and g["n"][d] >= g["ng"]) for d in range(g["dim"]))


def block_shape(g):
    bx = 1
    while bx < g["n"][2] and bx < 256:
        bx *= 2
    return bx, 256 // bx


def lin(g, t):
    return (t[0] * g["gn"][1] + t[1]) * g["gn"][2] + t[2]


def fused(g, invd, x, phi, num_sms):
    """k_solution_to_field, thread by thread; returns the writes it makes."""
    n0, n1, n2 = g["n"]
    ncell, nghost = n0 * n1 * n2, g["gn"][0] * g["gn"][1] * g["gn"][2]
    bx, by = block_shape(g)
    rows = n0 * n1
    blocks = max(1, min(-(-rows // by), num_sms * 8))        # grid_blocks(ctx, rows, by, 8)
    xw, fw = {}, {}
    for b, ty, tx in itertools.product(range(blocks), range(by), range(bx)):
        r = b * by + ty
        while r < rows:
            i = r // n1
            j = r - i * n1
            k = tx
            while k < n2:
                c = r * n2 + k
                assert 0 <= c < ncell
                v = invd[c] * x[c] if invd is not None else x[c]
                if invd is not None:
                    assert c not in xw
                    xw[c] = v
                q = (i, j, k)
                ind = [i + g["og"][0], j + g["og"][1], k + g["og"][2]]
                targets = [list(ind)]
                for d in range(g["dim"]):
                    if not g["periodic"][d]:
                        continue
                    if q[d] < g["ng"]:
                        t = list(ind)
                        t[d] = g["og"][d] + g["n"][d] + q[d]
                        targets.append(t)
                    if q[d] >= g["n"][d] - g["ng"]:
                        t = list(ind)
                        t[d] = q[d] - g["n"][d] + g["ng"]
                        targets.append(t)
                for t in targets:
                    assert all(0 <= t[d] < g["gn"][d] for d in range(3)), (t, g)
                    o = lin(g, t)
                    assert 0 <= o < nghost and o not in fw, (t, g)
                    fw[o] = v
                k += bx
            r += blocks * by
    return xw, fw


def three_kernels(g, invd, x, phi):
    """k_scale, k_scatter_to_field, then k_halo_fill along each periodic dimension."""
    x = x.copy() if invd is None else invd * x
    phi = phi.copy()
    n0, n1, n2 = g["n"]
    for c in range(n0 * n1 * n2):
        i, j, k = c // (n1 * n2), (c // n2) % n1, c % n2
        phi[lin(g, (i + g["og"][0], j + g["og"][1], k + g["og"][2]))] = x[c]
    for d in range(g["dim"]):
        if not g["periodic"][d]:
            continue
        e1, e2 = (1 if d == 0 else 0), (1 if d == 2 else 2)
        for layer, a, b in itertools.product(range(2 * g["ng"]), range(g["n"][e1]), range(g["n"][e2])):
            ind, src = [0, 0, 0], [0, 0, 0]
            ind[e1], ind[e2] = a + g["og"][e1], b + g["og"][e2]
            if layer < g["ng"]:
                ind[d] = layer
                src[d] = ind[d] + g["n"][d]
            else:
                ind[d] = g["og"][d] + g["n"][d] + layer - g["ng"]
                src[d] = ind[d] - g["n"][d]
            src[e1], src[e2] = ind[e1], ind[e2]
            phi[lin(g, ind)] = phi[lin(g, src)]
    return x, phi


CASES = [
    (1, (7,), 2, (1,)), (1, (2,), 2, (1,)), (1, (3,), 3, (1,)), (1, (9,), 2, (0,)),
    (2, (5, 6), 2, (1, 1)), (2, (4, 3), 3, (1, 0)), (2, (2, 2), 2, (0, 1)), (2, (6, 40), 2, (1, 1)),
    (3, (3, 4, 5), 2, (1, 1, 1)), (3, (2, 3, 2), 2, (1, 1, 1)), (3, (4, 3, 6), 3, (0, 1, 1)),
    (3, (3, 3, 4), 2, (1, 0, 0)), (3, (2, 2, 300), 2, (1, 1, 1)), (3, (3, 5, 7), 2, (0, 0, 0)),
]


@pytest.mark.parametrize("num_sms", [1, 148])
@pytest.mark.parametrize("dim,n,ng,periodic", CASES)
@pytest.mark.parametrize("jacobi", [True, False])
def test_fused_exit_writes_what_the_three_kernels_wrote(dim, n, ng, periodic, jacobi, num_sms):
    g = grid_dev(dim, n, ng, periodic)
    assert fused_ok(g)
    rng = np.random.default_rng(dim * 100 + sum(n) + ng)
    ncell = int(np.prod(g["n"]))
    nghost = int(np.prod(g["gn"]))
    x = rng.normal(size=ncell)
    invd = rng.uniform(0.5, 2.0, size=ncell) if jacobi else None
    phi0 = rng.normal(size=nghost)                   # the field before: stale values everywhere
    xw, fw = fused(g, invd, x, phi0, num_sms)
    x_new = x.copy()
    for c, v in xw.items():
        x_new[c] = v
    phi_new = phi0.copy()
    for o, v in fw.items():
        phi_new[o] = v
    x_ref, phi_ref = three_kernels(g, invd, x, phi0)
    np.testing.assert_array_equal(x_new, x_ref)
    np.testing.assert_array_equal(phi_new, phi_ref)
    # the same cells the oracle's CopyTo + ExchangeHaloCells write
    og = O.make_grid(dim, n, None, ng, periodic)
    phi_o = phi0.copy()
    O.copy_to_field(og, x_ref, phi_o)
    O.exchange_halo(og, phi_o)
    np.testing.assert_array_equal(phi_new, phi_o)


def test_grids_the_fused_exit_refuses():
    """A periodic dimension with fewer cells than ghost layers: the images
    would not cover the ghosts, so the solve keeps the three kernels."""
    assert not fused_ok(grid_dev(1, (1,), 2, (1,)))
    assert not fused_ok(grid_dev(3, (4, 2, 4), 3, (0, 1, 0)))
    assert fused_ok(grid_dev(3, (4, 1, 4), 3, (0, 0, 0)))
