"""Slab decomposition of the implicit step's solve (the reference's MPI
distribution, restated in oracle/slabs.py for the multi-GPU slab path): a
rank owns runs of i-planes, exchanges one boundary plane with each
i-neighbour before every SpMV and sums every dot product over ranks.  Run as
gloo ranks on CPU and checked against the serial oracle solve."""
import json
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import oracle as O
from oracle import slabs as S
from tests.helpers import interleave_csr, oracle_assembly, oracle_grid, oracle_timeloop

N = (9, 6, 5)


def _system(periodic, seed=21):
    """A TVD convection-diffusion implicit step (van Leer, diffusion, DDT) as
    the oracle assembles and exports it."""
    rng = np.random.default_rng(seed)
    case = {"n": N, "size": (1.0, 0.8, 1.3), "periodic": periodic, "dt": 0.02, "D": 3e-3,
            "phi0": rng.random(tuple(x + 4 for x in N)), "limiter": "VANLEER",
            "face_vel": [rng.normal(size=tuple(x + (1 if e == d else 0) for e, x in enumerate(N)))
                         for d in range(3)]}
    # a non-periodic axis gets a Dirichlet face below and a Neumann face above
    case["bc"] = {2 * d + 1: (1, 1.0 + d) for d in range(3) if not periodic[d]}
    case["bc"].update({2 * d + 2: (2, 0.0) for d in range(3) if not periodic[d]})
    og = oracle_grid(case)
    phi = np.ascontiguousarray(case["phi0"].reshape(-1))
    diag, rhs, mask = O.assemble(oracle_assembly(og, case), phi, phi)
    rp, cols, vals = O.export_csr(og, diag, mask)
    x0 = O.field_to_vector(og, phi)
    tol = 1e-12 * float(np.linalg.norm(rhs))
    return rp, cols, vals, rhs, x0, tol


def _serial(periodic, jacobi):
    rp, cols, vals, rhs, x0, tol = _system(periodic)
    slab = S.Slab(N, rp, cols, vals, 0, N[0], bool(periodic[0]))
    return S.bicgstab2(slab, S.Comm(None, 0, 1, bool(periodic[0])), rhs, x0, tol, 500, jacobi)


@pytest.mark.parametrize("jacobi", [False, True])
def test_serial_restatement_matches_oracle(jacobi):
    periodic = (1, 1, 1)
    rp, cols, vals, rhs, x0, tol = _system(periodic)
    x, info = _serial(periodic, jacobi)
    ox, oinfo = O.bicgstab2(rp, cols, vals, rhs, x0, tol, 500, O.PREC_JACOBI if jacobi else O.PREC_NONE)
    assert info["converged"] and oinfo["converged"]
    assert abs(info["iters"] - oinfo["iters"]) <= 1
    assert np.linalg.norm(x - ox) <= 1e-10 * np.linalg.norm(ox)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, periodic, jacobi, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rp, cols, vals, rhs, x0, tol = _system(periodic)
    i0, i1 = S.slab_range(N[0], world, rank)
    P = N[1] * N[2]
    slab = S.Slab(N, rp, cols, vals, i0, i1, bool(periodic[0]))
    x, info = S.bicgstab2(slab, S.Comm(dist, rank, world, bool(periodic[0])), rhs[i0 * P:i1 * P],
                          x0[i0 * P:i1 * P], tol, 500, jacobi)
    dist.barrier()
    dist.destroy_process_group()
    np.save(os.path.join(out, f"x{rank}.npy"), x)
    with open(os.path.join(out, f"i{rank}.json"), "w") as fh:
        json.dump({"i0": i0, "i1": i1, **{k: float(v) for k, v in info.items()}}, fh)


@pytest.mark.parametrize("world,periodic,jacobi", [(2, (1, 1, 1), False), (3, (1, 0, 1), True),
                                                   (2, (0, 1, 1), True)])
def test_slab_ranks_match_serial_solve(tmp_path, world, periodic, jacobi):
    mp.spawn(_rank, args=(world, _free_port(), periodic, jacobi, str(tmp_path)), nprocs=world, join=True)
    infos = [json.load(open(tmp_path / f"i{r}.json")) for r in range(world)]
    # the slabs tile the planes in order
    assert infos[0]["i0"] == 0 and infos[-1]["i1"] == N[0]
    assert all(infos[r]["i1"] == infos[r + 1]["i0"] for r in range(world - 1))
    # every rank takes the same decisions (the scalars come from the same sums)
    assert len({(i["iters"], i["status"], i["converged"]) for i in infos}) == 1
    x = np.concatenate([np.load(tmp_path / f"x{r}.npy") for r in range(world)])
    sx, sinfo = _serial(periodic, jacobi)
    rp, cols, vals, rhs, x0, tol = _system(periodic)
    ox, oinfo = O.bicgstab2(rp, cols, vals, rhs, x0, tol, 500, O.PREC_JACOBI if jacobi else O.PREC_NONE)
    assert infos[0]["converged"] == 1
    assert abs(infos[0]["iters"] - sinfo["iters"]) <= 1 and abs(infos[0]["iters"] - oinfo["iters"]) <= 1
    # partial sums are added in another order across ranks: rounding-level differences only
    assert np.linalg.norm(x - sx) <= 1e-10 * np.linalg.norm(sx)
    assert np.linalg.norm(x - ox) <= 1e-9 * np.linalg.norm(ox)


def _system2(periodic):
    """Two components, each its own velocity and field (no coupling), rows
    and columns cell * 2 + c."""
    a, b = _system(periodic, 21), _system(periodic, 22)
    rp, cols, vals = interleave_csr([a[:3], b[:3]])
    rhs = np.stack([a[3], b[3]], axis=1).reshape(-1)
    x0 = np.stack([a[4], b[4]], axis=1).reshape(-1)
    return rp, cols, vals, rhs, x0, 1e-12 * float(np.linalg.norm(rhs))


def _rank2(rank, world, port, periodic, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rp, cols, vals, rhs, x0, tol = _system2(periodic)
    i0, i1 = S.slab_range(N[0], world, rank)
    P = N[1] * N[2] * 2
    slab = S.Slab(N, rp, cols, vals, i0, i1, bool(periodic[0]), ncomp=2)
    x, info = S.bicgstab2(slab, S.Comm(dist, rank, world, bool(periodic[0])), rhs[i0 * P:i1 * P],
                          x0[i0 * P:i1 * P], tol, 500, True)
    dist.barrier()
    dist.destroy_process_group()
    np.save(os.path.join(out, f"x{rank}.npy"), x)
    with open(os.path.join(out, f"i{rank}.json"), "w") as fh:
        json.dump({k: float(v) for k, v in info.items()}, fh)


def test_slab_ranks_two_components(tmp_path):
    periodic = (1, 1, 1)
    mp.spawn(_rank2, args=(2, _free_port(), periodic, str(tmp_path)), nprocs=2, join=True)
    infos = [json.load(open(tmp_path / f"i{r}.json")) for r in range(2)]
    assert infos[0] == infos[1] and infos[0]["converged"] == 1
    x = np.concatenate([np.load(tmp_path / f"x{r}.npy") for r in range(2)])
    rp, cols, vals, rhs, x0, tol = _system2(periodic)
    ox, oinfo = O.bicgstab2(rp, cols, vals, rhs, x0, tol, 500, O.PREC_JACOBI)
    assert abs(infos[0]["iters"] - oinfo["iters"]) <= 1
    assert np.linalg.norm(x - ox) <= 1e-9 * np.linalg.norm(ox)


def test_slab_assembly_from_two_halo_planes():
    """A rank assembles its own rows from its planes of phi and phi_old plus
    two planes from each i-neighbour (the van Leer face of cell i reads
    i - 2: HaloBuffer's ghost width is 2) and its slice of the face
    velocities; the result is the global assembly's rows, bit for bit.
    (A slab is emulated as a grid periodic along i whose ghost planes hold
    the neighbours' planes.  On a periodic axis the staggered field's last
    face is its first (CartesianRepresentation.inl:64-76), so the i-faces
    here do not vary along i: the slab's upper face then equals the
    neighbour's first face either way.)"""
    n0, n1, n2 = 10, 6, 5
    h = 0.125   # dx exactly representable, hence the same on every slab
    rng = np.random.default_rng(5)
    phi = rng.random((n0 + 4, n1 + 4, n2 + 4))
    old = rng.random((n0 + 4, n1 + 4, n2 + 4))
    fv = [rng.normal(size=tuple(x + (1 if e == d else 0) for e, x in enumerate((n0, n1, n2)))) for d in range(3)]
    fv[0] = np.ascontiguousarray(np.broadcast_to(fv[0][:1], fv[0].shape))
    case = {"n": (n0, n1, n2), "size": (n0 * h, 0.75, 1.25), "periodic": (1, 1, 1), "dt": 0.02, "D": 3e-3,
            "limiter": "VANLEER", "face_vel": fv}
    og = oracle_grid(case)
    pf, of = phi.reshape(-1).copy(), old.reshape(-1).copy()
    O.exchange_halo(og, pf)
    O.exchange_halo(og, of)
    diag, rhs, _ = O.assemble(oracle_assembly(og, case), pf, of)
    phi3, old3 = pf.reshape(phi.shape), of.reshape(old.shape)
    P = n1 * n2
    for world in (2, 3):
        for rank in range(world):
            i0, i1 = S.slab_range(n0, world, rank)
            nl = i1 - i0
            # ghosted planes of the slab = global ghosted planes i0 .. i1 + 3
            lp = np.ascontiguousarray(phi3[i0:i1 + 4]).reshape(-1)
            lo = np.ascontiguousarray(old3[i0:i1 + 4]).reshape(-1)
            lcase = dict(case, n=(nl, n1, n2), size=(nl * h, 0.75, 1.25),
                         face_vel=[np.ascontiguousarray(fv[0][i0:i1 + 1]), np.ascontiguousarray(fv[1][i0:i1]),
                                   np.ascontiguousarray(fv[2][i0:i1])])
            desc = oracle_assembly(oracle_grid(lcase), lcase)
            ld, lr, _ = O.assemble(desc, lp, lo)
            assert np.array_equal(ld, diag[:, i0 * P:i1 * P]) and np.array_equal(lr, rhs[i0 * P:i1 * P])
            # with only one halo plane per side the TVD corrections differ
            bad = lp.reshape(nl + 4, n1 + 4, n2 + 4).copy()
            bad[0] += 10.0
            bad[-1] += 10.0
            bd, br, _ = O.assemble(desc, np.ascontiguousarray(bad.reshape(-1)), lo)
            assert not np.array_equal(br, rhs[i0 * P:i1 * P])


STEPS = 2


def _steps_case():
    """A periodic van Leer convection-diffusion case whose i-faces do not vary
    along i (see the assembly test) and whose ghosts are already exchanged."""
    n0, n1, n2, h = 10, 6, 5, 0.125
    rng = np.random.default_rng(9)
    fv = [rng.normal(size=tuple(x + (1 if e == d else 0) for e, x in enumerate((n0, n1, n2)))) for d in range(3)]
    fv[0] = np.ascontiguousarray(np.broadcast_to(fv[0][:1], fv[0].shape))
    case = {"n": (n0, n1, n2), "size": (n0 * h, 0.75, 1.25), "periodic": (1, 1, 1), "dt": 0.02, "D": 3e-3,
            "limiter": "VANLEER", "face_vel": fv, "rel_tol": 1e-12}
    phi = rng.random((n0 + 4) * (n1 + 4) * (n2 + 4))
    O.exchange_halo(oracle_grid(case), phi)
    case["phi0"] = phi.reshape(n0 + 4, n1 + 4, n2 + 4)
    return case, h


def _rank_steps(rank, world, port, out):
    """One rank of the distributed driver loop: assemble the slab, solve it,
    copy back, exchange two halo planes of the field, keep it as the old level."""
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    case, h = _steps_case()
    n0, n1, n2 = case["n"]
    i0, i1 = S.slab_range(n0, world, rank)
    nl = i1 - i0
    fv = case["face_vel"]
    lcase = dict(case, n=(nl, n1, n2), size=(nl * h, 0.75, 1.25),
                 face_vel=[np.ascontiguousarray(fv[0][i0:i1 + 1]), np.ascontiguousarray(fv[1][i0:i1]),
                           np.ascontiguousarray(fv[2][i0:i1])])
    lg = oracle_grid(lcase)
    desc = oracle_assembly(lg, lcase)
    comm = S.Comm(dist, rank, world, True)
    phi = np.ascontiguousarray(case["phi0"][i0:i1 + 4]).reshape(-1).copy()
    old = phi.copy()
    iters = []
    for _ in range(STEPS):
        diag, rhs, mask = O.assemble(desc, phi, old)
        slab = S.Slab.from_local((nl, n1, n2), *O.export_csr(lg, diag, mask))
        x0 = O.field_to_vector(lg, phi)
        tol = case["rel_tol"] * float(np.sqrt(comm.allsum([float(np.dot(rhs, rhs))])[0]))
        x, info = S.bicgstab2(slab, comm, rhs, x0, tol, 5000, True)
        O.copy_to_field(lg, x, phi)
        O.exchange_halo(lg, phi)            # the j and k ghosts (its i ghosts are replaced next)
        f3 = phi.reshape(nl + 4, n1 + 4, n2 + 4)
        below, above = comm.swap(f3[2:4].copy(), f3[nl:nl + 2].copy())
        f3[0:2], f3[nl + 2:nl + 4] = below, above
        old[:] = phi
        iters.append(info["iters"])
    dist.barrier()
    dist.destroy_process_group()
    np.save(os.path.join(out, f"f{rank}.npy"), phi.reshape(nl + 4, n1 + 4, n2 + 4)[2:nl + 2])
    with open(os.path.join(out, f"s{rank}.json"), "w") as fh:
        json.dump({"iters": iters}, fh)


@pytest.mark.parametrize("world", [2, 3])
def test_slab_time_steps_match_serial_loop(tmp_path, world):
    """The reference's driver loop (Build, Solve, CopyTo, ExchangeHaloCells,
    CopyDataVectorsToOldTimeStep) distributed over slabs gives the serial
    loop's field."""
    mp.spawn(_rank_steps, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    case, _ = _steps_case()
    hist, siters = oracle_timeloop(case, STEPS)
    n0, n1, n2 = case["n"]
    want = hist[-1].reshape(n0 + 4, n1 + 4, n2 + 4)[2:n0 + 2]
    got = np.concatenate([np.load(tmp_path / f"f{r}.npy") for r in range(world)])
    iters = [json.load(open(tmp_path / f"s{r}.json"))["iters"] for r in range(world)]
    assert all(it == iters[0] for it in iters)
    assert all(abs(a - b) <= 1 for a, b in zip(iters[0], siters))
    assert np.linalg.norm(got - want) <= 1e-10 * np.linalg.norm(want)
