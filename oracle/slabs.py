"""Slab decomposition of the implicit step's solve over ranks: the
reference's MPI distribution restated on CPU processes.

TEST INFRASTRUCTURE ONLY: this pins the semantics of a distributed solve
(which rows a rank owns, which values cross between ranks, where the
reductions sit) for the multi-GPU slab path.  Nothing in the product
imports it; tests run it as torch.distributed gloo ranks.

The reference distributes the Cartesian grid over MPI ranks
(Grid/Cartesian/CartesianDistribution.h:94-380); a rank's matrix rows are
its own cells, the columns of a 7-point row reach the ghost layer filled by
HaloBuffer::Exchange (MPI/HaloBuffer.inl:30-208), Tpetra imports the SpMV
operand's off-rank entries once per A.apply, and every dot product and norm
of BiCGStab2 (BiCGStab2.inl:339, 368, 408, 431, 488-501, 559) is one
MPI_Allreduce.  Here the slabs are runs of whole i-planes, the import is the
exchange of one boundary plane with each i-neighbour, and the reductions are
all_reduce(SUM) of the ranks' partial dots.

`bicgstab2` follows the oracle's dor_bicgstab2 (oracle/dare_oracle.c) step
for step -- itself the restatement of BiCGStab2.inl:166-582 -- with the
vector operations on the rank's rows and the two exchange points pluggable;
with one rank it is the serial solve.
"""
from __future__ import annotations

import numpy as np

LD = np.longdouble  # the reference keeps omega, mu, nu, tau in long double


def slab_range(n0: int, world: int, rank: int):
    """Planes [i0, i1) of `rank`: n0 split into `world` runs, the first
    n0 % world of them one plane longer."""
    base, extra = divmod(n0, world)
    i0 = rank * base + min(rank, extra)
    return i0, i0 + base + (1 if rank < extra else 0)


class Slab:
    """The rows of one rank: CSR rows of the cells of planes [i0, i1) with
    their columns renumbered into the extended local vector
    [plane i0 - 1 | own planes | plane i1] (the halo planes, wrapped when
    the grid is periodic along i).  With `ncomp` components the rows and
    columns are cell * ncomp + c (MatrixBlock_Cartesian.inl:127-240), so a
    plane holds n1 n2 ncomp entries."""

    def __init__(self, n, rowptr, cols, vals, i0: int, i1: int, periodic_i: bool, ncomp: int = 1):
        n0, n1, n2 = n
        self.P = n1 * n2 * ncomp
        self.n0, self.i0, self.i1 = n0, i0, i1
        self.periodic_i = periodic_i
        r0, r1 = i0 * self.P, i1 * self.P
        self.nrows = r1 - r0
        lo = rowptr[r0]
        self.rowptr = (rowptr[r0:r1 + 1] - lo).astype(np.int64)
        gcols = cols[lo:rowptr[r1]].astype(np.int64)
        self.vals = vals[lo:rowptr[r1]].astype(np.float64)
        plane = gcols // self.P
        inplane = gcols - plane * self.P
        # plane offset relative to the slab: -1 (lower halo), 0 .. nplanes-1, nplanes (upper halo)
        rel = plane - i0
        if periodic_i and n0 > 1:
            rel = np.where(rel < -1, rel + n0, rel)
            rel = np.where(rel > (i1 - i0), rel - n0, rel)
        if np.any(rel < -1) or np.any(rel > i1 - i0):
            raise ValueError("a row reaches past the neighbouring planes: not a 7-point slab")
        self.lcols = (rel + 1) * self.P + inplane   # index into [halo_lo | own | halo_hi]

    @classmethod
    def from_local(cls, n_local, rowptr, cols, vals, ncomp: int = 1):
        """A slab from the CSR a rank exports for its own grid of n_local[0]
        planes numbered as if periodic along i: a column one plane below the
        first plane (or above the last) wrapped onto the far plane, and is
        renumbered into the halo by its plane offset from the row
        (needs at least three planes)."""
        nl = n_local[0]
        if nl < 3:
            raise ValueError("a slab of fewer than three planes cannot tell a wrapped column from an own one")
        self = cls.__new__(cls)
        self.P = n_local[1] * n_local[2] * ncomp
        self.n0, self.i0, self.i1, self.periodic_i = nl, 0, nl, True
        self.nrows = nl * self.P
        self.rowptr = np.asarray(rowptr, dtype=np.int64)
        self.vals = np.asarray(vals, dtype=np.float64)
        gcols = np.asarray(cols, dtype=np.int64)
        rplane = np.repeat(np.arange(self.nrows) // self.P, np.diff(self.rowptr))
        cplane = gcols // self.P
        delta = (cplane - rplane + 1) % nl - 1
        if np.any(delta > 1):
            raise ValueError("a row reaches past the neighbouring planes: not a 7-point slab")
        self.lcols = (rplane + delta + 1) * self.P + (gcols - cplane * self.P)
        return self

    def spmv(self, xext: np.ndarray) -> np.ndarray:
        """y = A x for the own rows; `xext` is the extended local vector."""
        prod = self.vals * xext[self.lcols]
        y = np.empty(self.nrows)
        for r in range(self.nrows):  # the oracle's row order of additions
            s = 0.0
            for p in range(self.rowptr[r], self.rowptr[r + 1]):
                s += prod[p]
            y[r] = s
        return y


class Comm:
    """The exchange points of a distributed solve over torch.distributed
    (gloo on CPU): the halo planes of an SpMV operand, and sums over ranks."""

    def __init__(self, dist, rank: int, world: int, periodic_i: bool):
        self.dist, self.rank, self.world, self.periodic_i = dist, rank, world, periodic_i

    def _neighbours(self):
        lo = self.rank - 1 if self.rank > 0 else (self.world - 1 if self.periodic_i else None)
        hi = self.rank + 1 if self.rank < self.world - 1 else (0 if self.periodic_i else None)
        return lo, hi

    def swap(self, first: np.ndarray, last: np.ndarray):
        """Sends `first` (this rank's lowest planes) to the lower neighbour and
        `last` (its highest) to the upper one; returns what they sent in
        return: (the lower neighbour's highest planes, the upper neighbour's
        lowest).  Zeros where there is no neighbour."""
        below, above = np.zeros_like(first), np.zeros_like(last)
        lo, hi = self._neighbours()
        if self.world == 1:
            if self.periodic_i:
                below, above = last.copy(), first.copy()
            return below, above
        import torch
        t_below, t_above = torch.from_numpy(below), torch.from_numpy(above)
        reqs = []
        # tag 0: planes travelling up (my highest are the upper rank's lower halo), tag 1: down
        if lo is not None:
            reqs.append(self.dist.irecv(t_below, src=lo, tag=0))
            reqs.append(self.dist.isend(torch.from_numpy(np.ascontiguousarray(first)), dst=lo, tag=1))
        if hi is not None:
            reqs.append(self.dist.irecv(t_above, src=hi, tag=1))
            reqs.append(self.dist.isend(torch.from_numpy(np.ascontiguousarray(last)), dst=hi, tag=0))
        for r in reqs:
            r.wait()
        return below, above

    def extend(self, x: np.ndarray, P: int) -> np.ndarray:
        """[plane below | x | plane above], the planes from the neighbouring
        ranks (zeros where there is none: those columns do not occur)."""
        below, above = self.swap(x[:P], x[-P:])
        return np.concatenate([below, x, above])

    def allsum(self, values) -> np.ndarray:
        """Sums over ranks of a vector of partial sums (one all_reduce)."""
        v = np.asarray(values, dtype=np.float64)
        if self.world == 1:
            return v
        import torch
        t = torch.from_numpy(v.copy())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return t.numpy()


def bicgstab2(slab: Slab, comm: Comm, b: np.ndarray, x: np.ndarray, tol: float, max_it: int, jacobi: bool):
    """dor_bicgstab2 on the rank's rows (b, x: its slices of the global
    vectors).  Returns (x, info) with info = {status, converged, iters, res}."""
    P = slab.P
    dot = lambda a, c: float(comm.allsum([float(np.dot(a, c))])[0])
    norm2 = lambda a: float(np.sqrt(dot(a, a)))
    inv_diag = None
    if jacobi:
        d = np.zeros(slab.nrows)
        own = slab.lcols - P  # column of the own cell is row index r
        for r in range(slab.nrows):
            for p in range(slab.rowptr[r], slab.rowptr[r + 1]):
                if own[p] == r:
                    d[r] = slab.vals[p]
        inv_diag = 1.0 / d

    def apply_op(src):
        if jacobi:
            src = inv_diag * src
        return slab.spmv(comm.extend(src, P))

    info = {"status": 0, "converged": 0, "iters": 0, "res": 0.0}
    n = slab.nrows
    x = x.astype(np.float64).copy()
    x0 = x.copy()
    r = b.astype(np.float64).copy()
    if jacobi:
        x0 = inv_diag * x0
    v = slab.spmv(comm.extend(x0, P))          # (0) r = r_hat_0 = b - A x0
    r = 1.0 * r + (-1.0) * v
    r_hat_0 = r.copy()
    u, v, w = np.zeros(n), np.zeros(n), np.zeros(n)   # (1)
    rho = [1.0, 0.0]
    omega_1 = omega_2 = LD(1.0)
    alpha, k = 0.0, 0
    r_norm_0 = norm2(r)
    conv = r_norm_0
    if conv < tol:
        info.update(iters=k, res=conv, converged=1)
        return x0, info
    k += 1
    s = t = None
    while True:
        if k > max_it:
            break
        rho[0] = float(-omega_2 * LD(rho[0]))    # (3)
        if rho[0] == 0.0:
            info["status"] = 3
            break
        rho[1] = dot(r_hat_0, r)                   # (4)
        beta = alpha * rho[1] / rho[0]
        rho[0] = rho[1]
        if rho[0] == 0.0:
            info["status"] = 4
            break
        u = 1.0 * r + (-beta) * u                  # (5)
        v = apply_op(u)                            # (6)
        gamma = dot(v, r_hat_0)                    # (7)
        if gamma == 0.0:
            info["status"] = 7
            break
        alpha = rho[0] / gamma
        r = (-alpha) * v + 1.0 * r                 # (8)
        s = apply_op(r)                            # (9)
        x = alpha * u + 1.0 * x                    # (10)
        rho[1] = dot(r_hat_0, s)                   # (11)
        beta = alpha * rho[1] / rho[0]
        rho[0] = rho[1]
        v = 1.0 * s + (-beta) * v                  # (12)
        w = apply_op(v)                            # (13)
        gamma = dot(w, r_hat_0)                    # (14)
        if gamma == 0.0:
            info["status"] = 14
            break
        alpha = rho[0] / gamma
        u = 1.0 * r + (-beta) * u                  # (15)
        r = (-alpha) * v + 1.0 * r                 # (16)
        s = (-alpha) * w + 1.0 * s                 # (17)
        t = apply_op(s)                            # (18)
        # (19), (20): five dot products, one all_reduce as Tpetra's fused reductions would need
        part = [float(np.dot(r, s)), float(np.dot(s, s)), float(np.dot(s, t)), float(np.dot(t, t)),
                float(np.dot(r, t))]
        tot = comm.allsum(part)
        omega_1, mu, nu, tau, omega_2 = (LD(float(z)) for z in tot)
        if mu == 0.0:
            info["status"] = 20
            break
        tau -= nu * nu / mu                        # (21)
        if tau == 0.0:
            # BiCGStab2.inl:407-424: the true residual decides; when it does
            # not converge the common exit applies M^-1 a second time
            if jacobi:
                x = inv_diag * x
            rr = (-1.0) * slab.spmv(comm.extend(x, P)) + 1.0 * b
            conv = norm2(rr)
            if conv <= tol:
                info.update(converged=1, iters=k, res=conv)
                return x, info
            info["status"] = 21
            break
        omega_2 = (omega_2 - (nu * omega_1) / mu) / tau   # (22), (23)
        omega_1 = (omega_1 - nu * omega_2) / mu
        x = float(omega_1) * r + float(omega_2) * s + 1.0 * x   # (24): alpha a + beta b + gamma z
        x = alpha * u + 1.0 * x
        r = float(-omega_1) * s + float(-omega_2) * t + 1.0 * r  # (25)
        conv = norm2(r)
        if conv <= tol and k > 1:
            break
        u = float(-omega_1) * v + float(-omega_2) * w + 1.0 * u
        k += 1
    if jacobi:
        x = inv_diag * x
    info.update(iters=k, res=conv, converged=int(conv <= tol))
    return x, info
