"""The 3-D assembly's 16-byte paired staging, checked on the CPU.

k_assemble3 (dare_b200/csrc/dare_assembly3.cu) stages, per plane, a phi
tile with its two-cell halo (12 rows of 36), phi_old and the face arrays of
its 32 x 8 cells.  With an even n2 and ghost width (the PAIR form) it copies
pairs of cells with one 16-byte copy: the phi tile, phi_old, the x faces and
the y faces of the velocity and of face D; the z faces (rows of n2 + 1)
stay single.  This restates both copy assignments and checks, for edge and
inner tiles, both periodicities, face D and ghost widths 2 and 4, that the
paired one fills exactly the same shared-memory elements from the same
source cells (zero past the grid) as the per-cell one, each element once,
every 16-byte copy aligned in shared and global memory.
"""
import itertools

import pytest

import itertools
K, J = 32, 8; PW, PH = K + 4, J + 4; PHI = PW * PH; CELL = K * J
FY = (J + 1) * K; FZW = K + 1; FZ = J * FZW
OffPO = PHI; OffVX = OffPO + CELL; OffVY = OffVX + CELL; OffVZ = OffVY + FY; OffDX = OffVZ + FZ; OffDY = OffDX + CELL; OffDZ = OffDY + FY

def old_map(tid, j0, k0, n1, n2, og1, og2, gn1, gn2, p1, p2, fd):
    m = {}
    lane, ty = tid % K, tid // K
    jj, kk = j0 + ty, k0 + lane
    active = kk < n2 and jj < n1
    for h in range(2):
        e = tid + h * 256
        if e < PHI:
            j = j0 - 2 + e // PW; k = k0 - 2 + e % PW
            off = (j + og1) * gn2 + k + og2 if (0 <= j + og1 < gn1 and 0 <= k + og2 < gn2) else -1
            m[e] = ('phi', off)
        if e < FY:
            f = j0 + e // K; k = k0 + e % K
            if f == n1 and p1: f = 0
            off = f * n2 + k if (f <= n1 and k < n2) else -1
            m[OffVY + e] = ('vy', off)
            if fd: m[OffDY + e] = ('dy', off)
    cell_gh = (jj + og1) * gn2 + kk + og2
    m[OffPO + tid] = ('old', cell_gh if active else -1)
    m[OffVX + tid] = ('vx', jj * n2 + kk if active else -1)
    if fd: m[OffDX + tid] = ('dx', jj * n2 + kk if active else -1)
    return m

def new_map(tid, j0, k0, n1, n2, og1, og2, gn1, gn2, p1, p2, fd):
    m = {}
    def put(sm, arr, off, nb=2):
        assert (sm * 8) % (8 * nb) == 0, ('dst align', arr, sm)
        if off >= 0: assert (off * 8) % (8 * nb) == 0, ('src align', arr, off)
        for c in range(nb): m[sm + c] = (arr, off + c if off >= 0 else -1)
    if tid < PHI // 2:
        row = tid // (PW // 2); col = 2 * (tid - row * (PW // 2))
        j = j0 - 2 + row; k = k0 - 2 + col
        off = (j + og1) * gn2 + k + og2 if (0 <= j + og1 < gn1 and 0 <= k + og2 < gn2) else -1
        put(row * PW + col, 'phi', off)
    t2 = tid & 127; row = t2 >> 4; c2 = 2 * (t2 & 15)
    pj, pk = j0 + row, k0 + c2; act = pj < n1 and pk < n2
    if tid < 128:
        put(OffPO + row * K + c2, 'old', (pj + og1) * gn2 + pk + og2 if act else -1)
        if fd: put(OffDX + row * K + c2, 'dx', pj * n2 + pk if act else -1)
    else:
        put(OffVX + row * K + c2, 'vx', pj * n2 + pk if act else -1)
    if tid < FY // 2:
        row = tid >> 4; c2 = 2 * (tid & 15)
        f = j0 + row; k = k0 + c2
        if f == n1 and p1: f = 0
        off = f * n2 + k if (f <= n1 and k < n2) else -1
        put(OffVY + row * K + c2, 'vy', off)
        if fd: put(OffDY + row * K + c2, 'dy', off)
    return m



@pytest.mark.parametrize("og", [2, 4])
@pytest.mark.parametrize("fd", [0, 1])
def test_paired_staging_fills_the_same_elements(og, fd):
    tiles = 0
    for n1, n2 in [(8, 32), (9, 34), (16, 64), (17, 66), (5, 10), (3, 6), (64, 256), (23, 70)]:
        for p1, p2 in itertools.product([0, 1], [0, 1]):
            gn1, gn2 = n1 + 2 * og, n2 + 2 * og
            for j0 in range(0, n1, J):
                for k0 in range(0, n2, K):
                    mo, mn = {}, {}
                    for tid in range(256):
                        for e, v in old_map(tid, j0, k0, n1, n2, og, og, gn1, gn2, p1, p2, fd).items():
                            assert e not in mo
                            mo[e] = v
                        for e, v in new_map(tid, j0, k0, n1, n2, og, og, gn1, gn2, p1, p2, fd).items():
                            assert e not in mn, ("written twice", e)
                            mn[e] = v
                    assert mn == mo, (n1, n2, p1, p2, j0, k0)
                    tiles += 1
    assert tiles > 0
