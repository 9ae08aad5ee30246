"""The marching kernel's 16-byte vector staging, checked on the CPU.

k_march (dare_b200/csrc/dare_march.cuh) with PAIR stages every value as part
of a 16-byte copy: FP64 with one cell per thread (two doubles per copy),
FP32 with two cells per thread (four floats).  Each thread's copies are
computed from its index: operand tile rows j0-1 .. j0+TJ as 16-byte copies
plus the single halo cells k0-1 and k0+TW of the interior rows, and for the
per-cell streams one 16-byte copy per stream of the thread's half.  This
restates that arithmetic and checks, for the tile shapes the solver picks,
that every copy starts on its own size in shared and global memory (a
misaligned cp.async faults), stays inside the stage and the plane, is written
once, and that every value the 7-point row reads comes from the right cell
(periodic wrap, zero past a bounded face) -- before the kernel ever runs.
"""
import itertools

import pytest

import itertools
def jk_offset(j, k, n1, n2, p1, p2):
    if j < 0:
        if not p1: return -1
        j += n1
    elif j >= n1:
        if not p1: return -1
        j -= n1
    if k < 0:
        if not p2: return -1
        k += n2
    elif k >= n2:
        if not p2: return -1
        k -= n2
    if not (0 <= j < n1 and 0 <= k < n2): return -1
    return j * n2 + k

def _check(tsize, CPT, TK, TJ, NZ, NP, n1, n2, p1, p2):
    VEC = 16 // tsize
    TW = TK * CPT; NT = TK * TJ; NCT = TW * TJ
    IC = VEC; W = TW + 2 * IC; H = TJ + 2; ZT = W * H; STAGE = NZ * ZT + NP * NCT
    hw = TW // VEC; SETS = VEC // CPT; nvec = NCT // VEC
    if not (n2 % VEC == 0 and TW % VEC == 0 and (TJ + 2) * hw + 2 * TJ <= NT): return False
    assert STAGE * tsize % 16 == 0 and ZT * tsize % 16 == 0 and NZ * ZT * tsize % 16 == 0
    tiles_x = (n2 + TW - 1) // TW; tiles_y = (n1 + TJ - 1) // TJ
    for tile in range(tiles_x * tiles_y):
        tj0 = (tile // tiles_x) * TJ; tk0 = (tile % tiles_x) * TW
        op_w = {}   # smem elem -> source offset (or -1 zero)
        st_w = {}
        for tid in range(NT):
            par = tid // nvec; e = tid - par * nvec
            pr_row = e // hw; pr_col = VEC * (e - pr_row * hw)
            npr = (TJ + 2) * hw
            kind = 0
            if tid < npr:
                kind = 2; row = tid // hw; dk = VEC * (tid - row * hw); col = IC + dk; nb = 16
            elif tid < npr + 2 * TJ:
                e2 = tid - npr; kind = 1; row = 1 + (e2 >> 1); dk = TW if (e2 & 1) else -1; col = IC + dk; nb = tsize
            if kind:
                o = jk_offset(tj0 - 1 + row, tk0 + dk, n1, n2, p1, p2)
                dst = row * W + col
                assert (dst * tsize) % nb == 0, ('op dst align', tid, dst)
                assert 0 <= dst and dst + nb // tsize <= ZT, ('op dst bounds', tid)
                if o >= 0:
                    assert (o * tsize) % nb == 0, ('op src align', tid, o)
                    assert o + nb // tsize <= n1 * n2, ('op src bounds', tid, o)
                for c in range(nb // tsize):
                    assert dst + c not in op_w, ('op double write', tid)
                    op_w[dst + c] = (o + c) if o >= 0 else -1
            # streams: this thread's pair/quad for q % SETS == par
            pj = tj0 + pr_row; pk = tk0 + pr_col
            o_pair = pj * n2 + pk if (pj < n1 and pk < n2) else -1
            for q in range(NP):
                if q % SETS != par: continue
                dst = NZ * ZT + q * NCT + pr_row * TW + pr_col
                assert (dst * tsize) % 16 == 0 and dst + VEC <= STAGE
                if o_pair >= 0: assert (o_pair * tsize) % 16 == 0 and o_pair + VEC <= n1 * n2
                for c in range(VEC):
                    key = (q, pr_row * TW + pr_col + c)
                    assert key not in st_w
                    st_w[key] = (o_pair + c) if o_pair >= 0 else -1
        # coverage of what the compute reads
        for r in range(TJ):
            for c in range(TW):
                j = tj0 + r; k = tk0 + c
                if not (j < n1 and k < n2): continue
                for (dr, dc) in [(0, 0), (-1, 0), (1, 0), (0, -1), (0, 1)]:
                    elem = (r + 1 + dr) * W + IC + c + dc
                    want = jk_offset(j + dr, k + dc, n1, n2, p1, p2)
                    got = op_w.get(elem, 'missing')
                    assert got == want, ('operand', r, c, dr, dc, got, want)
                for q in range(NP):
                    assert st_w.get((q, r * TW + c)) == j * n2 + k, ('stream', q, r, c)
    return True



@pytest.mark.parametrize("tsize,cpt", [(8, 1), (4, 2)], ids=["fp64-one-cell", "fp32-two-cells"])
@pytest.mark.parametrize("tj", [8, 4])
def test_vector_staging_alignment_bounds_and_coverage(tsize, cpt, tj):
    checked = 0
    for nz, np_ in [(1, 6), (1, 8), (2, 7), (2, 8), (1, 10)]:
        for n1, n2 in [(8, 32), (5, 36), (9, 64), (17, 68), (3, 8), (12, 4)]:
            for p1, p2 in itertools.product([0, 1], [0, 1]):
                checked += _check(tsize, cpt, 32, tj, nz, np_, n1, n2, p1, p2)
    assert checked > 0


@pytest.mark.parametrize("tsize,cpt", [(8, 1), (4, 2)], ids=["fp64-one-cell", "fp32-two-cells"])
def test_flat_tiles_keep_the_per_cell_copies(tsize, cpt):
    """Tiles of one or two rows have fewer threads than operand copies: the
    launch condition refuses the vector staging there (the kernel then copies
    per cell)."""
    for tj in (1, 2):
        assert not _check(tsize, cpt, 32, tj, 2, 7, 9, 64, 1, 1)


def test_a_single_cell_copy_of_the_wrong_size_is_caught():
    """An 8-byte copy of one FP32 halo cell (a development version did this
    and faulted with a misaligned address) fails the alignment check."""
    ns = {"jk_offset": jk_offset}
    code = __import__("inspect").getsource(_check).replace("col = IC + dk; nb = tsize", "col = IC + dk; nb = 8")
    exec(code, ns)
    with pytest.raises(AssertionError):
        ns["_check"](4, 2, 32, 8, 2, 7, 9, 64, 1, 1)
