"""The slicing of dare_timesteps_host, checked on the CPU.

On single-component 3-D grids the host-resident time loop
(dare_b200/csrc/dare_step.cu) uploads the ghosted field in 16 slices
of whole 4 KB multiples and, as each slice lands, assembles the internal
planes whose stencil it completes: internal plane i reads the ghosted planes
i + og0 - 2 .. i + og0 + 2 (og0 = ghost layers), so after the bytes
[0, end) have landed the planes below floor(end / plane) - 2 - og0 are ready.
This restates that arithmetic and checks, for grid sizes and ghost widths
the API accepts, that every internal plane is assembled exactly once, in
order, and never before every ghosted plane its stencil reads is on the
device.
"""
import pytest

CHUNKS = 16


def slices(n0, n1, n2, ng):
    gn0, gn1, gn2 = n0 + 2 * ng, n1 + 2 * ng, n2 + 2 * ng
    total = gn0 * gn1 * gn2 * 8
    chunk = (total + CHUNKS - 1) // CHUNKS
    chunk = (chunk + 4095) // 4096 * 4096
    plane_bytes = gn1 * gn2 * 8
    nslices = 0
    for c in range(CHUNKS):
        if c * chunk >= total:
            break
        nslices = c + 1
    done, out = 0, []
    for c in range(nslices):
        off = c * chunk
        length = min(chunk, total - off)
        planes_in = gn0 if c == nslices - 1 else (off + length) // plane_bytes
        upto = min(max(planes_in - 2 - ng, 0), n0)
        if c == nslices - 1:
            upto = n0
        if upto > done:
            out.append((c, off + length, done, upto))
            done = upto
    return out, plane_bytes, total


@pytest.mark.parametrize("ng", [2, 3])
@pytest.mark.parametrize("n", [(3, 3, 3), (4, 5, 6), (16, 16, 16), (20, 20, 20), (24, 24, 24), (33, 7, 129),
                               (64, 64, 64), (128, 64, 32), (256, 256, 256), (17, 300, 5)])
def test_every_plane_assembled_once_after_its_stencil_landed(n, ng):
    n0 = n[0]
    ranges, plane_bytes, total = slices(*n, ng)
    covered = []
    for c, landed, ib, ie in ranges:
        covered.extend(range(ib, ie))
        # the last ghosted plane the range reads: (ie - 1) + ng + 2
        last_needed = (ie - 1) + ng + 2
        assert (last_needed + 1) * plane_bytes <= landed or landed == total, (c, ib, ie)
    assert covered == list(range(n0))
