"""The tiling of the bulk-staged CG vector kernels (csrc/solver_kernels.cuh,
`cg_update_bulk_kernel` / `cg_pupdate_bulk_kernel`), restated and checked:
the (column, chunk) items cover each column exactly, every bulk copy is
16-byte aligned with a size that is a multiple of 16 bytes and fits its
4 KB stage, and the stage / mbarrier-parity sequence a CTA waits on matches
the copies it issued, across the items of a grid-stride loop. No GPU needed."""
import pytest

STAGES, TILE_BYTES = 2, 4096


def items(colstride, nchunks, elem):
    """(e0, e1) element range of each chunk of a column: whole 16-byte groups."""
    v = 16 // elem
    ng = colstride // v
    return [(ng * c // nchunks * v, ng * (c + 1) // nchunks * v) for c in range(nchunks)]


def cta_schedule(ranges, elem):
    """Per tile, in the order one CTA handles its items: (issue stage, wait
    stage, wait parity, byte offset, bytes), with tiles counted over items."""
    te = TILE_BYTES // elem
    g0, out = 0, []
    for e0, e1 in ranges:
        ntile = -(-(e1 - e0) // te)
        issued = {}
        for t in range(min(STAGES, ntile)):
            issued[t] = (g0 + t) % STAGES
        for t in range(ntile):
            g = g0 + t
            b0 = e0 + t * te
            nbytes = min(te, e1 - b0) * elem
            out.append((issued[t], g % STAGES, (g // STAGES) & 1, b0 * elem, nbytes))
            if t + STAGES < ntile:
                issued[t + STAGES] = (g0 + t + STAGES) % STAGES
        g0 += ntile
    return out


@pytest.mark.parametrize("elem", [4, 8])
@pytest.mark.parametrize("n1, n2, n3", [(9, 17, 17), (9, 33, 33), (21, 81, 81), (33, 129, 129), (11, 11, 11),
                                        (13, 13, 13), (25, 25, 25)])
def test_tiles_cover_columns_and_stay_aligned(elem, n1, n2, n3):
    ps = -(-n1 * n2 // 4) * 4                      # plane padded to 4 elements
    colstride = 6 * n3 * ps
    nchunks = max(1, -(-colstride // 16384))
    assert colstride * elem % 16 == 0               # every column starts on a 16-byte boundary
    ranges = items(colstride, nchunks, elem)
    assert ranges[0][0] == 0 and ranges[-1][1] == colstride
    assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
    assert all(e1 > e0 for e0, e1 in ranges)
    for ncta_items in (1, 2, 5, len(ranges)):       # items one CTA takes in its grid-stride loop
        sched = cta_schedule(ranges[:ncta_items], elem)
        covered = []
        for issue_stage, wait_stage, parity, off, nbytes in sched:
            assert issue_stage == wait_stage         # the copy lands where the CTA waits
            assert off % 16 == 0 and nbytes % 16 == 0 and 0 < nbytes <= TILE_BYTES
            covered.append((off, off + nbytes))
        # every stage's waits alternate parity 0, 1, 0, ... (one phase per tile)
        for s in range(STAGES):
            par = [p for _, st, p, _, _ in sched if st == s]
            assert par == [i & 1 for i in range(len(par))]
        # tiles of the CTA's items cover those items exactly
        want = []
        for e0, e1 in ranges[:ncta_items]:
            want.append((e0 * elem, e1 * elem))
        got, k = [], 0
        for e0, e1 in ranges[:ncta_items]:
            lo = e0 * elem
            while k < len(covered) and covered[k][0] < e1 * elem:
                assert covered[k][0] == lo
                lo = covered[k][1]
                k += 1
            got.append((e0 * elem, lo))
        assert got == want
