"""The x3 split of FP64-input stencil launches (csrc/plane_march.cuh, the
segment bounds at the top of `plane_march_kernel`; csrc/eqd_host.cu,
`segmented`), restated here and checked for every axis length and split:
every plane's components are stored by exactly one segment, every value a
segment stores has all its inputs marched inside that segment, and the
step blocks (the units the dot products are summed over) do not depend on
the split. No GPU needed."""
import pytest

PBLK, NSLOT = 8, 6


def segmented(nblk, ctas, num_sms=148):
    """(nseg, segblk) for a launch of `ctas` CTAs (eqd_host.cu `segmented`)."""
    target = 2 * num_sms
    if ctas >= target or nblk <= 1:
        return 1, nblk
    want = min(-(-target // ctas), nblk)
    segblk = -(-nblk // want)
    return -(-nblk // segblk), segblk


def bounds(n3, seg, segblk):
    """The kernel's per-segment bounds."""
    q0 = seg * segblk * PBLK
    q1 = min(q0 + segblk * PBLK, n3)
    blk0 = q0 // PBLK
    nbs = -(-(q1 - q0) // PBLK)
    o_beg = q0 + 3
    s_end = n3 + 6 if q1 == n3 else q1 + 3
    s_beg = (q0 - 9) // NSLOT * NSLOT if q0 > 9 else 0
    ing_end = min(n3, s_end)
    p_lo, p_hi = max(q0 - 6, 0), min(n3, s_end - 3)
    return dict(q0=q0, q1=q1, blk0=blk0, nbs=nbs, o_beg=o_beg, s_end=s_end, s_beg=s_beg, ing_end=ing_end,
                p_lo=p_lo, p_hi=p_hi)


def block_of(s, nblk):
    return min((s - 3) // PBLK, nblk - 1)


def march(n3, seg, segblk):
    """What one segment does: stored planes per component group, the block of
    every owned step, and the planes each stored value needs."""
    b = bounds(n3, seg, segblk)
    nblk = -(-n3 // PBLK)
    out12, out3, steps = [], [], []
    for s in range(b["o_beg"], b["s_end"]):
        p, z = s - 3, s - 6
        if p < n3:
            out12.append(p)
        if 0 <= z < n3:
            out3.append(z)
        steps.append((s, block_of(s, nblk)))
    return b, out12, out3, steps


@pytest.mark.parametrize("n3", list(range(1, 70)) + [81, 129])
def test_every_split_stores_each_plane_once_with_its_inputs(n3):
    nblk = -(-n3 // PBLK)
    for segblk in range(1, nblk + 1):
        nseg = -(-nblk // segblk)
        out12, out3, blocks = [], [], {}
        for seg in range(nseg):
            b, o12, o3, steps = march(n3, seg, segblk)
            assert b["q0"] < n3 and b["nbs"] >= 1
            out12 += o12
            out3 += o3
            for s, blk in steps:
                assert b["blk0"] <= blk < b["blk0"] + b["nbs"]      # a segment flushes only its own blocks
                blocks.setdefault(blk, []).append(s)
            # components 1, 2 of plane p need the planes p-3..p+3 ingested
            for p in o12:
                assert b["p_lo"] <= p < b["p_hi"]
                for q in range(p - 3, p + 4):
                    assert q < 0 or q >= n3 or b["s_beg"] <= q < b["ing_end"]
            # component 3 of plane z needs F3 of planes z-3..z+3, each formed by in-plane work
            for z in o3:
                for q in range(z - 3, z + 4):
                    if 0 <= q < n3:
                        assert b["p_lo"] <= q < b["p_hi"]
                        for r in range(q - 3, q + 4):
                            assert r < 0 or r >= n3 or b["s_beg"] <= r < b["ing_end"]
            assert b["s_beg"] % NSLOT == 0                        # ring slot of plane q is q % NSLOT
            assert b["p_lo"] >= b["s_beg"] and b["p_hi"] <= n3
        assert sorted(out12) == list(range(n3))                   # each plane once
        assert sorted(out3) == list(range(n3))
        # the steps of a block are the same whatever the split
        whole = {}
        for s, blk in march(n3, 0, nblk)[3]:
            whole.setdefault(blk, []).append(s)
        assert {k: sorted(v) for k, v in blocks.items()} == whole


def test_split_choice():
    assert segmented(5, 1) == (5, 1)        # one CTA: as many segments as blocks
    assert segmented(5, 296) == (1, 5)      # two CTAs per SM already: no split
    assert segmented(1, 1) == (1, 1)        # one block: nothing to split
    nseg, segblk = segmented(11, 60)        # 60 CTAs want 5 segments of 11 blocks
    assert (nseg, segblk) == (4, 3) and nseg * segblk >= 11
    for nblk in range(1, 40):
        for ctas in (1, 2, 3, 7, 50, 147, 295):
            nseg, segblk = segmented(nblk, ctas)
            assert (nseg - 1) * segblk < nblk <= nseg * segblk  # no empty segment
