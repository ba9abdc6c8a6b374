"""Index maps of two kernels restated in Python (no GPU), so their coverage is checked
by construction:

- the digit product's tile order (tc_ozaki.cu, oz_gemm_kernel): groups of 8 row
  blocks walked column block by column block must visit every (row block, column
  block) tile exactly once;
- the R^k table of the assembly (assemble.cu): rkb_pad_kernel writes every element of
  the zero-margined table except the valid band |i - j| < ks, rkb_band_kernel writes
  exactly that band, and outside the band the interval ranges of (i, ip) and (j, jp)
  never overlap, so the factorised product is the whole value there."""
import pytest

OZ_GM = 8


def tile_of(bid, mblk, nblk):
    per = OZ_GM * nblk
    grp = bid // per
    m0b = grp * OZ_GM
    gs = min(mblk - m0b, OZ_GM)
    rr = bid - grp * per
    return m0b + rr % gs, rr // gs


@pytest.mark.parametrize("mblk", [1, 2, 7, 8, 9, 16, 17, 62, 63])
@pytest.mark.parametrize("nblk", [1, 3, 13, 64, 123])
def test_digit_gemm_tile_order_is_a_bijection(mblk, nblk):
    seen = set()
    for bid in range(mblk * nblk):
        mb, nb = tile_of(bid, mblk, nblk)
        assert 0 <= mb < mblk and 0 <= nb < nblk
        seen.add((mb, nb))
    assert len(seen) == mblk * nblk


def iv_range(i, ip, ks, nv):
    lo = max(0, i + ip - (ks - 1))
    hi = min(i, nv - 1)
    return lo, hi


@pytest.mark.parametrize("ns,ks", [(12, 3), (20, 4), (30, 8), (40, 10)])
def test_rk_table_pad_and_band_partition(ns, ks):
    nv = ns - ks + 1
    PL = ks - 1
    NP = ns + PL + 40 + PL           # the exchange tile's overhang (XTY = 40) as the high margin
    for ip in range(ks):
        for jp in range(ks):
            # rkb_band_kernel: diagonals d = -(ks-1) .. ks-1, valid elements only
            band = set()
            for d in range(-(ks - 1), ks):
                for i in range(((ns + 255) // 256) * 256):
                    j = i + d
                    if i >= ns or j < 0 or j >= ns or i + ip >= ns or j + jp >= ns:
                        continue
                    band.add((i, j))
            # rkb_pad_kernel: every padded element, skipping the valid band
            pad = set()
            for pr in range(NP):
                i = pr - PL
                irow = 0 <= i and i + ip < ns
                for pc in range(NP):
                    j = pc - PL
                    if irow and 0 <= j and j + jp < ns:
                        if j - i < ks and i - j < ks:
                            continue
                        ilo, ihi = iv_range(i, ip, ks, nv)
                        jlo, jhi = iv_range(j, jp, ks, nv)
                        # outside the band the interval ranges are disjoint, and the factorised
                        # branch the kernel takes is the one that holds
                        assert ihi < jlo or jhi < ilo
                        if not ihi < jlo:
                            assert jhi < ilo
                    pad.add((i, j))
            assert not (band & pad)
            valid = {(i, j) for i in range(ns) for j in range(ns) if i + ip < ns and j + jp < ns}
            assert band == {(i, j) for (i, j) in valid if abs(i - j) < ks}
            assert len(band) + len(pad) == NP * NP
