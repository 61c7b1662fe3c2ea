"""Copy addressing of the lean FP64 GEMM, checked on the host (no GPU).

`TileCopy<CL, SL, NT>` (evd4sc2025_b200/csrc/gemm_f64.cu) fixes each thread's
share of a tile copy at kernel start: contiguous index ci = (t % (CL/2)) * 2,
strided line si0 = t / (CL/2), lines si0 + r * SS (SS = NT / (CL/2)) for
r < R = SL / SS, one 16-byte cp.async per line, shortened to 8 or 0 bytes by
`cbytes(rem)` along the contiguous direction and switched off by `smask(lim)`
along the strided one.  For every instantiation the library launches and for
ragged edges, each enabled copy must read inside the matrix and write inside
the stage buffer [SL][CL + kPad], and the enabled copies must cover exactly
the valid part of the tile.
"""
import itertools

import pytest

KPAD = 4


def cbytes(rem):
    return 16 if rem >= 2 else (8 if rem == 1 else 0)


def tile_copies(CL, SL, NT, rem_contig, lim_strided):
    """(thread, line, contiguous start, elements) of every enabled copy."""
    CH = CL // 2
    assert NT % CH == 0
    SS = NT // CH
    assert SL % SS == 0
    R = SL // SS
    out = []
    for t in range(NT):
        ci, si0 = (t % CH) * 2, t // CH
        nb = cbytes(rem_contig - ci)
        for r in range(R):
            line = si0 + r * SS
            if line < lim_strided and nb:
                out.append((t, line, ci, nb // 8))
    return out


# (CL, SL, NT) of every TileCopy the dispatcher instantiates: 64x64 tiles with
# four 32x32 warps (A and B, both transposes) and 64x32 skinny tiles with four
# 16x32 warps; BK = 16
CONFIGS = [(64, 16, 128), (16, 64, 128), (32, 16, 128), (16, 32, 128)]


@pytest.mark.parametrize("CL,SL,NT", sorted(set(CONFIGS)))
@pytest.mark.parametrize("rem_contig,lim_strided", [(64, 16), (63, 16), (1, 16), (33, 7),
                                                     (2, 1), (17, 64), (64, 64), (5, 3)])
def test_tile_copy_in_bounds_and_complete(CL, SL, NT, rem_contig, lim_strided):
    rem_contig = min(rem_contig, CL)
    lim_strided = min(lim_strided, SL)
    copies = tile_copies(CL, SL, NT, rem_contig, lim_strided)
    covered = set()
    for t, line, ci, ne in copies:
        # global: contiguous elements [ci, ci + ne) of strided line `line`
        assert ci + ne <= rem_contig and line < lim_strided
        # shared: [line][CL + kPad] layout, inside the stage buffer
        off = line * (CL + KPAD) + ci
        assert off + ne <= SL * (CL + KPAD) and ci + ne <= CL
        for e in range(ne):
            assert (line, ci + e) not in covered
            covered.add((line, ci + e))
    want = {(l, c) for l, c in itertools.product(range(lim_strided), range(rem_contig))}
    assert covered == want
