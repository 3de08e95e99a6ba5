"""Host check of the two-body Gram kernel's block index rules (density.cu: k_gram,
k_gram_finish), for every M the library builds (1..16).

Each thread of k_gram owns one 4x4 block: rows aa + r*NB and columns
bb + c*NB (r, c < 4) of the K x K pair Gram matrix, K = M(M+1)/2, NB = ceil(K/4),
inside a shared tile padded to KP = 4*NB rows. For one state (phi = psi) only
the blocks with aa <= bb are reduced, enumerated by the kernel's triangular
walk, and the finish kernel reads entry (a, b) from (b, a), conjugated, when
a mod NB > b mod NB. The rules below restate those lines; the test checks
that every index stays inside the padded tile, that the walk visits each upper
block once, that every entry of the matrix is produced exactly once (computed
directly or by its mirror), and that the 16-byte bank slots of a warp's column
loads spread as the kernel's comment states."""
import pytest

LD = 33   # tile row stride in double2
TILE = 32


def walk(blk, NB):
    """The kernel's triangular walk: block number -> (aa, bb), aa <= bb."""
    aa, rem = 0, blk
    while rem >= NB - aa:
        rem -= NB - aa
        aa += 1
    return aa, aa + rem


@pytest.mark.parametrize("M", range(1, 17))
def test_hermitian_half_covers_every_entry(M):
    K = M * (M + 1) // 2
    NB = (K + 3) // 4
    KP = 4 * NB
    blocks = [walk(b, NB) for b in range(NB * (NB + 1) // 2)]
    assert sorted(blocks) == [(a, b) for a in range(NB) for b in range(a, NB)]
    written = {}
    for aa, bb in blocks:
        for r in range(4):
            for c in range(4):
                a, b = aa + r * NB, bb + c * NB
                assert a < KP and b < KP   # shared tile rows
                if a < K and b < K:
                    assert (a, b) not in written
                    written[(a, b)] = (aa, bb)
    for a in range(K):
        for b in range(K):
            mirror = (a % NB) > (b % NB)
            src = (b, a) if mirror else (a, b)
            assert src in written, (a, b)
            # a mirrored entry is never also computed directly
            assert not (mirror and (a, b) in written)


@pytest.mark.parametrize("M", range(1, 17))
def test_full_grid_covers_every_entry(M):
    K = M * (M + 1) // 2
    NB = (K + 3) // 4
    seen = set()
    for blk in range(NB * NB):
        aa, bb = blk // NB, blk % NB
        for r in range(4):
            for c in range(4):
                a, b = aa + r * NB, bb + c * NB
                assert a < 4 * NB and b < 4 * NB
                if a < K and b < K:
                    assert (a, b) not in seen
                    seen.add((a, b))
    assert len(seen) == K * K


def test_column_loads_spread_over_bank_slots():
    # M = 10: a warp's distinct column blocks bb read rows bb + c*NB at column t;
    # row x of the tile starts in 16-byte slot (x*LD + t) mod 8
    M = 10
    K = M * (M + 1) // 2
    NB = (K + 3) // 4
    for warp in range(0, NB * NB, 32):
        bbs = {blk % NB for blk in range(warp, min(warp + 32, NB * NB))}
        for t in range(TILE):
            for c in range(4):
                slots = {((bb + c * NB) * LD + t) % 8 for bb in bbs}
                # interleaved rows: as many slots as distinct addresses allow
                assert len(slots) == min(8, len(bbs))
                consecutive = {((4 * bb + c) * LD + t) % 8 for bb in bbs}
                assert len(consecutive) <= 2
