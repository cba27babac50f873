"""CPU check of the register-tile layouts (slices_tile.cu, adjoint_tile.cu)
for every lattice shape the kernels accept: each site is held by exactly one
active lane, the lanes a thread shuffles its left and right neighbours from
hold the columns next to its own (periodic in L1), the strips' edge rows and
the shared-memory sizes stay in their buffers, and in the force sweep every
(site, link) term is summed by exactly one thread.

The shape tables restate `tile_shape` (slices_tile.cu) and `adj_tile_shape`
(adjoint_tile.cu): (W columns per lane, LPR lanes per row group, H rows per
strip, R vectors or KG vector groups per CTA, maximum threads); the
acceptance rules are theirs."""
import pytest

SLICE_SHAPES = {48: (3, 16, 2, 1, 384), 24: (3, 8, 1, 2, 256), 16: (1, 16, 2, 2, 256),
                12: (1, 16, 2, 2, 256), 8: (1, 8, 2, 4, 256)}
ADJ_SHAPES = {24: (3, 8, 1, 2, 384), 16: (1, 16, 2, 2, 256), 12: (1, 16, 2, 2, 256), 8: (1, 8, 2, 2, 256)}


def slice_accepts(L1, L2):
    W, LPR, H, R, maxT = SLICE_SHAPES[L1]
    G = 32 // LPR
    if L2 < 2 or L2 % H or (L2 // H) % G:
        return False
    threads = 32 * (L2 // H) // G
    smem = 8 * 2 * R * (L2 // H) * L1
    return 32 <= threads <= maxT and smem <= 48 * 1024


def adj_accepts(L1, L2):
    W, LPR, H, KG, maxT = ADJ_SHAPES[L1]
    Gl = 32 // LPR
    if L2 < 2 or L2 % H or (L2 // H) % Gl:
        return False
    threads = KG * 32 * (L2 // H) // Gl
    smem = 4 * 6 * L1 * L2 + 8 * 2 * KG * 9 * (L2 // H) * L1
    return 32 <= threads <= maxT and smem <= 227 * 1024


def tile_threads(L1, L2, W, LPR, H, nthreads, warp_offset=0):
    """The geometry of tile_of (slices_tile.cu) for threads 0..nthreads-1."""
    G, ncl, NS = 32 // LPR, L1 // W, L2 // H
    geo = {}
    for tid in range(nthreads):
        lane, warp = tid % 32, tid // 32 - warp_offset
        g, cl = lane // LPR, lane % LPR
        s = warp * G + g
        act = cl < ncl
        a0 = cl * W if act else 0
        lm = g * LPR + ((ncl - 1 if cl == 0 else cl - 1) if act else 0)
        lp = g * LPR + ((0 if cl + 1 == ncl else cl + 1) if act else 0)
        geo[tid] = (s, act, a0, s * H, lm, lp)
    return geo, NS


def check_cover(geo, L1, L2, W, H, NS):
    own = {}
    for tid, (s, act, a0, b0, lm, lp) in geo.items():
        assert 0 <= s < NS and b0 + H <= L2
        if not act:
            continue
        for h in range(H):
            for k in range(W):
                site = (a0 + k, b0 + h)
                assert site not in own
                own[site] = tid
        base = tid - tid % 32
        left, right = geo[base + lm], geo[base + lp]
        assert left[0] == s and right[0] == s
        assert left[2] + W - 1 == (a0 - 1) % L1
        assert right[2] == (a0 + W) % L1
    assert len(own) == L1 * L2


@pytest.mark.parametrize("L1", sorted(SLICE_SHAPES))
def test_slice_tiles_cover_the_lattice(L1):
    W, LPR, H, R, maxT = SLICE_SHAPES[L1]
    n = 0
    for L2 in range(2, 97):
        if not slice_accepts(L1, L2):
            continue
        threads = 32 * (L2 // H) // (32 // LPR)
        geo, NS = tile_threads(L1, L2, W, LPR, H, threads)
        check_cover(geo, L1, L2, W, H, NS)
        n += 1
    assert n > 0
    assert slice_accepts(L1, L1)  # the square lattices of the checkpointing and batch workloads


@pytest.mark.parametrize("L1", sorted(ADJ_SHAPES))
def test_force_tiles_sum_every_link_once(L1):
    W, LPR, H, KG, maxT = ADJ_SHAPES[L1]
    Gl = 32 // LPR
    n = 0
    for L2 in range(2, 97):
        if not adj_accepts(L1, L2):
            continue
        NWg = (L2 // H) // Gl
        for g in range(KG):
            geo, NS = tile_threads(L1, L2, W, LPR, H, 32 * NWg * (g + 1), warp_offset=0)
            geo = {t: v for t, v in geo.items() if t >= 32 * NWg * g}
            # the group's warps are numbered from its first warp
            geo = {t: (v[0] - g * NWg * Gl,) + v[1:3] + (v[3] - g * NWg * Gl * H,) + v[4:] for t, v in geo.items()}
            check_cover(geo, L1, L2, W, H, NS)
            links = {}
            for tid, (s, act, a0, b0, lm, lp) in geo.items():
                if not act:
                    continue
                for h in range(H):
                    for k in range(W):
                        a, b = a0 + k, b0 + h
                        for key in ((a, b, 0), (a, b, 1), ((a + 1) % L1, b, 2)):
                            links[key] = links.get(key, 0) + 1
            assert len(links) == 3 * L1 * L2 and set(links.values()) == {1}
        n += 1
    assert n > 0
    assert adj_accepts(L1, L1)
