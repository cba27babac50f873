"""CPU check of the neighbour rule of the shared-memory force sweep
(adjoint.cu, k_adjoint): the FP32 instances keep, per site, only the offset p
of the site's three forward neighbours in its stencil event list, and read
neighbour k as src[p + k].

The host enables this per lattice (neighbours_in_events, context.cu, into
LatticeDev::nb_in_events) only when the rule holds for every site; the test
checks that it holds on every triangular lattice except those of one row
(L2 = 1), where each site is its own upper neighbour and the incoming copy of
that link sorts between the site's own links 1 and 2, and that it fails
there, so that those lattices keep the neighbour table.

The event lists restate build_event_tables (context.cu): site j receives, for
every link (i, k) of the forward table nnt[6i + 2k] (construct_triangular,
simulation/organic_lattice.c:10-46), the term "here" (key 2(3i + k), source
n) at i and "there" (key 2(3i + k) + 1, source i) at n, sorted by key.  A
site's own links have the keys 6j, 6j + 2, 6j + 4 and every incoming key is
odd, so the own block is contiguous with 0..3 incoming terms before it.  The
kernel takes the smallest q in 0..2 whose three entries match, else 3; on
lattices small enough for a site to appear twice that may not be the
structural offset, but it always yields the same three neighbours."""
import numpy as np
import pytest

from oracle import forward_neighbours


def event_sources(l1, l2):
    nb = forward_neighbours(l1, l2)
    V = l1 * l2
    per = [[] for _ in range(V)]
    for i in range(V):
        for k in range(3):
            n = int(nb[i, k])
            base = (3 * i + k) * 2
            per[i].append((base, n))
            per[n].append((base + 1, i))
    src = np.empty((V, 6), dtype=np.int64)
    for j in range(V):
        assert len(per[j]) == 6
        src[j] = [s for _, s in sorted(per[j])]
    return nb, src


def kernel_offset(src_j, nb_j):
    p = 3
    for q in (2, 1, 0):
        if all(src_j[q + k] == nb_j[k] for k in range(3)):
            p = q
    return p


def rule_holds(l1, l2):
    """neighbours_in_events restated, through the kernel's choice of p"""
    nb, src = event_sources(l1, l2)
    for j in range(l1 * l2):
        p = kernel_offset(src[j], nb[j])
        if [src[j][p + k] for k in range(3)] != list(nb[j]):
            return False
    return True


# one column (L1 = 1) has a self-link too (each site is its own right
# neighbour), but its incoming copy sorts between own links 0 and 1 and has
# the same source, so three matching entries remain
SHAPES = [(l1, l2) for l1 in range(1, 13) for l2 in range(1, 13) if l1 * l2 > 1] + [(32, 32), (48, 48), (3, 50), (50, 3)]


@pytest.mark.parametrize("l1,l2", SHAPES)
def test_forward_neighbours_from_event_offset(l1, l2):
    assert rule_holds(l1, l2) == (l2 != 1), (l1, l2)
