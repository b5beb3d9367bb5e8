"""CPU check of the L2 pull's index arithmetic (no GPU).

The single-mesh bulk-copy and tensor-core stage kernels with AHEAD, and the pool's
per-N bulk kernels at 6 and 9 points, have thread 0 of each block pull the u_in and k
of a later block's tile into L2 with cp.async.bulk.prefetch.L2.  This restates, in
numpy, the block -> tile map (bulk_tile_index, z-column order included), the block
ahead (tile_ahead: block + SM ids x MINB x AHEAD / 2, only when inside the grid) and
the 16-byte-rounded node range each prefetch covers (prefetch_nodes_l2), for every
AHEAD shape of the launch-shape lists and for meshes with ragged last tiles, and
checks that every range lies inside its [6][stride] state arrays and is a legal bulk
prefetch (16-byte aligned start, a multiple of 16 bytes long).
"""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
VARIANTS = os.path.join(ROOT, "nekwave_b200", "csrc", "stage_variants.h")


def shapes(N):
    """(ks, epb, ksm, minb, alg) of the launch-shape list of N points per direction."""
    text = open(VARIANTS).read()
    line = re.search(rf"#define NWB_VARIANTS_{N}\(X\)(.*)", text).group(1)
    return [tuple(int(v) for v in m.groups())
            for m in re.finditer(r"X\((\d+), (\d+), (\d+), (\d+), (\d+)\)", line)]


def pulled_shapes():
    """(N, epb, minb, ahead, zcol) of every shape with the L2 pull."""
    out = []
    for N in range(2, 11):
        for ks, epb, ksm, minb, alg in shapes(N):
            if alg in (211, 212):
                out.append((N, epb, minb, alg - 210, False))
            elif alg >= 1000 and (alg - 1000) & 768:
                fl = alg - 1000
                assert fl < 1024 and (fl & 768) != 768, alg  # one distance only
                assert fl & 2 and ks == 2, alg                 # the field split
                out.append((N, epb, minb, 2 if fl & 512 else 1, bool(fl & 1)))
    return out


def tile_index(b, nel, epb, zcol, structured):
    """bulk_tile_index: tiles in z-column order on structured boxes whose x rows hold
    whole tiles, else in memory order."""
    nx, ny, nz = nel
    if zcol and structured and nx % epb == 0:
        col, ez = b // nz, b % nz
        ntx = nx // epb
        ey, xt = col // ntx, col % ntx
        return xt + ntx * (ey + ny * ez)
    return b


def node_range(e0, n, n3):
    """prefetch_nodes_l2: [a0, a1) rounded out to even node indices (16 bytes)."""
    g0 = e0 * n3
    return g0 & ~1, (g0 + n * n3 + 1) & ~1


def test_every_pull_shape_is_listed_and_well_formed():
    got = pulled_shapes()
    # the defaults at 6 and 9 points pull half a wave ahead (entry 0 of their lists)
    assert shapes(6)[0] == (2, 2, 0, 3, 1314) and shapes(9)[0] == (2, 1, 0, 2, 1315)
    assert {N for N, *_ in got} == {5, 6, 7, 8, 9}
    for N, epb, minb, ahead, zcol in got:
        assert ahead in (1, 2) and minb >= 1 and epb >= 1


MESHES = [(1, 1, 1), (2, 1, 1), (3, 3, 2), (5, 4, 3), (16, 16, 12), (34, 34, 34), (64, 64, 32),
          (22, 22, 22), (29, 29, 29), (7, 11, 13)]


@pytest.mark.parametrize("nsm", [148, 160, 256])
def test_single_mesh_pull_ranges_stay_inside_the_state(nsm):
    for N, epb, minb, ahead, zcol in pulled_shapes():
        n3 = N ** 3
        for nel in MESHES:
            nelt = nel[0] * nel[1] * nel[2]
            npts = nelt * n3
            stride = (npts + 63) // 64 * 64
            grid = (nelt + epb - 1) // epb
            for structured in (True, False):
                b = np.arange(grid, dtype=np.int64)
                t = tile_index(b, nel, epb, zcol, structured)
                # every tile is some block's own tile exactly once
                assert np.array_equal(np.sort(t), b), (N, nel, zcol, structured)
                b2 = b + (nsm * minb * ahead) // 2
                b2 = b2[b2 < grid]
                if b2.size == 0:
                    continue
                e = tile_index(b2, nel, epb, zcol, structured) * epb
                n = np.minimum(epb, nelt - e)
                assert (n >= 1).all()
                a0, a1 = node_range(e, n, n3)
                assert (a0 >= 0).all() and (a1 <= stride).all() and (a1 > a0).all()
                assert (a0 % 2 == 0).all() and ((a1 - a0) % 2 == 0).all()  # 16-byte rules


@pytest.mark.parametrize("seed", [0, 1])
def test_pool_pull_ranges_stay_inside_each_cavity(seed):
    """The per-N pool kernels at 6 and 9 points: block b's pull reads work item b + d
    of that N's list (one block per item), whose cavity, first element and count set
    the range, inside that cavity's own [6][stride] arrays."""
    rng = np.random.default_rng(seed)
    for N, epb, minb in ((6, 2, 3), (9, 1, 2)):
        n3 = N ** 3
        cav = []  # (nelt, stride) per cavity of this N
        work = []  # (cavity, e0)
        for c in range(int(rng.integers(1, 60))):
            nel = rng.integers(1, 13, size=3)
            nelt = int(np.prod(nel))
            cav.append((nelt, (nelt * n3 + 63) // 64 * 64))
            work += [(c, e0) for e0 in range(0, nelt, epb)]
        work = np.array(work, dtype=np.int64)
        for nsm in (148, 160):
            d = (nsm * minb * 1) // 2
            b2 = np.arange(len(work)) + d
            b2 = b2[b2 < len(work)]
            for c, e0 in work[b2]:
                nelt, stride = cav[c]
                n = min(epb, nelt - e0)
                assert n >= 1
                a0, a1 = node_range(e0, n, n3)
                assert 0 <= a0 < a1 <= stride and a0 % 2 == 0 and (a1 - a0) % 2 == 0
