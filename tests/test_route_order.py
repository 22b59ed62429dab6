"""The fast path's per-substep order, restated on the host (no GPU).

Each substep the fast path does not sort the particles again: G2P counts, per
destination block, how many particles arrived from each of the 27 neighbour
directions; the block scan (k_bins) turns those counts into block ranges and
group offsets, writing each group's offset into the row of the block it came
from; the routing (k_route) gives every slot of a previous block its place
(group offset + rank among that block's slots of the same direction, in slot
order).  Particles that left the domain follow the valid ones, in slot order.
This test restates those three steps with numpy and checks the claim the GPU
test (tests/test_gpu_parity.py) checks on the kernels: the result is exactly a
stable sort of the slots by block.  The same grouping serves the reference's
scatter binning (GATHER_SCATTER::Prepare_Scatter,
Hybrid_Methods/Iterators/GATHER_SCATTER.cpp:33-87).
"""
import numpy as np
import pytest

INVALID = -1


def directions():
    """(dx, dy, dz) of direction d = (dx+1) 9 + (dy+1) 3 + dz+1."""
    return [(d // 9 - 1, (d // 3) % 3 - 1, d % 3 - 1) for d in range(27)]


def route(nb, old_block, new_block):
    """Destination of every slot.  old_block: block of each slot in the previous
    order (slots grouped by block, blocks ascending); new_block: block after the
    move (a neighbour of the old one) or INVALID."""
    nx, ny, nz = nb
    nblk = nx * ny * nz
    dirs = directions()
    coords = lambda b: (b // (ny * nz), (b // nz) % ny, b % nz)
    n = len(old_block)
    d_of = np.full(n, 28)
    for j in range(n):
        if new_block[j] == INVALID:
            continue
        o, b = coords(old_block[j]), coords(new_block[j])
        d_of[j] = dirs.index(tuple(bb - oo for bb, oo in zip(b, o)))
    # G2P: counts by destination row and direction; departures by source block
    dcount = np.zeros((nblk, 27), np.int64)
    inv = np.zeros(nblk, np.int64)
    for j in range(n):
        if d_of[j] == 28:
            inv[old_block[j]] += 1
        else:
            dcount[new_block[j], d_of[j]] += 1
    # k_bins: block ranges, each destination's groups (source blocks ascending =
    # direction descending), the offsets written into the source blocks' rows
    arrivals = dcount.sum(1)
    start = np.concatenate([[0], np.cumsum(arrivals)[:-1]])
    nvalid = int(arrivals.sum())
    inv_off = np.concatenate([[0], np.cumsum(inv)[:-1]])
    src_row = np.zeros((nblk, 27), np.int64)
    for b in range(nblk):
        run = start[b]
        bx, by, bz = coords(b)
        for d in range(26, -1, -1):
            if dcount[b, d]:
                dx, dy, dz = dirs[d]
                src = ((bx - dx) * ny + (by - dy)) * nz + (bz - dz)
                src_row[src, d] = run
                run += dcount[b, d]
    # k_route: slots of each previous block in slot order, ranked per direction
    dest = np.empty(n, np.int64)
    seen = {}
    for j in range(n):
        o, d = old_block[j], d_of[j]
        r = seen.get((o, d), 0)
        seen[(o, d)] = r + 1
        dest[j] = nvalid + inv_off[o] + r if d == 28 else src_row[o, d] + r
    return dest, nvalid


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_routed_order_is_a_stable_sort_by_block(seed):
    rng = np.random.default_rng(seed)
    nb = (5, 4, 6)
    nblk = int(np.prod(nb))
    per = rng.integers(0, 9, nblk)                  # particles per previous block, some empty
    old_block = np.repeat(np.arange(nblk), per)
    n = len(old_block)
    nx, ny, nz = nb
    o = np.stack([old_block // (ny * nz), (old_block // nz) % ny, old_block % nz], 1)
    step = rng.integers(-1, 2, (n, 3)) * (rng.random((n, 1)) < 0.3)   # 30 % of particles move
    c = o + step
    inside = np.all((c >= 0) & (c < np.array(nb)), 1)
    leave = rng.random(n) < 0.05                    # 5 % leave the domain
    new_block = np.where(inside & ~leave, (c[:, 0] * ny + c[:, 1]) * nz + c[:, 2], INVALID)
    dest, nvalid = route(nb, old_block, new_block)
    assert sorted(dest.tolist()) == list(range(n))  # a permutation of the slots
    order = np.empty(n, np.int64)
    order[dest] = np.arange(n)                      # order[position] = slot
    valid = new_block != INVALID
    expect = np.flatnonzero(valid)[np.argsort(new_block[valid], kind="stable")]
    np.testing.assert_array_equal(order[:nvalid], expect)
    np.testing.assert_array_equal(order[nvalid:], np.flatnonzero(~valid))
