"""CPU checks of the two facts the device's node growth rests on (no GPU needed).

1. The greedy overlap check of AppendNodeFromVertexHost (NodeGraph.cu:652-704), a
   sequential loop, equals the fixed point of the round rule the device runs: a candidate
   is rejected once an earlier neighbour is kept and kept once all of them are rejected.
   The rounds here are Jacobi rounds (every decision of a round reads the previous round's
   state); the device's in-place rounds only decide earlier, with the same decisions.
2. The dedup grid: in float32, two candidates that pass the overlap test have cell
   coordinates (floor of the coordinate times 1 / (1.125 r), clamped to +-2^18) that differ
   by at most one per axis, so the 27 cells around a candidate hold all its neighbours.
"""
import numpy as np
import pytest

CELL_SCALE = np.float32(1.125)
CLAMP = np.float32(262144.0)


def overlap_d2(a, b):
    """((dx*dx + dy*dy) + dz*dz) in float32, dx = a - b, as the host loop sums it."""
    d = (a - b).astype(np.float32)
    return ((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]).astype(np.float32) + d[..., 2] * d[..., 2]).astype(
        np.float32)


def greedy_sequential(c, thr):
    kept = []
    for i in range(len(c)):
        if not kept or not (overlap_d2(c[kept], c[i]) <= thr).any():
            kept.append(i)
    return np.array(kept, dtype=np.int64)


def earlier_neighbours(c, thr):
    n = len(c)
    d2 = overlap_d2(c[:, None, :], c[None, :, :])
    lower = np.tril(np.ones((n, n), bool), -1)
    i, j = np.nonzero((d2 <= thr) & lower)
    return i, j


def greedy_rounds(c, thr):
    n = len(c)
    i, j = earlier_neighbours(c, thr)
    state = np.zeros(n, np.int8)            # 0 open, 1 kept, 2 rejected
    rounds = 0
    while (state == 0).any():
        rounds += 1
        assert rounds <= n + 1
        kept_nb = np.zeros(n, bool)
        open_nb = np.zeros(n, bool)
        np.logical_or.at(kept_nb, i, state[j] == 1)
        np.logical_or.at(open_nb, i, state[j] == 0)
        new = state.copy()
        new[(state == 0) & kept_nb] = 2
        new[(state == 0) & ~kept_nb & ~open_nb] = 1
        state = new
    return np.nonzero(state == 1)[0], rounds


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_rounds_reach_the_sequential_greedy(seed):
    rng = np.random.default_rng(seed)
    radius = np.float32(0.025)
    r = np.float32(0.85) * radius
    thr = np.float32(r * r)
    # a noisy surface patch in voxel order, plus exact duplicates and points on a lattice
    # (distances equal to the threshold's neighbourhood, ties)
    p = rng.uniform(0, 0.3, (600, 3)).astype(np.float32)
    p[:, 2] = (0.05 * np.sin(8 * p[:, 0]) + 0.002 * rng.standard_normal(600)).astype(np.float32)
    lattice = (np.stack(np.meshgrid(np.arange(6), np.arange(6), [0], indexing="ij"), -1).reshape(-1, 3)
               * np.float32(0.7) * radius).astype(np.float32)
    c = np.concatenate([p, p[::50], lattice + np.float32(0.31)]).astype(np.float32)
    key = np.floor(c / (np.float32(0.7) * radius)).astype(np.int64)
    c = c[np.lexsort((key[:, 0], key[:, 1], key[:, 2]))]
    seq = greedy_sequential(c, thr)
    par, rounds = greedy_rounds(c, thr)
    np.testing.assert_array_equal(par, seq)
    assert 1 < rounds < len(c)


def cells(v, r):
    inv_cell = np.float32(1.0) / (CELL_SCALE * r)
    t = (v.astype(np.float32) * inv_cell).astype(np.float32)
    return np.floor(np.clip(t, -CLAMP, CLAMP)).astype(np.int64)


@pytest.mark.parametrize("radius,scale", [(0.025, 1.0), (0.006, 1.0), (0.001, 20.0), (0.0001, 40.0)])
def test_overlapping_candidates_lie_in_adjacent_cells(radius, scale):
    """Pairs built at the edge of the overlap test (|d| just under r along one axis, or
    spread over three), far from the origin where the scaled coordinates are large, and
    beyond the clamp."""
    rng = np.random.default_rng(7)
    radius = np.float32(radius)
    r = np.float32(0.85) * radius
    thr = np.float32(r * r)
    n = 200_000
    a = (rng.uniform(-scale, scale, (n, 3))).astype(np.float32)
    direction = rng.standard_normal((n, 3))
    direction[: n // 2, 1:] = 0.0                      # half the pairs along x alone
    direction /= np.linalg.norm(direction, axis=1, keepdims=True)
    length = r * (1.0 - np.abs(rng.standard_normal(n)) * 1e-6)
    b = (a + direction * length[:, None]).astype(np.float32)
    hit = overlap_d2(b, a) <= thr
    assert hit.mean() > 0.4
    diff = np.abs(cells(a[hit], r) - cells(b[hit], r))
    assert diff.max() <= 1


def test_cells_beyond_the_clamp_stay_adjacent():
    r = np.float32(0.85) * np.float32(0.0001)
    edge = np.float32(262144.0) * CELL_SCALE * r        # where the scaled coordinate reaches the clamp
    thr = np.float32(r * r)
    for x in (edge * np.float32(0.999999), edge * np.float32(1.5), -edge * np.float32(1.000001), -edge):
        a = np.array([x, 0, 0], np.float32)
        b = np.array([x + r, 0, 0], np.float32)
        while overlap_d2(a, b) > thr:                   # the farthest float that still overlaps
            b[0] = np.nextafter(b[0], a[0])
        assert np.abs(cells(a, r) - cells(b, r)).max() <= 1
