"""CPU checks of the oracle: known-answer tests derived from the reference's
definitions, independent Python restatements of its integer rules, and
properties of the assembled system.  No GPU."""
import numpy as np
import pytest


# ---------------------------------------------------------------------------
# Node graph: half-precision distances + strict-< heap + Lomuto quicksort
# (libs/star/geometry/node_graph/NodeGraph.cu:10-101, brute_force_knn.cuh:52-135)
# ---------------------------------------------------------------------------
def py_knn(dist_row, k, init):
    d = [init] * k
    idx = [0] * k

    def refresh():
        m = 0
        for i in range(1, k):
            if d[i] > d[m]:
                m = i
        return m

    m = refresh()
    for j, v in enumerate(dist_row):
        if v < d[m]:
            d[m] = v
            idx[m] = j
        m = refresh()

    def qs(lo, hi):
        if lo < hi:
            piv = d[hi]
            i = lo - 1
            for j in range(lo, hi):
                if d[j] < piv:
                    i += 1
                    d[i], d[j] = d[j], d[i]
                    idx[i], idx[j] = idx[j], idx[i]
            d[i + 1], d[hi] = d[hi], d[i + 1]
            idx[i + 1], idx[hi] = idx[hi], idx[i + 1]
            qs(lo, i)
            qs(i + 2, hi)

    qs(0, k - 1)
    return idx, d


def half_sq_dist(a, b):
    hi, lo = (a, b)
    dx = np.float32(hi[0] - lo[0])
    dy = np.float32(hi[1] - lo[1])
    dz = np.float32(hi[2] - lo[2])
    # fma(dz, dz, fma(dy, dy, dx*dx)) evaluated exactly in float64 then rounded once per fma
    t = np.float32(dx * dx)
    t = np.float32(np.float64(dy) * np.float64(dy) + np.float64(t))
    t = np.float32(np.float64(dz) * np.float64(dz) + np.float64(t))
    return float(np.float32(np.float16(t)))


@pytest.mark.parametrize("k", [4, 8])
def test_node_graph_matches_python_restatement(orc, k):
    rng = np.random.default_rng(3)
    pts = rng.uniform(-0.1, 0.1, size=(40, 3)).astype(np.float32)
    pts[5] = pts[6]          # exact duplicates -> ties
    pts[7] = pts[6]
    nodes = np.concatenate([np.zeros((2, 3), np.float32), pts])
    nodes4 = np.concatenate([nodes, np.ones((len(nodes), 1), np.float32)], 1)
    knn, w, edges = orc.OracleGeometry().node_graph(nodes4, k, 0.025)
    for a in range(len(nodes)):
        row = [half_sq_dist(nodes[max(a, b)], nodes[min(a, b)]) for b in range(len(nodes))]
        idx, d = py_knn(row, k, 1e3)
        assert list(knn[a]) == idx, f"node {a}"
        ww = np.exp(-np.array(d, np.float32) / np.float32(2 * np.float32(0.025) * np.float32(0.025)))
        np.testing.assert_allclose(w[a], ww / ww.sum(), rtol=1e-5)
    assert (edges[:, 0] == np.repeat(np.arange(len(nodes)), k)).all()
    assert (edges[:, 2] == np.tile(np.arange(k), len(nodes))).all()


def test_node_graph_self_is_first(orc):
    rng = np.random.default_rng(4)
    nodes4 = np.concatenate([rng.uniform(-1, 1, (50, 3)), np.ones((50, 1))], 1).astype(np.float32)
    knn, _, _ = orc.OracleGeometry().node_graph(nodes4, 4, 0.025)
    assert (knn[:, 0] == np.arange(50)).all()


def test_skinning_matches_python(orc):
    rng = np.random.default_rng(8)
    nodes = np.concatenate([rng.uniform(-0.2, 0.2, (30, 3)), np.ones((30, 1))], 1).astype(np.float32)
    verts = np.concatenate([rng.uniform(-0.2, 0.2, (200, 3)), np.ones((200, 1))], 1).astype(np.float32)
    knn, sw, cw = orc.OracleGeometry().skinning(nodes, verts, 0.025)
    for v in range(200):
        diff = (verts[v, :3] - nodes[:, :3]).astype(np.float32)
        row = []
        for d in diff:
            t = np.float32(d[0] * d[0])
            t = np.float32(np.float64(d[1]) ** 2 + np.float64(t))
            t = np.float32(np.float64(d[2]) ** 2 + np.float64(t))
            row.append(float(t))
        idx, _ = py_knn(row, 4, 1e6)
        assert list(knn[v]) == idx
    assert (cw == 1.0).all()
    np.testing.assert_allclose(sw.sum(1), 1.0, rtol=1e-6)


def test_voxel_subsample_kat(orc):
    v = 0.01
    pts = np.array([[0.0012, 0.0011, 0.0010, 1], [0.0049, 0.0051, 0.0050, 1],   # voxel (0,0,0): 2nd is nearer the centre
                    [0.0150, 0.0010, 0.0010, 1],                                 # voxel (1,0,0)
                    [-0.0050, 0.0050, 0.0050, 1],                                # voxel (-1,0,0)
                    [0.0052, 0.0049, 0.0050, 1]], np.float32)                    # ties with point 1? farther
    out = orc.OracleGeometry().voxel_subsample(pts, v)
    # keys sort (x+512) + (y+512)*1024 + ...: voxel x = -1 first, then 0, then 1
    np.testing.assert_array_equal(out[:, :3], pts[[3, 1, 2], :3])


def test_init_nodes_prepends_anchors_and_dedups(orc):
    rng = np.random.default_rng(1)
    pts = np.concatenate([rng.uniform(0, 0.2, (5000, 3)), np.ones((5000, 1))], 1).astype(np.float32)
    nodes = orc.OracleGeometry().init_nodes(pts, 0.025)
    np.testing.assert_array_equal(nodes[:2], [[0, 0, 0, 1], [0, 0, 0, 1]])
    real = nodes[2:, :3].astype(np.float64)
    d2 = ((real[:, None] - real[None]) ** 2).sum(-1)
    np.fill_diagonal(d2, 1.0)
    assert d2.min() > (0.85 * 0.025) ** 2 * (1 - 1e-5)


# ---------------------------------------------------------------------------
# Index build KATs (ImageTermKNNFetcher.cu:56-88, Node2TermsIndex.cu:6-121,
# NodePair2TermsIndex.cu:11-193)
# ---------------------------------------------------------------------------
def test_compact_pixels_kat(orc):
    from starhub_b200.scenes import Camera

    class S:
        pass
    s = S()
    s.camera = Camera(4, 3, 1, 1, 0, 0)
    idx = np.full((3, 4), 0xFFFFFFFF, np.uint32)
    idx[0, 1] = 2
    idx[1, 0] = 0
    idx[2, 3] = 1
    s.index_map = idx
    flow = np.zeros((3, 4, 2), np.float32)
    flow[0, 1] = [0.5, 1.5]      # 1.5 -> 2 (ties to even), 1.5 -> 2
    flow[1, 0] = [-3.0, 0.49]    # negative saturates to 0; 1.49 -> 1
    flow[2, 3] = [2.5, -0.5]     # 5.5 -> 6, 1.5 -> 2
    s.flow = flow
    s.surfel_knn = np.array([[0, 1, 2, 3], [4, 5, 6, 7], [8, 9, 10, 11]], np.uint16)
    s.surfel_sw = np.arange(12, dtype=np.float32).reshape(3, 4)
    s.surfel_cw = np.ones((3, 4), np.float32)
    pix, knn, sw, cw = orc.compact_pixels(s)
    np.testing.assert_array_equal(pix, [[1, 0, 2, 2], [0, 1, 0, 1], [3, 2, 6, 2]])
    np.testing.assert_array_equal(knn, s.surfel_knn[[2, 0, 1]])
    np.testing.assert_array_equal(sw, s.surfel_sw[[2, 0, 1]])


def test_node2term_kat(orc):
    dense = np.array([[0, 1, 2, 3], [2, 3, 4, 1]], np.uint16)
    edges = np.array([[0, 0, 0], [0, 4, 1], [2, 3, 1]], np.uint16)
    off, ti = orc.node2term(dense, edges, 5)
    # term ids: dense 0,1 | reg 2,3,4 | node-motion 5..9 ; self edge 2 -> invalid keys at the end
    expect = {0: [0, 3, 5], 1: [0, 1, 6], 2: [0, 1, 4, 7], 3: [0, 1, 4, 8], 4: [1, 3, 9]}
    for n, lst in expect.items():
        assert list(ti[off[n]:off[n + 1]]) == lst
    assert off[5] == sum(len(v) for v in expect.values())
    assert list(ti[off[5]:]) == [2, 2]


def test_nodepair2term_kat(orc):
    dense = np.array([[3, 1, 2, 0], [2, 3, 4, 1]], np.uint16)
    edges = np.array([[0, 0, 0], [4, 0, 1], [1, 3, 1]], np.uint16)
    m = orc.nodepair2term(dense, edges, 5)
    pairs = list(zip(m["half_rows"], m["half_cols"]))
    # dense 0 -> (1,3),(2,3),(0,3),(1,2),(0,1),(0,2); dense 1 -> (2,3),(2,4),(3,4),(1,2),(1,3),(1,4)
    # reg: (0,4) term 3, (1,3) term 4, self edge term 2 -> no pair
    expect = {(0, 1): [0], (0, 2): [0], (0, 3): [0], (0, 4): [3], (1, 2): [0, 1], (1, 3): [0, 1, 4],
              (1, 4): [1], (2, 3): [0, 1], (2, 4): [1], (3, 4): [1]}
    assert pairs == sorted(expect)
    for k, (b, e) in enumerate(zip(m["half_begin"], m["half_end"])):
        assert list(m["term_index"][b:e]) == expect[pairs[k]]
    sym = list(zip(m["sym_rows"], m["sym_cols"]))
    assert sym == sorted(sym) and len(sym) == 2 * len(pairs)
    assert list(m["blkrow_offset"]) == [0, 4, 8, 12, 16, 20]


def test_binblock_csr_structure(orc):
    m = orc.nodepair2term(np.array([[0, 1, 2, 3]], np.uint16), np.zeros((0, 3), np.uint16), 4)
    rp, col = orc.binblock_csr(4, m["sym_rows"], m["sym_cols"])
    # 24 scalar rows in one bin; every block row has 4 blocks -> bin length 24, 32 rows * 24 entries
    assert list(rp[:33]) == list(range(32)) + [32 * 24]
    nblk = rp[32] // 6
    used = col[:nblk]
    # row 0 of block-row 0 lists the diagonal (0) then columns 6, 12, 18
    assert [used[0 + 32 * s] for s in range(4)] == [0, 6, 12, 18]
    assert [used[6 + 32 * s] for s in range(4)] == [6, 0, 12, 18]
    assert (used[24:32] == -1).all()


# ---------------------------------------------------------------------------
# Solve properties
# ---------------------------------------------------------------------------
def test_aligned_scene_gives_identity(orc, tiny_scene):
    """Measurement equal to the rendered reference: zero residuals, zero step."""
    import dataclasses
    sc = dataclasses.replace(tiny_scene, meas_vertex=tiny_scene.ref_vertex.copy(),
                             meas_normal=tiny_scene.ref_normal.copy())
    dq = orc.solve(sc, gn_iters=3, pcg_iters=10)
    ident = np.tile(np.array([0, 0, 0, 1, 0, 0, 0, 0], np.float32), (sc.num_nodes, 1))
    np.testing.assert_allclose(dq, ident, atol=1e-6)


def test_system_symmetric_and_preconditioner(orc, tiny_scene):
    _, info = orc.solve(tiny_scene, gn_iters=1, pcg_iters=10, debug=True)
    rows, cols, off = info["sym_rows"], info["sym_cols"], info["offdiag"].reshape(-1, 6, 6)
    lookup = {(r, c): k for k, (r, c) in enumerate(zip(rows, cols))}
    for k, (r, c) in enumerate(zip(rows, cols)):
        np.testing.assert_allclose(off[k], off[lookup[(c, r)]].T, rtol=1e-5, atol=1e-9)
    D = info["diag"].reshape(-1, 6, 6)
    M = info["inv_diag"].reshape(-1, 6, 6)
    eye = np.einsum("nij,njk->nik", D.astype(np.float64), M.astype(np.float64))
    np.testing.assert_allclose(eye, np.broadcast_to(np.eye(6), eye.shape), atol=2e-3)
    assert (np.diagonal(D, axis1=1, axis2=2) >= 1e-3 * (1 - 1e-6)).all()


def test_fp32_reference_mode_close_to_fp64(orc, tiny_scene):
    from starhub_b200.scenes import twist_error
    d64 = orc.solve(tiny_scene, precision=orc.ORC_PREC_FP64)
    d32 = orc.solve(tiny_scene, precision=orc.ORC_PREC_FP32_REFERENCE)
    assert twist_error(d32, d64, tiny_scene.nodes) < 5e-3


def test_mixed_mode_node_centred_matches_fp64(orc, small_scene):
    """FP32 bulk with FP64 reductions and node-centred twists: within 1e-4 twist and 1e-5 m
    of the all-FP64 solve (the device design, restated on the CPU)."""
    from starhub_b200.scenes import position_error, twist_error
    d64 = orc.solve(small_scene)
    dmx = orc.solve(small_scene, precision=orc.ORC_PREC_MIXED)
    assert twist_error(dmx, d64, small_scene.nodes) < 1e-4
    assert position_error(small_scene, dmx, d64) < 1e-5


def test_node_centred_first_step_is_a_change_of_variables(orc, small_scene):
    """Block-Jacobi PCG is invariant under per-node changes of twist coordinates: the
    node-centred step maps back onto the origin-twist step."""
    _, a = orc.solve(small_scene, gn_iters=1, pcg_iters=5, debug=True)
    _, b = orc.solve(small_scene, gn_iters=1, pcg_iters=5, debug=True, precision=orc.ORC_PREC_MIXED)
    c = small_scene.nodes[:, :3].astype(np.float64)
    xo = b["step"].astype(np.float64).copy()
    xo[:, 3:] += np.cross(c, xo[:, :3])
    np.testing.assert_allclose(xo, a["step"], atol=1e-5 * np.abs(a["step"]).max(), rtol=0)


def test_voxel_keys_sort_as_signed_ints(orc):
    """The reference sorts encodeVoxel's int keys (VoxelSubsamplerSorting.cu:8-21 with cub's
    signed order): a voxel below -512 in z has a negative key and comes first, before a voxel
    whose key is positive, whatever the input order."""
    voxel = np.float32(0.01)
    pts = np.array([[0.0, 0.0, 1.0, 1.0], [0.0, 0.0, -6.0, 1.0]], np.float32)   # vz = 100, vz = -600
    out = orc.OracleGeometry().voxel_subsample(pts, voxel)
    np.testing.assert_array_equal(out[:, 2], np.array([-6.0, 1.0], np.float32))


def test_render_solver_maps_rules(orc):
    """The oracle's restatement of the solver-map pass (shaders/solver_map.vert:29-33) on a hand
    case: nearest surfel wins a pixel, equal depth keeps the lower id, z >= max depth and z <= 0
    are culled, an unstable surfel is culled unless recently observed."""
    from starhub_b200.scenes import Camera
    cam = Camera(8, 6, 10.0, 10.0, 4.0, 3.0)
    vc = np.array([[0.0, 0.0, 1.0, 5.0],      # pixel (4, 3), z = 1
                   [0.0, 0.0, 0.5, 5.0],      # same pixel, nearer: wins
                   [0.0, 0.0, 0.5, 5.0],      # same depth, higher id: loses
                   [0.1, 0.0, 2.0, 5.0],      # z = max depth: culled
                   [0.0, 0.1, -1.0, 5.0],     # behind the camera: culled
                   [0.2, 0.0, 1.0, 0.5],      # unstable, observed at t = 9 (|9 - 10| < 3): drawn
                   [-0.2, 0.0, 1.0, 0.5]],    # unstable, observed at t = 2: culled
                  np.float32)
    nr = np.tile(np.array([[0, 0, -1, 0.002]], np.float32), (len(vc), 1))
    ct = np.zeros((len(vc), 4), np.float32)
    ct[:, 2] = [10, 10, 10, 10, 10, 9, 2]
    idx, vmap, nmap, rgbd = orc.render_solver_maps(vc, nr, ct, cam, np.eye(4), max_depth=2.0, current_time=10.0)
    assert idx[3, 4] == 1
    assert idx[3, 6] == 5                       # floor(10 * 0.2 / 1 + 4 + 0.5) = 6
    assert (idx != 0xFFFFFFFF).sum() == 2
    np.testing.assert_array_equal(vmap[3, 4], [0.0, 0.0, 0.5, 1.0])
    np.testing.assert_array_equal(nmap[3, 4], [0.0, 0.0, -1.0, 0.0])
    assert rgbd[3, 4, 3] == np.float32(2.0)
    assert (vmap[idx == 0xFFFFFFFF] == 0).all()
    # without the recent-observation pass every unstable surfel is culled
    idx2, _, _, _ = orc.render_solver_maps(vc, nr, ct, cam, np.eye(4), max_depth=2.0, current_time=10.0,
                                           time_threshold=-1.0)
    assert (idx2 != 0xFFFFFFFF).sum() == 1


def test_render_observation_maps_rules(orc):
    """The oracle's restatement of the observation-map pass (geometry.vert:40-86 with
    observation_map.frag:13-17): a surfel facing the camera is a point as wide as its disk's image
    (radius 106 mm at 1 m and f = 10: about 3 pixels, so a 3 x 3 square), a tiny surfel still draws
    one pixel (GL's minimum point size), the nearer surfel wins, the culls are the solver map's,
    and the colour is (byte / 255) * 2 - 1 with 1 / z beside it."""
    from starhub_b200.scenes import Camera
    cam = Camera(16, 12, 10.0, 10.0, 8.0, 6.0)
    vc = np.array([[0.0, 0.0, 1.0, 5.0],      # 0: 3 x 3 square around pixel (8, 6)
                   [0.2, 0.0, 1.0, 5.0],      # 1: tiny, pixel (10, 6)
                   [0.0, 0.0, 0.5, 5.0],      # 2: tiny and nearer: wins (8, 6)
                   [0.0, 0.0, -1.0, 5.0],     # 3: behind the camera: culled
                   [0.1, 0.0, 3.0, 5.0],      # 4: z = max depth: culled
                   [-0.3, 0.0, 1.0, 0.5],     # 5: unstable, observed at t = 2: culled
                   [0.3, 0.2, 1.0, 0.5]],     # 6: unstable, observed at t = 9: pixel (11, 8)
                  np.float32)
    nr = np.tile(np.array([[0, 0, -1, 1.0]], np.float32), (len(vc), 1))
    nr[0, 3] = 106.0
    ct = np.zeros((len(vc), 4), np.float32)
    ct[:, 2] = [10, 10, 10, 10, 10, 2, 9]
    ct[0, 0] = np.array([0x00FF0080], np.int32).view(np.float32)[0]   # colour bytes (255, 0, 128)
    idx, rgbd = orc.render_observation_maps(vc, nr, ct, cam, np.eye(4), max_depth=3.0, current_time=10.0)
    want = np.full((12, 16), 0xFFFFFFFF, np.uint32)
    want[5:8, 7:10] = 0
    want[6, 8] = 2
    want[6, 10] = 1
    want[8, 11] = 6
    np.testing.assert_array_equal(idx, want)
    third = np.float32(np.float32(128) / np.float32(255)) * np.float32(2) - np.float32(1)
    np.testing.assert_array_equal(rgbd[5, 7], np.array([1.0, -1.0, third, 1.0], np.float32))
    assert rgbd[6, 8, 3] == np.float32(2.0)
    assert (rgbd[idx == 0xFFFFFFFF] == 0).all()
    # without the recent-observation pass the unstable surfel 6 goes too
    idx2, _ = orc.render_observation_maps(vc, nr, ct, cam, np.eye(4), max_depth=3.0, current_time=10.0,
                                          time_threshold=-1.0)
    assert idx2[8, 11] == 0xFFFFFFFF and (idx2 != 0xFFFFFFFF).sum() == 10
