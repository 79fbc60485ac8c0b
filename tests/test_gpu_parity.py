"""GPU parity against the oracle, through the C ABI (libbt.so).

Integer and index results (sample counts, path reservations, segments, splat
counts, grid cell ids, neighbour counts) must be bit-exact. Positions, blurred
and normalised density are expected bit-exact too, since both sides evaluate
the same f32 operation sequence; the stated tolerances (1e-4 of the canvas
extent = 2e-4 clip units for positions, 1e-5 relative for density) are the
contract and are asserted as well.
"""
import json

import numpy as np
import pytest

import bundling_thingy_b200 as bt
from bundling_thingy_b200 import synthetic

from conftest import oracle_config

pytestmark = pytest.mark.gpu

POS_TOL = 2e-4          # 1e-4 of the canvas extent (2 clip units)
DENSITY_RTOL = 1e-5


def opts_for(w: synthetic.Workload, **kw) -> bt.Options:
    o = bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                   blur_sigma=w.sigma, blur_shrink=w.shrink, record_neighbors=True)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def pair(oracle, xy, starts, opts, threads=0):
    gpu = bt.Gpu(opts)
    ora = oracle.Pipeline(oracle_config(oracle, opts, threads))
    n_gpu = gpu.upload((xy, starts))
    n_ora = ora.upload(xy, starts)
    assert n_gpu == n_ora
    return gpu, ora


def check_geometry(gpu, ora):
    np.testing.assert_array_equal(gpu.read_paths(), ora.paths())
    np.testing.assert_array_equal(gpu.read_segments(), ora.segments())
    np.testing.assert_array_equal(gpu.read_edges(), ora.edges())


def check_points(gpu, ora):
    gxy, gid = gpu.read_points()
    oxy, oid = ora.points()
    np.testing.assert_array_equal(gid, oid)
    assert np.abs(gxy - oxy).max(initial=0) <= POS_TOL
    np.testing.assert_array_equal(gxy, oxy)


def check_density(gpu, ora):
    np.testing.assert_array_equal(gpu.read_counts(), ora.counts())
    graw, gpeak = gpu.read_density_raw()
    _, overt, opeak = ora.blurred()
    assert gpeak == opeak
    np.testing.assert_allclose(graw, overt, rtol=DENSITY_RTOL, atol=DENSITY_RTOL * max(opeak, 1e-30))
    np.testing.assert_array_equal(graw, overt)
    np.testing.assert_array_equal(gpu.read_density(), ora.normalized())


def check_neighbors(gpu, ora):
    np.testing.assert_array_equal(gpu.read_neighbors(), ora.neighbors())


def test_upload_small_config(oracle):
    w = synthetic.small()
    gpu, ora = pair(oracle, w.xy, w.starts, opts_for(w))
    check_geometry(gpu, ora)
    check_points(gpu, ora)
    check_density(gpu, ora)


def test_iterate_small_config_with_kernel_shrink(oracle):
    w = synthetic.small()
    gpu, ora = pair(oracle, w.xy, w.starts, opts_for(w))
    for it in range(w.iterations):
        gpu.iterate(1)
        ora.iterate(1)
        check_points(gpu, ora)
        check_neighbors(gpu, ora)
        check_density(gpu, ora)
    assert gpu.info().iterations == w.iterations


def test_reference_mode_full_canvas(oracle):
    # The reference's own settings: 1600^2 canvas, one-texel spacing, fixed
    # sigma-6 blur (src/gpu.rs:21, resampling.wgsl:87, blur.wgsl:41-60).
    w = synthetic.small()
    o = bt.Options(neighbor_radius=4, record_neighbors=True)
    gpu, ora = pair(oracle, w.xy, w.starts, o)
    check_geometry(gpu, ora)
    check_points(gpu, ora)
    check_density(gpu, ora)
    gpu.iterate(3)
    ora.iterate(3)
    check_points(gpu, ora)
    check_neighbors(gpu, ora)
    check_density(gpu, ora)


def test_iterate_mid_config(oracle):
    w = synthetic.mid()
    gpu, ora = pair(oracle, w.xy, w.starts, opts_for(w))
    check_geometry(gpu, ora)
    for _ in range(3):
        gpu.iterate(2)
        ora.iterate(2)
        check_points(gpu, ora)
        check_neighbors(gpu, ora)
    check_density(gpu, ora)


def test_large_config_upload_and_first_iteration(oracle):
    w = synthetic.large()
    gpu, ora = pair(oracle, w.xy, w.starts, opts_for(w))
    assert 4_500_000 < gpu.info().samples < 5_500_000
    check_geometry(gpu, ora)
    check_points(gpu, ora)
    check_density(gpu, ora)
    gpu.iterate(1)
    ora.iterate(1)
    check_points(gpu, ora)
    check_neighbors(gpu, ora)
    check_density(gpu, ora)


def test_large_config_invariants_over_iterations():
    # Size-independent properties at full size: endpoints stay fixed, every
    # sample is splatted once, positions stay inside the fitted box, the
    # normalised density peaks at 1, and reruns are identical.
    w = synthetic.large()
    runs = []
    for _ in range(2):
        gpu = bt.Gpu(opts_for(w))
        gpu.upload((w.xy, w.starts))
        base, _ = gpu.read_points()
        gpu.iterate(5)
        xy, ids = gpu.read_points()
        paths = gpu.read_paths()
        ends = np.concatenate([paths[:, 0], paths[:, 0] + paths[:, 2] - 1])
        np.testing.assert_array_equal(xy[ends], base[ends])
        assert gpu.read_counts().sum() == gpu.info().samples
        assert np.abs(xy).max() <= 0.95 + 1e-6
        dens = gpu.read_density()
        assert dens.max() == 1.0 and dens.min() >= 0.0
        runs.append(xy)
    np.testing.assert_array_equal(runs[0], runs[1])


@pytest.mark.parametrize("fine,fine_x", [(1, 0), (3, 0), (0, 0), (2, 8), (6, 24), (12, 12), (1, 5)])
def test_search_cell_size_does_not_change_results(oracle, fine, fine_x):
    # Square and flat search cells enumerate the same N(p).
    w = synthetic.small()
    o = opts_for(w, neighbor_radius=6, fine_cells=fine, fine_cells_x=fine_x)
    gpu, ora = pair(oracle, w.xy, w.starts, o)
    gpu.iterate(2)
    ora.iterate(2)
    check_points(gpu, ora)
    check_neighbors(gpu, ora)


@pytest.mark.parametrize("mode", [0, 1])
def test_search_modes_match_oracle(oracle, mode):
    # Interior cells from prefix sums (0) and testing every candidate (1)
    # enumerate the same N(p) and give identical sums.
    w = synthetic.mid()
    gpu, ora = pair(oracle, w.xy, w.starts, opts_for(w, search_mode=mode))
    gpu.iterate(2)
    ora.iterate(2)
    check_points(gpu, ora)
    check_neighbors(gpu, ora)


@pytest.mark.parametrize("radius,size", [(40, 1024), (33, 1600), (1, 512)])
def test_interior_bounds_at_other_radii(oracle, radius, size):
    # Large radii stress the conservative interior bounds; radius 1 has one
    # search cell per grid cell.
    w = synthetic.mid()
    o = bt.Options(width=size, height=size, neighbor_radius=radius, sample_spacing=w.spacing,
                   blur_sigma=w.sigma, record_neighbors=True)
    gpu, ora = pair(oracle, w.xy, w.starts, o)
    gpu.iterate(2)
    ora.iterate(2)
    check_points(gpu, ora)
    check_neighbors(gpu, ora)


def test_graphs_and_direct_launches_agree():
    w = synthetic.small()
    out = []
    for graphs in (True, False):
        gpu = bt.Gpu(opts_for(w, blur_shrink=1.0, use_graphs=graphs))
        gpu.upload((w.xy, w.starts))
        gpu.iterate(4)
        out.append((gpu.read_points()[0], gpu.read_density()))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_grid_cells_and_binning(oracle):
    w = synthetic.small()
    gpu, ora = pair(oracle, w.xy, w.starts, opts_for(w, neighbor_radius=5))
    gpu.iterate(1)
    ora.iterate(1)
    cells, gw, gh = ora.cells()
    np.testing.assert_array_equal(gpu.read_cells(), cells)
    info = gpu.info()
    assert (info.grid_width, info.grid_height) == (gw, gh)
    slots, starts = gpu.read_binning()
    ky, kx = info.fine_cells, info.fine_cells_x
    fw = gw * kx
    assert starts[-1] == info.samples
    assert np.all(np.diff(starts.astype(np.int64)) >= 0)
    assert np.array_equal(np.sort(slots), np.arange(info.samples))
    # Every sample sits in a search cell inside its grid cell, so each grid
    # cell's population equals the oracle's (compared as sets of samples).
    cell_of_slot = np.repeat(np.arange(starts.size - 1), np.diff(starts))
    fx, fy = cell_of_slot % fw, cell_of_slot // fw
    coarse = (fy // ky) * gw + (fx // kx)
    np.testing.assert_array_equal(coarse, cells[slots])


def test_kat_graphs_on_gpu(oracle):
    # Straight segment, short closed path, two-sample path (see the oracle KATs).
    cp = np.float32([[0, 0], [10, 0], [50, 0.1], [50.2, 0.1], [50, 0.1], [0, 5], [0.001, 5], [3, 7], [9, 2]])
    starts = np.uint32([0, 2, 5, 7, 9])
    o = bt.Options(width=101, height=101, neighbor_radius=3, record_neighbors=True)
    gpu, ora = pair(oracle, cp, starts, o)
    check_geometry(gpu, ora)
    check_points(gpu, ora)
    gpu.iterate(3)
    ora.iterate(3)
    check_points(gpu, ora)
    check_neighbors(gpu, ora)
    check_density(gpu, ora)


def test_long_paths_and_many_segments(oracle):
    # Paths with thousands of samples per segment and many control points
    # exercise the warp-parallel emit across chunks.
    rng = np.random.default_rng(5)
    cp = np.concatenate([np.float32([[0, 0], [1, 1]]), rng.random((300, 2), dtype=np.float32)])
    starts = np.uint32([0, 2, 302])
    o = bt.Options(width=4096, height=4096, neighbor_radius=8, record_neighbors=True)
    gpu, ora = pair(oracle, cp, starts, o)
    check_geometry(gpu, ora)
    check_points(gpu, ora)
    check_density(gpu, ora)
    gpu.iterate(1)
    ora.iterate(1)
    check_points(gpu, ora)


def test_edge_id_coloring_skips_density(oracle):
    w = synthetic.small()
    o = opts_for(w, color_by=bt.COLOR_BY_EDGE_ID)
    gpu, ora = pair(oracle, w.xy, w.starts, o)
    gpu.iterate(2)
    ora.iterate(2)
    check_points(gpu, ora)
    with pytest.raises(bt.BtError) as e:
        gpu.read_density()
    assert e.value.status == 8


def test_errors_follow_the_reference():
    w = synthetic.small()
    gpu = bt.Gpu(bt.Options(width=256, height=256))
    with pytest.raises(bt.BtError) as e:
        gpu.iterate(1)
    assert e.value.status == 8 and "neighbor radius is not configured" in e.value.message
    gpu = bt.Gpu(bt.Options(width=256, height=256, neighbor_radius=2))
    with pytest.raises(bt.BtError) as e:
        gpu.iterate(1)
    assert e.value.status == 4 and "no uploaded graph" in e.value.message
    bad = [
        (w.xy, np.uint32([0, 2, 5])),                          # starts do not end at the point count
        (np.float32([[0, 0], [np.nan, 1]]), np.uint32([0, 2])),
        (np.float32([[0, 0], [1, 1], [2, 2]]), np.uint32([0, 1, 3])),   # one-point edge
        (np.float32([[1, 1], [1, 1]]), np.uint32([0, 2])),     # zero extent
    ]
    for xy, starts in bad:
        with pytest.raises(bt.BtError) as e:
            gpu.upload((xy, starts))
        assert e.value.status == 3
    # The context stays usable after rejected input.
    assert gpu.upload((w.xy, w.starts)) > 0
    gpu.iterate(1)


def test_capacity_overflow_matches_oracle(oracle):
    # Allocation::new (resampling.rs:321-397): a 1 MiB budget leaves room for
    # a few thousand samples; the reference reports overflow 1.
    w = synthetic.small()
    o = opts_for(w, neighbor_radius=None, max_graph_memory_mib=1)
    gpu = bt.Gpu(o)
    with pytest.raises(bt.BtError) as e:
        gpu.upload((w.xy, w.starts))
    assert e.value.status == 1
    cap = gpu.info().capacity
    cfg = oracle_config(oracle, o)
    cfg.capacity = cap
    with pytest.raises(oracle.OracleError) as e2:
        oracle.Pipeline(cfg).upload(w.xy, w.starts)
    assert e2.value.status == 1


def test_reupload_releases_previous_graph(oracle):
    a, b = synthetic.small(), synthetic.small(seed_offset=100)
    o = opts_for(a)
    gpu = bt.Gpu(o)
    gpu.upload((a.xy, a.starts))
    gpu.iterate(2)
    gpu.upload((b.xy, b.starts))
    ora = oracle.Pipeline(oracle_config(oracle, o))
    ora.upload(b.xy, b.starts)
    assert gpu.info().iterations == 0
    check_points(gpu, ora)
    gpu.iterate(2)
    ora.iterate(2)
    check_points(gpu, ora)


def test_distortion_matches_oracle(oracle):
    w = synthetic.small()
    o = opts_for(w, evaluate_distortion=True)
    gpu, ora = pair(oracle, w.xy, w.starts, o)
    base, _ = ora.points()
    assert gpu.distortion(bt.SIZE).distortion == 0.0
    gpu.iterate(3)
    ora.iterate(3)
    cur, _ = ora.points()
    d, px = oracle.distortion(ora.paths(), base, cur, bt.SIZE)
    m = gpu.distortion(bt.SIZE)
    assert abs(m.distortion - d) <= 1e-12 * max(d, 1e-30)
    assert abs(m.rms_displacement_pixels - px) <= 1e-12 * max(px, 1e-30)
    # The host readers reproduce it from the 12-byte records (geometry.rs).
    layout = gpu.distortion_layout()
    snap = gpu.distortion_snapshot(layout)
    np.testing.assert_array_equal(snap.positions, cur)


def test_stage_timings():
    w = synthetic.small()
    gpu = bt.Gpu(opts_for(w, timing=True))
    gpu.upload((w.xy, w.starts))
    up = gpu.stage_times()
    assert {"graph.count", "graph.emit", "density.blur_horizontal"} <= set(up)
    gpu.iterate(2)
    it = gpu.stage_times()
    assert {"graph.neighbor_mean", "graph.grid_scan", "graph.grid_scatter",
            "density.blur_vertical_and_maximum", "density.normalize"} <= set(it)
    assert all(v >= 0 for v in it.values())


def test_autotune_returns_an_equivalent_shape(oracle):
    w = synthetic.small()
    tuned, ms = bt.autotune(opts_for(w), w.xy, w.starts, 2)
    assert ms > 0
    assert tuned.fine_cells >= 1 and tuned.fine_cells_x >= tuned.fine_cells
    gpu, ora = pair(oracle, w.xy, w.starts, tuned)
    gpu.iterate(2)
    ora.iterate(2)
    check_points(gpu, ora)


def test_upload_picks_flat_search_cells_for_dense_graphs(oracle):
    # The shape is chosen from the graph's density at upload; any shape
    # enumerates the same neighbourhoods.
    w = synthetic.mid()
    gpu, ora = pair(oracle, w.xy, w.starts, opts_for(w))
    info = gpu.info()
    assert info.fine_cells_x > info.fine_cells >= 1
    gpu.iterate(2)
    ora.iterate(2)
    check_points(gpu, ora)
    check_density(gpu, ora)


def test_headless_distortion_report(oracle, tmp_path, capsys):
    # The headless run's distortion.json (src/main.rs:104-191): the device and
    # host measurements agree, and iteration 3 matches the oracle.
    from bundling_thingy_b200 import report

    w = synthetic.small()
    trl = tmp_path / "g.trl"
    synthetic.write_trl(trl, w.xy, w.starts)
    base = dict(width=w.width, height=w.height, sample_spacing=w.spacing, blur_sigma=w.sigma,
                blur_shrink=w.shrink)
    (tmp_path / "out").mkdir()
    (tmp_path / "out" / "distortion.json").write_text("stale")
    r_dev = report.headless_distortion(trl, tmp_path / "out", neighbor_radius=w.radius, iterations=3,
                                       options=bt.Options(**base))
    printed = capsys.readouterr().out.splitlines()
    assert printed[0] == "original.png distortion=0 rms_displacement_pixels=0"
    assert printed[1].startswith("iteration-01.png distortion=")
    r_host = report.headless_distortion(trl, tmp_path / "host", neighbor_radius=w.radius, iterations=3,
                                        options=bt.Options(**base), measure="host", echo=False)
    assert [i["file"] for i in r_dev["images"]] == ["original.png", "iteration-01.png", "iteration-02.png",
                                                    "iteration-03.png"]
    for a, b in zip(r_dev["images"], r_host["images"]):
        assert abs(a["distortion"] - b["distortion"]) <= 1e-12 * max(b["distortion"], 1e-30)
        assert abs(a["rms_displacement_pixels"] - b["rms_displacement_pixels"]) <= \
            1e-12 * max(b["rms_displacement_pixels"], 1e-30)
    assert json.loads((tmp_path / "out" / "distortion.json").read_text()) == r_dev
    assert r_dev["bundling"] == {"neighbor_radius": w.radius, "iterations": 3}
    # Iteration 3 against the oracle run of the same parsed graph.
    g = bt.Graph.load(trl)
    o = bt.Options(neighbor_radius=w.radius, evaluate_distortion=True, **base)
    gpu, ora = pair(oracle, g.points(), g.starts(), o)
    b0, _ = ora.points()
    ora.iterate(3)
    d, px = oracle.distortion(ora.paths(), b0, ora.points()[0], bt.SIZE)
    last = r_dev["images"][-1]
    assert abs(last["distortion"] - d) <= 1e-12 * d
    assert abs(last["rms_displacement_pixels"] - px) <= 1e-12 * px
    assert r_dev["geometry"]["active_samples"] == gpu.info().samples


@pytest.mark.parametrize("size,sigma", [(1001, 8.0), (512, 20.0), (1600, 0.0)])
def test_density_paths_with_and_without_tma(oracle, size, sigma):
    # The context's blur passes are TMA-staged when the map's sides are
    # multiples of 4 and the halo is at most 48 texels (sigma <= 16), and
    # element-staged otherwise: an odd side, a wide halo, and the reference's
    # sigma-6 table on its 1600^2 canvas all match the oracle bit for bit.
    w = synthetic.small()
    o = bt.Options(width=size, height=size, neighbor_radius=4, blur_sigma=sigma, record_neighbors=True)
    gpu, ora = pair(oracle, w.xy, w.starts, o)
    check_density(gpu, ora)
    gpu.iterate(2)
    ora.iterate(2)
    check_points(gpu, ora)
    check_density(gpu, ora)
