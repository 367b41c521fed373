"""cap3d front-end on the device: a small cap3d case (two wires over a ground
plane, two plate media, one dielectric block) extracted through the
front-end gives exactly the engine's result on the structure it builds, and
a physically consistent capacitance row."""
import numpy as np
import pytest

from deeprwcap_b200 import cap3d as C
from deeprwcap_b200 import engine
from test_cap3d import CASE

pytestmark = pytest.mark.gpu


def test_front_end_equals_engine(ctx, tmp_path):
    c = C.parse(CASE)
    res = C.extract(c, ctx=ctx, max_walks=200_000, p_tol=0.005)
    s = C.to_structure(c)
    p = C.job_params(s, 1, p_tol=0.005, c_ratio=0.9, max_walks=200_000)
    ref = engine.extract(s, p, ctx)
    assert res["walks"] == ref.walks and res["hops"] == ref.hops
    np.testing.assert_array_equal(res["cap_fF"], ref.cap[:4])
    row = res["row_F"]
    assert res["master"] == "A" and row["A"] > 0
    assert all(row[k] > 0 for k in ("GROUND", "B"))      # coupling magnitudes
    # the Maxwell row sums to zero in expectation: self = the sum of the
    # coupling magnitudes (window included), here to well inside 5 %
    coup = sum(v for k, v in row.items() if k != "A")
    assert abs(coup - row["A"]) <= 0.05 * row["A"]
    C.write_dspf([res], tmp_path / "a.dspf")
    back = C.parse_result(tmp_path / "a.dspf")
    err, self_err = C.compute_error({"A": row}, back)
    assert err < 1e-6 and self_err["A"] < 1e-6


def test_reference_case5_against_quickcap(ctx):
    """The reference's test case 5 (tests/golden/cap3d_case5.json, written from
    testcases/cap3d/case5.cap3d and its QuickCap result ref/case5.dspf by
    tests/golden/make_cap3d_fixtures.py), 2^20 walks at N = 16: the coupling
    row scored with the reference's metric (run_script.py:179-197) against
    QuickCap. Converged runs of this case score 0.2 %; the bar leaves room
    for the statistics of a fixed walk budget."""
    from pathlib import Path
    c, ref = C.load_case((Path(__file__).parent / "golden" / "cap3d_case5.json").read_text())
    res = C.extract(c, ctx=ctx, max_walks=1 << 20, p_tol=1e-9, c_tol=1e-9)
    assert res["walks"] == 1 << 20
    err, self_err = C.compute_error({res["master"]: res["row_F"]}, ref)
    assert err < 0.02, (err, res["row_F"], ref)
    assert self_err[res["master"]] < 0.01, self_err


def test_box_following_gauss_surface_agrees_with_bounding_box(ctx):
    """The small case's master A is L-shaped: its bounding box and the
    boundary of its own grown boxes are two different Gaussian surfaces
    around the same conductor, so they give the same capacitance row within
    the statistics (independent estimates)."""
    c = C.parse(CASE)
    s = C.to_structure(c)
    p0 = C.job_params(s, 1, p_tol=1e-9, c_tol=1e-9, max_walks=400_000)
    p1 = C.job_params(s, 1, p_tol=1e-9, c_tol=1e-9, max_walks=400_000)
    p1.gauss_surface = 1
    p1.gauss_offset = 0.5 * C.box_clearance(s, 1)
    p1.stop_dist = 1e-4 * p1.gauss_offset
    r0 = engine.extract(s, p0, ctx)
    r1 = engine.extract(s, p1, ctx)
    assert r0.walks == r1.walks == 400_000 and r1.lost == 0
    for e in range(s.n_nets + 1):
        z = abs(r1.cap[e] - r0.cap[e]) / np.hypot(r0.stderr[e], r1.stderr[e])
        assert z < 4.0, (e, r0.cap, r1.cap)
