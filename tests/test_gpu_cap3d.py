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
