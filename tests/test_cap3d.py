"""cap3d front-end on the CPU: parsing, the engine structure it builds, the
Gaussian-surface clearance, and the reference's result parsers and error
metric (executable/run_script.py:24-75, 179-197) on small files written
here."""
import numpy as np
import pytest

from deeprwcap_b200 import cap3d as C

CASE = """<cap3d>
<window>
\tname box
\tv1(-2.0,-2.0,0.0)
\tv2(4.0,3.0,5.0)
</window>
<plate_medium>
\tname TOP
\tdiel 2.5
\tz_top 5.0
</plate_medium>
<plate_medium>
\tname BOT
\tdiel 3.9
\tz_top 1.0
</plate_medium>
<medium>
\tname blob
\t<block>
\t\tlayer 0
\t\tbasepoint(1.0,1.0,2.5)
\t\tv1(0.5,0,0)
\t\tv2(0,0.5,0)
\t\thvector(0,0,0.5)
\t</block>
\tdiel 7.0
</medium>
<conductor>
\tname GROUND
\t<block>
\t\tname 0
\t\tlayer 2
\t\tbasepoint(-2.0,-2.0,0.0)
\t\tv1(6.0,0,0)
\t\tv2(0,5.0,0)
\t\thvector(0,0,0.2)
\t</block>
</conductor>
<conductor>
\tname A
\t<block>
\t\tname 0
\t\tlayer 5
\t\tbasepoint(0.0,0.0,1.2)
\t\tv1(2.0,0,0)
\t\tv2(0,0.3,0)
\t\thvector(0,0,0.3)
\t</block>
\t<block>
\t\tname 1
\t\tlayer 5
\t\tbasepoint(2.0,0.3,1.2)
\t\tv1(-0.3,0,0)
\t\tv2(0,1.0,0)
\t\thvector(0,0,0.3)
\t</block>
</conductor>
<conductor>
\tname B
\t<block>
\t\tname 0
\t\tlayer 5
\t\tbasepoint(0.0,2.0,1.2)
\t\tv1(1.0,0,0)
\t\tv2(0,0.3,0)
\t\thvector(0,0,0.3)
\t</block>
</conductor>
<layer>
\tname M1
\tid 5
\ttype interconnect
</layer>
<task>
\t<capacitance>
\t\tA
\t</capacitance>
</task>
<parameter>
\tc-ratio 0.900000
</parameter>
</cap3d>
"""


def test_parse_sections():
    c = C.parse(CASE)
    np.testing.assert_array_equal(c.window_lo, [-2, -2, 0])
    np.testing.assert_array_equal(c.window_hi, [4, 3, 5])
    assert c.net_names == ["GROUND", "A", "B"] and c.masters == ["A"] and c.c_ratio == 0.9
    assert [p[:2] for p in c.plates] == [("TOP", 2.5), ("BOT", 3.9)]
    # a negative edge vector spans the box below its base point
    np.testing.assert_allclose(c.conductors[1][1][1], [1.7, 0.3, 1.2, 2.0, 1.3, 1.5])


def test_structure():
    s = C.to_structure(C.parse(CASE))
    assert s.n_nets == 3 and list(s.nets) == [0, 1, 1, 2]
    # layers sorted by z_top: BOT from the window bottom, TOP from BOT's top
    np.testing.assert_array_equal(s.layer_zlo, [0.0, 1.0])
    np.testing.assert_array_equal(s.layer_eps, [3.9, 2.5])
    np.testing.assert_allclose(s.diel, [[1.0, 1.0, 2.5, 1.5, 1.5, 3.0, 7.0]])
    np.testing.assert_array_equal(s.encl_lo, [-2, -2, 0])


def test_pieces_of_a_net_are_merged():
    text = CASE.replace("\tname B\n", "\tname 12__B\n").replace(
        "<layer>", "<conductor>\n\tname 3__B\n\t<block>\n\t\tbasepoint(3.0,2.0,1.2)\n"
        "\t\tv1(0.5,0,0)\n\t\tv2(0,0.3,0)\n\t\thvector(0,0,0.3)\n\t</block>\n"
        "</conductor>\n<conductor>\n\tname A\n\t<block>\n\t\tbasepoint(-1.0,-1.0,3.0)\n"
        "\t\tv1(0.2,0,0)\n\t\tv2(0,0.2,0)\n\t\thvector(0,0,0.2)\n\t</block>\n"
        "</conductor>\n<layer>", 1)
    c = C.parse(text)
    assert len(c.conductors) == 5 and c.net_names == ["GROUND", "A", "B"]
    s = C.to_structure(c)
    assert s.n_nets == 3 and list(s.nets) == [0, 1, 1, 2, 2, 1]
    assert C.net_of("9__signalGND") == "signalGND" and C.net_of("ln_14") == "ln_14"


def test_clearance_and_job_params():
    c = C.parse(CASE)
    s = C.to_structure(c)
    # master A's box [0, 2] x [0, 1.3] x [1.2, 1.5]: B is 0.7 away in y,
    # the ground plane 1.0 below
    assert C.clearance(s, 1) == pytest.approx(0.7)
    p = C.job_params(s, 1, c_ratio=c.c_ratio)
    assert p.gauss_offset == pytest.approx(0.35) and p.stop_dist == pytest.approx(0.35e-4)
    assert p.master == 1 and p.c_ratio == pytest.approx(0.9) and p.gauss_surface == 0
    # B reaches into A's (L-shaped) bounding box without touching A's boxes:
    # the Gaussian surface follows A's boxes, grown by half their gap to B
    s.boxes[3, 1] = 1.2
    p = C.job_params(s, 1)
    assert p.gauss_surface == 1 and C.box_clearance(s, 1) == pytest.approx(0.7)
    assert p.stop_dist == pytest.approx(0.35e-4)  # offsets per box, up to gauss_offset
    s.boxes[3, 3] = 1.7  # B now touches A's second box
    with pytest.raises(ValueError):
        C.job_params(s, 1)


def test_rejects_malformed_blocks():
    bad = CASE.replace("v1(2.0,0,0)", "v1(2.0,0.1,0)")
    with pytest.raises(ValueError):
        C.parse(bad)
    with pytest.raises(ValueError):
        C.parse(CASE.replace("</conductor>\n<layer>", "<layer>", 1))


def _close(a, b):
    assert a.keys() == b.keys()
    for m in a:
        assert a[m].keys() == b[m].keys()
        for k in a[m]:
            assert a[m][k] == pytest.approx(b[m][k], rel=1e-7)


def test_result_parsers_and_metric(tmp_path):
    dspf = ("*|NET A 1.0e-15\nC0 A B 2.0e-16\nC1 A 0 5.0e-16\nC2 A B 4.0e-16\n")
    ref = C.parse_dspf(dspf)
    # "0" is GROUND; a pair listed twice keeps the mean
    assert ref == {"A": {"A": 1.0e-15, "B": 3.0e-16, "GROUND": 5.0e-16}}
    spice = ("** A 1.0fF * (+/-0.2%) (total)\nCp1 A B 0.3fF * (+/-1%)\n"
             "Cp2 A 0 0.0005pF * (+/-1%)\n")
    _close(C.parse_spice(spice), ref)
    assert C.parse_cap_unit("2.5fF") == pytest.approx(2.5e-15)
    mine = {"A": {"A": 1.1e-15, "B": 2.7e-16, "WINDOW": 1e-17}}
    err, self_err = C.compute_error(mine, ref)
    # |1.1-1.0| + |0.27-0.3| + |0-0.5| over 1.0 + 0.3 + 0.5
    assert err == pytest.approx((0.1 + 0.03 + 0.5) / 1.8)
    assert self_err["A"] == pytest.approx(0.1)
    out = tmp_path / "r.dspf"
    C.write_dspf([{"master": "A", "row_F": {"A": 1.0e-15, "B": 3.0e-16, "GROUND": 5.0e-16}}], out)
    _close(C.parse_result(out), ref)


def test_reference_case5_fixture_round_trip():
    """The committed fixture of the reference's case 5 (parsed structure and
    QuickCap couplings) loads back into the front-end's structure."""
    from pathlib import Path
    text = (Path(__file__).parent / "golden" / "cap3d_case5.json").read_text()
    c, ref = C.load_case(text)
    assert C.dump_case(c, ref) == text
    s = C.to_structure(c)
    master = C.net_of(c.masters[0])
    assert master in ref and set(ref[master]) <= set(c.net_names)
    assert len(s.boxes) == 25 and len(s.diel) == 38 and len(c.plates) == 32
    assert C.clearance(s, c.net_names.index(master)) > 0
