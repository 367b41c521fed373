"""Write the cap3d fixture in this folder from the reference's own test case.

    python tests/golden/make_cap3d_fixtures.py [OUT_DIR] [CASE ...]

Reads testcases/cap3d/<case>.cap3d and its QuickCap result
testcases/cap3d/ref/<case>.dspf (or .spice) from the reference tree
($DRWC_REFERENCE_DIR, else ``reference`` beside this repository's folder),
parses them with deeprwcap_b200.cap3d (the same parser the front-end uses)
and stores the parsed structure and the QuickCap couplings as JSON:
cap3d_<case>.json. Default: case5 into this folder (the committed fixture).
"""
from __future__ import annotations

import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from deeprwcap_b200 import cap3d  # noqa: E402
from oracle.oracle import reference_dir  # noqa: E402


def main() -> None:
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE
    cases = sys.argv[2:] or ["case5"]
    base = reference_dir() / "testcases" / "cap3d"
    out.mkdir(parents=True, exist_ok=True)
    for case in cases:
        c = cap3d.parse(base / f"{case}.cap3d")
        refp = base / "ref" / f"{case}.dspf"
        if not refp.exists():
            refp = base / "ref" / f"{case}.spice"
        ref = cap3d.parse_result(refp)
        (out / f"cap3d_{case}.json").write_text(cap3d.dump_case(c, ref))
        print("wrote", out / f"cap3d_{case}.json")


if __name__ == "__main__":
    main()
