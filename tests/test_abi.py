"""CPU checks of the C-ABI boundary: the library loads and exports every
entry point include/drwc.h declares (no compute calls: no GPU here)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    txt = (ROOT / "include" / "drwc.h").read_text()
    return sorted(set(re.findall(r"DRWC_API\s+[\w\s\*]+?\b(drwc_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "drwc_ggft_solve" in syms and "drwc_frw_run" in syms
    from deeprwcap_b200 import abi
    assert sorted(abi.EXPORTS) == syms


def test_library_exports_every_declared_symbol():
    from deeprwcap_b200 import abi
    if not abi.LIB_PATH.exists():
        from deeprwcap_b200 import build
        build.build()
    lib = C.CDLL(str(abi.LIB_PATH))
    for s in declared_symbols():
        assert hasattr(lib, s), s


def test_pure_entry_points_without_device():
    """Calls that touch no device: version, status strings, defaults and the
    argument checks that run before any CUDA call."""
    from deeprwcap_b200 import abi
    L = abi.load()
    assert b"sm_100a" in L.drwc_version()
    assert L.drwc_status_string(0) == b"ok"
    o = abi.default_fdm_opts()
    assert o.tol == 1e-10 and o.max_outer == 8
    p = abi.default_job_params()
    assert p.N == 16 and p.max_hops == 10000
    assert L.drwc_ggft_solve(None, 16, None, 0, 0.0, None, None) == 1
    assert L.drwc_ctx_destroy(None) == 1
    h = C.c_void_p()
    rc = L.drwc_ctx_create(0, C.byref(h))
    assert rc in (0, 5)  # no device in this container -> DRWC_ERR_NO_DEVICE
    if rc == 0:
        L.drwc_ctx_destroy(h)


def test_product_does_not_import_oracle():
    """The product package never reaches into oracle/."""
    for f in (ROOT / "deeprwcap_b200").rglob("*"):
        if f.suffix in (".py", ".cu", ".cuh", ".cpp", ".h"):
            txt = f.read_text()
            assert "oracle" not in re.sub(r"#.*|//.*", "", txt).replace("oracle/_ref", ""), f


def test_server_defaults_and_argument_checks_without_device():
    """The server's option defaults (struct layout shared with the header)
    and the checks that reject a request before any CUDA call."""
    from deeprwcap_b200 import abi, engine
    L = abi.load()
    o = engine.server_opts()
    # slots 0 / fdm_hops 0 / straggler_hops 0: defaults applied at creation (65536 slots,
    # up to 64 hops per step for a walk past its 32nd hop or in a job's tail)
    assert (o.slots, o.max_jobs, o.hbm_budget, o.n_sizes) == (0, 32, 1 << 30, 3)
    assert o.fdm_hops == 0 and o.straggler_hops == 0
    assert C.sizeof(abi.ServerOpts) == 80  # static_assert in csrc/serve.cu
    assert list(o.sizes[:3]) == [16, 21, 23] and o.steps_per_graph == 2
    assert o.max_materials == 16 and o.max_nets == 64 and abs(o.audit_frac - 0.01) < 1e-7
    o2 = engine.server_opts(sizes=(16, 23), slots=1024)
    assert o2.n_sizes == 2 and list(o2.sizes[:2]) == [16, 23] and o2.slots == 1024
    h = C.c_void_p()
    assert L.drwc_server_create(None, C.byref(o), None, 0, C.byref(h)) == 1
    assert L.drwc_server_destroy(None) == 1
    st = abi.ServerStats()
    assert L.drwc_server_stats_get(None, C.byref(st)) == 1
    jid = C.c_int64()
    assert L.drwc_server_submit(None, None, None, C.byref(jid)) == 1
