"""Build ``deeprwcap_b200/libdrwc.so`` from ``deeprwcap_b200/csrc`` for sm_100a.

    python -m deeprwcap_b200.build [--verbose] [--ptxas-v]

Each ``.cu`` file is compiled to an object in ``deeprwcap_b200/_build`` (in
parallel), then linked into one shared library with the C ABI of
``include/drwc.h``. Objects are rebuilt when their source or any header is
newer. The library is built in-tree so it travels with the repository.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = Path(os.environ.get("DRWC_BUILD_DIR", str(PKG / "_build")))
LIB = Path(os.environ.get("DRWC_LIBRARY", str(PKG / "libdrwc.so")))

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", str(ROOT / "include")]
# Extra -D flags (tuning sweeps build variants into another folder with these).
EXTRA = os.environ.get("DRWC_NVCC_DEFINES", "").split()


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def _headers():
    return list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))


def _deps(dep: Path) -> list[Path] | None:
    """Headers a source included at its last compile (nvcc -MD output)."""
    if not dep.exists():
        return None
    text = dep.read_text().replace("\\\n", " ")
    names = text.split(":", 1)[1].split() if ":" in text else []
    return [Path(n) for n in names]


def _compile(src: Path, verbose: bool, ptxas_v: bool) -> tuple[Path, str]:
    obj = BUILD / (src.stem + ".o")
    dep = BUILD / (src.stem + ".d")
    deps = _deps(dep)
    if deps is None or not all(d.exists() for d in deps):
        deps = _headers()
    newest = max([src.stat().st_mtime] + [h.stat().st_mtime for h in deps])
    if obj.exists() and obj.stat().st_mtime >= newest and not ptxas_v:
        return obj, ""
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *EXTRA, "-MD", "-MF", str(dep), "-c", str(src),
           "-o", str(obj)]
    if ptxas_v:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr}\n{r.stdout}")
    return obj, (r.stderr if (verbose or ptxas_v) else "")


def build(verbose: bool = False, ptxas_v: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    jobs = jobs or min(len(sources), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose, ptxas_v), sources))
    for obj, log in results:
        if log:
            print(f"--- {obj.name}\n{log}", file=sys.stderr)
    objs = [str(o) for o, _ in results]
    newest_obj = max(Path(o).stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest_obj:
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas_v, a.j))


if __name__ == "__main__":
    main()
