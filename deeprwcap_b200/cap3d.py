"""cap3d front-end: read a cap3d structure, extract the capacitance row of its
task's master net with the FRW engine, write it as a DSPF net, and score a
result against a QuickCap reference with the reference's error metric.

    python -m deeprwcap_b200.cap3d CASE.cap3d [--ref REF.dspf|REF.spice] [--N 16]
        [-p 0.01] [-c 0.01] [--c-ratio R] [--out OUT.dspf] [--max-walks 1e7]

cap3d sections read (the format of the reference's test cases,
testcases/cap3d/*.cap3d); lengths in um:

    <window> v1(x,y,z) v2(x,y,z)        the simulation box: the grounded enclosure
    <plate_medium> diel, z_top           stratified dielectric, stacked by z_top
    <medium> <block>...</block> diel     dielectric blocks (a later one overrides an earlier)
    <conductor> name <block>...</block>  conductors; a "<k>__" name prefix numbers
                                         the pieces of one net, and conductors
                                         of the same name are one net
    <block> basepoint(..) v1(..) v2(..) hvector(..)
                                         an axis-aligned box spanned by three
                                         edge vectors from its base point
    <task> <capacitance> NAME ...        master net(s)
    <parameter> c-ratio R                the coupling-convergence ratio
    <layer> ...                          process-layer metadata (not needed)

The engine's Gaussian surface is the master's bounding box grown by an
offset; by default half the L-infinity clearance between that box and the
nearest other conductor (or the window), so it cuts no other net. The
result row is the engine's (fF, Maxwell row: self positive, couplings
negative, the window last); the DSPF output lists the total and each
coupling magnitude in F, as QuickCap does.

Result parsing and the error metric restate executable/run_script.py:
``parse_cap_unit`` (:24-31), ``parse_spice`` (:32-54), ``parse_dspf``
(:55-75) and ``compute_error`` (:179-197): the summed absolute coupling
error over the summed reference magnitudes, plus the relative self-
capacitance error per master.
"""
from __future__ import annotations

import argparse
import json
import re
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import workloads as W

_VEC = re.compile(r"^(\w+)\s*\(([^)]*)\)\s*$")


@dataclass
class Cap3d:
    window_lo: np.ndarray
    window_hi: np.ndarray
    plates: list = field(default_factory=list)      # (name, eps, z_top)
    media: list = field(default_factory=list)       # (name, eps, [box [6]])
    conductors: list = field(default_factory=list)  # (name, [box [6]])
    masters: list = field(default_factory=list)
    c_ratio: float | None = None

    @property
    def net_names(self) -> list:
        """Nets in order of first appearance (conductors of one net merged)."""
        out = []
        for name, _ in self.conductors:
            n = net_of(name)
            if n not in out:
                out.append(n)
        return out


def net_of(conductor: str) -> str:
    """Net of a conductor: a ``<digits>__`` prefix numbers the pieces of one
    net (``9__signalGND`` is a piece of ``signalGND``), and conductors of the
    same name are one net."""
    m = re.match(r"^\d+__(.+)$", conductor)
    return m.group(1) if m else conductor


def _box(b: dict, where: str) -> list:
    """[lo xyz, hi xyz] of a block; every edge vector must lie along one axis
    and the three along different axes."""
    base = np.asarray(b.get("basepoint"), dtype=np.float64)
    vs = [np.asarray(b.get(k), dtype=np.float64) for k in ("v1", "v2", "hvector")]
    if base.shape != (3,) or any(v.shape != (3,) for v in vs):
        raise ValueError(f"{where}: block needs basepoint, v1, v2 and hvector")
    axes = []
    for v in vs:
        nz = np.flatnonzero(v)
        if len(nz) != 1:
            raise ValueError(f"{where}: only axis-aligned blocks are supported")
        axes.append(int(nz[0]))
    if sorted(axes) != [0, 1, 2]:
        raise ValueError(f"{where}: block edges must span three axes")
    lo, hi = base.copy(), base.copy()
    for v in vs:
        lo += np.minimum(v, 0.0)
        hi += np.maximum(v, 0.0)
    return [*lo, *hi]


def parse(source) -> Cap3d:
    """Parse cap3d text (a path or the text itself)."""
    text = Path(source).read_text() if isinstance(source, Path) or (
        isinstance(source, str) and "\n" not in source and Path(source).exists()) else source
    stack: list = []
    cur: dict = {}
    block: dict | None = None
    win: dict = {}
    cap = None
    plates, media, conductors, masters = [], [], [], []
    c_ratio = None
    for ln, raw in enumerate(text.splitlines(), 1):
        line = raw.strip()
        if not line or line.startswith("#"):
            continue
        where = f"line {ln}"
        if line.startswith("</"):
            tag = line[2:-1]
            if not stack or stack[-1] != tag:
                raise ValueError(f"{where}: unexpected </{tag}>")
            stack.pop()
            if tag == "block":
                cur.setdefault("blocks", []).append(_box(block, where))
                block = None
            elif tag == "plate_medium":
                plates.append((cur.get("name", ""), float(cur["diel"]), float(cur["z_top"])))
            elif tag == "medium":
                media.append((cur.get("name", ""), float(cur["diel"]), cur.get("blocks", [])))
            elif tag == "conductor":
                if not cur.get("blocks"):
                    raise ValueError(f"{where}: conductor {cur.get('name')} has no block")
                conductors.append((cur["name"], cur["blocks"]))
            elif tag == "window":
                win = dict(cur)
            continue
        if line.startswith("<"):
            tag = line[1:-1]
            stack.append(tag)
            if tag == "block":
                block = {}
            elif tag in ("plate_medium", "medium", "conductor", "window", "layer"):
                cur = {}
            continue
        ctx = stack[-1] if stack else ""
        m = _VEC.match(line)
        if m:
            vec = [float(t) for t in m.group(2).split(",")]
            (block if ctx == "block" else cur)[m.group(1)] = vec
            continue
        key, _, val = line.partition(" ")
        val = val.strip()
        if ctx == "capacitance":
            masters.extend(line.split())
        elif ctx == "parameter":
            if key == "c-ratio":
                c_ratio = float(val)
        elif ctx == "block":
            block[key] = val
        else:
            cur[key] = val
    if stack:
        raise ValueError(f"unclosed <{stack[-1]}>")
    if "v1" not in win or "v2" not in win:
        raise ValueError("no <window>")
    a, b = np.asarray(win["v1"]), np.asarray(win["v2"])
    cap = Cap3d(np.minimum(a, b), np.maximum(a, b), plates, media, conductors, masters, c_ratio)
    if not conductors:
        raise ValueError("no <conductor>")
    return cap


def dump_case(c: Cap3d, ref: dict | None = None) -> str:
    """The parsed case (and a reference result, {master: {net: F}}) as JSON
    text; ``load_case`` reads it back."""
    def boxes(bl):
        return [list(map(float, b)) for b in bl]
    return json.dumps({
        "window_lo": list(map(float, c.window_lo)), "window_hi": list(map(float, c.window_hi)),
        "plates": [[n, float(e), float(z)] for n, e, z in c.plates],
        "media": [[n, float(e), boxes(bl)] for n, e, bl in c.media],
        "conductors": [[n, boxes(bl)] for n, bl in c.conductors],
        "masters": list(c.masters), "c_ratio": c.c_ratio, "ref": ref})


def load_case(text: str) -> tuple[Cap3d, dict | None]:
    d = json.loads(text)
    c = Cap3d(np.asarray(d["window_lo"]), np.asarray(d["window_hi"]),
              [tuple(p) for p in d["plates"]], [(n, e, bl) for n, e, bl in d["media"]],
              [(n, bl) for n, bl in d["conductors"]], list(d["masters"]), d["c_ratio"])
    return c, d["ref"]


# Which of several overlapping media blocks holds a point: the one listed
# last ("last": a later <medium> is painted over the earlier ones, as the
# reference's cases nest conformal shells outer to inner), the one listed
# first ("first"), or the smallest ("smallest"). Scored against QuickCap on
# the reference's cases, "last" is the format's rule (case7: 3.2 % error,
# 37 % with "first").
MEDIA_ORDER = "last"


def to_structure(c: Cap3d, media_order: str | None = None) -> W.StructureSpec:
    """The engine structure: conductor boxes with net ids in order of the
    nets' first appearance (pieces of one net merged, see ``net_of``),
    plate media as layers (layer l from the previous z_top, the first from
    the window bottom), media blocks as dielectric blocks ordered so that
    the engine's first containing block is the one ``media_order`` (default
    MEDIA_ORDER) picks, the window as the grounded enclosure."""
    boxes, nets = [], []
    ids = {n: i for i, n in enumerate(c.net_names)}
    for name, bl in c.conductors:
        boxes.extend(bl)
        nets.extend([ids[net_of(name)]] * len(bl))
    plates = sorted(c.plates, key=lambda p: p[2])
    if plates:
        zlo = [float(c.window_lo[2])] + [p[2] for p in plates[:-1]]
        eps = [p[1] for p in plates]
    else:
        zlo, eps = [float(c.window_lo[2])], [1.0]
    diel = [[*b, e] for _, e, bl in c.media for b in bl]
    order = media_order or MEDIA_ORDER
    if order == "last":
        diel = diel[::-1]
    elif order == "smallest":
        diel = sorted(diel, key=lambda d: (d[3] - d[0]) * (d[4] - d[1]) * (d[5] - d[2]))
    return W.StructureSpec(np.asarray(boxes, dtype=np.float64).reshape(-1, 6),
                           np.asarray(nets, dtype=np.int32), len(ids),
                           np.asarray(zlo, dtype=np.float64), np.asarray(eps, dtype=np.float64),
                           np.asarray(diel, dtype=np.float64).reshape(-1, 7),
                           c.window_lo.astype(np.float64), c.window_hi.astype(np.float64))


def clearance(s: W.StructureSpec, master: int) -> float:
    """L-infinity gap between the master's bounding box and the nearest other
    conductor box or window wall (<= 0: the box touches another net)."""
    mb = s.boxes[s.nets == master]
    lo, hi = mb[:, :3].min(axis=0), mb[:, 3:].max(axis=0)
    gap = min(float((lo - s.encl_lo).min()), float((s.encl_hi - hi).min()))
    other = s.boxes[s.nets != master]
    if len(other):
        sep = np.maximum(other[:, :3] - hi, lo - other[:, 3:]).max(axis=1)
        gap = min(gap, float(sep.min()))
    return gap


def box_clearance(s: W.StructureSpec, master: int) -> float:
    """L-infinity gap between the master's own boxes and the nearest other
    conductor box or window wall."""
    mb = s.boxes[s.nets == master]
    gap = min(float((mb[:, :3] - s.encl_lo).min()), float((s.encl_hi - mb[:, 3:]).min()))
    other = s.boxes[s.nets != master]
    if len(other):
        sep = np.maximum(other[None, :, :3] - mb[:, None, 3:],
                         mb[:, None, :3] - other[None, :, 3:]).max(axis=2)
        gap = min(gap, float(sep.min()))
    return gap


def job_params(s: W.StructureSpec, master: int, N: int = 16, p_tol: float = 0.01,
               c_tol: float = 0.01, c_ratio: float = 0.95, offset: float | None = None,
               stop_rel: float = 1e-4, seed: int = 1, max_walks: int = 10_000_000,
               batch_walks: int = 1 << 16):
    """Job parameters for one master. The Gaussian surface is the master's
    bounding box grown by half its clearance when that box cuts no other
    net; otherwise (a master of many pieces wrapped around other nets) the
    outer boundary of the master's boxes, each grown by half its own gap to
    the other nets (gauss_surface = 1, the engine sizes each box's offset;
    gauss_offset is then the largest offset allowed, stop_dist scales with
    the smallest)."""
    gap = clearance(s, master)
    mode = 0
    stop_ref = None
    if not gap > 0:
        gap = box_clearance(s, master)
        mode = 1
        if not gap > 0:
            raise ValueError("the master's boxes touch another conductor; no Gaussian "
                             "surface around them avoids the other nets")
        stop_ref = 0.5 * gap
        gap = float(np.max(s.encl_hi - s.encl_lo))  # no cap below each box's own half gap
    off = 0.5 * gap if offset is None else float(offset)
    stop = stop_rel * (off if stop_ref is None else min(off, stop_ref))
    return W.job_params_plain(N=N, master=master, seed=seed, p_tol=p_tol, c_tol=c_tol,
                              c_ratio=c_ratio, gauss_offset=off, stop_dist=stop,
                              min_walks=min(batch_walks, max_walks), max_walks=max_walks,
                              batch_walks=batch_walks, tol=1e-8, gauss_surface=mode)


def extract(c: Cap3d, master: str | None = None, ctx=None, **kw) -> dict:
    """Capacitance row of one master (default: the task's first) through
    ``engine.extract``; couplings in F keyed by net name (the window as
    ``WINDOW``), plus the engine's raw row and run statistics."""
    from . import engine
    s = to_structure(c)
    name = net_of(master) if master else (net_of(c.masters[0]) if c.masters else c.net_names[0])
    if name not in c.net_names:
        raise ValueError(f"master {name!r} is not a conductor")
    mi = c.net_names.index(name)
    if c.c_ratio is not None:
        kw.setdefault("c_ratio", c.c_ratio)
    p = job_params(s, mi, **kw)
    t0 = time.time()
    r = engine.extract(s, p, ctx)
    secs = time.time() - t0
    names = c.net_names + ["WINDOW"]
    row = {name: float(r.cap[mi]) * 1e-15}
    for j, nm in enumerate(names):
        if j != mi:
            row[nm] = -float(r.cap[j]) * 1e-15
    return {"master": name, "row_F": row, "cap_fF": [float(v) for v in r.cap[:len(names)]],
            "stderr_fF": [float(v) for v in r.stderr[:len(names)]], "walks": int(r.walks),
            "hops": int(r.hops), "converged": bool(r.converged), "seconds": secs,
            "gauss_offset_um": p.gauss_offset, "stop_dist_um": p.stop_dist,
            "gauss_surface": int(p.gauss_surface), "lost": int(r.lost)}


def write_dspf(results, path) -> None:
    """One ``*|NET master total`` line and ``C<k> master other value`` lines
    (F) per master."""
    lines = []
    k = 0
    for res in results:
        m, row = res["master"], res["row_F"]
        lines.append(f"*|NET {m} {row[m]:.7e}")
        for nm, v in row.items():
            if nm != m:
                lines.append(f"C{k} {m} {nm} {v:.7e}")
                k += 1
    Path(path).write_text("\n".join(lines) + "\n")


# -------------------------------------------------- reference result files
def parse_cap_unit(s: str) -> float:
    s = s.strip()
    if s.endswith("pF"):
        return float(s[:-2]) * 1e-12
    if s.endswith("fF"):
        return float(s[:-2]) * 1e-15
    return float(s)


def _add_coupling(capmat: dict, a: str, b: str, v: float) -> None:
    """Coupling a-b: ground may be written "0"; a pair listed twice keeps the
    mean; the row of b (when b is a master) gets the same value. A first
    net with no total line starts a row here (the reference reader stops on
    a KeyError there)."""
    if b == "0":
        b = "GROUND"
    if a in capmat and b in capmat[a]:
        v = (capmat[a][b] + v) / 2  # a pair listed twice: the mean
    capmat.setdefault(a, {})[b] = v
    if b in capmat:
        capmat[b][a] = v


def parse_dspf(text: str) -> dict:
    """{master: {master: total, other: coupling}} from DSPF text."""
    lines = text.splitlines()
    capmat: dict = {}
    for line in lines:
        if line.startswith("*|NET "):
            t = line.split(" ")
            capmat[t[1]] = {t[1]: float(t[2])}
    for line in lines:
        if line.startswith("C"):
            t = line.split(" ")
            _add_coupling(capmat, t[1], t[2], float(t[3]))
    return capmat


def parse_spice(text: str) -> dict:
    """Same from QuickCap's SPICE listing (``** NET total (total)`` and
    ``Cp<k> a b value`` lines, values with fF / pF units)."""
    lines = text.splitlines()
    capmat: dict = {}
    for line in lines:
        if line.startswith("** ") and "(total)" in line:
            t = line.split(" ")
            capmat[t[1]] = {t[1]: parse_cap_unit(t[2])}
    for line in lines:
        if line.startswith("Cp"):
            t = line.split(" ")
            _add_coupling(capmat, t[1], t[2], parse_cap_unit(t[3]))
    return capmat


def parse_result(path) -> dict:
    text = Path(path).read_text()
    return parse_spice(text) if str(path).endswith(".spice") else parse_dspf(text)


def compute_error(mat: dict, ref: dict):
    """(summed |cap - ref| over summed |ref| across every reference entry of
    every master present in ``mat``, {master: |self / ref self - 1|})."""
    abserr = abssum = 0.0
    self_err = {}
    for m, row in ref.items():
        if m not in mat or m not in mat[m]:
            continue
        self_err[m] = abs(mat[m][m] / row[m] - 1)
        for nm, rv in row.items():
            abserr += abs(mat[m].get(nm, 0.0) - rv)
            abssum += abs(rv)
    return (0.0 if abssum == 0 else abserr / abssum), self_err


def main() -> None:
    ap = argparse.ArgumentParser(description="extract a cap3d case with the FRW engine")
    ap.add_argument("case")
    ap.add_argument("--ref", default=None)
    ap.add_argument("--N", type=int, default=16)
    ap.add_argument("-p", type=float, default=0.01)
    ap.add_argument("-c", type=float, default=0.01)
    ap.add_argument("--c-ratio", type=float, default=None)
    ap.add_argument("--offset", type=float, default=None, help="Gaussian-surface offset (um)")
    ap.add_argument("--max-walks", type=float, default=1e7)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    c = parse(Path(a.case))
    kw = dict(N=a.N, p_tol=a.p, c_tol=a.c, offset=a.offset, max_walks=int(a.max_walks))
    if a.c_ratio is not None:
        kw["c_ratio"] = a.c_ratio
    res = [extract(c, m, **kw) for m in (c.masters or c.net_names[:1])]
    out = {"case": Path(a.case).name, "conductors": len(c.conductors), "nets": len(c.net_names),
           "boxes": sum(len(b) for _, b in c.conductors),
           "media_blocks": sum(len(b) for _, _, b in c.media), "plates": len(c.plates),
           "results": res}
    if a.out:
        write_dspf(res, a.out)
    if a.ref:
        err, self_err = compute_error({r["master"]: r["row_F"] for r in res}, parse_result(a.ref))
        out["error"] = err
        out["selfcap_error"] = self_err
    print(json.dumps(out))


if __name__ == "__main__":
    main()
