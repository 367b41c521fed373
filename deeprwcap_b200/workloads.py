"""Seeded synthetic inputs for the FRW transition engine.

The reference publishes no benchmark inputs for this path; these generators
produce inputs with the shapes, sizes and value distributions of the
workloads the engine is measured on:

* ``fdm_cubes``: transition cubes of resolution N with 1-4 horizontal
  dielectric layers (uniform random z cuts, eps ~ U[2,8]) and 0-2 random
  axis-aligned dielectric boxes (eps ~ U[2,8]); optionally per-voxel noise
  (a quarter of the voxels replaced by eps log-uniform in [1,12]).
  Cubes are described in the dnnsolver's cube-normalised [-1,1] layer/cuboid
  form (dnn_solver.cpp:165-250) and voxelised at cell centres (2i+1)/N - 1
  with the fill rule of cuda_kernels.cu:39-83 (last layer with min_z <= z,
  first containing cuboid overrides), in FP64.
* ``mixed_fdm_batch``: uneven-N batch (N drawn from {16, 21, 23}), 10% of the
  cubes with voxel noise.
* ``two_layer_crossing``: 8 conductors in two orthogonal metal layers of 4
  wires (w = s = t = 0.1 um, L = 2 um, 0.2 um vertical gap), a 3-layer
  stratified dielectric (3.9 / 2.7 / 4.2, boundaries at the wire-layer
  mid-planes) in a grounded box with a 1 um margin.
* ``wire_stack``: generalised wire stacks (2-4 layers, 4-16 wires per layer,
  optional random dielectric blocks) for the denser and serving workloads.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from .abi import (MAX_CUBOIDS, MAX_LAYERS, PADDING, Box, DielBox, JobParams, Structure,
                  default_job_params)


# --------------------------------------------------------------------------- cubes
def random_cube_structure(rng: np.random.Generator):
    """One cube's layers [(min_z, eps)] (sorted) and boxes [(x0,y0,z0,x1,y1,z1,eps)]."""
    nl = int(rng.integers(1, 5))
    cuts = np.sort(rng.uniform(-1.0, 1.0, nl - 1))
    zlo = np.concatenate([[-1.0], cuts])
    layers = [(float(z), float(rng.uniform(2.0, 8.0))) for z in zlo]
    nb = int(rng.integers(0, 3))
    boxes = []
    for _ in range(nb):
        a = rng.uniform(-1.0, 1.0, 3)
        b = rng.uniform(-1.0, 1.0, 3)
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        boxes.append((*map(float, lo), *map(float, hi), float(rng.uniform(2.0, 8.0))))
    return layers, boxes


def voxelise_f64(layers, boxes, N: int) -> np.ndarray:
    """eps[k, j, i] at cell centres (2i+1)/N - 1 (FP64)."""
    c = (2.0 * np.arange(N) + 1.0) / N - 1.0
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    zlo = np.array([l[0] for l in layers])
    val = np.array([l[1] for l in layers])
    li = np.zeros(Z.shape, dtype=np.int64)
    for idx in range(len(layers)):
        li = np.where(Z >= zlo[idx], idx, li)
    eps = val[li]
    done = np.zeros(Z.shape, dtype=bool)
    for b in boxes:
        inside = ((X >= b[0]) & (X <= b[3]) & (Y >= b[1]) & (Y <= b[4]) & (Z >= b[2]) &
                  (Z <= b[5]) & ~done)
        eps = np.where(inside, b[6], eps)
        done |= inside
    return np.ascontiguousarray(eps)


def to_query_arrays(layers, boxes):
    """Padded float32 (30,), (105,) arrays in the dnnsolver query layout."""
    lay = np.full((MAX_LAYERS, 2), PADDING, dtype=np.float32)
    cub = np.full((MAX_CUBOIDS, 7), PADDING, dtype=np.float32)
    for i, l in enumerate(layers[:MAX_LAYERS]):
        lay[i] = l
    for i, b in enumerate(boxes[:MAX_CUBOIDS]):
        cub[i] = b
    return lay.reshape(-1), cub.reshape(-1)


def add_voxel_noise(eps: np.ndarray, rng: np.random.Generator, frac: float = 0.25):
    mask = rng.uniform(size=eps.shape) < frac
    noise = np.exp(rng.uniform(np.log(1.0), np.log(12.0), size=eps.shape))
    return np.where(mask, noise, eps)


def fdm_cubes(n: int, N: int, seed: int = 0, noise_frac: float = 0.0):
    """n cubes of resolution N: eps [n, N, N, N] FP64 and the structure list."""
    rng = np.random.default_rng(seed)
    eps = np.empty((n, N, N, N))
    structs = []
    for c in range(n):
        layers, boxes = random_cube_structure(rng)
        e = voxelise_f64(layers, boxes, N)
        if noise_frac > 0 and rng.uniform() < noise_frac:
            e = add_voxel_noise(e, rng)
        eps[c] = e
        structs.append((layers, boxes))
    return eps, structs


def query_batch(n: int, seed: int = 0):
    """n dnnsolver queries (layers [n,30], cuboids [n,105] float32)."""
    rng = np.random.default_rng(seed)
    L = np.empty((n, 30), dtype=np.float32)
    Cb = np.empty((n, 105), dtype=np.float32)
    for q in range(n):
        layers, boxes = random_cube_structure(rng)
        L[q], Cb[q] = to_query_arrays(layers, boxes)
    return L, Cb


@dataclass
class MixedBatch:
    N: np.ndarray            # [ncubes] int32
    eps_off: np.ndarray      # [ncubes] int64 (elements)
    out_off: np.ndarray      # [ncubes] int64 (elements)
    eps: np.ndarray          # concatenated FP64 permittivity
    noisy: np.ndarray        # [ncubes] bool

    @property
    def ncubes(self) -> int:
        return int(self.N.size)

    def cube(self, c: int) -> np.ndarray:
        n = int(self.N[c])
        return self.eps[self.eps_off[c]:self.eps_off[c] + n ** 3].reshape(n, n, n)

    @property
    def out_size(self) -> int:
        return int(self.out_off[-1] + 6 * int(self.N[-1]) ** 2)

    @property
    def cells(self) -> int:
        return int(np.sum(self.N.astype(np.int64) ** 3))


def mixed_fdm_batch(n: int = 8192, Ns=(16, 21, 23), seed: int = 0,
                    noise_frac: float = 0.10) -> MixedBatch:
    rng = np.random.default_rng(seed)
    Nc = rng.choice(np.asarray(Ns, dtype=np.int32), size=n).astype(np.int32)
    sizes = Nc.astype(np.int64) ** 3
    eps_off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    out_off = np.concatenate([[0], np.cumsum(6 * Nc.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
    eps = np.empty(int(sizes.sum()))
    noisy = np.zeros(n, dtype=bool)
    # voxelise once per distinct structure; cubes are independent
    for c in range(n):
        N = int(Nc[c])
        layers, boxes = random_cube_structure(rng)
        e = voxelise_f64(layers, boxes, N)
        if rng.uniform() < noise_frac:
            e = add_voxel_noise(e, rng)
            noisy[c] = True
        eps[eps_off[c]:eps_off[c] + N ** 3] = e.reshape(-1)
    return MixedBatch(Nc, eps_off, out_off, eps, noisy)


# ---------------------------------------------------------------------- structures
@dataclass
class StructureSpec:
    """A 3-D interconnect structure: conductor boxes (with net ids), stratified
    dielectric layers, dielectric blocks and the grounded enclosure (um)."""
    boxes: np.ndarray          # [nb, 6] lo xyz, hi xyz
    nets: np.ndarray           # [nb] int32
    n_nets: int
    layer_zlo: np.ndarray      # [nl]
    layer_eps: np.ndarray      # [nl]
    diel: np.ndarray           # [nd, 7] lo xyz, hi xyz, eps
    encl_lo: np.ndarray
    encl_hi: np.ndarray
    name: str = ""
    _keep: list = field(default_factory=list, repr=False)

    def to_c(self) -> Structure:
        nb, nd, nl = len(self.boxes), len(self.diel), len(self.layer_zlo)
        bx = (Box * max(nb, 1))()
        for i in range(nb):
            bx[i].lo[:] = list(self.boxes[i, :3])
            bx[i].hi[:] = list(self.boxes[i, 3:])
            bx[i].net = int(self.nets[i])
        db = (DielBox * max(nd, 1))()
        for i in range(nd):
            db[i].lo[:] = list(self.diel[i, :3])
            db[i].hi[:] = list(self.diel[i, 3:6])
            db[i].eps = float(self.diel[i, 6])
        zlo = (C.c_double * max(nl, 1))(*self.layer_zlo)
        le = (C.c_double * max(nl, 1))(*self.layer_eps)
        s = Structure()
        s.n_boxes, s.n_nets, s.n_layers, s.n_diel = nb, int(self.n_nets), nl, nd
        s.boxes = C.cast(bx, C.POINTER(Box))
        s.diel = C.cast(db, C.POINTER(DielBox))
        s.layer_zlo = C.cast(zlo, C.POINTER(C.c_double))
        s.layer_eps = C.cast(le, C.POINTER(C.c_double))
        s.encl_lo[:] = list(map(float, self.encl_lo))
        s.encl_hi[:] = list(map(float, self.encl_hi))
        s._keep = (bx, db, zlo, le)  # keep the buffers alive with the struct
        return s


def wire_stack(n_layers: int = 2, wires_per_layer: int = 4, width: float = 0.1,
               spacing: float = 0.1, thickness: float = 0.1, length: float = 2.0,
               gap: float = 0.2, margin: float = 1.0, diel_eps=None, n_diel_blocks: int = 0,
               seed: int = 0, name: str = "") -> StructureSpec:
    """Metal layers of parallel wires, alternating x/y direction, layer l at
    z in [l*(t+gap), l*(t+gap)+t]. Dielectric: len(diel_eps) stratified layers
    with boundaries at the wire-layer mid-planes (and, beyond the wire layers,
    evenly spaced), plus n_diel_blocks random dielectric blocks that avoid the
    conductors."""
    rng = np.random.default_rng(seed)
    pitch = width + spacing
    bundle = wires_per_layer * width + (wires_per_layer - 1) * spacing
    boxes, nets = [], []
    net = 0
    centre = length / 2.0
    for l in range(n_layers):
        z0 = l * (thickness + gap)
        for w in range(wires_per_layer):
            a0 = centre - bundle / 2.0 + w * pitch
            if l % 2 == 0:   # along x
                boxes.append([0.0, a0, z0, length, a0 + width, z0 + thickness])
            else:            # along y
                boxes.append([a0, 0.0, z0, a0 + width, length, z0 + thickness])
            nets.append(net)
            net += 1
    boxes = np.array(boxes, dtype=np.float64)
    lo = boxes[:, :3].min(axis=0)
    hi = boxes[:, 3:].max(axis=0)
    if diel_eps is None:
        diel_eps = [3.9, 2.7, 4.2]
    nd = len(diel_eps)
    mids = [l * (thickness + gap) + thickness / 2.0 for l in range(n_layers)]
    zb = list(mids[:nd - 1])
    while len(zb) < nd - 1:  # more dielectric layers than wire layers: spread above
        top = hi[2] + margin
        k = len(zb) - (n_layers - 1)
        zb.append(mids[-1] + (top - mids[-1]) * (k + 1) / (nd - n_layers + 1))
    layer_zlo = np.array([lo[2] - margin] + zb, dtype=np.float64)
    layer_eps = np.array(diel_eps, dtype=np.float64)
    diel = []
    tries = 0
    while len(diel) < n_diel_blocks and tries < 10000:
        tries += 1
        size = rng.uniform(0.05, 0.4, 3)
        c = rng.uniform(lo - 0.3, hi + 0.3)
        b = np.concatenate([c - size / 2, c + size / 2])
        clear = True
        for cb in boxes:  # keep a 0.02 um clearance from every conductor
            if np.all(b[:3] < cb[3:] + 0.02) and np.all(b[3:] > cb[:3] - 0.02):
                clear = False
                break
        if clear:
            diel.append(list(b) + [float(rng.uniform(2.5, 4.5))])
    diel = np.array(diel, dtype=np.float64).reshape(-1, 7)
    return StructureSpec(boxes, np.array(nets, dtype=np.int32), net, layer_zlo, layer_eps,
                         diel, lo - margin, hi + margin, name=name)


def two_layer_crossing() -> StructureSpec:
    """8 conductors: two orthogonal layers of 4 wires (w=s=t=0.1, L=2.0 um),
    layer 2 0.2 um above layer 1; dielectric 3.9/2.7/4.2 split at the wire
    mid-planes; grounded box with 1.0 um margin. Master = wire 0."""
    return wire_stack(2, 4, name="two_layer_crossing")


def dense_stack(seed: int = 0) -> StructureSpec:
    """24 conductors: 3 orthogonal-alternating layers of 8 wires, 5 stratified
    dielectric layers (eps ~ U[2.5, 4.5]) and 10 random dielectric blocks."""
    rng = np.random.default_rng(seed)
    eps = list(rng.uniform(2.5, 4.5, 5))
    return wire_stack(3, 8, diel_eps=eps, n_diel_blocks=10, seed=seed, name="dense_stack")


def job_params(N: int = 16, master: int = 0, seed: int = 1, p_tol: float = 0.01,
               c_tol: float = 0.01, c_ratio: float = 0.95, gauss_offset: float = 0.05,
               stop_dist: float = 1e-5, max_walks: int = 1 << 26,
               batch_walks: int = 1 << 16) -> JobParams:
    p = default_job_params()
    p.master, p.N, p.seed = master, N, seed
    p.p_tol, p.c_tol, p.c_ratio = p_tol, c_tol, c_ratio
    p.gauss_offset, p.stop_dist = gauss_offset, stop_dist
    p.max_walks, p.batch_walks = max_walks, batch_walks
    return p


def job_params_plain(N: int = 16, master: int = 0, seed: int = 1, **kw) -> JobParams:
    """JobParams without loading the CUDA library (for CPU-only callers)."""
    p = JobParams()
    p.master, p.N, p.seed = master, N, seed
    p.gauss_offset = kw.get("gauss_offset", 0.05)
    p.stop_dist = kw.get("stop_dist", 1e-5)
    p.p_tol = kw.get("p_tol", 0.01)
    p.c_tol = kw.get("c_tol", 0.01)
    p.c_ratio = kw.get("c_ratio", 0.95)
    p.min_walks = kw.get("min_walks", 4096)
    p.max_walks = kw.get("max_walks", 1 << 26)
    p.batch_walks = kw.get("batch_walks", 1 << 16)
    p.max_hops = kw.get("max_hops", 10000)
    p.gauss_surface = kw.get("gauss_surface", 0)
    p.fdm.tol = kw.get("tol", 1e-10)
    p.fdm.inner_tol = kw.get("inner_tol", 1e-5)
    p.fdm.max_outer = kw.get("max_outer", 8)
    p.fdm.max_inner = kw.get("max_inner", 0)
    p.fdm.warm_start = kw.get("warm_start", 1)
    p.fdm.extra_outer = kw.get("extra_outer", 8)
    return p


# ---------------------------------------------------------------------- serving
@dataclass
class ServeJob:
    """One request of a serving stream: arrival time (s after the stream
    starts), structure, cube resolution, walk count and seed."""
    arrival: float
    structure: StructureSpec
    N: int
    walks: int
    seed: int


def serving_stream(n_jobs: int = 16, rate: float = 50.0, seed: int = 0,
                   walks=(1e5, 1e7), Ns=(16, 21, 23)) -> list:
    """Poisson arrivals (mean `rate` jobs/s) of extraction jobs: 2-4 metal
    layers of 4-16 wires (8-64 conductors), the dielectric of the
    two-layer crossing (3 stratified layers) or of the dense stack (5 layers,
    eps ~ U[2.5, 4.5], 10 blocks), N drawn from Ns, walks log-uniform in
    `walks`. Everything is seeded."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_jobs):
        t += float(rng.exponential(1.0 / rate))
        nl = int(rng.integers(2, 5))
        nw = int(rng.integers(4, 17))
        if rng.random() < 0.5:
            eps, blocks = [3.9, 2.7, 4.2], 0
        else:
            eps, blocks = list(rng.uniform(2.5, 4.5, 5)), 10
        s = wire_stack(nl, nw, diel_eps=eps, n_diel_blocks=blocks, seed=seed * 1000 + i,
                       name=f"stack{nl}x{nw}")
        N = int(Ns[int(rng.integers(0, len(Ns)))])
        lo, hi = np.log(walks[0]), np.log(walks[1])
        nwalks = int(np.exp(rng.uniform(lo, hi)))
        out.append(ServeJob(t, s, N, nwalks, seed * 1000 + i + 1))
    return out


def serve_params(job: ServeJob, batch: int = 1 << 16, **kw) -> JobParams:
    """A fixed-size job: exactly job.walks walks (master = wire 0)."""
    return job_params_plain(N=job.N, seed=job.seed, min_walks=job.walks, max_walks=job.walks,
                            batch_walks=min(batch, job.walks), **kw)
