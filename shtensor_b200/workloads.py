"""Seeded synthetic block-sparse workloads (the reference ships no data sets).

Each workload is a contraction ``expr`` over tensors given as :class:`HostBlockSparse` in
the reference's storage layout (blocks sorted by column-major rolled id, each block dense
and column-major, packed in id order -- src/Tensor/BaseTensor.cpp:117-251).

* ``c0``  C[i,j,k] = sum_l A[i,j,l] B[l,k]; each mode 20 blocks with sizes uniform in
          [5,15]; blocks present independently with p=0.3; values uniform in [-1,1].
* ``c1``  C[i,j,a,b] = sum_P A[i,a,P] B[j,b,P]; i,j extent 64 in blocks from {5,9,13};
          a,b extent 512 in blocks from {13,25,32}; P extent 2048 in blocks from {32,48,64}
          (sizes are drawn until the extent is reached, so an extent can overshoot by less
          than one block); occupancy 15%; values N(0,1) times a per-block factor
          exp(-|blk_x - blk_P'|/4), with x = a for A and b for B and P' the P block index
          rescaled to the a/b block range.
* ``c2``  c1 shapes with per-block magnitudes 10^U(-6,2).
* ``c3``  C[a,b,i,j] = sum_{c,d} V[a,b,c,d] T[c,d,i,j]; a..d blocks of 24-48, i,j blocks of
          8-16; V stores a block when exp(-0.5*spread(a,b,c,d)) >= v_keep (spread = max-min
          of the four block indices), T when exp(-0.5*(|c-d|+|i-j|)) >= t_keep; values
          N(0,1) times the block's decay factor.  ``scale`` shrinks the extents (the full
          768-extent V would need terabytes).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class HostBlockSparse:
    block_sizes: list
    ids: np.ndarray
    offsets: np.ndarray
    data: np.ndarray
    rows: np.ndarray | None = None

    @property
    def order(self):
        return len(self.block_sizes)

    @property
    def nnz(self):
        return int(self.data.size)

    def index_lists(self):
        """Per-mode block-index lists (VArray<N>) of the stored blocks."""
        nblk = [len(b) for b in self.block_sizes]
        gstride = np.concatenate([[1], np.cumprod(nblk)[:-1]]).astype(np.int64)
        return [((self.ids // gstride[d]) % nblk[d]).astype(np.int32) for d in range(self.order)]

    def block_dims(self):
        idx = self.index_lists()
        return np.stack([np.asarray(self.block_sizes[d], np.int64)[idx[d]] for d in range(self.order)], axis=1) \
            if len(self.ids) else np.zeros((0, self.order), np.int64)


@dataclass
class Workload:
    name: str
    expr: str
    A: HostBlockSparse
    B: HostBlockSparse
    C: HostBlockSparse
    alpha: float = 1.0
    beta: float = 0.0
    screen_eps: float = 0.0
    meta: dict = field(default_factory=dict)


def split_extent(rng, extent: int, choices=None, lo=None, hi=None):
    sizes = []
    total = 0
    while total < extent:
        s = int(rng.choice(choices)) if choices is not None else int(rng.integers(lo, hi + 1))
        sizes.append(s)
        total += s
    return sizes


def build_tensor(rng, block_sizes, keep_mask_fn, scale_fn, dist: str) -> HostBlockSparse:
    nblk = [len(b) for b in block_sizes]
    total = int(np.prod(nblk))
    ids = np.arange(total, dtype=np.int64)
    gstride = np.concatenate([[1], np.cumprod(nblk)[:-1]]).astype(np.int64)
    coords = [(ids // gstride[d]) % nblk[d] for d in range(len(nblk))]
    keep = keep_mask_fn(coords)
    ids = ids[keep]
    coords = [c[keep] for c in coords]
    sizes = np.ones(len(ids), np.int64)
    for d in range(len(nblk)):
        sizes *= np.asarray(block_sizes[d], np.int64)[coords[d]]
    offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64) if len(ids) else np.zeros(0, np.int64)
    nnz = int(sizes.sum())
    if dist == "uniform":
        vals = rng.uniform(-1.0, 1.0, nnz)
    else:
        vals = rng.standard_normal(nnz)
    scales = scale_fn(coords) if scale_fn is not None else None
    if scales is not None and nnz:
        vals *= np.repeat(np.asarray(scales, np.float64), sizes)
    return HostBlockSparse([list(map(int, b)) for b in block_sizes], ids, offsets, vals)


def empty_tensor(block_sizes) -> HostBlockSparse:
    return HostBlockSparse([list(map(int, b)) for b in block_sizes], np.zeros(0, np.int64), np.zeros(0, np.int64),
                           np.zeros(0, np.float64))


def c0(seed: int = 1, nblocks: int = 20, p: float = 0.3) -> Workload:
    rng = np.random.default_rng(seed)
    i, j, l, k = (list(map(int, rng.integers(5, 16, nblocks))) for _ in range(4))
    A = build_tensor(rng, [i, j, l], lambda c: rng.random(len(c[0])) < p, None, "uniform")
    B = build_tensor(rng, [l, k], lambda c: rng.random(len(c[0])) < p, None, "uniform")
    return Workload("c0", "ijl, lk -> ijk", A, B, empty_tensor([i, j, k]),
                    meta={"extent": "~200 per mode", "blocks_per_mode": nblocks, "occupancy": p})


def _c1_shapes(rng, scale: float = 1.0):
    i = split_extent(rng, int(64 * scale), choices=[5, 9, 13])
    j = split_extent(rng, int(64 * scale), choices=[5, 9, 13])
    a = split_extent(rng, int(512 * scale), choices=[13, 25, 32])
    b = split_extent(rng, int(512 * scale), choices=[13, 25, 32])
    P = split_extent(rng, int(2048 * scale), choices=[32, 48, 64])
    return i, j, a, b, P


def c1(seed: int = 1, scale: float = 1.0, occupancy: float = 0.15, magnitudes: str = "decay") -> Workload:
    rng = np.random.default_rng(seed)
    i, j, a, b, P = _c1_shapes(rng, scale)
    na, nb, nP = len(a), len(b), len(P)

    def decay(nx):
        return lambda c: np.exp(-np.abs(c[1] - np.rint(c[2] * (nx - 1) / max(nP - 1, 1))) / 4.0)

    def mags(c):
        return 10.0 ** rng.uniform(-6.0, 2.0, len(c[0]))

    fA = decay(na) if magnitudes == "decay" else mags
    fB = decay(nb) if magnitudes == "decay" else mags
    A = build_tensor(rng, [i, a, P], lambda c: rng.random(len(c[0])) < occupancy, fA, "normal")
    B = build_tensor(rng, [j, b, P], lambda c: rng.random(len(c[0])) < occupancy, fB, "normal")
    return Workload("c1" if magnitudes == "decay" else "c2", "iaP, jbP -> ijab", A, B, empty_tensor([i, j, a, b]),
                    meta={"scale": scale, "occupancy": occupancy, "magnitudes": magnitudes})


def c2(seed: int = 1, scale: float = 1.0, occupancy: float = 0.15) -> Workload:
    return c1(seed, scale, occupancy, magnitudes="mixed")


def c3(seed: int = 1, scale: float = 0.125, v_keep: float = 0.1, t_keep: float = 1e-10,
       screen_eps: float = 1e-10) -> Workload:
    rng = np.random.default_rng(seed)
    big = [split_extent(rng, int(768 * scale), lo=24, hi=48) for _ in range(4)]
    small = [split_extent(rng, max(int(96 * scale), 8), lo=8, hi=16) for _ in range(2)]
    a, b, c, d = big
    i, j = small

    def v_spread(cc):
        st = np.stack(cc[:4])
        return st.max(0) - st.min(0)

    V = build_tensor(rng, [a, b, c, d], lambda cc: np.exp(-0.5 * v_spread(cc)) >= v_keep,
                     lambda cc: np.exp(-0.5 * v_spread(cc)), "normal")

    def t_delta(cc):
        return np.abs(cc[0] - cc[1]) + np.abs(cc[2] - cc[3])

    T = build_tensor(rng, [c, d, i, j], lambda cc: np.exp(-0.5 * t_delta(cc)) >= t_keep,
                     lambda cc: np.exp(-0.5 * t_delta(cc)), "normal")
    return Workload("c3", "abcd, cdij -> abij", V, T, empty_tensor([a, b, i, j]), screen_eps=screen_eps,
                    meta={"scale": scale, "v_keep": v_keep, "t_keep": t_keep})



def c4_request(rng, max_scale: float = 1.0) -> Workload:
    """One request of the serving mix: a family drawn from c0..c3, its extents scaled by
    U(0.25, 1) (times ``max_scale``) and, for c0..c2, occupancy drawn from U(0.05, 0.4).
    c3 keeps its own decay-and-screening sparsity at its default scale times the draw."""
    fam = int(rng.integers(0, 4))
    u = float(rng.uniform(0.25, 1.0)) * max_scale
    occ = float(rng.uniform(0.05, 0.4))
    seed = int(rng.integers(1, 1 << 30))
    if fam == 0:
        w = c0(seed=seed, nblocks=max(2, int(round(20 * u))), p=occ)
    elif fam == 1:
        w = c1(seed=seed, scale=u, occupancy=occ)
    elif fam == 2:
        w = c2(seed=seed, scale=u, occupancy=occ)
    else:
        w = c3(seed=seed, scale=0.125 * u)
    w.meta.update({"family": w.name, "u": u, "occupancy": occ})
    return w
