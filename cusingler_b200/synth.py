"""Seeded synthetic single-cell CSR data with the shapes of the benchmark workloads.

There is no public dataset in this environment, so every workload is generated:

* per gene a mean ``mu_g ~ logUniform(0.5, 20)``;
* counts ``x ~ NegBin(mean = mu_g * marker_factor, dispersion 0.3)`` (a Gamma-Poisson mixture);
* a logistic, mean-dependent dropout (a Splatter-style detection curve)
  ``P(detected) = 1 / (1 + exp(-k (ln mean - x0)))`` with ``x0`` solved so that the stored fraction
  hits the target density; highly expressed genes and raised marker genes are detected in most
  cells, which is what gives per-label medians (and so marker genes) their signal;
* stored value ``log2(1 + x)`` as float32, CSR rows with ascending column indices and no explicit
  zeros;
* label proportions ``~ Dirichlet(1)`` floored at ``1/(4L)``; each label has a marker block of genes whose mean is
  multiplied by a factor.  Family configurations give every label of a family a shared block plus a
  few label-specific genes with a small factor, so labels inside a family are near-identical.

Seeds: the "world" (gene means, marker blocks, label proportions) and the reference cells use
``seed``; the query uses ``seed + 1``; the MLP training set uses ``seed + 2``.  Generation is split
into fixed row chunks, each with its own child seed, so the output does not depend on how many
worker processes are used.
"""

from __future__ import annotations

import dataclasses
import os
from concurrent.futures import ProcessPoolExecutor
import multiprocessing as mp

import numpy as np

DISPERSION = 0.3
DROPOUT_SLOPE = 3.0
_CHUNK_ROWS = 4096


@dataclasses.dataclass
class Workload:
    name: str
    n_ref: int
    n_qry: int
    n_genes: int
    n_labels: int
    density: float
    # per-label marker block: (min genes, max genes, min factor, max factor)
    block: tuple
    # families: (n_families, labels per family, (min, max) private genes, private factor)
    families: tuple | None = None


WORKLOADS = {
    # 1,900 ref x 800 query x 15,000 genes, 13 labels, ~10 % nonzero, 60-gene 4x marker blocks.
    "small": Workload("small", 1900, 800, 15000, 13, 0.10, (60, 60, 4.0, 4.0)),
    # 20,000 ref x 100,000 query x 25,000 genes, 30 labels, ~6 %, 40-80 gene 3-5x blocks.
    "mid": Workload("mid", 20000, 100000, 25000, 30, 0.06, (40, 80, 3.0, 5.0)),
    # 50,000 ref x 500,000 query, 60 labels in 12 families of 5 (8-15 private genes at 1.5x).
    "stress": Workload("stress", 50000, 500000, 25000, 60, 0.06, (40, 80, 3.0, 5.0),
                       families=(12, 5, (8, 15), 1.5)),
    # 100,000 ref x 2,000,000 query x 30,000 genes, 120 labels in 20 families of 6, ~5 %.
    "full": Workload("full", 100000, 2000000, 30000, 120, 0.05, (40, 80, 3.0, 5.0),
                     families=(20, 6, (8, 15), 1.5)),
}


@dataclasses.dataclass
class World:
    mu: np.ndarray            # (W,) float64 gene means
    props: np.ndarray         # (L,) label proportions
    factor: np.ndarray        # (L, W) float32 multiplicative marker factors
    x0: float                 # dropout midpoint (log mean)


@dataclasses.dataclass
class CSR:
    n_rows: int
    n_cols: int
    data: np.ndarray          # float32
    indices: np.ndarray       # int32
    indptr: np.ndarray        # int32 (int64 if nnz >= 2**31)
    labels: np.ndarray        # int32 true label per row

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    def rows(self, start: int, stop: int) -> "CSR":
        a, b = int(self.indptr[start]), int(self.indptr[stop])
        return CSR(stop - start, self.n_cols, self.data[a:b], self.indices[a:b],
                   (self.indptr[start:stop + 1] - a).astype(self.indptr.dtype),
                   self.labels[start:stop])

    def take(self, rows) -> "CSR":
        """The given rows (any order, repeats allowed) as a new CSR."""
        rows = np.asarray(rows, dtype=np.int64)
        lens = (self.indptr[rows + 1] - self.indptr[rows]).astype(np.int64)
        indptr = np.zeros(rows.shape[0] + 1, dtype=np.int64)
        np.cumsum(lens, out=indptr[1:])
        src = np.repeat(self.indptr[rows].astype(np.int64) - indptr[:-1], lens) + np.arange(indptr[-1])
        idt = np.int32 if indptr[-1] < 2**31 else np.int64
        return CSR(rows.shape[0], self.n_cols, self.data[src], self.indices[src], indptr.astype(idt),
                   self.labels[rows])


def make_world(wl: Workload, seed: int = 0) -> World:
    rng = np.random.default_rng([seed, 7919])
    W, L = wl.n_genes, wl.n_labels
    mu = np.exp(rng.uniform(np.log(0.5), np.log(20.0), size=W))
    # Dirichlet(1) proportions, floored at 1/(4L) so that every label has reference cells (the
    # reference cannot handle a label without any)
    props = rng.dirichlet(np.ones(L))
    props = np.maximum(props, 0.25 / L)
    props = props / props.sum()
    factor = np.ones((L, W), dtype=np.float32)
    perm = rng.permutation(W)
    pos = 0
    gmin, gmax, fmin, fmax = wl.block
    if wl.families is None:
        for lab in range(L):
            m = int(rng.integers(gmin, gmax + 1))
            genes = perm[pos:pos + m]
            pos += m
            factor[lab, genes] = rng.uniform(fmin, fmax)
    else:
        n_fam, per_fam, (pmin, pmax), pfac = wl.families
        assert n_fam * per_fam == L
        for fam in range(n_fam):
            m = int(rng.integers(gmin, gmax + 1))
            block = perm[pos:pos + m]
            pos += m
            f = rng.uniform(fmin, fmax)
            for j in range(per_fam):
                lab = fam * per_fam + j
                factor[lab, block] = f
                p = int(rng.integers(pmin, pmax + 1))
                private = perm[pos:pos + p]
                pos += p
                factor[lab, private] = pfac
    x0 = _solve_midpoint(mu, props, factor, wl.density)
    return World(mu, props, factor, x0)


def _detect(mean, x0):
    return 1.0 / (1.0 + np.exp(-DROPOUT_SLOPE * (np.log(mean) - x0)))


def _p_pos(mean):
    r = 1.0 / DISPERSION
    return 1.0 - (r / (r + mean)) ** r


def _solve_midpoint(mu, props, factor, density):
    """Bisection for x0 so that E[stored fraction] = density over the label mix."""
    mean = mu[None, :] * factor.astype(np.float64)
    pp = _p_pos(mean)
    lo, hi = -10.0, 15.0
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        d = float((props[:, None] * _detect(mean, mid) * pp).sum(0).mean())
        if d > density:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def _bucket_genes(pmax):
    """Group genes by their largest detection probability (buckets of ratio 0.7)."""
    edges = [1.0]
    while edges[-1] > 1e-5:
        edges.append(edges[-1] * 0.7)
    b = np.searchsorted(-np.asarray(edges), -pmax, side="left") - 1
    b = np.clip(b, 0, len(edges) - 1)
    return [(edges[i], np.nonzero(b == i)[0]) for i in range(len(edges)) if np.any(b == i)]


def _gen_chunk(args):
    (child_seed, n_rows, W, mu, props, factor, x0) = args
    rng = np.random.default_rng(child_seed)
    labels = rng.choice(props.shape[0], size=n_rows, p=props).astype(np.int32)
    mean_lg = mu[None, :] * factor.astype(np.float64)
    P = _detect(mean_lg, x0)                       # (L, W) detection probability
    rows_all, cols_all = [], []
    # Candidates per gene bucket at the bucket's top rate, then thinned to each entry's own rate.
    for pm, genes in _bucket_genes(P.max(0)):
        total = n_rows * genes.shape[0]
        expect = total * pm
        n_draw = int(expect + 6.0 * np.sqrt(expect) + 64)
        flat = np.cumsum(rng.geometric(pm, size=n_draw).astype(np.int64)) - 1
        while flat[-1] < total:
            more = rng.geometric(pm, size=n_draw).astype(np.int64)
            flat = np.concatenate([flat, flat[-1] + np.cumsum(more)])
        flat = flat[flat < total]
        row = flat // genes.shape[0]
        col = genes[flat % genes.shape[0]]
        keep = rng.random(row.shape[0]) < P[labels[row], col] / pm
        rows_all.append(row[keep])
        cols_all.append(col[keep].astype(np.int32))
    row = np.concatenate(rows_all)
    col = np.concatenate(cols_all)
    order = np.lexsort((col, row))
    row, col = row[order], col[order]
    mean = mean_lg[labels[row], col]
    r = 1.0 / DISPERSION
    lam = rng.gamma(shape=r, scale=mean / r)
    x = rng.poisson(lam)
    nz = x > 0
    row, col, x = row[nz], col[nz], x[nz]
    data = np.log2(1.0 + x).astype(np.float32)
    counts = np.bincount(row, minlength=n_rows)
    indptr = np.zeros(n_rows + 1, dtype=np.int64)
    np.cumsum(counts, out=indptr[1:])
    return data, col, indptr, labels


def generate(world: World, n_rows: int, seed: int, workers: int | None = None) -> CSR:
    """Generate ``n_rows`` cells.  Deterministic in (world, n_rows, seed)."""
    W = world.factor.shape[1]
    n_chunks = max(1, (n_rows + _CHUNK_ROWS - 1) // _CHUNK_ROWS)
    children = np.random.SeedSequence([seed, 104729]).spawn(n_chunks)
    jobs = []
    for c in range(n_chunks):
        rows = min(_CHUNK_ROWS, n_rows - c * _CHUNK_ROWS)
        jobs.append((children[c], rows, W, world.mu, world.props, world.factor, world.x0))
    if workers is None:
        workers = min(len(jobs), os.cpu_count() or 1, 32)
    if workers > 1 and len(jobs) > 1:
        # spawn, never fork: callers may already hold a CUDA context
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            parts = list(ex.map(_gen_chunk, jobs))
    else:
        parts = [_gen_chunk(j) for j in jobs]
    nnz = sum(int(p[2][-1]) for p in parts)
    idt = np.int32 if nnz < 2**31 else np.int64
    data = np.empty(nnz, dtype=np.float32)
    indices = np.empty(nnz, dtype=np.int32)
    indptr = np.empty(n_rows + 1, dtype=idt)
    labels = np.empty(n_rows, dtype=np.int32)
    off, r0 = 0, 0
    indptr[0] = 0
    for d, c, ip, lab in parts:
        n = d.shape[0]
        k = lab.shape[0]
        data[off:off + n] = d
        indices[off:off + n] = c
        indptr[r0 + 1:r0 + k + 1] = ip[1:] + off
        labels[r0:r0 + k] = lab
        off += n
        r0 += k
    return CSR(n_rows, W, data, indices, indptr, labels)


def make_dataset(name: str, n_ref: int | None = None, n_qry: int | None = None, seed: int = 0,
                 workers: int | None = None):
    """Return (world, ref CSR, query CSR) for a named workload, optionally with fewer cells."""
    wl = WORKLOADS[name]
    world = make_world(wl, seed)
    ref = generate(world, wl.n_ref if n_ref is None else n_ref, seed, workers)
    qry = generate(world, wl.n_qry if n_qry is None else n_qry, seed + 1, workers)
    return world, ref, qry


def custom_dataset(n_ref: int, n_qry: int, n_genes: int, n_labels: int, density: float,
                   block=(20, 40, 3.0, 5.0), families=None, seed: int = 0, workers: int = 1):
    """A small ad-hoc workload for tests."""
    wl = Workload("custom", n_ref, n_qry, n_genes, n_labels, density, block, families)
    world = make_world(wl, seed)
    ref = generate(world, n_ref, seed, workers)
    qry = generate(world, n_qry, seed + 1, workers)
    return world, ref, qry


def names(prefix: str, n: int) -> list[str]:
    return [f"{prefix}{i}" for i in range(n)]
