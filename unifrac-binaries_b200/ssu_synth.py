"""Seeded synthetic phylogenies and feature tables for the UniFrac engine.

Trees come out in the balanced-parentheses (BP) array form that the C API's
`support_bptree_t` carries (reference: src/api.hpp:163-168): `structure[i]`
is True for an opening parenthesis, and the name and branch length of a node
sit at its opening index, as BPTree stores them (src/tree.cpp:72-99,
src/tree.cpp:441-455).  Tables come out as the observation-major CSR of
`support_biom_t` (src/api.hpp:145-154): row `i` of `indptr` spans the
samples in which feature `i` is non-zero, `indices` holds sample positions.

Every generator takes an integer seed and is deterministic for it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class BPTree:
    structure: np.ndarray          # bool[n_parens]
    lengths: np.ndarray            # float64[n_parens]
    names: list                    # str[n_parens]

    @property
    def n_parens(self) -> int:
        return int(self.structure.shape[0])

    def tip_names(self):
        s = self.structure
        return [self.names[i] for i in range(len(s) - 1) if s[i] and not s[i + 1]]

    def tip_lengths(self):
        s = self.structure
        return [float(self.lengths[i]) for i in range(len(s) - 1) if s[i] and not s[i + 1]]


@dataclass
class Table:
    obs_ids: list
    sample_ids: list
    indptr: np.ndarray             # uint32[n_obs + 1]
    indices: np.ndarray            # uint32[nnz], sample positions
    data: np.ndarray               # float64[nnz]
    extra: dict = field(default_factory=dict)

    @property
    def n_obs(self) -> int:
        return len(self.obs_ids)

    @property
    def n_samples(self) -> int:
        return len(self.sample_ids)

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    @classmethod
    def from_dense(cls, dense, obs_ids, sample_ids) -> "Table":
        """Observation-major CSR of a dense features x samples array (non-zero
        entries kept)."""
        dense = np.asarray(dense, dtype=np.float64)
        rows, cols = np.nonzero(dense)
        indptr = np.zeros(dense.shape[0] + 1, dtype=np.uint32)
        np.add.at(indptr, rows + 1, 1)
        return cls(list(obs_ids), list(sample_ids), np.cumsum(indptr).astype(np.uint32),
                   cols.astype(np.uint32), dense[rows, cols].copy())

    def dense(self) -> np.ndarray:
        out = np.zeros((self.n_obs, self.n_samples), dtype=np.float64)
        for i in range(self.n_obs):
            a, b = int(self.indptr[i]), int(self.indptr[i + 1])
            out[i, self.indices[a:b]] = self.data[a:b]
        return out


# ---------------------------------------------------------------- trees

def tree_from_children(children, lengths, names, root) -> BPTree:
    """Serialise a rooted tree given as child lists into BP arrays (iterative)."""
    n_nodes = len(children)
    structure = np.zeros(2 * n_nodes, dtype=bool)
    bp_len = np.zeros(2 * n_nodes, dtype=np.float64)
    bp_names = [""] * (2 * n_nodes)
    pos = 0
    stack = [(root, False)]
    while stack:
        node, closing = stack.pop()
        if closing:
            structure[pos] = False
            pos += 1
            continue
        structure[pos] = True
        bp_len[pos] = lengths[node]
        bp_names[pos] = names[node]
        pos += 1
        stack.append((node, True))
        for c in reversed(children[node]):
            stack.append((c, False))
    assert pos == 2 * n_nodes
    return BPTree(structure, bp_len, bp_names)


def random_binary_tree(n_tips: int, mean_length: float, seed: int, tip_prefix: str = "T") -> BPTree:
    """Rooted binary tree by uniform random pair-joining of `n_tips` tips.

    Branch lengths are iid Exponential(mean_length); the root's length is 0.
    """
    rng = np.random.default_rng(seed)
    n_nodes = 2 * n_tips - 1
    children = [[] for _ in range(n_nodes)]
    active = list(range(n_tips))
    picks = rng.random((max(n_tips - 1, 0), 2))
    for step in range(n_tips - 1):
        m = len(active)
        i = int(picks[step, 0] * m)
        a = active[i]
        active[i] = active[-1]
        active.pop()
        m -= 1
        j = int(picks[step, 1] * m)
        b = active[j]
        parent = n_tips + step
        children[parent] = [a, b]
        active[j] = parent
    root = active[0]
    lengths = rng.exponential(mean_length, size=n_nodes)
    lengths[root] = 0.0
    names = [f"{tip_prefix}{i}" for i in range(n_tips)] + [""] * (n_nodes - n_tips)
    return tree_from_children(children, lengths, names, root)


def parse_newick(newick: str, float_lengths: bool = True) -> BPTree:
    """Newick -> BP arrays.  Lengths are rounded through float32 as the
    reference's `std::stof` does (src/tree.cpp:446,449) unless disabled."""
    s = newick.strip()
    if s.endswith(";"):
        s = s[:-1]
    children, lengths, names = [], [], []

    def new_node():
        children.append([])
        lengths.append(0.0)
        names.append("")
        return len(children) - 1

    root = new_node()
    stack = []
    cur = root
    i = 0
    n = len(s)

    def read_label(i):
        start = i
        if i < n and s[i] == "'":
            j = s.index("'", i + 1)
            i = j + 1
        while i < n and s[i] not in "(),;":
            i += 1
        return s[start:i], i

    while i < n:
        c = s[i]
        if c == "(":
            stack.append(cur)
            cur = new_node()
            children[stack[-1]].append(cur)
            i += 1
        elif c == ",":
            cur = new_node()
            children[stack[-1]].append(cur)
            i += 1
        elif c == ")":
            cur = stack.pop()
            i += 1
        elif c.isspace():
            i += 1
        else:
            label, i = read_label(i)
            label = label.strip()
            if ":" in label:
                k = label.rfind(":")
                name, ln = label[:k], float(label[k + 1:])
                if float_lengths:
                    ln = float(np.float32(ln))
            else:
                name, ln = label, 0.0
            names[cur] = name
            lengths[cur] = ln
    return tree_from_children(children, lengths, names, root)


# ---------------------------------------------------------------- tables

def _csr_from_flat(flat: np.ndarray, n_obs: int, n_samples: int, values: np.ndarray):
    obs = (flat // n_samples).astype(np.int64)
    samp = (flat % n_samples).astype(np.uint32)
    counts = np.bincount(obs, minlength=n_obs)
    indptr = np.zeros(n_obs + 1, dtype=np.uint32)
    np.cumsum(counts, out=indptr[1:])
    return indptr, samp, values.astype(np.float64)


def random_positions(n_obs: int, n_samples: int, density: float, rng) -> np.ndarray:
    """Sorted distinct flat indices (obs * n_samples + sample), each (obs,
    sample) cell present with probability `density`."""
    total = n_obs * n_samples
    target = rng.binomial(total, density)
    if density > 0.2:
        flat = np.flatnonzero(rng.random(total) < density)
        return flat
    flat = np.unique(rng.integers(0, total, size=int(target * 1.02) + 16, dtype=np.int64))
    if flat.shape[0] > target:
        keep = np.sort(rng.choice(flat.shape[0], size=target, replace=False))
        flat = flat[keep]
    return flat


def make_table(obs_ids, n_samples: int, flat: np.ndarray, values: np.ndarray, sample_prefix="S") -> Table:
    indptr, indices, data = _csr_from_flat(flat, len(obs_ids), n_samples, values)
    return Table(list(obs_ids), [f"{sample_prefix}{j}" for j in range(n_samples)], indptr, indices, data)


def geometric_table(obs_ids, n_samples, density, mean, seed) -> Table:
    rng = np.random.default_rng(seed)
    flat = random_positions(len(obs_ids), n_samples, density, rng)
    vals = rng.geometric(1.0 / mean, size=flat.shape[0]).astype(np.float64) + 1.0
    return make_table(obs_ids, n_samples, flat, vals)


def lognormal_table(obs_ids, n_samples, density, mu, sigma, seed) -> Table:
    rng = np.random.default_rng(seed)
    flat = random_positions(len(obs_ids), n_samples, density, rng)
    vals = np.round(rng.lognormal(mu, sigma, size=flat.shape[0])) + 1.0
    return make_table(obs_ids, n_samples, flat, vals)


def negbin_table(obs_ids, n_samples, density, mean, dispersion, seed) -> Table:
    """Counts ~ NegBinomial(mean, dispersion) drawn as Gamma-Poisson, floored at 1."""
    rng = np.random.default_rng(seed)
    flat = random_positions(len(obs_ids), n_samples, density, rng)
    lam = rng.gamma(dispersion, mean / dispersion, size=flat.shape[0])
    vals = np.maximum(rng.poisson(lam), 1).astype(np.float64)
    return make_table(obs_ids, n_samples, flat, vals)


def presence_table(obs_ids, n_samples, rich_lo, rich_hi, seed) -> Table:
    """Per sample, a log-uniform richness r in [rich_lo, rich_hi] of distinct
    features chosen uniformly, each with count 1."""
    rng = np.random.default_rng(seed)
    n_obs = len(obs_ids)
    rich = np.exp(rng.uniform(math.log(rich_lo), math.log(rich_hi), size=n_samples)).astype(np.int64)
    rich = np.minimum(rich, n_obs)
    obs_all = []
    samp_all = []
    for j in range(n_samples):
        obs_all.append(rng.choice(n_obs, size=int(rich[j]), replace=False))
        samp_all.append(np.full(int(rich[j]), j, dtype=np.int64))
    obs_all = np.concatenate(obs_all)
    samp_all = np.concatenate(samp_all)
    flat = np.sort(obs_all * n_samples + samp_all)
    return make_table(obs_ids, n_samples, flat, np.ones(flat.shape[0]))


def rarefy(table: Table, depth: int, seed: int) -> Table:
    """Subsample every sample to `depth` counts without replacement; samples
    below `depth` are dropped and features left empty are removed, as the
    reference's rarefaction does (src/biom_subsampled.cpp:287-353).  Each
    sample's draw is a multivariate hypergeometric taken feature by feature
    (univariate hypergeometric of the feature's count against the rest),
    vectorised across samples.  The random stream is this generator's own:
    both engines are fed the same output."""
    rng = np.random.default_rng(seed)
    n_obs, n = table.n_obs, table.n_samples
    indptr = np.asarray(table.indptr, dtype=np.int64)
    obs = np.repeat(np.arange(n_obs), np.diff(indptr))
    samp = np.asarray(table.indices, dtype=np.int64)
    vals = np.asarray(table.data, dtype=np.float64).astype(np.int64)
    totals = np.bincount(samp, weights=vals, minlength=n).astype(np.int64)
    keep = np.flatnonzero(totals >= depth)
    new_col = np.full(n, -1, dtype=np.int64)
    new_col[keep] = np.arange(keep.shape[0])
    sel = new_col[samp] >= 0
    obs, samp, vals = obs[sel], new_col[samp[sel]], vals[sel]
    order = np.lexsort((obs, samp))  # sample-major, features in order
    obs, samp, vals = obs[order], samp[order], vals[order]
    m = keep.shape[0]
    counts = np.bincount(samp, minlength=m)
    start = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(counts, out=start[1:])
    rank = np.arange(obs.shape[0]) - start[samp]
    width = int(counts.max()) if m else 0
    grid = np.zeros((m, max(width, 1)), dtype=np.int64)
    grid[samp, rank] = vals
    left = grid.sum(axis=1)
    need = np.full(m, depth, dtype=np.int64)
    drawn = np.zeros_like(grid)
    for k in range(width):
        good = grid[:, k]
        bad = left - good
        x = rng.hypergeometric(np.maximum(good, 0), np.maximum(bad, 0), need) if m else good
        x = np.where(good > 0, x, 0)
        drawn[:, k] = x
        need -= x
        left -= good
    d = drawn[samp, rank].astype(np.float64)
    pos = d > 0
    obs, samp, d = obs[pos], samp[pos], d[pos]
    rows = np.unique(obs)
    row_new = np.full(n_obs, -1, dtype=np.int64)
    row_new[rows] = np.arange(rows.shape[0])
    flat = row_new[obs] * m + samp
    order = np.argsort(flat)
    t = make_table([table.obs_ids[i] for i in rows], m, flat[order], d[order])
    t.sample_ids = [table.sample_ids[j] for j in keep]
    return t


# ---------------------------------------------------------------- workloads

def geometric_1k_tips_128_samples(seed: int = 1):
    """1,000-tip tree (Exp mean 0.1); 1,000 x 128 table, 5% non-zero, Geometric(20)+1."""
    tree = random_binary_tree(1000, 0.1, seed)
    table = geometric_table(tree.tip_names(), 128, 0.05, 20.0, seed + 1000)
    return tree, table


def lognormal_20k_tips_2048_samples(seed: int = 2, n_samples: int = 2048, n_tips: int = 20000):
    """20,000-tip tree (Exp mean 0.05); 20,000 x 2,048 table, 1% non-zero,
    round(LogNormal(2, 1.5)) + 1."""
    tree = random_binary_tree(n_tips, 0.05, seed)
    table = lognormal_table(tree.tip_names(), n_samples, 0.01, 2.0, 1.5, seed + 1000)
    return tree, table


def presence_100k_tips_25k_samples(seed: int = 3, n_samples: int = 25000, n_tips: int = 100000):
    """100,000-tip tree (Exp mean 0.02); presence table, richness LogUniform[50, 2000]."""
    tree = random_binary_tree(n_tips, 0.02, seed)
    table = presence_table(tree.tip_names(), n_samples, 50, min(2000, n_tips), seed + 1000)
    return tree, table


def rarefied_replicates_10k_tips_5k_samples(seed: int = 4, n_replicates: int = 100, n_samples: int = 5000,
                                             n_tips: int = 10000, depth: int = 1000):
    """10,000-tip tree (Exp mean 0.1); base 10,000 x 5,000 table, 2% non-zero,
    NegBinomial(50, 0.5); replicates rarefied to `depth` with seed+r."""
    tree = random_binary_tree(n_tips, 0.1, seed)
    base = negbin_table(tree.tip_names(), n_samples, 0.02, 50.0, 0.5, seed + 1000)
    reps = [rarefy(base, depth, seed + r) for r in range(n_replicates)]
    return tree, base, reps


def uneven_tables_50k_tips(seed: int = 5, n_tables: int = 64, n_tips: int = 50000, lo: int = 64, hi: int = 4096):
    """One 50,000-tip tree (Exp mean 0.03); tables with log-uniform sample
    counts in [lo, hi], 1% non-zero, round(LogNormal(2, 1.5)) + 1."""
    tree = random_binary_tree(n_tips, 0.03, seed)
    rng = np.random.default_rng(seed + 1)
    sizes = np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), size=n_tables))).astype(int)
    tips = tree.tip_names()
    tables = [lognormal_table(tips, int(sizes[t]), 0.01, 2.0, 1.5, seed + 1000 + t) for t in range(n_tables)]
    return tree, tables
