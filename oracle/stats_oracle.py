"""Test infrastructure only: numpy restatement of the statistics the
reference runs on a distance matrix.

The reference delegates PCoA and PERMANOVA to scikit-bio-binaries
(src/skbio_alt.cpp:144-234: skbb_center_distance_matrix_*, skbb_pcoa_fsvd_*,
skbb_fsvd_inplace_*, skbb_permanova_*), a dependency that is not vendored in
its tree and has no pinned version there (conda package
scikit-bio-binaries).  Its published methods are scikit-bio's
(skbio.stats.ordination.pcoa, skbio.stats.distance.permanova); this module
restates them exactly (dense symmetric eigendecomposition instead of the
randomized fsvd, which approximates the same eigenpairs):

* centring: F = (I - 11'/n)(-D*D/2)(I - 11'/n)      (src/skbio_alt.cpp:144-157)
* PCoA: the largest eigenpairs of F; coordinates eigvec * sqrt(eigval);
  proportion explained eigval / trace(F), the fsvd form  (:176-199)
* PERMANOVA: s_T = sum_{i<j} d^2 / n, s_W = sum over groups of
  sum_{i<j in g} d^2 / n_g, F = (s_A / (G-1)) / (s_W / (n-G)),
  p = (1 + #{F_perm >= F}) / (1 + perms)                   (:219-234)

Pinned against the reference's own known answers in src/test_ska.cpp
(test_center_mat, test_pcoa, test_pcoa_big, test_permanova_*) and the
scikit-bio values its validation script checks (src/testdata/
validation_tests.sh), by tests/test_stats_oracle.py.

Only tests/ import this module; the product never does.
"""
from __future__ import annotations

import itertools

import numpy as np


def center(d):
    """Gower-centred -d^2/2 (src/skbio_alt.cpp:144-157)."""
    d = np.asarray(d, dtype=np.float64)
    e = -0.5 * d * d
    return e - e.mean(axis=0, keepdims=True) - e.mean(axis=1, keepdims=True) + e.mean()


def eigens(a, dims):
    """The `dims` largest eigenpairs of the symmetric matrix a: (values
    descending, vectors [n][dims])."""
    w, v = np.linalg.eigh(np.asarray(a, dtype=np.float64))
    order = np.argsort(w)[::-1][:dims]
    return w[order], v[:, order]


def pcoa(d, dims):
    """(eigenvalues, samples [n][dims], proportion explained) of scikit-bio's
    PCoA with the fsvd proportion (eigenvalue / trace of the centred matrix)."""
    f = center(d)
    w, v = eigens(f, dims)
    return w, v * np.sqrt(np.maximum(w, 0.0)), w / np.trace(f)


def _labels(grouping):
    _, inv = np.unique(np.asarray(grouping), return_inverse=True)
    return inv


def permanova_f(d, grouping):
    """PERMANOVA pseudo-F over the upper triangle of d (j > i)."""
    d = np.asarray(d, dtype=np.float64)
    g = _labels(grouping)
    n = d.shape[0]
    n_groups = g.max() + 1
    iu = np.triu_indices(n, 1)
    d2 = d[iu] ** 2
    s_t = d2.sum() / n
    sizes = np.bincount(g, minlength=n_groups).astype(np.float64)
    same = g[iu[0]] == g[iu[1]]
    s_w = (d2[same] / sizes[g[iu[0]][same]]).sum()
    return ((s_t - s_w) / (n_groups - 1)) / (s_w / (n - n_groups))


def permanova_p_exact(d, grouping):
    """The p-value a PERMANOVA with infinitely many permutations converges to:
    the share of all distinct relabelings whose F is >= the observed F
    (small n only)."""
    g = list(np.asarray(grouping))
    f0 = permanova_f(d, g)
    seen = set()
    ge = 0
    for perm in itertools.permutations(g):
        if perm in seen:
            continue
        seen.add(perm)
        ge += permanova_f(d, perm) >= f0 - 1e-12 * abs(f0)
    return ge / len(seen)
