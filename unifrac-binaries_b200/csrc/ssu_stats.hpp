// Consumers of the distance matrix on the device: principal coordinates
// (PCoA) and PERMANOVA.  The reference hands both to scikit-bio-binaries
// (src/skbio_alt.cpp:144-234: skbb_pcoa_fsvd_*, skbb_permanova_*), a
// dependency not carried in its tree; these restate the published methods
// of scikit-bio (ordination.pcoa with method "fsvd", stats.distance.permanova).
#pragma once

#include <cstdint>
#include <string>

namespace ssu {

// Matrices are n x n row-major, in host memory (copied to the device) or in
// device memory (read in place).
//
// PCoA of the distance matrix `mat`:
// E = -D^2 / 2 Gower-centred, F = (I - 11'/n) E (I - 11'/n); the `dims`
// largest eigenpairs of F by randomized subspace iteration with Rayleigh-Ritz
// (Halko, Martinsson, Tropp 2011, algorithm 4.4 with 10 extra columns; power
// steps until the wanted Ritz values move by at most 1e-12 of the largest,
// 4 to 60 of them), done in fp64 whatever TIn.  eigenvalues[dims]: descending;
// samples[n][dims]: eigenvector * sqrt(max(eigenvalue, 0)), each vector's
// largest-magnitude entry positive; proportion[dims]: eigenvalue / trace(F).
// Returns 0, or 6 with `err` set.
template <typename TIn>
int pcoa_device(const TIn *mat, uint32_t n, uint32_t dims, double *eigenvalues, double *samples, double *proportion,
                std::string &err);

// The `dims` largest eigenpairs of the symmetric matrix `mat` (already
// centred: the reference's find_eigens_fast), by the same iteration:
// eigenvalues[dims] descending, vectors[n][dims] unit eigenvectors with their
// largest-magnitude entry positive.  Returns 0, or 6 with `err` set.
template <typename TIn>
int eigens_device(const TIn *mat, uint32_t n, uint32_t dims, double *eigenvalues, double *vectors, std::string &err);

// PERMANOVA pseudo-F of `grouping` (n labels in [0, n_groups)) over the
// distance matrix `mat`, upper triangle read (j > i): s_T = sum_{i<j} d^2 / n,
// s_W = sum_groups sum_{i<j in g} d^2 / n_g, F = ((s_T - s_W) / (G - 1)) /
// (s_W / (n - G)); p = (1 + #{F of a permuted grouping >= F}) / (1 + perms),
// the permutations drawn from `seed`.  F and p are NaN when G < 2 or G == n
// (p also when perms == 0).  At most 65535 groups.  Returns 0, or 6 with
// `err` set.
template <typename TIn>
int permanova_device(const TIn *mat, uint32_t n, const uint32_t *grouping, uint32_t n_groups, uint32_t perms,
                     uint64_t seed, double &fstat, double &pvalue, std::string &err);

}  // namespace ssu
