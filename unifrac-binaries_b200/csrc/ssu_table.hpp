// Host-side feature table for the B200 UniFrac engine: an observation-major
// CSR (the reference's biom_inmem sparse layout, src/biom_inmem.cpp:130-157),
// borrowed from the caller or owned after filtering / rarefaction.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <string_view>
#include <unordered_map>
#include <vector>

namespace ssu {

struct TipMatch;
class NameMap;

struct Table {
    Table() = default;
    Table(const Table &) = delete;  // owned arrays are referenced by pointer
    Table &operator=(const Table &) = delete;
    Table(Table &&) = default;
    Table &operator=(Table &&) = default;

    uint32_t n_obs = 0;
    uint32_t n_samples = 0;
    const uint32_t *indptr = nullptr;   // n_obs + 1
    const uint32_t *indices = nullptr;  // sample positions
    const double *data = nullptr;
    // views into the caller's id strings (valid for the call)
    std::vector<std::string_view> obs_ids;
    std::vector<std::string_view> sample_ids;
    std::vector<double> totals;  // per-sample sum, accumulated in observation order
    // a borrowed CSR that cannot be indexed safely: offsets not starting at 0
    // or decreasing, or a sample position >= n_samples (such entries are left
    // out of the totals; validation rejects the table before device work)
    bool malformed = false;
    // no entry below zero (found while the totals are summed)
    bool nonneg = true;

    // Name matching of this table against the call's tree, made once by the
    // validation and reused by the shear (host-side cache of one call).
    mutable std::shared_ptr<const NameMap> names;
    mutable uint32_t distinct_names = 0;
    mutable std::shared_ptr<const TipMatch> tip_match;

    // storage when the table owns its arrays (and, for tables read from a
    // file, the bytes its id views point into)
    std::vector<uint32_t> own_indptr, own_indices;
    std::vector<double> own_data;
    std::unique_ptr<char[]> own_names;

    uint64_t nnz() const { return n_obs ? indptr[n_obs] : 0; }

    // Borrow a caller's CSR (not copied, as src/biom_inmem.cpp:129-157).
    static Table borrow(uint32_t n_obs, uint32_t n_samples, const uint32_t *indptr, const uint32_t *indices,
                        const double *data, const char *const *obs_ids, const char *const *sample_ids);
    // Two dense samples; only strictly positive values are kept
    // (src/biom_inmem.cpp:160-190).
    static Table dense_pair(uint32_t n_obs, const char *const *obs_ids, const double *s1, const double *s2);

    // Samples with total >= min_total, re-numbered, and observations that
    // keep at least one entry (src/biom_inmem.cpp:284-338).  Totals are the
    // parent's.
    Table filtered(double min_total) const;

    void compute_totals();
    std::unordered_map<std::string_view, uint32_t> obs_index() const;
    // point indptr / indices / data at the owned arrays
    void adopt() { adopt_owned(); }

  private:
    void adopt_owned();
};

}  // namespace ssu
