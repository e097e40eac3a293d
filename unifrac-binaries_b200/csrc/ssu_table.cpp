// Host-side feature table: borrow, dense pair, filter, rarefy, totals.
#include "ssu_table.hpp"

#include <algorithm>
#include <cmath>

#include "ssu_host.hpp"


namespace ssu {

void Table::adopt_owned() {
    indptr = own_indptr.data();
    indices = own_indices.data();
    data = own_data.data();
}

// Per-sample totals in observation order, with the shape checks.  Large
// tables are summed by observation ranges on several threads first: when
// every entry is an integer and the sum of magnitudes stays below 2^52,
// every partial and final sum is an integer that fp64 holds exactly, so the
// ranges' sums added in any order equal the observation-order sum bit for
// bit (counts, presence and rarefied tables).  Other tables (proportions,
// fractional abundances) are summed again in observation order.
void Table::compute_totals() {
    totals.assign(n_samples, 0.0);
    nonneg = true;
    malformed = false;
    if (n_obs && indptr[0] != 0) malformed = true;
    const uint64_t nnz_hint = n_obs ? indptr[n_obs] : 0;
    const unsigned threads = host_threads(8);
    if (threads > 1 && n_obs >= 1024 && nnz_hint >= (uint64_t(1) << 21)) {
        struct Part {
            std::vector<double> sum;
            double mag = 0.0;
            bool integral = true, nonneg = true, malformed = false;
        };
        std::vector<Part> parts(threads);
        // ranges of about nnz / threads entries (cuts kept in order for any indptr)
        std::vector<uint32_t> cut(threads + 1, 0);
        cut[threads] = n_obs;
        for (unsigned p = 1; p < threads; p++) {
            const uint64_t target = nnz_hint * p / threads;
            const uint32_t *at = std::lower_bound(indptr, indptr + n_obs, static_cast<uint32_t>(target));
            cut[p] = std::max(cut[p - 1], static_cast<uint32_t>(at - indptr));
        }
        parallel_for(threads, threads, [&](unsigned p) {
            // flags in locals: the parts share cache lines
            std::vector<double> sum(n_samples, 0.0);
            double mag = 0.0;
            bool integral = true, nneg = true, bad = false;
            for (uint32_t i = cut[p]; i < cut[p + 1]; i++) {
                if (indptr[i + 1] < indptr[i]) {
                    bad = true;
                    continue;
                }
                for (uint32_t q = indptr[i]; q < indptr[i + 1]; q++) {
                    const uint32_t j = indices[q];
                    const double x = data[q];
                    nneg = nneg && x >= 0.0;
                    integral = integral && x == std::trunc(x);
                    mag += std::fabs(x);
                    if (j < n_samples)
                        sum[j] += x;
                    else
                        bad = true;
                }
            }
            Part &r = parts[p];
            r.sum.swap(sum);
            r.mag = mag;
            r.integral = integral;
            r.nonneg = nneg;
            r.malformed = bad;
        });
        bool integral = true;
        double mag = 0.0;
        for (const Part &r : parts) {
            malformed = malformed || r.malformed;
            nonneg = nonneg && r.nonneg;
            integral = integral && r.integral;
            mag += r.mag;
        }
        if (integral && mag < 4503599627370496.0) {  // 2^52
            for (const Part &r : parts)
                for (uint32_t j = 0; j < n_samples; j++) totals[j] += r.sum[j];
            return;
        }
        totals.assign(n_samples, 0.0);
        nonneg = true;
        malformed = n_obs && indptr[0] != 0;
    }
    for (uint32_t i = 0; i < n_obs; i++) {
        if (indptr[i + 1] < indptr[i]) {
            malformed = true;
            continue;
        }
        for (uint32_t q = indptr[i]; q < indptr[i + 1]; q++) {
            const uint32_t j = indices[q];
            if (!(data[q] >= 0.0)) nonneg = false;
            if (j < n_samples)
                totals[j] += data[q];
            else
                malformed = true;
        }
    }
}

Table Table::borrow(uint32_t n_obs, uint32_t n_samples, const uint32_t *indptr, const uint32_t *indices,
                    const double *data, const char *const *obs_ids, const char *const *sample_ids) {
    Table t;
    t.n_obs = n_obs;
    t.n_samples = n_samples;
    t.indptr = indptr;
    t.indices = indices;
    t.data = data;
    t.obs_ids.reserve(n_obs);
    for (uint32_t i = 0; i < n_obs; i++) t.obs_ids.emplace_back(obs_ids[i]);
    t.sample_ids.reserve(n_samples);
    for (uint32_t j = 0; j < n_samples; j++) t.sample_ids.emplace_back(sample_ids[j]);
    t.compute_totals();
    return t;
}

Table Table::dense_pair(uint32_t n_obs, const char *const *obs_ids, const double *s1, const double *s2) {
    Table t;
    t.n_obs = n_obs;
    t.n_samples = 2;
    t.own_indptr.assign(n_obs + 1, 0);
    for (uint32_t i = 0; i < n_obs; i++) {
        if (s1[i] > 0.0) { t.own_indices.push_back(0); t.own_data.push_back(s1[i]); }
        if (s2[i] > 0.0) { t.own_indices.push_back(1); t.own_data.push_back(s2[i]); }
        t.own_indptr[i + 1] = static_cast<uint32_t>(t.own_indices.size());
        t.obs_ids.emplace_back(obs_ids[i]);
    }
    t.sample_ids = {"Sample1", "Sample2"};
    t.adopt_owned();
    t.compute_totals();
    return t;
}

Table Table::filtered(double min_total) const {
    Table t;
    std::vector<uint32_t> new_idx(n_samples, UINT32_MAX);
    for (uint32_t j = 0; j < n_samples; j++) {
        if (totals[j] >= min_total) {
            new_idx[j] = t.n_samples++;
            t.sample_ids.push_back(sample_ids[j]);
            t.totals.push_back(totals[j]);
        }
    }
    t.own_indptr.push_back(0);
    for (uint32_t i = 0; i < n_obs; i++) {
        const size_t before = t.own_indices.size();
        for (uint32_t q = indptr[i]; q < indptr[i + 1]; q++) {
            if (new_idx[indices[q]] == UINT32_MAX) continue;
            t.own_indices.push_back(new_idx[indices[q]]);
            t.own_data.push_back(data[q]);
            if (!(data[q] >= 0.0)) t.nonneg = false;
        }
        if (t.own_indices.size() > before) {
            t.obs_ids.push_back(obs_ids[i]);
            t.own_indptr.push_back(static_cast<uint32_t>(t.own_indices.size()));
        }
    }
    t.n_obs = static_cast<uint32_t>(t.obs_ids.size());
    if (t.n_obs == 0 || t.n_samples == 0) {
        t.n_obs = 0;
        t.n_samples = 0;
    }
    t.adopt_owned();
    return t;
}

std::unordered_map<std::string_view, uint32_t> Table::obs_index() const {
    std::unordered_map<std::string_view, uint32_t> m;
    m.reserve(n_obs * 2 + 1);
    for (uint32_t i = 0; i < n_obs; i++) m[obs_ids[i]] = i;
    return m;
}

}  // namespace ssu
