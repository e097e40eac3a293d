// Host-side feature table: borrow, dense pair, filter, rarefy, totals.
#include "ssu_table.hpp"

#include <random>

namespace ssu {

void Table::adopt_owned() {
    indptr = own_indptr.data();
    indices = own_indices.data();
    data = own_data.data();
}

void Table::compute_totals() {
    totals.assign(n_samples, 0.0);
    nonneg = true;
    malformed = false;
    if (n_obs && indptr[0] != 0) malformed = true;
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

Table Table::rarefied(uint32_t depth, bool with_replacement, uint64_t seed) const {
    // sample-major view of the kept samples
    std::vector<uint32_t> keep;
    for (uint32_t j = 0; j < n_samples; j++)
        if (totals[j] >= depth) keep.push_back(j);
    std::vector<uint32_t> new_idx(n_samples, UINT32_MAX);
    for (uint32_t jj = 0; jj < keep.size(); jj++) new_idx[keep[jj]] = jj;
    std::vector<std::vector<std::pair<uint32_t, double>>> cols(keep.size());
    for (uint32_t i = 0; i < n_obs; i++)
        for (uint32_t q = indptr[i]; q < indptr[i + 1]; q++)
            if (new_idx[indices[q]] != UINT32_MAX) cols[new_idx[indices[q]]].emplace_back(i, data[q]);

    std::mt19937_64 gen(seed);
    std::vector<std::vector<double>> sub(keep.size());
    for (uint32_t jj = 0; jj < keep.size(); jj++) {
        auto &col = cols[jj];
        std::vector<double> out(col.size(), 0.0);
        if (with_replacement) {
            std::vector<double> w(col.size());
            for (size_t e = 0; e < col.size(); e++) w[e] = col[e].second;
            std::discrete_distribution<size_t> pick(w.begin(), w.end());
            for (uint32_t d = 0; d < depth; d++) out[pick(gen)] += 1.0;
        } else {
            // `depth` draws without replacement from the multiset of integer
            // counts: partial Fisher-Yates over the expanded items
            std::vector<uint32_t> items;
            for (size_t e = 0; e < col.size(); e++) {
                const uint64_t c = static_cast<uint64_t>(col[e].second);
                items.insert(items.end(), c, static_cast<uint32_t>(e));
            }
            for (uint32_t d = 0; d < depth && d < items.size(); d++) {
                std::uniform_int_distribution<size_t> u(d, items.size() - 1);
                std::swap(items[d], items[u(gen)]);
                out[items[d]] += 1.0;
            }
        }
        sub[jj] = std::move(out);
    }
    // back to observation-major, dropping observations left without counts
    std::vector<std::vector<std::pair<uint32_t, double>>> rows(n_obs);
    for (uint32_t jj = 0; jj < keep.size(); jj++)
        for (size_t e = 0; e < cols[jj].size(); e++)
            rows[cols[jj][e].first].emplace_back(jj, sub[jj][e]);
    Table t;
    t.n_samples = static_cast<uint32_t>(keep.size());
    for (uint32_t jj = 0; jj < keep.size(); jj++) t.sample_ids.push_back(sample_ids[keep[jj]]);
    t.own_indptr.push_back(0);
    for (uint32_t i = 0; i < n_obs; i++) {
        bool any = false;
        for (auto &e : rows[i]) any = any || e.second > 0.0;
        if (!any) continue;
        for (auto &e : rows[i]) {
            if (e.second <= 0.0) continue;
            t.own_indices.push_back(e.first);
            t.own_data.push_back(e.second);
        }
        t.obs_ids.push_back(obs_ids[i]);
        t.own_indptr.push_back(static_cast<uint32_t>(t.own_indices.size()));
    }
    t.n_obs = static_cast<uint32_t>(t.obs_ids.size());
    t.adopt_owned();
    t.compute_totals();
    return t;
}

std::unordered_map<std::string_view, uint32_t> Table::obs_index() const {
    std::unordered_map<std::string_view, uint32_t> m;
    m.reserve(n_obs * 2 + 1);
    for (uint32_t i = 0; i < n_obs; i++) m[obs_ids[i]] = i;
    return m;
}

}  // namespace ssu
