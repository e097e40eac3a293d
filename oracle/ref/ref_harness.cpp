/*
 * Test infrastructure only (the oracle), never linked into the product.
 *
 * A C-ABI harness around the reference's own CPU hot path, compiled from the
 * reference sources (tree.cpp, biom_inmem.cpp, unifrac_internal.cpp,
 * unifrac.cpp, unifrac_cmp.cpp) by oracle/Makefile into oracle/_ref/.  The
 * reference's api.cpp cannot be built here (HDF5, LZ4 and libskbb are absent),
 * so this file redoes the few steps of its in-memory entry point
 * `one_off_matrix_T` (src/api.cpp:639-696) with the reference's own types:
 *   biom_inmem over the caller's CSR        (src/api.cpp:796-802)
 *   BPTree from arrays                      (src/api.cpp:804-807)
 *   VALIDATE_TREE_TABLE / SYNC_TREE_TABLE   (src/api.cpp:90-100)
 *   SET_METHOD                              (src/api.cpp:55-88)
 *   set_tasks                               (src/api.cpp:447-491)
 *   su::process_stripes                     (src/unifrac.cpp:521-554)
 *   stripes_to_matrix_T / condensed form    (src/unifrac.cpp:99-120, 229-328)
 * and of `faith_pd_one_off` (src/api.cpp:569-603).
 */
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_set>
#include <vector>

#include "biom_inmem.hpp"
#include "tree.hpp"
#include "unifrac.hpp"

namespace {

// Method-name table of SET_METHOD, src/api.cpp:55-88 (bare names are fp32).
bool parse_method(const char *m, su::Method &out) {
    struct Entry { const char *name; su::Method method; };
    static const Entry table[] = {
        {"unweighted", su::unweighted_fp32},
        {"weighted_normalized", su::weighted_normalized_fp32},
        {"weighted_unnormalized", su::weighted_unnormalized_fp32},
        {"unweighted_unnormalized", su::unweighted_unnormalized_fp32},
        {"generalized", su::generalized_fp32},
        {"unweighted_fp64", su::unweighted},
        {"weighted_normalized_fp64", su::weighted_normalized},
        {"weighted_unnormalized_fp64", su::weighted_unnormalized},
        {"unweighted_unnormalized_fp64", su::unweighted_unnormalized},
        {"generalized_fp64", su::generalized},
        {"unweighted_fp32", su::unweighted_fp32},
        {"weighted_normalized_fp32", su::weighted_normalized_fp32},
        {"weighted_unnormalized_fp32", su::weighted_unnormalized_fp32},
        {"unweighted_unnormalized_fp32", su::unweighted_unnormalized_fp32},
        {"generalized_fp32", su::generalized_fp32},
    };
    for (const Entry &e : table)
        if (std::strcmp(m, e.name) == 0) { out = e.method; return true; }
    return false;
}

// Balanced split of [start, stop) into n tasks, as set_tasks (src/api.cpp:447-491).
std::vector<su::task_parameters> split_tasks(double alpha, unsigned n_samples, unsigned start, unsigned stop,
                                             bool bypass, bool normalize, unsigned n_tasks) {
    if (stop <= start) stop = (n_samples + 1) / 2;
    const unsigned span = stop - start;
    const unsigned big = (span + n_tasks - 1) / n_tasks;
    const unsigned small = span / n_tasks;
    unsigned n_big = span % n_tasks;
    if (n_big == 0) n_big = n_tasks;
    std::vector<su::task_parameters> tasks(n_tasks);
    unsigned s = start;
    for (unsigned t = 0; t < n_tasks; t++) {
        tasks[t].tid = t;
        tasks[t].start = s;
        tasks[t].bypass_tips = bypass;
        tasks[t].normalize_sample_counts = normalize;
        s += (t < n_big) ? big : small;
        tasks[t].stop = s;
        tasks[t].n_samples = n_samples;
        tasks[t].g_unifrac_alpha = alpha;
    }
    return tasks;
}

su::BPTree sheared_tree(const su::BPTree &tree, const su::biom_interface &table) {
    std::unordered_set<std::string> keep(table.get_obs_ids().begin(), table.get_obs_ids().end());
    return tree.shear(keep).collapse();
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

/* Status codes follow ComputeStatus (src/status_enum.hpp:4). */
int ssu_ref_one_off(const uint32_t *indptr, const uint32_t *indices, const double *data, int n_obs, int n_samples,
                    const char *const *obs_ids, const char *const *sample_ids, const bool *structure,
                    const double *lengths, const char *const *names, int n_parens, const char *method,
                    bool variance_adjust, double alpha, bool bypass_tips, bool normalize, unsigned n_substeps,
                    unsigned stripe_start, unsigned stripe_stop, double *out_stripes, double *out_matrix,
                    double *out_condensed, uint64_t *out_n_embedded, double *out_seconds) {
    su::Method m;
    if (!parse_method(method, m)) return 4;  // unknown_method
    if (n_samples <= 0 || n_obs <= 0) return 3;  // table_empty
    su::biom_inmem table(obs_ids, sample_ids, const_cast<uint32_t *>(indices), const_cast<uint32_t *>(indptr),
                         const_cast<double *>(data), n_obs, n_samples);
    su::BPTree tree(structure, lengths, names, n_parens);
    if (su::test_table_ids_are_subset_of_tree(table, tree) != "") return 5;  // table_and_tree_do_not_overlap
    su::BPTree tree_sheared = sheared_tree(tree, table);

    const unsigned n = table.n_samples;
    const unsigned n_stripes = (n + 1) / 2;
    if (stripe_stop == 0 || stripe_stop <= stripe_start) { stripe_start = 0; stripe_stop = n_stripes; }
    if (stripe_stop > n_stripes) return 6;  // output_error: the reference exits here (src/api.cpp:553-556)
    if (n_substeps == 0) n_substeps = 1;
    if (n_substeps > stripe_stop - stripe_start) n_substeps = stripe_stop - stripe_start;

    if (out_n_embedded) {
        uint64_t internal_and_tips = tree_sheared.nparens / 2 - 1;
        uint64_t tips = 0;
        for (uint32_t i = 0; i + 1 < tree_sheared.nparens; i++)
            if (tree_sheared.isleaf(i)) tips++;
        *out_n_embedded = bypass_tips ? internal_and_tips - tips : internal_and_tips;
    }

    std::vector<double *> dm_stripes(n_stripes, nullptr);
    std::vector<double *> dm_stripes_total(n_stripes, nullptr);
    std::vector<su::task_parameters> tasks =
        split_tasks(alpha, n, stripe_start, stripe_stop, bypass_tips, normalize, n_substeps);

    auto t0 = std::chrono::steady_clock::now();
    su::process_stripes(table, tree_sheared, m, variance_adjust, dm_stripes, dm_stripes_total, tasks);
    double t_stripes = seconds_since(t0);

    if (out_stripes)
        for (unsigned s = stripe_start; s < stripe_stop; s++)
            std::memcpy(out_stripes + (uint64_t)(s - stripe_start) * n, dm_stripes[s], sizeof(double) * n);
    double t_matrix = 0.0;
    if (out_matrix && stripe_start == 0 && stripe_stop == n_stripes) {
        auto t1 = std::chrono::steady_clock::now();
        su::MemoryStripes ms(dm_stripes);
        su::stripes_to_matrix_T<double>(ms, n, n_stripes, out_matrix, 128 / sizeof(double));
        t_matrix = seconds_since(t1);
    }
    if (out_condensed && stripe_start == 0 && stripe_stop == n_stripes)
        su::stripes_to_condensed_form(dm_stripes, n, out_condensed, 0, n_stripes);
    if (out_seconds) { out_seconds[0] = t_stripes; out_seconds[1] = t_matrix; }

    for (unsigned s = 0; s < n_stripes; s++) {
        free(dm_stripes[s]);
        free(dm_stripes_total[s]);
    }
    return 0;
}

/* Faith PD with the zero-count sample filter of faith_pd_one_off
 * (src/api.cpp:569-603).  out_values and out_kept need n_samples slots;
 * *out_n_kept receives how many samples survived the filter and out_kept
 * their original indices. */
int ssu_ref_faith_pd(const uint32_t *indptr, const uint32_t *indices, const double *data, int n_obs, int n_samples,
                     const char *const *obs_ids, const char *const *sample_ids, const bool *structure,
                     const double *lengths, const char *const *names, int n_parens, double *out_values,
                     uint32_t *out_kept, uint32_t *out_n_kept, double *out_seconds) {
    if (n_samples <= 0 || n_obs <= 0) return 3;
    su::biom_inmem table(obs_ids, sample_ids, const_cast<uint32_t *>(indices), const_cast<uint32_t *>(indptr),
                         const_cast<double *>(data), n_obs, n_samples);
    su::BPTree tree(structure, lengths, names, n_parens);
    if (su::test_table_ids_are_subset_of_tree(table, tree) != "") return 5;
    su::biom_inmem table_nz(table, 1.0);
    auto t0 = std::chrono::steady_clock::now();
    if (table_nz.n_samples == 0 || table_nz.n_obs == 0) {
        *out_n_kept = table.n_samples;
        for (uint32_t i = 0; i < table.n_samples; i++) { out_values[i] = 0.0; out_kept[i] = i; }
    } else {
        su::BPTree tree_sheared = sheared_tree(tree, table_nz);
        std::vector<double> values(table_nz.n_samples, 0.0);
        su::faith_pd(table_nz, tree_sheared, values.data());
        *out_n_kept = table_nz.n_samples;
        const std::vector<std::string> &kept_ids = table_nz.get_sample_ids();
        uint32_t j = 0;
        for (uint32_t i = 0; i < (uint32_t)n_samples && j < table_nz.n_samples; i++) {
            if (kept_ids[j] == sample_ids[i]) {
                out_kept[j] = i;
                out_values[j] = values[j];
                j++;
            }
        }
    }
    if (out_seconds) out_seconds[0] = seconds_since(t0);
    return 0;
}

}  // extern "C"
