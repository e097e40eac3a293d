// C ABI of the B200 UniFrac engine (include/unifrac_b200.h).
//
// Host orchestration mirrors the reference's API layer (src/api.cpp):
// validate table and tree, shear and collapse the tree to the table's
// features, run the device plan, and hand back malloc'ed results that the
// caller releases through destroy_*().  Nothing here exits the process.
#include "unifrac_b200.h"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <fcntl.h>
#include <sched.h>
#include <system_error>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <sys/mman.h>
#include <map>
#include <mutex>
#include <thread>
#include <unistd.h>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <cuda_runtime.h>

#include "ssu_biom.hpp"
#include "ssu_engine.hpp"
#include "ssu_grouping.hpp"
#include "ssu_partial.hpp"
#include "ssu_rarefy.hpp"
#include "ssu_stats.hpp"
#include "ssu_table.hpp"
#include "ssu_tree.hpp"
#include "ssu_host.hpp"

namespace {

constexpr uint32_t kMmapFdMask = 0x0fff;  // src/api.cpp:27-28
constexpr uint32_t kMmapFlag = 0x1000;
constexpr uint32_t kPinnedFlag = 0x2000;  // matrix from the page-locked result pool
constexpr size_t kHugeAlign = size_t(2) << 20;

std::atomic<uint64_t> g_seed{5489u};

using ssu::host_threads;
using ssu::parallel_for;

bool env_yes(const char *name) {
    const char *v = std::getenv(name);
    if (!v) return false;
    const std::string s(v);
    return !(s == "NO" || s == "N" || s == "no" || s == "n" || s == "NEVER" || s == "never");
}

// UNIFRAC_TIMING_INFO step timer, as the reference's SETUP_TDBG/TDBG_STEP
// (src/api.cpp:34-49) with millisecond resolution.
struct StepTimer {
    const char *what;
    bool on;
    std::chrono::steady_clock::time_point t0;
    explicit StepTimer(const char *w) : what(w), on(env_yes("UNIFRAC_TIMING_INFO")), t0(std::chrono::steady_clock::now()) {
        if (on) std::printf("INFO (unifrac): Starting %s\n", what);
    }
    void step(const char *name) {
        if (!on) return;
        auto t1 = std::chrono::steady_clock::now();
        std::printf("INFO (unifrac): dt %8.3f ms : Completed %s.%s\n",
                    std::chrono::duration<double, std::milli>(t1 - t0).count(), what, name);
        t0 = t1;
    }
};

// Select the device as the reference's OpenACC runtime does (ACC_DEVICE_NUM).
bool select_device(std::string &err) {
    static std::atomic<bool> announced{false};
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        err = "no CUDA device available";
        return false;
    }
    if (const char *d = std::getenv("ACC_DEVICE_NUM")) {
        const int id = std::atoi(d);
        if (id >= 0 && id < count && cudaSetDevice(id) != cudaSuccess) {
            err = "cudaSetDevice failed";
            return false;
        }
    }
    if (env_yes("UNIFRAC_GPU_INFO") && !announced.exchange(true)) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, dev) == cudaSuccess)
            std::printf("INFO (unifrac): Using GPU %d (%s), B200 engine\n", dev, p.name);
    }
    return true;
}

void report(const std::string &where, const std::string &err) {
    if (!err.empty()) std::fprintf(stderr, "unifrac-b200: %s: %s\n", where.c_str(), err.c_str());
}

ComputeStatus is_fp64_method(const char *m, bool &fp64) {
    ssu::Method method;
    if (!ssu::parse_method(m, method, fp64)) return unknown_method;
    return okay;
}

char **copy_ids(const std::vector<std::string_view> &ids) {
    char **out = static_cast<char **>(std::malloc(sizeof(char *) * (ids.size() ? ids.size() : 1)));
    for (size_t i = 0; i < ids.size(); i++) {
        out[i] = static_cast<char *>(std::malloc(ids[i].size() + 1));
        std::memcpy(out[i], ids[i].data(), ids[i].size());
        out[i][ids[i].size()] = '\0';
    }
    return out;
}

ssu::Table table_from(const support_biom_t *t) {
    return ssu::Table::borrow(static_cast<uint32_t>(t->n_obs), static_cast<uint32_t>(t->n_samples), t->indptr,
                              t->indices, t->data, t->obs_ids, t->sample_ids);
}

// The caller's arrays outlive the call: names are viewed, not copied.
ssu::BPTree tree_from(const support_bptree_t *t, bool copy_names = false) {
    return ssu::BPTree::from_arrays(t->structure, t->lengths, t->names, t->n_parens, copy_names);
}

const ssu::NameMap &obs_map(const ssu::Table &table);

// The caller's table and tree, read side by side for large trees: the
// tree's arrays on a helper thread while this thread reads the table (ids,
// per-sample totals) and builds its name map.  Small trees are read inline,
// where a thread would cost more than it saves.
void read_inputs(const support_biom_t *table_data, const support_bptree_t *tree_data, ssu::Table &table,
                 ssu::BPTree &tree) {
    constexpr int kThreadedParens = 16384;
    if (tree_data->n_parens < kThreadedParens) {
        table = table_from(table_data);
        tree = tree_from(tree_data);
        return;
    }
    std::thread reader([&tree, tree_data] { tree = tree_from(tree_data); });
    table = table_from(table_data);
    obs_map(table);
    reader.join();
}

// Observation name -> row (the last row wins for a repeated name, as the
// reference's obs_id_index map), built once per table and call; the table
// keeps it with its number of distinct names.
const ssu::NameMap &obs_map(const ssu::Table &table) {
    if (!table.names) {
        auto m = std::make_shared<ssu::NameMap>(table.n_obs);
        uint32_t d = 0;
        for (uint32_t i = 0; i < table.n_obs; i++) d += m->set(table.obs_ids[i], i) ? 1u : 0u;
        table.distinct_names = d;
        table.names = std::move(m);
    }
    return *table.names;
}

// The table's tips matched against `tree`, computed once per call.
const ssu::TipMatch &tip_match(const ssu::Table &table, const ssu::BPTree &tree) {
    if (!table.tip_match || table.tip_match->tree_id != tree.open.data() ||
        table.tip_match->tree_size != tree.size())
        table.tip_match = std::make_shared<ssu::TipMatch>(tree.match_tips(obs_map(table), table.n_obs));
    return *table.tip_match;
}

// VALIDATE_TREE_TABLE (src/api.cpp:94-100): every table id is a tip name.
ComputeStatus validate(const ssu::Table &table, const ssu::BPTree &tree) {
    if (table.n_samples == 0 || table.n_obs == 0) return table_empty;
    if (table.malformed) {
        report("table", "malformed CSR (offsets or sample positions out of range)");
        return table_missing;
    }
    if (tree.malformed) {
        report("tree", "parentheses do not pair up");
        return tree_missing;
    }
    const ssu::TipMatch &m = tip_match(table, tree);
    return m.rows_matched == table.distinct_names ? okay : table_and_tree_do_not_overlap;
}

// SYNC_TREE_TABLE (src/api.cpp:90-92) + flattening for the device.  The kept
// tips carry their table rows; when every tip is in the table the shear is
// the tree itself, and a tree without single-child nodes collapses to itself.
ssu::FlatTree sync_tree(const ssu::Table &table, const ssu::BPTree &tree, bool bypass_tips) {
    const ssu::TipMatch &m = tip_match(table, tree);
    bool single = false;
    if (m.all_tips) {
        ssu::FlatTree f = ssu::flatten(tree, bypass_tips, &m.tags, &single);
        if (!single) return f;
        return ssu::flatten(tree.collapse(&m.tags), bypass_tips);
    }
    const ssu::BPTree sheared = tree.shear_matched(m);
    ssu::FlatTree f = ssu::flatten(sheared, bypass_tips, nullptr, &single);
    if (!single) return f;
    return ssu::flatten(sheared.collapse(), bypass_tips);
}

// UNIFRAC_B200_UNWEIGHTED_MODE: "gemm" runs unweighted methods on the
// tensor-core contraction for fp64 results too (max relative error ~1e-7
// instead of the stripe form's bit-level agreement); "stripe" keeps the
// presence-word stripe kernel for fp32 results as well.
void unweighted_mode(ssu::MethodSpec &spec) {
    if (const char *mode = std::getenv("UNIFRAC_B200_UNWEIGHTED_MODE")) {
        spec.unweighted_gemm = std::string(mode) == "gemm";
        spec.unweighted_stripe = std::string(mode) == "stripe";
    }
}

struct Request {
    const char *method;
    bool vaw;
    double alpha;
    bool bypass;
    bool normalize;
};

ComputeStatus make_plan(const ssu::Table &table, const ssu::BPTree &tree, const Request &r,
                        std::unique_ptr<ssu::Plan> &plan, StepTimer &timer) {
    ssu::MethodSpec spec;
    if (!ssu::parse_method(r.method, spec.method, spec.fp64)) return unknown_method;
    spec.vaw = r.vaw;
    spec.alpha = r.alpha;
    spec.bypass_tips = r.bypass;
    spec.normalize = r.normalize;
    unweighted_mode(spec);
    std::string err;
    if (!select_device(err)) {
        report("device", err);
        return output_error;
    }
    const ssu::FlatTree flat = sync_tree(table, tree, r.bypass);
    timer.step("sync_tree_table");
    ssu::Plan *p = nullptr;
    const int rc = ssu::Plan::create(table, flat, spec, nullptr, &p, err);
    if (rc) {
        report("plan", err);
        return static_cast<ComputeStatus>(rc);
    }
    plan.reset(p);
    timer.step("upload");
    return okay;
}

// Page-locked host memory for full results: the copy-out then runs at the
// link's rate with no per-call page registration.  Blocks released through
// destroy_mat_full_* are kept for later results (best fit, up to twice the
// request) while the pool holds at most UNIFRAC_B200_PINNED_BYTES (default:
// a sixteenth of the host's memory, within [4, 16] GiB) live and cached
// together; beyond that results use pageable memory.
class PinnedPool {
  public:
    static PinnedPool &get() {
        static PinnedPool p;
        return p;
    }
    void *take(size_t bytes) {
        std::lock_guard<std::mutex> lock(mu_);
        auto it = free_.lower_bound(bytes);
        if (it != free_.end() && it->first <= 2 * bytes) {
            void *p = it->second;
            cached_ -= it->first;
            live_bytes_ += it->first;
            live_[p] = it->first;
            free_.erase(it);
            return p;
        }
        while (held() + bytes > limit_ && !free_.empty()) {  // make room from the cache
            auto big = std::prev(free_.end());
            cudaFreeHost(big->second);
            cached_ -= big->first;
            free_.erase(big);
        }
        if (held() + bytes > limit_) return nullptr;
        void *p = nullptr;
        if (cudaMallocHost(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        live_[p] = bytes;
        live_bytes_ += bytes;
        return p;
    }
    void give(void *p) {
        std::lock_guard<std::mutex> lock(mu_);
        auto it = live_.find(p);
        if (it == live_.end()) return;
        const size_t cap = it->second;
        live_.erase(it);
        live_bytes_ -= cap;
        free_.emplace(cap, p);
        cached_ += cap;
    }

  private:
    PinnedPool() {
        const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGESIZE);
        if (pages > 0 && page > 0)
            limit_ = std::min(std::max(static_cast<size_t>(pages) * static_cast<size_t>(page) / 16, size_t(4) << 30),
                              size_t(16) << 30);
        if (const char *v = std::getenv("UNIFRAC_B200_PINNED_BYTES")) limit_ = std::strtoull(v, nullptr, 10);
    }
    size_t held() const { return live_bytes_ + cached_; }
    std::mutex mu_;
    std::multimap<size_t, void *> free_;
    std::unordered_map<void *, size_t> live_;
    size_t live_bytes_ = 0, cached_ = 0;
    size_t limit_ = size_t(4) << 30;
};

template <class TReal, class TMat>
bool alloc_full(TMat *&result, const std::vector<std::string_view> &ids, const char *mmap_dir) {
    result = static_cast<TMat *>(std::malloc(sizeof(TMat)));
    result->n_samples = static_cast<uint32_t>(ids.size());
    result->flags = 0;
    result->sample_ids = copy_ids(ids);
    const uint64_t n = ids.size();
    const uint64_t bytes = sizeof(TReal) * n * n;
    if (mmap_dir && mmap_dir[0]) {
        std::string tmpl = std::string(mmap_dir) + "/su_mmap_XXXXXX";
        int fd = mkstemp(&tmpl[0]);
        result->matrix = nullptr;
        if (fd >= 0) {
            unlink(tmpl.c_str());
            if (ftruncate(fd, static_cast<off_t>(bytes)) == 0) {
                void *m = mmap(nullptr, bytes ? bytes : 1, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_NORESERVE, fd, 0);
                if (m != MAP_FAILED) {
                    result->matrix = static_cast<TReal *>(m);
                    result->flags = (static_cast<uint32_t>(fd) & kMmapFdMask) | kMmapFlag;
                }
            }
            if (!result->matrix) close(fd);
        }
    } else if (bytes >= kHugeAlign) {
        void *p = PinnedPool::get().take(bytes);
        if (p) {
            result->matrix = static_cast<TReal *>(p);
            result->flags = kPinnedFlag;
            return true;
        }
        // 2 MiB-aligned with transparent huge pages: ~500x fewer page faults
        // when the result is written; still released with free()
        if (posix_memalign(&p, kHugeAlign, bytes) == 0) {
            madvise(p, bytes, MADV_HUGEPAGE);
            result->matrix = static_cast<TReal *>(p);
        } else {
            result->matrix = nullptr;
        }
    } else {
        result->matrix = static_cast<TReal *>(std::malloc(bytes ? bytes : 1));
    }
    return result->matrix != nullptr;
}

// Touch every page of a fresh host buffer on a few threads (run while the
// GPU computes, so the copy-out finds resident pages).
void prefault(void *p, size_t bytes) {
    const unsigned hw = host_threads(8);
    const size_t slice = ((bytes / hw) + kHugeAlign - 1) / kHugeAlign * kHugeAlign;
    const unsigned parts = static_cast<unsigned>((bytes + slice - 1) / slice);
    parallel_for(parts, hw, [&](unsigned t) {
        const size_t a = t * slice;
        std::memset(static_cast<char *>(p) + a, 0, std::min(slice, bytes - a));
    });
}

template <class TMat, class TReal>
void destroy_full(TMat **result) {
    if (!result || !*result) return;
    TMat *r = *result;
    for (uint32_t i = 0; i < r->n_samples; i++) std::free(r->sample_ids[i]);
    std::free(r->sample_ids);
    if (r->matrix) {
        if (r->flags & kPinnedFlag) {
            PinnedPool::get().give(r->matrix);
        } else if ((r->flags & kMmapFlag) == 0) {
            std::free(r->matrix);
        } else {
            const uint64_t n = r->n_samples;
            const size_t bytes = sizeof(TReal) * n * n;
            munmap(r->matrix, bytes ? bytes : 1);
            close(static_cast<int>(r->flags & kMmapFdMask));
        }
        r->matrix = nullptr;
    }
    std::free(r);
    *result = nullptr;
}

// one_off_matrix_T (src/api.cpp:639-696) over an already validated table.
template <class TReal, class TMat>
ComputeStatus full_matrix(const ssu::Table &table, const ssu::BPTree &tree, const Request &r, const char *mmap_dir,
                          TMat **result) {
    StepTimer timer("one_off_matrix_inmem");
    std::unique_ptr<ssu::Plan> plan;
    ComputeStatus st = make_plan(table, tree, r, plan, timer);
    if (st != okay) return st;
    bool allocated = false;
    if (*result == nullptr) {
        if (!alloc_full<TReal, TMat>(*result, table.sample_ids, mmap_dir)) {
            destroy_full<TMat, TReal>(result);
            report("one_off_matrix", "result allocation failed");
            return output_error;
        }
        allocated = true;
    }
    timer.step(((*result)->flags & kPinnedFlag) ? "result_alloc (page-locked)" : "result_alloc (pageable)");
    if ((*result)->matrix == nullptr || (*result)->n_samples != table.n_samples) {
        report("one_off_matrix", "caller-provided result does not match the table");
        return output_error;
    }
    std::string err;
    bool method_fp64 = false;
    is_fp64_method(r.method, method_fp64);
    const size_t elems = static_cast<size_t>(table.n_samples) * table.n_samples;
    const bool convert = method_fp64 != (sizeof(TReal) == sizeof(double));
    int rc = convert ? plan->execute(nullptr) : 0;
    if (rc == 0 && convert) {
        // the file-based calls compute in the method's precision and write
        // the result type's (stripes_to_matrix_T<TReal>, src/api.cpp:684-690)
        if (method_fp64) {
            std::vector<double> tmp(elems);
            rc = plan->download_full(tmp.data(), false, err);
            for (size_t i = 0; rc == 0 && i < elems; i++) (*result)->matrix[i] = static_cast<TReal>(tmp[i]);
        } else {
            std::vector<float> tmp(elems);
            rc = plan->download_full(tmp.data(), false, err);
            for (size_t i = 0; rc == 0 && i < elems; i++) (*result)->matrix[i] = static_cast<TReal>(tmp[i]);
        }
    } else if (rc == 0) {
        // a fresh pageable result is faulted in while the device computes and
        // page-locked for the copy; a pooled one is page-locked already
        const bool fresh = allocated && (*result)->flags == 0;
        const size_t bytes = sizeof(TReal) * elems;
        if ((*result)->flags & kPinnedFlag) {
            // page-locked: the copy-out runs alongside the computation
            rc = plan->execute_download((*result)->matrix, false, err);
        } else {
            rc = plan->execute(nullptr);
            if (rc == 0) {
                if (fresh && bytes >= kHugeAlign) prefault((*result)->matrix, bytes);
                rc = plan->download_full((*result)->matrix, fresh, err);
            } else {
                err = "launch failed";
            }
        }
    } else {
        err = "launch failed";
    }
    timer.step("stripes_to_matrix");
    if (rc) {
        report("one_off_matrix", err);
        if (allocated) destroy_full<TMat, TReal>(result);
        return static_cast<ComputeStatus>(rc);
    }
    return okay;
}

// skbio_biom_subsampled (src/biom_subsampled.cpp:287-353) once, drawn on the
// device with the current seed (the replicate-batch calls' replicate 0).
ComputeStatus rarefied_once(const ssu::Table &table, unsigned int depth, bool with_replacement, ssu::Table &out) {
    std::string err;
    if (!select_device(err)) {
        report("device", err);
        return output_error;
    }
    std::vector<ssu::Table> reps;
    if (ssu::rarefy_on_device(table, depth, with_replacement, g_seed.load(), 1, reps, err)) {
        report("subsample", err);
        return output_error;
    }
    out = std::move(reps[0]);
    return out.n_samples == 0 || out.n_obs == 0 ? table_empty : okay;
}

// one_off_matrix_v3_T (src/api.cpp:700-717): optional rarefaction first.
template <class TReal, class TMat>
ComputeStatus full_matrix_v3(const support_biom_t *table_data, const support_bptree_t *tree_data, const Request &r,
                             bool want_fp64, unsigned int subsample_depth, bool with_replacement, const char *mmap_dir,
                             TMat **result) {
    bool fp64 = false;
    ComputeStatus st = is_fp64_method(r.method, fp64);
    if (st != okay) return st;
    if (fp64 != want_fp64) return invalid_method;
    if (!table_data || table_data->n_samples <= 0 || table_data->n_obs <= 0) return table_empty;
    if (!tree_data) return tree_missing;
    StepTimer timer("one_off_matrix_v3");
    ssu::Table table;
    ssu::BPTree tree;
    read_inputs(table_data, tree_data, table, tree);
    timer.step("read_table_tree");
    st = validate(table, tree);
    timer.step("validate");
    if (st != okay) return st;
    if (subsample_depth > 0) {
        ssu::Table sub;
        st = rarefied_once(table, subsample_depth, with_replacement, sub);
        if (st != okay) return st;
        return full_matrix<TReal, TMat>(sub, tree, r, mmap_dir, result);
    }
    return full_matrix<TReal, TMat>(table, tree, r, mmap_dir, result);
}

// ------------------------------------------------------------------ batches

// Host side of a batch: per-table validation, the tree sheared to the union
// of the tables' observations and collapsed, each table's rows of the union
// observations, and each table's own embedded node count.
struct BatchHost {
    ssu::FlatTree flat;
    ssu::TableSet set;
};

ComputeStatus batch_prepare(const std::vector<const ssu::Table *> &tables, const ssu::BPTree &tree, bool bypass,
                            BatchHost &bh) {
    if (tables.empty() || tables.size() > 65535) return table_empty;
    if (tree.malformed) {
        report("tree", "parentheses do not pair up");
        return tree_missing;
    }
    size_t total_obs = 0;
    for (const ssu::Table *t : tables) {
        if (t->n_samples == 0 || t->n_obs == 0) return table_empty;
        if (t->malformed) {
            report("table", "malformed CSR (offsets or sample positions out of range)");
            return table_missing;
        }
        total_obs += t->n_obs;
    }
    ssu::NameMap uni(total_obs);
    std::vector<std::vector<uint32_t>> uid(tables.size());
    uint32_t n_union = 0;
    for (size_t t = 0; t < tables.size(); t++) {
        const ssu::Table &tb = *tables[t];
        uid[t].resize(tb.n_obs);
        for (uint32_t i = 0; i < tb.n_obs; i++) {
            int64_t u = uni.find(tb.obs_ids[i]);
            if (u < 0) {
                uni.set(tb.obs_ids[i], n_union);
                u = n_union++;
            }
            uid[t][i] = static_cast<uint32_t>(u);
        }
    }
    // VALIDATE_TREE_TABLE (src/api.cpp:94-100) for every table: each of its
    // observations names a tip
    std::vector<uint8_t> in_tree(n_union, 0);
    for (uint32_t i = 0; i + 1 < tree.size(); i++) {
        if (!tree.leaf(i)) continue;
        const int64_t u = uni.find(tree.name[i]);
        if (u >= 0) in_tree[u] = 1;
    }
    for (size_t t = 0; t < tables.size(); t++)
        for (uint32_t u : uid[t])
            if (!in_tree[u]) return table_and_tree_do_not_overlap;
    bh.flat = ssu::flatten(tree.shear_to(uni, n_union, nullptr).collapse(), bypass);
    bh.set.tables = tables;
    bh.set.obs_row.assign(tables.size(), std::vector<int32_t>(n_union, -1));
    bh.set.embedded.resize(tables.size());
    if (bypass) bh.set.row_active.resize(tables.size());
    for (size_t t = 0; t < tables.size(); t++) {
        for (uint32_t i = 0; i < tables[t]->n_obs; i++) bh.set.obs_row[t][uid[t][i]] = static_cast<int32_t>(i);
        bh.set.embedded[t] =
            ssu::table_embedded(bh.flat, bh.set.obs_row[t], bypass, bypass ? &bh.set.row_active[t] : nullptr);
    }
    return okay;
}

ComputeStatus batch_plan(const std::vector<const ssu::Table *> &tables, const ssu::BPTree &tree, const Request &r,
                         const ssu::BatchOptions &opts, std::unique_ptr<ssu::Plan> &plan, StepTimer &timer) {
    ssu::MethodSpec spec;
    if (!ssu::parse_method(r.method, spec.method, spec.fp64)) return unknown_method;
    spec.vaw = r.vaw;
    spec.alpha = r.alpha;
    spec.bypass_tips = r.bypass;
    spec.normalize = r.normalize;
    unweighted_mode(spec);
    std::string err;
    if (!select_device(err)) {
        report("device", err);
        return output_error;
    }
    BatchHost bh;
    ComputeStatus st = batch_prepare(tables, tree, r.bypass, bh);
    if (st != okay) return st;
    timer.step("sync_tree_tables");
    ssu::Plan *p = nullptr;
    const int rc = ssu::Plan::create_batch(bh.set, bh.flat, spec, opts, nullptr, &p, err);
    if (rc) {
        report("batch plan", err);
        return static_cast<ComputeStatus>(rc);
    }
    plan.reset(p);
    // the caller's CSR arrays are read by the uploads queued above
    if (plan->synchronize()) return output_error;
    timer.step("upload");
    return okay;
}

template <class TReal, class TMat>
ComputeStatus batch_matrices(const std::vector<const ssu::Table *> &tables, const ssu::BPTree &tree,
                             const Request &r, TMat **results) {
    StepTimer timer("one_off_batch_inmem");
    std::unique_ptr<ssu::Plan> plan;
    ComputeStatus st = batch_plan(tables, tree, r, ssu::BatchOptions{}, plan, timer);
    if (st != okay) return st;
    const size_t T = tables.size();
    for (size_t t = 0; t < T; t++) results[t] = nullptr;
    auto release = [&] {
        for (size_t t = 0; t < T; t++) destroy_full<TMat, TReal>(&results[t]);
    };
    for (size_t t = 0; t < T; t++)
        if (!alloc_full<TReal, TMat>(results[t], tables[t]->sample_ids, nullptr)) {
            release();
            report("one_off_batch", "result allocation failed");
            return output_error;
        }
    std::string err;
    int rc = plan->execute(nullptr);
    if (rc == 0) {
        for (size_t t = 0; t < T; t++) {  // overlaps the device work
            const size_t bytes = sizeof(TReal) * static_cast<size_t>(tables[t]->n_samples) * tables[t]->n_samples;
            if (results[t]->flags == 0 && bytes >= kHugeAlign) prefault(results[t]->matrix, bytes);
        }
        for (size_t t = 0; t < T && rc == 0; t++) {
            const uint64_t n = tables[t]->n_samples;
            rc = plan->download_range(plan->table_offset(static_cast<uint32_t>(t)), n * n, results[t]->matrix,
                                      results[t]->flags == 0, err);
        }
    } else {
        err = "launch failed";
    }
    timer.step("batch_to_matrices");
    if (rc) {
        report("one_off_batch", err);
        release();
        return static_cast<ComputeStatus>(rc);
    }
    return okay;
}

template <class TReal, class TMat>
ComputeStatus batch_v3(const support_biom_t *const *tables_data, unsigned int n_tables,
                       const support_bptree_t *tree_data, const Request &r, bool want_fp64, TMat **results) {
    bool fp64 = false;
    ComputeStatus st = is_fp64_method(r.method, fp64);
    if (st != okay) return st;
    if (fp64 != want_fp64) return invalid_method;
    if (!tables_data || n_tables == 0 || !results) return table_empty;
    if (!tree_data) return tree_missing;
    std::vector<ssu::Table> tables;
    tables.reserve(n_tables);
    for (unsigned int t = 0; t < n_tables; t++) {
        const support_biom_t *td = tables_data[t];
        if (!td || td->n_samples <= 0 || td->n_obs <= 0) return table_empty;
        tables.push_back(table_from(td));
    }
    std::vector<const ssu::Table *> ptrs;
    for (const ssu::Table &t : tables) ptrs.push_back(&t);
    return batch_matrices<TReal, TMat>(ptrs, tree_from(tree_data), r, results);
}

template <class TReal, class TMat>
ComputeStatus subsample_batch_v3(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                 const Request &r, bool want_fp64, unsigned int n_subsamples, unsigned int depth,
                                 bool with_replacement, TMat **results) {
    bool fp64 = false;
    ComputeStatus st = is_fp64_method(r.method, fp64);
    if (st != okay) return st;
    if (fp64 != want_fp64) return invalid_method;
    if (!table_data || table_data->n_samples <= 0 || table_data->n_obs <= 0 || n_subsamples == 0 || depth == 0 ||
        !results)
        return table_empty;
    if (!tree_data) return tree_missing;
    ssu::Table table;
    ssu::BPTree tree;
    read_inputs(table_data, tree_data, table, tree);
    st = validate(table, tree);
    if (st != okay) return st;
    // The replicates are drawn on the device (ssu_rarefy.cu): replicate i's
    // draws depend only on the seed, i and the sample.
    std::string err;
    if (!select_device(err)) {
        report("device", err);
        return output_error;
    }
    std::vector<ssu::Table> reps;
    if (ssu::rarefy_on_device(table, depth, with_replacement, g_seed.load(), n_subsamples, reps, err)) {
        report("subsample", err);
        return output_error;
    }
    for (const ssu::Table &t : reps)
        if (t.n_samples == 0 || t.n_obs == 0) return table_empty;
    std::vector<const ssu::Table *> ptrs;
    for (const ssu::Table &t : reps) ptrs.push_back(&t);
    return batch_matrices<TReal, TMat>(ptrs, tree, r, results);
}

ComputeStatus condensed(const ssu::Table &table, const ssu::BPTree &tree, const Request &r, mat_t **result) {
    StepTimer timer("one_off");
    std::unique_ptr<ssu::Plan> plan;
    ComputeStatus st = make_plan(table, tree, r, plan, timer);
    if (st != okay) return st;
    const uint64_t n = table.n_samples;
    mat_t *m = static_cast<mat_t *>(std::malloc(sizeof(mat_t)));
    m->n_samples = table.n_samples;
    m->cf_size = static_cast<unsigned int>(n * (n - 1) / 2);
    m->is_upper_triangle = true;
    m->condensed_form = static_cast<double *>(std::malloc(sizeof(double) * (m->cf_size ? m->cf_size : 1)));
    m->sample_ids = copy_ids(table.sample_ids);
    std::string err;
    const int rc = plan->run_condensed(m->condensed_form, err);
    timer.step("stripes_to_condensed_form");
    if (rc) {
        report("one_off", err);
        destroy_mat(&m);
        return static_cast<ComputeStatus>(rc);
    }
    *result = m;
    return okay;
}

ComputeStatus partial_stripes(const ssu::Table &table, const ssu::BPTree &tree, const Request &r,
                              unsigned int stripe_start, unsigned int stripe_stop, partial_mat_t **result) {
    StepTimer timer("partial");
    const uint32_t n_stripes = (table.n_samples + 1) / 2;
    if (stripe_stop <= stripe_start) stripe_stop = n_stripes;  // as set_tasks, src/api.cpp:455-456
    if (stripe_stop > n_stripes || stripe_start >= n_stripes) {
        report("partial", "stopping stripe is out of bounds, max " + std::to_string(n_stripes));
        return output_error;
    }
    std::unique_ptr<ssu::Plan> plan;
    ComputeStatus st = make_plan(table, tree, r, plan, timer);
    if (st != okay) return st;
    partial_mat_t *p = static_cast<partial_mat_t *>(std::malloc(sizeof(partial_mat_t)));
    p->n_samples = table.n_samples;
    p->sample_ids = copy_ids(table.sample_ids);
    p->stripe_start = stripe_start;
    p->stripe_stop = stripe_stop;
    p->stripe_total = n_stripes;
    p->is_upper_triangle = true;
    p->stripes = static_cast<double **>(std::malloc(sizeof(double *) * (stripe_stop - stripe_start)));
    for (uint32_t s = 0; s < stripe_stop - stripe_start; s++)
        p->stripes[s] = static_cast<double *>(std::calloc(table.n_samples, sizeof(double)));
    std::string err;
    const int rc = plan->run_stripes(stripe_start, stripe_stop, p->stripes, err);
    timer.step("process_stripes");
    if (rc) {
        report("partial", err);
        destroy_partial_mat(&p);
        return static_cast<ComputeStatus>(rc);
    }
    *result = p;
    return okay;
}

ComputeStatus inmem_common(const support_biom_t *table_data, const support_bptree_t *tree_data, ssu::Table &table,
                           ssu::BPTree &tree) {
    if (!table_data || table_data->n_samples <= 0 || table_data->n_obs <= 0) return table_empty;
    if (!tree_data) return tree_missing;
    read_inputs(table_data, tree_data, table, tree);
    return validate(table, tree);
}

// faith_pd_one_off (src/api.cpp:569-603) over an in-memory table.
ComputeStatus faith_pd(const ssu::Table &table, const ssu::BPTree &tree, r_vec **result) {
    StepTimer timer("faith_pd");
    ssu::Table nz = table.filtered(1.0);
    r_vec *rv = static_cast<r_vec *>(std::malloc(sizeof(r_vec)));
    if (nz.n_samples == 0 || nz.n_obs == 0) {
        std::fprintf(stderr, "WARNING: All samples had zero counts. Forcing zero result.\n");
        rv->n_samples = table.n_samples;
        rv->values = static_cast<double *>(std::calloc(table.n_samples ? table.n_samples : 1, sizeof(double)));
        rv->sample_ids = copy_ids(table.sample_ids);
        *result = rv;
        return okay;
    }
    if (nz.n_samples != table.n_samples || nz.n_obs != table.n_obs)
        std::fprintf(stderr, "WARNING: Some samples had zero counts and were filtered out.\n");
    rv->n_samples = nz.n_samples;
    rv->values = static_cast<double *>(std::calloc(nz.n_samples, sizeof(double)));
    rv->sample_ids = copy_ids(nz.sample_ids);
    std::string err;
    if (!select_device(err)) {
        report("faith_pd", err);
        destroy_results_vec(&rv);
        return output_error;
    }
    const ssu::FlatTree flat = sync_tree(nz, tree, false);
    timer.step("sync_tree_table");
    ssu::Plan *p = nullptr;
    int rc = ssu::Plan::create_faith(nz, flat, nullptr, &p, err);
    if (!rc) {
        std::unique_ptr<ssu::Plan> plan(p);
        rc = plan->run_faith(rv->values, err);
    }
    timer.step("faith_pd");
    if (rc) {
        report("faith_pd", err);
        destroy_results_vec(&rv);
        return static_cast<ComputeStatus>(rc);
    }
    *result = rv;
    return okay;
}

bool file_exists(const char *path) {
    if (!path) return false;
    std::ifstream f(path);
    return f.good();
}

bool read_text(const char *path, std::string &out) {
    std::ifstream f(path);
    if (!f.good()) return false;
    std::stringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

// CHECK_FILE + PARSE_TREE_TABLE (src/api.cpp:115-121, 127-135): the table
// file read as BIOM-HDF5 (ssu_biom.cpp), the tree file as newick.
ComputeStatus load_table_file(const char *biom_filename, ssu::Table &table) {
    std::string err;
    if (!ssu::read_biom_hdf5(biom_filename, table, err)) {
        report("table", std::string(biom_filename) + ": " + err);
        return table_missing;
    }
    return okay;
}

ComputeStatus load_tree_file(const char *tree_filename, ssu::BPTree &tree) {
    std::string text;
    if (!read_text(tree_filename, text) || !ssu::BPTree::from_newick(text, tree)) return tree_missing;
    return okay;
}

struct OpaqueTree {
    ssu::BPTree tree;
};

// Both files (or the table file and a pre-parsed tree), read and validated:
// table_missing / tree_missing for missing or unreadable files, then
// VALIDATE_TREE_TABLE's statuses.
ComputeStatus load_files(const char *biom_filename, const char *tree_filename, ssu::Table &table,
                         ssu::BPTree &tree) {
    if (!file_exists(biom_filename)) return table_missing;
    if (!file_exists(tree_filename)) return tree_missing;
    ComputeStatus st = load_tree_file(tree_filename, tree);
    if (st != okay) return st;
    st = load_table_file(biom_filename, table);
    if (st != okay) return st;
    return validate(table, tree);
}

ComputeStatus load_files_wtree(const char *biom_filename, const opaque_bptree_t *tree_data, ssu::Table &table,
                               ssu::BPTree &tree) {
    if (!tree_data) return tree_missing;
    if (!file_exists(biom_filename)) return table_missing;
    tree = reinterpret_cast<const OpaqueTree *>(tree_data)->tree;
    const ComputeStatus st = load_table_file(biom_filename, table);
    if (st != okay) return st;
    return validate(table, tree);
}

// merge_partial_to_matrix_T (src/api.cpp:2454-2478): the partials checked,
// the result allocated (malloc, or a file under mmap_dir), every stripe read
// (from memory, or its file when only the header was read), scattered to
// both triangles and released; stripes are independent, so they go to host
// threads.
template <class TReal, class TMat>
MergeStatus merge_partials(partial_dyn_mat_t **mats, int n, const char *mmap_dir, TMat **result) {
    if (!result) return incomplete_stripe_set;
    if (mmap_dir && !mmap_dir[0]) mmap_dir = nullptr;
    const MergeStatus err = ssu::partial_check(mats, n, false);
    if (err != merge_okay) return err;
    const uint32_t ns = mats[0]->n_samples;
    std::vector<std::string_view> ids(ns);
    for (uint32_t j = 0; j < ns; j++) ids[j] = mats[0]->sample_ids[j];
    struct Job {
        partial_dyn_mat_t *p;
        uint32_t idx;
        uint64_t off;
    };
    std::vector<Job> jobs;
    for (int i = 0; i < n; i++) {
        partial_dyn_mat_t *p = mats[i];
        const uint32_t cnt = p->stripe_stop - p->stripe_start;
        bool all_in_memory = true;
        for (uint32_t s = 0; s < cnt; s++) all_in_memory = all_in_memory && p->stripes && p->stripes[s];
        std::vector<uint64_t> offs(cnt, 0);
        if (!all_in_memory) {
            if (!p->filename || !p->offsets ||
                ssu::partial_stripe_offsets(p->filename, p->offsets[0], cnt, offs) != read_okay)
                return incomplete_stripe_set;
        }
        for (uint32_t s = 0; s < cnt; s++) jobs.push_back(Job{p, s, offs[s]});
    }
    *result = nullptr;
    if (!alloc_full<TReal, TMat>(*result, ids, mmap_dir)) {
        destroy_full<TMat, TReal>(result);
        return incomplete_stripe_set;
    }
    TReal *m = (*result)->matrix;
    std::atomic<bool> bad{false};
    try {
        parallel_for(static_cast<unsigned>(jobs.size()), host_threads(16), [&](unsigned j) {
            const Job &jb = jobs[j];
            double *owned = jb.p->stripes ? jb.p->stripes[jb.idx] : nullptr;
            const double *stripe = owned;
            std::vector<double> local;
            if (!stripe) {
                local.resize(ns);
                if (ssu::partial_read_stripe_at(jb.p->filename, jb.off, ns, local.data()) != read_okay) {
                    bad = true;
                    return;
                }
                stripe = local.data();
            }
            const uint64_t s = jb.p->stripe_start + jb.idx;
            for (uint64_t k = 0; k < ns; k++) {
                const uint64_t l = (k + s + 1) % ns;
                m[k * ns + l] = static_cast<TReal>(stripe[k]);
                m[l * ns + k] = static_cast<TReal>(stripe[k]);
            }
            // a stripe held in memory is released once used (the reference's
            // PartialStripes::release_stripe, src/api.cpp:2441-2450)
            if (owned) {
                std::free(owned);
                jb.p->stripes[jb.idx] = nullptr;
            }
        });
    } catch (const std::exception &) {
        bad = true;
    }
    if (bad) {
        destroy_full<TMat, TReal>(result);
        return incomplete_stripe_set;
    }
    for (uint64_t k = 0; k < ns; k++) m[k * ns + k] = 0;
    return merge_okay;
}

}  // namespace

// =================================================== reference-compatible

extern "C" {

void ssu_set_random_seed(unsigned int new_seed) { g_seed.store(new_seed); }

IOStatus read_bptree_opaque(const char *tree_filename, opaque_bptree_t **tree_data) {
    if (tree_data == nullptr) return unexpected_end;
    std::string text;
    if (!read_text(tree_filename, text)) return open_error;
    OpaqueTree *t = new OpaqueTree();
    if (!ssu::BPTree::from_newick(text, t->tree)) {
        delete t;
        return unexpected_end;
    }
    *tree_data = reinterpret_cast<opaque_bptree_t *>(t);
    return read_okay;
}

void load_bptree_opaque(const char *newick, opaque_bptree_t **tree_data) {
    OpaqueTree *t = new OpaqueTree();
    if (!newick || !ssu::BPTree::from_newick(newick, t->tree)) t->tree = ssu::BPTree();
    *tree_data = reinterpret_cast<opaque_bptree_t *>(t);
}

void convert_bptree_opaque(const support_bptree_t *in_tree, opaque_bptree_t **tree_data) {
    OpaqueTree *t = new OpaqueTree();
    t->tree = tree_from(in_tree, true);
    *tree_data = reinterpret_cast<opaque_bptree_t *>(t);
}

void destroy_bptree_opaque(opaque_bptree_t **tree_data) {
    if (tree_data && *tree_data) {
        delete reinterpret_cast<OpaqueTree *>(*tree_data);
        *tree_data = nullptr;
    }
}

int get_bptree_opaque_els(opaque_bptree_t *tree_data) {
    if (!tree_data) return 0;
    return static_cast<int>(reinterpret_cast<OpaqueTree *>(tree_data)->tree.tip_names().size());
}

void destroy_mat(mat_t **result) {
    if (!result || !*result) return;
    mat_t *m = *result;
    for (unsigned int i = 0; i < m->n_samples; i++) std::free(m->sample_ids[i]);
    std::free(m->sample_ids);
    std::free(m->condensed_form);
    std::free(m);
    *result = nullptr;
}

void destroy_mat_full_fp64(mat_full_fp64_t **result) { destroy_full<mat_full_fp64_t, double>(result); }
void destroy_mat_full_fp32(mat_full_fp32_t **result) { destroy_full<mat_full_fp32_t, float>(result); }

void destroy_partial_mat(partial_mat_t **result) {
    if (!result || !*result) return;
    partial_mat_t *p = *result;
    if (p->sample_ids) {
        for (uint32_t i = 0; i < p->n_samples; i++) std::free(p->sample_ids[i]);
        std::free(p->sample_ids);
    }
    if (p->stripes) {
        for (uint32_t s = 0; s < p->stripe_stop - p->stripe_start; s++) std::free(p->stripes[s]);
        std::free(p->stripes);
    }
    std::free(p);
    *result = nullptr;
}

void destroy_partial_dyn_mat(partial_dyn_mat_t **result) {
    if (!result || !*result) return;
    partial_dyn_mat_t *p = *result;
    if (p->sample_ids) {
        for (uint32_t i = 0; i < p->n_samples; i++) std::free(p->sample_ids[i]);
        std::free(p->sample_ids);
    }
    if (p->stripes) {
        for (uint32_t s = 0; s < p->stripe_stop - p->stripe_start; s++) std::free(p->stripes[s]);
        std::free(p->stripes);
    }
    std::free(p->offsets);
    std::free(p->filename);
    std::free(p);
    *result = nullptr;
}

MergeStatus merge_partial_to_matrix(partial_dyn_mat_t **partial_mats, int n_partials, mat_full_fp64_t **result) {
    return merge_partials<double, mat_full_fp64_t>(partial_mats, n_partials, nullptr, result);
}

MergeStatus merge_partial_to_matrix_fp32(partial_dyn_mat_t **partial_mats, int n_partials,
                                         mat_full_fp32_t **result) {
    return merge_partials<float, mat_full_fp32_t>(partial_mats, n_partials, nullptr, result);
}

MergeStatus merge_partial_to_mmap_matrix(partial_dyn_mat_t **partial_mats, int n_partials, const char *mmap_dir,
                                         mat_full_fp64_t **result) {
    return merge_partials<double, mat_full_fp64_t>(partial_mats, n_partials, mmap_dir, result);
}

MergeStatus merge_partial_to_mmap_matrix_fp32(partial_dyn_mat_t **partial_mats, int n_partials,
                                              const char *mmap_dir, mat_full_fp32_t **result) {
    return merge_partials<float, mat_full_fp32_t>(partial_mats, n_partials, mmap_dir, result);
}

void destroy_results_vec(r_vec **result) {
    if (!result || !*result) return;
    r_vec *r = *result;
    for (unsigned int i = 0; i < r->n_samples; i++) std::free(r->sample_ids[i]);
    std::free(r->sample_ids);
    std::free(r->values);
    std::free(r);
    *result = nullptr;
}

ComputeStatus one_off_matrix_inmem_v3(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                      const char *unifrac_method, bool variance_adjust, double alpha,
                                      bool bypass_tips, bool normalize_sample_counts, unsigned int,
                                      unsigned int subsample_depth, bool subsample_with_replacement,
                                      const char *mmap_dir, mat_full_fp64_t **result) {
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return full_matrix_v3<double, mat_full_fp64_t>(table_data, tree_data, r, true, subsample_depth,
                                                    subsample_with_replacement, mmap_dir, result);
}

ComputeStatus one_off_matrix_inmem_v2(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                      const char *unifrac_method, bool variance_adjust, double alpha,
                                      bool bypass_tips, unsigned int n_substeps, unsigned int subsample_depth,
                                      bool subsample_with_replacement, const char *mmap_dir,
                                      mat_full_fp64_t **result) {
    return one_off_matrix_inmem_v3(table_data, tree_data, unifrac_method, variance_adjust, alpha, bypass_tips, true,
                                   n_substeps, subsample_depth, subsample_with_replacement, mmap_dir, result);
}

ComputeStatus one_off_inmem(const support_biom_t *table_data, const support_bptree_t *tree_data,
                            const char *unifrac_method, bool variance_adjust, double alpha, bool bypass_tips,
                            unsigned int n_substeps, mat_full_fp64_t **result) {
    return one_off_matrix_inmem_v3(table_data, tree_data, unifrac_method, variance_adjust, alpha, bypass_tips, true,
                                   n_substeps, 0, false, nullptr, result);
}

ComputeStatus one_off_matrix_inmem_fp32_v3(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                           const char *unifrac_method, bool variance_adjust, double alpha,
                                           bool bypass_tips, bool normalize_sample_counts, unsigned int,
                                           unsigned int subsample_depth, bool subsample_with_replacement,
                                           const char *mmap_dir, mat_full_fp32_t **result) {
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return full_matrix_v3<float, mat_full_fp32_t>(table_data, tree_data, r, false, subsample_depth,
                                                   subsample_with_replacement, mmap_dir, result);
}

ComputeStatus one_off_matrix_inmem_fp32_v2(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                           const char *unifrac_method, bool variance_adjust, double alpha,
                                           bool bypass_tips, unsigned int n_substeps, unsigned int subsample_depth,
                                           bool subsample_with_replacement, const char *mmap_dir,
                                           mat_full_fp32_t **result) {
    return one_off_matrix_inmem_fp32_v3(table_data, tree_data, unifrac_method, variance_adjust, alpha, bypass_tips,
                                        true, n_substeps, subsample_depth, subsample_with_replacement, mmap_dir,
                                        result);
}

ComputeStatus one_off_inmem_fp32(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                 const char *unifrac_method, bool variance_adjust, double alpha, bool bypass_tips,
                                 unsigned int n_substeps, mat_full_fp32_t **result) {
    return one_off_matrix_inmem_fp32_v3(table_data, tree_data, unifrac_method, variance_adjust, alpha, bypass_tips,
                                        true, n_substeps, 0, false, nullptr, result);
}

// one_dense_pair (src/api.cpp:729-766)
static ComputeStatus dense_pair(unsigned int n_obs, const char **obs_ids, const double *sample1,
                                const double *sample2, const ssu::BPTree &tree, const char *unifrac_method,
                                bool variance_adjust, double alpha, bool bypass_tips, bool normalize,
                                double *result) {
    bool fp64 = false;
    ComputeStatus st = is_fp64_method(unifrac_method, fp64);
    if (st != okay) return st;
    ssu::Table table = ssu::Table::dense_pair(n_obs, obs_ids, sample1, sample2);
    st = validate(table, tree);
    if (st != okay) return st;
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize};
    if (fp64) {
        mat_full_fp64_t *m = nullptr;
        st = full_matrix<double, mat_full_fp64_t>(table, tree, r, nullptr, &m);
        if (st == okay) {
            *result = m->matrix[1];
            destroy_mat_full_fp64(&m);
        }
    } else {
        mat_full_fp32_t *m = nullptr;
        st = full_matrix<float, mat_full_fp32_t>(table, tree, r, nullptr, &m);
        if (st == okay) {
            *result = m->matrix[1];
            destroy_mat_full_fp32(&m);
        }
    }
    return st;
}

ComputeStatus one_dense_pair_v3t(unsigned int n_obs, const char **obs_ids, const double *sample1,
                                 const double *sample2, const opaque_bptree_t *tree_data, const char *unifrac_method,
                                 bool variance_adjust, double alpha, bool bypass_tips, bool normalize_sample_counts,
                                 double *result) {
    if (!tree_data) return tree_missing;
    const ssu::BPTree &tree = reinterpret_cast<const OpaqueTree *>(tree_data)->tree;
    return dense_pair(n_obs, obs_ids, sample1, sample2, tree, unifrac_method, variance_adjust, alpha, bypass_tips,
                      normalize_sample_counts, result);
}

ComputeStatus one_dense_pair_v3(unsigned int n_obs, const char **obs_ids, const double *sample1,
                                const double *sample2, const support_bptree_t *tree_data, const char *unifrac_method,
                                bool variance_adjust, double alpha, bool bypass_tips, bool normalize_sample_counts,
                                double *result) {
    if (!tree_data) return tree_missing;
    const ssu::BPTree tree = tree_from(tree_data);
    return dense_pair(n_obs, obs_ids, sample1, sample2, tree, unifrac_method, variance_adjust, alpha, bypass_tips,
                      normalize_sample_counts, result);
}

ComputeStatus one_dense_pair_v2t(unsigned int n_obs, const char **obs_ids, const double *sample1,
                                 const double *sample2, const opaque_bptree_t *tree_data, const char *unifrac_method,
                                 bool variance_adjust, double alpha, bool bypass_tips, double *result) {
    return one_dense_pair_v3t(n_obs, obs_ids, sample1, sample2, tree_data, unifrac_method, variance_adjust, alpha,
                              bypass_tips, true, result);
}

ComputeStatus one_dense_pair_v2(unsigned int n_obs, const char **obs_ids, const double *sample1,
                                const double *sample2, const support_bptree_t *tree_data, const char *unifrac_method,
                                bool variance_adjust, double alpha, bool bypass_tips, double *result) {
    return one_dense_pair_v3(n_obs, obs_ids, sample1, sample2, tree_data, unifrac_method, variance_adjust, alpha,
                             bypass_tips, true, result);
}

ComputeStatus one_off_v3(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                         bool variance_adjust, double alpha, bool bypass_tips, bool normalize_sample_counts,
                         unsigned int, mat_t **result) {
    ssu::Table table;
    ssu::BPTree tree;
    const ComputeStatus st = load_files(biom_filename, tree_filename, table, tree);
    if (st != okay) return st;
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return condensed(table, tree, r, result);
}

ComputeStatus one_off_wtree_v3(const char *biom_filename, const opaque_bptree_t *tree_data,
                               const char *unifrac_method, bool variance_adjust, double alpha, bool bypass_tips,
                               bool normalize_sample_counts, unsigned int, mat_t **result) {
    ssu::Table table;
    ssu::BPTree tree;
    const ComputeStatus st = load_files_wtree(biom_filename, tree_data, table, tree);
    if (st != okay) return st;
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return condensed(table, tree, r, result);
}

ComputeStatus one_off(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                      bool variance_adjust, double alpha, bool bypass_tips, unsigned int n_substeps, mat_t **result) {
    return one_off_v3(biom_filename, tree_filename, unifrac_method, variance_adjust, alpha, bypass_tips, true,
                      n_substeps, result);
}

ComputeStatus one_off_wtree(const char *biom_filename, const opaque_bptree_t *tree_data, const char *unifrac_method,
                            bool variance_adjust, double alpha, bool bypass_tips, unsigned int n_substeps,
                            mat_t **result) {
    return one_off_wtree_v3(biom_filename, tree_data, unifrac_method, variance_adjust, alpha, bypass_tips, true,
                            n_substeps, result);
}

}  // extern "C"

namespace {

// one_off_matrix_v3_T over a loaded table (src/api.cpp:700-717): optional
// rarefaction, the method's precision for the arithmetic, TReal for the result.
template <class TReal, class TMat>
ComputeStatus file_matrix(ComputeStatus loaded, const ssu::Table &table, const ssu::BPTree &tree, const Request &r,
                          unsigned int subsample_depth, bool with_replacement, const char *mmap_dir, TMat **result) {
    if (loaded != okay) return loaded;
    if (!result) return output_error;
    if (mmap_dir && mmap_dir[0] == 0) mmap_dir = nullptr;
    if (subsample_depth > 0) {
        ssu::Table sub;
        const ComputeStatus st = rarefied_once(table, subsample_depth, with_replacement, sub);
        if (st != okay) return st;
        return full_matrix<TReal, TMat>(sub, tree, r, mmap_dir, result);
    }
    return full_matrix<TReal, TMat>(table, tree, r, mmap_dir, result);
}

}  // namespace

extern "C" {

ComputeStatus one_off_matrix_v3(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                                bool variance_adjust, double alpha, bool bypass_tips, bool normalize_sample_counts,
                                unsigned int, unsigned int subsample_depth, bool subsample_with_replacement,
                                const char *mmap_dir, mat_full_fp64_t **result) {
    ssu::Table table;
    ssu::BPTree tree;
    const ComputeStatus st = load_files(biom_filename, tree_filename, table, tree);
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return file_matrix<double, mat_full_fp64_t>(st, table, tree, r, subsample_depth, subsample_with_replacement,
                                                mmap_dir, result);
}

ComputeStatus one_off_matrix_fp32_v3(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                                     bool variance_adjust, double alpha, bool bypass_tips,
                                     bool normalize_sample_counts, unsigned int, unsigned int subsample_depth,
                                     bool subsample_with_replacement, const char *mmap_dir,
                                     mat_full_fp32_t **result) {
    ssu::Table table;
    ssu::BPTree tree;
    const ComputeStatus st = load_files(biom_filename, tree_filename, table, tree);
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return file_matrix<float, mat_full_fp32_t>(st, table, tree, r, subsample_depth, subsample_with_replacement,
                                               mmap_dir, result);
}

ComputeStatus one_off_matrix_v3t(const char *biom_filename, const opaque_bptree_t *tree_data,
                                 const char *unifrac_method, bool variance_adjust, double alpha, bool bypass_tips,
                                 bool normalize_sample_counts, unsigned int, unsigned int subsample_depth,
                                 bool subsample_with_replacement, const char *mmap_dir, mat_full_fp64_t **result) {
    ssu::Table table;
    ssu::BPTree tree;
    const ComputeStatus st = load_files_wtree(biom_filename, tree_data, table, tree);
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return file_matrix<double, mat_full_fp64_t>(st, table, tree, r, subsample_depth, subsample_with_replacement,
                                                mmap_dir, result);
}

ComputeStatus one_off_matrix_fp32_v3t(const char *biom_filename, const opaque_bptree_t *tree_data,
                                      const char *unifrac_method, bool variance_adjust, double alpha,
                                      bool bypass_tips, bool normalize_sample_counts, unsigned int,
                                      unsigned int subsample_depth, bool subsample_with_replacement,
                                      const char *mmap_dir, mat_full_fp32_t **result) {
    ssu::Table table;
    ssu::BPTree tree;
    const ComputeStatus st = load_files_wtree(biom_filename, tree_data, table, tree);
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return file_matrix<float, mat_full_fp32_t>(st, table, tree, r, subsample_depth, subsample_with_replacement,
                                               mmap_dir, result);
}

ComputeStatus one_off_matrix_v2(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                                bool variance_adjust, double alpha, bool bypass_tips, unsigned int n_substeps,
                                unsigned int subsample_depth, bool subsample_with_replacement, const char *mmap_dir,
                                mat_full_fp64_t **result) {
    return one_off_matrix_v3(biom_filename, tree_filename, unifrac_method, variance_adjust, alpha, bypass_tips, true,
                             n_substeps, subsample_depth, subsample_with_replacement, mmap_dir, result);
}

ComputeStatus one_off_matrix_v2t(const char *biom_filename, const opaque_bptree_t *tree_data,
                                 const char *unifrac_method, bool variance_adjust, double alpha, bool bypass_tips,
                                 unsigned int n_substeps, unsigned int subsample_depth,
                                 bool subsample_with_replacement, const char *mmap_dir, mat_full_fp64_t **result) {
    return one_off_matrix_v3t(biom_filename, tree_data, unifrac_method, variance_adjust, alpha, bypass_tips, true,
                              n_substeps, subsample_depth, subsample_with_replacement, mmap_dir, result);
}

ComputeStatus one_off_matrix(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                             bool variance_adjust, double alpha, bool bypass_tips, unsigned int n_substeps,
                             const char *mmap_dir, mat_full_fp64_t **result) {
    return one_off_matrix_v3(biom_filename, tree_filename, unifrac_method, variance_adjust, alpha, bypass_tips, true,
                             n_substeps, 0, false, mmap_dir, result);
}

ComputeStatus one_off_matrix_fp32_v2(const char *biom_filename, const char *tree_filename,
                                     const char *unifrac_method, bool variance_adjust, double alpha,
                                     bool bypass_tips, unsigned int n_substeps, unsigned int subsample_depth,
                                     bool subsample_with_replacement, const char *mmap_dir,
                                     mat_full_fp32_t **result) {
    return one_off_matrix_fp32_v3(biom_filename, tree_filename, unifrac_method, variance_adjust, alpha, bypass_tips,
                                  true, n_substeps, subsample_depth, subsample_with_replacement, mmap_dir, result);
}

ComputeStatus one_off_matrix_fp32_v2t(const char *biom_filename, const opaque_bptree_t *tree_data,
                                      const char *unifrac_method, bool variance_adjust, double alpha,
                                      bool bypass_tips, unsigned int n_substeps, unsigned int subsample_depth,
                                      bool subsample_with_replacement, const char *mmap_dir,
                                      mat_full_fp32_t **result) {
    return one_off_matrix_fp32_v3t(biom_filename, tree_data, unifrac_method, variance_adjust, alpha, bypass_tips,
                                   true, n_substeps, subsample_depth, subsample_with_replacement, mmap_dir, result);
}

ComputeStatus one_off_matrix_fp32(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                                  bool variance_adjust, double alpha, bool bypass_tips, unsigned int n_substeps,
                                  const char *mmap_dir, mat_full_fp32_t **result) {
    return one_off_matrix_fp32_v3(biom_filename, tree_filename, unifrac_method, variance_adjust, alpha, bypass_tips,
                                  true, n_substeps, 0, false, mmap_dir, result);
}

ComputeStatus faith_pd_one_off(const char *biom_filename, const char *tree_filename, r_vec **result) {
    ssu::Table table;
    ssu::BPTree tree;
    const ComputeStatus st = load_files(biom_filename, tree_filename, table, tree);
    if (st != okay) return st;
    return faith_pd(table, tree, result);
}

ComputeStatus partial_v3(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                         bool variance_adjust, double alpha, bool bypass_tips, bool normalize_sample_counts,
                         unsigned int, unsigned int stripe_start, unsigned int stripe_stop, partial_mat_t **result) {
    if (!file_exists(biom_filename)) return table_missing;
    if (!file_exists(tree_filename)) return tree_missing;
    bool fp64 = false;
    if (is_fp64_method(unifrac_method, fp64) != okay) return unknown_method;  // SET_METHOD before parsing
    ssu::Table table;
    ssu::BPTree tree;
    const ComputeStatus st = load_files(biom_filename, tree_filename, table, tree);
    if (st != okay) return st;
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return partial_stripes(table, tree, r, stripe_start, stripe_stop, result);
}

ComputeStatus partial(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                      bool variance_adjust, double alpha, bool bypass_tips, unsigned int n_substeps,
                      unsigned int stripe_start, unsigned int stripe_stop, partial_mat_t **result) {
    return partial_v3(biom_filename, tree_filename, unifrac_method, variance_adjust, alpha, bypass_tips, true,
                      n_substeps, stripe_start, stripe_stop, result);
}

// ================================================================ extensions

IOStatus ssu_b200_read_biom(const char *biom_filename, support_biom_t **table) {
    if (!table) return unexpected_end;
    *table = nullptr;
    if (!file_exists(biom_filename)) return open_error;
    ssu::Table t;
    std::string err;
    if (!ssu::read_biom_hdf5(biom_filename, t, err)) {
        report("table", std::string(biom_filename) + ": " + err);
        return read_error;
    }
    support_biom_t *b = static_cast<support_biom_t *>(std::calloc(1, sizeof(support_biom_t)));
    b->n_obs = static_cast<int>(t.n_obs);
    b->n_samples = static_cast<int>(t.n_samples);
    b->nnz = static_cast<int>(t.nnz());
    b->obs_ids = copy_ids(t.obs_ids);
    b->sample_ids = copy_ids(t.sample_ids);
    b->indptr = static_cast<uint32_t *>(std::malloc(sizeof(uint32_t) * (t.n_obs + 1)));
    b->indices = static_cast<uint32_t *>(std::malloc(sizeof(uint32_t) * std::max<uint64_t>(t.nnz(), 1)));
    b->data = static_cast<double *>(std::malloc(sizeof(double) * std::max<uint64_t>(t.nnz(), 1)));
    std::memcpy(b->indptr, t.indptr, sizeof(uint32_t) * (t.n_obs + 1));
    std::memcpy(b->indices, t.indices, sizeof(uint32_t) * t.nnz());
    std::memcpy(b->data, t.data, sizeof(double) * t.nnz());
    *table = b;
    return read_okay;
}

ComputeStatus ssu_b200_rarefy_batch(const support_biom_t *table_data, unsigned int n_subsamples,
                                    unsigned int depth, bool with_replacement, support_biom_t **results) {
    if (!table_data || table_data->n_samples <= 0 || table_data->n_obs <= 0 || n_subsamples == 0 || depth == 0 ||
        !results)
        return table_empty;
    ssu::Table table = table_from(table_data);
    if (table.malformed) {
        report("table", "malformed CSR (offsets or sample positions out of range)");
        return table_missing;
    }
    std::string err;
    if (!select_device(err)) {
        report("device", err);
        return output_error;
    }
    std::vector<ssu::Table> reps;
    if (ssu::rarefy_on_device(table, depth, with_replacement, g_seed.load(), n_subsamples, reps, err)) {
        report("subsample", err);
        return output_error;
    }
    for (unsigned int r = 0; r < n_subsamples; r++) {
        const ssu::Table &t = reps[r];
        support_biom_t *b = static_cast<support_biom_t *>(std::calloc(1, sizeof(support_biom_t)));
        b->n_obs = static_cast<int>(t.n_obs);
        b->n_samples = static_cast<int>(t.n_samples);
        b->nnz = static_cast<int>(t.nnz());
        b->obs_ids = copy_ids(t.obs_ids);
        b->sample_ids = copy_ids(t.sample_ids);
        b->indptr = static_cast<uint32_t *>(std::malloc(sizeof(uint32_t) * (t.n_obs + 1)));
        b->indices = static_cast<uint32_t *>(std::malloc(sizeof(uint32_t) * std::max<uint64_t>(t.nnz(), 1)));
        b->data = static_cast<double *>(std::malloc(sizeof(double) * std::max<uint64_t>(t.nnz(), 1)));
        if (t.n_obs) std::memcpy(b->indptr, t.indptr, sizeof(uint32_t) * (t.n_obs + 1));
        else b->indptr[0] = 0;
        if (t.nnz()) {
            std::memcpy(b->indices, t.indices, sizeof(uint32_t) * t.nnz());
            std::memcpy(b->data, t.data, sizeof(double) * t.nnz());
        }
        results[r] = b;
    }
    return okay;
}

void ssu_b200_destroy_biom(support_biom_t **table) {
    if (!table || !*table) return;
    support_biom_t *b = *table;
    for (int i = 0; i < b->n_obs; i++) std::free(b->obs_ids[i]);
    for (int j = 0; j < b->n_samples; j++) std::free(b->sample_ids[j]);
    std::free(b->obs_ids);
    std::free(b->sample_ids);
    std::free(b->indptr);
    std::free(b->indices);
    std::free(b->data);
    std::free(b);
    *table = nullptr;
}

ComputeStatus ssu_b200_one_off_inmem_v3(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                        const char *unifrac_method, bool variance_adjust, double alpha,
                                        bool bypass_tips, bool normalize_sample_counts, unsigned int,
                                        mat_t **result) {
    bool fp64 = false;
    ComputeStatus st = is_fp64_method(unifrac_method, fp64);
    if (st != okay) return st;
    ssu::Table table;
    ssu::BPTree tree;
    st = inmem_common(table_data, tree_data, table, tree);
    if (st != okay) return st;
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return condensed(table, tree, r, result);
}

ComputeStatus ssu_b200_partial_inmem_v3(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                        const char *unifrac_method, bool variance_adjust, double alpha,
                                        bool bypass_tips, bool normalize_sample_counts, unsigned int,
                                        unsigned int stripe_start, unsigned int stripe_stop,
                                        partial_mat_t **result) {
    bool fp64 = false;
    ComputeStatus st = is_fp64_method(unifrac_method, fp64);
    if (st != okay) return st;
    ssu::Table table;
    ssu::BPTree tree;
    st = inmem_common(table_data, tree_data, table, tree);
    if (st != okay) return st;
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return partial_stripes(table, tree, r, stripe_start, stripe_stop, result);
}

ComputeStatus ssu_b200_faith_pd_inmem(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                      r_vec **result) {
    ssu::Table table;
    ssu::BPTree tree;
    const ComputeStatus st = inmem_common(table_data, tree_data, table, tree);
    if (st != okay) return st;
    return faith_pd(table, tree, result);
}

int ssu_b200_shear_collapse(const support_bptree_t *in_tree, const char *const *names, int n_names,
                            int do_collapse, bool *out_structure, double *out_lengths, const char **out_names,
                            int *out_n) {
    if (!in_tree || !out_n) return 1;
    const ssu::BPTree tree = tree_from(in_tree);
    ssu::NameSet keep;
    if (names)
        for (int i = 0; i < n_names; i++) keep.insert(names[i]);
    else
        keep = tree.tip_names();
    const ssu::BPTree sheared = tree.shear(keep);
    const ssu::BPTree r = do_collapse ? sheared.collapse() : sheared;
    // names are handed back as pointers into the input tree's strings
    *out_n = static_cast<int>(r.size());
    for (uint32_t i = 0; i < r.size(); i++) {
        out_structure[i] = r.open[i] != 0;
        out_lengths[i] = r.length[i];
        out_names[i] = r.name[i].data();  // a view into in_tree->names
    }
    return 0;
}

int ssu_b200_tree_arrays(const opaque_bptree_t *tree_data, int capacity, bool *out_structure, double *out_lengths,
                         const char **out_names, int *out_n) {
    if (!tree_data || !out_n) return 1;
    const ssu::BPTree &t = reinterpret_cast<const OpaqueTree *>(tree_data)->tree;
    *out_n = static_cast<int>(t.size());
    if (static_cast<int>(t.size()) > capacity) return 2;
    for (uint32_t i = 0; i < t.size(); i++) {
        out_structure[i] = t.open[i] != 0;
        out_lengths[i] = t.length[i];
        out_names[i] = t.name[i].data();  // owned, NUL-terminated strings
    }
    return 0;
}

struct ssu_b200_plan {
    std::unique_ptr<ssu::Plan> plan;
};

ComputeStatus ssu_b200_plan_create(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                   const char *unifrac_method, bool variance_adjust, double alpha, bool bypass_tips,
                                   bool normalize_sample_counts, ssu_b200_plan_t **plan) {
    bool fp64 = false;
    ComputeStatus st = is_fp64_method(unifrac_method, fp64);
    if (st != okay) return st;
    ssu::Table table;
    ssu::BPTree tree;
    st = inmem_common(table_data, tree_data, table, tree);
    if (st != okay) return st;
    StepTimer timer("plan_create");
    auto *h = new ssu_b200_plan();
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    st = make_plan(table, tree, r, h->plan, timer);
    if (st != okay) {
        delete h;
        return st;
    }
    // the plan owns copies of everything it needs on the device
    if (h->plan->synchronize()) {
        delete h;
        return output_error;
    }
    *plan = h;
    return okay;
}

ComputeStatus ssu_b200_plan_execute(ssu_b200_plan_t *plan, void *stream) {
    if (!plan) return output_error;
    return plan->plan->execute(stream) ? output_error : okay;
}

const void *ssu_b200_plan_device_result(const ssu_b200_plan_t *plan) {
    return plan ? plan->plan->device_result() : nullptr;
}

ComputeStatus ssu_b200_plan_copy_result(ssu_b200_plan_t *plan, void *host_out, void *stream) {
    if (!plan) return output_error;
    return plan->plan->copy_result(host_out, stream) ? output_error : okay;
}

uint64_t ssu_b200_plan_work_units(const ssu_b200_plan_t *plan) { return plan ? plan->plan->work_units() : 0; }
uint32_t ssu_b200_plan_n_samples(const ssu_b200_plan_t *plan) { return plan ? plan->plan->n_samples() : 0; }
uint64_t ssu_b200_plan_n_embedded(const ssu_b200_plan_t *plan) { return plan ? plan->plan->n_embedded() : 0; }
uint32_t ssu_b200_plan_launches(const ssu_b200_plan_t *plan) { return plan ? plan->plan->launches() : 0; }
uint64_t ssu_b200_plan_tensor_flops(const ssu_b200_plan_t *plan) { return plan ? plan->plan->tensor_flops() : 0; }
void ssu_b200_plan_set_timing(ssu_b200_plan_t *plan, int enable) {
    if (plan) plan->plan->set_timing(enable != 0);
}

int ssu_b200_plan_stage_ms(ssu_b200_plan_t *plan, float *embed_ms, float *pair_ms, float *finalize_ms) {
    if (!plan) return 1;
    ssu::StageTimes t;
    if (plan->plan->stage_times(t)) return 1;
    if (embed_ms) *embed_ms = t.embed_ms;
    if (pair_ms) *pair_ms = t.pair_ms;
    if (finalize_ms) *finalize_ms = t.finalize_ms;
    return 0;
}

void ssu_b200_plan_destroy(ssu_b200_plan_t **plan) {
    if (plan && *plan) {
        delete *plan;
        *plan = nullptr;
    }
}

ComputeStatus ssu_b200_one_off_batch_inmem_v3(const support_biom_t *const *tables, unsigned int n_tables,
                                              const support_bptree_t *tree_data, const char *unifrac_method,
                                              bool variance_adjust, double alpha, bool bypass_tips,
                                              bool normalize_sample_counts, mat_full_fp64_t **results) {
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return batch_v3<double, mat_full_fp64_t>(tables, n_tables, tree_data, r, true, results);
}

ComputeStatus ssu_b200_one_off_batch_inmem_fp32_v3(const support_biom_t *const *tables, unsigned int n_tables,
                                                   const support_bptree_t *tree_data, const char *unifrac_method,
                                                   bool variance_adjust, double alpha, bool bypass_tips,
                                                   bool normalize_sample_counts, mat_full_fp32_t **results) {
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return batch_v3<float, mat_full_fp32_t>(tables, n_tables, tree_data, r, false, results);
}

ComputeStatus ssu_b200_subsample_batch_inmem_v3(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                                const char *unifrac_method, bool variance_adjust, double alpha,
                                                bool bypass_tips, bool normalize_sample_counts,
                                                unsigned int n_subsamples, unsigned int subsample_depth,
                                                bool subsample_with_replacement, mat_full_fp64_t **results) {
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return subsample_batch_v3<double, mat_full_fp64_t>(table_data, tree_data, r, true, n_subsamples, subsample_depth,
                                                       subsample_with_replacement, results);
}

ComputeStatus ssu_b200_subsample_batch_inmem_fp32_v3(const support_biom_t *table_data,
                                                     const support_bptree_t *tree_data, const char *unifrac_method,
                                                     bool variance_adjust, double alpha, bool bypass_tips,
                                                     bool normalize_sample_counts, unsigned int n_subsamples,
                                                     unsigned int subsample_depth, bool subsample_with_replacement,
                                                     mat_full_fp32_t **results) {
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    return subsample_batch_v3<float, mat_full_fp32_t>(table_data, tree_data, r, false, n_subsamples,
                                                      subsample_depth, subsample_with_replacement, results);
}

ComputeStatus ssu_b200_batch_plan_create(const support_biom_t *const *tables_data, unsigned int n_tables,
                                         const support_bptree_t *tree_data, const char *unifrac_method,
                                         bool variance_adjust, double alpha, bool bypass_tips,
                                         bool normalize_sample_counts, uint64_t group_bytes, int autotune,
                                         ssu_b200_plan_t **plan) {
    bool fp64 = false;
    ComputeStatus st = is_fp64_method(unifrac_method, fp64);
    if (st != okay) return st;
    if (!tables_data || n_tables == 0 || !plan) return table_empty;
    if (!tree_data) return tree_missing;
    std::vector<ssu::Table> tables;
    tables.reserve(n_tables);
    for (unsigned int t = 0; t < n_tables; t++) {
        const support_biom_t *td = tables_data[t];
        if (!td || td->n_samples <= 0 || td->n_obs <= 0) return table_empty;
        tables.push_back(table_from(td));
    }
    std::vector<const ssu::Table *> ptrs;
    for (const ssu::Table &t : tables) ptrs.push_back(&t);
    StepTimer timer("batch_plan_create");
    ssu::BatchOptions opts;
    opts.group_bytes = group_bytes;
    opts.autotune = autotune;
    auto *h = new ssu_b200_plan();
    const Request r{unifrac_method, variance_adjust, alpha, bypass_tips, normalize_sample_counts};
    st = batch_plan(ptrs, tree_from(tree_data), r, opts, h->plan, timer);
    if (st != okay) {
        delete h;
        return st;
    }
    *plan = h;
    return okay;
}

uint32_t ssu_b200_plan_n_tables(const ssu_b200_plan_t *plan) { return plan ? plan->plan->n_tables() : 0; }
uint32_t ssu_b200_plan_n_groups(const ssu_b200_plan_t *plan) { return plan ? plan->plan->n_groups() : 0; }
uint32_t ssu_b200_plan_table_samples(const ssu_b200_plan_t *plan, uint32_t table) {
    return plan ? plan->plan->table_samples(table) : 0;
}
uint64_t ssu_b200_plan_table_offset(const ssu_b200_plan_t *plan, uint32_t table) {
    return plan ? plan->plan->table_offset(table) : 0;
}
uint64_t ssu_b200_plan_table_embedded(const ssu_b200_plan_t *plan, uint32_t table) {
    return plan ? plan->plan->table_embedded(table) : 0;
}
void ssu_b200_plan_set_graph(ssu_b200_plan_t *plan, int enable) {
    if (plan) plan->plan->set_graph(enable != 0);
}
const char *ssu_b200_plan_tuning(const ssu_b200_plan_t *plan) { return plan ? plan->plan->tuning() : ""; }

const char *ssu_b200_plan_pair_kernel(const ssu_b200_plan_t *plan) {
    return plan ? plan->plan->pair_kernel_name() : "";
}

const char *ssu_b200_version(void) { return "unifrac-b200 0.1 (sm_100a)"; }

}  // extern "C"

// ============================================= PCoA and PERMANOVA (device)

namespace {

template <typename TOut>
void free_outputs(TOut **a, TOut **b, TOut **c) {
    for (TOut **p : {a, b, c}) {
        std::free(*p);
        *p = nullptr;
    }
}

// src/api.cpp:2537-2547 (su::pcoa, src/skbio_alt.cpp:176-199): malloc'ed
// eigenvalues[n_dims], samples[n_samples][n_dims], proportion[n_dims]; all
// three NULL after a failure (reported on stderr).
template <typename TOut, typename TIn>
void pcoa_T(const TIn *mat, uint32_t n, uint32_t dims, TOut **eigenvalues, TOut **samples, TOut **proportion) {
    if (!eigenvalues || !samples || !proportion) return;
    const size_t nd = static_cast<size_t>(n) * dims;
    *eigenvalues = static_cast<TOut *>(std::malloc(sizeof(TOut) * std::max<size_t>(dims, 1)));
    *samples = static_cast<TOut *>(std::malloc(sizeof(TOut) * std::max<size_t>(nd, 1)));
    *proportion = static_cast<TOut *>(std::malloc(sizeof(TOut) * std::max<size_t>(dims, 1)));
    if (!*eigenvalues || !*samples || !*proportion) {
        free_outputs(eigenvalues, samples, proportion);
        report("pcoa", "out of host memory");
        return;
    }
    std::string err;
    try {
        if (!mat && n) throw std::invalid_argument("no matrix");
        if (!select_device(err)) throw std::runtime_error(err);
        std::vector<double> ev(dims), sm(nd), pr(dims);
        if (ssu::pcoa_device(mat, n, dims, ev.data(), sm.data(), pr.data(), err)) throw std::runtime_error(err);
        for (uint32_t c = 0; c < dims; c++) {
            (*eigenvalues)[c] = static_cast<TOut>(ev[c]);
            (*proportion)[c] = static_cast<TOut>(pr[c]);
        }
        for (size_t k = 0; k < nd; k++) (*samples)[k] = static_cast<TOut>(sm[k]);
    } catch (const std::exception &e) {
        free_outputs(eigenvalues, samples, proportion);
        report("pcoa", e.what());
    }
}

// src/api.cpp:2501-2507 (su::find_eigens_fast): eigenvalues[n_dims] and
// unit eigenvectors[n_samples][n_dims] of an already centred matrix.
template <typename TReal>
void eigens_T(uint32_t n, uint32_t dims, const TReal *centered, TReal **eigenvalues, TReal **eigenvectors) {
    if (!eigenvalues || !eigenvectors) return;
    const size_t nd = static_cast<size_t>(n) * dims;
    *eigenvalues = static_cast<TReal *>(std::malloc(sizeof(TReal) * std::max<size_t>(dims, 1)));
    *eigenvectors = static_cast<TReal *>(std::malloc(sizeof(TReal) * std::max<size_t>(nd, 1)));
    std::string err;
    try {
        if (!*eigenvalues || !*eigenvectors) throw std::runtime_error("out of host memory");
        if (!centered && n) throw std::invalid_argument("no matrix");
        if (!select_device(err)) throw std::runtime_error(err);
        std::vector<double> ev(dims), vec(nd);
        if (ssu::eigens_device(centered, n, dims, ev.data(), vec.data(), err)) throw std::runtime_error(err);
        for (uint32_t c = 0; c < dims; c++) (*eigenvalues)[c] = static_cast<TReal>(ev[c]);
        for (size_t k = 0; k < nd; k++) (*eigenvectors)[k] = static_cast<TReal>(vec[k]);
    } catch (const std::exception &e) {
        std::free(*eigenvalues);
        std::free(*eigenvectors);
        *eigenvalues = nullptr;
        *eigenvectors = nullptr;
        report("find_eigens_fast", e.what());
    }
}

// Labels of any values renumbered 0, 1, ... by first appearance.
uint32_t dense_labels(const uint32_t *grouping, uint32_t n, std::vector<uint32_t> &out) {
    std::unordered_map<uint32_t, uint32_t> ids;
    out.resize(n);
    for (uint32_t i = 0; i < n; i++)
        out[i] = ids.emplace(grouping[i], static_cast<uint32_t>(ids.size())).first->second;
    return static_cast<uint32_t>(ids.size());
}

template <typename TReal>
ComputeStatus permanova_T(const TReal *mat, uint32_t n, const uint32_t *grouping, uint32_t n_groups,
                          unsigned int perms, uint64_t seed, TReal &fstat, TReal &pvalue) {
    std::string err;
    try {
        if (!select_device(err)) throw std::runtime_error(err);
        double f = 0.0, p = 0.0;
        if (ssu::permanova_device(mat, n, grouping, n_groups, perms, seed, f, p, err)) throw std::runtime_error(err);
        fstat = static_cast<TReal>(f);
        pvalue = static_cast<TReal>(p);
        return okay;
    } catch (const std::exception &e) {
        report("permanova", e.what());
        return output_error;
    }
}

// src/api.cpp:949-975: each grouping column read from the TSV (any failure:
// grouping_missing) and tested on the matrix.  Column i's permutations are
// drawn from the library seed (ssu_set_random_seed) + i.
template <typename TReal, typename TMat>
ComputeStatus compute_permanova_T(const char *grouping_filename, unsigned int n_columns, const char **columns,
                                  TMat *result, unsigned int perms, TReal *fstats, TReal *pvalues) {
    if (!result || !result->matrix || !result->sample_ids || (n_columns && (!columns || !fstats || !pvalues)))
        return grouping_missing;
    if (!grouping_filename || !file_exists(grouping_filename)) return grouping_missing;
    std::vector<uint32_t> grouping;
    for (unsigned int i = 0; i < n_columns; i++) {
        uint32_t n_groups = 0;
        std::string err;
        if (!columns[i] || !ssu::read_grouping_tsv(grouping_filename, columns[i], result->n_samples,
                                                   result->sample_ids, grouping, n_groups, err)) {
            report("grouping", err);
            return grouping_missing;
        }
        const ComputeStatus st = permanova_T<TReal>(result->matrix, result->n_samples, grouping.data(), n_groups,
                                                    perms, g_seed.load() + i, fstats[i], pvalues[i]);
        if (st != okay) return st;
    }
    return okay;
}

}  // namespace

extern "C" {

void pcoa(const double *mat, const uint32_t n_samples, const uint32_t n_dims, double **eigenvalues,
          double **samples, double **proportion_explained) {
    pcoa_T<double>(mat, n_samples, n_dims, eigenvalues, samples, proportion_explained);
}

void pcoa_fp32(const float *mat, const uint32_t n_samples, const uint32_t n_dims, float **eigenvalues,
               float **samples, float **proportion_explained) {
    pcoa_T<float>(mat, n_samples, n_dims, eigenvalues, samples, proportion_explained);
}

void pcoa_mixed(const double *mat, const uint32_t n_samples, const uint32_t n_dims, float **eigenvalues,
                float **samples, float **proportion_explained) {
    pcoa_T<float>(mat, n_samples, n_dims, eigenvalues, samples, proportion_explained);
}

void find_eigens_fast(const uint32_t n_samples, const uint32_t n_dims, double *centered, double **eigenvalues,
                      double **eigenvectors) {
    eigens_T<double>(n_samples, n_dims, centered, eigenvalues, eigenvectors);
}

void find_eigens_fast_fp32(const uint32_t n_samples, const uint32_t n_dims, float *centered, float **eigenvalues,
                           float **eigenvectors) {
    eigens_T<float>(n_samples, n_dims, centered, eigenvalues, eigenvectors);
}

ComputeStatus compute_permanova_fp64(const char *grouping_filename, unsigned int n_columns, const char **columns,
                                     mat_full_fp64_t *result, unsigned int permanova_perms, double *fstats,
                                     double *pvalues) {
    return compute_permanova_T<double>(grouping_filename, n_columns, columns, result, permanova_perms, fstats,
                                       pvalues);
}

ComputeStatus compute_permanova_fp32(const char *grouping_filename, unsigned int n_columns, const char **columns,
                                     mat_full_fp32_t *result, unsigned int permanova_perms, float *fstats,
                                     float *pvalues) {
    return compute_permanova_T<float>(grouping_filename, n_columns, columns, result, permanova_perms, fstats,
                                      pvalues);
}

ComputeStatus ssu_b200_read_grouping(const char *grouping_filename, const char *column, uint32_t n_samples,
                                     const char *const *sample_ids, uint32_t *grouping, uint32_t *n_groups) {
    if (!grouping_filename || !column || (n_samples && (!sample_ids || !grouping)) || !n_groups)
        return grouping_missing;
    std::vector<uint32_t> g;
    std::string err;
    if (!ssu::read_grouping_tsv(grouping_filename, column, n_samples, sample_ids, g, *n_groups, err)) {
        report("grouping", err);
        return grouping_missing;
    }
    std::copy(g.begin(), g.end(), grouping);
    return okay;
}

ComputeStatus ssu_b200_permanova_fp64(const double *mat, uint32_t n_samples, const uint32_t *grouping,
                                      unsigned int permanova_perms, double *fstat, double *pvalue) {
    if (!mat || !grouping || !fstat || !pvalue) return output_error;
    std::vector<uint32_t> labels;
    const uint32_t g = dense_labels(grouping, n_samples, labels);
    return permanova_T<double>(mat, n_samples, labels.data(), g, permanova_perms, g_seed.load(), *fstat, *pvalue);
}

ComputeStatus ssu_b200_permanova_fp32(const float *mat, uint32_t n_samples, const uint32_t *grouping,
                                      unsigned int permanova_perms, float *fstat, float *pvalue) {
    if (!mat || !grouping || !fstat || !pvalue) return output_error;
    std::vector<uint32_t> labels;
    const uint32_t g = dense_labels(grouping, n_samples, labels);
    return permanova_T<float>(mat, n_samples, labels.data(), g, permanova_perms, g_seed.load(), *fstat, *pvalue);
}

IOStatus ssu_b200_read_h5_doubles(const char *filename, const char *dataset, double **values, uint32_t *rank,
                                  uint64_t *dims) {
    if (!filename || !dataset || !values || !rank || !dims) return read_error;
    *values = nullptr;
    *rank = 0;
    if (!file_exists(filename)) return open_error;
    ssu::H5Data d;
    std::string err;
    if (!ssu::read_hdf5_dataset(filename, dataset, d, err) || d.is_string || d.dims.size() > 8) {
        report("hdf5", std::string(filename) + ":" + dataset + ": " + (err.empty() ? "not a numeric dataset" : err));
        return read_error;
    }
    *values = static_cast<double *>(std::malloc(sizeof(double) * std::max<size_t>(d.values.size(), 1)));
    if (!*values) return read_error;
    std::copy(d.values.begin(), d.values.end(), *values);
    *rank = static_cast<uint32_t>(d.dims.size());
    std::copy(d.dims.begin(), d.dims.end(), dims);
    return read_okay;
}

IOStatus ssu_b200_read_h5_strings(const char *filename, const char *dataset, char ***strings, uint64_t *n) {
    if (!filename || !dataset || !strings || !n) return read_error;
    *strings = nullptr;
    *n = 0;
    if (!file_exists(filename)) return open_error;
    ssu::H5Data d;
    std::string err;
    if (!ssu::read_hdf5_dataset(filename, dataset, d, err) || !d.is_string) {
        report("hdf5", std::string(filename) + ":" + dataset + ": " + (err.empty() ? "not a string dataset" : err));
        return read_error;
    }
    std::vector<std::string_view> views(d.strings.begin(), d.strings.end());
    *strings = copy_ids(views);
    *n = d.strings.size();
    return read_okay;
}

void ssu_b200_free_h5_strings(char **strings, uint64_t n) {
    if (!strings) return;
    for (uint64_t i = 0; i < n; i++) std::free(strings[i]);
    std::free(strings);
}

}  // extern "C"
