// Device plan of the B200 UniFrac engine (host-visible interface; no CUDA
// types cross this header so the C API layer stays plain C++).
//
// A plan holds one table, or a batch of tables that share one tree (many
// rarefied replicates of a table, or many tables of uneven sample counts).
// A batch is laid out as groups of tables whose embeddings fit the device
// together; each group is embedded in one pass and its pair stage is one
// persistent launch over the tiles of all its tables.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "ssu_table.hpp"
#include "ssu_tree.hpp"

namespace ssu {

// su::Method (src/unifrac.hpp:22) without the precision axis, which is `fp64`.
enum class Method : int { unweighted = 0, unweighted_unnormalized, weighted_normalized, weighted_unnormalized, generalized };

struct MethodSpec {
    Method method = Method::unweighted;
    bool fp64 = true;
    bool vaw = false;
    double alpha = 1.0;
    bool bypass_tips = false;
    bool normalize = true;
    // unweighted (non variance-adjusted) only: the tcgen05 contraction is
    // the default for fp32 results; unweighted_gemm asks for it with fp64
    // results too, unweighted_stripe keeps the presence-word stripe kernel
    bool unweighted_gemm = false;
    bool unweighted_stripe = false;
};

// Method-name table of the reference (src/api.cpp:55-88): bare names are fp32.
bool parse_method(const char *name, Method &method, bool &fp64);

enum class OutMode : int { full = 0, stripes = 1, condensed = 2 };

// Tables of a batch plan, all flattened against one tree.
struct TableSet {
    std::vector<const Table *> tables;
    // obs_row[i][o]: row in table i of the tree's observation o
    // (FlatTree::leaf_obs), or -1
    std::vector<std::vector<int32_t>> obs_row;
    // embedded node count of each table's own sheared and collapsed tree
    // (the reference's work per pair)
    std::vector<uint32_t> embedded;
    // with bypassed tips: row_active[i][row] says whether an embedded row
    // of the shared tree is an embedded row of table i's own tree (rows whose
    // subtree holds a single tip of table i merge into that tip there)
    std::vector<std::vector<uint8_t>> row_active;
};

struct BatchOptions {
    // device bytes one group may use for its embedding (0: a share of the
    // free memory at plan creation)
    size_t group_bytes = 0;
    // pair-kernel tile shape: -1 engine default (tuned for batches), 0 the
    // heuristic choice, 1 measured on the plan's own data
    int autotune = -1;
};

// Stage timings of the last execute (ms), filled when timing is on.
struct StageTimes {
    float embed_ms = 0, pair_ms = 0, finalize_ms = 0;
};

struct PlanImpl;

class Plan {
  public:
    // Uploads the table (CSR + per-sample totals) and the flattened tree and
    // allocates the embedding and result buffers.  `stream` is a cudaStream_t
    // (nullptr: the plan creates its own).  Returns 0 or a ComputeStatus code
    // with `err` set.
    static int create(const Table &table, const FlatTree &tree, const MethodSpec &spec, void *stream, Plan **out,
                      std::string &err);
    // Batch plan: full results of every table, in table order, one after
    // the other in device memory.
    static int create_batch(const TableSet &set, const FlatTree &tree, const MethodSpec &spec,
                            const BatchOptions &opts, void *stream, Plan **out, std::string &err);
    // Faith PD plan: embedding of every non-root node in fp64, no pair stage.
    static int create_faith(const Table &table, const FlatTree &tree, void *stream, Plan **out, std::string &err);
    ~Plan();

    // Recompute the full n x n matrix (of every table) into device memory
    // (T = double for fp64 methods, float otherwise).  Asynchronous on
    // `stream` (nullptr: the plan's stream).  With graph mode on, the first
    // call captures the whole sequence as one CUDA graph and later calls
    // launch it.
    int execute(void *stream);
    void set_graph(bool on);
    // One execute with the result written for the stripes [start, stop) into
    // host arrays stripes[s - start][0..n) (double).
    int run_stripes(uint32_t start, uint32_t stop, double *const *host_stripes, std::string &err);
    // Condensed upper triangle (double, n(n-1)/2) into host memory.
    int run_condensed(double *host_cf, std::string &err);
    // Full matrix into host memory as double or float (converted on device).
    int run_full(void *host_out, bool out_fp64, std::string &err);
    // Faith PD values of every sample (plan from create_faith).
    int run_faith(double *host_values, std::string &err);

    // Copy the full result of the last execute into host memory; with
    // `pin`, the destination is page-locked for the copy (cudaHostRegister)
    // and released after.  Synchronises and checks device-side errors.
    int download_full(void *host_out, bool pin, std::string &err);
    // execute(nullptr) then download_full, with the copy-out overlapped with
    // the computation where the plan allows it (one table on the tensor-core
    // path: bands of rows are copied as soon as every launch writing to them
    // has finished); otherwise the two calls in turn.
    int execute_download(void *host_out, bool pin, std::string &err);
    // Same for `count` result elements starting at element `offset` (one
    // table of a batch: table_offset(t), n_t * n_t).
    int download_range(uint64_t offset, uint64_t count, void *host_out, bool pin, std::string &err);

    const void *device_result() const;
    int copy_result(void *host_out, void *stream);
    int synchronize();
    // Error code raised by a device-side bounded wait since the last check
    // (0 = none); synchronises the plan's stream.
    int device_error();

    uint32_t n_samples() const;  // all tables
    uint32_t n_tables() const;
    uint32_t n_groups() const;
    uint32_t table_samples(uint32_t t) const;
    uint64_t table_offset(uint32_t t) const;  // elements into device_result()
    uint64_t table_embedded(uint32_t t) const;
    // how the pair kernel was chosen ("default", "tuned ...", "cache ...")
    const char *tuning() const;
    uint64_t n_embedded() const;
    uint64_t work_units() const;
    // tensor-core flops (2 x multiply-adds) one execute issues; 0 off the
    // tensor-core path
    uint64_t tensor_flops() const;
    uint32_t launches() const;
    const char *pair_kernel_name() const;
    void set_timing(bool on);
    int stage_times(StageTimes &out);

  private:
    Plan() = default;
    PlanImpl *impl_ = nullptr;
};

}  // namespace ssu
