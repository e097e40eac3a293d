// Device plan of the B200 UniFrac engine (host-visible interface; no CUDA
// types cross this header so the C API layer stays plain C++).
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
    // unweighted (non variance-adjusted) only: run the tcgen05 contraction
    // instead of the presence-word stripe kernel
    bool unweighted_gemm = false;
};

// Method-name table of the reference (src/api.cpp:55-88): bare names are fp32.
bool parse_method(const char *name, Method &method, bool &fp64);

enum class OutMode : int { full = 0, stripes = 1, condensed = 2 };

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
    // Faith PD plan: embedding of every non-root node in fp64, no pair stage.
    static int create_faith(const Table &table, const FlatTree &tree, void *stream, Plan **out, std::string &err);
    ~Plan();

    // Recompute the full n x n matrix into device memory (T = double for
    // fp64 methods, float otherwise).  Asynchronous on `stream` (nullptr: the
    // plan's stream).
    int execute(void *stream);
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

    const void *device_result() const;
    int copy_result(void *host_out, void *stream);
    int synchronize();
    // Error code raised by a device-side bounded wait since the last check
    // (0 = none); synchronises the plan's stream.
    int device_error();

    uint32_t n_samples() const;
    uint64_t n_embedded() const;
    uint64_t work_units() const;
    uint32_t launches() const;
    const char *pair_kernel_name() const;
    void set_timing(bool on);
    int stage_times(StageTimes &out);

  private:
    Plan() = default;
    PlanImpl *impl_ = nullptr;
};

}  // namespace ssu
