// Device plan of the B200 UniFrac engine: upload, embedding, pair stage,
// output layouts.  One plan = one table, or a batch of tables sharing a
// tree, on one GPU and one stream.
#include "ssu_engine.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cuda.h>
#include <cuda_runtime.h>
#include <fstream>
#include <map>
#include <future>
#include <mutex>
#include <thread>

#include "ssu_gemm.cuh"
#include "ssu_host.hpp"
#include "ssu_kernels.cuh"
#include "ssu_pairs.cuh"
#include "ssu_sparse.cuh"
#include "ssu_union.cuh"

namespace ssu {

bool parse_method(const char *name, Method &method, bool &fp64) {
    struct Entry {
        const char *name;
        Method method;
        bool fp64;
    };
    static const Entry table[] = {
        {"unweighted", Method::unweighted, false},
        {"weighted_normalized", Method::weighted_normalized, false},
        {"weighted_unnormalized", Method::weighted_unnormalized, false},
        {"unweighted_unnormalized", Method::unweighted_unnormalized, false},
        {"generalized", Method::generalized, false},
        {"unweighted_fp64", Method::unweighted, true},
        {"weighted_normalized_fp64", Method::weighted_normalized, true},
        {"weighted_unnormalized_fp64", Method::weighted_unnormalized, true},
        {"unweighted_unnormalized_fp64", Method::unweighted_unnormalized, true},
        {"generalized_fp64", Method::generalized, true},
        {"unweighted_fp32", Method::unweighted, false},
        {"weighted_normalized_fp32", Method::weighted_normalized, false},
        {"weighted_unnormalized_fp32", Method::weighted_unnormalized, false},
        {"unweighted_unnormalized_fp32", Method::unweighted_unnormalized, false},
        {"generalized_fp32", Method::generalized, false},
    };
    if (!name) return false;
    for (const Entry &e : table)
        if (std::strcmp(name, e.name) == 0) {
            method = e.method;
            fp64 = e.fp64;
            return true;
        }
    return false;
}

namespace {

constexpr int kOutputError = 6;  // ComputeStatus output_error

// One stream-ordered memory pool per device, owned by the library, that
// keeps freed blocks cached (no release threshold): repeated calls reuse the
// embedding and result buffers instead of re-mapping them.
// Host -> device copies from pageable memory (the caller's table arrays)
// through page-locked staging: up to four host threads each copy 8 MiB
// pieces into two staging buffers of their own and issue an asynchronous
// copy from each on a stream of their own (a buffer is refilled once its
// last copy has landed), so host memory is read by several threads while
// the copies run; the driver's own pageable path stages on the calling
// thread (11-12 GB/s on the B200 hosts here).  The staging buffers are made
// once per process, for the first device that uploads; other devices, a
// second upload while one is running, and small uploads (below 32 MiB) take
// the plain path.  On return the copies are ordered before later work on s.
struct HostPiece {
    void *dst;
    const void *src;
    size_t bytes;
};
class Staging {
  public:
    static constexpr size_t kPiece = size_t(8) << 20;
    static constexpr int kWorkers = 4;

    static Staging &get() {
        static Staging st;
        return st;
    }
    // 0 on success; any CUDA error code otherwise
    cudaError_t upload(const std::vector<HostPiece> &pieces, cudaStream_t s, int dev) {
        size_t total = 0;
        for (const HostPiece &p : pieces) total += p.bytes;
        std::unique_lock<std::mutex> lock(mu_, std::try_to_lock);
        const unsigned workers = std::min<unsigned>(kWorkers, host_threads(kWorkers));
        if (total < (size_t(32) << 20) || !lock.owns_lock() || workers < 2 || !ready(dev)) {
            for (const HostPiece &p : pieces)
                if (p.bytes) {
                    const cudaError_t e = cudaMemcpyAsync(p.dst, p.src, p.bytes, cudaMemcpyHostToDevice, s);
                    if (e != cudaSuccess) return e;
                }
            return cudaSuccess;
        }
        // the destinations are stream-ordered allocations on s: copies start after them
        cudaError_t e0 = cudaEventRecord(start_, s);
        for (unsigned w = 0; w < workers && e0 == cudaSuccess; w++) e0 = cudaStreamWaitEvent(streams_[w], start_, 0);
        if (e0 != cudaSuccess) return e0;
        std::vector<HostPiece> cuts;  // 8 MiB pieces, in order
        for (const HostPiece &p : pieces)
            for (size_t o = 0; o < p.bytes; o += kPiece)
                cuts.push_back({static_cast<char *>(p.dst) + o, static_cast<const char *>(p.src) + o,
                                std::min(kPiece, p.bytes - o)});
        std::vector<cudaError_t> err(workers, cudaSuccess);
        auto work = [&](unsigned w) {
            cudaError_t e = cudaSetDevice(dev);
            unsigned use = 0;
            for (size_t i = w; i < cuts.size() && e == cudaSuccess; i += workers, use++) {
                const unsigned b = w * 2 + (use & 1);
                e = cudaEventSynchronize(landed_[b]);  // its previous copy has landed
                if (e != cudaSuccess) break;
                std::memcpy(buf_[b], cuts[i].src, cuts[i].bytes);
                e = cudaMemcpyAsync(cuts[i].dst, buf_[b], cuts[i].bytes, cudaMemcpyHostToDevice, streams_[w]);
                if (e == cudaSuccess) e = cudaEventRecord(landed_[b], streams_[w]);
            }
            err[w] = e;
        };
        std::vector<std::thread> pool;
        for (unsigned w = 1; w < workers; w++) {
            try {
                pool.emplace_back(work, w);
            } catch (const std::system_error &) {
                err[w] = cudaErrorLaunchFailure;  // reported below; its pieces were not copied
            }
        }
        work(0);
        for (std::thread &t : pool) t.join();
        for (unsigned w = 0; w < workers; w++)
            if (err[w] != cudaSuccess) {
                // nothing may still write the destinations once the caller frees them
                for (unsigned v = 0; v < workers; v++) cudaStreamSynchronize(streams_[v]);
                return err[w];
            }
        for (unsigned w = 0; w < workers; w++) {
            cudaError_t e = cudaEventRecord(done_[w], streams_[w]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, done_[w], 0);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

  private:
    bool ready(int dev) {
        if (dev_ >= 0) return dev_ == dev && ok_;
        dev_ = dev;
        ok_ = cudaEventCreateWithFlags(&start_, cudaEventDisableTiming) == cudaSuccess;
        for (int w = 0; w < kWorkers && ok_; w++) {
            ok_ = cudaStreamCreateWithFlags(&streams_[w], cudaStreamNonBlocking) == cudaSuccess &&
                  cudaEventCreateWithFlags(&done_[w], cudaEventDisableTiming) == cudaSuccess;
            for (int b = 2 * w; b < 2 * w + 2 && ok_; b++)
                ok_ = cudaHostAlloc(&buf_[b], kPiece, cudaHostAllocDefault) == cudaSuccess &&
                      cudaEventCreateWithFlags(&landed_[b], cudaEventDisableTiming) == cudaSuccess;
        }
        if (!ok_) cudaGetLastError();  // the plain path stands in
        return ok_;
    }
    std::mutex mu_;
    int dev_ = -1;
    bool ok_ = false;
    cudaStream_t streams_[kWorkers] = {};
    cudaEvent_t done_[kWorkers] = {};
    void *buf_[2 * kWorkers] = {};
    cudaEvent_t landed_[2 * kWorkers] = {};
    cudaEvent_t start_ = nullptr;
};

cudaMemPool_t device_pool(int dev) {
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    if (pools.size() <= static_cast<size_t>(dev)) pools.resize(dev + 1, nullptr);
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
        uint64_t threshold = UINT64_MAX;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &threshold);
        pools[dev] = p;
    }
    return pools[dev];
}

#define SSU_CK(call)                                                                                  \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            last_error = std::string(#call) + ": " + cudaGetErrorString(e_);                          \
            return kOutputError;                                                                      \
        }                                                                                             \
    } while (0)

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// 2-D tensor map over a row-major [rows][cols] matrix of bytes with a
// 128-column x box_rows box and 128-byte swizzle (the UMMA K-major layout);
// rows past `rows` read as zero.
bool make_u8_map(CUtensorMap *map, void *base, uint64_t rows, uint64_t cols, uint32_t box_rows) {
    EncodeTiledFn f = encode_tiled();
    if (!f) return false;
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {cols};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(tc::BLOCK_K), box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return f(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 2-D tensor map over the first `rows` rows of a row-major [.][cols] matrix of
// T (fp64 or fp32), box 64 columns x 16 rows, no swizzle; rows past `rows`
// read as zero.  cols * sizeof(T) must be a multiple of 16.
template <typename T>
bool make_rows_map(CUtensorMap *map, const void *base, uint64_t rows, uint64_t cols) {
    EncodeTiledFn f = encode_tiled();
    if (!f) return false;
    const cuuint64_t dims[2] = {cols, std::max<uint64_t>(rows, 1)};
    const cuuint64_t strides[1] = {cols * sizeof(T)};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(dev::UT), static_cast<cuuint32_t>(dev::URS)};
    const cuuint32_t estr[2] = {1, 1};
    return f(map, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
             const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tiles of one table (columns [base, base + n) of its group) holding at
// least one pair k < l; with a stripe window only those whose pairs reach a
// stripe in [start, stop).  x and y are block indices in the group's
// columns, z is the table.
void append_tiles(std::vector<uint4> &tiles, uint32_t table, uint32_t base, uint32_t n, int BM, int BN,
                  bool windowed, uint32_t start, uint32_t stop) {
    const uint32_t nbk = (n + BM - 1) / BM, nbl = (n + BN - 1) / BN;
    for (uint32_t kb = 0; kb < nbk; kb++) {
        const int64_t kmin = static_cast<int64_t>(kb) * BM;
        const int64_t kmax = std::min<int64_t>(n, kmin + BM) - 1;
        for (uint32_t lb = 0; lb < nbl; lb++) {
            const int64_t lmin = static_cast<int64_t>(lb) * BN;
            const int64_t lmax = std::min<int64_t>(n, lmin + BN) - 1;
            if (kmin >= lmax) continue;
            if (windowed) {
                const int64_t dmin = std::max<int64_t>(1, lmin - kmax), dmax = lmax - kmin;
                const int64_t s1lo = dmin - 1, s1hi = dmax - 1;
                const int64_t s2lo = static_cast<int64_t>(n) - dmax - 1, s2hi = static_cast<int64_t>(n) - dmin - 1;
                const bool hit1 = s1lo < static_cast<int64_t>(stop) && s1hi >= static_cast<int64_t>(start);
                const bool hit2 = s2lo < static_cast<int64_t>(stop) && s2hi >= static_cast<int64_t>(start);
                if (!hit1 && !hit2) continue;
            }
            tiles.push_back(make_uint4(base / BM + kb, base / BN + lb, table, 0));
        }
    }
}

// Pair-kernel shapes chosen by measurement, per problem class, for the life
// of the process and, with UNIFRAC_B200_TUNE_CACHE=<file>, across processes
// (one "key<TAB>shape" line per choice).
class TuneCache {
  public:
    static TuneCache &get() {
        static TuneCache c;
        return c;
    }
    bool find(const std::string &key, std::string &shape) {
        std::lock_guard<std::mutex> lock(mu_);
        load();
        auto it = entries_.find(key);
        if (it == entries_.end()) return false;
        shape = it->second;
        return true;
    }
    void put(const std::string &key, const std::string &shape) {
        std::lock_guard<std::mutex> lock(mu_);
        load();
        entries_[key] = shape;
        const char *path = std::getenv("UNIFRAC_B200_TUNE_CACHE");
        if (path && *path) {
            std::ofstream f(path, std::ios::app);
            if (f) f << key << '\t' << shape << '\n';
        }
    }

  private:
    void load() {
        if (loaded_) return;
        loaded_ = true;
        const char *path = std::getenv("UNIFRAC_B200_TUNE_CACHE");
        if (!path || !*path) return;
        std::ifstream f(path);
        std::string line;
        while (std::getline(f, line)) {
            const size_t tab = line.find('\t');
            if (tab != std::string::npos) entries_[line.substr(0, tab)] = line.substr(tab + 1);
        }
    }
    std::mutex mu_;
    bool loaded_ = false;
    std::map<std::string, std::string> entries_;
};

int log2_bucket(uint64_t x) {
    int b = 0;
    while (x > 1) {
        x >>= 1;
        b++;
    }
    return b;
}

// UNIFRAC_TIMING_INFO: host time of the plan's setup steps, printed as the
// API layer prints its own steps.
struct SetupTimer {
    bool on;
    std::chrono::steady_clock::time_point t0;
    SetupTimer() : on(std::getenv("UNIFRAC_TIMING_INFO") != nullptr), t0(std::chrono::steady_clock::now()) {}
    void step(const char *name) {
        if (!on) return;
        const auto t1 = std::chrono::steady_clock::now();
        std::printf("INFO (unifrac): dt %8.3f ms : plan.%s\n",
                    std::chrono::duration<double, std::milli>(t1 - t0).count(), name);
        std::fflush(stdout);
        t0 = t1;
    }
};

int env_int(const char *name, int fallback) {
    const char *v = std::getenv(name);
    return (v && *v) ? std::atoi(v) : fallback;
}

}  // namespace

// Tables that are embedded together: one column slab of the embedding each.
struct Group {
    uint32_t t0 = 0, t1 = 0;             // tables [t0, t1)
    uint64_t ld = 0;                     // columns = row stride of the embedding
    int32_t *d_tip_obs = nullptr;        // [tip][t1 - t0]: the tip's row in each table, or -1
    double *d_totals = nullptr;          // per column, fp64
    void *d_tot = nullptr;               // per column in T (variance adjusted)
    uint32_t *d_block_table = nullptr;   // per 128 columns: the table (per-table lengths)
    std::vector<double> totals;
    uint4 *d_tiles = nullptr;
    uint32_t n_tiles = 0, splits = 1, rows_per_split = 0;
    // tensor-core path: per operand row, the starting columns of its tips
    uint32_t *d_sample_ptr = nullptr;
    int32_t *d_start_col = nullptr;
    // tensor-core path, one table: first work unit and first row of each
    // band of row blocks (one extra entry closes the list)
    std::vector<uint32_t> band_unit, band_row;
};

// Host-built layout of the tensor-core operands (see build_gemm_layout).
struct GemmLayout {
    std::vector<double> lsorted, scale;  // lengths in column order; 2^-s_c per chunk
    std::vector<uint32_t> chunk_end;     // first K block after chunk c
    std::vector<uint8_t> digits;         // u, s, v, t rows of k_pad bytes
    std::vector<int32_t> parent_col;     // embedded parent's column, or -1
    std::vector<int32_t> start_of_obs;   // column where a tree observation's path starts, or -1
    std::string error;
};
GemmLayout build_gemm_layout(const FlatTree &tree);

struct PlanImpl {
    MethodSpec spec;
    bool faith = false;
    bool batch = false;
    uint32_t n = 0;  // samples of all tables
    uint32_t K = 0, E = 0;
    uint64_t ld = 0;      // widest group
    uint32_t max_table_n = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int n_sms = 148;
    std::string last_error;

    // tables: concatenated CSR, descriptors, groups
    std::vector<dev::TableDesc> tdesc;
    dev::TableDesc *d_tdesc = nullptr;
    std::vector<uint64_t> table_E;
    std::vector<Group> groups;
    uint32_t *d_indptr = nullptr, *d_indices = nullptr;
    double *d_data = nullptr;
    // tensor-core layout built on a worker thread while setup() uploads
    // (built in setup_gemm instead when no thread can be started)
    std::future<GemmLayout> gemm_layout;
    void start_gemm_layout(const FlatTree &tree) {
        try {
            gemm_layout = std::async(std::launch::async, build_gemm_layout, std::cref(tree));
        } catch (const std::exception &) {
            gemm_layout = std::future<GemmLayout>();
        }
    }

    // tree
    uint32_t n_tips = 0;
    uint32_t *d_tip_rows = nullptr;
    uint32_t *d_child_ptr = nullptr, *d_child_rows = nullptr, *d_level_rows = nullptr;
    std::vector<uint32_t> level_ptr;
    uint32_t *d_post_rows = nullptr;
    double *d_len_rows = nullptr;
    void *d_len = nullptr;  // embedded lengths in T; per table when len_stride > 0
    uint64_t len_stride = 0;
    std::vector<double> host_len;
    std::vector<std::vector<uint8_t>> row_active;

    // embedding and method buffers, sized for the widest group
    void *d_U = nullptr, *d_C = nullptr;
    void *d_W = nullptr, *d_part = nullptr;
    uint32_t n_parts = 0, part_chunk = 0;
    unsigned long long *d_P = nullptr;
    void *d_lut = nullptr;
    uint64_t lut_stride = 0;
    uint32_t n_words = 0;
    void *d_full = nullptr;
    uint64_t full_elems = 0;

    // weighted methods over the sparse embedding (dense rows in registers,
    // sparse rows on their intersections, flagged tiles recomputed exactly)
    bool hybrid = false;
    uint32_t hybrid_div = 8;  // rows non-zero in more than ld / hybrid_div columns are dense
    bool hybrid_atomic = false;  // sparse updates with shared-memory atomics (fp32 default)
    bool hybrid_scatter = false;  // sparse rows as per-pair fixed-point sums (sparse_pairs_kernel)
    unsigned long long *d_Sq = nullptr;  // those sums; the fp64 result buffer doubles as them
    unsigned long long *d_sc_next = nullptr;  // the scatter's next (sparse row, table) task
    uint64_t scatter_band_bytes = 40ull << 20;  // sums per scatter band (UNIFRAC_B200_SCATTER_BAND_BYTES, 0: one band)
    double sq_scale = 1.0;
    bool nonneg_data = true;  // no negative count in any table
    unsigned long long *d_masks = nullptr;
    uint32_t *d_counts = nullptr, *d_dense_rows = nullptr, *d_sparse_rows = nullptr, *d_nrows = nullptr;
    uint8_t *d_row_class = nullptr;
    double *d_Ws = nullptr, *d_ws_part = nullptr, *d_hpartial = nullptr;
    int *d_flags = nullptr;
    size_t hpartial_bytes = 0;
    template <typename T>
    int setup_hybrid();
    template <typename T>
    int hybrid_stage(cudaStream_t s, const Group &g, const dev::OutSpec &out, const uint4 *tiles, uint32_t ntiles,
                     uint32_t splits, bool last);
    // generalized and variance-adjusted methods over the union of the two
    // samples' supports (same masks and row classes as the hybrid)
    bool union_mode = false;
    double *d_upartial = nullptr;
    size_t upartial_bytes = 0;
    void *d_slen = nullptr;  // union kernel: branch lengths in T, zero-padded to whole 16-row stages
    // budget of one mbarrier wait in the union kernel (UNIFRAC_B200_WAIT_CYCLES,
    // default about one second), and its test switch UNIFRAC_B200_TEST_STALL=1
    // (the kernel's producer issues nothing, so its waits run out and the call
    // returns output_error: host-side failure injection, no fault)
    long long union_wait_cycles = 2000000000LL;
    int union_stall = 0;
    // the same for the tensor-core kernel, whose longest legitimate wait (a
    // chunk of 127 K blocks) is about 35 us: default about 0.1 s
    long long gemm_wait_cycles = 200000000LL;
    int sparse_prep_alloc();
    template <typename T>
    int sparse_prep(cudaStream_t s, const Group &g, uint32_t div);
    template <typename T>
    int setup_union();
    template <typename T>
    int union_stage(cudaStream_t s, const Group &g, const dev::OutSpec &out, const uint4 *tiles, uint32_t ntiles,
                    uint32_t splits, bool last);

    // pair stage
    PairKernel<double> kd;
    PairKernel<float> kf;
    void *d_partial = nullptr;
    size_t partial_bytes = 0;
    int autotune = 0;
    std::string tuning = "default";

    // tensor-core unweighted path (one table)
    bool gemm = false;
    uint32_t n_pad = 0, k_pad = 0, n_chunks = 0;
    uint8_t *d_A = nullptr, *d_B = nullptr, *d_lq = nullptr;
    double *d_r = nullptr, *d_lsorted = nullptr, *d_chunk_scale = nullptr;
    uint32_t *d_chunk_end = nullptr;
    int32_t *d_parent_col = nullptr;
    int *d_error = nullptr;
    CUtensorMap map_A{}, map_B{};
    int setup_gemm(const TableSet &set, const FlatTree &tree);
    int build_units(uint32_t band);
    int tune_band();
    bool device_error_pending();
    uint32_t tc_band = 4;
    int execute_gemm(cudaStream_t s, const dev::OutSpec &out);
    int execute_gemm_overlap(void *host);
    // overlapped copy-out: a second compute stream, the copy stream, and an
    // event per band of rows
    cudaStream_t aux[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> band_ev;

    // CUDA graph of execute()
    bool graph_on = false, capturing = false;
    cudaGraphExec_t graph = nullptr;

    template <typename T>
    PairKernel<T> &kern();

    bool timing = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    uint32_t launches = 0;
    std::vector<void *> allocations;

    cudaMemPool_t pool = nullptr;

    template <typename P>
    cudaError_t alloc(P **p, size_t bytes) {
        void *q = nullptr;
        cudaError_t e = pool ? cudaMallocFromPoolAsync(&q, std::max<size_t>(bytes, 256), pool, stream)
                             : cudaMallocAsync(&q, std::max<size_t>(bytes, 256), stream);
        if (e == cudaSuccess) {
            allocations.push_back(q);
            *p = static_cast<P *>(q);
        }
        return e;
    }
    template <typename P>
    cudaError_t upload(P **p, const void *src, size_t bytes) {
        cudaError_t e = alloc(p, bytes);
        if (e != cudaSuccess || bytes == 0) return e;
        return cudaMemcpyAsync(*p, src, bytes, cudaMemcpyHostToDevice, stream);
    }

    bool bits() const {
        return !faith && !spec.vaw &&
               (spec.method == Method::unweighted || spec.method == Method::unweighted_unnormalized);
    }
    bool timed() const { return timing && !capturing; }

    int setup(const TableSet &set, const FlatTree &tree, const BatchOptions &opts);
    template <typename T>
    int setup_method();
    template <typename T>
    int tune(std::vector<PairKernel<T>> &cands, size_t &chosen);
    template <typename T>
    int embed(cudaStream_t s, const Group &g);
    template <typename T>
    int prepare(cudaStream_t s, const Group &g);
    template <typename T>
    int pair_stage(cudaStream_t s, const Group &g, const dev::OutSpec &out, const uint4 *tiles, uint32_t n_tiles,
                   uint32_t splits, uint32_t rows_per_split, bool last);
    template <typename T>
    void choose_splits(const PairKernel<T> &k, uint32_t tiles, uint32_t &splits, uint32_t &rows_per_split) const;
    template <typename T>
    int execute_T(cudaStream_t s, const dev::OutSpec &out);
    int execute_all(cudaStream_t s);
    int run_windowed(int mode, void *d_out, uint32_t start, uint32_t stop);
    void zero_diagonal(cudaStream_t s, void *out);
};

template <>
PairKernel<double> &PlanImpl::kern<double>() {
    return kd;
}
template <>
PairKernel<float> &PlanImpl::kern<float>() {
    return kf;
}

int PlanImpl::setup(const TableSet &set, const FlatTree &tree, const BatchOptions &opts) {
    SetupTimer timer;
    const uint32_t n_tables = static_cast<uint32_t>(set.tables.size());
    K = tree.n_nodes;
    E = faith ? tree.n_nodes : tree.n_embedded;
    int dev_id = 0;
    SSU_CK(cudaGetDevice(&dev_id));
    SSU_CK(cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, dev_id));
    pool = device_pool(dev_id);
    if (!stream) {
        SSU_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        own_stream = true;
    }

    // table descriptors and the concatenated CSR
    tdesc.assign(n_tables, dev::TableDesc{});
    table_E.assign(n_tables, E);
    uint64_t nnz_total = 0, indptr_total = 0;
    full_elems = 0;
    for (uint32_t t = 0; t < n_tables; t++) {
        const Table &tb = *set.tables[t];
        if (!tb.nonneg) nonneg_data = false;
        dev::TableDesc &d = tdesc[t];
        d.n = tb.n_samples;
        d.out_off = full_elems;
        d.nnz_off = nnz_total;
        d.indptr_off = static_cast<uint32_t>(indptr_total);
        full_elems += static_cast<uint64_t>(tb.n_samples) * tb.n_samples;
        nnz_total += tb.nnz();
        indptr_total += static_cast<uint64_t>(tb.n_obs) + 1;
        n += tb.n_samples;
        max_table_n = std::max(max_table_n, tb.n_samples);
        if (!set.embedded.empty()) table_E[t] = set.embedded[t];
    }
    if (indptr_total > UINT32_MAX) {
        last_error = "too many observations in one plan";
        return kOutputError;
    }
    SSU_CK(alloc(&d_indptr, sizeof(uint32_t) * indptr_total));
    SSU_CK(alloc(&d_indices, sizeof(uint32_t) * nnz_total));
    SSU_CK(alloc(&d_data, sizeof(double) * nnz_total));
    {
        std::vector<HostPiece> pieces;
        for (uint32_t t = 0; t < n_tables; t++) {
            const Table &tb = *set.tables[t];
            const dev::TableDesc &d = tdesc[t];
            pieces.push_back({d_indptr + d.indptr_off, tb.indptr, sizeof(uint32_t) * (tb.n_obs + 1)});
            pieces.push_back({d_indices + d.nnz_off, tb.indices, sizeof(uint32_t) * tb.nnz()});
            pieces.push_back({d_data + d.nnz_off, tb.data, sizeof(double) * tb.nnz()});
        }
        SSU_CK(Staging::get().upload(pieces, stream, dev_id));
    }

    timer.step("csr_upload");
    // groups of tables whose embedding fits the budget together
    const size_t el = (spec.fp64 || faith) ? sizeof(double) : sizeof(float);
    n_words = bits() ? (E + 63) / 64 : 0;
    if (!faith && !spec.vaw && spec.method == Method::weighted_normalized) {
        part_chunk = 512;
        n_parts = std::max<uint32_t>(1, (E + part_chunk - 1) / part_chunk);
    }
    const bool counts = spec.vaw && !faith;
    size_t per_col = el * std::max<uint32_t>(K, 1) * (counts ? 2 : 1) + sizeof(double) + (counts ? el : 0) +
                     sizeof(unsigned long long) * n_words + (n_parts ? el * (n_parts + 1) : 0);
    if (gemm) {
        // 8-bit operand rows (A0, A1, B0, B1) over the padded nodes (chunk
        // padding included, allowing for 128 chunks) and r
        const uint64_t kp = (static_cast<uint64_t>(E) + tc::BLOCK_K - 1) / tc::BLOCK_K * tc::BLOCK_K + 128 * tc::BLOCK_K;
        per_col = 2 * tc::PRODUCTS * kp + sizeof(double);
    }
    size_t budget = opts.group_bytes;
    if (!budget) {
        if (const char *b = std::getenv("UNIFRAC_B200_GROUP_BYTES")) budget = std::strtoull(b, nullptr, 10);
    }
    if (!budget && n_tables > 1) {  // one table is one group whatever the budget
        size_t free_b = 0, total_b = 0;
        SSU_CK(cudaMemGetInfo(&free_b, &total_b));
        // (fp32 weighted plans also hold the pair-scatter sums: 8 bytes per result)
        const bool weighted = spec.method == Method::weighted_normalized || spec.method == Method::weighted_unnormalized;
        const size_t fixed = el * full_elems + 12 * nnz_total + (weighted && !spec.fp64 && !faith ? 8 * full_elems : 0);
        budget = free_b > fixed ? (free_b - fixed) / 2 : 0;
    }
    uint64_t max_cols = std::max<uint64_t>(128, budget / per_col);
    // the hybrid weighted kernel gathers rows at random: narrow groups keep
    // its rows close in memory (measured on 20 replicates of 5,000 samples:
    // 414 ms as one 100k-column group, 377 ms as 5k-column groups)
    hybrid = !faith && !gemm && !spec.vaw && nonneg_data && set.row_active.empty() &&
             (spec.method == Method::weighted_normalized || spec.method == Method::weighted_unnormalized);
    if (const char *m = std::getenv("UNIFRAC_B200_WEIGHTED_MODE"))
        if (std::string(m) == "dense") hybrid = false;
    // generalized and variance-adjusted methods: only the union of the two
    // samples' supports adds to a pair (needs u >= 0 so presence is u > 0)
    union_mode = !faith && !gemm && nonneg_data && set.row_active.empty() &&
                 (spec.vaw || spec.method == Method::generalized);
    if (const char *m = std::getenv("UNIFRAC_B200_UNION_MODE"))
        if (std::string(m) == "dense") union_mode = false;
    // Sparse-kernel groups hold as many tables as the memory budget allows:
    // the whole batch in one embedding pass and one persistent pair launch
    // where it fits (100 config-4 replicates: 1,440 ms as one group against
    // 1,432 ms as 100 groups of one; 64 config-5 tables: generalized 1,449
    // against 1,468 ms as 10 groups of <= 8,192 columns, VAW weighted 1,822
    // against 1,847 ms).  UNIFRAC_B200_SPARSE_GROUP_COLS caps their columns.
    if ((hybrid || union_mode) && env_int("UNIFRAC_B200_SPARSE_GROUP_COLS", 0) > 0) {
        const uint64_t cap = static_cast<uint64_t>(std::max(128, env_int("UNIFRAC_B200_SPARSE_GROUP_COLS", 0)));
        max_cols = std::min<uint64_t>(max_cols, std::max<uint64_t>(cap, (max_table_n + 127) / 128 * 128));
    }
    groups.clear();
    uint64_t cols = 0;
    for (uint32_t t = 0; t < n_tables; t++) {
        const uint64_t w = std::max<uint64_t>(128, (static_cast<uint64_t>(tdesc[t].n) + 127) / 128 * 128);
        if (groups.empty() || (cols > 0 && cols + w > max_cols)) {
            if (!groups.empty()) groups.back().ld = cols;
            groups.emplace_back();
            groups.back().t0 = t;
            cols = 0;
        }
        tdesc[t].base = static_cast<uint32_t>(cols);
        cols += w;
        groups.back().t1 = t + 1;
    }
    if (groups.empty()) groups.emplace_back();
    groups.back().ld = std::max<uint64_t>(cols, 128);
    ld = 0;
    for (const Group &g : groups) ld = std::max(ld, g.ld);
    if (ld > UINT32_MAX) {
        last_error = "too many samples in one group";
        return kOutputError;
    }

    // per group: the tips' rows in each table, the per-column totals
    n_tips = static_cast<uint32_t>(tree.leaf_rows.size());
    const bool per_table_len = !faith && !set.row_active.empty();
    for (Group &g : groups) {
        const uint32_t tg = g.t1 - g.t0;
        std::vector<int32_t> tip_obs(static_cast<size_t>(n_tips) * std::max<uint32_t>(tg, 1), -1);
        for (uint32_t i = 0; i < n_tips; i++) {
            const int32_t o = tree.leaf_obs[tree.leaf_rows[i]];
            for (uint32_t j = 0; j < tg; j++) {
                int32_t v = o;
                if (!set.obs_row.empty()) {
                    const std::vector<int32_t> &m = set.obs_row[g.t0 + j];
                    v = (o >= 0 && static_cast<size_t>(o) < m.size()) ? m[o] : -1;
                }
                tip_obs[static_cast<size_t>(i) * tg + j] = v;
            }
        }
        SSU_CK(upload(&g.d_tip_obs, tip_obs.data(), sizeof(int32_t) * tip_obs.size()));
        g.totals.assign(g.ld, 0.0);
        for (uint32_t t = g.t0; t < g.t1; t++)
            std::copy(set.tables[t]->totals.begin(), set.tables[t]->totals.end(), g.totals.begin() + tdesc[t].base);
        SSU_CK(upload(&g.d_totals, g.totals.data(), sizeof(double) * g.ld));
        if (per_table_len) {
            std::vector<uint32_t> bt(g.ld / 128, 0);
            for (uint32_t t = g.t0; t < g.t1; t++) {
                const uint64_t w = std::max<uint64_t>(128, (static_cast<uint64_t>(tdesc[t].n) + 127) / 128 * 128);
                for (uint64_t c = tdesc[t].base / 128; c < (tdesc[t].base + w) / 128; c++) bt[c] = t;
            }
            SSU_CK(upload(&g.d_block_table, bt.data(), sizeof(uint32_t) * bt.size()));
        }
    }
    SSU_CK(upload(&d_tdesc, tdesc.data(), sizeof(dev::TableDesc) * std::max<uint32_t>(n_tables, 1)));
    timer.step("groups");

    // tree
    SSU_CK(upload(&d_tip_rows, tree.leaf_rows.data(), sizeof(uint32_t) * n_tips));
    SSU_CK(upload(&d_child_ptr, tree.child_ptr.data(), sizeof(uint32_t) * tree.child_ptr.size()));
    SSU_CK(upload(&d_child_rows, tree.child_rows.data(), sizeof(uint32_t) * tree.child_rows.size()));
    SSU_CK(upload(&d_level_rows, tree.level_rows.data(), sizeof(uint32_t) * tree.level_rows.size()));
    level_ptr = tree.level_ptr;
    if (faith) {
        SSU_CK(upload(&d_post_rows, tree.postorder_row.data(), sizeof(uint32_t) * tree.postorder_row.size()));
        SSU_CK(upload(&d_len_rows, tree.length.data(), sizeof(double) * tree.length.size()));
    }
    // embedded lengths in T, rows [0, E); per table (zero where a row is
    // not embedded in that table's own tree) with bypassed tips in a batch
    host_len.assign(tree.length.begin(), tree.length.begin() + E);
    const uint32_t n_len = per_table_len ? n_tables : 1;
    len_stride = per_table_len ? E : 0;
    if (spec.fp64 || faith) {
        std::vector<double> len(static_cast<size_t>(E) * n_len);
        for (uint32_t t = 0; t < n_len; t++)
            for (uint32_t e = 0; e < E; e++)
                len[static_cast<size_t>(t) * E + e] = (!per_table_len || set.row_active[t][e]) ? host_len[e] : 0.0;
        SSU_CK(upload(reinterpret_cast<double **>(&d_len), len.data(), sizeof(double) * len.size()));
    } else {
        std::vector<float> len(static_cast<size_t>(E) * n_len);
        for (uint32_t t = 0; t < n_len; t++)
            for (uint32_t e = 0; e < E; e++)
                len[static_cast<size_t>(t) * E + e] =
                    (!per_table_len || set.row_active[t][e]) ? static_cast<float>(host_len[e]) : 0.0f;
        SSU_CK(upload(reinterpret_cast<float **>(&d_len), len.data(), sizeof(float) * len.size()));
    }
    for (auto &e : ev) SSU_CK(cudaEventCreate(&e));
    timer.step("tree_upload");
    return 0;
}

template <typename T>
void PlanImpl::choose_splits(const PairKernel<T> &k, uint32_t tiles, uint32_t &out_splits,
                             uint32_t &out_rows) const {
    const uint32_t units = bits() ? n_words : E;
    const uint32_t q = static_cast<uint32_t>(k.row_quantum);
    const uint32_t slots = static_cast<uint32_t>(std::max(1, n_sms * k.blocks_per_sm));
    uint32_t best_s = 1;
    double best_cost = 1e300;
    const uint32_t max_s = std::max<uint32_t>(1, std::min<uint32_t>(64, units / (8 * q)));
    for (uint32_t s = 1; s <= max_s; s++) {
        const double ctas = static_cast<double>(tiles) * s;
        const double waves = std::ceil(ctas / slots);
        const double cost = waves / s * (1.0 + 0.005 * (s - 1));
        if (cost < best_cost - 1e-12) {
            best_cost = cost;
            best_s = s;
        }
    }
    uint32_t rows = units ? (units + best_s - 1) / best_s : 0;
    rows = ((rows + q - 1) / q) * q;
    out_rows = rows;
    out_splits = rows ? (units + rows - 1) / rows : 1;
    if (out_splits == 0) out_splits = 1;
}

template <typename T>
int PlanImpl::setup_method() {
    std::vector<PairKernel<T>> cands;
    for (PairKernel<T> k : pair_candidates<T>(spec)) {
        int bps = 0;
        if (k.configure(k.smem) != cudaSuccess || k.occupancy(&bps, k.threads, k.smem) != cudaSuccess || bps < 1) {
            cudaGetLastError();
            continue;
        }
        k.blocks_per_sm = bps;
        cands.push_back(k);
    }
    if (cands.empty()) {
        last_error = "pair kernel does not fit on the device";
        return kOutputError;
    }
    const uint32_t n_tables = static_cast<uint32_t>(tdesc.size());

    const size_t rowbytes = sizeof(T) * ld;
    SSU_CK(alloc(&d_U, rowbytes * std::max<uint32_t>(K, 1)));
    if (spec.vaw) {
        SSU_CK(alloc(&d_C, rowbytes * std::max<uint32_t>(K, 1)));
        for (Group &g : groups) {
            std::vector<T> tot(g.ld, T(0));
            for (uint64_t j = 0; j < g.ld; j++) tot[j] = static_cast<T>(g.totals[j]);
            SSU_CK(upload(reinterpret_cast<T **>(&g.d_tot), tot.data(), sizeof(T) * g.ld));
        }
    }
    if (bits()) {
        const uint32_t n_lut = len_stride ? n_tables : 1;
        lut_stride = len_stride ? static_cast<uint64_t>(2048) * n_words : 0;
        SSU_CK(alloc(&d_P, sizeof(unsigned long long) * ld * std::max<uint32_t>(n_words, 1)));
        SSU_CK(alloc(&d_lut, sizeof(T) * 2048 * std::max<uint32_t>(n_words, 1) * n_lut));
        if (n_words) {
            dev::build_lut_kernel<T><<<dim3(n_words * 8, n_lut), 256, 0, stream>>>(
                static_cast<const T *>(d_len), E, static_cast<T *>(d_lut), len_stride, lut_stride);
            SSU_CK(cudaGetLastError());
        }
    }
    if (n_parts) {
        SSU_CK(alloc(&d_W, sizeof(T) * ld));
        SSU_CK(alloc(&d_part, sizeof(T) * ld * n_parts));
    }
    SSU_CK(alloc(&d_full, sizeof(T) * std::max<uint64_t>(full_elems, 1)));

    size_t chosen = 0;
    // `hybrid` was settled by setup(): weighted methods with counts >= 0
    // (min(a, b) = 0 off the intersection of the supports), both precisions
    // (the fp32 form accumulates in fp64 too; measured on 2,048 samples x 40k
    // nodes: 6.1 ms against 7.4 ms for the fp32 dense kernel)
    if (hybrid) {
        // the exact recomputation of flagged tiles runs the 128 x 128 shape
        chosen = 0;
        tuning = "sparse hybrid";
    } else if (union_mode) {
        tuning = "sparse union";
    } else if (cands.size() > 1 && autotune == 1) {
        const int rc = tune<T>(cands, chosen);
        if (rc) return rc;
    }
    kern<T>() = cands[chosen];
    const PairKernel<T> &k = kern<T>();
    if (hybrid) return setup_hybrid<T>();
    if (union_mode) return setup_union<T>();

    partial_bytes = 0;
    for (Group &g : groups) {
        std::vector<uint4> tiles;
        for (uint32_t t = g.t0; t < g.t1; t++) append_tiles(tiles, t, tdesc[t].base, tdesc[t].n, k.BM, k.BN, false, 0, 0);
        g.n_tiles = static_cast<uint32_t>(tiles.size());
        SSU_CK(upload(&g.d_tiles, tiles.data(), sizeof(uint4) * tiles.size()));
        choose_splits<T>(k, g.n_tiles, g.splits, g.rows_per_split);
        if (g.splits > 1)
            partial_bytes = std::max(partial_bytes, sizeof(T) * k.partial_per_tile * g.n_tiles * g.splits);
    }
    if (partial_bytes) SSU_CK(alloc(&d_partial, partial_bytes));
    return 0;
}

template <typename T>
int PlanImpl::setup_hybrid() {
    hybrid_div = static_cast<uint32_t>(std::max(1, env_int("UNIFRAC_B200_HYBRID_DIV", 8)));
    if (const int rc = sparse_prep_alloc()) return rc;
    SSU_CK(alloc(&d_Ws, sizeof(double) * ld));
    part_chunk = part_chunk ? part_chunk : 512;
    n_parts = std::max<uint32_t>(1, (E + part_chunk - 1) / part_chunk);
    SSU_CK(alloc(&d_ws_part, sizeof(double) * ld * n_parts));
    // UNIFRAC_B200_DETERMINISTIC=1: fp32 plans also take the owner walk, so
    // their results repeat bit for bit (about 13% slower on replicate tables)
    hybrid_atomic = sizeof(T) == 4 && !env_int("UNIFRAC_B200_DETERMINISTIC", 0);
    // UNIFRAC_B200_HYBRID_SCATTER=0: the tile kernel walks the sparse rows
    // itself instead of reading per-pair sums
    hybrid_scatter = env_int("UNIFRAC_B200_HYBRID_SCATTER", 1) != 0;
    if (hybrid_scatter) {
        // no pair's sum of L min(a, b) exceeds the sum of |L| over the
        // embedded rows times the largest embedded value: 1 for proportions,
        // the largest sample total for raw counts.  The unit 2^-s keeps
        // every sum below 2^62.
        double vmax = 1.0;
        if (!spec.normalize)
            for (const Group &g : groups)
                for (double t : g.totals) vmax = std::max(vmax, std::fabs(t));
        double bound = 0.0;
        for (uint32_t e = 0; e < E; e++) bound += std::fabs(host_len[e]);
        bound *= vmax * (1.0 + 1e-12);
        const int s2 = 62 - static_cast<int>(std::ceil(std::log2(std::max(bound, 1e-300))));
        sq_scale = std::ldexp(1.0, std::min(s2, 1000));
        if (sizeof(T) == sizeof(double))
            d_Sq = static_cast<unsigned long long *>(d_full);  // written only after its sum is read
        else
            SSU_CK(alloc(&d_Sq, sizeof(unsigned long long) * std::max<uint64_t>(full_elems, 1)));
        SSU_CK(alloc(&d_sc_next, sizeof(unsigned long long)));
        if (const char *b = std::getenv("UNIFRAC_B200_SCATTER_BAND_BYTES"))
            scatter_band_bytes = std::strtoull(b, nullptr, 10);
    }
    const int smem = static_cast<int>(dev::hybrid_smem<T>());
    SSU_CK(cudaFuncSetAttribute(dev::pair_hybrid_kernel<T, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem));
    SSU_CK(cudaFuncSetAttribute(dev::pair_hybrid_kernel<T, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem));
    SSU_CK(cudaFuncSetAttribute(dev::pair_hybrid_kernel<T, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem));
    SSU_CK(cudaFuncSetAttribute(dev::pair_hybrid_kernel<T, false, false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    uint32_t max_tiles = 0;
    hpartial_bytes = 0;
    for (Group &g : groups) {
        std::vector<uint4> tiles;
        for (uint32_t t = g.t0; t < g.t1; t++) append_tiles(tiles, t, tdesc[t].base, tdesc[t].n, dev::HB, dev::HB, false, 0, 0);
        g.n_tiles = static_cast<uint32_t>(tiles.size());
        SSU_CK(upload(&g.d_tiles, tiles.data(), sizeof(uint4) * tiles.size()));
        // node splits so the tiles fill the SMs (one CTA per SM)
        uint32_t best_s = 1;
        double best = 1e300;
        const uint32_t max_s = std::max<uint32_t>(1, std::min<uint32_t>(64, E / 128));
        for (uint32_t sp = 1; sp <= max_s; sp++) {
            const double cost = std::ceil(static_cast<double>(g.n_tiles) * sp / n_sms) / sp * (1.0 + 0.02 * (sp - 1));
            if (cost < best - 1e-12) {
                best = cost;
                best_s = sp;
            }
        }
        g.splits = best_s;
        max_tiles = std::max(max_tiles, g.n_tiles);
        if (g.splits > 1)
            hpartial_bytes = std::max(hpartial_bytes, sizeof(double) * dev::HB * dev::HB * g.n_tiles * g.splits);
    }
    SSU_CK(alloc(&d_flags, sizeof(int) * std::max<uint32_t>(max_tiles, 1)));
    if (hpartial_bytes) SSU_CK(alloc(&d_hpartial, hpartial_bytes));
    return 0;
}

// Hybrid weighted pair stage of one group (its embedding and W ready):
// masks and counts, dense / sparse row lists, sparse one-sided sums, the
// hybrid tile kernel (+ split finalize), then the exact dense kernel on the
// tiles it flagged.
template <typename T>
int PlanImpl::hybrid_stage(cudaStream_t s, const Group &g, const dev::OutSpec &out, const uint4 *tiles,
                           uint32_t ntiles, uint32_t splits, bool last) {
    const T *U = static_cast<const T *>(d_U);
    if (const int rc = sparse_prep<T>(s, g, hybrid_div)) return rc;
    if (d_W) {
        // weighted normalized: W and Ws in one pass over the embedding
        dim3 grid(static_cast<uint32_t>((g.ld + 127) / 128), n_parts);
        dev::hybrid_sums_partial_kernel<T><<<grid, 128, 0, s>>>(U, static_cast<const T *>(d_len), d_row_class, E,
                                                                g.ld, part_chunk, static_cast<T *>(d_part), d_ws_part);
        dev::reduce_partials_kernel<T><<<static_cast<uint32_t>((g.ld + 255) / 256), 256, 0, s>>>(
            static_cast<const T *>(d_part), n_parts, g.ld, static_cast<T *>(d_W));
        launches += 2;
    } else {
        // weighted unnormalized: Ws only, reading the sparse rows alone
        dim3 grid(static_cast<uint32_t>((g.ld + 255) / 256), n_parts);
        dev::sparse_sums_partial_kernel<T><<<grid, 256, 0, s>>>(U, static_cast<const T *>(d_len), d_sparse_rows,
                                                                d_nrows, g.ld, part_chunk, d_ws_part);
        launches++;
    }
    dev::reduce_partials_kernel<double><<<static_cast<uint32_t>((g.ld + 255) / 256), 256, 0, s>>>(
        d_ws_part, n_parts, g.ld, d_Ws);
    launches++;
    if (ntiles == 0) return 0;
    SSU_CK(cudaMemsetAsync(d_flags, 0, sizeof(int) * ntiles, s));
    if (hybrid_scatter) {
        dev::ScatterArgs<T> sa{};
        sa.next = d_sc_next;
        sa.sparse_rows = d_sparse_rows;
        sa.n_rows = d_nrows;
        sa.masks = d_masks;
        sa.E = E;
        sa.tables = d_tdesc;
        sa.U = U;
        sa.len = static_cast<const T *>(d_len);
        sa.ld = g.ld;
        sa.Sq = d_Sq;
        sa.scale = sq_scale;
        // one table at a time, its sums zeroed just before: the zeroing leaves
        // the table's sums partly in L2 for the atomics that follow (100
        // config-4 replicates, weighted fp32: 645 ms per step against 836 ms
        // with every table zeroed first and one launch over all of them)
        for (uint32_t t = g.t0; t < g.t1; t++) {
            const uint64_t nt = tdesc[t].n;
            SSU_CK(cudaMemsetAsync(d_Sq + tdesc[t].out_off, 0, sizeof(unsigned long long) * nt * nt, s));
            SSU_CK(cudaMemsetAsync(d_sc_next, 0, sizeof(unsigned long long), s));
            sa.t0 = t;
            sa.n_tables = 1;
            // bands of rows k whose sums fit L2 well (at most 16 bands)
            uint64_t br = std::max<uint64_t>(nt, 1);
            if (scatter_band_bytes && nt * nt * 8 > scatter_band_bytes)
                br = std::max<uint64_t>({64, scatter_band_bytes / (8 * nt), (nt + 15) / 16});
            sa.band_rows = static_cast<uint32_t>(br);
            sa.n_bands = static_cast<uint32_t>((std::max<uint64_t>(nt, 1) + br - 1) / br);
            dev::sparse_pairs_kernel<T><<<static_cast<uint32_t>(n_sms) * 8, dev::SC_WARPS * 32, 0, s>>>(sa);
            launches++;
        }
    }
    dev::HybridArgs<T> h{};
    h.tiles = tiles;
    h.n_tiles = ntiles;
    h.n_splits = std::max<uint32_t>(splits, 1);
    h.tables = d_tdesc;
    h.U = U;
    h.len = static_cast<const T *>(d_len);
    h.masks = d_masks;
    h.row_class = d_row_class;
    h.E = E;
    h.ld = g.ld;
    h.dense_rows = d_dense_rows;
    h.n_rows = d_nrows;
    h.W = static_cast<const T *>(d_W);
    h.Ws = d_Ws;
    h.tau = 0.02;
    h.tile_flags = d_flags;
    h.partial = h.n_splits > 1 ? d_hpartial : nullptr;
    if (h.n_splits > 1 && sizeof(double) * dev::HB * dev::HB * ntiles * h.n_splits > hpartial_bytes) {
        h.n_splits = 1;
        h.partial = nullptr;
    }
    h.out = out;
    h.Sq = hybrid_scatter ? d_Sq : nullptr;
    h.sq_unit = 1.0 / sq_scale;
    const bool norm = spec.method == Method::weighted_normalized;
    const uint32_t ctas = static_cast<uint32_t>(
        std::min<uint64_t>(static_cast<uint64_t>(ntiles) * h.n_splits, static_cast<uint64_t>(n_sms)));
    const size_t smem = dev::hybrid_smem<T>();
    if (norm && hybrid_atomic)
        dev::pair_hybrid_kernel<T, true, true><<<ctas, dev::HTHREADS, smem, s>>>(h);
    else if (norm)
        dev::pair_hybrid_kernel<T, true, false><<<ctas, dev::HTHREADS, smem, s>>>(h);
    else if (hybrid_atomic)
        dev::pair_hybrid_kernel<T, false, true><<<ctas, dev::HTHREADS, smem, s>>>(h);
    else
        dev::pair_hybrid_kernel<T, false, false><<<ctas, dev::HTHREADS, smem, s>>>(h);
    launches++;
    if (h.partial) {
        if (norm)
            dev::hybrid_finalize_kernel<T, true><<<ntiles, dev::HTHREADS, 0, s>>>(h);
        else
            dev::hybrid_finalize_kernel<T, false><<<ntiles, dev::HTHREADS, 0, s>>>(h);
        launches++;
    }
    if (last && timed()) SSU_CK(cudaEventRecord(ev[2], s));
    // exact |a - b| recomputation of the flagged tiles (all nodes)
    const PairKernel<T> &k = kern<T>();
    dev::PairArgs<T> a{};
    a.tiles = tiles;
    a.n_tiles = ntiles;
    a.n_splits = 1;
    a.tables = d_tdesc;
    a.U = U;
    a.len = static_cast<const T *>(d_len);
    a.W = static_cast<const T *>(d_W);
    a.E = E;
    a.ld = g.ld;
    a.rows_per_split = E;
    a.out = out;
    a.tile_flags = d_flags;
    k.launch(a, static_cast<uint32_t>(std::min<uint64_t>(ntiles, static_cast<uint64_t>(n_sms) * k.blocks_per_sm)),
             k.smem, s);
    launches++;
    SSU_CK(cudaGetLastError());
    return 0;
}

// Buffers of the per-call row classification shared by the hybrid and union
// paths: word-major presence masks, non-zero counts, classes, row lists.
int PlanImpl::sparse_prep_alloc() {
    const uint64_t words = ld / 64;
    SSU_CK(alloc(&d_masks, sizeof(unsigned long long) * std::max<uint64_t>(static_cast<uint64_t>(E) * words, 1)));
    SSU_CK(alloc(&d_counts, sizeof(uint32_t) * std::max<uint32_t>(E, 1)));
    SSU_CK(alloc(&d_row_class, std::max<uint32_t>(E, 1)));
    SSU_CK(alloc(&d_dense_rows, sizeof(uint32_t) * std::max<uint32_t>(E, 1)));
    SSU_CK(alloc(&d_sparse_rows, sizeof(uint32_t) * std::max<uint32_t>(E, 1)));
    SSU_CK(alloc(&d_nrows, sizeof(uint32_t) * 2));
    return 0;
}

// Row classes of the group's embedding (dense: non-zero in more than ld / div
// columns), from the counts the embedding wrote with the masks.
template <typename T>
int PlanImpl::sparse_prep(cudaStream_t s, const Group &g, uint32_t div) {
    if (!E) SSU_CK(cudaMemsetAsync(d_counts, 0, sizeof(uint32_t), s));
    dev::classify_rows_kernel<<<1, 1024, 0, s>>>(d_counts, E, static_cast<uint32_t>(g.ld / div), d_dense_rows,
                                                 d_sparse_rows, d_row_class, d_nrows);
    launches++;
    SSU_CK(cudaGetLastError());
    return 0;
}

template <typename T>
int PlanImpl::setup_union() {
    if (const char *w = std::getenv("UNIFRAC_B200_WAIT_CYCLES")) union_wait_cycles = std::max(0LL, std::atoll(w));
    union_stall = env_int("UNIFRAC_B200_TEST_STALL", 0) ? 1 : 0;
    if (const int rc = sparse_prep_alloc()) return rc;
    size_t smem = 0;
    SSU_CK(dev::union_configure<T>(spec, &smem));
    upartial_bytes = 0;
    for (Group &g : groups) {
        std::vector<uint4> tiles;
        for (uint32_t t = g.t0; t < g.t1; t++)
            append_tiles(tiles, t, tdesc[t].base, tdesc[t].n, dev::UT, dev::UT, false, 0, 0);
        g.n_tiles = static_cast<uint32_t>(tiles.size());
        SSU_CK(upload(&g.d_tiles, tiles.data(), sizeof(uint4) * tiles.size()));
        // node splits so the tiles fill the SMs (one CTA per SM)
        uint32_t best_s = 1;
        double best = 1e300;
        const uint32_t max_s = std::max<uint32_t>(1, std::min<uint32_t>(64, E / 128));
        for (uint32_t sp = 1; sp <= max_s; sp++) {
            const double cost = std::ceil(static_cast<double>(g.n_tiles) * sp / n_sms) / sp * (1.0 + 0.02 * (sp - 1));
            if (cost < best - 1e-12) {
                best = cost;
                best_s = sp;
            }
        }
        g.splits = best_s;
        if (g.splits > 1)
            upartial_bytes = std::max(upartial_bytes, sizeof(double) * 2 * dev::UT * dev::UT * g.n_tiles * g.splits);
    }
    if (upartial_bytes) SSU_CK(alloc(&d_upartial, upartial_bytes));
    // branch lengths in T, zero-padded to whole stages (a stage copies 16)
    std::vector<T> lens((static_cast<size_t>(E) + dev::URS - 1) / dev::URS * dev::URS + dev::URS, T(0));
    for (uint32_t e = 0; e < E; e++) lens[e] = static_cast<T>(host_len[e]);
    SSU_CK(upload(reinterpret_cast<T **>(&d_slen), lens.data(), sizeof(T) * lens.size()));
    if (!d_error) {
        SSU_CK(alloc(&d_error, sizeof(int)));
        SSU_CK(cudaMemsetAsync(d_error, 0, sizeof(int), stream));
    }
    return 0;
}

// Union pair stage of one group (its embedding and presence words ready):
// the union tile kernel (+ split finalize) over 2-D maps of the group's
// proportions and counts.
template <typename T>
int PlanImpl::union_stage(cudaStream_t s, const Group &g, const dev::OutSpec &out, const uint4 *tiles,
                          uint32_t ntiles, uint32_t splits, bool last) {
    if (ntiles == 0) return 0;
    CUtensorMap tmU{}, tmC{};
    if (!make_rows_map<T>(&tmU, d_U, E, g.ld) || (spec.vaw && !make_rows_map<T>(&tmC, d_C, E, g.ld))) {
        last_error = "cuTensorMapEncodeTiled failed";
        return kOutputError;
    }
    dev::UnionArgs<T> u{};
    u.tiles = tiles;
    u.n_tiles = ntiles;
    u.n_splits = std::max<uint32_t>(splits, 1);
    if (u.n_splits > 1 && sizeof(double) * 2 * dev::UT * dev::UT * ntiles * u.n_splits > upartial_bytes)
        u.n_splits = 1;
    u.tables = d_tdesc;
    u.tot = static_cast<const T *>(g.d_tot);
    u.len = static_cast<const T *>(d_slen);
    u.masks = d_masks;
    u.E = E;
    u.ld = g.ld;
    u.alpha = spec.alpha;
    u.partial = u.n_splits > 1 ? d_upartial : nullptr;
    u.out = out;
    u.error = d_error;
    u.wait_cycles = union_wait_cycles;
    u.stall = union_stall;
    const uint32_t ctas = static_cast<uint32_t>(
        std::min<uint64_t>(static_cast<uint64_t>(ntiles) * u.n_splits, static_cast<uint64_t>(n_sms)));
    SSU_CK(dev::union_launch<T>(spec, tmU, spec.vaw ? tmC : tmU, u, ctas, s));
    launches += u.partial ? 2 : 1;
    if (last && timed()) SSU_CK(cudaEventRecord(ev[2], s));
    return 0;
}

// Pick the tile shape: predicted pair-stage time = waves x (time of one
// full wave of the shape over a probe of node rows, measured on the plan's
// own group-0 data) x (rows per split / probe rows).
template <typename T>
int PlanImpl::tune(std::vector<PairKernel<T>> &cands, size_t &chosen) {
    const Group &g = groups[0];
    const std::string key = std::string(cands[0].name) + (sizeof(T) == 8 ? "|f64" : "|f32") + "|a" +
                            std::to_string(alpha_kind(spec.alpha)) + "|E" + std::to_string(log2_bucket(E)) + "|c" +
                            std::to_string(log2_bucket(g.ld)) + "|n" + std::to_string(log2_bucket(max_table_n)) +
                            "|sm" + std::to_string(n_sms);
    std::string shape;
    if (TuneCache::get().find(key, shape)) {
        for (size_t i = 0; i < cands.size(); i++)
            if (shape == cands[i].shape) {
                chosen = i;
                tuning = "cache " + shape;
                return 0;
            }
    }
    int rc = embed<T>(stream, g);
    if (!rc) rc = prepare<T>(stream, g);
    if (rc) return rc;
    cudaEvent_t a = nullptr, b = nullptr;
    SSU_CK(cudaEventCreate(&a));
    SSU_CK(cudaEventCreate(&b));
    const uint32_t units = bits() ? n_words : E;
    double best = 1e300;
    std::string report;
    for (size_t i = 0; i < cands.size(); i++) {
        const PairKernel<T> &k = cands[i];
        std::vector<uint4> tiles;
        for (uint32_t t = g.t0; t < g.t1; t++) append_tiles(tiles, t, tdesc[t].base, tdesc[t].n, k.BM, k.BN, false, 0, 0);
        if (tiles.empty() || units == 0) continue;
        uint4 *d_t = nullptr;
        SSU_CK(upload(&d_t, tiles.data(), sizeof(uint4) * tiles.size()));
        uint32_t splits = 1, rows = 0;
        choose_splits<T>(k, static_cast<uint32_t>(tiles.size()), splits, rows);
        const uint32_t slots = static_cast<uint32_t>(std::max(1, n_sms * k.blocks_per_sm));
        const uint32_t q = static_cast<uint32_t>(k.row_quantum);
        uint32_t probe = std::min<uint32_t>(units, bits() ? 32 : 2048);
        probe = std::max<uint32_t>(q, probe / q * q);
        dev::PairArgs<T> pa{};
        pa.tiles = d_t;
        pa.n_tiles = std::min<uint32_t>(static_cast<uint32_t>(tiles.size()), slots);
        pa.n_splits = 1;
        pa.tables = d_tdesc;
        pa.U = static_cast<const T *>(d_U);
        pa.C = static_cast<const T *>(d_C);
        pa.len = static_cast<const T *>(d_len);
        pa.len_stride = len_stride;
        pa.tot = static_cast<const T *>(g.d_tot);
        pa.W = static_cast<const T *>(d_W);
        pa.P = d_P;
        pa.lut = static_cast<const T *>(d_lut);
        pa.lut_stride = lut_stride;
        pa.E = units;
        pa.ld = g.ld;
        pa.rows_per_split = probe;
        pa.alpha = static_cast<T>(spec.alpha);
        pa.out = dev::OutSpec{0, d_full, 0, 0};
        pa.partial = nullptr;
        k.launch(pa, pa.n_tiles, k.smem, stream);
        SSU_CK(cudaEventRecord(a, stream));
        for (int r = 0; r < 3; r++) k.launch(pa, pa.n_tiles, k.smem, stream);
        SSU_CK(cudaEventRecord(b, stream));
        SSU_CK(cudaEventSynchronize(b));
        float ms = 0;
        SSU_CK(cudaEventElapsedTime(&ms, a, b));
        const double waves = std::ceil(static_cast<double>(tiles.size()) * splits / slots);
        const double pred = waves * (ms / 3.0) * (static_cast<double>(rows) / probe);
        char buf[96];
        std::snprintf(buf, sizeof(buf), "%s%s=%.3gms", report.empty() ? "" : " ", k.shape, pred);
        report += buf;
        if (pred < best) {
            best = pred;
            chosen = i;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    TuneCache::get().put(key, cands[chosen].shape);
    tuning = std::string("tuned ") + cands[chosen].shape + " (" + report + ")";
    return 0;
}

template <typename T>
int PlanImpl::embed(cudaStream_t s, const Group &g) {
    if (K == 0) return 0;
    const bool counts = spec.vaw && !faith;
    T *U = static_cast<T *>(d_U);
    T *C = static_cast<T *>(d_C);
    const bool normalize = faith ? true : spec.normalize;
    const uint32_t tg = g.t1 - g.t0;
    // the sparse pair kernels' presence masks and counts, filled as rows are
    // embedded (no separate pass over U)
    dev::MaskOut mo{nullptr, nullptr, E};
    if ((hybrid || union_mode) && d_masks && E) {
        SSU_CK(cudaMemsetAsync(d_masks, 0, sizeof(unsigned long long) * E * (g.ld / 64), s));
        SSU_CK(cudaMemsetAsync(d_counts, 0, sizeof(uint32_t) * E, s));
        mo.masks = d_masks;
        mo.counts = d_counts;
    }
    if (n_tips) {
        const uint32_t grid = std::min<uint32_t>(n_tips, 65535u * 8);
        if (counts)
            dev::embed_tips_kernel<T, true><<<grid, 256, 0, s>>>(d_tip_rows, g.d_tip_obs, n_tips, tg, d_tdesc + g.t0,
                                                                 d_indptr, d_indices, d_data, g.d_totals, normalize,
                                                                 U, C, g.ld, mo);
        else
            dev::embed_tips_kernel<T, false><<<grid, 256, 0, s>>>(d_tip_rows, g.d_tip_obs, n_tips, tg,
                                                                  d_tdesc + g.t0, d_indptr, d_indices, d_data,
                                                                  g.d_totals, normalize, U, C, g.ld, mo);
        launches++;
    }
    const uint64_t nvec = g.ld / dev::Vec16<T>::n;
    const uint32_t threads = 128;
    const uint32_t col_blocks = static_cast<uint32_t>((nvec + threads - 1) / threads);
    for (size_t h = 1; h < level_ptr.size(); h++) {
        const uint32_t a = level_ptr[h - 1], b = level_ptr[h];
        if (b == a) continue;
        const uint64_t blocks = static_cast<uint64_t>(b - a) * col_blocks;
        const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>(blocks, 1u << 20));
        if (counts)
            dev::embed_level_kernel<T, true><<<grid, threads, 0, s>>>(d_level_rows + a, b - a, d_child_ptr,
                                                                      d_child_rows, U, C, g.ld, col_blocks, mo);
        else
            dev::embed_level_kernel<T, false><<<grid, threads, 0, s>>>(d_level_rows + a, b - a, d_child_ptr,
                                                                       d_child_rows, U, C, g.ld, col_blocks, mo);
        launches++;
    }
    SSU_CK(cudaGetLastError());
    return 0;
}

template <typename T>
int PlanImpl::prepare(cudaStream_t s, const Group &g) {
    const T *U = static_cast<const T *>(d_U);
    const T *len = static_cast<const T *>(d_len);
    if (d_W && !hybrid) {  // the hybrid sums W with its Ws (hybrid_stage)
        dim3 grid(static_cast<uint32_t>((g.ld + 127) / 128), n_parts);
        dev::weighted_sums_partial_kernel<T><<<grid, 128, 0, s>>>(U, len, E, g.ld, part_chunk,
                                                                 static_cast<T *>(d_part),
                                                                 len_stride ? g.d_block_table : nullptr, len_stride);
        dev::reduce_partials_kernel<T><<<static_cast<uint32_t>((g.ld + 255) / 256), 256, 0, s>>>(
            static_cast<const T *>(d_part), n_parts, g.ld, static_cast<T *>(d_W));
        launches += 2;
    }
    if (d_P && n_words) {
        const uint64_t total = static_cast<uint64_t>(n_words) * g.ld;
        const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>((total + 255) / 256, 1u << 20));
        dev::pack_presence_kernel<T><<<grid, 256, 0, s>>>(U, E, g.ld, n_words, d_P);
        launches++;
    }
    SSU_CK(cudaGetLastError());
    return 0;
}

template <typename T>
int PlanImpl::pair_stage(cudaStream_t s, const Group &g, const dev::OutSpec &out, const uint4 *tiles,
                         uint32_t ntiles, uint32_t nsplits, uint32_t rows, bool last) {
    const PairKernel<T> &k = kern<T>();
    if (ntiles == 0) return 0;
    dev::PairArgs<T> a{};
    a.tiles = tiles;
    a.n_tiles = ntiles;
    a.tables = d_tdesc;
    a.U = static_cast<const T *>(d_U);
    a.C = static_cast<const T *>(d_C);
    a.len = static_cast<const T *>(d_len);
    a.len_stride = len_stride;
    a.tot = static_cast<const T *>(g.d_tot);
    a.W = static_cast<const T *>(d_W);
    a.P = d_P;
    a.lut = static_cast<const T *>(d_lut);
    a.lut_stride = lut_stride;
    a.E = bits() ? n_words : E;
    a.ld = g.ld;
    a.alpha = static_cast<T>(spec.alpha);
    a.out = out;
    if (nsplits <= 1) {
        nsplits = 1;
        rows = a.E;
        a.partial = nullptr;
    } else {
        a.partial = static_cast<T *>(d_partial);
    }
    a.n_splits = nsplits;
    a.rows_per_split = rows;
    const uint64_t work = static_cast<uint64_t>(ntiles) * nsplits;
    const uint64_t slots = static_cast<uint64_t>(std::max(1, n_sms * k.blocks_per_sm));
    k.launch(a, static_cast<uint32_t>(std::min(work, slots)), k.smem, s);
    launches++;
    if (last && timed()) SSU_CK(cudaEventRecord(ev[2], s));
    if (nsplits > 1) {
        k.finalize(a, s);
        launches++;
    }
    SSU_CK(cudaGetLastError());
    return 0;
}

void PlanImpl::zero_diagonal(cudaStream_t s, void *out) {
    if (!max_table_n || tdesc.empty()) return;
    const uint32_t bx = std::min<uint32_t>((max_table_n + 255) / 256, 64);
    dev::zero_diagonal_kernel<<<dim3(bx, static_cast<uint32_t>(tdesc.size())), 256, 0, s>>>(out, d_tdesc,
                                                                                          spec.fp64 ? 1 : 0);
    launches++;
}

template <typename T>
int PlanImpl::execute_T(cudaStream_t s, const dev::OutSpec &out) {
    launches = 0;
    if (timed()) SSU_CK(cudaEventRecord(ev[0], s));
    for (size_t gi = 0; gi < groups.size(); gi++) {
        const Group &g = groups[gi];
        int rc = embed<T>(s, g);
        if (!rc) rc = prepare<T>(s, g);
        if (rc) return rc;
        if (gi == 0 && timed()) SSU_CK(cudaEventRecord(ev[1], s));
        rc = union_mode ? union_stage<T>(s, g, out, g.d_tiles, g.n_tiles, g.splits, gi + 1 == groups.size())
             : hybrid ? hybrid_stage<T>(s, g, out, g.d_tiles, g.n_tiles, g.splits, gi + 1 == groups.size())
                    : pair_stage<T>(s, g, out, g.d_tiles, g.n_tiles, g.splits, g.rows_per_split,
                                    gi + 1 == groups.size());
        if (rc) return rc;
        if (gi + 1 == groups.size() && g.n_tiles == 0 && timed()) SSU_CK(cudaEventRecord(ev[2], s));
    }
    if (out.mode == 0) zero_diagonal(s, out.ptr);
    if (timed()) SSU_CK(cudaEventRecord(ev[3], s));
    SSU_CK(cudaGetLastError());
    return 0;
}

int PlanImpl::execute_all(cudaStream_t s) {
    dev::OutSpec o{0, d_full, 0, 0};
    if (gemm) return execute_gemm(s, o);
    return spec.fp64 ? execute_T<double>(s, o) : execute_T<float>(s, o);
}

// One table only: its stripes [start, stop) (mode 1) or condensed form (2).
int PlanImpl::run_windowed(int mode, void *d_out, uint32_t start, uint32_t stop) {
    if (gemm) {
        dev::OutSpec o{mode, d_out, start, stop};
        return execute_gemm(stream, o);
    }
    const Group &g = groups[0];
    const int BM = union_mode ? dev::UT : spec.fp64 ? kd.BM : kf.BM;
    const int BN = union_mode ? dev::UT : spec.fp64 ? kd.BN : kf.BN;
    std::vector<uint4> tiles;
    append_tiles(tiles, 0, 0, tdesc[0].n, BM, BN, mode == 1, start, stop);
    uint4 *d_t = nullptr;
    SSU_CK(upload(&d_t, tiles.data(), sizeof(uint4) * tiles.size()));
    // (the hybrid and union stages below also take the full matrix's splits)
    if (union_mode) {
        dev::OutSpec o{mode, d_out, start, stop};
        launches = 0;
        const uint32_t nt = static_cast<uint32_t>(tiles.size());
        int rc = 0;
        if (spec.fp64) {
            rc = embed<double>(stream, g);
            if (!rc) rc = union_stage<double>(stream, g, o, d_t, nt, g.splits, true);
        } else {
            rc = embed<float>(stream, g);
            if (!rc) rc = union_stage<float>(stream, g, o, d_t, nt, g.splits, true);
        }
        return rc;
    }
    if (hybrid) {
        dev::OutSpec o{mode, d_out, start, stop};
        launches = 0;
        const uint32_t nt = static_cast<uint32_t>(tiles.size());
        int rc = 0;
        if (spec.fp64) {
            rc = embed<double>(stream, g);
            if (!rc) rc = prepare<double>(stream, g);
            if (!rc) rc = hybrid_stage<double>(stream, g, o, d_t, nt, g.splits, true);
        } else {
            rc = embed<float>(stream, g);
            if (!rc) rc = prepare<float>(stream, g);
            if (!rc) rc = hybrid_stage<float>(stream, g, o, d_t, nt, g.splits, true);
        }
        return rc;
    }
    // the full matrix's node splits: every tile of the window sums its nodes
    // in the same order as in the full matrix, so stripes of a window are
    // bit-identical to the full matrix's (the window never holds more tiles,
    // so the plan's partial buffer fits)
    const uint32_t s = g.splits, rows = g.rows_per_split;
    dev::OutSpec o{mode, d_out, start, stop};
    launches = 0;
    const uint32_t nt = static_cast<uint32_t>(tiles.size());
    int rc = 0;
    if (spec.fp64) {
        rc = embed<double>(stream, g);
        if (!rc) rc = prepare<double>(stream, g);
        if (!rc) rc = pair_stage<double>(stream, g, o, d_t, nt, s, rows, true);
    } else {
        rc = embed<float>(stream, g);
        if (!rc) rc = prepare<float>(stream, g);
        if (!rc) rc = pair_stage<float>(stream, g, o, d_t, nt, s, rows, true);
    }
    return rc;
}

// --------------------------------------------------- tensor-core unweighted

// Tensor-core work units: per table, the (256-row block, 128-column block)
// pairs holding some pair k < l, ordered in bands of `band` row blocks walked
// column by column.  Clusters start in launch order as SMs free up, so a
// unit reads the column block of B that its predecessor is reading and the
// row block of A that the unit a band height earlier read, both still in L2:
// each B block comes from DRAM about once per band, each A block about once
// per table.  The order changes no result (every unit is independent).
int PlanImpl::build_units(uint32_t band) {
    band = std::max(1u, band);
    for (Group &g : groups) {
        std::vector<uint4> tiles;
        g.band_unit.clear();
        g.band_row.clear();
        for (uint32_t t = g.t0; t < g.t1; t++) {
            const uint32_t n = tdesc[t].n;
            const uint32_t nkb = (n + tc::UMMA_M - 1) / tc::UMMA_M, nlb = (n + tc::COLS - 1) / tc::COLS;
            for (uint32_t k0 = 0; k0 < nkb; k0 += band) {
                g.band_unit.push_back(static_cast<uint32_t>(tiles.size()));
                g.band_row.push_back(k0 * tc::UMMA_M);
                for (uint32_t lb = 0; lb < nlb; lb++)
                    for (uint32_t kb = k0; kb < std::min(nkb, k0 + band); kb++)
                        if (static_cast<uint64_t>(kb) * tc::UMMA_M <
                            std::min<uint64_t>(n, static_cast<uint64_t>(lb + 1) * tc::COLS) - 1)
                            tiles.push_back(make_uint4(kb, lb, t, 0));
            }
            g.band_unit.push_back(static_cast<uint32_t>(tiles.size()));
            g.band_row.push_back(n);
        }
        g.n_tiles = static_cast<uint32_t>(tiles.size());
        if (!g.d_tiles) SSU_CK(alloc(&g.d_tiles, sizeof(uint4) * std::max<size_t>(tiles.size(), 1)));
        if (!tiles.empty())
            SSU_CK(cudaMemcpyAsync(g.d_tiles, tiles.data(), sizeof(uint4) * tiles.size(), cudaMemcpyHostToDevice,
                                   stream));
        SSU_CK(cudaStreamSynchronize(stream));  // the host list is released on return
    }
    tc_band = band;
    return 0;
}

// With tuning on: the band height of the unit order by measurement (one
// untimed and one timed execute per candidate), cached per (table sizes,
// nodes, SM count) for the process and UNIFRAC_B200_TUNE_CACHE.
int PlanImpl::tune_band() {
    const std::string key = "tc_band|n" + std::to_string(log2_bucket(max_table_n)) + "|c" +
                            std::to_string(log2_bucket(ld)) + "|E" + std::to_string(log2_bucket(E)) + "|sm" +
                            std::to_string(n_sms);
    std::string v;
    if (TuneCache::get().find(key, v) && v.rfind("band=", 0) == 0) {
        const int b = std::atoi(v.c_str() + 5);
        if (b > 0) {
            tuning = "cache band " + std::to_string(b);
            return build_units(static_cast<uint32_t>(b));
        }
    }
    cudaEvent_t a = nullptr, b = nullptr;
    SSU_CK(cudaEventCreate(&a));
    SSU_CK(cudaEventCreate(&b));
    const dev::OutSpec out{0, d_full, 0, 0};
    uint32_t best_band = tc_band;
    float best = 1e30f;
    std::string report;
    int rc = 0;
    for (uint32_t cand : {2u, 4u, 8u}) {
        if ((rc = build_units(cand))) break;
        if ((rc = execute_gemm(stream, out))) break;
        SSU_CK(cudaEventRecord(a, stream));
        if ((rc = execute_gemm(stream, out))) break;
        SSU_CK(cudaEventRecord(b, stream));
        SSU_CK(cudaEventSynchronize(b));
        float ms = 0.f;
        SSU_CK(cudaEventElapsedTime(&ms, a, b));
        report += (report.empty() ? "" : ", ") + std::to_string(cand) + ": " + std::to_string(ms) + " ms";
        if (ms < best) {
            best = ms;
            best_band = cand;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    if (device_error_pending()) {
        last_error = "device wait expired while tuning";
        return kOutputError;
    }
    TuneCache::get().put(key, "band=" + std::to_string(best_band));
    tuning = "measured band " + std::to_string(best_band) + " (" + report + ")";
    return build_units(best_band);
}

// Tree-only host part of the tensor-core setup (no CUDA call, so it runs on
// a worker thread while the plan's CSR and tree are uploaded).
// Embedded nodes grouped by the binary exponent of |length|, largest first,
// packed into chunks of whole 128-node K blocks: a chunk closes (its last
// block padded with zero-length columns) where the exponent changes or at
// MAX_CHUNK_KB blocks.  Chunk c is scaled by 2^s_c so that its exponent's
// largest length lies in [2^22, 2^23), which puts all its lengths there;
// q = round(L 2^s_c) is then written as 256 u v + s t with 8-bit digits
// (`digits::split_length`).
GemmLayout build_gemm_layout(const FlatTree &tree) {
    GemmLayout lay;
    const uint32_t E = tree.n_embedded;
    // order by binary exponent of |length|, largest first, by row within an
    // exponent (one counting pass): every length of an exponent lies within a
    // factor of two of the others, which is all the chunks need
    constexpr int kExp = 2048;  // biased fp64 exponents; 0 holds zeros (and subnormals)
    auto exponent = [](double a) {
        uint64_t b;
        std::memcpy(&b, &a, sizeof b);
        return static_cast<int>((b >> 52) & 0x7FF);
    };
    std::vector<uint32_t> count(kExp, 0), order(E);
    std::vector<double> emax(kExp, 0.0);
    for (uint32_t e = 0; e < E; e++) {
        const double a = std::fabs(tree.length[e]);
        const int x = exponent(a);
        count[x]++;
        emax[x] = std::max(emax[x], a);
    }
    {
        uint32_t at = 0;
        for (int x = kExp - 1; x >= 0; x--) {
            const uint32_t c = count[x];
            count[x] = at;
            at += c;
        }
        for (uint32_t e = 0; e < E; e++) order[count[exponent(std::fabs(tree.length[e]))]++] = e;
    }
    std::vector<int32_t> col_of_row(tree.n_nodes, -1);
    std::vector<uint32_t> lq;  // 23-bit fixed-point lengths
    lq.reserve(E + 128 * tc::BLOCK_K);
    lay.lsorted.reserve(E + 128 * tc::BLOCK_K);
    const uint32_t max_cols = static_cast<uint32_t>(tc::MAX_CHUNK_KB) * tc::BLOCK_K;
    auto pad_to_block = [&] {
        while (lay.lsorted.size() % tc::BLOCK_K) {
            lay.lsorted.push_back(0.0);
            lq.push_back(0u);
        }
        lay.chunk_end.push_back(static_cast<uint32_t>(lay.lsorted.size() / tc::BLOCK_K));
    };
    // A chunk holds lengths of one exponent (at most MAX_CHUNK_KB blocks),
    // scaled by 2^sig so that the exponent's largest lies in [2^22, 2^23):
    // every length of the chunk then lies in [2^22, 2^23) too.
    const double qmax = std::ldexp(1.0, tc::QBITS) - 1.0;
    int cur = -1, sig = 0;
    double pw = 1.0;
    bool by_mul = true;
    size_t chunk_first = 0;
    double first = -1.0;
    for (uint32_t i = 0; i < E; i++) {
        const double L = tree.length[order[i]];
        const int xe = exponent(std::fabs(L));
        if (xe != cur || lay.lsorted.size() - chunk_first >= max_cols) {
            if (cur >= 0) pad_to_block();
            cur = xe;
            first = emax[xe];
            chunk_first = lay.lsorted.size();
            // floor(log2) of a normal double is its unbiased exponent, exactly
            const int lg = xe > 0 ? xe - 1023 : (first > 0 ? static_cast<int>(std::floor(std::log2(first))) : 0);
            sig = first > 0 ? (tc::QBITS - 1) - lg : 0;
            lay.scale.push_back(std::ldexp(1.0, -sig));
            by_mul = sig >= -1022 && sig <= 1023;  // 2^sig itself a normal double
            pw = by_mul ? std::ldexp(1.0, sig) : 1.0;
        }
        col_of_row[order[i]] = static_cast<int32_t>(lay.lsorted.size());
        const double x = by_mul ? L * pw : std::ldexp(L, sig);  // exact: a power of two
        lay.lsorted.push_back(L);
        lq.push_back(static_cast<uint32_t>(std::min(std::floor(std::max(x, 0.0) + 0.5), qmax)));
    }
    if (first < 0) lay.scale.push_back(1.0);  // no embedded node: one chunk of padding
    pad_to_block();
    const uint32_t k_pad = static_cast<uint32_t>(lay.lsorted.size());
    // digits u, s, v, t of every column, one k_pad row each
    lay.digits.assign(static_cast<size_t>(2 * tc::PRODUCTS) * k_pad, 0);
    for (uint32_t c = 0; c < k_pad; c++) {
        uint8_t d[4];
        if (!digits::split_length(lq[c], d)) {
            lay.error = "length has no 8-bit product form";
            return lay;
        }
        for (int i = 0; i < 4; i++) lay.digits[static_cast<size_t>(i) * k_pad + c] = d[i];
    }
    // parents among embedded nodes
    std::vector<int32_t> parent_row(tree.n_nodes, -1);
    for (uint32_t r = 0; r < tree.n_nodes; r++)
        for (uint32_t c = tree.child_ptr[r]; c < tree.child_ptr[r + 1]; c++) parent_row[tree.child_rows[c]] = r;
    lay.parent_col.assign(k_pad, -1);
    for (uint32_t r = 0; r < E; r++) {
        const int32_t p = parent_row[r];
        lay.parent_col[col_of_row[r]] = (p >= 0 && static_cast<uint32_t>(p) < E) ? col_of_row[p] : -1;
    }
    // starting column of each tree observation: its tip, or the tip's parent
    // when tips are bypassed
    uint32_t n_obs_tree = 0;
    for (uint32_t r : tree.leaf_rows) n_obs_tree = std::max<uint32_t>(n_obs_tree, tree.leaf_obs[r] + 1);
    lay.start_of_obs.assign(n_obs_tree, -1);
    for (uint32_t r : tree.leaf_rows) {
        const int32_t obs = tree.leaf_obs[r];
        if (obs < 0) continue;
        int32_t node = static_cast<int32_t>(r);
        if (r >= E) node = parent_row[r];
        lay.start_of_obs[obs] = (node >= 0 && static_cast<uint32_t>(node) < E) ? col_of_row[node] : -1;
    }
    return lay;
}

int PlanImpl::setup_gemm(const TableSet &set, const FlatTree &tree) {
    SetupTimer timer;
    GemmLayout lay = gemm_layout.valid() ? gemm_layout.get() : build_gemm_layout(tree);
    timer.step("gemm_layout");
    if (!lay.error.empty()) {
        last_error = lay.error;
        return kOutputError;
    }
    k_pad = static_cast<uint32_t>(lay.lsorted.size());
    n_chunks = static_cast<uint32_t>(lay.chunk_end.size());
    const std::vector<int32_t> &start_of_obs = lay.start_of_obs;
    const uint32_t n_obs_tree = static_cast<uint32_t>(start_of_obs.size());
    // per group: operand rows = the group's columns; each row's list of
    // starting columns (one per table row of an observation with a positive
    // count), built on the device from the uploaded CSR: count, scan, place
    for (Group &g : groups) {
        uint64_t nnz_g = 0;
        for (uint32_t t = g.t0; t < g.t1; t++) nnz_g += set.tables[t]->nnz();
        uint32_t *d_count = nullptr, *d_fill = nullptr;
        SSU_CK(alloc(&d_count, sizeof(uint32_t) * g.ld));
        SSU_CK(alloc(&d_fill, sizeof(uint32_t) * g.ld));
        SSU_CK(alloc(&g.d_sample_ptr, sizeof(uint32_t) * (g.ld + 1)));
        SSU_CK(alloc(&g.d_start_col, sizeof(int32_t) * std::max<uint64_t>(nnz_g, 1)));
        SSU_CK(cudaMemsetAsync(d_count, 0, sizeof(uint32_t) * g.ld, stream));
        std::vector<int32_t *> d_row_start(g.t1 - g.t0, nullptr);
        for (uint32_t t = g.t0; t < g.t1; t++) {
            const Table &tb = *set.tables[t];
            std::vector<int32_t> row_start(std::max<uint32_t>(tb.n_obs, 1), -1);
            if (set.obs_row.empty()) {
                for (uint32_t o = 0; o < n_obs_tree && o < tb.n_obs; o++) row_start[o] = start_of_obs[o];
            } else {
                const std::vector<int32_t> &m = set.obs_row[t];
                for (uint32_t o = 0; o < n_obs_tree && o < m.size(); o++)
                    if (m[o] >= 0 && static_cast<uint32_t>(m[o]) < tb.n_obs) row_start[m[o]] = start_of_obs[o];
            }
            SSU_CK(upload(&d_row_start[t - g.t0], row_start.data(), sizeof(int32_t) * row_start.size()));
        }
        for (int pass = 0; pass < 2; pass++) {
            if (pass == 1) {
                tc::exclusive_scan_kernel<<<1, 1024, 0, stream>>>(d_count, static_cast<uint32_t>(g.ld),
                                                                  g.d_sample_ptr);
                SSU_CK(cudaMemcpyAsync(d_fill, g.d_sample_ptr, sizeof(uint32_t) * g.ld, cudaMemcpyDeviceToDevice,
                                       stream));
            }
            for (uint32_t t = g.t0; t < g.t1; t++) {
                const Table &tb = *set.tables[t];
                const dev::TableDesc &d = tdesc[t];
                if (tb.n_obs == 0 || tb.nnz() == 0) continue;
                const uint64_t threads = static_cast<uint64_t>(tb.n_obs) * 32;
                tc::sample_lists_kernel<<<static_cast<uint32_t>((threads + 255) / 256), 256, 0, stream>>>(
                    d_indptr + d.indptr_off, d_indices + d.nnz_off, d_data + d.nnz_off, d_row_start[t - g.t0],
                    tb.n_obs, d.base, d_count, pass ? d_fill : nullptr, g.d_start_col);
            }
        }
        SSU_CK(cudaGetLastError());
    }
    timer.step("gemm_sample_lists");
    const uint32_t band = static_cast<uint32_t>(std::max(1, env_int("UNIFRAC_B200_TC_BAND", 4)));
    if (const int rc = build_units(band)) return rc;
    timer.step("gemm_tiles");
    n_pad = static_cast<uint32_t>(ld);
    const size_t op_bytes = static_cast<size_t>(n_pad) * k_pad;
    SSU_CK(alloc(&d_A, tc::PRODUCTS * op_bytes));
    SSU_CK(alloc(&d_B, tc::PRODUCTS * op_bytes));
    SSU_CK(alloc(&d_r, sizeof(double) * n_pad));
    SSU_CK(upload(&d_lq, lay.digits.data(), lay.digits.size()));
    SSU_CK(upload(&d_lsorted, lay.lsorted.data(), sizeof(double) * k_pad));
    SSU_CK(upload(&d_chunk_scale, lay.scale.data(), sizeof(double) * n_chunks));
    SSU_CK(upload(&d_chunk_end, lay.chunk_end.data(), sizeof(uint32_t) * n_chunks));
    SSU_CK(upload(&d_parent_col, lay.parent_col.data(), sizeof(int32_t) * k_pad));
    SSU_CK(alloc(&d_error, sizeof(int)));
    SSU_CK(cudaMemsetAsync(d_error, 0, sizeof(int), stream));
    if (const char *w = std::getenv("UNIFRAC_B200_WAIT_CYCLES")) gemm_wait_cycles = std::max(0LL, std::atoll(w));
    union_stall = env_int("UNIFRAC_B200_TEST_STALL", 0) ? 1 : 0;
    if (!make_u8_map(&map_A, d_A, static_cast<uint64_t>(tc::PRODUCTS) * n_pad, k_pad, tc::ROWS) ||
        !make_u8_map(&map_B, d_B, static_cast<uint64_t>(tc::PRODUCTS) * n_pad, k_pad, tc::B_ROWS)) {
        last_error = "cuTensorMapEncodeTiled failed";
        return kOutputError;
    }
    SSU_CK(cudaFuncSetAttribute(tc::unweighted_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(tc::SMEM_BYTES)));
    const size_t bits_smem = sizeof(uint32_t) * (k_pad / 32);
    if (bits_smem > 200 * 1024) {
        last_error = "tree too large for the tensor-core presence kernel";
        return kOutputError;
    }
    SSU_CK(cudaFuncSetAttribute(tc::presence_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(bits_smem)));
    SSU_CK(alloc(&d_full, (spec.fp64 ? sizeof(double) : sizeof(float)) * std::max<uint64_t>(full_elems, 1)));
    SSU_CK(cudaStreamSynchronize(stream));
    timer.step("gemm_buffers");
    tuning = "band " + std::to_string(tc_band);
    if (autotune == 1 && !std::getenv("UNIFRAC_B200_TC_BAND")) {
        if (const int rc = tune_band()) return rc;
        timer.step("gemm_tune");
    }
    return 0;
}

bool PlanImpl::device_error_pending() {
    int h = 0;
    if (!d_error || cudaMemcpy(&h, d_error, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    return h != 0;
}

int PlanImpl::execute_gemm(cudaStream_t s, const dev::OutSpec &out) {
    launches = 0;
    if (timed()) SSU_CK(cudaEventRecord(ev[0], s));
    const size_t bits_smem = sizeof(uint32_t) * (k_pad / 32);
    for (size_t gi = 0; gi < groups.size(); gi++) {
        const Group &g = groups[gi];
        tc::presence_rows_kernel<<<static_cast<uint32_t>(g.ld), 256, bits_smem, s>>>(
            g.d_sample_ptr, g.d_start_col, d_parent_col, d_lq, d_lsorted, static_cast<uint32_t>(g.ld), k_pad,
            static_cast<uint64_t>(n_pad) * k_pad, d_A, d_B, d_r);
        launches++;
        if (gi == 0 && timed()) SSU_CK(cudaEventRecord(ev[1], s));
        if (g.n_tiles) {
            tc::GemmArgs a{};
            a.tiles = g.d_tiles;
            a.n_tiles = g.n_tiles;
            a.tables = d_tdesc;
            a.n_kblocks = k_pad / tc::BLOCK_K;
            a.plane_rows = n_pad;
            a.n_chunks = n_chunks;
            a.chunk_end = d_chunk_end;
            a.chunk_scale = d_chunk_scale;
            a.r = d_r;
            a.normalized = spec.method == Method::unweighted ? 1 : 0;
            a.out_fp64 = spec.fp64 ? 1 : 0;
            a.out = out;
            a.error = d_error;
            a.wait_cycles = gemm_wait_cycles;
            a.stall = union_stall;
            // two CTAs (one cluster) per work unit, started in unit order
            tc::unweighted_tc_kernel<<<2 * g.n_tiles, tc::THREADS, tc::SMEM_BYTES, s>>>(map_A, map_B, a);
            launches++;
        }
        if (gi + 1 == groups.size() && timed()) SSU_CK(cudaEventRecord(ev[2], s));
    }
    if (out.mode == 0) zero_diagonal(s, out.ptr);
    if (timed()) SSU_CK(cudaEventRecord(ev[3], s));
    SSU_CK(cudaGetLastError());
    return 0;
}

// One table on the tensor-core path, result copied out while it is being
// computed.  The work units are ordered in bands of row blocks, and a unit of
// band p writes the upper-triangle entries of its rows (band p) and their
// mirror images in rows of bands >= p.  So rows of band p are final once the
// launches of bands 0..p are done: each band is one launch, alternating
// between two streams (the next band's clusters fill SMs as the previous
// band drains), and the copy stream copies band p's rows after waiting for
// band p's launch - the earlier bands' copies having waited for theirs.
// (25,000 samples: the copy-out, about 43 GB/s while the kernel runs against
// 57 GB/s alone, ends ~25 ms after the last band; copying per band the rows
// and columns it finished, all bands on one stream, or two copy streams
// measured the same.)
int PlanImpl::execute_gemm_overlap(void *host) {
    const Group &g = groups[0];
    const uint32_t nb = static_cast<uint32_t>(g.band_unit.size()) - 1;
    const uint32_t n_t = tdesc[0].n;
    const size_t el = spec.fp64 ? sizeof(double) : sizeof(float);
    for (cudaStream_t &a : aux)
        if (!a) SSU_CK(cudaStreamCreateWithFlags(&a, cudaStreamNonBlocking));
    while (band_ev.size() < nb + 2) {
        cudaEvent_t e = nullptr;
        SSU_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        band_ev.push_back(e);
    }
    cudaStream_t s = stream, s1 = aux[0], sc = aux[1];
    launches = 0;
    dev::OutSpec out{};
    out.mode = 0;
    out.ptr = d_full;
    zero_diagonal(s, d_full);  // the units never write the diagonal
    const size_t bits_smem = sizeof(uint32_t) * (k_pad / 32);
    tc::presence_rows_kernel<<<static_cast<uint32_t>(g.ld), 256, bits_smem, s>>>(
        g.d_sample_ptr, g.d_start_col, d_parent_col, d_lq, d_lsorted, static_cast<uint32_t>(g.ld), k_pad,
        static_cast<uint64_t>(n_pad) * k_pad, d_A, d_B, d_r);
    launches++;
    SSU_CK(cudaEventRecord(band_ev[nb], s));
    SSU_CK(cudaStreamWaitEvent(s1, band_ev[nb], 0));
    for (uint32_t p = 0; p < nb; p++) {
        cudaStream_t st = (p & 1) ? s1 : s;
        const uint32_t u0 = g.band_unit[p], u1 = g.band_unit[p + 1];
        if (u1 > u0) {
            tc::GemmArgs a{};
            a.tiles = g.d_tiles + u0;
            a.n_tiles = u1 - u0;
            a.tables = d_tdesc;
            a.n_kblocks = k_pad / tc::BLOCK_K;
            a.plane_rows = n_pad;
            a.n_chunks = n_chunks;
            a.chunk_end = d_chunk_end;
            a.chunk_scale = d_chunk_scale;
            a.r = d_r;
            a.normalized = spec.method == Method::unweighted ? 1 : 0;
            a.out_fp64 = spec.fp64 ? 1 : 0;
            a.out = out;
            a.error = d_error;
            a.wait_cycles = gemm_wait_cycles;
            a.stall = union_stall;
            tc::unweighted_tc_kernel<<<2 * (u1 - u0), tc::THREADS, tc::SMEM_BYTES, st>>>(map_A, map_B, a);
            launches++;
        }
        SSU_CK(cudaEventRecord(band_ev[p], st));
        SSU_CK(cudaStreamWaitEvent(sc, band_ev[p], 0));
        const uint64_t r0 = g.band_row[p], r1 = std::min<uint64_t>(g.band_row[p + 1], n_t);
        if (r1 > r0)
            SSU_CK(cudaMemcpyAsync(static_cast<char *>(host) + el * r0 * n_t,
                                   static_cast<const char *>(d_full) + el * r0 * n_t, el * (r1 - r0) * n_t,
                                   cudaMemcpyDeviceToHost, sc));
    }
    SSU_CK(cudaGetLastError());
    SSU_CK(cudaEventRecord(band_ev[nb + 1], sc));
    SSU_CK(cudaStreamWaitEvent(s, band_ev[nb + 1], 0));
    SSU_CK(cudaEventRecord(band_ev[nb], s1));
    SSU_CK(cudaStreamWaitEvent(s, band_ev[nb], 0));
    return 0;
}

// ------------------------------------------------------------------ Plan

namespace {

int resolve_autotune(int requested, bool batch) {
    if (requested >= 0) return requested;
    return env_int("UNIFRAC_B200_AUTOTUNE", batch ? 1 : 0);
}

}  // namespace

namespace {

// Unweighted methods (not variance adjusted) on the tensor-core contraction:
// by default for fp32 results (its ~1e-8 relative error is far inside the
// fp32 stripe form's own), on request for fp64.  Presence is "proportion >
// 0", the OR of the tips below a node, so it needs counts that are not
// negative, and the lengths are fixed-point magnitudes, so they must not be
// negative either.  A batch with bypassed tips keeps the stripe form (its
// tables' trees differ in which rows carry length).
bool use_tensor_cores(const MethodSpec &spec, const TableSet &set, const FlatTree &tree, bool batch) {
    if (spec.vaw || !(spec.method == Method::unweighted || spec.method == Method::unweighted_unnormalized))
        return false;
    bool want = spec.unweighted_gemm || (!spec.fp64 && !spec.unweighted_stripe);
    if (batch && spec.bypass_tips) want = false;
    for (uint32_t e = 0; want && e < tree.n_embedded; e++)
        if (!(tree.length[e] >= 0.0 && std::isfinite(tree.length[e]))) want = false;
    for (const Table *t : set.tables)
        if (!t->nonneg) want = false;  // found while the table's totals were summed
    return want;
}

}  // namespace

int Plan::create(const Table &table, const FlatTree &tree, const MethodSpec &spec, void *stream, Plan **out,
                 std::string &err) {
    Plan *p = new Plan();
    p->impl_ = new PlanImpl();
    PlanImpl &m = *p->impl_;
    m.spec = spec;
    m.stream = static_cast<cudaStream_t>(stream);
    m.autotune = resolve_autotune(-1, false);
    TableSet set;
    set.tables.push_back(&table);
    set.embedded.push_back(tree.n_embedded);
    m.gemm = use_tensor_cores(spec, set, tree, false);
    if (m.gemm) m.start_gemm_layout(tree);
    int rc = m.setup(set, tree, BatchOptions{});
    if (!rc) rc = m.gemm ? m.setup_gemm(set, tree) : spec.fp64 ? m.setup_method<double>() : m.setup_method<float>();
    if (rc) {
        err = m.last_error;
        delete p;
        return rc;
    }
    *out = p;
    return 0;
}

int Plan::create_batch(const TableSet &set, const FlatTree &tree, const MethodSpec &spec, const BatchOptions &opts,
                       void *stream, Plan **out, std::string &err) {
    if (set.tables.empty() || set.tables.size() > 65535 ||
        (!set.obs_row.empty() && set.obs_row.size() != set.tables.size()) ||
        (!set.row_active.empty() && set.row_active.size() != set.tables.size())) {
        err = "bad table set";
        return kOutputError;
    }
    Plan *p = new Plan();
    p->impl_ = new PlanImpl();
    PlanImpl &m = *p->impl_;
    m.spec = spec;
    m.batch = true;
    m.stream = static_cast<cudaStream_t>(stream);
    m.autotune = resolve_autotune(opts.autotune, true);
    m.gemm = use_tensor_cores(spec, set, tree, true);
    if (m.gemm) m.start_gemm_layout(tree);
    int rc = m.setup(set, tree, opts);
    if (!rc) rc = m.gemm ? m.setup_gemm(set, tree) : spec.fp64 ? m.setup_method<double>() : m.setup_method<float>();
    if (rc) {
        err = m.last_error;
        delete p;
        return rc;
    }
    *out = p;
    return 0;
}

int Plan::create_faith(const Table &table, const FlatTree &tree, void *stream, Plan **out, std::string &err) {
    Plan *p = new Plan();
    p->impl_ = new PlanImpl();
    PlanImpl &m = *p->impl_;
    m.faith = true;
    m.spec.fp64 = true;
    m.spec.normalize = true;
    m.stream = static_cast<cudaStream_t>(stream);
    TableSet set;
    set.tables.push_back(&table);
    int rc = m.setup(set, tree, BatchOptions{});
    if (!rc) {
        if (m.alloc(&m.d_U, sizeof(double) * m.ld * std::max<uint32_t>(m.K, 1)) != cudaSuccess) {
            err = "device allocation failed";
            delete p;
            return kOutputError;
        }
    }
    if (rc) {
        err = m.last_error;
        delete p;
        return rc;
    }
    *out = p;
    return 0;
}

Plan::~Plan() {
    if (!impl_) return;
    PlanImpl &m = *impl_;
    if (m.graph) cudaGraphExecDestroy(m.graph);
    if (m.stream) {
        for (void *q : m.allocations) cudaFreeAsync(q, m.stream);
        cudaStreamSynchronize(m.stream);
    }
    for (auto &e : m.ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : m.band_ev)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t a : m.aux)
        if (a) {
            cudaStreamSynchronize(a);
            cudaStreamDestroy(a);
        }
    if (m.own_stream && m.stream) cudaStreamDestroy(m.stream);
    delete impl_;
}

void Plan::set_graph(bool on) {
    PlanImpl &m = *impl_;
    if (!on && m.graph) {
        cudaGraphExecDestroy(m.graph);
        m.graph = nullptr;
    }
    m.graph_on = on;
}

int Plan::execute(void *stream) {
    PlanImpl &m = *impl_;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : m.stream;
    if (!m.graph_on) return m.execute_all(s);
    if (!m.graph) {
        // capture on a stream of our own so the caller's stream may be the
        // legacy default stream
        cudaStream_t cs = m.stream;
        if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            m.last_error = "stream capture failed";
            return kOutputError;
        }
        m.capturing = true;
        const int rc = m.execute_all(cs);
        m.capturing = false;
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(cs, &g);
        if (rc || e != cudaSuccess || !g) {
            if (g) cudaGraphDestroy(g);
            m.last_error = "stream capture failed";
            return kOutputError;
        }
        const cudaError_t ie = cudaGraphInstantiate(&m.graph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            m.graph = nullptr;
            m.last_error = cudaGetErrorString(ie);
            return kOutputError;
        }
    }
    return cudaGraphLaunch(m.graph, s) == cudaSuccess ? 0 : kOutputError;
}

int Plan::device_error() {
    PlanImpl &m = *impl_;
    if (!m.d_error) return 0;
    int h = 0;
    if (cudaMemcpyAsync(&h, m.d_error, sizeof(int), cudaMemcpyDeviceToHost, m.stream) != cudaSuccess ||
        cudaStreamSynchronize(m.stream) != cudaSuccess)
        return kOutputError;
    if (h) cudaMemsetAsync(m.d_error, 0, sizeof(int), m.stream);
    return h;
}

int Plan::run_full(void *host_out, bool out_fp64, std::string &err) {
    PlanImpl &m = *impl_;
    if (out_fp64 != m.spec.fp64) {
        err = "result precision does not match the method";
        return kOutputError;
    }
    int rc = execute(nullptr);
    if (!rc) {
        const size_t bytes = (m.spec.fp64 ? sizeof(double) : sizeof(float)) * m.full_elems;
        cudaError_t e = cudaMemcpyAsync(host_out, m.d_full, bytes, cudaMemcpyDeviceToHost, m.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(m.stream);
        if (e != cudaSuccess) {
            m.last_error = cudaGetErrorString(e);
            rc = kOutputError;
        } else if (const int de = device_error()) {
            m.last_error = "device wait expired (code " + std::to_string(de) + ")";
            rc = kOutputError;
        }
    }
    if (rc) err = m.last_error;
    return rc;
}

int Plan::execute_download(void *host_out, bool pin, std::string &err) {
    PlanImpl &m = *impl_;
    const bool overlap = m.gemm && !m.graph_on && m.groups.size() == 1 && m.groups[0].t1 - m.groups[0].t0 == 1 &&
                         m.groups[0].band_unit.size() > 2 && m.full_elems > 0;
    if (!overlap) {
        const int rc = execute(nullptr);
        if (rc) {
            err = m.last_error.empty() ? "launch failed" : m.last_error;
            return rc;
        }
        return download_full(host_out, pin, err);
    }
    const size_t bytes = (m.spec.fp64 ? sizeof(double) : sizeof(float)) * m.full_elems;
    bool registered = false;
    if (pin && bytes >= (size_t(1) << 20))
        registered = cudaHostRegister(host_out, bytes, cudaHostRegisterDefault) == cudaSuccess;
    if (pin && !registered) cudaGetLastError();  // a refused registration only means pageable copies
    int rc = m.execute_gemm_overlap(host_out);
    cudaError_t e = cudaStreamSynchronize(m.stream);
    if (registered) cudaHostUnregister(host_out);
    if (rc) {
        err = m.last_error;
        return rc;
    }
    if (e != cudaSuccess) {
        err = cudaGetErrorString(e);
        return kOutputError;
    }
    if (const int de = device_error()) {
        err = "device wait expired (code " + std::to_string(de) + ")";
        return kOutputError;
    }
    return 0;
}

int Plan::download_full(void *host_out, bool pin, std::string &err) {
    return download_range(0, impl_->full_elems, host_out, pin, err);
}

int Plan::download_range(uint64_t offset, uint64_t count, void *host_out, bool pin, std::string &err) {
    PlanImpl &m = *impl_;
    const size_t el = m.spec.fp64 ? sizeof(double) : sizeof(float);
    if (offset > m.full_elems || count > m.full_elems - offset) {
        err = "result range out of bounds";
        return kOutputError;
    }
    const size_t bytes = el * count;
    bool registered = false;
    if (pin && bytes >= (size_t(1) << 20))
        registered = cudaHostRegister(host_out, bytes, cudaHostRegisterDefault) == cudaSuccess;
    if (pin && !registered) cudaGetLastError();  // a refused registration only means a pageable copy
    cudaError_t e = bytes ? cudaMemcpyAsync(host_out, static_cast<const char *>(m.d_full) + el * offset, bytes,
                                            cudaMemcpyDeviceToHost, m.stream)
                          : cudaSuccess;
    if (e == cudaSuccess) e = cudaStreamSynchronize(m.stream);
    if (registered) cudaHostUnregister(host_out);
    if (e != cudaSuccess) {
        err = cudaGetErrorString(e);
        return kOutputError;
    }
    if (const int de = device_error()) {
        err = "device wait expired (code " + std::to_string(de) + ")";
        return kOutputError;
    }
    return 0;
}

int Plan::run_stripes(uint32_t start, uint32_t stop, double *const *host_stripes, std::string &err) {
    PlanImpl &m = *impl_;
    const size_t count = static_cast<size_t>(stop - start) * m.n;
    double *d_out = nullptr;
    if (m.alloc(&d_out, sizeof(double) * std::max<size_t>(count, 1)) != cudaSuccess ||
        cudaMemsetAsync(d_out, 0, sizeof(double) * std::max<size_t>(count, 1), m.stream) != cudaSuccess) {
        err = "device allocation failed";
        return kOutputError;
    }
    int rc = m.run_windowed(1, d_out, start, stop);
    if (!rc) {
        std::vector<double> host(count);
        cudaError_t e = cudaMemcpyAsync(host.data(), d_out, sizeof(double) * count, cudaMemcpyDeviceToHost, m.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(m.stream);
        if (e != cudaSuccess) {
            m.last_error = cudaGetErrorString(e);
            rc = kOutputError;
        } else if (const int de = device_error()) {
            m.last_error = "device wait expired (code " + std::to_string(de) + ")";
            rc = kOutputError;
        } else {
            for (uint32_t s = start; s < stop; s++)
                std::memcpy(host_stripes[s - start], host.data() + static_cast<size_t>(s - start) * m.n,
                            sizeof(double) * m.n);
        }
    }
    if (rc) err = m.last_error;
    return rc;
}

int Plan::run_condensed(double *host_cf, std::string &err) {
    PlanImpl &m = *impl_;
    const size_t count = static_cast<size_t>(m.n) * (m.n - 1) / 2;
    double *d_out = nullptr;
    if (m.alloc(&d_out, sizeof(double) * std::max<size_t>(count, 1)) != cudaSuccess) {
        err = "device allocation failed";
        return kOutputError;
    }
    int rc = m.run_windowed(2, d_out, 0, 0);
    if (!rc && count) {
        cudaError_t e = cudaMemcpyAsync(host_cf, d_out, sizeof(double) * count, cudaMemcpyDeviceToHost, m.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(m.stream);
        if (e != cudaSuccess) {
            m.last_error = cudaGetErrorString(e);
            rc = kOutputError;
        } else if (const int de = device_error()) {
            m.last_error = "device wait expired (code " + std::to_string(de) + ")";
            rc = kOutputError;
        }
    }
    if (rc) err = m.last_error;
    return rc;
}

int Plan::run_faith(double *host_values, std::string &err) {
    PlanImpl &m = *impl_;
    m.launches = 0;
    const Group &g = m.groups[0];
    int rc = m.embed<double>(m.stream, g);
    if (rc) {
        err = m.last_error;
        return rc;
    }
    const uint32_t chunk = 1024;
    const uint32_t parts = std::max<uint32_t>(1, (m.K + chunk - 1) / chunk);
    double *d_part = nullptr, *d_out = nullptr;
    if (m.alloc(&d_part, sizeof(double) * g.ld * parts) != cudaSuccess ||
        m.alloc(&d_out, sizeof(double) * g.ld) != cudaSuccess) {
        err = "device allocation failed";
        return kOutputError;
    }
    dim3 grid(static_cast<uint32_t>((g.ld + 255) / 256), parts);
    dev::faith_partial_kernel<<<grid, 256, 0, m.stream>>>(static_cast<const double *>(m.d_U), m.d_len_rows,
                                                          m.d_post_rows, m.K, g.ld, chunk, d_part);
    dev::reduce_partials_kernel<double><<<static_cast<uint32_t>((g.ld + 255) / 256), 256, 0, m.stream>>>(
        d_part, parts, g.ld, d_out);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(host_values, d_out, sizeof(double) * m.n, cudaMemcpyDeviceToHost, m.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m.stream);
    if (e != cudaSuccess) {
        err = cudaGetErrorString(e);
        return kOutputError;
    }
    return 0;
}

const void *Plan::device_result() const { return impl_->d_full; }

int Plan::copy_result(void *host_out, void *stream) {
    PlanImpl &m = *impl_;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : m.stream;
    const size_t bytes = (m.spec.fp64 ? sizeof(double) : sizeof(float)) * m.full_elems;
    if (cudaMemcpyAsync(host_out, m.d_full, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess) return kOutputError;
    if (cudaStreamSynchronize(s) != cudaSuccess) return kOutputError;
    return device_error() ? kOutputError : 0;
}

int Plan::synchronize() { return cudaStreamSynchronize(impl_->stream) == cudaSuccess ? 0 : kOutputError; }

uint32_t Plan::n_samples() const { return impl_->n; }
uint32_t Plan::n_tables() const { return static_cast<uint32_t>(impl_->tdesc.size()); }
uint32_t Plan::n_groups() const { return static_cast<uint32_t>(impl_->groups.size()); }
uint32_t Plan::table_samples(uint32_t t) const { return t < impl_->tdesc.size() ? impl_->tdesc[t].n : 0; }
uint64_t Plan::table_offset(uint32_t t) const { return t < impl_->tdesc.size() ? impl_->tdesc[t].out_off : 0; }
uint64_t Plan::table_embedded(uint32_t t) const { return t < impl_->table_E.size() ? impl_->table_E[t] : 0; }
uint64_t Plan::n_embedded() const { return impl_->E; }
uint64_t Plan::work_units() const {
    uint64_t u = 0;
    for (size_t t = 0; t < impl_->tdesc.size(); t++) {
        const uint64_t n = impl_->tdesc[t].n;
        u += n * (n - (n ? 1 : 0)) / 2 * impl_->table_E[t];
    }
    return u;
}
uint64_t Plan::tensor_flops() const {
    if (!impl_->gemm) return 0;
    uint64_t units = 0;
    for (const auto &g : impl_->groups) units += g.n_tiles;
    return 2ull * tc::PRODUCTS * tc::UMMA_M * tc::UMMA_N * impl_->k_pad * units;
}
uint32_t Plan::launches() const { return impl_->launches; }
const char *Plan::pair_kernel_name() const {
    if (impl_->gemm) return "unweighted_tc_kernel";
    if (impl_->union_mode) return impl_->spec.vaw ? "pair_union<variance_adjusted>" : "pair_union<generalized>";
    if (impl_->hybrid)
        return impl_->spec.method == Method::weighted_normalized ? "pair_hybrid<weighted_normalized>"
                                                                 : "pair_hybrid<weighted_unnormalized>";
    return impl_->spec.fp64 ? impl_->kd.name : impl_->kf.name;
}
const char *Plan::tuning() const {
    static thread_local std::string s;
    if (impl_->gemm) {
        s = "tensor-core units, " + impl_->tuning;
        return s.c_str();
    }
    if (impl_->union_mode) return "sparse union 64x64";
    s = impl_->tuning + " " + (impl_->spec.fp64 ? impl_->kd.shape : impl_->kf.shape);
    return s.c_str();
}
void Plan::set_timing(bool on) { impl_->timing = on; }

int Plan::stage_times(StageTimes &out) {
    PlanImpl &m = *impl_;
    if (!m.timing || m.graph_on) return kOutputError;
    if (cudaEventSynchronize(m.ev[3]) != cudaSuccess) return kOutputError;
    cudaEventElapsedTime(&out.embed_ms, m.ev[0], m.ev[1]);
    cudaEventElapsedTime(&out.pair_ms, m.ev[1], m.ev[2]);
    cudaEventElapsedTime(&out.finalize_ms, m.ev[2], m.ev[3]);
    return 0;
}

}  // namespace ssu
