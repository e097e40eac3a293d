// Device plan of the B200 UniFrac engine: upload, embedding, pair stage,
// output layouts.  One plan = one table on one GPU, one stream.
#include "ssu_engine.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <mutex>

#include "ssu_gemm.cuh"
#include "ssu_kernels.cuh"

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

// 2-D fp16 tensor map over a row-major [rows][cols] matrix with a
// 64-column x 128-row box and 128-byte swizzle (the UMMA K-major layout).
bool make_fp16_map(CUtensorMap *map, void *base, uint64_t rows, uint64_t cols) {
    EncodeTiledFn f = encode_tiled();
    if (!f) return false;
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {cols * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(tc::BLOCK_K), static_cast<cuuint32_t>(tc::BLOCK_M)};
    const cuuint32_t estr[2] = {1, 1};
    return f(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Type-erased pair stage: one kernel family with its tile shape.
template <typename T>
struct PairKernel {
    int BM = 0, BN = 0, threads = 0;
    int row_quantum = 1;     // node rows (or words) per pipeline stage
    size_t smem = 0;
    size_t partial_per_tile = 0;  // accumulator values per tile
    int blocks_per_sm = 1;
    const char *name = "";
    void (*launch)(const dev::PairArgs<T> &, dim3, size_t, cudaStream_t) = nullptr;
    void (*finalize)(const dev::PairArgs<T> &, uint32_t, cudaStream_t) = nullptr;
    cudaError_t (*configure)(size_t) = nullptr;
    cudaError_t (*occupancy)(int *, int, size_t) = nullptr;
};

template <typename T, class Op, int BM, int BN, int TM, int TN, int KC>
PairKernel<T> values_kernel(const char *name) {
    PairKernel<T> k;
    k.BM = BM;
    k.BN = BN;
    k.threads = (BM / TM) * (BN / TN);
    k.row_quantum = KC;
    k.smem = dev::pair_values_smem<T, Op, BM, BN, KC>();
    k.partial_per_tile = static_cast<size_t>(BM) * BN * Op::NACC;
    k.name = name;
    k.launch = [](const dev::PairArgs<T> &a, dim3 grid, size_t smem, cudaStream_t s) {
        dev::pair_values_kernel<T, Op, BM, BN, TM, TN, KC><<<grid, (BM / TM) * (BN / TN), smem, s>>>(a);
    };
    k.finalize = [](const dev::PairArgs<T> &a, uint32_t splits, cudaStream_t s) {
        dev::split_finalize_kernel<T, Op, BM, BN, TM, TN><<<a.n_tiles, (BM / TM) * (BN / TN), 0, s>>>(a, splits);
    };
    k.configure = [](size_t smem) {
        return cudaFuncSetAttribute(dev::pair_values_kernel<T, Op, BM, BN, TM, TN, KC>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    };
    k.occupancy = [](int *blocks, int threads, size_t smem) {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, dev::pair_values_kernel<T, Op, BM, BN, TM, TN, KC>,
                                                             threads, smem);
    };
    return k;
}

template <typename T, bool NORM, int BM, int BN, int TM, int TN, int KW>
PairKernel<T> bits_kernel(const char *name) {
    using Op = dev::OpUnweightedBits<T, NORM>;
    PairKernel<T> k;
    k.BM = BM;
    k.BN = BN;
    k.threads = (BM / TM) * (BN / TN);
    k.row_quantum = KW;
    k.smem = dev::pair_bits_smem<T, BM, BN, KW>();
    k.partial_per_tile = static_cast<size_t>(BM) * BN * Op::NACC;
    k.name = name;
    k.launch = [](const dev::PairArgs<T> &a, dim3 grid, size_t smem, cudaStream_t s) {
        dev::pair_bits_kernel<T, NORM, BM, BN, TM, TN, KW><<<grid, (BM / TM) * (BN / TN), smem, s>>>(a);
    };
    k.finalize = [](const dev::PairArgs<T> &a, uint32_t splits, cudaStream_t s) {
        dev::split_finalize_kernel<T, Op, BM, BN, TM, TN><<<a.n_tiles, (BM / TM) * (BN / TN), 0, s>>>(a, splits);
    };
    k.configure = [](size_t smem) {
        return cudaFuncSetAttribute(dev::pair_bits_kernel<T, NORM, BM, BN, TM, TN, KW>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    };
    k.occupancy = [](int *blocks, int threads, size_t smem) {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, dev::pair_bits_kernel<T, NORM, BM, BN, TM, TN, KW>,
                                                             threads, smem);
    };
    return k;
}

// alpha kind: 1 -> sqrt, 2 -> identity, 3 -> constant 1, 0 -> pow
int alpha_kind(double alpha) {
    if (alpha == 0.5) return 1;
    if (alpha == 1.0) return 2;
    if (alpha == 0.0) return 3;
    return 0;
}

template <typename T, template <typename, int> class OpT>
PairKernel<T> generalized_family(double alpha, const char *name) {
    switch (alpha_kind(alpha)) {
    case 1: return values_kernel<T, OpT<T, 1>, 128, 64, 8, 4, 16>(name);
    case 2: return values_kernel<T, OpT<T, 2>, 128, 64, 8, 4, 16>(name);
    case 3: return values_kernel<T, OpT<T, 3>, 128, 64, 8, 4, 16>(name);
    default: return values_kernel<T, OpT<T, 0>, 128, 64, 8, 4, 16>(name);
    }
}

template <typename T>
PairKernel<T> select_kernel(const MethodSpec &s) {
    constexpr bool D = sizeof(T) == 8;
    constexpr int KCW = D ? 16 : 32;
    if (s.vaw) {
        switch (s.method) {
        case Method::unweighted:
            return values_kernel<T, dev::OpVawUnweighted<T, true>, 128, 64, 8, 4, 16>("pair_values<vaw_unweighted>");
        case Method::unweighted_unnormalized:
            return values_kernel<T, dev::OpVawUnweighted<T, false>, 128, 64, 8, 4, 16>(
                "pair_values<vaw_unweighted_unnormalized>");
        case Method::weighted_normalized:
            return values_kernel<T, dev::OpVawWeighted<T, true>, 128, 64, 8, 4, 16>(
                "pair_values<vaw_weighted_normalized>");
        case Method::weighted_unnormalized:
            return values_kernel<T, dev::OpVawWeighted<T, false>, 128, 64, 8, 4, 16>(
                "pair_values<vaw_weighted_unnormalized>");
        case Method::generalized:
            return generalized_family<T, dev::OpVawGeneralized>(s.alpha, "pair_values<vaw_generalized>");
        }
    }
    switch (s.method) {
    case Method::unweighted:
        return bits_kernel<T, true, 128, 64, 8, 4, D ? 2 : 4>("pair_bits<unweighted>");
    case Method::unweighted_unnormalized:
        return bits_kernel<T, false, 128, 64, 8, 4, D ? 2 : 4>("pair_bits<unweighted_unnormalized>");
    case Method::weighted_normalized:
        return values_kernel<T, dev::OpWeighted<T, true>, 128, 128, 8, 8, KCW>("pair_values<weighted_normalized>");
    case Method::weighted_unnormalized:
        return values_kernel<T, dev::OpWeighted<T, false>, 128, 128, 8, 8, KCW>(
            "pair_values<weighted_unnormalized>");
    case Method::generalized:
        return generalized_family<T, dev::OpGeneralized>(s.alpha, "pair_values<generalized>");
    }
    return PairKernel<T>();
}

// Tiles (kb, lb) holding at least one pair k < l; with a stripe window only
// those whose pairs reach a stripe in [start, stop).
std::vector<uint2> make_tiles(uint32_t n, int BM, int BN, bool windowed, uint32_t start, uint32_t stop) {
    std::vector<uint2> tiles;
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
            tiles.push_back(make_uint2(kb, lb));
        }
    }
    return tiles;
}

}  // namespace

struct PlanImpl {
    MethodSpec spec;
    bool faith = false;
    uint32_t n = 0, K = 0, E = 0;
    uint64_t ld = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int n_sms = 148;
    std::string last_error;

    // inputs
    uint32_t *d_indptr = nullptr, *d_indices = nullptr;
    double *d_data = nullptr, *d_totals = nullptr;
    uint32_t *d_tip_rows = nullptr;
    int32_t *d_tip_obs = nullptr;
    uint32_t n_tips = 0;
    uint32_t *d_child_ptr = nullptr, *d_child_rows = nullptr, *d_level_rows = nullptr;
    std::vector<uint32_t> level_ptr;
    uint32_t *d_post_rows = nullptr;
    double *d_len_rows = nullptr;

    // embedding and method buffers
    void *d_U = nullptr, *d_C = nullptr, *d_len = nullptr, *d_tot = nullptr;
    void *d_W = nullptr, *d_part = nullptr;
    uint32_t n_parts = 0, part_chunk = 0;
    unsigned long long *d_P = nullptr;
    void *d_lut = nullptr;
    uint32_t n_words = 0;
    void *d_full = nullptr;

    // pair stage
    PairKernel<double> kd;
    PairKernel<float> kf;
    uint2 *d_tiles = nullptr;
    uint32_t n_tiles = 0, splits = 1, rows_per_split = 0;
    void *d_partial = nullptr;
    size_t partial_bytes = 0;

    std::vector<double> host_totals;  // per-sample totals, padded to ld

    // tensor-core unweighted path
    bool gemm = false;
    uint32_t n_pad = 0, k_pad = 0, n_chunks = 0;
    __half *d_A = nullptr, *d_Bh = nullptr, *d_Bl = nullptr, *d_lhi = nullptr, *d_llo = nullptr;
    double *d_r = nullptr, *d_lsorted = nullptr, *d_chunk_scale = nullptr, *d_G = nullptr;
    int32_t *d_parent_col = nullptr, *d_start_col = nullptr;
    uint32_t *d_sample_ptr = nullptr;
    int *d_error = nullptr;
    CUtensorMap map_A{}, map_Bh{}, map_Bl{};
    int setup_gemm(const Table &table, const FlatTree &tree);
    int execute_gemm(cudaStream_t s, const dev::OutSpec &out, const uint2 *tiles, uint32_t ntiles);

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

    int setup(const Table &table, const FlatTree &tree);
    template <typename T>
    int setup_method();
    template <typename T>
    int embed(cudaStream_t s);
    template <typename T>
    int prepare(cudaStream_t s);
    template <typename T>
    int pair_stage(cudaStream_t s, const dev::OutSpec &out, const uint2 *tiles, uint32_t n_tiles, uint32_t splits);
    template <typename T>
    int choose_splits(uint32_t tiles, uint32_t &splits, uint32_t &rows_per_split);
    template <typename T>
    int execute_T(cudaStream_t s, const dev::OutSpec &out, const uint2 *tiles, uint32_t n_tiles, uint32_t splits);
    int run_windowed(int mode, void *d_out, uint32_t start, uint32_t stop);
};

template <>
PairKernel<double> &PlanImpl::kern<double>() {
    return kd;
}
template <>
PairKernel<float> &PlanImpl::kern<float>() {
    return kf;
}

int PlanImpl::setup(const Table &table, const FlatTree &tree) {
    n = table.n_samples;
    K = tree.n_nodes;
    E = faith ? tree.n_nodes : tree.n_embedded;
    ld = ((static_cast<uint64_t>(n) + 127) / 128) * 128;
    int dev_id = 0;
    SSU_CK(cudaGetDevice(&dev_id));
    SSU_CK(cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, dev_id));
    pool = device_pool(dev_id);
    if (!stream) {
        SSU_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        own_stream = true;
    }
    const uint64_t nnz = table.nnz();
    SSU_CK(upload(&d_indptr, table.indptr, sizeof(uint32_t) * (table.n_obs + 1)));
    SSU_CK(upload(&d_indices, table.indices, sizeof(uint32_t) * nnz));
    SSU_CK(upload(&d_data, table.data, sizeof(double) * nnz));
    host_totals.assign(ld, 0.0);
    std::copy(table.totals.begin(), table.totals.end(), host_totals.begin());
    SSU_CK(upload(&d_totals, host_totals.data(), sizeof(double) * ld));

    std::vector<int32_t> tip_obs;
    tip_obs.reserve(tree.leaf_rows.size());
    for (uint32_t r : tree.leaf_rows) tip_obs.push_back(tree.leaf_obs[r]);
    n_tips = static_cast<uint32_t>(tree.leaf_rows.size());
    SSU_CK(upload(&d_tip_rows, tree.leaf_rows.data(), sizeof(uint32_t) * n_tips));
    SSU_CK(upload(&d_tip_obs, tip_obs.data(), sizeof(int32_t) * n_tips));
    SSU_CK(upload(&d_child_ptr, tree.child_ptr.data(), sizeof(uint32_t) * tree.child_ptr.size()));
    SSU_CK(upload(&d_child_rows, tree.child_rows.data(), sizeof(uint32_t) * tree.child_rows.size()));
    SSU_CK(upload(&d_level_rows, tree.level_rows.data(), sizeof(uint32_t) * tree.level_rows.size()));
    level_ptr = tree.level_ptr;
    if (faith) {
        SSU_CK(upload(&d_post_rows, tree.postorder_row.data(), sizeof(uint32_t) * tree.postorder_row.size()));
        SSU_CK(upload(&d_len_rows, tree.length.data(), sizeof(double) * tree.length.size()));
    }
    // embedded lengths in T, rows [0, E)
    if (spec.fp64 || faith) {
        std::vector<double> len(tree.length.begin(), tree.length.begin() + E);
        SSU_CK(upload(reinterpret_cast<double **>(&d_len), len.data(), sizeof(double) * E));
    } else {
        std::vector<float> len(E);
        for (uint32_t e = 0; e < E; e++) len[e] = static_cast<float>(tree.length[e]);
        SSU_CK(upload(reinterpret_cast<float **>(&d_len), len.data(), sizeof(float) * E));
    }
    for (auto &e : ev) SSU_CK(cudaEventCreate(&e));
    return 0;
}

template <typename T>
int PlanImpl::choose_splits(uint32_t tiles, uint32_t &out_splits, uint32_t &out_rows) {
    const PairKernel<T> &k = kern<T>();
    const uint32_t units = (spec.method == Method::unweighted || spec.method == Method::unweighted_unnormalized) &&
                                   !spec.vaw
                               ? n_words
                               : E;
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
    return 0;
}

template <typename T>
int PlanImpl::setup_method() {
    PairKernel<T> k = select_kernel<T>(spec);
    SSU_CK(k.configure(k.smem));
    int bps = 0;
    SSU_CK(k.occupancy(&bps, k.threads, k.smem));
    if (bps < 1) {
        last_error = "pair kernel does not fit on the device";
        return kOutputError;
    }
    k.blocks_per_sm = bps;
    kern<T>() = k;

    const size_t rowbytes = sizeof(T) * ld;
    SSU_CK(alloc(&d_U, rowbytes * std::max<uint32_t>(K, 1)));
    if (spec.vaw) {
        SSU_CK(alloc(&d_C, rowbytes * std::max<uint32_t>(K, 1)));
        std::vector<T> tot(ld, T(0));
        for (uint64_t j = 0; j < ld; j++) tot[j] = static_cast<T>(host_totals[j]);
        SSU_CK(upload(reinterpret_cast<T **>(&d_tot), tot.data(), sizeof(T) * ld));
    }
    const bool bits = !spec.vaw && (spec.method == Method::unweighted || spec.method == Method::unweighted_unnormalized);
    if (bits) {
        n_words = (E + 63) / 64;
        SSU_CK(alloc(&d_P, sizeof(unsigned long long) * ld * std::max<uint32_t>(n_words, 1)));
        SSU_CK(alloc(&d_lut, sizeof(T) * 2048 * std::max<uint32_t>(n_words, 1)));
    }
    if (!spec.vaw && spec.method == Method::weighted_normalized) {
        part_chunk = 512;
        n_parts = std::max<uint32_t>(1, (E + part_chunk - 1) / part_chunk);
        SSU_CK(alloc(&d_W, sizeof(T) * ld));
        SSU_CK(alloc(&d_part, sizeof(T) * ld * n_parts));
    }
    SSU_CK(alloc(&d_full, sizeof(T) * static_cast<uint64_t>(n) * n));

    std::vector<uint2> tiles = make_tiles(n, k.BM, k.BN, false, 0, 0);
    n_tiles = static_cast<uint32_t>(tiles.size());
    SSU_CK(upload(&d_tiles, tiles.data(), sizeof(uint2) * tiles.size()));
    choose_splits<T>(n_tiles, splits, rows_per_split);
    if (splits > 1) {
        partial_bytes = sizeof(T) * k.partial_per_tile * n_tiles * splits;
        SSU_CK(alloc(&d_partial, partial_bytes));
    }
    return 0;
}

template <typename T>
int PlanImpl::embed(cudaStream_t s) {
    if (K == 0) return 0;
    const bool counts = spec.vaw && !faith;
    T *U = static_cast<T *>(d_U);
    T *C = static_cast<T *>(d_C);
    const bool normalize = faith ? true : spec.normalize;
    if (n_tips) {
        const uint32_t grid = std::min<uint32_t>(n_tips, 65535u * 8);
        if (counts)
            dev::embed_tips_kernel<T, true><<<grid, 256, 0, s>>>(d_tip_rows, d_tip_obs, n_tips, d_indptr, d_indices,
                                                                 d_data, d_totals, normalize, U, C, ld);
        else
            dev::embed_tips_kernel<T, false><<<grid, 256, 0, s>>>(d_tip_rows, d_tip_obs, n_tips, d_indptr, d_indices,
                                                                  d_data, d_totals, normalize, U, C, ld);
        launches++;
    }
    const uint64_t nvec = ld / dev::Vec16<T>::n;
    const uint32_t threads = 128;
    const uint32_t col_blocks = static_cast<uint32_t>((nvec + threads - 1) / threads);
    for (size_t h = 1; h < level_ptr.size(); h++) {
        const uint32_t a = level_ptr[h - 1], b = level_ptr[h];
        if (b == a) continue;
        const uint64_t blocks = static_cast<uint64_t>(b - a) * col_blocks;
        const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>(blocks, 1u << 20));
        if (counts)
            dev::embed_level_kernel<T, true><<<grid, threads, 0, s>>>(d_level_rows + a, b - a, d_child_ptr,
                                                                      d_child_rows, U, C, ld, col_blocks);
        else
            dev::embed_level_kernel<T, false><<<grid, threads, 0, s>>>(d_level_rows + a, b - a, d_child_ptr,
                                                                       d_child_rows, U, C, ld, col_blocks);
        launches++;
    }
    SSU_CK(cudaGetLastError());
    return 0;
}

template <typename T>
int PlanImpl::prepare(cudaStream_t s) {
    const T *U = static_cast<const T *>(d_U);
    const T *len = static_cast<const T *>(d_len);
    if (d_W) {
        dim3 grid(static_cast<uint32_t>((ld + 255) / 256), n_parts);
        dev::weighted_sums_partial_kernel<T><<<grid, 256, 0, s>>>(U, len, E, ld, part_chunk, static_cast<T *>(d_part));
        dev::reduce_partials_kernel<T><<<static_cast<uint32_t>((ld + 255) / 256), 256, 0, s>>>(
            static_cast<const T *>(d_part), n_parts, ld, static_cast<T *>(d_W));
        launches += 2;
    }
    if (d_P && n_words) {
        const uint64_t total = static_cast<uint64_t>(n_words) * ld;
        const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>((total + 255) / 256, 1u << 20));
        dev::pack_presence_kernel<T><<<grid, 256, 0, s>>>(U, E, ld, n_words, d_P);
        dev::build_lut_kernel<T><<<n_words * 8, 256, 0, s>>>(len, E, static_cast<T *>(d_lut));
        launches += 2;
    }
    SSU_CK(cudaGetLastError());
    return 0;
}

template <typename T>
int PlanImpl::pair_stage(cudaStream_t s, const dev::OutSpec &out, const uint2 *tiles, uint32_t ntiles,
                         uint32_t nsplits) {
    const PairKernel<T> &k = kern<T>();
    if (ntiles == 0) return 0;
    dev::PairArgs<T> a{};
    a.tiles = tiles;
    a.n_tiles = ntiles;
    a.U = static_cast<const T *>(d_U);
    a.C = static_cast<const T *>(d_C);
    a.len = static_cast<const T *>(d_len);
    a.tot = static_cast<const T *>(d_tot);
    a.W = static_cast<const T *>(d_W);
    a.P = d_P;
    a.lut = static_cast<const T *>(d_lut);
    const bool bits = d_P != nullptr;
    a.E = bits ? n_words : E;
    a.ld = ld;
    a.n = n;
    a.alpha = static_cast<T>(spec.alpha);
    a.out = out;
    uint32_t rows = rows_per_split;
    if (nsplits <= 1) {
        nsplits = 1;
        rows = bits ? n_words : E;
        a.partial = nullptr;
    } else {
        a.partial = static_cast<T *>(d_partial);
    }
    a.rows_per_split = rows;
    dim3 grid(ntiles, nsplits);
    k.launch(a, grid, k.smem, s);
    launches++;
    if (timing) SSU_CK(cudaEventRecord(ev[2], s));
    if (nsplits > 1) {
        k.finalize(a, nsplits, s);
        launches++;
    }
    SSU_CK(cudaGetLastError());
    return 0;
}

template <typename T>
int PlanImpl::execute_T(cudaStream_t s, const dev::OutSpec &out, const uint2 *tiles, uint32_t ntiles,
                        uint32_t nsplits) {
    launches = 0;
    if (timing) SSU_CK(cudaEventRecord(ev[0], s));
    int rc = embed<T>(s);
    if (rc) return rc;
    rc = prepare<T>(s);
    if (rc) return rc;
    if (timing) SSU_CK(cudaEventRecord(ev[1], s));
    rc = pair_stage<T>(s, out, tiles, ntiles, nsplits);
    if (rc) return rc;
    if (timing && ntiles == 0) SSU_CK(cudaEventRecord(ev[2], s));
    if (out.mode == 0 && n) {
        dev::zero_diagonal_kernel<<<(n + 255) / 256, 256, 0, s>>>(out.ptr, n, sizeof(T) == 8);
        launches++;
    }
    if (timing) SSU_CK(cudaEventRecord(ev[3], s));
    SSU_CK(cudaGetLastError());
    return 0;
}

int PlanImpl::run_windowed(int mode, void *d_out, uint32_t start, uint32_t stop) {
    if (gemm) {
        dev::OutSpec o{mode, d_out, start, stop};
        return execute_gemm(stream, o, d_tiles, n_tiles);
    }
    const int BM = spec.fp64 ? kd.BM : kf.BM, BN = spec.fp64 ? kd.BN : kf.BN;
    std::vector<uint2> tiles = make_tiles(n, BM, BN, mode == 1, start, stop);
    uint2 *d_t = nullptr;
    SSU_CK(upload(&d_t, tiles.data(), sizeof(uint2) * tiles.size()));
    uint32_t s = 1, rows = 0;
    (void)s;
    if (spec.fp64)
        choose_splits<double>(static_cast<uint32_t>(tiles.size()), s, rows);
    else
        choose_splits<float>(static_cast<uint32_t>(tiles.size()), s, rows);
    // the window never holds more tiles than the full matrix, so the plan's
    // partial buffer is large enough when the split count does not grow
    const size_t per_tile = spec.fp64 ? kd.partial_per_tile * sizeof(double) : kf.partial_per_tile * sizeof(float);
    if (s > 1 && per_tile * tiles.size() * s > partial_bytes) s = 1;
    const uint32_t saved = rows_per_split;
    rows_per_split = rows;
    dev::OutSpec o{mode, d_out, start, stop};
    int rc = spec.fp64 ? execute_T<double>(stream, o, d_t, static_cast<uint32_t>(tiles.size()), s)
                       : execute_T<float>(stream, o, d_t, static_cast<uint32_t>(tiles.size()), s);
    rows_per_split = saved;
    return rc;
}

// --------------------------------------------------- tensor-core unweighted

int PlanImpl::setup_gemm(const Table &table, const FlatTree &tree) {
    const uint32_t chunk_nodes = tc::CHUNK_KB * tc::BLOCK_K;
    n_pad = ((n + tc::BLOCK_M - 1) / tc::BLOCK_M) * tc::BLOCK_M;
    k_pad = std::max<uint32_t>(chunk_nodes, ((E + chunk_nodes - 1) / chunk_nodes) * chunk_nodes);
    n_chunks = k_pad / chunk_nodes;
    // embedded nodes sorted by decreasing length
    std::vector<uint32_t> order(E);
    for (uint32_t e = 0; e < E; e++) order[e] = e;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return tree.length[a] > tree.length[b]; });
    std::vector<int32_t> col_of_row(tree.n_nodes, -1);
    for (uint32_t c = 0; c < E; c++) col_of_row[order[c]] = static_cast<int32_t>(c);
    std::vector<double> lsorted(k_pad, 0.0), scale(n_chunks, 1.0);
    std::vector<__half> lhi(k_pad, __float2half(0.0f)), llo(k_pad, __float2half(0.0f));
    for (uint32_t c = 0; c < E; c++) lsorted[c] = tree.length[order[c]];
    for (uint32_t ch = 0; ch < n_chunks; ch++) {
        const double mx = lsorted[ch * chunk_nodes];
        int sig = 0;
        if (mx > 0) sig = 14 - static_cast<int>(std::floor(std::log2(mx)));
        scale[ch] = std::ldexp(1.0, -sig);
        for (uint32_t c = ch * chunk_nodes; c < (ch + 1) * chunk_nodes; c++) {
            const double x = std::ldexp(lsorted[c], sig);
            const __half h = __double2half(x);
            lhi[c] = h;
            llo[c] = __double2half(x - static_cast<double>(__half2float(h)));
        }
    }
    // parents among embedded nodes
    std::vector<int32_t> parent_row(tree.n_nodes, -1);
    for (uint32_t r = 0; r < tree.n_nodes; r++)
        for (uint32_t c = tree.child_ptr[r]; c < tree.child_ptr[r + 1]; c++) parent_row[tree.child_rows[c]] = r;
    std::vector<int32_t> parent_col(k_pad, -1);
    for (uint32_t c = 0; c < E; c++) {
        const int32_t p = parent_row[order[c]];
        parent_col[c] = (p >= 0 && static_cast<uint32_t>(p) < E) ? col_of_row[p] : -1;
    }
    // sample-major list of starting columns (tip, or its parent when tips are bypassed)
    std::vector<int32_t> start_of_obs(table.n_obs, -1);
    for (uint32_t r : tree.leaf_rows) {
        const int32_t obs = tree.leaf_obs[r];
        if (obs < 0) continue;
        int32_t node = static_cast<int32_t>(r);
        if (r >= E) node = parent_row[r];
        start_of_obs[obs] = (node >= 0 && static_cast<uint32_t>(node) < E) ? col_of_row[node] : -1;
    }
    std::vector<uint32_t> sample_ptr(n + 1, 0);
    for (uint32_t i = 0; i < table.n_obs; i++)
        for (uint32_t q = table.indptr[i]; q < table.indptr[i + 1]; q++)
            if (table.data[q] > 0.0 && start_of_obs[i] >= 0) sample_ptr[table.indices[q] + 1]++;
    for (uint32_t j = 0; j < n; j++) sample_ptr[j + 1] += sample_ptr[j];
    std::vector<int32_t> start_col(std::max<uint32_t>(sample_ptr[n], 1));
    std::vector<uint32_t> fill(sample_ptr.begin(), sample_ptr.end() - 1);
    for (uint32_t i = 0; i < table.n_obs; i++)
        for (uint32_t q = table.indptr[i]; q < table.indptr[i + 1]; q++)
            if (table.data[q] > 0.0 && start_of_obs[i] >= 0) start_col[fill[table.indices[q]]++] = start_of_obs[i];

    const size_t op_bytes = sizeof(__half) * static_cast<size_t>(n_pad) * k_pad;
    SSU_CK(alloc(&d_A, op_bytes));
    SSU_CK(alloc(&d_Bh, op_bytes));
    SSU_CK(alloc(&d_Bl, op_bytes));
    SSU_CK(alloc(&d_r, sizeof(double) * n_pad));
    SSU_CK(alloc(&d_G, sizeof(double) * static_cast<size_t>(n_pad) * n_pad));
    SSU_CK(upload(&d_lhi, lhi.data(), sizeof(__half) * k_pad));
    SSU_CK(upload(&d_llo, llo.data(), sizeof(__half) * k_pad));
    SSU_CK(upload(&d_lsorted, lsorted.data(), sizeof(double) * k_pad));
    SSU_CK(upload(&d_chunk_scale, scale.data(), sizeof(double) * n_chunks));
    SSU_CK(upload(&d_parent_col, parent_col.data(), sizeof(int32_t) * k_pad));
    SSU_CK(upload(&d_sample_ptr, sample_ptr.data(), sizeof(uint32_t) * (n + 1)));
    SSU_CK(upload(&d_start_col, start_col.data(), sizeof(int32_t) * start_col.size()));
    SSU_CK(alloc(&d_error, sizeof(int)));
    SSU_CK(cudaMemsetAsync(d_error, 0, sizeof(int), stream));
    if (!make_fp16_map(&map_A, d_A, n_pad, k_pad) || !make_fp16_map(&map_Bh, d_Bh, n_pad, k_pad) ||
        !make_fp16_map(&map_Bl, d_Bl, n_pad, k_pad)) {
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
    // every ordered tile of G, grouped 12 x 12 so concurrent CTAs share row
    // blocks in L2
    std::vector<uint2> tiles;
    const uint32_t nb = n_pad / tc::BLOCK_M;
    for (uint32_t gk = 0; gk < nb; gk += 12)
        for (uint32_t gl = 0; gl < nb; gl += 12)
            for (uint32_t kb = gk; kb < std::min(nb, gk + 12); kb++)
                for (uint32_t lb = gl; lb < std::min(nb, gl + 12); lb++) tiles.push_back(make_uint2(kb, lb));
    n_tiles = static_cast<uint32_t>(tiles.size());
    SSU_CK(upload(&d_tiles, tiles.data(), sizeof(uint2) * tiles.size()));
    gemm = true;
    return 0;
}

int PlanImpl::execute_gemm(cudaStream_t s, const dev::OutSpec &out, const uint2 *tiles, uint32_t ntiles) {
    launches = 0;
    if (timing) SSU_CK(cudaEventRecord(ev[0], s));
    const size_t bits_smem = sizeof(uint32_t) * (k_pad / 32);
    tc::presence_rows_kernel<<<n_pad, 256, bits_smem, s>>>(d_sample_ptr, d_start_col, d_parent_col, d_lhi, d_llo,
                                                           d_lsorted, n, k_pad, d_A, d_Bh, d_Bl, d_r);
    launches++;
    if (timing) SSU_CK(cudaEventRecord(ev[1], s));
    if (ntiles) {
        tc::GemmArgs g{};
        g.tiles = tiles;
        g.n_tiles = ntiles;
        g.n = n;
        g.n_kblocks = k_pad / tc::BLOCK_K;
        g.chunk_scale = d_chunk_scale;
        g.G = d_G;
        g.ldg = n_pad;
        g.error = d_error;
        g.wait_cycles = 2000000000LL;  // about one second per wait at B200 clocks
        tc::unweighted_tc_kernel<<<ntiles, tc::THREADS, tc::SMEM_BYTES, s>>>(map_A, map_Bh, map_Bl, g);
        launches++;
    }
    if (timing) SSU_CK(cudaEventRecord(ev[2], s));
    if (n) {
        const dim3 grid((n + 31) / 32, (n + 31) / 32);
        tc::finish_unweighted_kernel<<<grid, dim3(32, 8), 0, s>>>(d_G, n_pad, d_r, n,
                                                                  spec.method == Method::unweighted ? 1 : 0,
                                                                  spec.fp64 ? 1 : 0, out);
        launches++;
    }
    if (out.mode == 0 && n) {
        dev::zero_diagonal_kernel<<<(n + 255) / 256, 256, 0, s>>>(out.ptr, n, spec.fp64 ? 1 : 0);
        launches++;
    }
    if (timing) SSU_CK(cudaEventRecord(ev[3], s));
    SSU_CK(cudaGetLastError());
    return 0;
}

// ------------------------------------------------------------------ Plan

int Plan::create(const Table &table, const FlatTree &tree, const MethodSpec &spec, void *stream, Plan **out,
                 std::string &err) {
    Plan *p = new Plan();
    p->impl_ = new PlanImpl();
    PlanImpl &m = *p->impl_;
    m.spec = spec;
    m.stream = static_cast<cudaStream_t>(stream);
    int rc = m.setup(table, tree);
    bool want_gemm = spec.unweighted_gemm && !spec.vaw &&
                     (spec.method == Method::unweighted || spec.method == Method::unweighted_unnormalized);
    // presence is "proportion > 0": with no negative count it is the OR of
    // the tips below a node; other inputs keep the stripe kernel
    for (uint64_t q = 0; want_gemm && q < table.nnz(); q++)
        if (!(table.data[q] >= 0.0)) want_gemm = false;
    if (!rc && want_gemm) {
        rc = m.setup_gemm(table, tree);
        if (!rc && m.alloc(&m.d_full, (spec.fp64 ? sizeof(double) : sizeof(float)) * static_cast<uint64_t>(m.n) * m.n) !=
                       cudaSuccess) {
            m.last_error = "device allocation failed";
            rc = kOutputError;
        }
    } else if (!rc) {
        rc = spec.fp64 ? m.setup_method<double>() : m.setup_method<float>();
    }
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
    int rc = m.setup(table, tree);
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
    if (m.stream) {
        for (void *q : m.allocations) cudaFreeAsync(q, m.stream);
        cudaStreamSynchronize(m.stream);
    }
    for (auto &e : m.ev)
        if (e) cudaEventDestroy(e);
    if (m.own_stream && m.stream) cudaStreamDestroy(m.stream);
    delete impl_;
}

int Plan::execute(void *stream) {
    PlanImpl &m = *impl_;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : m.stream;
    dev::OutSpec o{0, m.d_full, 0, 0};
    if (m.gemm) return m.execute_gemm(s, o, m.d_tiles, m.n_tiles);
    return m.spec.fp64 ? m.execute_T<double>(s, o, m.d_tiles, m.n_tiles, m.splits)
                       : m.execute_T<float>(s, o, m.d_tiles, m.n_tiles, m.splits);
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
        const size_t bytes = (m.spec.fp64 ? sizeof(double) : sizeof(float)) * static_cast<size_t>(m.n) * m.n;
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

int Plan::download_full(void *host_out, bool pin, std::string &err) {
    PlanImpl &m = *impl_;
    const size_t bytes = (m.spec.fp64 ? sizeof(double) : sizeof(float)) * static_cast<size_t>(m.n) * m.n;
    bool registered = false;
    if (pin && bytes >= (size_t(1) << 20))
        registered = cudaHostRegister(host_out, bytes, cudaHostRegisterDefault) == cudaSuccess;
    if (pin && !registered) cudaGetLastError();  // a refused registration only means a pageable copy
    cudaError_t e = cudaMemcpyAsync(host_out, m.d_full, bytes, cudaMemcpyDeviceToHost, m.stream);
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
    int rc = m.embed<double>(m.stream);
    if (rc) {
        err = m.last_error;
        return rc;
    }
    const uint32_t chunk = 1024;
    const uint32_t parts = std::max<uint32_t>(1, (m.K + chunk - 1) / chunk);
    double *d_part = nullptr, *d_out = nullptr;
    if (m.alloc(&d_part, sizeof(double) * m.ld * parts) != cudaSuccess ||
        m.alloc(&d_out, sizeof(double) * m.ld) != cudaSuccess) {
        err = "device allocation failed";
        return kOutputError;
    }
    dim3 grid(static_cast<uint32_t>((m.ld + 255) / 256), parts);
    dev::faith_partial_kernel<<<grid, 256, 0, m.stream>>>(static_cast<const double *>(m.d_U), m.d_len_rows,
                                                          m.d_post_rows, m.K, m.ld, chunk, d_part);
    dev::reduce_partials_kernel<double><<<static_cast<uint32_t>((m.ld + 255) / 256), 256, 0, m.stream>>>(
        d_part, parts, m.ld, d_out);
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
    const size_t bytes = (m.spec.fp64 ? sizeof(double) : sizeof(float)) * static_cast<size_t>(m.n) * m.n;
    if (cudaMemcpyAsync(host_out, m.d_full, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess) return kOutputError;
    if (cudaStreamSynchronize(s) != cudaSuccess) return kOutputError;
    return device_error() ? kOutputError : 0;
}

int Plan::synchronize() { return cudaStreamSynchronize(impl_->stream) == cudaSuccess ? 0 : kOutputError; }

uint32_t Plan::n_samples() const { return impl_->n; }
uint64_t Plan::n_embedded() const { return impl_->E; }
uint64_t Plan::work_units() const {
    const uint64_t n = impl_->n;
    return n * (n - (n ? 1 : 0)) / 2 * impl_->E;
}
uint32_t Plan::launches() const { return impl_->launches; }
const char *Plan::pair_kernel_name() const {
    if (impl_->gemm) return "unweighted_tc_kernel";
    return impl_->spec.fp64 ? impl_->kd.name : impl_->kf.name;
}
void Plan::set_timing(bool on) { impl_->timing = on; }

int Plan::stage_times(StageTimes &out) {
    PlanImpl &m = *impl_;
    if (!m.timing) return kOutputError;
    if (cudaEventSynchronize(m.ev[3]) != cudaSuccess) return kOutputError;
    cudaEventElapsedTime(&out.embed_ms, m.ev[0], m.ev[1]);
    cudaEventElapsedTime(&out.pair_ms, m.ev[1], m.ev[2]);
    cudaEventElapsedTime(&out.finalize_ms, m.ev[2], m.ev[3]);
    return 0;
}

}  // namespace ssu
