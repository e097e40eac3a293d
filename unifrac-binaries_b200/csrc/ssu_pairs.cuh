// Pair-stage kernel registry: every (operator, tile shape) instance the
// engine can launch, type-erased so the plan and the autotuner pick among
// them at run time.  The instances of each method family are compiled in
// their own translation unit (ssu_pairs_*.cu).
#pragma once

#include <vector>

#include "ssu_engine.hpp"
#include "ssu_kernels.cuh"

namespace ssu {

template <typename T>
struct PairKernel {
    int BM = 0, BN = 0, threads = 0;
    int row_quantum = 1;          // node rows (or words) per pipeline stage
    size_t smem = 0;
    size_t partial_per_tile = 0;  // accumulator values per tile
    int blocks_per_sm = 1;
    const char *name = "";
    const char *shape = "";
    void (*launch)(const dev::PairArgs<T> &, uint32_t ctas, size_t smem, cudaStream_t) = nullptr;
    void (*finalize)(const dev::PairArgs<T> &, cudaStream_t) = nullptr;
    cudaError_t (*configure)(size_t) = nullptr;
    cudaError_t (*occupancy)(int *, int, size_t) = nullptr;
};

template <typename T, class Op, int BM, int BN, int TM, int TN, int KC>
PairKernel<T> values_kernel(const char *name, const char *shape) {
    PairKernel<T> k;
    k.BM = BM;
    k.BN = BN;
    k.threads = (BM / TM) * (BN / TN);
    k.row_quantum = KC;
    k.smem = dev::pair_values_smem<T, Op, BM, BN, KC>();
    k.partial_per_tile = static_cast<size_t>(BM) * BN * Op::NACC;
    k.name = name;
    k.shape = shape;
    k.launch = [](const dev::PairArgs<T> &a, uint32_t ctas, size_t smem, cudaStream_t s) {
        dev::pair_values_kernel<T, Op, BM, BN, TM, TN, KC><<<ctas, (BM / TM) * (BN / TN), smem, s>>>(a);
    };
    k.finalize = [](const dev::PairArgs<T> &a, cudaStream_t s) {
        dev::split_finalize_kernel<T, Op, BM, BN, TM, TN><<<a.n_tiles, (BM / TM) * (BN / TN), 0, s>>>(a, a.n_splits);
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
PairKernel<T> bits_kernel(const char *name, const char *shape) {
    using Op = dev::OpUnweightedBits<T, NORM>;
    PairKernel<T> k;
    k.BM = BM;
    k.BN = BN;
    k.threads = (BM / TM) * (BN / TN);
    k.row_quantum = KW;
    k.smem = dev::pair_bits_smem<T, BM, BN, KW>();
    k.partial_per_tile = static_cast<size_t>(BM) * BN * Op::NACC;
    k.name = name;
    k.shape = shape;
    k.launch = [](const dev::PairArgs<T> &a, uint32_t ctas, size_t smem, cudaStream_t s) {
        dev::pair_bits_kernel<T, NORM, BM, BN, TM, TN, KW><<<ctas, (BM / TM) * (BN / TN), smem, s>>>(a);
    };
    k.finalize = [](const dev::PairArgs<T> &a, cudaStream_t s) {
        dev::split_finalize_kernel<T, Op, BM, BN, TM, TN><<<a.n_tiles, (BM / TM) * (BN / TN), 0, s>>>(a, a.n_splits);
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
inline int alpha_kind(double alpha) {
    if (alpha == 0.5) return 1;
    if (alpha == 1.0) return 2;
    if (alpha == 0.0) return 3;
    return 0;
}

// Candidate instances of each family, the default (heuristic) choice first.
template <typename T>
std::vector<PairKernel<T>> weighted_candidates(bool normalized);
template <typename T>
std::vector<PairKernel<T>> generalized_candidates(int alpha_kind);
template <typename T>
std::vector<PairKernel<T>> vaw_candidates(Method method, int alpha_kind);
template <typename T>
std::vector<PairKernel<T>> bits_candidates(bool normalized);

template <typename T>
std::vector<PairKernel<T>> pair_candidates(const MethodSpec &s) {
    if (s.vaw) return vaw_candidates<T>(s.method, alpha_kind(s.alpha));
    switch (s.method) {
    case Method::unweighted: return bits_candidates<T>(true);
    case Method::unweighted_unnormalized: return bits_candidates<T>(false);
    case Method::weighted_normalized: return weighted_candidates<T>(true);
    case Method::weighted_unnormalized: return weighted_candidates<T>(false);
    case Method::generalized: return generalized_candidates<T>(alpha_kind(s.alpha));
    }
    return {};
}

}  // namespace ssu
