// Unweighted presence-word pair-kernel instances
// (src/unifrac_task_impl.hpp:1424-1753).
#include "ssu_pairs.cuh"

namespace ssu {

template <typename T>
std::vector<PairKernel<T>> bits_candidates(bool normalized) {
    constexpr int KW = sizeof(T) == 8 ? 2 : 4;
    if (normalized)
        return {bits_kernel<T, true, 128, 64, 8, 4, KW>("pair_bits<unweighted>", "128x64/8x4"),
                bits_kernel<T, true, 64, 64, 4, 4, KW>("pair_bits<unweighted>", "64x64/4x4")};
    return {bits_kernel<T, false, 128, 64, 8, 4, KW>("pair_bits<unweighted_unnormalized>", "128x64/8x4"),
            bits_kernel<T, false, 64, 64, 4, 4, KW>("pair_bits<unweighted_unnormalized>", "64x64/4x4")};
}

template std::vector<PairKernel<double>> bits_candidates<double>(bool);
template std::vector<PairKernel<float>> bits_candidates<float>(bool);

}  // namespace ssu
