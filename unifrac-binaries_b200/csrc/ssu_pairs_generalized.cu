// Generalized UniFrac pair-kernel instances (src/unifrac_task_impl.hpp:924-1040),
// one operator per alpha kind (sqrt, identity, constant, pow).
#include "ssu_pairs.cuh"

namespace ssu {

namespace {
template <typename T, int AK>
std::vector<PairKernel<T>> family() {
    using Op = dev::OpGeneralized<T, AK>;
    return {values_kernel<T, Op, 128, 64, 8, 4, 16>("pair_values<generalized>", "128x64/8x4"),
            values_kernel<T, Op, 64, 64, 4, 4, 16>("pair_values<generalized>", "64x64/4x4")};
}
}  // namespace

template <typename T>
std::vector<PairKernel<T>> generalized_candidates(int ak) {
    switch (ak) {
    case 1: return family<T, 1>();
    case 2: return family<T, 2>();
    case 3: return family<T, 3>();
    default: return family<T, 0>();
    }
}

template std::vector<PairKernel<double>> generalized_candidates<double>(int);
template std::vector<PairKernel<float>> generalized_candidates<float>(int);

}  // namespace ssu
