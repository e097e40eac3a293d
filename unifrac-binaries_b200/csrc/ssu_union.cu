// Instances of the union kernel, one per method operator (ssu_union.cuh).
#include "ssu_engine.hpp"
#include "ssu_pairs.cuh"
#include "ssu_union.cuh"

namespace ssu {
namespace dev {

namespace {

// The kernel's setmaxnreg split assumes the block launches with exactly
// UREG_LAUNCH registers per thread: with fewer, the consumers' increase could
// never be granted.  An instance built otherwise is refused here, before any
// launch.
template <typename T, class Op>
cudaError_t configure_one(size_t *smem) {
    *smem = union_smem<T, Op::COUNTS>();
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, pair_union_kernel<T, Op>);
    if (e != cudaSuccess) return e;
    if (fa.numRegs != UREG_LAUNCH || fa.maxThreadsPerBlock < UTHREADS) return cudaErrorInvalidConfiguration;
    return cudaFuncSetAttribute(pair_union_kernel<T, Op>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(*smem));
}

template <typename T, class Op>
cudaError_t launch_one(const CUtensorMap &tmU, const CUtensorMap &tmC, const UnionArgs<T> &a, uint32_t ctas,
                       cudaStream_t s) {
    pair_union_kernel<T, Op><<<ctas, UTHREADS, union_smem<T, Op::COUNTS>(), s>>>(tmU, tmC, a);
    if (a.partial) union_finalize_kernel<T, Op><<<a.n_tiles, UFIN_THREADS, 0, s>>>(a);
    return cudaGetLastError();
}

// Calls f.template operator()<Op>() for the method's operator in precision R.
template <typename R, class F>
cudaError_t with_op(const MethodSpec &spec, F &&f) {
    const int ak = alpha_kind(spec.alpha);
    if (!spec.vaw) {
        switch (ak) {
        case 1: return f.template operator()<OpGeneralized<R, 1>>();
        case 2: return f.template operator()<OpGeneralized<R, 2>>();
        case 3: return f.template operator()<OpGeneralized<R, 3>>();
        default: return f.template operator()<OpGeneralized<R, 0>>();
        }
    }
    switch (spec.method) {
    case Method::unweighted: return f.template operator()<OpVawUnweighted<R, true>>();
    case Method::unweighted_unnormalized: return f.template operator()<OpVawUnweighted<R, false>>();
    case Method::weighted_normalized: return f.template operator()<OpVawWeighted<R, true>>();
    case Method::weighted_unnormalized: return f.template operator()<OpVawWeighted<R, false>>();
    case Method::generalized:
        switch (ak) {
        case 1: return f.template operator()<OpVawGeneralized<R, 1>>();
        case 2: return f.template operator()<OpVawGeneralized<R, 2>>();
        case 3: return f.template operator()<OpVawGeneralized<R, 3>>();
        default: return f.template operator()<OpVawGeneralized<R, 0>>();
        }
    }
    return cudaErrorInvalidValue;
}

}  // namespace

template <typename T>
struct Configure {
    size_t *smem;
    template <class Op>
    cudaError_t operator()() const {
        return configure_one<T, Op>(smem);
    }
};

template <typename T>
struct Launch {
    const CUtensorMap &tmU, &tmC;
    const UnionArgs<T> &a;
    uint32_t ctas;
    cudaStream_t s;
    template <class Op>
    cudaError_t operator()() const {
        return launch_one<T, Op>(tmU, tmC, a, ctas, s);
    }
};

template <typename T>
cudaError_t union_configure(const MethodSpec &spec, size_t *smem) {
    return with_op<T>(spec, Configure<T>{smem});
}

template <typename T>
cudaError_t union_launch(const MethodSpec &spec, const CUtensorMap &tmU, const CUtensorMap &tmC,
                         const UnionArgs<T> &a, uint32_t ctas, cudaStream_t s) {
    return with_op<T>(spec, Launch<T>{tmU, tmC, a, ctas, s});
}

template cudaError_t union_configure<double>(const MethodSpec &, size_t *);
template cudaError_t union_configure<float>(const MethodSpec &, size_t *);
template cudaError_t union_launch<double>(const MethodSpec &, const CUtensorMap &, const CUtensorMap &,
                                          const UnionArgs<double> &, uint32_t, cudaStream_t);
template cudaError_t union_launch<float>(const MethodSpec &, const CUtensorMap &, const CUtensorMap &,
                                         const UnionArgs<float> &, uint32_t, cudaStream_t);

}  // namespace dev
}  // namespace ssu
