// Weighted UniFrac pair stage for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc (or any allocating routine) at the point
// where they want distances: code running inside a host framework that owns
// all device memory through its own arena or pool, a process with a fixed
// device-memory budget handed out up front, or an embedding where every
// buffer is carved out of one region before work starts.  They can still
// pass their own device buffers for inputs and outputs.  This entry point
// runs the weighted (normalized or unnormalized) pair kernel of the engine
// over such buffers and takes the little scratch it needs - the split-K
// partial tiles, the per-sample weighted sums and the tile list - from one
// file-scope device array instead of allocating.
//
// Limits and sharing rules (also stated in include/unifrac_b200.h):
//  * the scratch array is kScratchBytes (32 MiB) and lives on every GPU that
//    loads this library until the process exits;
//  * n_samples is limited to kMaxSamples, and a call whose scratch needs
//    exceed the array is rejected with output_error and a message;
//  * every call on a device shares the one array, which keeps whatever the
//    last call left there; calls that overlap on the GPU (different streams,
//    or different host threads without ordering) race on it;
//  * nothing in the scratch has to start at zero: every value a call reads is
//    written earlier in the same call (the tile list and the table descriptor
//    by a small kernel, so no call reads host memory once it has returned);
//  * d_embedding must be 16-byte aligned, d_lengths and d_out 8-byte aligned
//    (output_error otherwise);
//  * the first call on a device resolves the array's device address
//    (cudaGetSymbolAddress) and sets the pair kernel's shared-memory limit,
//    so that first call should come before any stream capture.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "ssu_kernels.cuh"
#include "unifrac_b200.h"

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr uint32_t kMaxSamples = 100000;
constexpr int BM = 128, BN = 128, TM = 8, TN = 8, KC = 16;
constexpr uint32_t kWChunk = 512;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

template <bool NORM>
using WeightedOp = ssu::dev::OpWeighted<double, NORM>;

struct DeviceSetup {
    bool ready = false;
    void *scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int n_sms = 0;
    int blocks_per_sm = 1;
};

std::mutex g_setup_mu;
std::vector<DeviceSetup> g_setup;

void note(const char *msg) { std::fprintf(stderr, "unifrac-b200 (no-alloc): %s\n", msg); }

// Once per device, with that device current: the host-side address of the
// scratch array (its name on the host is only a stand-in) and kernel limits.
bool setup_device(int dev, DeviceSetup &out) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (g_setup.size() <= static_cast<size_t>(dev)) g_setup.resize(dev + 1);
    DeviceSetup &s = g_setup[dev];
    if (!s.ready) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) {
            note(cudaGetErrorString(e));
            return false;
        }
        if (cudaDeviceGetAttribute(&s.n_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return false;
        const size_t smem = ssu::dev::pair_values_smem<double, WeightedOp<true>, BM, BN, KC>();
        auto k1 = ssu::dev::pair_values_kernel<double, WeightedOp<true>, BM, BN, TM, TN, KC>;
        auto k0 = ssu::dev::pair_values_kernel<double, WeightedOp<false>, BM, BN, TM, TN, KC>;
        if (cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
                cudaSuccess)
            return false;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s.blocks_per_sm, k1, (BM / TM) * (BN / TN), smem) !=
                cudaSuccess ||
            s.blocks_per_sm < 1)
            return false;
        s.scratch = ptr;
        s.ready = true;
    }
    out = s;
    return true;
}

// Tiles of the pair kernel: every 128 x 128 block (kb, lb) with kb <= lb,
// row-major, except the last diagonal block when it holds one sample (no pair
// k < l there): the blocks (kb, lb) with kb * 128 < min(n, (lb + 1) * 128) - 1.
uint32_t tile_count(uint32_t n) {
    const uint32_t nb = (n + BM - 1) / BM;
    return nb * (nb + 1) / 2 - (n % BM == 1 ? 1u : 0u);
}

// One thread per block row kb writes that row's tiles at their closed-form
// offset kb * nb - kb (kb - 1) / 2; thread 0 also writes the table descriptor.
__global__ void write_tiles_kernel(uint4 *tiles, ssu::dev::TableDesc *table, uint32_t n, uint32_t nb,
                                   uint32_t n_tiles) {
    const uint32_t kb = blockIdx.x * blockDim.x + threadIdx.x;
    if (kb == 0) {
        ssu::dev::TableDesc t{};
        t.n = n;
        *table = t;
    }
    if (kb >= nb) return;
    const uint32_t first = kb * nb - kb * (kb - 1) / 2;
    for (uint32_t lb = kb; lb < nb; lb++)
        if (first + (lb - kb) < n_tiles) tiles[first + (lb - kb)] = make_uint4(kb, lb, 0, 0);
}

template <bool NORM>
int run(const DeviceSetup &ds, const double *U, const double *len, uint32_t E, uint32_t n, uint64_t ld,
        double *out, cudaStream_t stream) {
    using Op = WeightedOp<NORM>;
    const uint32_t nb = (n + BM - 1) / BM;
    const uint32_t n_tiles = tile_count(n);

    // scratch layout: [table][tiles][W][W partials][split partials], 256-byte aligned
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    unsigned char *base = static_cast<unsigned char *>(ds.scratch);
    size_t off = 0;
    ssu::dev::TableDesc *d_table = reinterpret_cast<ssu::dev::TableDesc *>(base + off);
    off = align(off + sizeof(ssu::dev::TableDesc));
    uint4 *d_tiles = reinterpret_cast<uint4 *>(base + off);
    off = align(off + sizeof(uint4) * std::max<uint32_t>(n_tiles, 1));
    double *d_W = nullptr, *d_part = nullptr;
    uint32_t n_parts = 0, chunk = kWChunk;
    if (NORM) {
        d_W = reinterpret_cast<double *>(base + off);
        off = align(off + sizeof(double) * ld);
        n_parts = std::max<uint32_t>(1, (E + chunk - 1) / chunk);
        const size_t room = off < kScratchBytes ? (kScratchBytes - off) / (sizeof(double) * ld) : 0;
        if (room == 0) {
            note("n_samples too large for the scratch array");
            return output_error;
        }
        if (n_parts > room) {  // fewer, longer chunks
            n_parts = static_cast<uint32_t>(room);
            chunk = (E + n_parts - 1) / n_parts;
            n_parts = std::max<uint32_t>(1, (E + chunk - 1) / chunk);
        }
        d_part = reinterpret_cast<double *>(base + off);
        off = align(off + sizeof(double) * ld * n_parts);
    }
    if (off > kScratchBytes) {
        note("n_samples too large for the scratch array");
        return output_error;
    }
    // split count: waves over the SMs, capped by the scratch left for partials
    const size_t per_split = sizeof(double) * static_cast<size_t>(BM) * BN * Op::NACC * n_tiles;
    const uint32_t max_fit = static_cast<uint32_t>(std::min<size_t>(64, (kScratchBytes - off) / per_split));
    const uint32_t slots = static_cast<uint32_t>(ds.n_sms * ds.blocks_per_sm);
    uint32_t splits = 1;
    double best = 1e300;
    const uint32_t max_s = std::max<uint32_t>(1, std::min<uint32_t>(max_fit, E / (8 * KC)));
    for (uint32_t s = 1; s <= max_s; s++) {
        const double cost = std::ceil(static_cast<double>(n_tiles) * s / slots) / s * (1.0 + 0.005 * (s - 1));
        if (cost < best - 1e-12) {
            best = cost;
            splits = s;
        }
    }
    uint32_t rows = E ? (E + splits - 1) / splits : 0;
    rows = ((rows + KC - 1) / KC) * KC;
    splits = rows ? (E + rows - 1) / rows : 1;
    if (splits == 0) splits = 1;
    double *d_split = splits > 1 ? reinterpret_cast<double *>(base + off) : nullptr;

    // the tile list and the table descriptor are written on the device: the
    // call reads no host memory after it returns
    write_tiles_kernel<<<(nb + 127) / 128, 128, 0, stream>>>(d_tiles, d_table, n, nb, n_tiles);
    if (NORM) {
        dim3 grid(static_cast<uint32_t>((ld + 255) / 256), n_parts);
        ssu::dev::weighted_sums_partial_kernel<double><<<grid, 256, 0, stream>>>(U, len, E, ld, chunk, d_part,
                                                                                nullptr, 0);
        ssu::dev::reduce_partials_kernel<double><<<static_cast<uint32_t>((ld + 255) / 256), 256, 0, stream>>>(
            d_part, n_parts, ld, d_W);
    }
    ssu::dev::PairArgs<double> a{};
    a.tiles = d_tiles;
    a.n_tiles = n_tiles;
    a.n_splits = splits;
    a.tables = d_table;
    a.U = U;
    a.len = len;
    a.W = d_W;
    a.E = E;
    a.ld = ld;
    a.rows_per_split = splits > 1 ? rows : E;
    a.out = ssu::dev::OutSpec{0, out, 0, 0};
    a.partial = d_split;
    const size_t smem = ssu::dev::pair_values_smem<double, Op, BM, BN, KC>();
    if (n_tiles) {
        const uint64_t work = static_cast<uint64_t>(n_tiles) * splits;
        const uint32_t ctas =
            static_cast<uint32_t>(std::min<uint64_t>(work, static_cast<uint64_t>(ds.n_sms) * ds.blocks_per_sm));
        ssu::dev::pair_values_kernel<double, Op, BM, BN, TM, TN, KC>
            <<<ctas, (BM / TM) * (BN / TN), smem, stream>>>(a);
        if (splits > 1)
            ssu::dev::split_finalize_kernel<double, Op, BM, BN, TM, TN>
                <<<n_tiles, (BM / TM) * (BN / TN), 0, stream>>>(a, splits);
    }
    ssu::dev::zero_diagonal_kernel<<<dim3((n + 255) / 256, 1), 256, 0, stream>>>(out, d_table, 1);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        note(cudaGetErrorString(e));
        return output_error;
    }
    return okay;
}

}  // namespace

extern "C" ComputeStatus ssu_b200_weighted_pairs_noalloc(const double *d_embedding, const double *d_lengths,
                                                         uint32_t n_embedded, uint32_t n_samples, uint64_t ld,
                                                         int normalized, double *d_out, void *stream) {
    if (n_samples == 0) return table_empty;
    if (n_samples > kMaxSamples) {
        note("n_samples exceeds the limit of this entry point (100000)");
        return output_error;
    }
    if (ld < n_samples || ld % 128 != 0) {
        note("ld must be a multiple of 128 and at least n_samples");
        return output_error;
    }
    if (!d_embedding || !d_lengths || !d_out) {
        note("null device pointer");
        return output_error;
    }
    // the pair kernel stages embedding rows with 16-byte copies and reads
    // lengths and writes the matrix as doubles
    if (reinterpret_cast<uintptr_t>(d_embedding) % 16 != 0 || reinterpret_cast<uintptr_t>(d_lengths) % 8 != 0 ||
        reinterpret_cast<uintptr_t>(d_out) % 8 != 0) {
        note("d_embedding must be 16-byte aligned, d_lengths and d_out 8-byte aligned");
        return output_error;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return output_error;
    DeviceSetup ds;
    if (!setup_device(dev, ds)) {
        note("device set-up failed");
        return output_error;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int rc = normalized ? run<true>(ds, d_embedding, d_lengths, n_embedded, n_samples, ld, d_out, s)
                              : run<false>(ds, d_embedding, d_lengths, n_embedded, n_samples, ld, d_out, s);
    return static_cast<ComputeStatus>(rc);
}
