// Unweighted UniFrac as a tensor-core contraction on sm_100a (tcgen05).
//
// For presence X (samples x embedded nodes, 0/1) and branch lengths L:
//   G[k][l] = sum_n X[k][n] L[n] (1 - X[l][n])  (length in k and not in l)
//   r[k]    = sum_n X[k][n] L[n]                 (fp64)
//   xor sum  num = G[k][l] + G[l][k]
//   or  sum  den = r[k] + G[l][k]
//   unweighted d = num / den, unnormalized d = num
// which are the xor / or sums of the reference's unweighted tasks
// (src/unifrac_task_impl.hpp:1193-1278).  Every term is positive: unlike
// r_k + r_l - 2 X L X^T, nothing cancels when two samples share most of
// their length, so the relative error does not grow for close samples.
//
// Operands (fp16, K-major, built by `presence_rows_kernel`): A = X, and
// B_hi / B_lo = (1 - X) * (L 2^s_c) split into two fp16 terms (hi = fp16(x),
// lo = fp16(x - hi)), nodes sorted by decreasing length and scaled per
// 256-node chunk c by a power of two 2^s_c.  Each chunk is accumulated in
// fp32 in tensor memory (TMEM), then promoted to fp64 registers scaled back
// by 2^-s_c.  The contraction covers every ordered tile (kb, lb) and stores G
// in fp64; `finish_unweighted_kernel` forms num and den from G and its
// transpose.
//
// CTA: one 128 x 128 tile of G.  Warp 0 issues TMA loads (A, B_hi,
// B_lo: 128 rows x 64 nodes each, 128-byte swizzle) into a 4-stage ring;
// warp 1 (one thread) issues tcgen05.mma (M=128, N=128, K=16, two per K-step:
// hi and lo into the same accumulator) into one of two TMEM accumulators;
// warps 2..9 drain a finished accumulator (tcgen05.ld) into fp64 while the
// next chunk accumulates in the other.  Every mbarrier wait is bounded: on
// expiry the CTA records an error code, stops issuing, waits (bounded) for its
// own TMA copies and MMAs, frees its TMEM and returns.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "ssu_kernels.cuh"

namespace ssu {
namespace tc {

constexpr int BLOCK_M = 128;
constexpr int BLOCK_N = 128;
constexpr int BLOCK_K = 64;  // fp16 nodes per stage row: one 128-byte swizzle atom
constexpr int UMMA_K = 16;
constexpr int STAGES = 4;
constexpr int CHUNK_KB = 4;  // K blocks per fp64 promotion (256 nodes)
constexpr int TMEM_COLS = 2 * BLOCK_N;
constexpr int EPI_WARPS = 8;
constexpr int THREADS = 32 * (2 + EPI_WARPS);
constexpr uint32_t TILE_BYTES = BLOCK_M * BLOCK_K * 2;
constexpr uint32_t STAGE_BYTES = 3 * TILE_BYTES;
constexpr size_t SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;

enum : int { ERR_NONE = 0, ERR_FULL_WAIT = 1, ERR_EMPTY_WAIT = 2, ERR_ACC_FULL_WAIT = 3, ERR_ACC_EMPTY_WAIT = 4,
             ERR_DONE_WAIT = 5, ERR_DRAIN_WAIT = 6 };

// G block of one table: table t's rows are operand rows [base, base + ldg)
// and its G is ldg x ldg (row major) at G + g_off.
struct GemmTable {
    uint64_t g_off;
    uint32_t ldg;   // the table's samples rounded up to BLOCK_M
    uint32_t base;  // first operand row of the table
};

struct GemmArgs {
    const uint4 *tiles;   // x = row block of k, y = row block of l, z = table
    uint32_t n_tiles;
    const GemmTable *tables;
    uint32_t n_kblocks;   // padded nodes / BLOCK_K, a multiple of CHUNK_KB
    const double *chunk_scale;  // 2^-s_c per chunk
    double *G;
    int *error;           // first error code of any CTA
    long long wait_cycles;  // budget of one mbarrier wait
};

using dev::mbar_arrive;
using dev::mbar_expect_tx;
using dev::mbar_init;
using dev::mbar_try_wait;
using dev::mbar_wait;
using dev::smem_u32;

using dev::tma_load_2d;

// K-major operand tile in shared memory with 128-byte swizzle: rows of 128
// bytes, 8-row groups 1024 bytes apart (SBO), LBO unused (1), descriptor
// version 1, layout type 2 (SWIZZLE_128B).  The tile base is 1024-aligned.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);
    d |= static_cast<uint64_t>(1) << 16;
    d |= static_cast<uint64_t>(1024 >> 4) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    d |= static_cast<uint64_t>(2) << 61;
    return d;
}

// Instruction descriptor, kind::f16: D f32, A and B f16, both K-major, M x N.
__host__ __device__ constexpr uint32_t f16_idesc(int m, int n) {
    return (1u << 4) | (0u << 7) | (0u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void fail(int *shared_abort, int *global_err, int code) {
    atomicExch(shared_abort, 1);
    atomicCAS(global_err, ERR_NONE, code);
}

__global__ void __launch_bounds__(THREADS, 1)
    unweighted_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmBh,
                         const __grid_constant__ CUtensorMap tmBl, const GemmArgs args) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *accf = empty + STAGES;
    uint64_t *acce = accf + 2;
    uint64_t *done = acce + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint4 tile = args.tiles[blockIdx.x];
    const int m0 = static_cast<int>(tile.x) * BLOCK_M, n0 = static_cast<int>(tile.y) * BLOCK_N;
    const GemmTable gt = args.tables[tile.z];
    const uint32_t nkb = args.n_kblocks;
    const uint32_t nchunks = nkb / CHUNK_KB;
    const long long budget = args.wait_cycles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(accf + b, 1);
            mbar_init(acce + b, EPI_WARPS);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(tmem_slot);
    volatile int *vabort = abort_flag;

    if (warp == 0) {
        if (lane == 0) {
            // TMA producer
            uint32_t issued = 0;
            for (uint32_t kb = 0; kb < nkb; kb++) {
                const uint32_t s = kb % STAGES, use = kb / STAGES;
                if (*vabort) break;
                if (use > 0 && !mbar_wait(empty + s, (use - 1) & 1, budget)) {
                    fail(abort_flag, args.error, ERR_EMPTY_WAIT);
                    break;
                }
                uint8_t *st = smem + s * STAGE_BYTES;
                mbar_expect_tx(full + s, STAGE_BYTES);
                tma_load_2d(st, &tmA, full + s, static_cast<int>(kb) * BLOCK_K, m0);
                tma_load_2d(st + TILE_BYTES, &tmBh, full + s, static_cast<int>(kb) * BLOCK_K, n0);
                tma_load_2d(st + 2 * TILE_BYTES, &tmBl, full + s, static_cast<int>(kb) * BLOCK_K, n0);
                issued = kb + 1;
            }
            // never leave with copies in flight: each stage's last load must land
            for (uint32_t kb = issued > STAGES ? issued - STAGES : 0; kb < issued; kb++) {
                if (!mbar_wait(full + kb % STAGES, (kb / STAGES) & 1, budget))
                    fail(abort_flag, args.error, ERR_DRAIN_WAIT);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer
            constexpr uint32_t idesc = f16_idesc(BLOCK_M, BLOCK_N);
            for (uint32_t c = 0; c < nchunks && !*vabort; c++) {
                const uint32_t buf = c & 1, reuse = c >> 1;
                if (reuse > 0 && !mbar_wait(acce + buf, (reuse - 1) & 1, budget)) {
                    fail(abort_flag, args.error, ERR_ACC_EMPTY_WAIT);
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + buf * BLOCK_N;
                bool ok = true;
                for (uint32_t kk = 0; kk < CHUNK_KB; kk++) {
                    const uint32_t kb = c * CHUNK_KB + kk;
                    const uint32_t s = kb % STAGES, use = kb / STAGES;
                    if (!mbar_wait(full + s, use & 1, budget)) {
                        fail(abort_flag, args.error, ERR_FULL_WAIT);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = smem_u32(smem + s * STAGE_BYTES);
                    const uint64_t a0 = sw128_desc(st);
                    const uint64_t h0 = sw128_desc(st + TILE_BYTES);
                    const uint64_t l0 = sw128_desc(st + 2 * TILE_BYTES);
#pragma unroll
                    for (int ks = 0; ks < BLOCK_K / UMMA_K; ks++) {
                        // advance 16 fp16 = 32 bytes along K inside the swizzle atom
                        const uint64_t koff = static_cast<uint64_t>((ks * UMMA_K * 2) >> 4);
                        umma_f16(d, a0 + koff, h0 + koff, idesc, (kk | ks) != 0 ? 1u : 0u);
                        umma_f16(d, a0 + koff, l0 + koff, idesc, 1u);
                    }
                    umma_commit(empty + s);
                }
                if (!ok) break;
                umma_commit(accf + buf);
            }
            umma_commit(done);
        }
    } else {
        // epilogue: warp w reads TMEM lanes 32*(w%4).. and half (w-2)/4 of the columns
        const int q = warp & 3;
        const int half = (warp - 2) >> 2;
        const int row = q * 32 + lane;
        double acc[BLOCK_N / 2];
#pragma unroll
        for (int i = 0; i < BLOCK_N / 2; i++) acc[i] = 0.0;
        bool ok = true;
        for (uint32_t c = 0; c < nchunks; c++) {
            const uint32_t buf = c & 1, use = c >> 1;
            if (!mbar_wait(accf + buf, use & 1, budget)) {
                fail(abort_flag, args.error, ERR_ACC_FULL_WAIT);
                ok = false;
                break;
            }
            tc_fence_after();
            const double sc = args.chunk_scale[c];
            const uint32_t base = tmem + (static_cast<uint32_t>(q * 32) << 16) + buf * BLOCK_N + half * (BLOCK_N / 2);
#pragma unroll
            for (int j = 0; j < BLOCK_N / 2 / 16; j++) {
                uint32_t v[16];
                tmem_ld16(base + j * 16, v);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; i++)
                    acc[j * 16 + i] = fma(static_cast<double>(__uint_as_float(v[i])), sc, acc[j * 16 + i]);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(acce + buf);
        }
        if (ok && !*vabort) {
            double *g = args.G + gt.g_off + static_cast<uint64_t>(m0 - gt.base + row) * gt.ldg + (n0 - gt.base) +
                        half * (BLOCK_N / 2);
#pragma unroll
            for (int i = 0; i < BLOCK_N / 2; i += 2)
                *reinterpret_cast<double2 *>(g + i) = make_double2(acc[i], acc[i + 1]);
        }
    }
    __syncthreads();
    if (warp == 1) {
        // every MMA this CTA issued has completed before its TMEM is freed
        if (!mbar_wait(done, 0, budget)) fail(abort_flag, args.error, ERR_DONE_WAIT);
        tc_fence_after();
        __syncwarp();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// Presence rows for the contraction, one CTA per sample (padding rows too):
// walk up from every present tip, marking embedded ancestors in a shared
// bitmap (stopping at nodes already marked), then write the sample's rows of
// A = X and B_hi, B_lo = (1 - X) L (fp16) in full, 16 bytes per thread, and
// r = sum L of the present nodes (fp64, fixed reduction order).
__global__ void presence_rows_kernel(const uint32_t *__restrict__ sample_ptr, const int32_t *__restrict__ start_col,
                                     const int32_t *__restrict__ parent_col, const __half *__restrict__ l_hi,
                                     const __half *__restrict__ l_lo, const double *__restrict__ l_sorted,
                                     uint32_t n, uint32_t k_pad, __half *__restrict__ A, __half *__restrict__ Bh,
                                     __half *__restrict__ Bl, double *__restrict__ r) {
    extern __shared__ uint32_t bits[];  // k_pad / 32 words
    __shared__ double red[256];
    const uint32_t j = blockIdx.x;
    const uint32_t words = k_pad / 32;
    for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) bits[w] = 0u;
    __syncthreads();
    if (j < n) {
        for (uint32_t e = sample_ptr[j] + threadIdx.x; e < sample_ptr[j + 1]; e += blockDim.x) {
            int32_t c = start_col[e];
            while (c >= 0) {
                const uint32_t m = 1u << (c & 31);
                const uint32_t old = atomicOr(&bits[c >> 5], m);
                if (old & m) break;
                c = parent_col[c];
            }
        }
    }
    __syncthreads();
    const uint64_t row = static_cast<uint64_t>(j) * k_pad;
    double part = 0.0;
    for (uint32_t c8 = threadIdx.x * 8; c8 < k_pad; c8 += blockDim.x * 8) {
        const uint32_t b = (bits[c8 >> 5] >> (c8 & 31)) & 0xFFu;
        __align__(16) __half xa[8], xh[8], xl[8];
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const bool on = (b >> t) & 1u;
            xa[t] = on ? __float2half(1.0f) : __float2half(0.0f);
            xh[t] = on ? __float2half(0.0f) : l_hi[c8 + t];
            xl[t] = on ? __float2half(0.0f) : l_lo[c8 + t];
            if (on) part += l_sorted[c8 + t];
        }
        *reinterpret_cast<uint4 *>(A + row + c8) = *reinterpret_cast<const uint4 *>(xa);
        *reinterpret_cast<uint4 *>(Bh + row + c8) = *reinterpret_cast<const uint4 *>(xh);
        *reinterpret_cast<uint4 *>(Bl + row + c8) = *reinterpret_cast<const uint4 *>(xl);
    }
    red[threadIdx.x] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int t = 0; t < 256; t++) s += red[t];
        r[j] = s;
    }
}

// num = G[k][l] + G[l][k], den = r[k] + G[l][k] for k < l, then the output
// layout of the other pair kernels; grid.z = table of the group.
__global__ void finish_unweighted_kernel(const double *__restrict__ G, const GemmTable *__restrict__ gtables,
                                         const dev::TableDesc *__restrict__ tables, const double *__restrict__ r,
                                         int normalized, int out_fp64, dev::OutSpec out) {
    // 32 x 32 block of pairs per CTA; both G tiles through shared memory
    __shared__ double gt[32][33];
    const GemmTable g = gtables[blockIdx.z];
    const dev::TableDesc td = tables[blockIdx.z];
    const uint32_t n = td.n;
    const uint32_t k0 = blockIdx.y * 32, l0 = blockIdx.x * 32;
    if (k0 > l0 + 31 || k0 >= n || l0 >= n) return;
    const double *Gt = G + g.g_off;
    const uint32_t ldg = g.ldg;
    const double *rt = r + g.base;
    if (out.mode == 0) out.ptr = static_cast<char *>(out.ptr) + td.out_off * (out_fp64 ? sizeof(double) : sizeof(float));
    const uint32_t tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (uint32_t i = ty; i < 32; i += 8) {
        const uint32_t l = l0 + i, k = k0 + tx;
        gt[i][tx] = (l < n && k < n) ? Gt[static_cast<uint64_t>(l) * ldg + k] : 0.0;  // G[l][k]
    }
    __syncthreads();
    for (uint32_t i = ty; i < 32; i += 8) {
        const uint32_t k = k0 + i, l = l0 + tx;
        if (k < l && l < n) {
            const double gkl = Gt[static_cast<uint64_t>(k) * ldg + l];
            const double glk = gt[tx][i];
            const double num = gkl + glk;
            const double v = normalized ? num / (rt[k] + glk) : num;
            if (out.mode == 0 && !out_fp64)
                dev::emit_pair<float>(out, n, k, l, static_cast<float>(v));
            else
                dev::emit_pair<double>(out, n, k, l, v);
        }
    }
}

}  // namespace tc
}  // namespace ssu
