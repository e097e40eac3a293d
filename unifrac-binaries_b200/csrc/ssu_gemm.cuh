// Unweighted UniFrac as a tensor-core contraction on sm_100a (tcgen05).
//
// For presence X (samples x embedded nodes, 0/1) and branch lengths L:
//   G[k][l] = sum_n X[k][n] L[n] (1 - X[l][n])  (length in k and not in l)
//   r[k]    = sum_n X[k][n] L[n]                 (fp64)
// and for a pair k < l
//   or  sum  = r[l] + G[k][l]                    (l, plus what only k has)
//   xor sum  = 2 G[k][l] + r[l] - r[k]           (= G[k][l] + G[l][k])
//   unweighted d = xor / or, unnormalized d = xor
// which are the xor / or sums of the reference's unweighted tasks
// (src/unifrac_task_impl.hpp:1193-1278).  Only G[k][l] with k < l is
// contracted: the upper triangle of tiles.  The subtraction in the xor sum
// cannot lose relative accuracy to G's error: G[k][l] <= xor, so an error
// e * G[k][l] in G is at most 2 e of the result; r is an fp64 sum of the
// true lengths.
//
// Operands (8-bit, K-major, built by `presence_rows_kernel`).  The length of
// node n, scaled by its chunk's 2^s_c to q < 2^23, is written as
//   q = 256 u v + s t     (u, v, s, t in [0, 255]; u v, s t <= 32767)
// (every integer below 2^23 has such a form; the host picks one per node).
// Row operands A0 = X u and A1 = X s, column operands B0 = (1 - X) v and
// B1 = (1 - X) t, so that with P0 = A0 B0^T and P1 = A1 B1^T (`kind::i8`,
// unsigned, int32 accumulate: exact, a chunk holding at most 512 blocks x
// 128 nodes x 32767 < 2^31)
//   G[k][l] (chunk c) = 2^-s_c (256 P0[k][l] + P1[k][l]).
// Two products of 8-bit operands carry the 23-bit lengths: two MMAs per
// pair and node, where a 0/1 row operand against three byte planes of the
// lengths takes three.  Nodes are grouped by the binary exponent of their
// length and packed into chunks of whole 128-node K blocks of one exponent
// (zero-length padding columns close a chunk); scaled by 2^s_c every length
// of chunk c lies in [2^22, 2^23), so q = round(L 2^s_c) keeps 23
// significant bits.  Each chunk is accumulated in tensor memory (TMEM), then
// 256 P0 + P1 (exact in int64) is promoted to fp64 registers scaled back by
// 2^-s_c.  The only rounding before fp64 is the quantisation of each length
// (relative at most 2^-23).
//
// Work unit: a cluster of two CTAs (cta_group::2) owns 256 rows k x 128
// columns l of one table.  Per 32 nodes, two MMAs of M = 256 (128 rows per
// CTA) x N = 128 (64 columns of B held by each CTA), one per product, into
// TMEM columns [0, 128) and [128, 256) of one of two accumulators.  Per
// CTA: warp 0 issues its TMA loads (its 128 rows of A0 and of A1 and its 64
// rows of B0 and of B1, 128 nodes, 128-byte swizzle, no multicast) into a
// 4-stage ring whose full barriers live in CTA 0; in CTA 0 one thread of
// warp 1 issues the MMAs, and commits each stage's release and each chunk's
// completion to both CTAs; warps 2..9 of both CTAs drain a finished
// accumulator into fp64 registers while the next chunk accumulates, and
// finally form the distances and write them.  Every mbarrier wait is
// bounded: on expiry the CTA records an error code, stops issuing, lets its
// copies and MMAs finish, frees TMEM and returns.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "ssu_digits.hpp"
#include "ssu_kernels.cuh"

namespace ssu {
namespace tc {

constexpr int ROWS = 128;        // rows k per CTA (M = 256 per cluster)
constexpr int COLS = 128;        // columns l per work unit
constexpr int PRODUCTS = 2;      // operand pairs (A0, B0), (A1, B1)
constexpr int BLOCK_K = 128;     // 8-bit nodes per stage row: one 128-byte swizzle atom
constexpr int UMMA_K = 32;
constexpr int UMMA_M = 2 * ROWS;
constexpr int UMMA_N = COLS;           // per product
constexpr int B_ROWS = UMMA_N / 2;     // B rows of each product held by each CTA of the pair
constexpr int STAGES = 4;
constexpr int MAX_CHUNK_KB = 512;      // 512 x 128 x 32767 < 2^31: exact product sums
constexpr int QBITS = digits::kBits;   // fixed-point bits of the largest length of a chunk
constexpr int MAX_PART = static_cast<int>(digits::kMaxPart);  // largest u v and s t
constexpr int ACC_STRIDE = 256;        // TMEM columns between the two accumulators
constexpr int TMEM_COLS = 512;
constexpr int EPI_WARPS = 8;
constexpr int THREADS = 32 * (2 + EPI_WARPS);
constexpr uint32_t A_BYTES = ROWS * BLOCK_K;    // one product's A tile
constexpr uint32_t B_BYTES = B_ROWS * BLOCK_K;  // one product's B tile
constexpr uint32_t STAGE_BYTES = PRODUCTS * (A_BYTES + B_BYTES);  // per CTA
constexpr size_t SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
static_assert(UMMA_N % 16 == 0 && UMMA_N <= 256, "kind::i8 with M = 256 takes N in multiples of 16 up to 256");
static_assert(PRODUCTS * UMMA_N <= ACC_STRIDE && 2 * ACC_STRIDE <= TMEM_COLS,
              "two accumulators must fit the TMEM allocation");
static_assert(A_BYTES % 1024 == 0 && B_BYTES % 1024 == 0, "operand tiles must keep 1024-byte swizzle alignment");
static_assert(SMEM_BYTES <= 227 * 1024, "stage ring exceeds shared memory");
static_assert(static_cast<long long>(MAX_CHUNK_KB) * BLOCK_K * MAX_PART < (1LL << 31), "product sums must stay exact");
static_assert((static_cast<long long>(MAX_PART) << 8) + MAX_PART >= (1LL << QBITS) - 1,
              "256 u v + s t must reach the largest length");

enum : int { ERR_NONE = 0, ERR_FULL_WAIT = 1, ERR_EMPTY_WAIT = 2, ERR_ACC_FULL_WAIT = 3, ERR_ACC_EMPTY_WAIT = 4,
             ERR_DONE_WAIT = 5, ERR_DRAIN_WAIT = 6 };

struct GemmArgs {
    const uint4 *tiles;         // x = 256-row block k, y = 128-column block l, z = table
    uint32_t n_tiles;
    const dev::TableDesc *tables;
    uint32_t n_kblocks;         // padded nodes / BLOCK_K
    uint32_t plane_rows;        // operand rows of one product (A1 and B1 start there)
    uint32_t n_chunks;
    const uint32_t *chunk_end;  // first K block after chunk c
    const double *chunk_scale;  // 2^-s_c per chunk
    const double *r;            // per operand row: fp64 sum of the present lengths
    int normalized;
    int out_fp64;
    dev::OutSpec out;
    int *error;                 // first error code of any CTA
    long long wait_cycles;      // budget of one mbarrier wait
    int stall;                  // test switch: no copy is issued, so every wait runs out
};

using dev::mbar_expect_tx;
using dev::mbar_init;
using dev::smem_u32;

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

// Instruction descriptor, kind::i8: D s32, A and B unsigned 8-bit, both
// K-major, M x N (M counts both CTAs of the pair).
__host__ __device__ constexpr uint32_t i8_idesc(int m, int n) {
    return (2u << 4) | (0u << 7) | (0u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// shared::cluster address of the same shared-memory offset in CTA `rank`
__device__ __forceinline__ uint32_t map_to_rank(uint32_t saddr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
    return r;
}
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
// Bounded wait on a barrier of this CTA that other CTAs of the cluster
// arrive on (acquire at cluster scope).
__device__ __forceinline__ bool mbar_try_wait_cl(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_cl(uint64_t *bar, uint32_t parity, long long budget) {
    const uint32_t a = smem_u32(bar);
    if (mbar_try_wait_cl(a, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait_cl(a, parity))
        if (clock64() - t0 > budget) return false;
    return true;
}
// arrive on a barrier given by its shared::cluster address (any CTA of the cluster)
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cl_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cl_addr) : "memory");
}
// 2-D tiled TMA load into this CTA's shared memory completing on a barrier of
// either CTA of the pair (given by its shared::cluster address); no multicast.
__device__ __forceinline__ void tma_load_2d_pair(void *dst, const CUtensorMap *map, uint32_t bar_cl, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
        "%4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(bar_cl), "r"(x), "r"(y)
        : "memory");
}
__device__ __forceinline__ void umma_i8_pair(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}" ::"r"(
            d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0));
}
// Arrive once on the barrier at this offset in both CTAs of the pair when
// every MMA issued so far has completed.
__device__ __forceinline__ void umma_commit_pair(uint64_t *bar) {
    const uint16_t mask = 0x3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"(mask)
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

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(THREADS, 1)
    unweighted_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                         const GemmArgs args) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);  // used in CTA 0
    uint64_t *empty = full + STAGES;
    uint64_t *accf = empty + STAGES;
    uint64_t *acce = accf + 2;  // used in CTA 0: released by the epilogues of both CTAs
    uint64_t *done = acce + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

    const uint32_t rank = cluster_rank();
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint4 tile = args.tiles[blockIdx.x >> 1];
    const dev::TableDesc td = args.tables[tile.z];
    const uint32_t k0 = tile.x * UMMA_M + rank * ROWS;  // this CTA's first row, table-local
    const uint32_t l0 = tile.y * COLS;
    // this CTA's rows: 128 of A0 (A1 plane_rows further), and its half of the
    // unit's 128 columns of B0 (B1 likewise)
    const int arow = static_cast<int>(td.base + k0);
    const int brow = static_cast<int>(td.base + l0 + rank * B_ROWS);
    const int prow = static_cast<int>(args.plane_rows);
    const uint32_t nkb = args.n_kblocks, nchunks = args.n_chunks;
    const long long budget = args.wait_cycles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(accf + b, 1);
            mbar_init(acce + b, 2 * EPI_WARPS);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    // both CTAs' barriers are initialised before either signals the other
    cluster_sync();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(tmem_slot);
    volatile int *vabort = abort_flag;
    const uint32_t full0 = map_to_rank(smem_u32(full), 0);
    const uint32_t acce0 = map_to_rank(smem_u32(acce), 0);
    // once any cluster of the launch has recorded an error, the others stop
    // at once instead of each waiting out its budget
    if (threadIdx.x == 0 && *reinterpret_cast<volatile int *>(args.error) != ERR_NONE) *abort_flag = 1;
    __syncthreads();
    bool ok = true;
    uint32_t issued = 0;

    if (warp == 0) {
        if (lane == 0) {
            // TMA producer of this CTA; the pair's stage completes on CTA 0's barrier
            for (uint32_t kb = 0; kb < (args.stall ? 0u : nkb); kb++) {
                const uint32_t s = kb % STAGES, use = kb / STAGES;
                if (*vabort) break;
                if (use > 0 && !mbar_wait_cl(empty + s, (use - 1) & 1, budget)) {
                    fail(abort_flag, args.error, ERR_EMPTY_WAIT);
                    break;
                }
                uint8_t *st = smem + s * STAGE_BYTES;
                const int x = static_cast<int>(kb) * BLOCK_K;
                if (rank == 0) mbar_expect_tx(full + s, 2 * STAGE_BYTES);
                // stage layout: A0, A1, B0, B1
                tma_load_2d_pair(st, &tmA, full0 + s * 8, x, arow);
                tma_load_2d_pair(st + A_BYTES, &tmA, full0 + s * 8, x, arow + prow);
                tma_load_2d_pair(st + 2 * A_BYTES, &tmB, full0 + s * 8, x, brow);
                tma_load_2d_pair(st + 2 * A_BYTES + B_BYTES, &tmB, full0 + s * 8, x, brow + prow);
                issued = kb + 1;
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && rank == 0) {
            // MMA issuer for the pair
            constexpr uint32_t idesc = i8_idesc(UMMA_M, UMMA_N);
            uint32_t kb = 0;
            for (uint32_t c = 0; c < nchunks && !*vabort; c++) {
                const uint32_t buf = c & 1, reuse = c >> 1;
                if (reuse > 0 && !mbar_wait_cl(acce + buf, (reuse - 1) & 1, budget)) {
                    fail(abort_flag, args.error, ERR_ACC_EMPTY_WAIT);
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + buf * ACC_STRIDE;
                const uint32_t kstart = kb, kend = args.chunk_end[c];
                bool good = true;
                for (; kb < kend; kb++) {
                    const uint32_t s = kb % STAGES, use = kb / STAGES;
                    if (!mbar_wait_cl(full + s, use & 1, budget)) {
                        fail(abort_flag, args.error, ERR_FULL_WAIT);
                        good = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = smem_u32(smem + s * STAGE_BYTES);
                    const uint64_t a0 = sw128_desc(st);
                    const uint64_t a1 = sw128_desc(st + A_BYTES);
                    const uint64_t b0 = sw128_desc(st + 2 * A_BYTES);
                    const uint64_t b1 = sw128_desc(st + 2 * A_BYTES + B_BYTES);
#pragma unroll
                    for (int ks = 0; ks < BLOCK_K / UMMA_K; ks++) {
                        // advance 32 bytes along K inside the swizzle atom
                        const uint64_t koff = static_cast<uint64_t>((ks * UMMA_K) >> 4);
                        const uint32_t accum = (kb != kstart || ks != 0) ? 1u : 0u;
                        umma_i8_pair(d, a0 + koff, b0 + koff, idesc, accum);
                        umma_i8_pair(d + UMMA_N, a1 + koff, b1 + koff, idesc, accum);
                    }
                    umma_commit_pair(empty + s);
                }
                if (!good) break;
                umma_commit_pair(accf + buf);
            }
            umma_commit_pair(done);
        }
    } else {
        // epilogue: warp w reads TMEM lanes 32*(w%4).. and half (w-2)/4 of the
        // 128 columns, each column's two product sums
        const int q = warp & 3;
        const int half = (warp - 2) >> 2;
        constexpr int HC = COLS / 2;  // columns per epilogue warp
        double acc[HC];
#pragma unroll
        for (int i = 0; i < HC; i++) acc[i] = 0.0;
        for (uint32_t c = 0; c < nchunks; c++) {
            const uint32_t buf = c & 1, use = c >> 1;
            if (*vabort || !mbar_wait_cl(accf + buf, use & 1, budget)) {
                fail(abort_flag, args.error, ERR_ACC_FULL_WAIT);
                ok = false;
                break;
            }
            tc_fence_after();
            const double sc = args.chunk_scale[c];
            const uint32_t base = tmem + (static_cast<uint32_t>(q * 32) << 16) + buf * ACC_STRIDE + half * HC;
#pragma unroll
            for (int g = 0; g < HC / 16; g++) {
                // 16 columns of each product
                uint32_t v0[16], v1[16];
                tmem_ld16(base + g * 16, v0);
                tmem_ld16(base + UMMA_N + g * 16, v1);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const unsigned long long t = (static_cast<unsigned long long>(v0[i]) << 8) + v1[i];
                    acc[g * 16 + i] = fma(static_cast<double>(t), sc, acc[g * 16 + i]);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(acce0 + buf * 8);
        }
        const uint32_t n = td.n;
        const uint32_t k = k0 + q * 32 + lane;
        if (ok && !*vabort && k < n) {
            dev::OutSpec o = args.out;
            if (o.mode == 0)
                o.ptr = static_cast<char *>(o.ptr) + td.out_off * (args.out_fp64 ? sizeof(double) : sizeof(float));
            const double *rt = args.r + td.base;
            const double rk = rt[k];
            const uint32_t lb = l0 + half * HC;
            // fully unrolled: acc stays in registers
#pragma unroll
            for (int j = 0; j < HC; j++) {
                const uint32_t l = lb + j;
                if (k < l && l < n) {
                    const double rl = rt[l];
                    const double g = acc[j];
                    const double x = 2.0 * g + (rl - rk);
                    const double v = args.normalized ? x / (rl + g) : x;
                    if (o.mode == 0 && !args.out_fp64)
                        dev::emit_pair<float>(o, n, k, l, static_cast<float>(v));
                    else
                        dev::emit_pair<double>(o, n, k, l, v);
                }
            }
        }
    }
    __syncthreads();
    if (warp == 1) {
        // every MMA that writes this CTA's TMEM or reads its shared memory has completed
        if (lane == 0 && !mbar_wait_cl(done, 0, budget)) fail(abort_flag, args.error, ERR_DONE_WAIT);
        __syncwarp();
        tc_fence_after();
    }
    if (threadIdx.x == 0 && *vabort && issued > 0) {
        // after an expired wait, give copies still in flight into this CTA's
        // shared memory time to land (about 20 ms at B200 clocks) before it is released
        const long long t0 = clock64();
        while (clock64() - t0 < budget / 100) __nanosleep(1000);
    }
    __syncthreads();
    // neither CTA frees TMEM or leaves while the other may still signal it
    cluster_sync();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// Per-sample lists of starting columns, built from one table's CSR on the
// device: table row i (one warp) whose observation starts at column
// row_start[i] >= 0 gives every sample j with a positive count one entry in
// operand row base + j.  Counting pass (fill == nullptr): count[base + j]++;
// placing pass: start_col[fill[base + j]++] = row_start[i].  The order within
// a sample's list varies; the rows kernel only takes the union of the paths.
__global__ void sample_lists_kernel(const uint32_t *__restrict__ indptr, const uint32_t *__restrict__ indices,
                                    const double *__restrict__ data, const int32_t *__restrict__ row_start,
                                    uint32_t n_rows, uint32_t base, uint32_t *__restrict__ count,
                                    uint32_t *__restrict__ fill, int32_t *__restrict__ start_col) {
    const uint64_t w = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const uint32_t lane = threadIdx.x % 32;
    if (w >= n_rows) return;
    const int32_t st = row_start[w];
    if (st < 0) return;
    for (uint32_t q = indptr[w] + lane; q < indptr[w + 1]; q += 32) {
        if (!(data[q] > 0.0)) continue;
        const uint32_t col = base + indices[q];
        if (fill)
            start_col[atomicAdd(fill + col, 1u)] = st;
        else
            atomicAdd(count + col, 1u);
    }
}

// out[0] = 0, out[i + 1] = in[0] + ... + in[i] for i < n; one CTA of 1024.
__global__ void __launch_bounds__(1024) exclusive_scan_kernel(const uint32_t *__restrict__ in, uint32_t n,
                                                              uint32_t *__restrict__ out) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    const uint32_t lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    if (threadIdx.x == 0) {
        carry = 0;
        out[0] = 0;
    }
    __syncthreads();
    for (uint32_t b = 0; b < n; b += 1024) {
        const uint32_t i = b + threadIdx.x;
        uint32_t v = i < n ? in[i] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= static_cast<uint32_t>(o)) v += y;
        }
        if (lane == 31) warp_tot[warp] = v;
        __syncthreads();
        if (warp == 0) {
            uint32_t t = warp_tot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= static_cast<uint32_t>(o)) t += y;
            }
            warp_tot[lane] = t;  // inclusive over warps
        }
        __syncthreads();
        const uint32_t before = carry + (warp ? warp_tot[warp - 1] : 0u);
        if (i < n) out[i + 1] = before + v;
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_tot[31];
        __syncthreads();
    }
}

// Presence rows for the contraction, one CTA per sample (padding rows too):
// walk up from every present tip, marking embedded ancestors in a shared
// bitmap (stopping at nodes already marked), then write the sample's rows of
// A0 = X u, A1 = X s, B0 = (1 - X) v and B1 = (1 - X) t (8-bit, 16 nodes and
// 16 bytes per store; A1 and B1 `plane` bytes after A0 and B0), and
// r = sum L of the present nodes (fp64, fixed reduction order).  lq holds
// the node digits u, s, v, t: digit i at lq + i * k_pad.
__global__ void presence_rows_kernel(const uint32_t *__restrict__ sample_ptr, const int32_t *__restrict__ start_col,
                                     const int32_t *__restrict__ parent_col, const uint8_t *__restrict__ lq,
                                     const double *__restrict__ l_sorted, uint32_t n, uint32_t k_pad, uint64_t plane,
                                     uint8_t *__restrict__ A, uint8_t *__restrict__ B, double *__restrict__ r) {
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
    for (uint32_t c16 = threadIdx.x * 16; c16 < k_pad; c16 += blockDim.x * 16) {
        const uint32_t b = (bits[c16 >> 5] >> (c16 & 31)) & 0xFFFFu;
        uint32_t keep[4];  // 0xFF in the bytes of present nodes
#pragma unroll
        for (int w = 0; w < 4; w++) {
            const uint32_t nib = (b >> (4 * w)) & 0xFu;
            keep[w] = ((nib & 1u) | (((nib >> 1) & 1u) << 8) | (((nib >> 2) & 1u) << 16) |
                       (((nib >> 3) & 1u) << 24)) * 0xFFu;
        }
#pragma unroll
        for (int i = 0; i < 2 * PRODUCTS; i++) {
            const uint4 d = *reinterpret_cast<const uint4 *>(lq + static_cast<uint64_t>(i) * k_pad + c16);
            const bool row_side = i < PRODUCTS;
            uint8_t *dst = (row_side ? A : B) + static_cast<uint64_t>(i % PRODUCTS) * plane + row + c16;
            const uint32_t m0 = row_side ? keep[0] : ~keep[0], m1 = row_side ? keep[1] : ~keep[1];
            const uint32_t m2 = row_side ? keep[2] : ~keep[2], m3 = row_side ? keep[3] : ~keep[3];
            *reinterpret_cast<uint4 *>(dst) = make_uint4(d.x & m0, d.y & m1, d.z & m2, d.w & m3);
        }
#pragma unroll
        for (int t = 0; t < 16; t++)
            if ((b >> t) & 1u) part += l_sorted[c16 + t];
    }
    red[threadIdx.x] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int t = 0; t < 256; t++) s += red[t];
        r[j] = s;
    }
}

}  // namespace tc
}  // namespace ssu
