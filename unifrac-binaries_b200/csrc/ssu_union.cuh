// Generalized and variance-adjusted UniFrac over a sparse embedding (sm_100a).
//
// A node adds nothing to a pair where neither sample has it: the VAW weight
// mi (m - mi) is 0 there (mi = counts of both samples), and so is the
// generalized u + v.  Per node, only the pairs with the row sample present
// (row pass: every column of the tile) or only the column sample present
// (column pass: the rows without it) are evaluated, each with the method's
// own term - no rearrangement, so the result matches the dense form up to
// the order of the summation (no cancellation, nothing to recompute).
//
// Tile: 64 (k) x 64 (l) pairs; 16 consumer warps and a producer warpgroup
// (one thread issues the copies; the group hands most of its registers to
// the consumers through setmaxnreg, so accumulators and terms stay in
// registers).  The embedded rows stream through in order, 32 consecutive
// rows per stage: one 2-D TMA box (32 rows x 64 columns) per block (k, l)
// and per array (proportions; counts for VAW) and one copy of the 32 branch
// lengths - five copies a stage, not one per row - into a ring of
// mbarrier-guarded stages (no multicast).  Each consumer warp waits only
// for the stage it reads, so a warp with little work runs ahead.  Which
// staged rows hold a tile row or column comes from the embedding's presence
// words (one 64-bit word per row and 64 columns; lane n holds staged row
// n's words of both blocks), read a stage ahead.  Row
// pass: warp w owns rows 4w .. 4w + 3 (lanes over the 64 columns); column
// pass: warp w owns columns 4w .. 4w + 3 (lanes over the 64 rows); both in
// registers, one owner per element (deterministic sums); the two parts meet
// in shared memory for the epilogue.  A staged row with more than 40 of the
// tile's 128 samples present is evaluated for every pair of the warp's rows
// instead (eight independent terms per thread, no item search).  Every mbarrier wait is bounded: on
// expiry the block records an error, stops, and lets its copies land.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "ssu_kernels.cuh"

namespace ssu {
namespace dev {

template <typename T>
struct UnionArgs {
    const uint4 *tiles;  // 64 x 64 tiles: x block of k, y block of l, z table
    uint32_t n_tiles, n_splits;
    const TableDesc *tables;
    const T *tot;        // per-column totals (variance adjusted)
    const T *len;        // per embedded row, zero-padded to a multiple of URS rows and one stage more
    const unsigned long long *masks;  // presence words: [ld / 64][E], bit c of word (w, e): U[e][64 w + c] > 0
    uint32_t E;
    uint64_t ld;
    double alpha;
    double *partial;     // per (split, tile) 2 x 64 x 64 fp64; nullptr: no splits
    OutSpec out;
    int *error;          // first error code of any block
    long long wait_cycles;
    int stall;           // test switch: the producer issues nothing, so every
                         // consumer wait runs out (off in normal use)
};

enum : int { UNION_ERR_FULL_WAIT = 11, UNION_ERR_EMPTY_WAIT = 12, UNION_ERR_DRAIN_WAIT = 13 };
constexpr long long kDrainCycles = 2000000000LL;  // about one second at B200 clocks

constexpr int UT = 64;                    // tile: 64 (k) x 64 (l)
constexpr int UCW = 16;                   // consumer warps (four warpgroups)
constexpr int UCT = 32 * UCW;             // consumer threads
constexpr int UTHREADS = UCT + 128;       // + the producer warpgroup (one thread copies)
// Register split (setmaxnreg): the block launches with 96 per thread
// (65,536 / 640, rounded down to a multiple of 8); the producer warpgroup
// hands back all but 32 and the consumer warpgroups take them, 112 each.
constexpr int UREG_LAUNCH = 96;
constexpr int UREG_PRODUCER = 32;
constexpr int UREG_CONSUMER = 112;
static_assert(UREG_CONSUMER * UCT + UREG_PRODUCER * 128 <= UREG_LAUNCH * UTHREADS,
              "the warpgroups' register shares exceed the block's launch registers");
static_assert(UREG_LAUNCH * UTHREADS <= 65536 && UREG_CONSUMER % 8 == 0 && UREG_PRODUCER % 8 == 0,
              "setmaxnreg counts are multiples of 8 within the register file");
constexpr int UR = UT / UCW;              // rows (row pass) / columns (column pass) per warp
// embedded rows per ring stage (the box height): one per lane.  Measured on
// the 64 uneven tables (five methods, one step): 32 rows 8.59 s, 16 rows
// 9.28 s, 8 rows 11.07 s, 4 rows 15.27 s (per-stage waits, copy issue and
// presence words outweigh the finer balance of short stages)
constexpr int URS = 32;
// A staged row with more than this many of the tile's 128 samples present
// (about 31%) is evaluated for every pair of the warp's rows: past it the
// item path issues more term slots (about 16 p per lane at presence p,
// masked lanes included) than the eight of the all-pairs path.
constexpr int UDENSE_BITS = 40;
constexpr int UFIN_THREADS = 256;

// one staged box: URS rows x 64 columns, densely packed
template <typename T>
__host__ __device__ constexpr size_t union_box_bytes() {
    return sizeof(T) * URS * UT;
}
// one ring stage: boxes (k then l block; proportions, then counts for VAW)
// and the 16 lengths, padded so every stage starts on 128 bytes
template <typename T, bool CNT>
__host__ __device__ constexpr size_t union_stage_bytes() {
    return (union_box_bytes<T>() * (CNT ? 4 : 2) + sizeof(T) * URS + 127) / 128 * 128;
}
// bytes a stage's copies deliver (the mbarrier's transaction count)
template <typename T, bool CNT>
__host__ __device__ constexpr uint32_t union_stage_tx() {
    return static_cast<uint32_t>(union_box_bytes<T>() * (CNT ? 4 : 2) + sizeof(T) * URS);
}
template <typename T, bool CNT>
__host__ __device__ constexpr int union_stages() {
    return 204800 / union_stage_bytes<T, CNT>() < 16 ? static_cast<int>(204800 / union_stage_bytes<T, CNT>()) : 16;
}
// the epilogue's shared tiles, laid over the ring once it has drained
constexpr size_t kUnionTileBytes = 2 * sizeof(double) * UT * UT;
template <typename T, bool CNT>
__host__ __device__ constexpr size_t union_ring_bytes() {
    return union_stages<T, CNT>() * union_stage_bytes<T, CNT>() > kUnionTileBytes
               ? union_stages<T, CNT>() * union_stage_bytes<T, CNT>()
               : kUnionTileBytes;
}
template <typename T, bool CNT>
__host__ __device__ constexpr size_t union_smem() {
    return union_ring_bytes<T, CNT>() + sizeof(double) * 2 * UT + sizeof(uint64_t) * 2 * union_stages<T, CNT>() + 16;
}

// Layout checks for every instance: whole 128-byte stages (each TMA box
// lands 128-aligned), a transaction count within the mbarrier's range, and
// the block's shared memory within the 227 KB a CTA may have.
template <typename T, bool CNT>
constexpr bool union_layout_ok() {
    return union_stage_bytes<T, CNT>() % 128 == 0 && union_box_bytes<T>() % 128 == 0 &&
           union_stage_tx<T, CNT>() <= union_stage_bytes<T, CNT>() && union_stage_tx<T, CNT>() < (1u << 20) &&
           union_smem<T, CNT>() <= 227u * 1024u && union_stages<T, CNT>() >= 2;
}
static_assert(union_layout_ok<double, true>() && union_layout_ok<double, false>() &&
                  union_layout_ok<float, true>() && union_layout_ok<float, false>(),
              "union kernel shared-memory layout");

__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void union_fail(int *abort_flag, int *error, int code) {
    atomicExch(abort_flag, 1);
    if (error) atomicCAS(error, 0, code);
}

__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(UCT) : "memory"); }

template <int N>
__device__ __forceinline__ void regs_release() {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(N));
}
template <int N>
__device__ __forceinline__ void regs_take() {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(N));
}

// The scalar type an operator computes its terms in.
template <class Op> struct op_real;
template <typename R, int AK> struct op_real<OpGeneralized<R, AK>> { using type = R; };
template <typename R, int AK> struct op_real<OpVawGeneralized<R, AK>> { using type = R; };
template <typename R, bool N> struct op_real<OpVawWeighted<R, N>> { using type = R; };
template <typename R, bool N> struct op_real<OpVawUnweighted<R, N>> { using type = R; };

// Whether staged rows dense in a tile take the all-pairs path: not for the
// general-alpha operators, whose eight unrolled pow evaluations outgrow the
// instruction cache (measured 1.5x slower); their dense rows stay on the
// item path.
template <class Op> struct op_dense_rows { static constexpr bool value = true; };
template <typename R> struct op_dense_rows<OpGeneralized<R, 0>> { static constexpr bool value = false; };
template <typename R> struct op_dense_rows<OpVawGeneralized<R, 0>> { static constexpr bool value = false; };

// One term of the method added to fp64 sums: fp64 operators accumulate
// directly; fp32 operators (fp32 plans, as the reference fp32 build's terms)
// compute the term in single precision and add it in fp64.
template <class Op>
__device__ __forceinline__ void union_term(double *acc, double a, double b, double ca, double cb, double m, double L,
                                           double alpha) {
    using R = typename op_real<Op>::type;
    if constexpr (sizeof(R) == 8) {
        Op::term(acc, a, b, ca, cb, m, L, alpha);
    } else {
        R t[2] = {R(0), R(0)};
        Op::term(t, static_cast<R>(a), static_cast<R>(b), static_cast<R>(ca), static_cast<R>(cb), static_cast<R>(m),
                 static_cast<R>(L), static_cast<R>(alpha));
        acc[0] += static_cast<double>(t[0]);
        if (Op::NACC > 1) acc[1] += static_cast<double>(t[1]);
    }
}

// The distance from the fp64 sums: num / den for the two-sum operators, num
// for the one-sum (unnormalized variance-adjusted) ones.
template <typename T, class Op>
__device__ __forceinline__ void union_emit(const TableDesc &td, OutSpec o, uint32_t kc, uint32_t lc, double num,
                                           double den) {
    const uint32_t k = kc - td.base, l = lc - td.base;
    if (!(k < l && l < td.n)) return;
    emit_pair<T>(o, td.n, k, l, static_cast<T>(Op::NACC > 1 ? num / den : num));
}

// Op: the method's operator, in the plan's precision (its term).  tmU / tmC:
// 2-D maps over the group's proportions / counts ([E rows][ld columns], box
// 16 x 64; rows past E read as zero).
template <typename T, class Op>
__global__ void __launch_bounds__(UTHREADS, 1)
    pair_union_kernel(const __grid_constant__ CUtensorMap tmU, const __grid_constant__ CUtensorMap tmC,
                      const UnionArgs<T> a) {
    constexpr bool CNT = Op::COUNTS;
    constexpr int NS = union_stages<T, CNT>();
    constexpr size_t SB = union_stage_bytes<T, CNT>();
    constexpr size_t BOX = union_box_bytes<T>();
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *ring = smem;
    double *Ts = reinterpret_cast<double *>(smem + union_ring_bytes<T, CNT>());  // [2UT] k then l totals
    uint64_t *full = reinterpret_cast<uint64_t *>(Ts + 2 * UT);
    uint64_t *empty = full + NS;
    int *abort_flag = reinterpret_cast<int *>(empty + NS);
    // after the ring has drained
    double *Mn = reinterpret_cast<double *>(smem);  // [64][64] numerator
    double *Md = Mn + UT * UT;                      // [64][64] denominator

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long budget = a.wait_cycles;
    if (tid == 0) {
        for (int s = 0; s < NS; s++) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, UCW);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    volatile int *vabort = abort_flag;

    // rows of a split: a multiple of the stage height
    const uint32_t sr = ((a.E + a.n_splits - 1) / a.n_splits + URS - 1) / URS * URS;
    const uint32_t n_work = a.n_tiles * a.n_splits;
    // Each role runs its own loop over the work items; per item both take
    // the same two block barriers (ring drained; shared tiles free again).
    uint32_t g = 0;  // stages used so far (same count in every warp)
    if (warp >= UCW) {
        regs_release<UREG_PRODUCER>();
        for (uint32_t w = blockIdx.x; w < n_work; w += gridDim.x) {
            const uint32_t split = w / a.n_tiles, ti = w - split * a.n_tiles;
            const uint32_t r_begin = min(a.E, split * sr), r_end = min(a.E, r_begin + sr);
            const uint32_t n_chunks = (r_end - r_begin + URS - 1) / URS;
            if (tid == UCT) {
                // ---- producer: five copies per stage
                const uint4 tile = a.tiles[ti];
                const int k0 = static_cast<int>(tile.x * UT), l0 = static_cast<int>(tile.y * UT);
                uint32_t issued = 0;
                for (uint32_t c = 0; c < (a.stall ? 0u : n_chunks); c++) {
                    const uint32_t gc = g + c, st = gc % NS, use = gc / NS;
                    if (*vabort) break;
                    if (use > 0 && !mbar_wait(empty + st, (use - 1) & 1, budget)) {
                        union_fail(abort_flag, a.error, UNION_ERR_EMPTY_WAIT);
                        break;
                    }
                    const int e0 = static_cast<int>(r_begin + c * URS);
                    unsigned char *sp = ring + st * SB;
                    mbar_expect_tx(full + st, union_stage_tx<T, CNT>());
                    tma_load_2d(sp, &tmU, full + st, k0, e0);
                    tma_load_2d(sp + BOX, &tmU, full + st, l0, e0);
                    if (CNT) {
                        tma_load_2d(sp + 2 * BOX, &tmC, full + st, k0, e0);
                        tma_load_2d(sp + 3 * BOX, &tmC, full + st, l0, e0);
                    }
                    bulk_load(sp + (CNT ? 4 : 2) * BOX, a.len + e0, URS * sizeof(T), full + st);
                    issued = c + 1;
                }
                // never leave with copies in flight: each stage's last fill lands
                // (at least about a second per wait, whatever the wait budget)
                const long long drain_budget = budget > kDrainCycles ? budget : kDrainCycles;
                for (uint32_t c = issued > static_cast<uint32_t>(NS) ? issued - NS : 0; c < issued; c++)
                    if (!mbar_wait(full + (g + c) % NS, ((g + c) / NS) & 1, drain_budget))
                        union_fail(abort_flag, a.error, UNION_ERR_DRAIN_WAIT);
            }
            g += n_chunks;
            __syncthreads();  // the ring has drained (every stage's copies landed and were read)
            const bool failed = *vabort != 0;
            __syncthreads();  // the consumers' epilogue is done with the shared tiles
            if (failed) break;
        }
        return;
    }

    regs_take<UREG_CONSUMER>();
    for (uint32_t w = blockIdx.x; w < n_work; w += gridDim.x) {
        const uint32_t split = w / a.n_tiles, ti = w - split * a.n_tiles;
        const uint4 tile = a.tiles[ti];
        const uint32_t k0 = tile.x * UT, l0 = tile.y * UT;
        const uint32_t r_begin = min(a.E, split * sr), r_end = min(a.E, r_begin + sr);
        const uint32_t n_chunks = (r_end - r_begin + URS - 1) / URS;
        if (CNT)
            for (int c = tid; c < 2 * UT; c += UCT)
                Ts[c] = static_cast<double>(a.tot[c < UT ? k0 + c : l0 + (c - UT)]);
        consumer_sync();

        // row pass: rows r0 + rr x columns lane + 32 j; column pass: rows
        // lane + 32 j x columns c0 + cc
        double A[UR][2][2], B[UR][2][2];
#pragma unroll
        for (int i = 0; i < UR; i++)
#pragma unroll
            for (int j = 0; j < 2; j++) A[i][j][0] = A[i][j][1] = B[i][j][0] = B[i][j][1] = 0.0;
        {
            const int r0 = UR * warp, c0 = UR * warp;
            const double tk0 = CNT ? Ts[lane] : 0.0, tk1 = CNT ? Ts[lane + 32] : 0.0;
            const double tl0 = CNT ? Ts[UT + lane] : 0.0, tl1 = CNT ? Ts[UT + lane + 32] : 0.0;
            // presence words of a stage: lane n the k and l blocks' words of staged row n
            auto words_of = [&](uint32_t c, unsigned long long &wk, unsigned long long &wl) {
                const uint32_t e = r_begin + c * URS + static_cast<uint32_t>(lane);
                const bool ok = c < n_chunks && lane < URS && e < r_end;
                wk = ok ? a.masks[(k0 / 64) * static_cast<uint64_t>(a.E) + e] : 0ull;
                wl = ok ? a.masks[(l0 / 64) * static_cast<uint64_t>(a.E) + e] : 0ull;
            };
            unsigned long long wk_next, wl_next;
            words_of(0, wk_next, wl_next);
            for (uint32_t c = 0; c < n_chunks; c++) {
                const unsigned long long wk = wk_next, wl = wl_next;
                words_of(c + 1, wk_next, wl_next);  // in flight while this stage is evaluated
                const uint32_t gc = g + c, st = gc % NS, use = gc / NS;
                int ok = *vabort ? 0 : 1;
                if (ok && !mbar_wait(full + st, use & 1, budget)) ok = 0;
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0 && !*vabort) union_fail(abort_flag, a.error, UNION_ERR_FULL_WAIT);
                    break;
                }
                const T *vk = reinterpret_cast<const T *>(ring + st * SB);  // [URS][64] k block
                const T *vl = vk + URS * UT;                                // [URS][64] l block
                const T *ck = vl + URS * UT;                                // counts (VAW)
                const T *cl = ck + URS * UT;
                const T *ls = vk + URS * UT * (CNT ? 4 : 2);                // [URS] lengths
                // bit n: staged row n has row r0 + rr (row pass) / column
                // c0 + cc (column pass)
                // staged rows dense in this tile (more than UDENSE_BITS of its
                // 128 samples present): every pair of the warp's rows, below
                uint32_t dm = 0;
                if constexpr (op_dense_rows<Op>::value) {
                    const int both = __popcll(wk) + __popcll(wl);
                    dm = __ballot_sync(0xffffffffu, both > UDENSE_BITS);
                }
                uint32_t rm[UR], cm[UR];
#pragma unroll
                for (int q = 0; q < UR; q++) {
                    rm[q] = __ballot_sync(0xffffffffu, (wk >> (r0 + q)) & 1ull) & ~dm;
                    cm[q] = __ballot_sync(0xffffffffu, (wl >> (c0 + q)) & 1ull) & ~dm;
                }
                // dense staged rows: rows r0 .. r0 + 3 x columns lane, lane +
                // 32, each pair's term (a pair with neither sample adds
                // nothing); eight independent terms per row
                for (uint32_t nd = op_dense_rows<Op>::value ? dm : 0u; nd;) {
                    const int n = __ffs(nd) - 1;
                    nd &= nd - 1;
                    const double L = static_cast<double>(ls[n]);
                    double bv[2], cb[2];
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        bv[j] = static_cast<double>(vl[n * UT + lane + 32 * j]);
                        cb[j] = CNT ? static_cast<double>(cl[n * UT + lane + 32 * j]) : 0.0;
                    }
#pragma unroll
                    for (int rr = 0; rr < UR; rr++) {
                        const double av = static_cast<double>(vk[n * UT + r0 + rr]);
                        const double ca = CNT ? static_cast<double>(ck[n * UT + r0 + rr]) : 0.0;
                        const double tk = CNT ? Ts[r0 + rr] : 0.0;
                        union_term<Op>(A[rr][0], av, bv[0], ca, cb[0], tk + tl0, L, a.alpha);
                        union_term<Op>(A[rr][1], av, bv[1], ca, cb[1], tk + tl1, L, a.alpha);
                    }
                }
#pragma unroll
                for (int rr = 0; rr < UR; rr++) {
                    uint32_t nm = rm[rr];
                    if (!nm) continue;
                    const int r = r0 + rr;
                    const double tk = CNT ? Ts[r] : 0.0;
                    while (nm) {
                        const int n = __ffs(nm) - 1;
                        nm &= nm - 1;
                        const T *v = vl + n * UT;
                        const T *cv = cl + n * UT;
                        const double L = static_cast<double>(ls[n]);
                        const double av = static_cast<double>(vk[n * UT + r]);
                        const double ca = CNT ? static_cast<double>(ck[n * UT + r]) : 0.0;
                        union_term<Op>(A[rr][0], av, static_cast<double>(v[lane]), ca,
                                       CNT ? static_cast<double>(cv[lane]) : 0.0, tk + tl0, L, a.alpha);
                        union_term<Op>(A[rr][1], av, static_cast<double>(v[lane + 32]), ca,
                                       CNT ? static_cast<double>(cv[lane + 32]) : 0.0, tk + tl1, L, a.alpha);
                    }
                }
#pragma unroll
                for (int cc = 0; cc < UR; cc++) {
                    uint32_t nm = cm[cc];
                    if (!nm) continue;
                    const int col = c0 + cc;
                    const double tl = CNT ? Ts[UT + col] : 0.0;
                    while (nm) {
                        const int n = __ffs(nm) - 1;
                        nm &= nm - 1;
                        const T *v = vk + n * UT;
                        const double L = static_cast<double>(ls[n]);
                        const double bv = static_cast<double>(vl[n * UT + col]);
                        const double cb = CNT ? static_cast<double>(cl[n * UT + col]) : 0.0;
                        if (v[lane] == T(0)) union_term<Op>(B[cc][0], 0.0, bv, 0.0, cb, tk0 + tl, L, a.alpha);
                        if (v[lane + 32] == T(0)) union_term<Op>(B[cc][1], 0.0, bv, 0.0, cb, tk1 + tl, L, a.alpha);
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(empty + st);
            }
        }
        g += n_chunks;
        __syncthreads();  // the ring has drained (every stage's copies landed and were read)
        const bool failed = *vabort != 0;

        if (!failed) {
            const int r0 = UR * warp, c0 = UR * warp;
#pragma unroll
            for (int rr = 0; rr < UR; rr++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    Mn[(r0 + rr) * UT + lane + 32 * j] = A[rr][j][0];
                    Md[(r0 + rr) * UT + lane + 32 * j] = A[rr][j][1];
                }
            consumer_sync();
#pragma unroll
            for (int cc = 0; cc < UR; cc++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    Mn[(lane + 32 * j) * UT + c0 + cc] += B[cc][j][0];
                    Md[(lane + 32 * j) * UT + c0 + cc] += B[cc][j][1];
                }
            consumer_sync();
            if (a.partial) {
                double *dst = a.partial + (static_cast<uint64_t>(split) * a.n_tiles + ti) * 2 * UT * UT;
                for (int e = tid; e < 2 * UT * UT; e += UCT) dst[e] = Mn[e];
            } else {
                const TableDesc td = a.tables[tile.z];
                OutSpec o = a.out;
                if (o.mode == 0) o.ptr = static_cast<T *>(o.ptr) + td.out_off;
                for (int e = tid; e < UT * UT; e += UCT)
                    union_emit<T, Op>(td, o, k0 + e / UT, l0 + e % UT, Mn[e], Md[e]);
            }
        }
        __syncthreads();  // the shared tiles lie over the next item's ring
        if (failed) break;
    }
}

// Split partials of each tile summed in split order, then the epilogue.
template <typename T, class Op>
__global__ void __launch_bounds__(UFIN_THREADS) union_finalize_kernel(const UnionArgs<T> a) {
    const uint32_t ti = blockIdx.x;
    const uint4 tile = a.tiles[ti];
    const TableDesc td = a.tables[tile.z];
    OutSpec o = a.out;
    if (o.mode == 0) o.ptr = static_cast<T *>(o.ptr) + td.out_off;
    for (int e = threadIdx.x; e < UT * UT; e += UFIN_THREADS) {
        double num = 0.0, den = 0.0;
        for (uint32_t s = 0; s < a.n_splits; s++) {
            const double *src = a.partial + (static_cast<uint64_t>(s) * a.n_tiles + ti) * 2 * UT * UT;
            num += src[e];
            den += src[UT * UT + e];
        }
        union_emit<T, Op>(td, o, tile.x * UT + e / UT, tile.y * UT + e % UT, num, den);
    }
}

// Method dispatch (ssu_union.cu): shared-memory limit of the method's
// instance, and the launch of its kernel (+ the split finalize).
template <typename T>
cudaError_t union_configure(const MethodSpec &spec, size_t *smem);
template <typename T>
cudaError_t union_launch(const MethodSpec &spec, const CUtensorMap &tmU, const CUtensorMap &tmC,
                         const UnionArgs<T> &a, uint32_t ctas, cudaStream_t s);

}  // namespace dev
}  // namespace ssu
