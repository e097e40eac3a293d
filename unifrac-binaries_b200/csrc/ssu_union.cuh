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
// (one warp issues the copies; the group hands most of its registers to the
// consumers through setmaxnreg, so accumulators and terms stay in
// registers).  Sparse rows: the producer streams the tile's k and l blocks
// of 16 rows at a time (1D bulk copies, no multicast) into a ring of
// mbarrier-guarded stages; each consumer warp waits only for the stage it
// reads, so a warp with little work runs ahead instead of idling at a block
// barrier.  Row pass: warp w owns rows 4w .. 4w + 3 (lanes over the 64
// columns); column pass: warp w owns columns 4w .. 4w + 3 (lanes over the 64
// rows); both in registers, one owner per element (deterministic sums).
// Dense rows (non-zero in more than ld / div columns) then run a
// register-tiled loop, and the three parts meet in shared memory.  Every
// mbarrier wait is bounded: on expiry the block records an error, stops, and
// lets its copies land.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ssu_kernels.cuh"

namespace ssu {
namespace dev {

template <typename T>
struct UnionArgs {
    const uint4 *tiles;  // 64 x 64 tiles: x block of k, y block of l, z table
    uint32_t n_tiles, n_splits;
    const TableDesc *tables;
    const T *U, *C;      // proportions, raw counts (variance adjusted)
    const T *tot;        // per-column totals (variance adjusted)
    const T *len;        // per embedded row
    const T *slen;       // per sparse row (in sparse-row order, padded by 16)
    uint32_t E;
    uint64_t ld;
    const uint32_t *dense_rows, *sparse_rows;
    const uint32_t *n_rows;  // {dense, sparse}
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
constexpr int UTHREADS = UCT + 128;       // + the producer warpgroup (one warp copies)
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
constexpr int URS = 16;                   // sparse rows per ring stage
constexpr int UKC = 8;                    // dense rows per dense stage
constexpr int UDS = 3;                    // dense stages
constexpr int UFIN_THREADS = 256;

// staged sparse row: k block, l block, 16 bytes of padding (bank spread)
template <typename T>
__host__ __device__ constexpr int union_pitch() {
    return 2 * UT + 16 / static_cast<int>(sizeof(T));
}
// one ring stage: values, counts (variance adjusted), lengths
template <typename T, bool CNT>
__host__ __device__ constexpr size_t union_stage_bytes() {
    return sizeof(T) * (static_cast<size_t>(URS) * union_pitch<T>() * (CNT ? 2 : 1) + URS);
}
template <typename T, bool CNT>
__host__ __device__ constexpr int union_stages() {
    return 204800 / union_stage_bytes<T, CNT>() < 16 ? static_cast<int>(204800 / union_stage_bytes<T, CNT>()) : 16;
}
// shared tiles and dense staging, laid over the ring once it has drained
template <typename T, bool CNT>
__host__ __device__ constexpr size_t union_dense_bytes() {
    return 2 * sizeof(double) * UT * UT + UDS * (sizeof(T) * UKC * 2 * UT * (CNT ? 2 : 1) + sizeof(T) * UKC);
}
template <typename T, bool CNT>
__host__ __device__ constexpr size_t union_ring_bytes() {
    return union_stages<T, CNT>() * union_stage_bytes<T, CNT>() > union_dense_bytes<T, CNT>()
               ? union_stages<T, CNT>() * union_stage_bytes<T, CNT>()
               : (union_dense_bytes<T, CNT>() + 15) / 16 * 16;
}
template <typename T, bool CNT>
__host__ __device__ constexpr size_t union_smem() {
    return union_ring_bytes<T, CNT>() + sizeof(double) * 2 * UT + sizeof(uint64_t) * 2 * union_stages<T, CNT>() + 16;
}

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

// Op: the method's operator, in the plan's precision (its term).
template <typename T, class Op>
__global__ void __launch_bounds__(UTHREADS, 1) pair_union_kernel(const UnionArgs<T> a) {
    constexpr bool CNT = Op::COUNTS;
    constexpr int P = union_pitch<T>();
    constexpr int NS = union_stages<T, CNT>();
    constexpr size_t SB = union_stage_bytes<T, CNT>();
    constexpr int VEC = 16 / sizeof(T);
    constexpr int CPR = 2 * UT / VEC;  // 16-byte pieces per dense staged row
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *ring = smem;
    double *Ts = reinterpret_cast<double *>(smem + union_ring_bytes<T, CNT>());  // [2UT] k then l totals
    uint64_t *full = reinterpret_cast<uint64_t *>(Ts + 2 * UT);
    uint64_t *empty = full + NS;
    int *abort_flag = reinterpret_cast<int *>(empty + NS);
    // after the ring has drained
    double *Mn = reinterpret_cast<double *>(smem);  // [64][64] numerator
    double *Md = Mn + UT * UT;                      // [64][64] denominator
    T *Dv = reinterpret_cast<T *>(Md + UT * UT);    // [UDS][UKC][2UT] dense values
    T *Dc = Dv + UDS * UKC * 2 * UT;                // [UDS][UKC][2UT] dense counts
    T *Dl = Dc + (CNT ? UDS * UKC * 2 * UT : 0);    // [UDS][UKC]

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

    const uint32_t n_dense = a.n_rows[0], n_sparse = a.n_rows[1];
    // sparse rows of a split: a multiple of the stage height, so every stage
    // starts on a 16-row boundary (aligned length copies)
    const uint32_t sr = ((n_sparse + a.n_splits - 1) / a.n_splits + URS - 1) / URS * URS;
    const uint32_t n_work = a.n_tiles * a.n_splits;
    // Each role runs its own loop over the work items; per item both take
    // the same two block barriers (ring drained; shared tiles free again).
    uint32_t g = 0;  // stages used so far (same count in every warp)
    if (warp >= UCW) {
        regs_release<UREG_PRODUCER>();
        for (uint32_t w = blockIdx.x; w < n_work; w += gridDim.x) {
            const uint32_t split = w / a.n_tiles, ti = w - split * a.n_tiles;
            const uint32_t s_begin = min(n_sparse, split * sr), s_end = min(n_sparse, s_begin + sr);
            const uint32_t n_chunks = (s_end - s_begin + URS - 1) / URS;
            if (warp == UCW) {
                const uint4 tile = a.tiles[ti];
                const uint32_t k0 = tile.x * UT, l0 = tile.y * UT;
                // ---- producer: lane r < 16 copies row r of each stage, lane 16
                // the stage's lengths; row ids fetched two stages ahead
                auto id_of = [&](uint32_t c) -> uint32_t {
                    const uint32_t i = s_begin + c * URS + static_cast<uint32_t>(lane);
                    return (lane < URS && c < n_chunks && i < s_end) ? a.sparse_rows[i] : 0u;
                };
                uint32_t e1 = id_of(0), e2 = id_of(1);
                uint32_t issued = 0;
                for (uint32_t c = 0; c < (a.stall ? 0u : n_chunks); c++) {
                    const uint32_t e = e1;
                    e1 = e2;
                    e2 = id_of(c + 2);
                    const uint32_t gc = g + c, st = gc % NS, use = gc / NS;
                    int ok = 1;
                    if (lane == 0) {
                        if (*vabort) {
                            ok = 0;
                        } else if (use > 0 && !mbar_wait(empty + st, (use - 1) & 1, budget)) {
                            union_fail(abort_flag, a.error, UNION_ERR_EMPTY_WAIT);
                            ok = 0;
                        }
                    }
                    if (!__shfl_sync(0xffffffffu, ok, 0)) break;
                    const uint32_t i0 = s_begin + c * URS;
                    const uint32_t nv = min(static_cast<uint32_t>(URS), s_end - i0);
                    unsigned char *sp = ring + st * SB;
                    if (lane == 0)
                        mbar_expect_tx(full + st, static_cast<uint32_t>(nv * 2 * UT * sizeof(T) * (CNT ? 2 : 1) +
                                                                        URS * sizeof(T)));
                    __syncwarp();
                    if (static_cast<uint32_t>(lane) < nv) {
                        const uint64_t base = static_cast<uint64_t>(e) * a.ld;
                        T *dv = reinterpret_cast<T *>(sp) + lane * P;
                        bulk_load(dv, a.U + base + k0, UT * sizeof(T), full + st);
                        bulk_load(dv + UT, a.U + base + l0, UT * sizeof(T), full + st);
                        if (CNT) {
                            T *dc = reinterpret_cast<T *>(sp) + URS * P + lane * P;
                            bulk_load(dc, a.C + base + k0, UT * sizeof(T), full + st);
                            bulk_load(dc + UT, a.C + base + l0, UT * sizeof(T), full + st);
                        }
                    } else if (lane == URS) {
                        T *dl = reinterpret_cast<T *>(sp) + URS * P * (CNT ? 2 : 1);
                        bulk_load(dl, a.slen + i0, URS * sizeof(T), full + st);
                    }
                    issued = c + 1;
                }
                // never leave with copies in flight: each stage's last fill lands
                // (at least about a second per wait, whatever the wait budget)
                const long long drain_budget = budget > kDrainCycles ? budget : kDrainCycles;
                if (lane == 0)
                    for (uint32_t c = issued > static_cast<uint32_t>(NS) ? issued - NS : 0; c < issued; c++)
                        if (!mbar_wait(full + (g + c) % NS, ((g + c) / NS) & 1, drain_budget))
                            union_fail(abort_flag, a.error, UNION_ERR_DRAIN_WAIT);
                __syncwarp();
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
        const uint32_t s_begin = min(n_sparse, split * sr), s_end = min(n_sparse, s_begin + sr);
        const uint32_t n_chunks = (s_end - s_begin + URS - 1) / URS;
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
            // ---- consumers
            const int r0 = UR * warp, c0 = UR * warp;
            const int hn = lane & 15, hq = lane >> 4;
            const double tk0 = CNT ? Ts[lane] : 0.0, tk1 = CNT ? Ts[lane + 32] : 0.0;
            const double tl0 = CNT ? Ts[UT + lane] : 0.0, tl1 = CNT ? Ts[UT + lane + 32] : 0.0;
            for (uint32_t c = 0; c < n_chunks; c++) {
                const uint32_t gc = g + c, st = gc % NS, use = gc / NS;
                int ok = *vabort ? 0 : 1;
                if (ok && !mbar_wait(full + st, use & 1, budget)) ok = 0;
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0 && !*vabort) union_fail(abort_flag, a.error, UNION_ERR_FULL_WAIT);
                    break;
                }
                const T *vs = reinterpret_cast<const T *>(ring + st * SB);
                const T *cs = vs + URS * P;
                const T *ls = vs + URS * P * (CNT ? 2 : 1);
                const uint32_t nv = min(static_cast<uint32_t>(URS), s_end - (s_begin + c * URS));
                const uint32_t nvm = (1u << nv) - 1u;
                // bit n of half-word h: staged row n has row r0 + 2q + h
                // (row pass) / column c0 + 2q + h (column pass)
                uint32_t rm[UR / 2], cm[UR / 2];
#pragma unroll
                for (int q = 0; q < UR / 2; q++) {
                    rm[q] = __ballot_sync(0xffffffffu, vs[hn * P + r0 + 2 * q + hq] > T(0));
                    cm[q] = __ballot_sync(0xffffffffu, vs[hn * P + UT + c0 + 2 * q + hq] > T(0));
                }
#pragma unroll
                for (int rr = 0; rr < UR; rr++) {
                    uint32_t nm = (rm[rr / 2] >> (16 * (rr % 2))) & nvm;
                    if (!nm) continue;
                    const int r = r0 + rr;
                    const double tk = CNT ? Ts[r] : 0.0;
                    while (nm) {
                        const int n = __ffs(nm) - 1;
                        nm &= nm - 1;
                        const T *v = vs + n * P;
                        const T *cv = cs + n * P;
                        const double L = static_cast<double>(ls[n]);
                        const double av = static_cast<double>(v[r]);
                        const double ca = CNT ? static_cast<double>(cv[r]) : 0.0;
                        union_term<Op>(A[rr][0], av, static_cast<double>(v[UT + lane]), ca,
                                 CNT ? static_cast<double>(cv[UT + lane]) : 0.0, tk + tl0, L, a.alpha);
                        union_term<Op>(A[rr][1], av, static_cast<double>(v[UT + lane + 32]), ca,
                                 CNT ? static_cast<double>(cv[UT + lane + 32]) : 0.0, tk + tl1, L, a.alpha);
                    }
                }
#pragma unroll
                for (int cc = 0; cc < UR; cc++) {
                    uint32_t nm = (cm[cc / 2] >> (16 * (cc % 2))) & nvm;
                    if (!nm) continue;
                    const int col = UT + c0 + cc;
                    const double tl = CNT ? Ts[col] : 0.0;
                    while (nm) {
                        const int n = __ffs(nm) - 1;
                        nm &= nm - 1;
                        const T *v = vs + n * P;
                        const double L = static_cast<double>(ls[n]);
                        const double bv = static_cast<double>(v[col]);
                        const double cb = CNT ? static_cast<double>(cs[n * P + col]) : 0.0;
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
            const int ctid = tid;
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

            // ---- dense rows: 4 (k) x 2 (l) pairs per thread in registers
            constexpr int TM = 4, TN = 2;
            const int ty = ctid / 32, tx = ctid % 32;
            const uint32_t dr = (n_dense + a.n_splits - 1) / a.n_splits;
            const uint32_t d_begin = min(n_dense, split * dr), d_end = min(n_dense, d_begin + dr);
            const uint32_t n_dchunks = d_end > d_begin ? (d_end - d_begin + UKC - 1) / UKC : 0;
            if (n_dchunks > 0) {
                double acc[TM][TN][2];
#pragma unroll
                for (int i = 0; i < TM; i++)
#pragma unroll
                    for (int j = 0; j < TN; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
                double tkd[TM], tld[TN];
#pragma unroll
                for (int i = 0; i < TM; i++) tkd[i] = CNT ? Ts[tile_row<UT, TM>(ty, i)] : 0.0;
#pragma unroll
                for (int j = 0; j < TN; j++) tld[j] = CNT ? Ts[UT + tx + 32 * j] : 0.0;
                // warp r < UKC stages row r of a chunk
                auto ok_of = [&](uint32_t chunk) {
                    return warp < UKC && chunk < n_dchunks && d_begin + chunk * UKC + warp < d_end;
                };
                auto load_row = [&](int sd, uint32_t chunk) {
                    if (warp >= UKC) return;
                    const bool ok = ok_of(chunk);
                    const uint32_t e = ok ? a.dense_rows[d_begin + chunk * UKC + warp] : 0u;
                    const uint64_t base = static_cast<uint64_t>(e) * a.ld;
                    T *dv = Dv + (sd * UKC + warp) * 2 * UT;
                    T *dc = Dc + (sd * UKC + warp) * 2 * UT;
                    for (int q = lane; q < CPR; q += 32) {
                        const uint32_t col = q < UT / VEC ? k0 + q * VEC : l0 + (q - UT / VEC) * VEC;
                        cp_async16(dv + q * VEC, a.U + base + col, ok ? 16 : 0);
                        if (CNT) cp_async16(dc + q * VEC, a.C + base + col, ok ? 16 : 0);
                    }
                    if (lane == 0)
                        cp_async_small<sizeof(T)>(Dl + sd * UKC + warp, a.len + e, ok ? (int)sizeof(T) : 0);
                };
                for (uint32_t c = 0; c + 1 < UDS; c++) {
                    if (c < n_dchunks) load_row(static_cast<int>(c), c);
                    cp_async_commit();
                }
                for (uint32_t ch = 0; ch < n_dchunks; ch++) {
                    const uint32_t nxt = ch + UDS - 1;
                    if (nxt < n_dchunks) load_row(static_cast<int>(nxt % UDS), nxt);
                    cp_async_commit();
                    cp_async_wait<UDS - 1>();
                    consumer_sync();
                    const int sd = static_cast<int>(ch % UDS);
                    const T *vs = Dv + sd * UKC * 2 * UT;
                    const T *cs = Dc + sd * UKC * 2 * UT;
                    for (int c = 0; c < UKC; c++) {
                        T av[TM], ac[TM];
                        load_half<T, TM / 2>(av, vs + c * 2 * UT + ty * (TM / 2));
                        load_half<T, TM / 2>(av + TM / 2, vs + c * 2 * UT + UT / 2 + ty * (TM / 2));
                        if (CNT) {
                            load_half<T, TM / 2>(ac, cs + c * 2 * UT + ty * (TM / 2));
                            load_half<T, TM / 2>(ac + TM / 2, cs + c * 2 * UT + UT / 2 + ty * (TM / 2));
                        }
                        const double L = static_cast<double>(Dl[sd * UKC + c]);
#pragma unroll
                        for (int j = 0; j < TN; j++) {
                            const double bv = static_cast<double>(vs[c * 2 * UT + UT + tx + 32 * j]);
                            const double bc = CNT ? static_cast<double>(cs[c * 2 * UT + UT + tx + 32 * j]) : 0.0;
#pragma unroll
                            for (int i = 0; i < TM; i++)
                                union_term<Op>(acc[i][j], static_cast<double>(av[i]), bv,
                                         CNT ? static_cast<double>(ac[i]) : 0.0, bc, tkd[i] + tld[j], L, a.alpha);
                        }
                    }
                    consumer_sync();
                }
                cp_async_wait<0>();
                consumer_sync();  // the column pass's additions are complete
#pragma unroll
                for (int i = 0; i < TM; i++)
#pragma unroll
                    for (int j = 0; j < TN; j++) {
                        const int at = tile_row<UT, TM>(ty, i) * UT + tx + 32 * j;
                        Mn[at] += acc[i][j][0];
                        Md[at] += acc[i][j][1];
                    }
            }
            consumer_sync();

            if (a.partial) {
                double *dst = a.partial + (static_cast<uint64_t>(split) * a.n_tiles + ti) * 2 * UT * UT;
                for (int e = ctid; e < 2 * UT * UT; e += UCT) dst[e] = Mn[e];
            } else {
                const TableDesc td = a.tables[tile.z];
                OutSpec o = a.out;
                if (o.mode == 0) o.ptr = static_cast<T *>(o.ptr) + td.out_off;
                for (int e = ctid; e < UT * UT; e += UCT)
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

// Per sparse row (in order) its branch length, so a ring stage can copy the
// lengths of its 16 rows in one piece.
template <typename T>
__global__ void gather_sparse_len_kernel(const uint32_t *__restrict__ sparse_rows, const uint32_t *__restrict__ n_rows,
                                         const T *__restrict__ len, uint32_t E, T *__restrict__ slen) {
    const uint32_t n = n_rows[1];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < E; i += gridDim.x * blockDim.x)
        slen[i] = i < n ? len[sparse_rows[i]] : T(0);
}

// Method dispatch (ssu_union.cu): shared-memory limit of the method's
// instance, and the launch of its kernel (+ the split finalize).
template <typename T>
cudaError_t union_configure(const MethodSpec &spec, size_t *smem);
template <typename T>
cudaError_t union_launch(const MethodSpec &spec, const UnionArgs<T> &a, uint32_t ctas, cudaStream_t s);

}  // namespace dev
}  // namespace ssu
