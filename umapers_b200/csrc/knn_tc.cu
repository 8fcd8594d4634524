// knn_tc.cu - exact kNN through tcgen05 tensor-core distance tiles.
//
// Replaces exact_nearest_neighbors{,_to_reference} (rust_umap/src/lib.rs:
// 2863-2928, 3346-3399) and exact_nearest_neighbors_cosine (lib.rs:2874-2889)
// for dense rows with the same result as the reference, bit for bit:
//
// 1. prep: every row becomes one FP16 operand row of K' = round_up(d + 6, 16)
//    columns.  Euclidean rows are first multiplied by a power of two s (the
//    same for every row, exact) that keeps the largest squared norm at or
//    below 2^15; cosine rows are divided by their L2 norm.  With h = fp16(row)
//    and a_i, b_j per-row terms split into three FP16 parts,
//        A = [alpha h | 1 1 1 | split3(a_i) | 0...]
//        B = [      h | split3(b_j) | 1 1 1 | 0...]
//    one GEMM gives L_ij = alpha h_i.h_j + a_i + b_j (alpha = -2, a = (1-c) n -
//    c0/2 for euclidean; alpha = -1, a = 1 - c0, b = 0 for cosine), a
//    certified LOWER bound of the reference's FP32 distance (scaled by s^2).
//    FP16 keeps 11 significant bits, so one product term h_i.h_j is within
//    2^-10 |x||y| of x.y; c and c0 also cover FP32 accumulation, the FP32
//    norms, the FP16 subnormal range and the reference's own rounding (see
//    bound_for).  By |x||y| <= (|x|^2 + |y|^2) / 2 the bound separates into a
//    row term and a column term, so it folds into the operands.
// 2. tc_knn_kernel: a persistent, warp-specialised tcgen05 kernel.  A CTA
//    keeps MT query tiles of 128 rows of A resident in shared memory, streams
//    BN-row candidate tiles of B through a TMA ring (SWIZZLE_128B, no
//    multicast), and one thread issues 128 x BN x 16 tcgen05.mma (kind::f16,
//    FP16 in, FP32 accumulate) into double-buffered TMEM accumulators.  A
//    last k-block of 16 or 32 columns is loaded as a narrow block (32- or
//    64-byte rows, SWIZZLE_32B / 64B) in the same ring stage as the block
//    before it.  One epilogue warp per (TMEM lane quarter, query tile,
//    64-column group) owns 32 rows x 64 columns of the accumulator: it reads
//    them with tcgen05.ld and keeps, per (row, 64-column group), the S = 32
//    smallest (L, index) keys in a global list.  A per-list threshold skips a
//    row's 64 columns with one vote in the common case; otherwise every
//    pending row of the warp is served at once, one per lane: the lane
//    appends its row's keys below the threshold behind the list's sorted
//    keys.  A list is merged (bitonic, one key per lane) only when its
//    appended keys would overflow, which also lowers its threshold.  When the
//    query tiles are fewer than the SMs, the candidate tiles are split too
//    (one wave of units), with lists per split.  A self kNN over at least one
//    wave of query groups first regroups its rows by nearest pivot ("cell
//    order" below), and each group starts its candidate walk at its own
//    cell, so the lists fill with near candidates first.
// 3. rerank: one warp per row recomputes exact FP32 distances in the
//    reference's summation order and keeps the k smallest (distance, index)
//    keys.  With U_j = L_j + 2 e_j and B the smallest largest-L of the full
//    lists, every candidate missing from the lists has d >= B, so the row is
//    certified when at least k candidates have U < B.  Only listed candidates
//    with L <= T, T the k-th smallest U, can rank in the top k, so only they
//    are recomputed.
// 4. Rows that fail (near-ties wider than the bound, or too few listed
//    candidates below B) run a second pass as a query set with at least two
//    candidate splits, i.e. twice as many lists per row, on operands in the
//    three-term FP16 split h.h' + h.l' + l.h' (l = fp16(x - h), K' =
//    3d + 6), whose bound is about 2^-21 of the norms; rows that still fail
//    (duplicates beyond the lists, zero cosine rows) are recomputed by
//    knn_plain.
//
// Every wait on an mbarrier is bounded by a %globaltimer deadline; a timeout
// sets an error word, stops all roles, drains in-flight copies and frees TMEM.
#include <cub/cub.cuh>
#include <cuda.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "kernels.cuh"
#include "tcgen05.cuh"

namespace umapb {
namespace {

using namespace tc;

constexpr int BM = 128;     // query rows per tile (UMMA M)
constexpr int BK = kBK;     // FP16 columns per k-block (one 128-byte swizzle row)
constexpr int UK = kUK;     // K of one tcgen05.mma kind::f16
constexpr int S = 32;       // shortlist length per list
constexpr int HC = 64;       // keys a list holds appended between merges
constexpr int LS = S + HC;  // slots per list: S sorted keys, then up to HC appended
constexpr int kMaxK = 62;   // neighbours per row on the tensor path (64-entry re-rank lists)
constexpr int kATileBytes = BM * BK * 2;  // 16 KiB: one query tile's k-block
constexpr int kBarBytes = 256;            // mbarriers, TMEM address, abort flag
constexpr int kNormCols = 6;              // 3 + 3 FP16 columns of the folded row terms
constexpr int kMaxStages = 8;
constexpr size_t kSmemLimit = 227 * 1024;

// Operand geometry for d features in `terms` product terms (1: h.h'; 3: the
// split h.h' + h.l' + l.h' with l = fp16(x - h)): K' columns used by the MMA
// (kmma), the stored row length (at least one 64-column block), k-blocks,
// and the k-steps of 16 columns issued in the last k-block.
struct Geom {
    int terms, kmma, kst, kb, tail;
};
inline Geom geom(int d, int terms = 1) {
    Geom g;
    g.terms = terms;
    g.kmma = ((terms * d + kNormCols + UK - 1) / UK) * UK;
    g.kst = std::max(g.kmma, BK);
    g.kb = (g.kmma + BK - 1) / BK;
    g.tail = (g.kmma - BK * (g.kb - 1)) / UK;
    return g;
}

// Error bound of one GEMM entry against the reference's FP32 distance, in
// the scaled units of the GEMM: e_ij = c (n_i + n_j) + c0 for euclidean (n the
// scaled FP32 squared norms), e = c0 for cosine.  Terms (u = 2^-11 the FP16
// unit roundoff, eta = 2^-25 half the FP16 subnormal spacing):
//   2u + u^2            the one-term FP16 product, |x||y| <= (n_i + n_j) / 2
//                       (3.1 * 2^-22 for the three-term split: |l| <= u|x|,
//                       |x - h - l| <= u^2 |x|)
//   2.01 K' 2^-23       FP32 accumulation of K' terms (truncating adders)
//   d 2^-24             the FP32 norms
//   2 (d + 16) 2^-24    the reference's FP32 sum and subtractions (d <= 2(n_i + n_j))
//   2 eta sqrt(d)       FP16 subnormals (absolute part in c0)
//   2^-23               the FP32 rounding of the folded row terms
// with 25% slack on the sum.
struct Bound {
    double c, c0;
};
inline Bound bound_for(int d, const Geom& g, bool cosine) {
    const double u = std::ldexp(1.0, -11), eta = std::ldexp(1.0, -25);
    const double sd = std::sqrt(static_cast<double>(d));
    const double prod = g.terms == 1 ? 2.0 * u + u * u : 3.1 * u * u;
    const double t = g.terms;  // subnormal errors enter once per product term
    Bound b;
    if (!cosine) {
        b.c = 1.25 * (prod + 2.01 * g.kmma * std::ldexp(1.0, -23) + d * std::ldexp(1.0, -24) +
                      2.0 * (d + 16) * std::ldexp(1.0, -24) + 2.0 * t * eta * sd * 1.01 +
                      std::ldexp(1.0, -23));
        b.c0 = 2.0 * (4.1 * t * eta * sd + 6.0 * eta);
    } else {
        // unit rows: |x^.y^ - cos| <= prod (1 + d 2^-23) + subnormals,
        // |cos_ref - cos| <= (2d + 16) 2^-24 (dot, norms, product, division)
        b.c = 0.0;
        b.c0 = 1.25 * (prod + 4.0 * t * eta * sd +
                       (3.0 * d + 2.01 * g.kmma + 16.0) * std::ldexp(1.0, -23)) +
               12.0 * eta;
    }
    return b;
}

// The power-of-two scale of euclidean rows: s = 2^e, s^2 = 2^(2e).
struct ScaleInfo {
    float s, s2;
};

// order-preserving map of a float to uint32 (negative values included)
__device__ __forceinline__ uint32_t f2o(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
    return (o & 0x80000000u) ? __uint_as_float(o & 0x7FFFFFFFu) : __uint_as_float(~o);
}

__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Minimum of the 64 FP32 values (bit patterns) of r[0] and r[1]: a tree of
// three-input mins, five levels deep (64 -> 22 -> 8 -> 3 -> 1).
__device__ __forceinline__ float min64(const uint32_t (&r)[2][32]) {
    float a[22];
#pragma unroll
    for (int i = 0; i < 21; ++i) {
        const int j = 3 * i;
        a[i] = min3f(__uint_as_float(r[j >> 5][j & 31]), __uint_as_float(r[(j + 1) >> 5][(j + 1) & 31]),
                     __uint_as_float(r[(j + 2) >> 5][(j + 2) & 31]));
    }
    a[21] = __uint_as_float(r[1][31]);
    float b[8];
#pragma unroll
    for (int i = 0; i < 7; ++i) b[i] = min3f(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
    b[7] = a[21];
    const float c0 = min3f(b[0], b[1], b[2]), c1 = min3f(b[3], b[4], b[5]), c2 = fminf(b[6], b[7]);
    return min3f(c0, c1, c2);
}

// Bitonic sort of one value per lane, ascending with the lane index.
template <typename T>
__device__ __forceinline__ T warp_sort_asc(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const T o = __shfl_xor_sync(0xffffffffu, v, stride);
            const bool up = (lane & size) == 0;
            const bool lower = (lane & stride) == 0;
            v = (lower == up) ? (v < o ? v : o) : (v < o ? o : v);
        }
    }
    return v;
}

// Two independent bitonic sorts (one value per lane each) stage by stage, so
// their shuffles overlap.
template <typename T>
__device__ __forceinline__ void warp_sort_asc2(T& a, T& b) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const T oa = __shfl_xor_sync(0xffffffffu, a, stride);
            const T ob = __shfl_xor_sync(0xffffffffu, b, stride);
            const bool keep_min = ((lane & size) == 0) == ((lane & stride) == 0);
            a = keep_min ? (a < oa ? a : oa) : (a < oa ? oa : a);
            b = keep_min ? (b < ob ? b : ob) : (b < ob ? ob : b);
        }
    }
}

// Merges 32 keys (one per lane, any order) into a list sorted ascending
// across the lanes and keeps the 32 smallest: sort the keys, reverse them,
// take the lane-wise minimum (a bitonic sequence holding the 32 smallest of
// both) and sort that with five compare-exchange stages.
__device__ __forceinline__ uint64_t warp_merge_keys(uint64_t list, uint64_t keys) {
    const int lane = threadIdx.x & 31;
    const uint64_t srt = warp_sort_asc<uint64_t>(keys);
    const uint64_t rev = __shfl_sync(0xffffffffu, srt, 31 - lane);
    uint64_t m = list < rev ? list : rev;
#pragma unroll
    for (int st = 16; st > 0; st >>= 1) {
        const uint64_t o = __shfl_xor_sync(0xffffffffu, m, st);
        m = (lane & st) ? (m > o ? m : o) : (m < o ? m : o);
    }
    return m;
}

// Sorts a bitonic sequence held one value per lane (five compare-exchange
// stages), ascending with the lane index.
template <typename T>
__device__ __forceinline__ T warp_bitonic_sort(T m) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int st = 16; st > 0; st >>= 1) {
        const T o = __shfl_xor_sync(0xffffffffu, m, st);
        m = (lane & st) ? (m > o ? m : o) : (m < o ? m : o);
    }
    return m;
}

// A sorted list of the 64 smallest values seen, two per lane: `lo` holds
// ranks 0-31 and `hi` ranks 32-63, each ascending across the lanes.
// Merging 32 new values (any order): the 32 smallest of lo and the chunk
// become lo; the 32 largest of those, merged with hi, give hi.
template <typename T>
__device__ __forceinline__ void warp_merge64(T& lo, T& hi, T chunk) {
    const int lane = threadIdx.x & 31;
    const T srt = warp_sort_asc<T>(chunk);
    const T rev = __shfl_sync(0xffffffffu, srt, 31 - lane);
    const T a = lo < rev ? lo : rev;
    const T b = lo < rev ? rev : lo;
    lo = warp_bitonic_sort<T>(a);
    const T rest = warp_bitonic_sort<T>(b);
    const T rrev = __shfl_sync(0xffffffffu, rest, 31 - lane);
    hi = warp_bitonic_sort<T>(hi < rrev ? hi : rrev);
}

// The value of rank r (< 64) of a lo/hi pair.
template <typename T>
__device__ __forceinline__ T rank_of(T lo, T hi, int r) {
    const T a = __shfl_sync(0xffffffffu, lo, r & 31);
    const T b = __shfl_sync(0xffffffffu, hi, r & 31);
    return r < 32 ? a : b;
}

// Held keys at or above this count are merged in one bitonic pass instead of
// key by key (about 6 sequential insertions cost as much).
constexpr int kBulkMergeMin = 6;

// A list occupies LS slots: its S smallest keys so far, sorted ascending
// (order-mapped L << 32 | index), then up to HC keys appended unsorted since
// the last merge, each below that merge's threshold and stored with L as raw
// FP32 bits (the epilogue appends without converting).
__device__ __forceinline__ uint64_t held_key(uint64_t raw) {
    return (static_cast<uint64_t>(f2o(__uint_as_float(static_cast<uint32_t>(raw >> 32)))) << 32) |
           static_cast<uint32_t>(raw);
}

// Merges the `held` appended keys (at most HC) into the sorted ones, one key
// per lane, and returns the new S-th smallest L, or +inf while the list holds
// fewer than S keys.
__device__ __forceinline__ float merge_held(uint64_t* lst, int held) {
    const int lane = threadIdx.x & 31;
    __syncwarp();  // the appended keys were stored by other lanes
    uint64_t lk = lst[lane];
    uint64_t h0 = lane < held ? held_key(lst[S + lane]) : ~0ull;
    uint64_t h1 = lane + 32 < held ? held_key(lst[S + 32 + lane]) : ~0ull;
    if (held > 32) {
        // both halves sorted at once; the 32 smallest of them (lane-wise min
        // of one and the other reversed, a bitonic sequence), sorted, then
        // merged with the list the same way
        warp_sort_asc2<uint64_t>(h0, h1);
        const uint64_t r1 = __shfl_sync(0xffffffffu, h1, 31 - lane);
        const uint64_t m = warp_bitonic_sort<uint64_t>(h0 < r1 ? h0 : r1);
        const uint64_t rm = __shfl_sync(0xffffffffu, m, 31 - lane);
        lk = warp_bitonic_sort<uint64_t>(lk < rm ? lk : rm);
    } else if (held >= kBulkMergeMin) {
        lk = warp_merge_keys(lk, h0);
    } else {
        for (int b = 0; b < held; ++b) {
            const uint64_t key = __shfl_sync(0xffffffffu, h0, b);
            const int pos = __popc(__ballot_sync(0xffffffffu, lk < key));
            const uint64_t up = __shfl_up_sync(0xffffffffu, lk, 1);
            if (lane > pos)
                lk = up;
            else if (lane == pos)
                lk = key;
        }
    }
    lst[lane] = lk;
    __syncwarp();
    const uint64_t last = __shfl_sync(0xffffffffu, lk, S - 1);
    return last == ~0ull ? INFINITY : o2f(static_cast<uint32_t>(last >> 32));
}

// Appends, for one lane's row, its values below t (columns below lim) as
// held keys at dst[h...]; returns the new count.
template <bool kAll>
__device__ __forceinline__ int append_row(const uint32_t (&r)[2][32], float t, int lim,
                                          int32_t col0, uint64_t* dst, int h) {
#pragma unroll
    for (int j = 0; j < 64; ++j) {
        if (__uint_as_float(r[j >> 5][j & 31]) < t && (kAll || j < lim)) {
            dst[h] = (static_cast<uint64_t>(r[j >> 5][j & 31]) << 32) |
                     static_cast<uint32_t>(col0 + j);
            ++h;
        }
    }
    return h;
}

// CTAs begin their candidate range at staggered tiles (16 groups, 2 tiles
// apart) so they do not all request the same tile at once.  The shortlist
// certificate does not depend on the visiting order.
constexpr int32_t kStaggerGroups = 16, kStaggerStep = 2;

struct TcArgs {
    int64_t n_q;
    int64_t n_r;
    int kb;               // k-blocks of 64 columns
    int tail;             // k-steps issued in the last k-block (1..4)
    int ntail;            // 16 or 32: the last k-block is a narrow block of that many
                          // columns, loaded with the last full one; 0: 64-column blocks only
    int st;               // stages of the candidate ring
    int64_t n_units;      // work units: (group of MT query tiles, candidate split)
    int n_split;          // candidate splits per group (1 unless query tiles are few)
    int64_t split_tiles;  // candidate tiles per split (the last split may hold fewer)
    int64_t n_ctiles;     // candidate tiles
    uint64_t* lists;      // n_q x n_split x (BN / 64) lists of LS slots of keys (L
                          // order-mapped << 32 | index), one list per (row, candidate split,
                          // 64-column group)
    const int32_t* start_tile;  // per query group, the first candidate tile to visit (rows in
                                // cell order, one split), or null for the staggered start
    int* err;
};

// Work unit u covers query group u / n_split and the candidate tiles of
// split u % n_split, visited from tile begin + rot onwards (cyclically).
// With rows in cell order a group starts at its own cell's first tile.
struct Unit {
    int32_t group, split, begin, len, rot;  // tile counts stay far below 2^31
};
__device__ __forceinline__ Unit unit_of(const TcArgs& p, int64_t u, int64_t stagger) {
    Unit r;
    r.group = static_cast<int32_t>(u / p.n_split);
    r.split = static_cast<int32_t>(u - static_cast<int64_t>(r.group) * p.n_split);
    r.begin = r.split * static_cast<int32_t>(p.split_tiles);
    r.len = static_cast<int32_t>(min(p.split_tiles, p.n_ctiles - r.begin));
    r.rot = p.start_tile != nullptr ? p.start_tile[r.group]
                                    : static_cast<int32_t>(stagger % kStaggerGroups) * kStaggerStep;
    if (r.rot >= r.len || r.rot < 0) r.rot = 0;
    return r;
}

// Candidate tile visited at step t of unit w.
__device__ __forceinline__ int32_t tile_at(int32_t t, const Unit& w) {
    const int32_t c = t + w.rot;
    return w.begin + (c >= w.len ? c - w.len : c);
}

// Kernel shapes: MT query tiles of 128 rows share each BN-row candidate tile;
// 2 TMEM buffers of MT x BN columns; one epilogue warp per (TMEM lane quarter,
// query tile, 64-column group).
// With SA (streamed A) the query tile is not resident: every ring stage
// carries the query tile's k-block beside the candidate tile's, so rows of
// any width fit shared memory at 1.5x the L2 reads of the resident form.
template <int MT, int BN>
constexpr int epi_warps() { return 4 * MT * (BN / 64); }
template <int MT, int BN>
constexpr int tc_threads() { return 64 + 32 * epi_warps<MT, BN>(); }

// The register file is split among the SM's four schedulers: with 18 warps
// two of them hold five warps, which caps a thread at 96 registers.
// The epilogue role of one warp.  Warp w reads TMEM lanes 32 * (w % 4)
// (hardware rule); the warps of each quarter split (query tile, 64-column
// group).  Units are first_unit, first_unit + unit_step, ...  False after a
// wait ran out.
template <int MT, int BN>
__device__ __forceinline__ bool tc_epilogue(const TcArgs& p, int warp, int lane,
                                            uint32_t tmem_base, uint32_t b_tfull,
                                            uint32_t b_tempty, int64_t first_unit,
                                            int64_t unit_step, int64_t stagger,
                                            volatile int* abort_flag) {
    constexpr int GPT = BN / 64;  // lists per candidate tile
    // Warp w reads TMEM lanes 32 * (w % 4) (hardware rule); the warps of
    // each quarter split (query tile, 64-column group).
    const int quarter = warp & 3;
    const int slot = (warp - 2) >> 2;
    const int mt = slot / GPT;
    const int cq = slot % GPT;
    uint64_t cg = 0;
    bool ok = true;
    for (int64_t unit = first_unit; unit < p.n_units && ok; unit += unit_step) {
        const Unit w = unit_of(p, unit, stagger);
        const int32_t row = (w.group * MT + mt) * BM + quarter * 32 + lane;
        const bool row_ok = row < p.n_q;
        const int32_t list_base = w.split * GPT + cq;  // list of (row, split, group)
        auto list_of = [&](int32_t srow) {
            return p.lists + (static_cast<int64_t>(srow) * GPT * p.n_split + list_base) * LS;
        };
        float tau = INFINITY;  // this row's list: its S-th smallest key at the last merge
        int held = 0;          // keys appended behind the sorted ones since then
        for (int32_t c = 0; c < w.len; ++c, ++cg) {
            const uint32_t buf = static_cast<uint32_t>(cg & 1);
            const uint32_t par = static_cast<uint32_t>((cg >> 1) & 1);
            if (!mbar_wait(b_tfull + 8 * buf, par, abort_flag)) {
                ok = false;
                break;
            }
            fence_after();
            const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) +
                                   buf * (MT * BN) + mt * BN + cq * 64;
            uint32_t r[2][32];
            tmem_ld32(taddr, r[0]);
            tmem_ld32(taddr + 32, r[1]);
            tmem_wait_ld();
            // the accumulator buffer can be overwritten as soon as it is in registers
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(b_tempty + 8 * buf);
            unsigned pend = __ballot_sync(0xffffffffu, row_ok && min64(r) < tau);
            if (pend == 0) continue;
            const int32_t colh = tile_at(c, w) * BN + cq * 64;
            const int32_t valid_cols = static_cast<int32_t>(p.n_r - colh);
            // Every pending row at once, one per lane: count the row's
            // values below its threshold, merge the lists whose appended
            // keys would overflow (one list at a time, across the warp),
            // then append each row's keys behind its sorted ones.
            const bool mine = (pend >> lane) & 1u;
            const bool all = valid_cols >= 64;
            float t = mine ? tau : -INFINITY;
            int cnt = 0;
#pragma unroll
            for (int j = 0; j < 64; ++j)
                cnt += (__uint_as_float(r[j >> 5][j & 31]) < t && (all || j < valid_cols))
                           ? 1
                           : 0;
            unsigned over = __ballot_sync(0xffffffffu, held + cnt > HC);
            while (over) {
                const int cur = __ffs(over) - 1;
                over &= over - 1;
                const float nt = merge_held(list_of(__shfl_sync(0xffffffffu, row, cur)),
                                            __shfl_sync(0xffffffffu, held, cur));
                if (lane == cur) {
                    tau = nt;
                    held = 0;
                }
            }
            t = mine ? tau : -INFINITY;
            uint64_t* dst = list_of(row) + S;
            held = all ? append_row<true>(r, t, 64, colh, dst, held)
                       : append_row<false>(r, t, valid_cols, colh, dst, held);
        }
        if (!ok) break;
        // every list of the unit ends sorted, with nothing held
        unsigned rest = __ballot_sync(0xffffffffu, held > 0);
        while (rest) {
            const int cur = __ffs(rest) - 1;
            rest &= rest - 1;
            merge_held(list_of(__shfl_sync(0xffffffffu, row, cur)),
                       __shfl_sync(0xffffffffu, held, cur));
        }
    }
    return ok;
}

// With a narrow last k-block (p.ntail, resident query tiles only) a tile
// takes KB - 1 ring stages; the last holds the final 64-column block and the
// narrow one (32- or 64-byte rows at the matching swizzle), so a 16-column
// tail costs 8 KiB of candidate loads per 256-row tile instead of 32.
template <int MT, int BN, bool SA>
__global__ void __launch_bounds__(tc_threads<MT, BN>(), 1)
    tc_knn_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                  const __grid_constant__ CUtensorMap tmAt,
                  const __grid_constant__ CUtensorMap tmBt, TcArgs p) {
    static_assert(MT * BN <= 256 && (BN == 128 || BN == 256), "at most 512 TMEM columns");
    constexpr int kEpiWarps = epi_warps<MT, BN>();
    constexpr int kBTileBytes = BN * BK * 2;
    constexpr int kStageB = SA ? MT * kATileBytes : 0;  // candidate tile within a stage
    constexpr uint32_t kIdesc = idesc_f16(BM, BN);
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int KB = p.kb, ST = p.st;
    const int NT = SA ? 0 : p.ntail;                  // narrow tail columns (0: none)
    const int KBM = NT ? KB - 1 : KB;                 // 64-column k-blocks (one stage each)
    const int TAIL = NT ? NT / UK : p.tail;           // k-steps of the last (or narrow) block
    const int ta_bytes = BM * NT * 2, tb_bytes = BN * NT * 2;
    const int stage_bytes = SA ? MT * kATileBytes + kBTileBytes : kBTileBytes + tb_bytes;
    const int a_bytes = SA ? 0 : MT * (KBM * kATileBytes + ta_bytes);  // resident query tiles
    const uint32_t sA = smem_u32(smem);
    const uint32_t sAt = sA + MT * KBM * kATileBytes;  // narrow blocks of the query tiles
    const uint32_t sB = sA + a_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + a_bytes + ST * stage_bytes);
    const uint32_t b_full = smem_u32(bars);
    const uint32_t b_empty = b_full + 8 * ST;
    const uint32_t b_tfull = b_empty + 8 * ST;
    const uint32_t b_tempty = b_tfull + 16;
    const uint32_t b_afull = b_tempty + 16;
    const uint32_t b_aempty = b_afull + 8;
    const uint32_t b_final = b_aempty + 8;
    uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(bars + 2 * ST + 7);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr uint32_t kTmemCols = 2 * MT * BN;  // 256 or 512: a power of two

    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(b_full + 8 * s, 1);
            mbar_init(b_empty + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(b_tfull + 8 * b, 1);
            mbar_init(b_tempty + 8 * b, kEpiWarps);
        }
        mbar_init(b_afull, 1);
        mbar_init(b_aempty, 1);
        mbar_init(b_final, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        tmem_alloc(smem_u32(tmem_holder), kTmemCols);
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem_base = *tmem_holder;

    auto fail = [&](int code) {
        *abort_flag = 1;
        atomicCAS(p.err, 0, code);
    };

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int64_t u_iter = 0;
            for (int64_t unit = blockIdx.x; unit < p.n_units && !*abort_flag;
                 unit += gridDim.x, ++u_iter) {
                const Unit w = unit_of(p, unit, blockIdx.x);
                if (!SA) {
                    if (u_iter > 0 &&
                        !mbar_wait(b_aempty, static_cast<uint32_t>((u_iter - 1) & 1), abort_flag)) {
                        fail(1);
                        break;
                    }
                    mbar_expect_tx(b_afull, a_bytes);
                    for (int mt = 0; mt < MT; ++mt) {
                        const int ya = static_cast<int>((w.group * MT + mt) * BM);
                        for (int kb = 0; kb < KBM; ++kb)
                            tma_load_2d(sA + (mt * KBM + kb) * kATileBytes, &tmA, b_afull, kb * BK,
                                        ya);
                        if (NT) tma_load_2d(sAt + mt * ta_bytes, &tmAt, b_afull, KBM * BK, ya);
                    }
                }
                bool ok = true;
                for (int32_t c = 0; c < w.len && ok; ++c) {
                    const int ty = static_cast<int>(tile_at(c, w) * BN);
                    for (int kb = 0; kb < KBM; ++kb) {
                        if (!mbar_wait(b_empty + 8 * stage, phase ^ 1, abort_flag)) {
                            fail(2);
                            ok = false;
                            break;
                        }
                        const uint32_t sbase = sB + stage * stage_bytes;
                        const bool narrow = NT && kb + 1 == KBM;
                        mbar_expect_tx(b_full + 8 * stage,
                                       SA ? stage_bytes : kBTileBytes + (narrow ? tb_bytes : 0));
                        if (SA)
                            for (int mt = 0; mt < MT; ++mt)
                                tma_load_2d(sbase + mt * kATileBytes, &tmA, b_full + 8 * stage,
                                            kb * BK, static_cast<int>((w.group * MT + mt) * BM));
                        tma_load_2d(sbase + kStageB, &tmB, b_full + 8 * stage, kb * BK, ty);
                        if (narrow)
                            tma_load_2d(sbase + kBTileBytes, &tmBt, b_full + 8 * stage, KBM * BK, ty);
                        if (++stage == ST) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                }
                if (!ok) break;
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------- MMA issuer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            uint64_t cg = 0;
            int64_t u_iter = 0;
            bool ok = true;
            for (int64_t unit = blockIdx.x; unit < p.n_units && ok; unit += gridDim.x, ++u_iter) {
                if (!SA) {
                    if (!mbar_wait(b_afull, static_cast<uint32_t>(u_iter & 1), abort_flag)) {
                        fail(3);
                        break;
                    }
                    fence_after();
                }
                const int32_t len = unit_of(p, unit, blockIdx.x).len;
                for (int32_t c = 0; c < len && ok; ++c, ++cg) {
                    const uint32_t buf = static_cast<uint32_t>(cg & 1);
                    if (!mbar_wait(b_tempty + 8 * buf, static_cast<uint32_t>(((cg >> 1) & 1) ^ 1),
                                   abort_flag)) {
                        fail(4);
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint32_t dcol = tmem_base + buf * (MT * BN);
                    for (int kb = 0; kb < KBM; ++kb) {
                        if (!mbar_wait(b_full + 8 * stage, phase, abort_flag)) {
                            fail(5);
                            ok = false;
                            break;
                        }
                        fence_after();
                        const int steps = NT || kb + 1 < KB ? BK / UK : TAIL;
                        const uint32_t sbase = sB + stage * stage_bytes;
                        const uint64_t db0 = desc_sw128(sbase + kStageB);
#pragma unroll
                        for (int ks = 0; ks < BK / UK; ++ks) {
                            if (ks < steps) {
#pragma unroll
                                for (int mt = 0; mt < MT; ++mt) {
                                    const uint64_t da =
                                        (SA ? desc_sw128(sbase + mt * kATileBytes)
                                            : desc_sw128(sA + (mt * KBM + kb) * kATileBytes)) +
                                        2 * ks;
                                    umma_bf16(dcol + mt * BN, da, db0 + 2 * ks, kIdesc,
                                              (kb | ks) != 0 ? 1u : 0u);
                                }
                            }
                        }
                        if (NT && kb + 1 == KBM) {
                            // the narrow block: rows of 2 * NT bytes, k-steps 32 bytes apart
                            const uint64_t dbt = desc_narrow(sbase + kBTileBytes, 2 * NT);
#pragma unroll
                            for (int ks = 0; ks < 2; ++ks) {
                                if (ks < TAIL) {
#pragma unroll
                                    for (int mt = 0; mt < MT; ++mt)
                                        umma_bf16(dcol + mt * BN,
                                                  desc_narrow(sAt + mt * ta_bytes, 2 * NT) + 2 * ks,
                                                  dbt + 2 * ks, kIdesc, 1u);
                                }
                            }
                        }
                        umma_commit(b_empty + 8 * stage);
                        if (++stage == ST) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                    if (ok) umma_commit(b_tfull + 8 * buf);
                }
                if (ok && !SA) umma_commit(b_aempty);
            }
            // every MMA issued by this thread has completed before TMEM is freed
            umma_commit(b_final);
            mbar_wait(b_final, 0, abort_flag);
        }
    } else {
        // --------------------------------------------------- epilogue
        if (!tc_epilogue<MT, BN>(p, warp, lane, tmem_base, b_tfull, b_tempty, blockIdx.x,
                                 gridDim.x, blockIdx.x, abort_flag))
            fail(6);
    }

    __syncthreads();
    if (*abort_flag) {
        // let copies already in flight land before the CTA's shared memory goes away
        const uint64_t t0 = global_ns();
        while (global_ns() - t0 < 2000000ull) {
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        tmem_dealloc(tmem_base, kTmemCols);
    }
}

// ------------------------------------------------------------ operands --
// Largest FP32 squared norm (non-negative floats order as unsigned ints).
__global__ void max_sq_kernel(const float* __restrict__ sq, int64_t n, unsigned* __restrict__ out) {
    float m = 0.0f;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        m = fmaxf(m, sq[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(out, __float_as_uint(m));
}

// s = 2^e with the largest e such that max_sq * s^2 <= 2^15: every scaled
// squared norm, every |2 h| and every folded row term then fits FP16
// (max 65504) with room to spare.
__global__ void scale_kernel(const unsigned* __restrict__ max_bits, ScaleInfo* __restrict__ out) {
    const float m = __uint_as_float(*max_bits);
    int e = 0;
    if (m > 0.0f && isfinite(m)) {
        int ex = 0;
        frexpf(m, &ex);  // m < 2^ex
        const int t = 15 - ex;
        e = t >= 0 ? t / 2 : -((-t + 1) / 2);
        e = max(-60, min(60, e));
    }
    out->s = ldexpf(1.0f, e);
    out->s2 = ldexpf(1.0f, 2 * e);
}

// Three FP16 parts whose sum is v within 2^-33 |v| (plus subnormal spacing).
__device__ __forceinline__ void split3(float v, __half* o) {
    const __half p1 = __float2half_rn(v);
    const float r1 = v - __half2float(p1);
    const __half p2 = __float2half_rn(r1);
    const float r2 = r1 - __half2float(p2);
    o[0] = p1;
    o[1] = p2;
    o[2] = __float2half_rn(r2);
}

// One warp per operand row: the FP16 row (scaled or unit-normalised) in one
// term ([alpha h] against [h]) or three ([alpha h | alpha h | alpha l]
// against [h | l | h]), the six folded columns, and zeros up to the stored
// width.  `sq` holds the FP32 squared norms in the reference's order
// (row_norms).
__global__ void prep_kernel(const float* __restrict__ X, const float* __restrict__ sq, int64_t n,
                            int d, int terms, int kst, const ScaleInfo* __restrict__ sc, double c,
                            double c0, bool cosine, bool is_query, __half* __restrict__ out) {
    const int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* x = X + row * d;
    __half* o = out + row * kst;
    const float n2 = sq[row];
    float mul;
    if (cosine) {
        const float nrm = __fsqrt_rn(n2);
        mul = nrm > 0.0f ? __frcp_rn(nrm) : 0.0f;
    } else {
        mul = sc->s;
    }
    const float alpha = cosine ? -1.0f : -2.0f;  // exact scalings of FP16 values
    for (int t = lane; t < d; t += 32) {
        const float v = x[t] * mul;
        const __half h = __float2half_rn(v);
        if (terms == 1) {
            o[t] = is_query ? __float2half_rn(alpha * __half2float(h)) : h;
        } else {
            const __half l = __float2half_rn(v - __half2float(h));
            if (is_query) {
                const __half ah = __float2half_rn(alpha * __half2float(h));
                o[t] = ah;
                o[d + t] = ah;
                o[2 * d + t] = __float2half_rn(alpha * __half2float(l));
            } else {
                o[t] = h;
                o[d + t] = l;
                o[2 * d + t] = h;
            }
        }
    }
    const int nc = terms * d;  // first folded column
    for (int t = nc + kNormCols + lane; t < kst; t += 32) o[t] = __float2half_rn(0.0f);
    if (lane == 0) {
        float a;
        if (cosine)
            a = is_query ? static_cast<float>(1.0 - c0) : 0.0f;
        else
            a = static_cast<float>((1.0 - c) * static_cast<double>(n2) *
                                       static_cast<double>(sc->s2) -
                                   0.5 * c0);
        const __half one = __float2half_rn(1.0f);
        __half parts[3];
        split3(a, parts);
        if (is_query) {
            o[nc] = one; o[nc + 1] = one; o[nc + 2] = one;
            o[nc + 3] = parts[0]; o[nc + 4] = parts[1]; o[nc + 5] = parts[2];
        } else {
            o[nc] = parts[0]; o[nc + 1] = parts[1]; o[nc + 2] = parts[2];
            o[nc + 3] = one; o[nc + 4] = one; o[nc + 5] = one;
        }
    }
}

// ------------------------------------------------------------ re-rank ---
// Squared euclidean distance with the reference's operations in its order
// (squared_distance, rust_umap/src/lib.rs:2445-2492: for d >= 64, eight
// strided lanes of acc + diff * diff summed in order, then the scalar tail).
__device__ __forceinline__ float sqdist_ref(const float* __restrict__ x, const float* __restrict__ y,
                                            int d) {
    if (d >= 64) {
        float lane[8];
#pragma unroll
        for (int l = 0; l < 8; ++l) lane[l] = 0.0f;
        int i = 0;
        if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0) {
            // the same operations in the same order, from 16-byte loads
            for (; i + 8 <= d; i += 8) {
                const float4 xa = *reinterpret_cast<const float4*>(x + i);
                const float4 xb = *reinterpret_cast<const float4*>(x + i + 4);
                const float4 ya = __ldg(reinterpret_cast<const float4*>(y + i));
                const float4 yb = __ldg(reinterpret_cast<const float4*>(y + i + 4));
                const float xs[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
                const float ys[8] = {ya.x, ya.y, ya.z, ya.w, yb.x, yb.y, yb.z, yb.w};
#pragma unroll
                for (int l = 0; l < 8; ++l) {
                    const float df = __fsub_rn(xs[l], ys[l]);
                    lane[l] = __fadd_rn(lane[l], __fmul_rn(df, df));
                }
            }
        }
        for (; i + 8 <= d; i += 8)
#pragma unroll
            for (int l = 0; l < 8; ++l) {
                const float df = __fsub_rn(x[i + l], y[i + l]);
                lane[l] = __fadd_rn(lane[l], __fmul_rn(df, df));
            }
        float s = lane[0];
#pragma unroll
        for (int l = 1; l < 8; ++l) s = __fadd_rn(s, lane[l]);
        for (; i < d; ++i) {
            const float df = __fsub_rn(x[i], y[i]);
            s = __fadd_rn(s, __fmul_rn(df, df));
        }
        return s;
    }
    float s = 0.0f;
    for (int i = 0; i < d; ++i) {
        const float df = __fsub_rn(x[i], y[i]);
        s = __fadd_rn(s, __fmul_rn(df, df));
    }
    return s;
}

// Dot product in the reference's order (dot_product_avx2 / _scalar,
// lib.rs:2653-2738: the same eight-lane layout as squared_distance for d >= 64).
__device__ __forceinline__ float dot_ref(const float* __restrict__ x, const float* __restrict__ y,
                                         int d) {
    if (d >= 64) {
        float lane[8];
#pragma unroll
        for (int l = 0; l < 8; ++l) lane[l] = 0.0f;
        int i = 0;
        for (; i + 8 <= d; i += 8)
#pragma unroll
            for (int l = 0; l < 8; ++l) lane[l] = __fadd_rn(lane[l], __fmul_rn(x[i + l], y[i + l]));
        float s = lane[0];
#pragma unroll
        for (int l = 1; l < 8; ++l) s = __fadd_rn(s, lane[l]);
        for (; i < d; ++i) s = __fadd_rn(s, __fmul_rn(x[i], y[i]));
        return s;
    }
    float s = 0.0f;
    for (int i = 0; i < d; ++i) s = __fadd_rn(s, __fmul_rn(x[i], y[i]));
    return s;
}

// cosine_distance_with_norms (lib.rs:2740-2765) from the dot and L2 norms.
__device__ __forceinline__ float cosine_ref(float dot, float xn, float yn) {
    if (xn == 0.0f && yn == 0.0f) return 0.0f;
    if (xn == 0.0f || yn == 0.0f) return 1.0f;
    float c = __fdiv_rn(dot, __fmul_rn(xn, yn));
    c = fminf(fmaxf(c, -1.0f), 1.0f);
    return __fsub_rn(1.0f, c);
}

struct RerankArgs {
    const float* Q;        // query rows in operand order
    const float* R;        // candidate rows in operand order
    const float* qsq;      // FP32 squared norms (reference order), operand order
    const float* rsq;
    const uint64_t* lists;
    int n_lists;
    int64_t n_q;
    int d, k;
    double c, c0;
    bool cosine;
    const ScaleInfo* sc;
    const int32_t* omap;   // query position -> output row (null: identity)
    const int32_t* rmap;   // candidate position -> original index (null: identity)
    int32_t* out_idx;
    float* out_dist;
    int* fb_count;
    int32_t* fb_rows;      // output rows that could not be certified
};

__global__ void rerank_kernel(RerankArgs a) {
    const int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= a.n_q) return;
    const int k = a.k, d = a.d;
    const int64_t orow = a.omap != nullptr ? a.omap[row] : row;
    const uint64_t* rl = a.lists + row * a.n_lists * LS;
    // The smallest bound a candidate missing from every list can have: a full
    // list left out only candidates with L >= its largest entry, a list that
    // is not full kept every candidate of its range.
    double bound = INFINITY;
    for (int h = 0; h < a.n_lists; ++h) {
        const uint64_t lk = rl[h * LS + lane];
        const bool valid = lk != ~0ull;
        float lmax = valid ? o2f(static_cast<uint32_t>(lk >> 32)) : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
        if (__popc(__ballot_sync(0xffffffffu, valid)) == S)
            bound = fmin(bound, static_cast<double>(lmax));
    }
    // Upper bounds U = L + 2e (rounded up to FP32): `below` counts the
    // candidates with U < bound (k of them certify the row), and T is the k-th
    // smallest U.  A candidate with L > T has k others with d <= U <= T < L <= d
    // ahead of it, so only candidates with L <= T can rank in the top k: each
    // list (sorted by L) contributes a prefix, usually empty.
    const double s2 = a.cosine ? 1.0 : static_cast<double>(a.sc->s2);
    const double nq = static_cast<double>(a.qsq[row]) * s2;
    int below = 0;
    // the 64 smallest U, sorted across the warp (hi stays +inf for k <= 32)
    float topu = INFINITY, topu_hi = INFINITY;
    const bool wide = k > 32;
    for (int h = 0; h < a.n_lists; ++h) {
        const uint64_t lk = rl[h * LS + lane];
        const float l0 = o2f(static_cast<uint32_t>(__shfl_sync(0xffffffffu, lk, 0) >> 32));
        double U = INFINITY;
        if (lk != ~0ull) {
            const double nc =
                a.cosine ? 0.0 : static_cast<double>(a.rsq[static_cast<uint32_t>(lk)]) * s2;
            U = static_cast<double>(o2f(static_cast<uint32_t>(lk >> 32))) +
                2.0 * (a.c * (nq + nc) + a.c0) * (1.0 + 1e-6);
        }
        below += __popc(__ballot_sync(0xffffffffu, U < bound));
        // a list whose smallest L already exceeds the k-th smallest U so far
        // cannot lower it
        if (!(l0 <= rank_of<float>(topu, topu_hi, k - 1))) continue;
        const float uc = __double2float_ru(U);
        if (wide) {
            warp_merge64<float>(topu, topu_hi, uc);
        } else {
            const float u = warp_sort_asc<float>(uc);
            const float ur = __shfl_sync(0xffffffffu, u, 31 - lane);
            topu = warp_bitonic_sort<float>(fminf(topu, ur));
        }
    }
    const float T = rank_of<float>(topu, topu_hi, k - 1);
    // Exact keys in the reference's order for the candidates with L <= T; the
    // 32 (k <= 32) or 64 smallest are kept sorted across the warp (bitonic
    // merge of each list's keys into them).
    const float* qrow = a.Q + row * d;
    const float qn = a.cosine ? __fsqrt_rn(a.qsq[row]) : 0.0f;
    uint64_t top = ~0ull, top_hi = ~0ull;
    for (int h = 0; h < a.n_lists; ++h) {
        const uint64_t lk = rl[h * LS + lane];
        const bool take = lk != ~0ull && o2f(static_cast<uint32_t>(lk >> 32)) <= T;
        if (__ballot_sync(0xffffffffu, take) == 0) continue;
        uint64_t key = ~0ull;
        if (take) {
            const uint32_t j = static_cast<uint32_t>(lk);
            const float* crow = a.R + static_cast<int64_t>(j) * d;
            const float dist = a.cosine
                                   ? cosine_ref(dot_ref(qrow, crow, d), qn, __fsqrt_rn(a.rsq[j]))
                                   : sqdist_ref(qrow, crow, d);
            key = knn_key(dist, a.rmap != nullptr ? static_cast<uint32_t>(a.rmap[j]) : j);
        }
        if (wide)
            warp_merge64<uint64_t>(top, top_hi, key);
        else
            top = warp_merge_keys(top, key);
    }
    // A zero cosine query has distance 0 to zero rows and 1 to the rest, which
    // its bound (built for unit rows) does not cover: it goes to the plain path.
    const bool failed = below < k || (a.cosine && a.qsq[row] == 0.0f);
    if (!failed) {
        for (int half = 0; half < 2; ++half) {
            const int r = half * 32 + lane;
            if (r >= k) break;
            const uint64_t key = half == 0 ? top : top_hi;
            a.out_idx[orow * k + r] = static_cast<int32_t>(key_index(key));
            const float kd = key_dist(key);
            a.out_dist[orow * k + r] = a.cosine ? kd : __fsqrt_rn(kd);
        }
    }
    if (failed && lane == 0) a.fb_rows[atomicAdd(a.fb_count, 1)] = static_cast<int32_t>(orow);
}

__global__ void gather_rows_kernel(const float* __restrict__ X, const int32_t* __restrict__ perm,
                                   int64_t n, int d, float* __restrict__ out) {
    const int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* src = X + static_cast<int64_t>(perm[row]) * d;
    float* dst = out + row * d;
    for (int t = lane; t < d; t += 32) dst[t] = src[t];
}

// --------------------------------------------------------------- host ----
// Kernel shape: MT query tiles x BN candidate rows, ring stages, and the
// width of a narrow last k-block (0: none).
struct Shape {
    int mt = 0, bn = 0, st = 0;
    bool stream = false;  // query tile streamed through the ring with the candidates
    size_t smem = 0;
    int ntail = 0;
    int lists() const { return bn / 64; }  // lists per row and candidate split
};

// The last k-block is loaded narrow when the operands span at least two
// k-blocks and it issues one or two k-steps (16 or 32 columns).
int narrow_cols(const Geom& g) { return g.kb >= 2 && g.tail <= 2 ? g.tail * UK : 0; }

size_t smem_bytes(int mt, int bn, int kb, int st, bool stream, int ntail) {
    // tiles + 1 KiB alignment slack + barriers/flags
    const int kbm = ntail ? kb - 1 : kb;
    const size_t a = stream ? 0
                            : static_cast<size_t>(mt) *
                                  (static_cast<size_t>(kbm) * kATileBytes + BM * ntail * 2);
    const size_t stage = static_cast<size_t>(bn) * BK * 2 + static_cast<size_t>(bn) * ntail * 2 +
                         (stream ? mt * kATileBytes : 0);
    return a + st * stage + 1024 + kBarBytes;
}

// One resident query tile against 256-candidate tiles (four lists per row)
// while the operands fit with at least three ring stages, else against
// 128-candidate tiles (two lists per row, eight epilogue warps); rows too
// wide for a resident tile stream it with 256-candidate tiles (64-column
// blocks only).
Shape shape_for(const Geom& g) {
    const int kb = g.kb, nt = narrow_cols(g);
    const int cand[2][2] = {{1, 256}, {1, 128}};
    for (const auto& c : cand) {
        int st = kMaxStages;
        while (st >= 2 && smem_bytes(c[0], c[1], kb, st, false, nt) > kSmemLimit) --st;
        if (st >= (c[1] == 256 ? 3 : 2))
            return Shape{c[0], c[1], st, false, smem_bytes(c[0], c[1], kb, st, false, nt), nt};
    }
    int st = kMaxStages;
    while (st >= 3 && smem_bytes(1, 256, kb, st, true, 0) > kSmemLimit) --st;
    return Shape{1, 256, st, true, smem_bytes(1, 256, kb, st, true, 0), 0};
}

// The operand maps of one side: 64-column blocks of `rows_box` rows, and the
// narrow last block when the shape uses one (else a copy of the first).
struct SideMaps {
    CUtensorMap full, tail;
};
SideMaps side_maps(const __half* X, int64_t n, const Geom& g, const Shape& sh, int rows_box) {
    SideMaps m;
    m.full = make_f16_map(X, n, g.kst, rows_box);
    m.tail = sh.ntail ? make_f16_tail_map(X, n, g.kst, sh.ntail, rows_box) : m.full;
    return m;
}

template <int MT, int BN, bool SA>
void launch_tc_t(const SideMaps& ma, const SideMaps& mb, const TcArgs& a, size_t smem,
                 cudaStream_t s) {
    auto kern = tc_knn_kernel<MT, BN, SA>;
    UMAPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
    int dev = 0, sms = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    UMAPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t grid = std::min<int64_t>(a.n_units, sms);
    kern<<<static_cast<unsigned>(grid), tc_threads<MT, BN>(), smem, s>>>(ma.full, mb.full,
                                                                          ma.tail, mb.tail, a);
    UMAPB_LAUNCH_CHECK();
}

void launch_tc(const Shape& sh, const SideMaps& ma, const SideMaps& mb, const TcArgs& a,
               cudaStream_t s) {
    if (sh.stream && sh.mt == 1 && sh.bn == 256)
        launch_tc_t<1, 256, true>(ma, mb, a, sh.smem, s);
    else if (!sh.stream && sh.mt == 1 && sh.bn == 256)
        launch_tc_t<1, 256, false>(ma, mb, a, sh.smem, s);
    else if (!sh.stream && sh.mt == 1 && sh.bn == 128)
        launch_tc_t<1, 128, false>(ma, mb, a, sh.smem, s);
    else
        invalid("tensor-core kNN: no kernel shape for these operands");
}

// Work decomposition: groups of MT query tiles; when the groups are fewer
// than the SMs the candidate tiles are split too (at least 8 per split, and
// no more units than SMs, so every unit starts at once), so small query sets
// still occupy the GPU.  `min_split` forces at least that many splits (more
// lists per row) where the candidate tiles allow.
TcArgs plan(int64_t n_q, int64_t n_r, const Geom& g, const Shape& sh, bool allow_split,
            int min_split) {
    TcArgs a{};
    a.n_q = n_q;
    a.n_r = n_r;
    a.kb = g.kb;
    a.tail = g.tail;
    a.ntail = sh.ntail;
    a.st = sh.st;
    a.n_ctiles = ceil_div(n_r, sh.bn);
    const int64_t groups = ceil_div(n_q, static_cast<int64_t>(BM) * sh.mt);
    int64_t split = 1;
    if (allow_split) {
        int dev = 0, sms = 0;
        UMAPB_CUDA(cudaGetDevice(&dev));
        UMAPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (groups < sms)
            split = std::min<int64_t>(std::max<int64_t>(sms / groups, 1),
                                      std::max<int64_t>(1, a.n_ctiles / 8));
    }
    split = std::max<int64_t>(split, std::min<int64_t>(min_split, a.n_ctiles));
    a.split_tiles = ceil_div(a.n_ctiles, split);
    a.n_split = static_cast<int>(ceil_div(a.n_ctiles, a.split_tiles));
    a.n_units = groups * a.n_split;
    return a;
}

// ------------------------------------------------------------ cell order --
// A self kNN over at least one wave of query groups runs on its rows
// regrouped by cell.
// - Every row joins the nearest of C pivot rows (rows p * (n / C)).
// - The rows are stably sorted by cell.
// - Each query group starts its candidate walk at its own cell's first tile.
// The shortlists then fill with near candidates in the first tiles. Their
// thresholds drop early, and later tiles rarely hold a qualifying key.
// The groups of one wave start within a few hundred tiles of each other, so
// they still stream the candidate operand in step through L2.
// The result does not change: the certificate does not depend on the
// visiting order, and the re-rank maps positions back to original rows.
constexpr int kMaxCells = 256;
constexpr int64_t kCellPivotFloats = 16384;  // 64 KiB of pivots in shared memory

// Cells: 32, 64, 128 or 256, as many as keep at least 2,048 rows per cell
// (512 at 32 cells) and the pivots within 64 KiB; 0 = rows stay in order.
int cell_count(int64_t n, int d) {
    int c = kMaxCells;
    while (c > 32 && (c * static_cast<int64_t>(d) > kCellPivotFloats || c * int64_t{2048} > n))
        c >>= 1;
    if (c * static_cast<int64_t>(d) > kCellPivotFloats || c * int64_t{512} > n) return 0;
    return c;
}

// One warp per row: lane l scores pivots l + 32 q (q < PPL) from shared
// memory ([d][C], conflict-free), the row's values broadcast by shuffle, and
// the warp keeps the pivot with the smallest |p|^2 - 2 x.p (lower on ties).
template <int PPL>
__global__ void __launch_bounds__(256) cell_assign_kernel(const float* __restrict__ X, int64_t n,
                                                          int d, int64_t stride,
                                                          uint8_t* __restrict__ cell,
                                                          int32_t* __restrict__ iota) {
    constexpr int C = 32 * PPL;
    extern __shared__ float piv[];
    float* pn = piv + static_cast<int64_t>(d) * C;
    for (int i = threadIdx.x; i < C * d; i += blockDim.x) {
        const int pc = i / d, t = i - pc * d;
        piv[t * C + pc] = X[static_cast<int64_t>(pc) * stride * d + t];
    }
    __syncthreads();
    for (int pc = threadIdx.x; pc < C; pc += blockDim.x) {
        float sq = 0.0f;
        for (int t = 0; t < d; ++t) sq = fmaf(piv[t * C + pc], piv[t * C + pc], sq);
        pn[pc] = sq;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; row < n;
         row += warps) {
        const float* x = X + row * d;
        float acc[PPL];
#pragma unroll
        for (int q = 0; q < PPL; ++q) acc[q] = 0.0f;
        for (int t0 = 0; t0 < d; t0 += 32) {
            const float xv = t0 + lane < d ? x[t0 + lane] : 0.0f;
            const int tn = min(32, d - t0);
            for (int j = 0; j < tn; ++j) {
                const float xj = __shfl_sync(0xffffffffu, xv, j);
                const float* pr = piv + (t0 + j) * C + lane;
#pragma unroll
                for (int q = 0; q < PPL; ++q) acc[q] = fmaf(xj, pr[32 * q], acc[q]);
            }
        }
        float best = INFINITY;
        int bi = C;
#pragma unroll
        for (int q = 0; q < PPL; ++q) {
            const float sc = pn[lane + 32 * q] - 2.0f * acc[q];
            if (sc < best) {
                best = sc;
                bi = lane + 32 * q;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob < best || (ob == best && oi < bi)) {
                best = ob;
                bi = oi;
            }
        }
        if (lane == 0) {
            cell[row] = static_cast<uint8_t>(bi < C ? bi : 0);
            iota[row] = static_cast<int32_t>(row);
        }
    }
}

// First candidate tile of each query group: the tile holding the first row
// of the cell that the group's first row belongs to (binary search in the
// sorted cell keys).
__global__ void group_start_kernel(const uint8_t* __restrict__ skey, int64_t groups,
                                   int rows_per_group, int tile_rows,
                                   int32_t* __restrict__ start_tile) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= groups) return;
    const int64_t r0 = g * rows_per_group;
    const uint8_t c = skey[r0];
    int64_t lo = 0, hi = r0;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (skey[mid] < c)
            lo = mid + 1;
        else
            hi = mid;
    }
    start_tile[g] = static_cast<int32_t>(lo / tile_rows);
}

struct CellOrder {
    DevBuf<float> rows;          // the rows in cell order
    DevBuf<int32_t> perm;        // position -> original row
    DevBuf<int32_t> start_tile;  // per query group
};

template <int PPL>
void launch_assign(const float* X, int64_t n, int d, uint8_t* cell, int32_t* iota,
                   cudaStream_t s) {
    constexpr int C = 32 * PPL;
    const size_t smem = (static_cast<size_t>(C) * d + C) * sizeof(float);
    auto kern = cell_assign_kernel<PPL>;
    UMAPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
    int dev = 0, sms = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    UMAPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 8), static_cast<int64_t>(sms) * 3);
    kern<<<static_cast<unsigned>(blocks), 256, smem, s>>>(X, n, d, n / C, cell, iota);
    UMAPB_LAUNCH_CHECK();
}

void cell_order(const float* X, int64_t n, int d, int cells, int rows_per_group, int64_t groups,
                int tile_rows, CellOrder& co, cudaStream_t s) {
    DevBuf<uint8_t> key(n, s), skey(n, s);
    DevBuf<int32_t> iota(n, s);
    co.perm.alloc(n, s);
    switch (cells) {
        case 32: launch_assign<1>(X, n, d, key.get(), iota.get(), s); break;
        case 64: launch_assign<2>(X, n, d, key.get(), iota.get(), s); break;
        case 128: launch_assign<4>(X, n, d, key.get(), iota.get(), s); break;
        default: launch_assign<8>(X, n, d, key.get(), iota.get(), s); break;
    }
    size_t tmp_bytes = 0;
    UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key.get(), skey.get(),
                                               iota.get(), co.perm.get(), static_cast<int>(n), 0,
                                               8, s));
    DevBuf<uint8_t> tmp(tmp_bytes, s);
    UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, key.get(), skey.get(),
                                               iota.get(), co.perm.get(), static_cast<int>(n), 0,
                                               8, s));
    co.start_tile.alloc(groups, s);
    group_start_kernel<<<static_cast<unsigned>(ceil_div(groups, 256)), 256, 0, s>>>(
        skey.get(), groups, rows_per_group, tile_rows, co.start_tile.get());
    UMAPB_LAUNCH_CHECK();
    co.rows.alloc(static_cast<size_t>(n) * d, s);
    gather_rows_kernel<<<static_cast<unsigned>(ceil_div(n * 32, 256)), 256, 0, s>>>(
        X, co.perm.get(), n, d, co.rows.get());
    UMAPB_LAUNCH_CHECK();
}


void launch_prep(const float* X, const float* sq, int64_t n, int d, const Geom& g,
                 const ScaleInfo* sc, const Bound& b, bool cosine, bool query, __half* out,
                 cudaStream_t s) {
    if (n == 0) return;
    prep_kernel<<<static_cast<unsigned>(ceil_div(n * 32, 256)), 256, 0, s>>>(
        X, sq, n, d, g.terms, g.kst, sc, b.c, b.c0, cosine, query, out);
    UMAPB_LAUNCH_CHECK();
}

void launch_max_sq(const float* sq, int64_t n, unsigned* out, cudaStream_t s) {
    if (n == 0) return;
    const int blocks = static_cast<int>(std::min<int64_t>(ceil_div(n, 256), 148 * 4));
    max_sq_kernel<<<blocks, 256, 0, s>>>(sq, n, out);
    UMAPB_LAUNCH_CHECK();
}

// Empties `count` lists: their S sorted slots become ~0 (the appended slots
// are only read below the count a list holds).
void clear_lists(uint64_t* lists, size_t count, cudaStream_t s) {
    if (count == 0) return;
    UMAPB_CUDA(cudaMemset2DAsync(lists, LS * sizeof(uint64_t), 0xFF, S * sizeof(uint64_t), count,
                                 s));
}

void launch_rerank(const RerankArgs& ra, cudaStream_t s) {
    rerank_kernel<<<static_cast<unsigned>(ceil_div(ra.n_q * 32, 256)), 256, 0, s>>>(ra);
    UMAPB_LAUNCH_CHECK();
}

float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    UMAPB_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
}

struct EventPair {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    EventPair() {
        UMAPB_CUDA(cudaEventCreate(&e0));
        UMAPB_CUDA(cudaEventCreate(&e1));
    }
    ~EventPair() {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    EventPair(const EventPair&) = delete;
    EventPair& operator=(const EventPair&) = delete;
};

}  // namespace

bool knn_tc_supported(int d, int k, int metric) {
    if (metric != UMAPB_METRIC_EUCLIDEAN && metric != UMAPB_METRIC_COSINE) return false;
    if (k < 1 || k > kMaxK || d < 1) return false;
    if (shape_for(geom(d)).st == 0) return false;
    // rows the certificate cannot settle go to the plain kernel, whose tiles
    // bound the width
    if (!knn_plain_supported(d, k)) return false;
    return device_is_sm100();
}

void knn_tc(const float* Q, int64_t n_q, const float* R, int64_t n_r, int d, int k, int metric,
            int32_t* out_idx, float* out_dist, TcKnnStats* stats, cudaStream_t s) {
    if (!knn_tc_supported(d, k, metric))
        invalid("the tensor-core kNN path does not support this metric/shape on this device");
    if (n_q == 0) return;
    if (k > n_r) invalid("kNN needs k <= number of reference rows");
    const bool cosine = metric == UMAPB_METRIC_COSINE;
    const bool self = Q == R && n_q == n_r;
    const float* const Q0 = Q;  // original rows: later passes read rows of these
    const float* const R0 = R;
    const Geom g = geom(d);
    const Shape sh = shape_for(g);
    const Bound bd = bound_for(d, g, cosine);
    TcArgs a = plan(n_q, n_r, g, sh, true, 1);
    CellOrder co;
    const int cells = self && a.n_split == 1 ? cell_count(n_q, d) : 0;
    if (cells > 0) {
        cell_order(Q, n_q, d, cells, sh.mt * BM, ceil_div(n_q, static_cast<int64_t>(BM) * sh.mt),
                   sh.bn, co, s);
        Q = R = co.rows.get();
        a.start_tile = co.start_tile.get();
    }
    const int32_t* perm = cells > 0 ? co.perm.get() : nullptr;
    DevBuf<float> qsq(n_q, s), rsq;
    row_norms(Q, n_q, d, nullptr, qsq.get(), s);
    if (!self) {
        rsq.alloc(n_r, s);
        row_norms(R, n_r, d, nullptr, rsq.get(), s);
    }
    const float* rsq_p = self ? qsq.get() : rsq.get();
    // flags: [0] pass-1 kernel error, [1] pass-1 failed rows, [2] pass-2 kernel
    // error, [3] pass-2 failed rows, [4] largest squared norm (bits)
    DevBuf<int> flags(8, s);
    UMAPB_CUDA(cudaMemsetAsync(flags.get(), 0, 8 * sizeof(int), s));
    unsigned* max_bits = reinterpret_cast<unsigned*>(flags.get() + 4);
    DevBuf<ScaleInfo> sc(1, s);
    if (!cosine) {
        launch_max_sq(qsq.get(), n_q, max_bits, s);
        if (!self) launch_max_sq(rsq.get(), n_r, max_bits, s);
    }
    scale_kernel<<<1, 1, 0, s>>>(max_bits, sc.get());
    UMAPB_LAUNCH_CHECK();
    DevBuf<__half> A(static_cast<size_t>(n_q) * g.kst, s), B(static_cast<size_t>(n_r) * g.kst, s);
    launch_prep(Q, qsq.get(), n_q, d, g, sc.get(), bd, cosine, true, A.get(), s);
    launch_prep(R, rsq_p, n_r, d, g, sc.get(), bd, cosine, false, B.get(), s);
    const int n_lists = sh.lists() * a.n_split;
    DevBuf<uint64_t> lists(static_cast<size_t>(n_q) * n_lists * LS, s);
    clear_lists(lists.get(), static_cast<size_t>(n_q) * n_lists, s);
    const SideMaps ma = side_maps(A.get(), n_q, g, sh, BM);
    const SideMaps mb = side_maps(B.get(), n_r, g, sh, sh.bn);
    a.lists = lists.get();
    a.err = flags.get();
    EventPair ev;
    UMAPB_CUDA(cudaEventRecord(ev.e0, s));
    launch_tc(sh, ma, mb, a, s);
    UMAPB_CUDA(cudaEventRecord(ev.e1, s));
    DevBuf<int32_t> fb_rows(n_q, s);
    RerankArgs ra{};
    ra.Q = Q;
    ra.R = R;
    ra.qsq = qsq.get();
    ra.rsq = rsq_p;
    ra.lists = lists.get();
    ra.n_lists = n_lists;
    ra.n_q = n_q;
    ra.d = d;
    ra.k = k;
    ra.c = bd.c;
    ra.c0 = bd.c0;
    ra.cosine = cosine;
    ra.sc = sc.get();
    ra.omap = perm;
    ra.rmap = perm;
    ra.out_idx = out_idx;
    ra.out_dist = out_dist;
    ra.fb_count = flags.get() + 1;
    ra.fb_rows = fb_rows.get();
    launch_rerank(ra, s);
    int h[2] = {0, 0};
    UMAPB_CUDA(cudaMemcpyAsync(h, flags.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    if (h[0] != 0)
        throw Error(UMAPB_ERR_CUDA, "tensor-core kNN kernel stopped on a wait timeout (code " +
                                        std::to_string(h[0]) + ")");
    float ms = elapsed_ms(ev.e0, ev.e1);
    const int64_t fb = h[1];
    int64_t fb_final = 0;
    if (fb > 0) {
        // Second pass: the failed rows as a query set, with at least two
        // candidate splits (twice as many lists per row) and, where the
        // operands fit shared memory, the three-term FP16 split, whose bound
        // is about 2^-21 of the norms instead of 2^-10.
        lists.release();
        A.release();
        Geom g2 = geom(d, 3);
        Shape sh2 = shape_for(g2);
        if (sh2.st == 0 || sh2.stream) {
            g2 = g;
            sh2 = sh;
        }
        const Bound bd2 = bound_for(d, g2, cosine);
        DevBuf<__half> B2;
        SideMaps mb2 = mb;
        if (g2.terms != g.terms) {
            B.release();
            B2.alloc(static_cast<size_t>(n_r) * g2.kst, s);
            launch_prep(R, rsq_p, n_r, d, g2, sc.get(), bd2, cosine, false, B2.get(), s);
            mb2 = side_maps(B2.get(), n_r, g2, sh2, sh2.bn);
        }
        DevBuf<float> Q2(static_cast<size_t>(fb) * d, s), q2sq(fb, s);
        gather_rows_kernel<<<static_cast<unsigned>(ceil_div(fb * 32, 256)), 256, 0, s>>>(
            Q0, fb_rows.get(), fb, d, Q2.get());
        UMAPB_LAUNCH_CHECK();
        row_norms(Q2.get(), fb, d, nullptr, q2sq.get(), s);
        DevBuf<__half> A2(static_cast<size_t>(fb) * g2.kst, s);
        launch_prep(Q2.get(), q2sq.get(), fb, d, g2, sc.get(), bd2, cosine, true, A2.get(), s);
        TcArgs a2 = plan(fb, n_r, g2, sh2, true, 2);
        const int n_lists2 = sh2.lists() * a2.n_split;
        DevBuf<uint64_t> lists2(static_cast<size_t>(fb) * n_lists2 * LS, s);
        clear_lists(lists2.get(), static_cast<size_t>(fb) * n_lists2, s);
        const SideMaps ma2 = side_maps(A2.get(), fb, g2, sh2, BM);
        a2.lists = lists2.get();
        a2.err = flags.get() + 2;
        EventPair ev2;
        UMAPB_CUDA(cudaEventRecord(ev2.e0, s));
        launch_tc(sh2, ma2, mb2, a2, s);
        UMAPB_CUDA(cudaEventRecord(ev2.e1, s));
        DevBuf<int32_t> fb2_rows(fb, s);
        RerankArgs rb = ra;
        rb.c = bd2.c;
        rb.c0 = bd2.c0;
        rb.Q = Q2.get();
        rb.qsq = q2sq.get();
        rb.lists = lists2.get();
        rb.n_lists = n_lists2;
        rb.n_q = fb;
        rb.omap = fb_rows.get();
        rb.rmap = perm;
        rb.fb_count = flags.get() + 3;
        rb.fb_rows = fb2_rows.get();
        launch_rerank(rb, s);
        int h2[2] = {0, 0};
        UMAPB_CUDA(cudaMemcpyAsync(h2, flags.get() + 2, sizeof(h2), cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaStreamSynchronize(s));
        if (h2[0] != 0)
            throw Error(UMAPB_ERR_CUDA, "tensor-core kNN kernel stopped on a wait timeout (code " +
                                            std::to_string(h2[0]) + ")");
        ms += elapsed_ms(ev2.e0, ev2.e1);
        fb_final = h2[1];
        if (fb_final > 0) {
            DevBuf<float> qn, rn;
            if (cosine) {
                qn.alloc(n_q, s);
                row_norms(Q0, n_q, d, qn.get(), nullptr, s);
                if (!self) {
                    rn.alloc(n_r, s);
                    row_norms(R0, n_r, d, rn.get(), nullptr, s);
                }
            }
            knn_plain(Q0, fb2_rows.get(), fb_final, R0, n_r, d, k, metric, qn.get(),
                      self ? qn.get() : rn.get(), out_idx, out_dist, s);
        }
    }
    if (stats) {
        stats->fallback_rows = fb_final;
        stats->second_pass_rows = fb;
        stats->kernel_ms = ms;
        stats->shortlist = S;
    }
}

}  // namespace umapb

// ===================================================== allocation-free entry
// umapb_knn_exact_noalloc: the tensor-core exact kNN for callers that cannot
// allocate device memory.  Its scratch (operands, shortlists, flags) lives in
// one file-scope device array of kNoAllocScratchBytes that every GPU loading
// this library holds until the process exits.  In host code the array's name
// is only a host-side stand-in, so the device address is fetched once per
// device with cudaGetSymbolAddress (on the first call made with that device
// current) and reused afterwards.  It runs one tensor-core pass; rows that
// pass cannot certify are recomputed on the plain path over the caller's
// rows, which needs no scratch.
namespace umapb {
namespace {
constexpr size_t kNoAllocScratchBytes = static_cast<size_t>(160) << 20;
}  // namespace
}  // namespace umapb

static __device__ __align__(256) unsigned char umapb_noalloc_scratch[umapb::kNoAllocScratchBytes];

namespace umapb {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kMaxDevices] = {};

unsigned char* noalloc_scratch() {
    int dev = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) invalid("device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        UMAPB_CUDA(cudaGetSymbolAddress(&p, umapb_noalloc_scratch));
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    return g_noalloc_ptr[dev];
}

inline size_t round256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

// bytes of scratch one call needs for n rows of d features
size_t noalloc_need(int64_t n, int d) {
    const size_t rows = static_cast<size_t>(n);
    const Geom g = geom(d);
    const Shape sh = shape_for(g);
    return round256(rows * 4) + 2 * round256(rows * g.kst * 2) +
           round256(rows * sh.lists() * LS * 8) + round256(8 * sizeof(int)) +
           round256(sizeof(ScaleInfo)) + round256(rows * 4);
}

void knn_noalloc(const float* X, int64_t n, int d, int k, int32_t* out_idx, float* out_dist,
                 cudaStream_t s) {
    if (n < 1 || d < 1) invalid("empty input");
    if (k < 1 || k > n) invalid("k must be in [1, n_rows]");
    if (!knn_tc_supported(d, k, UMAPB_METRIC_EUCLIDEAN))
        invalid("the allocation-free kNN runs the tensor-core path only (sm_100, euclidean, "
                "k <= 62, n_cols within the tensor-core operand limit)");
    const size_t need = noalloc_need(n, d);
    if (need > kNoAllocScratchBytes) {
        int64_t max_rows = 0;
        while (noalloc_need(max_rows + 1024, d) <= kNoAllocScratchBytes) max_rows += 1024;
        invalid("the allocation-free kNN needs " + std::to_string(need) +
                " bytes of scratch, above its static limit of " +
                std::to_string(kNoAllocScratchBytes) + " bytes (about " +
                std::to_string(max_rows) + " rows at " + std::to_string(d) + " columns)");
    }
    const Geom g = geom(d);
    const Shape sh = shape_for(g);
    const Bound bd = bound_for(d, g, false);
    unsigned char* base = noalloc_scratch();
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        unsigned char* p = base + off;
        off += round256(bytes);
        return p;
    };
    float* sq = reinterpret_cast<float*>(carve(static_cast<size_t>(n) * 4));
    __half* A = reinterpret_cast<__half*>(carve(static_cast<size_t>(n) * g.kst * 2));
    __half* B = reinterpret_cast<__half*>(carve(static_cast<size_t>(n) * g.kst * 2));
    uint64_t* lists =
        reinterpret_cast<uint64_t*>(carve(static_cast<size_t>(n) * sh.lists() * LS * 8));
    // [0] kernel error, [1] rows to recompute, [4] largest squared norm (bits)
    int* flags = reinterpret_cast<int*>(carve(8 * sizeof(int)));
    ScaleInfo* sc = reinterpret_cast<ScaleInfo*>(carve(sizeof(ScaleInfo)));
    int32_t* fb_rows = reinterpret_cast<int32_t*>(carve(static_cast<size_t>(n) * 4));

    // every call starts from cleared shortlists and flags (the array keeps
    // the previous call's contents)
    clear_lists(lists, static_cast<size_t>(n) * sh.lists(), s);
    UMAPB_CUDA(cudaMemsetAsync(flags, 0, 8 * sizeof(int), s));
    row_norms(X, n, d, nullptr, sq, s);
    unsigned* max_bits = reinterpret_cast<unsigned*>(flags + 4);
    launch_max_sq(sq, n, max_bits, s);
    scale_kernel<<<1, 1, 0, s>>>(max_bits, sc);
    UMAPB_LAUNCH_CHECK();
    launch_prep(X, sq, n, d, g, sc, bd, false, true, A, s);
    launch_prep(X, sq, n, d, g, sc, bd, false, false, B, s);
    const SideMaps ma = side_maps(A, n, g, sh, BM);
    const SideMaps mb = side_maps(B, n, g, sh, sh.bn);
    TcArgs a = plan(n, n, g, sh, false, 1);  // one split: the scratch holds one set of lists
    a.lists = lists;
    a.err = flags;
    launch_tc(sh, ma, mb, a, s);
    RerankArgs ra{};
    ra.Q = X;
    ra.R = X;
    ra.qsq = sq;
    ra.rsq = sq;
    ra.lists = lists;
    ra.n_lists = sh.lists();
    ra.n_q = n;
    ra.d = d;
    ra.k = k;
    ra.c = bd.c;
    ra.c0 = bd.c0;
    ra.cosine = false;
    ra.sc = sc;
    ra.out_idx = out_idx;
    ra.out_dist = out_dist;
    ra.fb_count = flags + 1;
    ra.fb_rows = fb_rows;
    launch_rerank(ra, s);
    int flags_h[2] = {0, 0};
    UMAPB_CUDA(cudaMemcpyAsync(flags_h, flags, sizeof(flags_h), cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaStreamSynchronize(s));
    if (flags_h[0] != 0)
        throw Error(UMAPB_ERR_CUDA, "tensor-core kNN kernel stopped on a wait timeout (code " +
                                        std::to_string(flags_h[0]) + ")");
    if (flags_h[1] > 0)
        knn_plain(X, fb_rows, flags_h[1], X, n, d, k, UMAPB_METRIC_EUCLIDEAN, nullptr, nullptr,
                  out_idx, out_dist, s, false);
    UMAPB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace
}  // namespace umapb

extern "C" int32_t umapb_knn_exact_noalloc(const float* data, int64_t n_rows, int64_t n_cols,
                                           int64_t k, int32_t* indices, float* dists,
                                           void* stream) {
    try {
        umapb::knn_noalloc(data, n_rows, static_cast<int>(n_cols), static_cast<int>(k), indices,
                           dists, static_cast<cudaStream_t>(stream));
        umapb::set_last_error("");
        return UMAPB_OK;
    } catch (const umapb::Error& e) {
        umapb::set_last_error(e.what());
        return e.status;
    } catch (const std::exception& e) {
        umapb::set_last_error(e.what());
        return UMAPB_ERR_CUDA;
    }
}
