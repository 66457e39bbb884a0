// LBVH construction and refit for sm_100a.
//
// Pipeline (one stream, no host synchronisation):
//   1. k_root_reduce   per-primitive boxes -> union (order-free atomics on ordered ints)
//   2. k_morton_hist   30-/63-bit Morton code of each box centroid, and the digit
//                      histograms of every sort pass from the same pass over the codes
//   3. radix sort      stable LSD sort of (code, input index), 8-bit digits: one
//                      k_onesweep launch per digit (local ranking, then the tile's digit
//                      offsets by a decoupled look-back over the earlier tiles)
//   4. k_karras        Karras 2012 hierarchy over the sorted codes (+ each node's range)
//   5. k_leaf_climb    leaf boxes + triangle records in sorted order, then one bottom-up
//                      climb per leaf that writes every child box into its parent: in
//                      shared memory while a node's leaves lie in the block's own leaves,
//                      through global memory above that
//
// Reference counterparts (src/): bvh/gpu_bvh.cu:135-149 (codes), 582-584 (sort),
// 151-180 (hierarchy), 182-214 (bottom-up boxes), 535-613 (build/refit drivers);
// bvh/cpu_lbvh_builder.h:163-259 (the host builder the results are bit-exact with).
// The reference's separate subtree-size, preorder and escape passes (gpu_bvh.cu:216-363)
// have no counterpart: traversal walks the Karras nodes directly.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "../../include/lux_gpu.h"
#include "lux_internal.h"

namespace lux {
namespace {

// Launch shapes; the LUX_* macros exist so that other shapes can be built and timed
// against these defaults (results do not depend on them).
#ifndef LUX_SORT_ITEMS
#define LUX_SORT_ITEMS 16
#endif
#ifndef LUX_CLIMB_THREADS
#define LUX_CLIMB_THREADS 256
#endif
#ifndef LUX_LOOKBACK_BATCH
#define LUX_LOOKBACK_BATCH 8
#endif
#ifndef LUX_SORT_THREADS
#define LUX_SORT_THREADS 512
#endif

constexpr int kThreads = 256;
constexpr int kRadix = 256;
constexpr int kSortItems = LUX_SORT_ITEMS;
constexpr int kSortThreads = LUX_SORT_THREADS;      // threads of a k_onesweep block
constexpr int kSortTile = kSortThreads * kSortItems;  // keys per tile
// The allocation-free sort's tiles (its scratch size is part of the ABI): fixed.
constexpr int kStaticItems = 16;
constexpr int kStaticTile = kThreads * kStaticItems;
constexpr int kScanThreads = 1024;
constexpr int kClimbBound = 160;                 // > max tree depth (64 + 96 bits)
constexpr int kMaxPasses = 8;                    // 8-bit digits of a 63-bit key
constexpr int kClimbThreads = LUX_CLIMB_THREADS; // leaves per climb block
constexpr int kClimbSmem = kClimbThreads * (6 * 8 + 4);   // k_leaf_climb's shared memory
constexpr long long kLookbackSpins = 1ll << 22;  // bound of one look-back wait

// Relaxed device-scope accesses of the look-back words (each word carries its own value,
// so no other ordering is needed) and an acquire-release add for the climb's flags.
LUX_D unsigned ld_relaxed(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
LUX_D void st_relaxed(unsigned* p, unsigned v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
LUX_D unsigned atomic_add_acq_rel(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
                 : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

LUX_D unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <int Kind>
LUX_D void load_prim(const float* prims, int i, f3& v0, f3& v1, f3& v2, box3& b) {
    if (Kind == LUX_PRIM_TRIANGLES) {
        const float* t = prims + static_cast<size_t>(i) * 9;
        v0 = make_f3(t[0], t[1], t[2]);
        v1 = make_f3(t[3], t[4], t[5]);
        v2 = make_f3(t[6], t[7], t[8]);
        b = triangle_box(v0, v1, v2);
    } else {
        const float* t = prims + static_cast<size_t>(i) * 6;
        b = box3{make_f3(t[0], t[1], t[2]), make_f3(t[3], t[4], t[5])};
        v0 = v1 = v2 = make_f3(0, 0, 0);
    }
}

// load_prim through 16-byte loads: the aligned window of three float4 (triangles, 36 B at
// any 4-byte offset) or two (boxes, 24 B at an 8-byte offset) that holds the primitive,
// the primitive's floats then selected from it.  Three load instructions instead of nine
// (two instead of six), each lane's bytes in at most three sectors.  Used when the
// buffer is 16-byte aligned and the window ends inside it; the scalar loads otherwise.
template <int Kind>
LUX_D void load_prim_vec(const float* prims, int n, int i, bool aligned, f3& v0, f3& v1,
                         f3& v2, box3& b) {
    constexpr int kFloats = Kind == LUX_PRIM_TRIANGLES ? 9 : 6;
    constexpr int kWindow = Kind == LUX_PRIM_TRIANGLES ? 12 : 8;
    const size_t off = static_cast<size_t>(i) * kFloats;
    const size_t base = off & ~size_t(3);
    if (!aligned || base + kWindow > static_cast<size_t>(n) * kFloats) {
        load_prim<Kind>(prims, i, v0, v1, v2, b);
        return;
    }
    const int r = static_cast<int>(off & 3);
    const float4* p = reinterpret_cast<const float4*>(prims + base);
    float w[kWindow];
#pragma unroll
    for (int q = 0; q < kWindow / 4; ++q) {
        const float4 x = __ldg(p + q);
        w[4 * q] = x.x; w[4 * q + 1] = x.y; w[4 * q + 2] = x.z; w[4 * q + 3] = x.w;
    }
    float t[kFloats];
#pragma unroll
    for (int j = 0; j < kFloats; ++j) {
        if (Kind == LUX_PRIM_TRIANGLES)
            t[j] = r == 0 ? w[j] : r == 1 ? w[j + 1] : r == 2 ? w[j + 2] : w[j + 3];
        else
            t[j] = r == 0 ? w[j] : w[j + 2];
    }
    if (Kind == LUX_PRIM_TRIANGLES) {
        v0 = make_f3(t[0], t[1], t[2]);
        v1 = make_f3(t[3], t[4], t[5]);
        v2 = make_f3(t[6], t[7], t[8]);
        b = triangle_box(v0, v1, v2);
    } else {
        b = box3{make_f3(t[0], t[1], t[2]), make_f3(t[3], t[4], t[5])};
        v0 = v1 = v2 = make_f3(0, 0, 0);
    }
}

LUX_D bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// ---------------------------------------------------------------- 1. root box

template <int Kind>
__global__ void __launch_bounds__(kThreads) k_root_reduce(const float* prims, int n,
                                                          unsigned* root_ord) {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        f3 v0, v1, v2;
        box3 b;
        load_prim<Kind>(prims, i, v0, v1, v2, b);
        lo[0] = fminf(lo[0], b.lo.x); lo[1] = fminf(lo[1], b.lo.y); lo[2] = fminf(lo[2], b.lo.z);
        hi[0] = fmaxf(hi[0], b.hi.x); hi[1] = fmaxf(hi[1], b.hi.y); hi[2] = fmaxf(hi[2], b.hi.z);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
        }
    }
    // The block's warps meet in shared memory; one atomic per block and value (the
    // atomics of every warp on six words serialised in L2).
    __shared__ float part[kThreads / 32][6];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            part[warp][a] = lo[a];
            part[warp][3 + a] = hi[a];
        }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int a = threadIdx.x;
        float v = part[0][a];
        for (int w = 1; w < kThreads / 32; ++w) v = a < 3 ? fminf(v, part[w][a]) : fmaxf(v, part[w][a]);
        if (a < 3) atomicMin(root_ord + a, float_to_ordered(v));
        else atomicMin(root_ord + a, ~float_to_ordered(v));
    }
}

LUX_D box3 decode_root(const unsigned* root_ord) {
    return box3{make_f3(ordered_to_float(root_ord[0]), ordered_to_float(root_ord[1]),
                        ordered_to_float(root_ord[2])),
                make_f3(ordered_to_float(~root_ord[3]), ordered_to_float(~root_ord[4]),
                        ordered_to_float(~root_ord[5]))};
}

// ---------------------------------------------------------------- 2. Morton codes

template <int Kind, typename Key>
__global__ void __launch_bounds__(kThreads) k_morton(const float* prims, int n,
                                                     const unsigned* root_ord, Key* codes) {
    box3 root = decode_root(root_ord);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        f3 v0, v1, v2;
        box3 b;
        load_prim<Kind>(prims, i, v0, v1, v2, b);
        if (sizeof(Key) == 4) {
            codes[i] = static_cast<Key>(morton30(b, root));
        } else {
            codes[i] = static_cast<Key>(morton63(b, root));
        }
    }
}

// ---------------------------------------------------------------- 3. radix sort

template <typename Key>
LUX_D unsigned digit_of(Key k, int shift) {
    return static_cast<unsigned>(k >> shift) & (kRadix - 1);
}

// Morton codes (as k_morton) plus, for every sort pass p, the count of each 8-bit digit
// of the codes: hist[p * kRadix + d], accumulated in shared memory (one copy per warp
// for 30-bit keys, two for the 63-bit keys' eight passes, to stay within 48 KB) and added
// to the global counts once per block.
template <int Kind, typename Key, int Passes>
__global__ void __launch_bounds__(kThreads) k_morton_hist(const float* prims, int n,
                                                          const unsigned* root_ord,
                                                          Key* codes, unsigned* hist) {
    constexpr int kCopies = Passes <= 4 ? kThreads / 32 : 2;
    __shared__ unsigned h[kCopies][Passes][kRadix];
    for (int i = threadIdx.x; i < kCopies * Passes * kRadix; i += kThreads) (&h[0][0][0])[i] = 0;
    __syncthreads();
    const int warp = (threadIdx.x >> 5) % kCopies;
    box3 root = decode_root(root_ord);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        f3 v0, v1, v2;
        box3 b;
        load_prim<Kind>(prims, i, v0, v1, v2, b);
        Key c = sizeof(Key) == 4 ? static_cast<Key>(morton30(b, root))
                                 : static_cast<Key>(morton63(b, root));
        codes[i] = c;
#pragma unroll
        for (int p = 0; p < Passes; ++p) atomicAdd(&h[warp][p][digit_of(c, 8 * p)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < Passes * kRadix; i += kThreads) {
        unsigned v = 0;
#pragma unroll
        for (int w = 0; w < kCopies; ++w) v += (&h[w][0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
}

// Exclusive prefix of each pass's digit counts: bases[p * kRadix + d] = the number of
// keys whose pass-p digit is below d.  One block of kRadix threads per pass.
__global__ void __launch_bounds__(kRadix) k_digit_bases(const unsigned* hist, unsigned* bases) {
    __shared__ unsigned warp_sums[kRadix / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned v = hist[blockIdx.x * kRadix + threadIdx.x];
    unsigned incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        unsigned o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += o;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    unsigned before = 0;
    for (int w = 0; w < warp; ++w) before += warp_sums[w];
    bases[blockIdx.x * kRadix + threadIdx.x] = before + incl - v;
}

// Lanes of the warp whose digit (and validity) equal this lane's: a validity ballot and
// one ballot per digit bit, ANDed (cheaper than a general match on sm_100a).
LUX_D unsigned digit_peers(unsigned d, bool valid) {
    unsigned peers = __ballot_sync(0xffffffffu, valid);
    if (!valid) peers = ~peers;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const bool bit = (d >> b) & 1u;
        const unsigned m = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? m : ~m;
    }
    return peers;
}

// Look-back words, 32 bits: 0 while not yet published; kTileAggregate | this tile's own
// count (at most kSortTile); kTilePrefix | the count over tiles 0..t (at most 2^30, the
// primitive limit, so it fits below the flag bit).
constexpr unsigned kTileAggregate = 1u << 30;
constexpr unsigned kTilePrefix = 1u << 31;
constexpr int kLookbackBatch = LUX_LOOKBACK_BATCH;   // earlier tiles' words loaded together

// One stable LSD pass over all keys.  Tiles of kSortTile keys are taken in launch order
// (an atomic counter), ranked inside the tile as k_sort_downsweep ranks them (per-warp
// digit counts in input order, so equal digits keep input order), and placed at
// bases[d] + (digit d's count in earlier tiles) + the rank in the tile.  The count in
// earlier tiles comes from a decoupled look-back: each tile publishes its per-digit
// count, then walks back over the earlier tiles' words until one holds an inclusive
// prefix, and publishes its own inclusive prefix.  A tile waits only on tiles that were
// handed out before it (and so are running or done); each wait is bounded and a wait
// that runs out reports through `error`.
template <typename Key, bool First>
__global__ void __launch_bounds__(kSortThreads) k_onesweep(const Key* keys_in,
                                                           const int* vals_in, Key* keys_out,
                                                           int* vals_out, int n, int shift,
                                                           const unsigned* bases,
                                                           unsigned* lookback,
                                                           unsigned* tile_counter, int* error) {
    static_assert(kSortThreads >= kRadix, "one thread per digit in the look-back");
    constexpr int kWarps = kSortThreads / 32;
    constexpr int kWarpSpan = kSortTile / kWarps;
    __shared__ unsigned wcount[kWarps][kRadix];
    __shared__ unsigned gbase[kRadix];
    __shared__ int tile_s;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) tile_s = static_cast<int>(atomicAdd(tile_counter, 1u));
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kSortThreads) (&wcount[0][0])[i] = 0;
    __syncthreads();
    const int tile = tile_s;

    const unsigned lt = lanemask_lt();
    const int base = tile * kSortTile + warp * kWarpSpan;
    Key k[kSortItems];
    int v[kSortItems];
    unsigned rank[kSortItems];
    // All of the warp's keys and values are loaded before the ranking starts, so their
    // loads are in flight together rather than one per ranking round.
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        int idx = base + j * 32 + lane;
        bool valid = idx < n;
        k[j] = valid ? keys_in[idx] : Key(0);
        v[j] = First ? idx : (valid ? vals_in[idx] : 0);
    }
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        int idx = base + j * 32 + lane;
        bool valid = idx < n;
        unsigned d = valid ? digit_of(k[j], shift) : 0u;
        unsigned peers = digit_peers(d, valid);
        unsigned before = valid ? wcount[warp][d] : 0u;
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wcount[warp][d] = before + __popc(peers);
        __syncwarp();
        rank[j] = valid ? before + __popc(peers & lt) : 0xffffffffu;
    }
    __syncthreads();
    if (threadIdx.x < kRadix) {
        const int d = threadIdx.x;
        unsigned total = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            unsigned c = wcount[w][d];
            wcount[w][d] = total;
            total += c;
        }
        unsigned* mine = lookback + static_cast<size_t>(tile) * kRadix + d;
        unsigned prefix = 0;
        if (tile == 0) {
            st_relaxed(mine, kTilePrefix | total);
        } else {
            st_relaxed(mine, kTileAggregate | total);
            // Walk back kLookbackBatch tiles at a time (their words are loaded together,
            // so a run of aggregates costs one load latency per batch): take every
            // published word up to the nearest inclusive prefix, and re-read from the
            // first word not yet published.
            int t = tile - 1;
            long long spins = 0;
            bool found = false;
            while (!found && t >= 0) {
                unsigned w[kLookbackBatch];
#pragma unroll
                for (int j = 0; j < kLookbackBatch; ++j)
                    w[j] = t - j >= 0 ? ld_relaxed(lookback + static_cast<size_t>(t - j) * kRadix + d)
                                      : 0u;
                int taken = 0;
                bool blocked = false;
#pragma unroll
                for (int j = 0; j < kLookbackBatch; ++j) {
                    if (found || blocked || t - j < 0) continue;
                    if (w[j] == 0) {          // not published yet: resume at this tile
                        blocked = true;
                        continue;
                    }
                    found = (w[j] & kTilePrefix) != 0;
                    prefix += w[j] & (found ? ~kTilePrefix : ~kTileAggregate);
                    taken = j + 1;
                }
                t -= taken;
                if (blocked && ++spins > kLookbackSpins) {
                    atomicOr(error, kErrLoopBound);
                    break;
                }
            }
            st_relaxed(mine, kTilePrefix | (prefix + total));
        }
        gbase[d] = bases[d] + prefix;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        if (rank[j] == 0xffffffffu) continue;
        unsigned d = digit_of(k[j], shift);
        unsigned pos = gbase[d] + wcount[warp][d] + rank[j];
        if (pos >= static_cast<unsigned>(n)) {  // cannot happen for consistent counts
            atomicOr(error, kErrLoopBound);
            continue;
        }
        keys_out[pos] = k[j];
        vals_out[pos] = v[j];
    }
}

// Per-tile digit counts, stored digit-major: hist[d * tiles + tile].
template <typename Key>
__global__ void __launch_bounds__(kThreads) k_sort_upsweep(const Key* keys, int n, int shift,
                                                           unsigned* hist, int tiles) {
    __shared__ unsigned counts[kRadix];
    counts[threadIdx.x] = 0;
    __syncthreads();
    int base = blockIdx.x * kStaticTile;
#pragma unroll 4
    for (int j = 0; j < kStaticItems; ++j) {
        int idx = base + j * kThreads + threadIdx.x;
        bool valid = idx < n;
        unsigned d = valid ? digit_of(keys[idx], shift) : kRadix;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        if (valid && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&counts[d], __popc(peers));
    }
    __syncthreads();
    hist[threadIdx.x * tiles + blockIdx.x] = counts[threadIdx.x];
}

// Exclusive scan of `count` words in place, one block.  count is a multiple of 4 and
// data 16-byte aligned: each pass covers 4096 words with one coalesced uint4 per
// thread, a warp-shuffle scan of the per-thread sums and a carry into the next pass.
__global__ void __launch_bounds__(kScanThreads) k_scan_exclusive(unsigned* data, int count) {
    constexpr int kWarps = kScanThreads / 32;
    __shared__ unsigned warp_sums[kWarps];
    __shared__ unsigned carry_s;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry_s = 0;
    uint4* data4 = reinterpret_cast<uint4*>(data);
    const int count4 = count >> 2;
    for (int base = 0; base < count4; base += kScanThreads) {
        int i = base + threadIdx.x;
        uint4 v = i < count4 ? data4[i] : make_uint4(0, 0, 0, 0);
        unsigned s = v.x + v.y + v.z + v.w;
        unsigned incl = s;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            unsigned o = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += o;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            unsigned w = warp_sums[lane];
            unsigned wi = w;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                unsigned o = __shfl_up_sync(0xffffffffu, wi, off);
                if (lane >= off) wi += o;
            }
            warp_sums[lane] = wi - w;  // exclusive prefix of warp totals
        }
        __syncthreads();
        unsigned carry = carry_s;
        unsigned run = carry + warp_sums[warp] + incl - s;
        if (i < count4) {
            uint4 o;
            o.x = run;
            o.y = run + v.x;
            o.z = o.y + v.y;
            o.w = o.z + v.z;
            data4[i] = o;
        }
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry_s = run + s;
        __syncthreads();
    }
}

// Stable scatter of one tile.  Warp w owns tile keys [w*512, w*512+512), visited in
// rounds of 32 consecutive keys; a key's rank is (count of its digit in this warp's
// earlier rounds) + (peers with the same digit in lower lanes), then offset by the same
// digit's counts in earlier warps and earlier tiles, so equal digits keep input order.
template <typename Key, bool First>
__global__ void __launch_bounds__(kThreads) k_sort_downsweep(const Key* keys_in,
                                                             const int* vals_in, Key* keys_out,
                                                             int* vals_out, int n, int shift,
                                                             const unsigned* scanned,
                                                             int tiles, int* error) {
    constexpr int kWarps = kThreads / 32;
    constexpr int kWarpSpan = kStaticTile / kWarps;
    __shared__ unsigned wcount[kWarps][kRadix];
    __shared__ unsigned gbase[kRadix];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kThreads) (&wcount[0][0])[i] = 0;
    gbase[threadIdx.x] = scanned[threadIdx.x * tiles + blockIdx.x];
    __syncthreads();

    const unsigned lt = lanemask_lt();
    const int base = blockIdx.x * kStaticTile + warp * kWarpSpan;
    Key k[kStaticItems];
    int v[kStaticItems];
    unsigned rank[kStaticItems];
#pragma unroll
    for (int j = 0; j < kStaticItems; ++j) {
        int idx = base + j * 32 + lane;
        bool valid = idx < n;
        k[j] = valid ? keys_in[idx] : Key(0);
        v[j] = First ? idx : (valid ? vals_in[idx] : 0);
        unsigned d = valid ? digit_of(k[j], shift) : kRadix;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        unsigned before = valid ? wcount[warp][d] : 0u;
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wcount[warp][d] = before + __popc(peers);
        __syncwarp();
        rank[j] = valid ? before + __popc(peers & lt) : 0xffffffffu;
    }
    __syncthreads();
    {
        unsigned run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            unsigned c = wcount[w][threadIdx.x];
            wcount[w][threadIdx.x] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kStaticItems; ++j) {
        if (rank[j] == 0xffffffffu) continue;
        unsigned d = digit_of(k[j], shift);
        unsigned pos = gbase[d] + wcount[warp][d] + rank[j];
        if (pos >= static_cast<unsigned>(n)) {  // cannot happen for a consistent histogram
            atomicOr(error, kErrLoopBound);
            continue;
        }
        keys_out[pos] = k[j];
        vals_out[pos] = v[j];
    }
}

// ---------------------------------------------------------------- 4. Karras hierarchy

LUX_D int clz64(unsigned long long x) { return __clzll(static_cast<long long>(x)); }

// Common-prefix length of sorted keys i and j.  30-bit codes: the reference's merged
// key (code << 32) | index (bvh/gpu_bvh.cu:66-74).  63-bit codes: the code prefix, and
// the index prefix beyond it when the codes are equal.
template <typename Key>
LUX_D int delta(const Key* codes, int i, int j) {
    if (sizeof(Key) == 4) {
        unsigned long long ki = (static_cast<unsigned long long>(codes[i]) << 32) | unsigned(i);
        unsigned long long kj = (static_cast<unsigned long long>(codes[j]) << 32) | unsigned(j);
        return clz64(ki ^ kj);
    } else {
        unsigned long long x = static_cast<unsigned long long>(codes[i] ^ codes[j]);
        if (x) return clz64(x);
        return 64 + __clz(static_cast<int>(unsigned(i) ^ unsigned(j)));
    }
}

// node_info[i]: (first leaf, last leaf, parent code, unused) of internal node i; the
// range is written by node i's thread, the parent code by its parent's.
template <typename Key>
__global__ void __launch_bounds__(kThreads) k_karras(const Key* codes, int n, BvhNode* nodes,
                                                     int* node_parent, int* leaf_parent,
                                                     int4* node_info) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int first, last;
    if (i == 0) {
        first = 0;
        last = n - 1;
        node_parent[0] = -1;
        reinterpret_cast<int*>(node_info)[2] = -1;
    } else {
        // determine_range (bvh/gpu_bvh.cu:76-105).
        int dl = delta(codes, i, i - 1);
        int dr = delta(codes, i, i + 1);
        int dir = dr > dl ? 1 : -1;
        int dmin = min(dl, dr);
        int lmax = 2;
        for (;;) {
            int c = i + dir * lmax;
            if (c < 0 || c >= n) break;
            if (delta(codes, i, c) <= dmin) break;
            lmax <<= 1;
        }
        int len = 0;
        for (int step = lmax >> 1; step > 0; step >>= 1) {
            int c = i + (len + step) * dir;
            if (c < 0 || c >= n) continue;
            if (delta(codes, i, c) > dmin) len += step;
        }
        int other = i + len * dir;
        first = dir < 0 ? other : i;
        last = dir < 0 ? i : other;
    }
    // find_split (bvh/gpu_bvh.cu:107-121).
    int node_delta = delta(codes, first, last);
    int split = first;
    int stride = last - first;
    do {
        stride = (stride + 1) >> 1;
        int mid = split + stride;
        if (mid < last && delta(codes, first, mid) > node_delta) split = mid;
    } while (stride > 1);

    int left = first == split ? ~split : split;
    int right = last == split + 1 ? ~(split + 1) : split + 1;
    reinterpret_cast<int2*>(&nodes[i].ch)[0] = make_int2(left, right);
    reinterpret_cast<int2*>(node_info + i)[0] = make_int2(first, last);
    if (left < 0) {
        leaf_parent[split] = i << 1;
    } else {
        node_parent[split] = i << 1;
        reinterpret_cast<int*>(node_info + split)[2] = i << 1;
    }
    if (right < 0) {
        leaf_parent[split + 1] = (i << 1) | 1;
    } else {
        node_parent[split + 1] = (i << 1) | 1;
        reinterpret_cast<int*>(node_info + split + 1)[2] = (i << 1) | 1;
    }
}

// ---------------------------------------------------------------- 5. boxes bottom-up

LUX_D void store_slot(BvhNode* node, int slot, const box3& b) {
    float* f = reinterpret_cast<float*>(node);
    if (slot == 0) {
        __stcg(reinterpret_cast<float4*>(f), make_float4(b.lo.x, b.lo.y, b.lo.z, b.hi.x));
        __stcg(reinterpret_cast<float2*>(f + 4), make_float2(b.hi.y, b.hi.z));
    } else {
        __stcg(reinterpret_cast<float2*>(f + 6), make_float2(b.lo.x, b.lo.y));
        __stcg(reinterpret_cast<float4*>(f + 8), make_float4(b.lo.z, b.hi.x, b.hi.y, b.hi.z));
    }
}

LUX_D box3 load_slot_cg(const BvhNode* node, int slot) {
    const float* f = reinterpret_cast<const float*>(node);
    if (slot == 0) {
        float4 a = __ldcg(reinterpret_cast<const float4*>(f));
        float2 b = __ldcg(reinterpret_cast<const float2*>(f + 4));
        return box3{make_f3(a.x, a.y, a.z), make_f3(a.w, b.x, b.y)};
    }
    float2 a = __ldcg(reinterpret_cast<const float2*>(f + 6));
    float4 b = __ldcg(reinterpret_cast<const float4*>(f + 8));
    return box3{make_f3(a.x, a.y, b.x), make_f3(b.y, b.z, b.w)};
}

// One thread per sorted leaf.  The leaf box (and, for triangles, the sorted triangle
// record) is written; then the thread climbs: it hands its box to the parent, and the
// second of the two children to arrive (a counter) unions both and continues upward, so
// every node box is the union of its children's boxes (merge_bounds_kernel,
// bvh/gpu_bvh.cu:182-214).  A node whose leaf range lies inside this block's leaves
// [lo, lo + kClimbThreads) has both its children climbing in this block and an index in
// that range too (a Karras node is numbered by one end of its range), so the hand-over
// goes through shared memory; above that through the node's slot in global memory with
// an acquire-release counter, which the second arrival resets to zero.  One 16-byte load
// of node_info per level gives the node's range and its parent link.
template <int Kind>
__global__ void __launch_bounds__(kClimbThreads) k_leaf_climb(const float* prims, int n,
                                                              const int* sorted_ids,
                                                              TriRecord* tris, BvhNode* nodes,
                                                              const int* leaf_parent,
                                                              const int4* node_info,
                                                              unsigned* flags, float* root,
                                                              int* error) {
    // Per node of the block: each child's box (three float2) and an arrival counter, in
    // dynamic shared memory (kClimbSmem bytes).
    extern __shared__ float2 climb_smem[];
    float2 (*sbox)[2][3] = reinterpret_cast<float2 (*)[2][3]>(climb_smem);
    unsigned* sflag = reinterpret_cast<unsigned*>(climb_smem + 6 * kClimbThreads);
    const int lo = blockIdx.x * kClimbThreads;
    sflag[threadIdx.x] = 0;
    __syncthreads();
    int k = lo + threadIdx.x;
    if (k >= n) return;
    // The leaf's id, its parent link and the parent's record are fetched before the
    // primitive, so the two dependent chains overlap.
    const int pid = sorted_ids[k];
    int code = n > 1 ? leaf_parent[k] : -1;
    int4 info = make_int4(0, -1, -1, 0);
    if (code >= 0 && (code >> 1) < n - 1) info = node_info[code >> 1];
    if (pid < 0 || pid >= n) {  // cannot happen for a consistent sort
        atomicOr(error, kErrLoopBound);
        return;
    }
    f3 v0, v1, v2;
    box3 b;
    load_prim_vec<Kind>(prims, n, pid, aligned16(prims), v0, v1, v2, b);
    if (Kind == LUX_PRIM_TRIANGLES) {
        TriRecord r;
        r.p0 = make_float4(v0.x, v0.y, v0.z, __int_as_float(pid));
        r.p1 = make_float4(v1.x, v1.y, v1.z, 0.0f);
        r.p2 = make_float4(v2.x, v2.y, v2.z, 0.0f);
        tris[k] = r;
    }
    if (n == 1) {
        root[0] = b.lo.x; root[1] = b.lo.y; root[2] = b.lo.z;
        root[3] = b.hi.x; root[4] = b.hi.y; root[5] = b.hi.z;
        return;
    }
    for (int level = 0; level < kClimbBound; ++level) {
        int p = code >> 1;
        int slot = code & 1;
        if (code < 0 || p >= n - 1) break;  // parent links out of range: report below
        // The grandparent's record is requested now, before the hand-over, so its load
        // overlaps this level's (for the half of the threads that go on).
        const int up = info.z;
        int4 next = make_int4(0, -1, -1, 0);
        if (up >= 0 && (up >> 1) < n - 1) next = node_info[up >> 1];
        const int s = p - lo;
        if (info.x >= lo && info.y < lo + kClimbThreads && s >= 0 && s < kClimbThreads) {
            // The block fences order the box's stores before the counter's add, and the
            // add before the sibling's box is read (they are also compiler barriers).
            float2* mine = &sbox[s][slot][0];
            mine[0] = make_float2(b.lo.x, b.lo.y);
            mine[1] = make_float2(b.lo.z, b.hi.x);
            mine[2] = make_float2(b.hi.y, b.hi.z);
            __threadfence_block();
            unsigned prior = atomicAdd(&sflag[s], 1u);
            if (prior == 0) return;  // the sibling finishes this node
            __threadfence_block();
            const float2* o = &sbox[s][slot ^ 1][0];
            const float2 o0 = o[0], o1 = o[1], o2 = o[2];
            box3 sib{make_f3(o0.x, o0.y, o1.x), make_f3(o1.y, o2.x, o2.y)};
            const box3 left = slot ? sib : b;
            const box3 right = slot ? b : sib;
            store_slot(nodes + p, 0, left);
            store_slot(nodes + p, 1, right);
            b = box_union(left, right);
        } else {
            store_slot(nodes + p, slot, b);
            unsigned prior = atomic_add_acq_rel(flags + p, 1u);
            if (prior == 0) return;  // the sibling finishes this node
            flags[p] = 0;
            box3 sib = load_slot_cg(nodes + p, slot ^ 1);
            b = slot ? box_union(sib, b) : box_union(b, sib);
        }
        if (p == 0) {
            root[0] = b.lo.x; root[1] = b.lo.y; root[2] = b.lo.z;
            root[3] = b.hi.x; root[4] = b.hi.y; root[5] = b.hi.z;
            return;
        }
        code = up;
        info = next;
    }
    atomicOr(error, kErrClimbBound);
}

// ---------------------------------------------------------------- export

// Host tree layout (bvh/cpu_bvh.h:15-32): internal i, then leaf k at n-1+k.
template <typename Key>
__global__ void k_export(BvhView v, const Key* codes, unsigned long long* codes64, int* left,
                         int* right, float* bounds) {
    int n = v.n;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && codes64) codes64[i] = static_cast<unsigned long long>(codes[i]);
    if (i >= 2 * n - 1) return;
    box3 b;
    int l = -1, r = -1;
    if (i < n - 1) {
        BvhNode nd = load_node(v.nodes, i);
        b = box_union(node_left_box(nd), node_right_box(nd));
        l = nd.ch.x < 0 ? n - 1 + ~nd.ch.x : nd.ch.x;
        r = nd.ch.y < 0 ? n - 1 + ~nd.ch.y : nd.ch.y;
    } else {
        b = leaf_box(v, i - (n - 1));
    }
    if (left) left[i] = l;
    if (right) right[i] = r;
    if (bounds) {
        float* o = bounds + static_cast<size_t>(i) * 6;
        o[0] = b.lo.x; o[1] = b.lo.y; o[2] = b.lo.z;
        o[3] = b.hi.x; o[4] = b.hi.y; o[5] = b.hi.z;
    }
}

int grid_for(int count, int threads = kThreads) { return (count + threads - 1) / threads; }

// Launches one kernel of the build chain on ctx's stream and counts it.
template <typename... Params, typename... Args>
cudaError_t chain_launch(lux_ctx* ctx, void (*kernel)(Params...), int grid, int block,
                         size_t smem, Args... args) {
    ctx->launches += 1;
    kernel<<<grid, block, smem, ctx->stream>>>(static_cast<Params>(args)...);
    return cudaGetLastError();
}

int stride_grid(const lux_ctx* ctx, int count) {
    return std::max(1, std::min(grid_for(count), ctx->sm_count * 8));
}

// Device scratch of a build: the sort's alternate keys and values, the digit counts and
// bases of every pass, the tile counters and the look-back words.
struct SortScratch {
    size_t key_bytes, val_bytes, counts_bytes, lookback_bytes;
    size_t total() const { return key_bytes + val_bytes + counts_bytes + lookback_bytes; }
};

SortScratch sort_scratch(int n, size_t key_size, int passes) {
    const size_t tiles = static_cast<size_t>((n + kSortTile - 1) / kSortTile);
    SortScratch s;
    s.key_bytes = (static_cast<size_t>(n) * key_size + 255) & ~size_t(255);
    s.val_bytes = (static_cast<size_t>(n) * sizeof(int) + 255) & ~size_t(255);
    // hist[kMaxPasses * kRadix], tile counters[kMaxPasses] (padded), bases[...]
    s.counts_bytes = 2 * sizeof(unsigned) * kMaxPasses * kRadix + 256;
    s.lookback_bytes = sizeof(unsigned) * kRadix * tiles * passes;
    return s;
}

// Morton codes of the primitives into `codes` and their stable sort with the input
// indices into (codes, vals): k_morton_hist, k_digit_bases, then one k_onesweep per
// 8-bit digit (an even count, so the result lands back in the caller's arrays).
template <int Kind, typename Key>
int morton_and_sort(lux_ctx* ctx, const float* prims, const unsigned* root_ord, Key* codes,
                    int* vals, int n) {
    constexpr int kPasses = sizeof(Key) == 4 ? 4 : 8;   // 30 bits: 4 digits; 63 bits: 8
    const int tiles = grid_for(n, kSortTile);
    const SortScratch layout = sort_scratch(n, sizeof(Key), kPasses);
    int st = ensure_scratch(ctx, layout.total());
    if (st) return st;
    char* s = static_cast<char*>(ctx->scratch);
    Key* keys_alt = reinterpret_cast<Key*>(s);
    int* vals_alt = reinterpret_cast<int*>(s + layout.key_bytes);
    unsigned* hist = reinterpret_cast<unsigned*>(s + layout.key_bytes + layout.val_bytes);
    unsigned* bases = hist + kMaxPasses * kRadix;
    unsigned* counters = bases + kMaxPasses * kRadix;
    auto* lookback = reinterpret_cast<unsigned*>(
        s + layout.key_bytes + layout.val_bytes + layout.counts_bytes);
    // Counts, tile counters and look-back words start at zero (reset by the caller
    // before the chain's first kernel, reset_sort_scratch).
    const int hist_grid = std::max(1, std::min(grid_for(n), ctx->sm_count * 2));
    cudaError_t err = chain_launch(ctx, k_morton_hist<Kind, Key, kPasses>, hist_grid, kThreads,
                                   0, prims, n, root_ord, codes, hist);
    if (err == cudaSuccess) err = chain_launch(ctx, k_digit_bases, kPasses, kRadix, 0, hist, bases);
    Key* kin = codes;
    int* vin = vals;
    Key* kout = keys_alt;
    int* vout = vals_alt;
    for (int p = 0; p < kPasses && err == cudaSuccess; ++p) {
        unsigned* words = lookback + static_cast<size_t>(p) * tiles * kRadix;
        err = chain_launch(ctx, p == 0 ? k_onesweep<Key, true> : k_onesweep<Key, false>, tiles,
                           kSortThreads, 0, kin, vin, kout, vout, n, 8 * p, bases + p * kRadix,
                           words, counters + p, ctx->d_error);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    return cuda_fail(err, "radix sort");
}

// Zeroes the sort's counts, tile counters and look-back words in ctx's scratch (laid out
// as morton_and_sort lays it out); grows the scratch first.
template <typename Key>
int reset_sort_scratch(lux_ctx* ctx, int n) {
    constexpr int kPasses = sizeof(Key) == 4 ? 4 : 8;
    const SortScratch layout = sort_scratch(n, sizeof(Key), kPasses);
    if (int st = ensure_scratch(ctx, layout.total())) return st;
    char* s = static_cast<char*>(ctx->scratch);
    unsigned* hist = reinterpret_cast<unsigned*>(s + layout.key_bytes + layout.val_bytes);
    unsigned* counters = hist + 2 * kMaxPasses * kRadix;
    cudaError_t err = cudaMemsetAsync(hist, 0, sizeof(unsigned) * kMaxPasses * kRadix,
                                      ctx->stream);
    if (err == cudaSuccess)
        err = cudaMemsetAsync(counters, 0, 256 + layout.lookback_bytes, ctx->stream);
    return err == cudaSuccess ? LUX_OK : cuda_fail(err, "sort scratch reset");
}

template <int Kind>
int climb(lux_ctx* ctx, lux_bvh* bvh, const float* prims) {
    if (kClimbSmem > 48 * 1024) {
        cudaError_t err = cudaFuncSetAttribute(
            k_leaf_climb<Kind>, cudaFuncAttributeMaxDynamicSharedMemorySize, kClimbSmem);
        if (err != cudaSuccess) return cuda_fail(err, "k_leaf_climb shared memory");
    }
    return cuda_fail(chain_launch(ctx, k_leaf_climb<Kind>, grid_for(bvh->n, kClimbThreads),
                                  kClimbThreads, kClimbSmem, prims, bvh->n, bvh->sorted_ids,
                                  bvh->tris, bvh->nodes, bvh->leaf_parent, bvh->node_info,
                                  bvh->flags, bvh->root, ctx->d_error),
                     "k_leaf_climb");
}

template <int Kind, typename Key>
int build_typed(lux_ctx* ctx, lux_bvh* bvh, const float* prims) {
    int n = bvh->n;
    Key* codes = static_cast<Key*>(bvh->codes);
    unsigned* root_ord = reinterpret_cast<unsigned*>(bvh->root + 8);
    // Every reset first, so that the kernels follow one another directly.
    cudaError_t err = cudaMemsetAsync(root_ord, 0xff, 6 * sizeof(unsigned), ctx->stream);
    if (err == cudaSuccess && n == 1)
        // A lone leaf has no parent (the storage may hold a larger earlier tree).
        err = cudaMemsetAsync(bvh->leaf_parent, 0xff, sizeof(int), ctx->stream);
    if (err != cudaSuccess) return cuda_fail(err, "memset root");
    if (int st = reset_sort_scratch<Key>(ctx, n)) return st;
    err = chain_launch(ctx, k_root_reduce<Kind>, stride_grid(ctx, n), kThreads, 0, prims, n,
                       root_ord);
    if (err != cudaSuccess) return cuda_fail(err, "k_root_reduce");
    int st = morton_and_sort<Kind, Key>(ctx, prims, root_ord, codes, bvh->sorted_ids, n);
    if (st) return st;
    if (n > 1) {
        err = chain_launch(ctx, k_karras<Key>, grid_for(n - 1), kThreads, 0, codes, n, bvh->nodes,
                           bvh->node_parent, bvh->leaf_parent, bvh->node_info);
        if (err != cudaSuccess) return cuda_fail(err, "k_karras");
    }
    return climb<Kind>(ctx, bvh, prims);
}

}  // namespace

size_t lbvh_scratch_bytes(int n, int morton_bits) {
    return morton_bits == 63 ? sort_scratch(n, 8, 8).total() : sort_scratch(n, 4, 4).total();
}

int lbvh_alloc(lux_ctx* ctx, lux_bvh* bvh) {
    (void)ctx;
    bvh->capacity = std::max(bvh->capacity, std::max(bvh->n, 1));
    int n = bvh->capacity;
    size_t key = bvh->morton_bits == 63 ? 8 : 4;
    struct Req {
        void** ptr;
        size_t bytes;
    } reqs[] = {
        {reinterpret_cast<void**>(&bvh->nodes), sizeof(BvhNode) * std::max(n - 1, 1)},
        {reinterpret_cast<void**>(&bvh->tris), sizeof(TriRecord) * n},
        {reinterpret_cast<void**>(&bvh->sorted_ids), sizeof(int) * n},
        {reinterpret_cast<void**>(&bvh->leaf_parent), sizeof(int) * n},
        {reinterpret_cast<void**>(&bvh->node_parent), sizeof(int) * std::max(n - 1, 1)},
        {reinterpret_cast<void**>(&bvh->node_info), sizeof(int4) * std::max(n - 1, 1)},
        {reinterpret_cast<void**>(&bvh->flags), sizeof(unsigned) * std::max(n - 1, 1)},
        {&bvh->codes, key * n},
        {reinterpret_cast<void**>(&bvh->root), sizeof(float) * 16},
    };
    for (auto& r : reqs) {
        cudaError_t err = cudaMalloc(r.ptr, r.bytes);
        if (err != cudaSuccess) {
            cudaGetLastError();
            lbvh_free(bvh);
            return fail(LUX_ERR_OUT_OF_MEMORY, "lbvh allocation failed");
        }
    }
    cudaError_t err = cudaMemset(bvh->flags, 0, sizeof(unsigned) * std::max(n - 1, 1));
    if (err == cudaSuccess) err = cudaMemset(bvh->leaf_parent, 0xff, sizeof(int) * n);
    return cuda_fail(err, "lbvh init");
}

void lbvh_free(lux_bvh* bvh) {
    void* ptrs[] = {bvh->nodes, bvh->tris, bvh->sorted_ids, bvh->leaf_parent, bvh->node_parent,
                    bvh->node_info, bvh->flags, bvh->codes, bvh->root, bvh->wide};
    bvh->wide = nullptr;
    bvh->wide_capacity = 0;
    bvh->wide_current = false;
    for (void* p : ptrs) {
        if (p) cudaFree(p);
    }
    bvh->nodes = nullptr;
    bvh->tris = nullptr;
    bvh->sorted_ids = nullptr;
    bvh->leaf_parent = nullptr;
    bvh->node_parent = nullptr;
    bvh->node_info = nullptr;
    bvh->flags = nullptr;
    bvh->codes = nullptr;
    bvh->root = nullptr;
}

int lbvh_build(lux_ctx* ctx, lux_bvh* bvh, const float* prims) {
    bvh->wide_current = false;
    if (bvh->n <= 0) return LUX_OK;
    bool wide = bvh->morton_bits == 63;
    if (bvh->kind == LUX_PRIM_TRIANGLES) {
        return wide ? build_typed<LUX_PRIM_TRIANGLES, unsigned long long>(ctx, bvh, prims)
                    : build_typed<LUX_PRIM_TRIANGLES, unsigned>(ctx, bvh, prims);
    }
    return wide ? build_typed<LUX_PRIM_AABBS, unsigned long long>(ctx, bvh, prims)
                : build_typed<LUX_PRIM_AABBS, unsigned>(ctx, bvh, prims);
}

namespace {

// Triangle records in sorted order from triangles given in input order.
__global__ void k_attach(const float* tris, int n, const int* sorted_ids, TriRecord* out,
                         int* error) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int pid = sorted_ids[k];
    if (pid < 0 || pid >= n) {
        atomicOr(error, kErrLoopBound);
        return;
    }
    f3 v0, v1, v2;
    box3 b;
    load_prim<LUX_PRIM_TRIANGLES>(tris, pid, v0, v1, v2, b);
    TriRecord r;
    r.p0 = make_float4(v0.x, v0.y, v0.z, __int_as_float(pid));
    r.p1 = make_float4(v1.x, v1.y, v1.z, 0.0f);
    r.p2 = make_float4(v2.x, v2.y, v2.z, 0.0f);
    out[k] = r;
}

}  // namespace

int lbvh_attach_triangles(lux_ctx* ctx, lux_bvh* bvh, const float* tris) {
    if (bvh->n <= 0) return LUX_OK;
    k_attach<<<grid_for(bvh->n), kThreads, 0, ctx->stream>>>(tris, bvh->n, bvh->sorted_ids,
                                                              bvh->tris, ctx->d_error);
    ctx->launches += 1;
    return cuda_fail(cudaGetLastError(), "k_attach");
}

int lbvh_refit(lux_ctx* ctx, lux_bvh* bvh, const float* prims) {
    bvh->wide_current = false;
    if (bvh->n <= 0) return LUX_OK;
    return bvh->kind == LUX_PRIM_TRIANGLES ? climb<LUX_PRIM_TRIANGLES>(ctx, bvh, prims)
                                           : climb<LUX_PRIM_AABBS>(ctx, bvh, prims);
}

namespace {

struct WideSlots {
    box3 box[4];
    int ch[4];
    int count;
    LUX_D void add(int handle, const box3& b) {
        if (count >= 4) return;
        box[count] = b;
        ch[count] = handle;
        ++count;
    }
};

// Biased exponent of an axis grid: from 2^e >= extent / 255, raised until the top grid
// point decodes at or above hi.
// Grid of one axis of a wide node whose children span [origin, hi] (the node's box):
// the smallest exponent e (biased into *biased) for which the grid's points k * 2^e,
// k = floor(origin / 2^e) with |k| <= 2^22, reach hi within 255 steps; *c = (k - 2^23) * 2^e
// (exact).  False when no exponent up to 103 does (the node is then left unbounded).
LUX_D bool wide_axis(float origin, float hi, unsigned* biased, float* c) {
    const float extent = sub(hi, origin);
    int e = -126;
    if (extent > 0.0f) {
        int ex;
        frexpf(extent / 255.0f, &ex);
        e = max(ex, -126);
    }
    for (; e <= 103; ++e) {
        const unsigned b = static_cast<unsigned>(e + 127);
        const float scale = wide_scale(b);
        const float inv = wide_scale(254u - b);  // 2^-e, exact for the exponents used
        const float k = floorf(mul(origin, inv));
        if (!(fabsf(k) <= 4194304.0f)) continue;            // 2^22
        const float cc = mul(sub(k, 8388608.0f), scale);    // (k - 2^23) * 2^e, exact
        if (wide_decode(cc, 255u, scale) < hi) continue;
        *biased = b;
        *c = cc;
        return true;
    }
    return false;
}

// Outward-rounded grid coordinates of [lo, hi]: the largest q_lo whose decode is <= lo
// and the smallest q_hi whose decode is >= hi (grid offset c, see wide_axis).
LUX_D void wide_quantize(float c, unsigned biased, float lo, float hi, unsigned& qlo,
                         unsigned& qhi) {
    const float scale = wide_scale(biased);
    const float inv = wide_scale(254u - biased);  // 2^-e, exact for the exponents used
    const float origin = wide_decode(c, 0u, scale);
    const float fa = floorf(mul(sub(lo, origin), inv));
    int a = fa >= 255.0f ? 255 : (fa > 0.0f ? static_cast<int>(fa) : 0);
    while (a > 0 && wide_decode(c, static_cast<unsigned>(a), scale) > lo) --a;
    const float fb = ceilf(mul(sub(hi, origin), inv));
    int b = fb >= 255.0f ? 255 : (fb > 0.0f ? static_cast<int>(fb) : 0);
    while (b < 255 && wide_decode(c, static_cast<unsigned>(b), scale) < hi) ++b;
    qlo = static_cast<unsigned>(a);
    qhi = static_cast<unsigned>(b);
}

// Wide node i from binary node i and its internal children (see WideNode).
__global__ void __launch_bounds__(kThreads) k_widen(const BvhNode* nodes, int n,
                                                    WideNode* wide, int* error) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    WideSlots s;
    s.count = 0;
    BvhNode nd = load_node(nodes, i);
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        int h = side ? nd.ch.y : nd.ch.x;
        if (h >= n - 1) {  // cannot happen for a consistent hierarchy
            atomicOr(error, kErrLoopBound);
            continue;
        }
        if (h >= 0) {
            BvhNode cn = load_node(nodes, h);
            s.add(cn.ch.x, node_left_box(cn));
            s.add(cn.ch.y, node_right_box(cn));
        } else {
            s.add(h, side ? node_right_box(nd) : node_left_box(nd));
        }
    }
    box3 u = box_union(node_left_box(nd), node_right_box(nd));
    float o[3] = {u.lo.x, u.lo.y, u.lo.z};
    float top[3] = {u.hi.x, u.hi.y, u.hi.z};
    bool finite = true;
    for (int a = 0; a < 3; ++a) finite = finite && isfinite(o[a]) && isfinite(top[a]);
    unsigned ebits[3] = {127u, 127u, 127u};
    float cgrid[3] = {0.0f, 0.0f, 0.0f};
    unsigned lo_w[3] = {0, 0, 0}, hi_w[3] = {0, 0, 0};
    for (int a = 0; a < 3 && finite; ++a) finite = wide_axis(o[a], top[a], &ebits[a], &cgrid[a]);
    if (finite) {
        for (int c = 0; c < s.count; ++c) {
            float lo[3] = {s.box[c].lo.x, s.box[c].lo.y, s.box[c].lo.z};
            float hi[3] = {s.box[c].hi.x, s.box[c].hi.y, s.box[c].hi.z};
            for (int a = 0; a < 3; ++a) {
                unsigned ql, qh;
                wide_quantize(cgrid[a], ebits[a], lo[a], hi[a], ql, qh);
                lo_w[a] |= ql << (8 * c);
                hi_w[a] |= qh << (8 * c);
            }
        }
    } else {
        for (int a = 0; a < 3; ++a) {
            ebits[a] = 127u;
            cgrid[a] = 0.0f;
        }
    }
    unsigned meta = ebits[0] | (ebits[1] << 8) | (ebits[2] << 16) |
                    (static_cast<unsigned>(s.count) << 24) | (finite ? 0u : kWideUnbounded);
    int ch[4] = {0, 0, 0, 0};
    for (int c = 0; c < s.count; ++c) ch[c] = s.ch[c];
    WideNode w;
    w.q0 = make_float4(cgrid[0], cgrid[1], cgrid[2], __uint_as_float(meta));
    w.q1 = make_float4(__uint_as_float(lo_w[0]), __uint_as_float(lo_w[1]),
                       __uint_as_float(lo_w[2]), __uint_as_float(hi_w[0]));
    w.q2 = make_float4(__uint_as_float(hi_w[1]), __uint_as_float(hi_w[2]), __int_as_float(ch[0]),
                       __int_as_float(ch[1]));
    w.q3 = make_float4(__int_as_float(ch[2]), __int_as_float(ch[3]), 0.0f, 0.0f);
    wide[i] = w;
}

}  // namespace

int lbvh_ensure_wide(lux_ctx* ctx, lux_bvh* bvh) {
    if (bvh->wide_current || bvh->n <= 1) return LUX_OK;
    int need = std::max(bvh->capacity - 1, 1);
    if (bvh->wide_capacity < need) {
        if (bvh->wide) cudaFree(bvh->wide);
        bvh->wide = nullptr;
        bvh->wide_capacity = 0;
        cudaError_t err = cudaMalloc(&bvh->wide, sizeof(WideNode) * size_t(need));
        if (err != cudaSuccess) {
            cudaGetLastError();
            bvh->wide = nullptr;
            return fail(LUX_ERR_OUT_OF_MEMORY, "wide node allocation failed");
        }
        bvh->wide_capacity = need;
    }
    k_widen<<<grid_for(bvh->n - 1), kThreads, 0, ctx->stream>>>(bvh->nodes, bvh->n, bvh->wide,
                                                                 ctx->d_error);
    ctx->launches += 1;
    int st = cuda_fail(cudaGetLastError(), "k_widen");
    if (!st) bvh->wide_current = true;
    return st;
}

int lbvh_export(lux_ctx* ctx, const lux_bvh* bvh, uint64_t* codes64, int* left, int* right,
                float* bounds) {
    int n = bvh->n;
    if (n <= 0) return LUX_OK;
    int count = 2 * n - 1;
    auto* c64 = reinterpret_cast<unsigned long long*>(codes64);
    if (bvh->morton_bits == 63) {
        k_export<unsigned long long><<<grid_for(count), kThreads, 0, ctx->stream>>>(
            bvh->view(), static_cast<const unsigned long long*>(bvh->codes), c64, left, right,
            bounds);
    } else {
        k_export<unsigned><<<grid_for(count), kThreads, 0, ctx->stream>>>(
            bvh->view(), static_cast<const unsigned*>(bvh->codes), c64, left, right, bounds);
    }
    ctx->launches += 1;
    return cuda_fail(cudaGetLastError(), "k_export");
}

}  // namespace lux

// ---------------------------------------------------------------- no-allocation sort
// lux_lbvh_morton_sort_static keeps every temporary of the Morton sort in this array
// instead of context scratch, so that a call allocates no device memory.  The module
// holds it on every GPU it is loaded on until the process exits.  Layout in bytes:
//   [0, 24)      six ordered-int root words (start at all ones: the identity of min)
//   [64, 68)     device error word (starts at zero)
//   [256, ...)   digit histograms, kRadix x tiles words (fully rewritten every pass)
//   then keys    LUX_STATIC_SORT_MAX_PRIMS x 8 bytes: 63-bit alternate keys, or both
//                30-bit key buffers
//   then values  LUX_STATIC_SORT_MAX_PRIMS x 4 bytes: alternate primitive ids
namespace lux {
namespace {

constexpr int kStaticMaxPrims = LUX_STATIC_SORT_MAX_PRIMS;
constexpr int kStaticMaxTiles = (kStaticMaxPrims + kStaticTile - 1) / kStaticTile;
constexpr size_t kStaticHeaderBytes = 256;
constexpr size_t kStaticHistBytes = size_t(kRadix) * kStaticMaxTiles * sizeof(unsigned);
constexpr size_t kStaticKeyBytes = size_t(kStaticMaxPrims) * 8;
constexpr size_t kStaticValBytes = size_t(kStaticMaxPrims) * 4;
constexpr size_t kStaticBytes = kStaticHeaderBytes + kStaticHistBytes + kStaticKeyBytes +
                                kStaticValBytes;
static_assert(kStaticBytes == LUX_STATIC_SORT_SCRATCH_BYTES, "static sort array size");
static_assert(kStaticHistBytes % 256 == 0 && kStaticKeyBytes % 256 == 0, "region alignment");
constexpr int kMaxDevices = 64;

}  // namespace
}  // namespace lux

static __device__ __align__(256) unsigned char lux_static_sort_scratch[lux::kStaticBytes];

namespace lux {
namespace {

// Device address of the array on `device`, which must be current.  Looked up once per
// device (the first call on it), then reused.
int static_sort_scratch(int device, unsigned char** out) {
    static std::mutex mu;
    static unsigned char* address[kMaxDevices] = {};
    if (device < 0 || device >= kMaxDevices)
        return fail(LUX_ERR_INVALID_ARGUMENT, "device ordinal out of range for the static sort");
    std::lock_guard<std::mutex> lk(mu);
    if (!address[device]) {
        void* p = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&p, lux_static_sort_scratch);
        if (err != cudaSuccess) return cuda_fail(err, "cudaGetSymbolAddress(static sort array)");
        address[device] = static_cast<unsigned char*>(p);
    }
    *out = address[device];
    return LUX_OK;
}

__global__ void k_widen_codes(const unsigned* codes, int n, unsigned long long* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = codes[i];
}

// Root box, Morton codes and the LSD sort over explicit buffers: the even pass count
// leaves the result in (keys, vals).
template <int Kind, typename Key>
int morton_sort_into(lux_ctx* ctx, const float* prims, int n, Key* keys, Key* keys_alt,
                     int* vals, int* vals_alt, unsigned* hist, unsigned* root_ord, int* error) {
    cudaStream_t stream = ctx->stream;
    k_root_reduce<Kind><<<stride_grid(ctx, n), kThreads, 0, stream>>>(prims, n, root_ord);
    k_morton<Kind, Key><<<stride_grid(ctx, n), kThreads, 0, stream>>>(prims, n, root_ord, keys);
    ctx->launches += 2;
    const int tiles = grid_for(n, kStaticTile);
    int passes = (sizeof(Key) == 4 ? 30 + 7 : 63 + 7) / 8;
    if (passes & 1) ++passes;
    Key* kin = keys;
    Key* kout = keys_alt;
    int* vin = vals;
    int* vout = vals_alt;
    for (int p = 0; p < passes; ++p) {
        int shift = 8 * p;
        k_sort_upsweep<Key><<<tiles, kThreads, 0, stream>>>(kin, n, shift, hist, tiles);
        k_scan_exclusive<<<1, kScanThreads, 0, stream>>>(hist, kRadix * tiles);
        if (p == 0) {
            k_sort_downsweep<Key, true><<<tiles, kThreads, 0, stream>>>(
                kin, vin, kout, vout, n, shift, hist, tiles, error);
        } else {
            k_sort_downsweep<Key, false><<<tiles, kThreads, 0, stream>>>(
                kin, vin, kout, vout, n, shift, hist, tiles, error);
        }
        ctx->launches += 3;
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    return cuda_fail(cudaGetLastError(), "static morton sort");
}

}  // namespace

int lbvh_morton_sort_static(lux_ctx* ctx, const float* prims, int n, int kind, int morton_bits,
                            uint64_t* sorted_codes, int* sorted_ids) {
    if (n < 0 || n > kStaticMaxPrims)
        return fail(LUX_ERR_INVALID_ARGUMENT,
                    "static morton sort: n = " + std::to_string(n) + " is outside 0.." +
                        std::to_string(kStaticMaxPrims) + " (the static array's limit)");
    unsigned char* base = nullptr;
    if (int st = static_sort_scratch(ctx->device, &base)) return st;
    if (n == 0) return LUX_OK;
    unsigned* root_ord = reinterpret_cast<unsigned*>(base);
    int* error = reinterpret_cast<int*>(base + 64);
    unsigned* hist = reinterpret_cast<unsigned*>(base + kStaticHeaderBytes);
    unsigned char* keys = base + kStaticHeaderBytes + kStaticHistBytes;
    int* vals_alt = reinterpret_cast<int*>(keys + kStaticKeyBytes);
    auto* codes64 = reinterpret_cast<unsigned long long*>(sorted_codes);
    cudaStream_t stream = ctx->stream;
    // The array keeps the previous call's contents: reset the words that must start at a
    // fixed value.  Histograms, keys and values are fully written before they are read.
    cudaError_t err = cudaMemsetAsync(root_ord, 0xff, 6 * sizeof(unsigned), stream);
    if (err == cudaSuccess) err = cudaMemsetAsync(error, 0, sizeof(int), stream);
    if (err != cudaSuccess) return cuda_fail(err, "static sort reset");
    int st;
    if (morton_bits == 63) {
        auto* alt = reinterpret_cast<unsigned long long*>(keys);
        st = kind == LUX_PRIM_TRIANGLES
                 ? morton_sort_into<LUX_PRIM_TRIANGLES>(ctx, prims, n, codes64, alt, sorted_ids,
                                                        vals_alt, hist, root_ord, error)
                 : morton_sort_into<LUX_PRIM_AABBS>(ctx, prims, n, codes64, alt, sorted_ids,
                                                    vals_alt, hist, root_ord, error);
    } else {
        auto* k30 = reinterpret_cast<unsigned*>(keys);
        auto* alt = k30 + kStaticMaxPrims;
        st = kind == LUX_PRIM_TRIANGLES
                 ? morton_sort_into<LUX_PRIM_TRIANGLES>(ctx, prims, n, k30, alt, sorted_ids,
                                                        vals_alt, hist, root_ord, error)
                 : morton_sort_into<LUX_PRIM_AABBS>(ctx, prims, n, k30, alt, sorted_ids,
                                                    vals_alt, hist, root_ord, error);
        if (!st) {
            k_widen_codes<<<stride_grid(ctx, n), kThreads, 0, stream>>>(k30, n, codes64);
            ctx->launches += 1;
            st = cuda_fail(cudaGetLastError(), "k_widen_codes");
        }
    }
    if (st) return st;
    err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) return cuda_fail(err, "static morton sort");
    int word = 0;
    err = cudaMemcpy(&word, error, sizeof(int), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return cuda_fail(err, "static sort error word");
    if (word) return fail(LUX_ERR_DEVICE_CHECK, "static morton sort: device check failed");
    return LUX_OK;
}

}  // namespace lux
