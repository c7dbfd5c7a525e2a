// Tiled greedy cosine for sm_100a: cms_cosine_greedy / cms_cosine_greedy_sparse.
//
// Replaces the reference's per-pair Numba kernel (cudams/similarity/
// spectrum_similarity_functions.py:39-262) and the batch loop around it
// (cudams/similarity/CudaCosineGreedy.py:138-226).  Results are identical to
// the plain kernel and to the oracle; only the way candidates are found and
// ordered differs.
//
// Pipeline of one call (all on one stream, no host synchronisation):
//   1. validate_kernel   offsets sane, spectra <= CMS_MAX_PEAKS; else every
//                        later kernel exits at once and the error word is set
//   2. norms_kernel      sqrt(sum (a*b)^2) per spectrum, sequential float64
//   3. order kernels     reference spectra ordered by peak count, largest
//                        first (log2 length classes), for load balance
//   4. index kernels     query spectra are cut into tiles of tile_spectra;
//                        each tile's peaks are bucketed by m/z (bucket width
//                        tol by default, buckets hashed modulo n_buckets) into a
//                        CSR "tile stream" of (m/z, query<<16 | peak)
//   5. join_kernel       persistent warps; one work item = (reference
//                        spectrum, query tile).  Lanes take reference peaks,
//                        jump through the bucket table to the tile-stream
//                        entries inside the tolerance window (the
//                        two-pointer sweep of the reference, with the second
//                        pointer advanced by the index instead of one step at
//                        a time), test them with exact float32 window bounds
//                        and push candidates into a per-warp pool (shared
//                        memory, extended in global memory).  The pool is
//                        counting-sorted by query; each query's run is then
//                        resolved greedily: 1-3 candidates in closed form by
//                        one lane, 4-8 by an 8-lane segment, 9-32 by the warp.
//                        The sweep is load-balanced: a chunk's window entries
//                        are expanded 32 at a time over the warp, and each
//                        query's candidates are chained through a per-warp
//                        head table (tagged by an epoch, so it is rarely
//                        cleared) instead of being counting-sorted.
//                        The dense row segment is zeroed with coalesced
//                        stores just before, and each run stores its result
//                        over its zeros.  Pairs with longer runs (or >=
//                        match_limit candidates) go to a spill list.
//   6. pair_kernel       one CTA per spilled pair (or per pair of the whole
//                        matrix in mode 2): exact generation-order sweep with
//                        match_limit truncation, bitonic sort of (key, gen)
//                        (in registers when there are eight candidates a
//                        thread, else in shared memory), warp greedy with
//                        per-chunk conflict masks and used-peak bitmasks.
//   7. mirror_kernel     (symmetric dense calls, csrc/mirror.cu) lower
//                        triangle copied from the upper one.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "cms_internal.cuh"

namespace cms {
namespace {

constexpr int kJoinWarps = 8;
constexpr int kJoinThreads = kJoinWarps * 32;
constexpr int kPool = 256;        // candidate pool entries per warp
constexpr int kLongRun = 32;      // longer runs go to the pair kernel
constexpr int kMidRun = 8;        // runs up to this length are resolved four per warp step
constexpr int kMaxTile = 4096;    // max query spectra per tile
constexpr int kOrderClasses = 17; // log2 length classes (0..16)
constexpr int kModifiedMaxPeaks = 32767;  // modified cosine: reference peak index in 15 bits

__device__ __forceinline__ double peak_a(const double* a, int64_t i) { return a ? a[i] : 1.0; }

// ---------------------------------------------------------------------------
// 1. validation
// ---------------------------------------------------------------------------
__global__ void validate_kernel(SpecSet S, uint32_t* bad, uint32_t* err,
                                int max_peaks = CMS_MAX_PEAKS) {
    const int64_t n = S.n;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t lo = S.off[s], hi = S.off[s + 1];
        uint32_t e = 0;
        if (lo < 0 || hi < lo || hi > S.n_peaks) e |= kErrBadOffsets;
        if (hi - lo > max_peaks) e |= kErrSpectrumTooLong;
        if (e) {
            atomicOr(err, e);
            atomicOr(bad, 1u);
        }
    }
}

// ---------------------------------------------------------------------------
// 2. norms: sn[s] = sqrt(sum_k (a_k*b_k)^2), summed in peak order
// ---------------------------------------------------------------------------
__global__ void norms_kernel(SpecSet S, double* sn, const uint32_t* bad) {
    if (*bad) return;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < S.n;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t lo = S.off[s], hi = S.off[s + 1];
        double acc = 0.0;
        for (int64_t k = lo; k < hi; ++k) {
            const double w = __dmul_rn(peak_a(S.a, k), S.b[k]);
            acc = __dadd_rn(acc, __dmul_rn(w, w));
        }
        sn[s] = sqrt(acc);
    }
}

// ---------------------------------------------------------------------------
// 3. reference order: largest length class first
// ---------------------------------------------------------------------------
__device__ __forceinline__ int length_class(int64_t len) {
    return len <= 0 ? 0 : min(kOrderClasses - 1, 64 - __clzll((unsigned long long)len));
}

__global__ void order_count_kernel(SpecSet S, uint32_t* cls_count, const uint32_t* bad) {
    if (*bad) return;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < S.n;
         s += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&cls_count[length_class(S.off[s + 1] - S.off[s])], 1u);
}

__global__ void order_scatter_kernel(SpecSet S, const uint32_t* cls_count, uint32_t* cls_cursor,
                                     int32_t* order, const uint32_t* bad) {
    if (*bad) return;
    __shared__ uint32_t base[kOrderClasses];
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int c = kOrderClasses - 1; c >= 0; --c) {
            base[c] = acc;
            acc += cls_count[c];
        }
    }
    __syncthreads();
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < S.n;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int c = length_class(S.off[s + 1] - S.off[s]);
        const uint32_t pos = base[c] + atomicAdd(&cls_cursor[c], 1u);
        order[pos] = (int32_t)s;
    }
}

// ---------------------------------------------------------------------------
// 4. tile index over the query side
// ---------------------------------------------------------------------------
// tile-stream entry: m/z, (query within tile << 16 | peak), intensity weight b
struct __align__(16) Entry {
    float mz;
    uint32_t id;
    double b;
};

struct IndexGeom {
    int tile;        // query spectra per tile
    int n_tiles;
    int nb;          // buckets per tile (power of two)
    double inv_w;    // 1 / bucket width
};

// Bucket of an m/z value: floor(mz / width), hashed modulo nb by the caller.
// Monotone non-decreasing in mz (one float64 multiply, then round down), so
// every entry inside [L, H] falls in a bucket of [bucket_of(L), bucket_of(H)].
// (float64 keeps one bucket per width even when mz / width exceeds 2^24.)
__device__ __forceinline__ long long bucket_of(float x, double inv_w) {
    return __double2ll_rd(__dmul_rn((double)x, inv_w));
}

// The value an index sorts a peak by: its m/z, or for the neutral-loss index
// of modified cosine (NL) its m/z minus its spectrum's precursor m/z, computed
// in float64 and rounded to float32 (the join widens its windows by a margin
// that covers this rounding and confirms each candidate exactly).
template <bool NL>
__device__ __forceinline__ float index_value(const SpecSet& B, int64_t s, int64_t k) {
    if (!NL) return B.mz[k];
    return __double2float_rn(__dsub_rn((double)B.mz[k], B.prec[s]));
}

// warp per spectrum: histogram of (tile, bucket)
template <bool NL>
__global__ void index_count_kernel(SpecSet B, IndexGeom g, uint32_t* cnt, const uint32_t* bad) {
    if (*bad) return;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const unsigned mask = (unsigned)(g.nb - 1);
    for (int64_t s = warp; s < B.n; s += nwarps) {
        const int64_t t = s / g.tile;
        const int64_t lo = B.off[s], hi = B.off[s + 1];
        uint32_t* c = cnt + t * (int64_t)g.nb;
        for (int64_t k = lo + lane; k < hi; k += 32) {
            const unsigned bk = (unsigned)bucket_of(index_value<NL>(B, s, k), g.inv_w) & mask;
            atomicAdd(&c[bk], 1u);
        }
    }
}

// CTA per tile: exclusive scan of the bucket counts into tab[t][0..nb], and
// reset the counters to the bucket starts (scatter cursors).
__global__ void index_scan_kernel(IndexGeom g, uint32_t* cnt_cur, uint32_t* tab,
                                  const uint32_t* bad) {
    if (*bad) return;
    const int t = blockIdx.x;
    uint32_t* c = cnt_cur + (int64_t)t * g.nb;
    uint32_t* out = tab + (int64_t)t * (g.nb + 1);
    const int per = (g.nb + blockDim.x - 1) / blockDim.x;
    const int begin = min(g.nb, (int)threadIdx.x * per);
    const int end = min(g.nb, begin + per);
    uint32_t local = 0;
    for (int k = begin; k < end; ++k) local += c[k];
    // block exclusive scan of `local`
    __shared__ uint32_t warp_sums[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = local;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t v = lane < nw ? warp_sums[lane] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, v, d);
            if (lane >= d) v += u;
        }
        if (lane < nw) warp_sums[lane] = v;
    }
    __syncthreads();
    uint32_t run = incl - local + (wid > 0 ? warp_sums[wid - 1] : 0u);
    for (int k = begin; k < end; ++k) {
        const uint32_t v = c[k];
        out[k] = run;
        c[k] = run;
        run += v;
    }
    if (threadIdx.x == blockDim.x - 1) out[g.nb] = run;
}

// warp per spectrum: scatter (value, q_local<<16 | peak) into the tile stream
template <bool NL>
__global__ void index_scatter_kernel(SpecSet B, IndexGeom g, uint32_t* cur, Entry* ent,
                                     const uint32_t* bad) {
    if (*bad) return;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const unsigned mask = (unsigned)(g.nb - 1);
    for (int64_t s = warp; s < B.n; s += nwarps) {
        const int64_t t = s / g.tile;
        const int64_t base = B.off[t * g.tile];
        const uint32_t ql = (uint32_t)(s - t * g.tile);
        const int64_t lo = B.off[s], hi = B.off[s + 1];
        uint32_t* c = cur + t * (int64_t)g.nb;
        for (int64_t k = lo + lane; k < hi; k += 32) {
            const float mz = index_value<NL>(B, s, k);
            const unsigned bk = (unsigned)bucket_of(mz, g.inv_w) & mask;
            const uint32_t pos = atomicAdd(&c[bk], 1u);
            Entry en;
            en.mz = mz;
            en.id = (ql << 16) | (uint32_t)(k - lo);
            en.b = B.b[k];
            ent[base + pos] = en;
        }
    }
}

// ---------------------------------------------------------------------------
// shared helpers for greedy resolution
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long order_key(double k) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(k);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double key_from_order(unsigned long long o) {
    const unsigned long long u = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
    return __longlong_as_double((long long)u);
}
// (key, gen) strictly precedes (key', gen') in the greedy order
__device__ __forceinline__ bool before(double k1, uint32_t g1, double k2, uint32_t g2) {
    return k1 > k2 || (k1 == k2 && g1 > g2);
}

__device__ __forceinline__ void emit_hit(const SparseOut& o, int r, int q, float sc, int mt,
                                         uint8_t ovf) {
    const bool both = o.mirror && r != q;
    const unsigned long long pos = atomicAdd(o.count, both ? 2ull : 1ull);
    if (pos < (unsigned long long)o.capacity) {
        o.r[pos] = r;
        o.q[pos] = q;
        o.score[pos] = sc;
        o.matches[pos] = mt;
        o.overflow[pos] = ovf;
    }
    if (both && pos + 1 < (unsigned long long)o.capacity) {
        o.r[pos + 1] = q;
        o.q[pos + 1] = r;
        o.score[pos + 1] = sc;
        o.matches[pos + 1] = mt;
        o.overflow[pos + 1] = ovf;
    }
}

// Optional per-work-item timing records (cms_trace_enable): 4 words each --
// tag | smid << 32, item index, %globaltimer at its start and end (ns).
struct TraceOut {
    unsigned long long* rec;
    unsigned long long* count;
    long long cap;
    unsigned int tag;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct SpillList {
    int2* pairs;  // (reference, query)
    unsigned int* count;
    unsigned int cap;
};

__device__ __forceinline__ void spill_push(const SpillList& sl, int r, int q, uint32_t* err) {
    const unsigned int pos = atomicAdd(sl.count, 1u);
    if (pos < sl.cap)
        sl.pairs[pos] = make_int2(r, q);
    else
        atomicOr(err, kErrSpillOverrun);
}

// ---------------------------------------------------------------------------
// 5. join kernel
// ---------------------------------------------------------------------------
struct JoinParams {
    SpecSet A;  // sweeping side (one spectrum per work item)
    SpecSet B;  // indexed side (tiles)
    const double* snA;
    const double* snB;
    const int32_t* a_order;
    const uint32_t* tab;
    const Entry* ent;
    const uint32_t* tab2;  // modified cosine: neutral-loss index (m/z - precursor)
    const Entry* ent2;
    IndexGeom g;
    double tol;
    double shift;
    int match_limit;
    float init_width_scale;  // first sub-range width = scale / n_A_peaks (0: whole tile)
    // first sub-range width per length class of the sweeping spectrum (the
    // tuner's measured candidate-pool split); 0: init_width_scale decides
    int width_by_class[kOrderClasses];
    int warp_smem_bytes;     // per-warp slice of dynamic shared memory
    int pool_max;            // candidates a sweep may hold: kPoolMax, or kPool without gpool
    int max_fetch;           // fetches of kFetch items per warp before it exits (0: no limit)
    unsigned char* gpool;    // global pool extension, kGPool * 16 bytes per warp (or null)
    // bounded launches: a CTA claims one of n_slots global-pool slices (a bit
    // of `slots`) for its lifetime instead of using slice blockIdx.x (null:
    // slice blockIdx.x, persistent launches)
    unsigned int* slots;
    int n_slots;
    TraceOut trace;          // per-item timing records (rec null: off)
    unsigned long long* work;
    SpillList spill;
    DenseOut dense;
    SparseOut sparse;
    uint32_t* err;
    const uint32_t* bad;
    int sym;  // only pairs (reference i, query j) with i <= j
};

constexpr int kFetch = 2;                  // work items taken per atomic (2: 0.8% faster than 4)
// rounds of 32 tile-stream entries a warp loads before testing the first (1
// measured fastest at 100k x 100k: 42.8 ms against 43.3 for 2 and 46.6 for 3,
// each extra round costing registers and spills)
constexpr int kRounds = 1;
constexpr int kSearchWaves = 4;            // waves of short-lived CTAs per library search
constexpr int kSlotWords = 64;             // slot bitmap words of a bounded join launch
constexpr int kPoolMax = 4096;             // candidates per sweep: smem pool + global extension
constexpr int kGPool = kPoolMax - kPool;   // global extension entries per warp
static_assert(kPoolMax <= 4096, "pool slots are packed into 12 bits");
static_assert(kMaxTile <= 4096, "query indices within a range are packed into 12 bits");

// Candidate metadata word: the query's index within the swept range (bits
// 0-11) and the slot of the previous candidate of the same query (bits 12-23,
// present when kHasNext is set).  A query's candidates form a chain that
// starts at the slot its head names (the candidate pushed last).
constexpr uint32_t kHasNext = 1u << 24;
__device__ __forceinline__ int meta_query(uint32_t m) { return (int)(m & 0xFFFu); }
__device__ __forceinline__ int meta_next(uint32_t m) { return (int)((m >> 12) & 0xFFFu); }

// A warp's candidate pool: the first kPool entries live in shared memory, the
// rest in a per-warp slice of global scratch (L2-resident), so that a large
// reference spectrum is swept once even when it has thousands of candidates
// in a tile.  Slots are indices into the concatenation.
struct Pool {
    double* skey;
    uint32_t* sgen;
    uint32_t* smeta;
    double* gkey;
    uint32_t* ggen;
    uint32_t* gmeta;
    __device__ __forceinline__ double key(int i) const { return i < kPool ? skey[i] : gkey[i - kPool]; }
    __device__ __forceinline__ uint32_t gen(int i) const { return i < kPool ? sgen[i] : ggen[i - kPool]; }
    __device__ __forceinline__ uint32_t meta(int i) const {
        return i < kPool ? smeta[i] : gmeta[i - kPool];
    }
    __device__ __forceinline__ void put(int i, double k, uint32_t g, uint32_t m) const {
        if (i < kPool) {
            skey[i] = k;
            sgen[i] = g;
            smeta[i] = m;
        } else {
            gkey[i - kPool] = k;
            ggen[i - kPool] = g;
            gmeta[i - kPool] = m;
        }
    }
};

// Per-warp shared-memory slice (offsets in bytes; the head table's length
// depends on the tile size, so the slice size is computed at launch).
//   key   double [kPool]     candidate key
//   gen   uint32 [kPool]     (p_ref << 16) | p_query
//   meta  uint32 [kPool]     query in range | previous candidate of the query
//   head  uint32 [tile/2]    two 16-bit heads per word, one per query of the
//                            range: (epoch << 12) | slot of its last candidate;
//                            a head of another epoch means "no candidate yet"
//   wa    double [32]        per-lane sweeping-peak weight of the current chunk
//   lh    float2 [32]        per-lane float32 window [L, H] of the current chunk
//   runs  uint32 [kLongRuns] runs of 4..32 candidates queued for the warp:
//                            slot of the chain head | length << 12; runs of at
//                            most kMidRun from the front, longer ones from the back
//   x     float  [32]        per-lane sweeping-peak m/z (modified cosine's exact test)
//   t0    uint64             %globaltimer at the current item's start (trace only)
constexpr int kLongRuns = 64;
__host__ __device__ constexpr int head_words(int tile) { return (((tile + 1) / 2) + 3) & ~3; }
__host__ __device__ constexpr int warp_slice_bytes(int tile) {
    return 16 * kPool + 4 * head_words(tile) + 8 * 32 + 8 * 32 + 4 * kLongRuns + 4 * 32 + 16;
}

// Reference peak of a candidate's generation word.  Modified cosine marks
// candidates of its second (precursor-shifted) pass in bit 31, which makes
// them later in generation order than every unshifted one (the order of
// matchms' concatenation) and limits its spectra to 32767 peaks.
template <bool MODIFIED>
__device__ __forceinline__ uint32_t gen_p1(uint32_t g) {
    return MODIFIED ? ((g >> 16) & 0x7FFFu) : (g >> 16);
}

// Neutral-loss window of modified cosine's shifted pass: entries whose
// m/z - precursor lies within tol of the sweeping peak's, widened by twice
// the float32 spacing there (the stored values are rounded to float32) and a
// float64 rounding allowance, rounded outwards; every entry inside is then
// confirmed with the exact test of the shifted window.
__device__ __forceinline__ bool nl_window(float mz, double prec, double tol, float& L, float& H) {
    const double zr = __dsub_rn((double)mz, prec);
    const float mag = __double2float_ru(fabs(zr) + tol + 1.0);
    const double m = 2.0 * (double)(nextafterf(mag, INFINITY) - mag) +
                     1e-9 * (fabs((double)mz) + fabs(prec) + 1.0);
    L = __double2float_rd(__dsub_rn(__dsub_rn(zr, tol), m));
    H = __double2float_ru(__dadd_rn(__dadd_rn(zr, tol), m));
    return isfinite(L) && isfinite(H);
}

// Exact float32 window of one sweeping peak.
//
// The float64 test of the reference (query peak y matches reference peak x iff
// !(y+shift > x+tol) && !(y+shift < x-tol)) is, for a fixed sweeping peak, a
// conjunction of a predicate non-decreasing in the indexed peak's m/z and one
// non-increasing in it.  So the float32 values it accepts form one interval
// [L, H] of float32 numbers.  It is found once per sweeping peak by rounding
// an estimate and stepping with nextafterf until the float64 predicates flip;
// each entry is then tested with two float32 compares, with exactly the same
// outcome as the float64 test.  The estimate is within an ulp or two; the
// step loops are capped, and a peak that does not converge (non-finite input)
// gets an empty window and an error flag.
template <bool A_IS_REF, bool NOSHIFT>
struct Window {
    // A_IS_REF: x = sweeping reference peak; lo/hi = x -+ tol
    // else:     c = sweeping query peak + shift
    __device__ __forceinline__ static bool not_below(float y, double lo, double c, double tol,
                                                     double shift) {
        if (A_IS_REF) return !(__dadd_rn((double)y, shift) < lo);
        return !(c > __dadd_rn((double)y, tol));
    }
    __device__ __forceinline__ static bool not_above(float y, double hi, double c, double tol,
                                                     double shift) {
        if (A_IS_REF) return !(__dadd_rn((double)y, shift) > hi);
        return !(c < __dsub_rn((double)y, tol));
    }
    __device__ static bool bounds(float mzA, double tol, double shift, float& L, float& H) {
        const double x = (double)mzA;
        if (A_IS_REF && NOSHIFT) {
            // y (float32, exact in float64) is accepted iff lo <= y <= hi: the
            // interval ends are lo rounded up and hi rounded down to float32
            L = __double2float_ru(__dsub_rn(x, tol));
            H = __double2float_rd(__dadd_rn(x, tol));
            return isfinite(L) && isfinite(H);
        }
        double lo = 0.0, hi = 0.0, c = 0.0, el, eh;
        if (A_IS_REF) {
            lo = __dsub_rn(x, tol);
            hi = __dadd_rn(x, tol);
            el = __dsub_rn(lo, shift);
            eh = __dsub_rn(hi, shift);
        } else {
            c = __dadd_rn(x, shift);
            el = __dsub_rn(c, tol);
            eh = __dadd_rn(c, tol);
        }
        float l = __double2float_rd(el), h = __double2float_ru(eh);
        int k = 0;
        for (; k < 16 && !not_below(l, lo, c, tol, shift); ++k) l = nextafterf(l, INFINITY);
        for (; k < 32 && not_below(nextafterf(l, -INFINITY), lo, c, tol, shift); ++k)
            l = nextafterf(l, -INFINITY);
        for (; k < 48 && !not_above(h, hi, c, tol, shift); ++k) h = nextafterf(h, -INFINITY);
        for (; k < 64 && not_above(nextafterf(h, INFINITY), hi, c, tol, shift); ++k)
            h = nextafterf(h, INFINITY);
        const bool ok = k < 64 && isfinite(l) && isfinite(h) && not_below(l, lo, c, tol, shift) &&
                        not_above(h, hi, c, tol, shift);
        L = l;
        H = h;
        return ok;
    }
};

// Three CTAs (24 warps) per SM: up to 85 registers a thread.
template <bool A_IS_REF, bool SPARSE, bool NOSHIFT, bool MODIFIED>
__global__ void __launch_bounds__(kJoinThreads, 3)
join_kernel(JoinParams P) {
    if (*P.bad) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int hw = head_words(P.g.tile);
    unsigned char* slice = smem_raw + (size_t)(threadIdx.x >> 5) * P.warp_smem_bytes;
    uint32_t* head = reinterpret_cast<uint32_t*>(slice + 16 * kPool);
    double* s_wa = reinterpret_cast<double*>(slice + 16 * kPool + 4 * hw);
    float2* s_lh = reinterpret_cast<float2*>(slice + 16 * kPool + 4 * hw + 8 * 32);
    uint32_t* long_runs = reinterpret_cast<uint32_t*>(slice + 16 * kPool + 4 * hw + 16 * 32);
    float* s_x = reinterpret_cast<float*>(slice + 16 * kPool + 4 * hw + 16 * 32 + 4 * kLongRuns);
    unsigned long long* s_t0 = reinterpret_cast<unsigned long long*>(
        slice + 16 * kPool + 4 * hw + 16 * 32 + 4 * kLongRuns + 4 * 32);
    // Global-pool slice of this CTA: blockIdx.x, or under bounded launches a
    // slice claimed from the slot bitmap (at most n_slots CTAs are resident at
    // once, so one is free; if a release has not landed yet the CTA runs with
    // the shared-memory pool only).  Every search is bounded by 2 passes over
    // the words and 32 attempts per word.
    __shared__ int s_slot;
    int pslot = (int)blockIdx.x;
    if (P.slots) {
        if (threadIdx.x == 0) {
            int got = -1;
            const int words = (P.n_slots + 31) >> 5;
            for (int i = 0; i < 2 * words && got < 0; ++i) {
                const int w = (int)((blockIdx.x + (unsigned)i) % (unsigned)words);
                const int nb = min(32, P.n_slots - 32 * w);
                const unsigned valid = nb >= 32 ? 0xffffffffu : ((1u << nb) - 1u);
                unsigned cur = atomicOr(&P.slots[w], 0u);
                for (int k = 0; k < 32 && got < 0; ++k) {
                    const unsigned freeb = ~cur & valid;
                    if (!freeb) break;
                    const unsigned bit = freeb & (0u - freeb);
                    const unsigned old = atomicOr(&P.slots[w], bit);
                    if (!(old & bit))
                        got = 32 * w + (__ffs(bit) - 1);
                    else
                        cur = old | bit;
                }
            }
            s_slot = got;
        }
        __syncthreads();
        pslot = s_slot;
    }
    const int pool_max = (P.gpool && pslot >= 0) ? P.pool_max : kPool;
    Pool pool;
    {
        const size_t gw = (size_t)(pslot >= 0 ? pslot : 0) * kJoinWarps + (threadIdx.x >> 5);
        unsigned char* g = (P.gpool && pslot >= 0) ? P.gpool + gw * (size_t)kGPool * 16 : nullptr;
        pool.skey = reinterpret_cast<double*>(slice);
        pool.sgen = reinterpret_cast<uint32_t*>(slice + 8 * kPool);
        pool.smeta = reinterpret_cast<uint32_t*>(slice + 12 * kPool);
        pool.gkey = reinterpret_cast<double*>(g);
        pool.ggen = reinterpret_cast<uint32_t*>(g ? g + 8 * kGPool : nullptr);
        pool.gmeta = reinterpret_cast<uint32_t*>(g ? g + 12 * kGPool : nullptr);
    }

    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const unsigned below = (1u << lane) - 1u;
    const int64_t nA = P.A.n;
    const int64_t n_items = nA * (int64_t)P.g.n_tiles;
    const unsigned nbmask = (unsigned)(P.g.nb - 1);
    const Entry* __restrict__ ent = P.ent;
    const uint32_t* __restrict__ tab = P.tab;
    // epoch of the head table (1..15): every swept range takes the next one,
    // so heads left by earlier ranges read as empty without clearing the
    // table; it is cleared once per 15 ranges (and before the first)
    unsigned epoch = 15;

    for (int fetches = 0; P.max_fetch == 0 || fetches < P.max_fetch; ++fetches) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(P.work, (unsigned long long)kFetch);
        base = __shfl_sync(full, base, 0);
        if ((int64_t)base >= n_items) break;
        // item = t * nA + ai: one division per fetch, then step ai
        int64_t tt = (int64_t)base / nA, ai = (int64_t)base - tt * nA;
        for (int f = 0; f < kFetch && (int64_t)(base + f) < n_items; ++f, ++ai) {
        while (ai >= nA) {
            ai -= nA;
            ++tt;
        }
        if (P.trace.rec && lane == 0) *s_t0 = global_ns();
        const int t = (int)tt;
        const int a = P.a_order[ai];
        const int64_t a0 = P.A.off[a];
        const int na = (int)(P.A.off[a + 1] - a0);
        const int b_begin = t * P.g.tile;
        const int tn = (int)min((int64_t)P.g.tile, P.B.n - b_begin);
        const int64_t tbase = P.B.off[b_begin];
        const uint32_t* T = tab + (int64_t)t * (P.g.nb + 1);
        const uint32_t* T2 = MODIFIED ? P.tab2 + (int64_t)t * (P.g.nb + 1) : nullptr;
        const double snA = P.snA[a];
        // a resolved run's result, stored straight into the dense output
        auto put_dense = [&](int bq, float sc, int mt) {
            const int64_t o = (int64_t)(A_IS_REF ? a : bq) * P.dense.ld + (A_IS_REF ? bq : a);
            __stcs(&P.dense.score[o], sc);
            __stcs(&P.dense.matches[o], mt);
        };
        auto store_result_n = [&](int bq, double score, int mt, double snB) {
            const float sc =
                (float)__ddiv_rn(score, A_IS_REF ? __dmul_rn(snA, snB) : __dmul_rn(snB, snA));
            if (SPARSE) {
                if (sc >= P.sparse.threshold)
                    emit_hit(P.sparse, A_IS_REF ? a : bq, A_IS_REF ? bq : a, sc, mt, 0);
            } else {
                put_dense(bq, sc, mt);
            }
        };
        auto store_result = [&](int bq, double score, int mt) {
            store_result_n(bq, score, mt, P.snB[bq]);
        };

        int width = tn;
        const int wc = P.width_by_class[length_class(na)];
        if (wc > 0)
            width = max(1, min(tn, wc));
        else if (P.init_width_scale > 0.f && na > 0)  // multiples of 32 keep row writes aligned
            width = max(32, min(tn, (int)(P.init_width_scale / (float)na) & ~31));
        // queries of this item: the whole tile, or under `sym` those on or
        // above the diagonal (reference index <= query index)
        int range_lo = 0, q_end = tn;
        if (P.sym) {
            if (A_IS_REF)
                range_lo = max(0, min(tn, a - b_begin));
            else
                q_end = max(0, min(tn, a - b_begin + 1));
        }
        while (range_lo < q_end) {
            const int range_hi = min(range_lo + width, q_end);
            const int rw = range_hi - range_lo;
            epoch = epoch == 15 ? 1u : epoch + 1u;
            if (epoch == 1u)
                for (int w = 4 * lane; w < hw; w += 128)
                    *reinterpret_cast<uint4*>(head + w) = make_uint4(0u, 0u, 0u, 0u);
            __syncwarp();
            // ---- sweep: candidates of (a, queries [range_lo, range_hi)) ----
            // Each lane takes one sweeping peak of a 32-peak chunk and finds
            // the tile-stream entries of its window's buckets (one run, or two
            // when the hashed bucket range wraps).  The chunk's entries are
            // then processed 32 at a time, flat entry k by lane k % 32, which
            // finds the peak that owns it by a binary search over the warp's
            // inclusive entry counts: every lane tests an entry in every
            // round, however unevenly the entries fall among the peaks.
            // Latency is hidden by running ahead: a step's bucket-table loads
            // are issued one step early (steps are chunks, or chunk x pass
            // for modified cosine), the peaks a probe needs one chunk early,
            // and the entries of kRounds rounds are loaded before the first is
            // tested.
            int n = 0;  // candidates found (warp-uniform)
            constexpr int kPasses = MODIFIED ? 2 : 1;
            const int n_steps = ((na + 31) >> 5) * kPasses;
            float mz_c = 0.f, mz_n = 0.f;  // chunks c, c+1
            double w_c = 0.0, w_n = 0.0;
            auto load_peak = [&](int pp, float& mz, double& w) {
                if (pp < na) {
                    mz = P.A.mz[a0 + pp];
                    w = __dmul_rn(peak_a(P.A.a, a0 + pp), P.A.b[a0 + pp]);
                }
            };
            load_peak(lane, mz_c, w_c);
            load_peak(32 + lane, mz_n, w_n);
            // one step's window and raw bucket-table values (consumed a step later)
            float pL = 1.0f, pH = 0.0f;
            uint32_t pt0 = 0, pt1 = 0, pt2 = 0, pt3 = 0;
            auto probe = [&](bool valid, float mz, bool shifted) {
                pL = 1.0f;
                pH = 0.0f;
                pt0 = pt1 = pt2 = pt3 = 0u;
                if (!valid) return;
                const bool ok = (MODIFIED && shifted)
                                    ? nl_window(mz, P.A.prec[a], P.tol, pL, pH)
                                    : Window<A_IS_REF, NOSHIFT>::bounds(mz, P.tol, P.shift, pL, pH);
                if (!ok) {
                    atomicOr(P.err, kErrBadOffsets);
                    pL = 1.0f;
                    pH = 0.0f;
                    return;
                }
                if (!(pL <= pH)) return;
                const uint32_t* TT = (MODIFIED && shifted) ? T2 : T;
                const long long blo = bucket_of(pL, P.g.inv_w);
                const long long bhi = bucket_of(pH, P.g.inv_w);
                if (bhi - blo + 1 >= P.g.nb) {
                    pt0 = __ldg(&TT[0]);
                    pt1 = __ldg(&TT[P.g.nb]);
                } else {
                    const unsigned bl = (unsigned)blo & nbmask, bh = (unsigned)bhi & nbmask;
                    pt0 = __ldg(&TT[bl]);
                    if (bl <= bh) {
                        pt1 = __ldg(&TT[bh + 1]);
                    } else {  // wrapped: [bl, nb) then [0, bh]
                        pt1 = __ldg(&TT[P.g.nb]);
                        pt2 = __ldg(&TT[0]);
                        pt3 = __ldg(&TT[bh + 1]);
                    }
                }
            };
            probe(lane < na, mz_c, false);
            for (int st = 0; st < n_steps; ++st) {
                const int pass = MODIFIED ? (st & 1) : 0;
                const int pc = (MODIFIED ? (st >> 1) : st) * 32;
                const int p = pc + lane;
                // this step's probe
                const float L = pL, H = pH;
                const uint32_t r0b = pt0, c0 = pt1 - pt0, r1b = pt2, c1 = pt3 - pt2;
                if (pass == 0) {
                    s_wa[lane] = w_c;
                    if (MODIFIED) s_x[lane] = mz_c;
                }
                // the next step's probe, in flight during this step's rounds
                if (st + 1 < n_steps) {
                    if (MODIFIED && pass == 0)
                        probe(p < na, mz_c, true);
                    else
                        probe(p + 32 < na, mz_n, false);
                }
                const Entry* EE = (MODIFIED && pass) ? P.ent2 : ent;
                s_lh[lane] = make_float2(L, H);
                const uint32_t c = c0 + c1;
                uint32_t incl = c;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const uint32_t v = __shfl_up_sync(full, incl, d);
                    if (lane >= d) incl += v;
                }
                const uint32_t excl = incl - c;
                const uint32_t E = __shfl_sync(full, incl, 31);
                const bool wrapped = __any_sync(full, c1 != 0u);
                const uint32_t off0 = r0b - excl;  // entry k of lane l: r0b + (k - excl)
                __syncwarp();
                // position of flat entry k, and the lane (peak) that owns it
                auto locate = [&](uint32_t k, int& o) -> uint32_t {
                    o = 0;
#pragma unroll
                    for (int step = 16; step > 0; step >>= 1) {
                        const uint32_t v = __shfl_sync(full, incl, o + step - 1);
                        if (v <= k) o += step;
                    }
                    if (!wrapped) return __shfl_sync(full, off0, o & 31) + k;
                    const uint32_t oex = __shfl_sync(full, excl, o & 31);
                    const uint32_t oc0 = __shfl_sync(full, c0, o & 31);
                    const uint32_t or0 = __shfl_sync(full, r0b, o & 31);
                    const uint32_t or1 = __shfl_sync(full, r1b, o & 31);
                    const uint32_t e = k - oex;
                    return e < oc0 ? or0 + e : or1 + (e - oc0);
                };
                for (uint32_t kb = 0; kb < E; kb += 32 * kRounds) {
                    // kRounds rounds' entries in flight before the first is tested
                    int ow[kRounds];
                    Entry enb[kRounds];
#pragma unroll
                    for (int u = 0; u < kRounds; ++u) {
                        const uint32_t k = kb + 32u * u + (uint32_t)lane;
                        const uint32_t pos = locate(k, ow[u]);
                        enb[u].id = 0;
                        if (k < E) enb[u] = EE[tbase + pos];
                    }
#pragma unroll
                    for (int u = 0; u < kRounds; ++u) {
                        if (kb + 32u * u >= E) break;
                        const uint32_t k = kb + 32u * u + (uint32_t)lane;
                        const int o = ow[u];
                        const Entry en = enb[u];
                        bool cand = false;
                        if (k < E) {
                            const float2 lh = s_lh[o];
                            const int bq = (int)(en.id >> 16);
                            cand = en.mz >= lh.x && en.mz <= lh.y && bq >= range_lo && bq < range_hi;
                            if (MODIFIED && pass && cand) {
                                // the shifted window exactly as matchms tests it:
                                // mz2 = mz_q + (prec_ref - prec_q) against mz_ref -+ tol
                                const int qb = b_begin + bq;
                                const float y = P.B.mz[P.B.off[qb] + (en.id & 0xFFFFu)];
                                const double mz2 =
                                    __dadd_rn((double)y, __dsub_rn(P.A.prec[a], P.B.prec[qb]));
                                const double x = (double)s_x[o];
                                cand = !(mz2 > __dadd_rn(x, P.tol)) && !(mz2 < __dsub_rn(x, P.tol));
                            }
                        }
                        const unsigned bal = __ballot_sync(full, cand);
                        const int slot = n + __popc(bal & below);
                        n += __popc(bal);
                        if (cand && slot < pool_max) {
                            const int bq = (int)(en.id >> 16);
                            const int pB = (int)(en.id & 0xFFFFu);
                            const int pa = pc + o;
                            const double aB = P.B.a ? P.B.a[P.B.off[b_begin + bq] + pB] : 1.0;
                            double key;
                            uint32_t gen;
                            if (A_IS_REF) {
                                key = __dmul_rn(__dmul_rn(s_wa[o], aB), en.b);
                                gen = ((uint32_t)pa << 16) | (uint32_t)pB;
                                if (MODIFIED) gen |= (uint32_t)pass << 31;
                            } else {
                                const double wB = __dmul_rn(aB, en.b);
                                key = __dmul_rn(__dmul_rn(wB, peak_a(P.A.a, a0 + pa)),
                                                P.A.b[a0 + pa]);
                                gen = ((uint32_t)pB << 16) | (uint32_t)pa;
                            }
                            // push onto the query's chain: swap the new slot into
                            // its 16-bit head; the old head, if of this epoch, is
                            // the chain's next element
                            const int qr = bq - range_lo;
                            uint32_t* hp = head + (qr >> 1);
                            const unsigned sh = (unsigned)(qr & 1) * 16u;
                            const unsigned nh = (epoch << 12) | (unsigned)slot;
                            unsigned cur = *reinterpret_cast<volatile uint32_t*>(hp), assumed, ph;
                            do {
                                assumed = cur;
                                ph = (assumed >> sh) & 0xFFFFu;
                                cur = atomicCAS(hp, assumed,
                                                (assumed & ~(0xFFFFu << sh)) | (nh << sh));
                            } while (cur != assumed);
                            uint32_t m = (uint32_t)qr;
                            if ((ph >> 12) == epoch) m |= ((ph & 0xFFFu) << 12) | kHasNext;
                            pool.put(slot, key, gen, m);
                        }
                    }
                    if (n > pool_max) break;
                }
                __syncwarp();  // s_lh / s_wa / s_x are rewritten by the next step
                if (n > pool_max) break;
                if (pass == kPasses - 1) {  // next chunk: rotate the prefetched peaks
                    mz_c = mz_n;
                    w_c = w_n;
                    load_peak(pc + 64 + lane, mz_n, w_n);
                }
            }
            __syncwarp();
            if (n > pool_max) {
                if (rw > 1) {
                    // too many candidates for one pool: retry a narrower range
                    width = max(1, (int)((long long)rw * pool_max / (2LL * n)));
                    width = min(width, rw / 2 > 0 ? rw / 2 : 1);
                    continue;
                }
                // a single pair has more candidates than the pool: pair kernel
                if (lane == 0) {
                    const int bq = b_begin + range_lo;
                    const int rr = A_IS_REF ? a : bq, qq = A_IS_REF ? bq : a;
                    spill_push(P.spill, rr, qq, P.err);
                    if (!SPARSE) {
                        const int64_t o = (int64_t)rr * P.dense.ld + qq;
                        P.dense.score[o] = __int_as_float(0x7fc00000);
                        P.dense.matches[o] = -1;
                        P.dense.overflow[o] = 0;
                    }
                }
                __syncwarp();
                range_lo = range_hi;
                width = max(32, width);
                continue;
            }

            // ---- zeros for the dense row segment of the range: queries without
            // a candidate keep them; the runs' results, stored by this warp
            // after the __syncwarp below, overwrite theirs (a spilled pair's
            // overflow flag is rewritten by the pair kernel).  Written just
            // before the runs are resolved, so that the lines are still in L2
            // when the results land in them (zeroing before the sweep let L2
            // evict ~1/3 of them first: +40% DRAM traffic).  Four queries per
            // lane, 16-byte streaming stores when aligned.
            if (!SPARSE) {
                const int64_t row = (int64_t)a * P.dense.ld + b_begin + range_lo;
                int qv = 0;
                if ((row & 3) == 0 && (P.dense.ld & 3) == 0) {
                    for (; qv + 128 <= rw; qv += 128) {
                        const int64_t o = row + qv + 4 * lane;
                        __stcs(reinterpret_cast<float4*>(P.dense.score + o),
                               make_float4(0.f, 0.f, 0.f, 0.f));
                        __stcs(reinterpret_cast<int4*>(P.dense.matches + o), make_int4(0, 0, 0, 0));
                        __stcs(reinterpret_cast<uchar4*>(P.dense.overflow + o),
                               make_uchar4(0, 0, 0, 0));
                    }
                }
                for (int qr = qv + lane; qr < rw; qr += 32) {
                    __stcs(&P.dense.score[row + qr], 0.f);
                    __stcs(&P.dense.matches[row + qr], 0);
                    __stcs(&P.dense.overflow[row + qr], (unsigned char)0);
                }
            }
            __syncwarp();

            // ---- resolve each query's run ----
            // Slot s owns its query's run when the query's head names it (it
            // was pushed last); the owner walks the chain.  Runs of 1 to 3
            // candidates are resolved by their lane in closed form; runs of
            // 4..32 are queued and resolved by the warp; longer runs (or runs
            // reaching match_limit) go to the pair kernel.
            int n_mid = 0, n_big = 0;
            auto flush_long = [&]() {
                __syncwarp();
                // runs of 4..8 candidates, four at a time: each 8-lane segment
                // sorts one run's (key, gen) descending in registers (bitonic),
                // then resolves it greedily by segment-wise ballot
                const int seg = lane >> 3, tq = lane & 7;
                for (int r = 0; r < n_mid; r += 4) {
                    const bool valid = r + seg < n_mid;
                    const unsigned e = valid ? long_runs[r + seg] : 0u;
                    const int s0 = (int)(e & 0xFFFu);
                    const int L = valid ? (int)(e >> 12) : 0;
                    double k = -INFINITY;
                    uint32_t g = 0;
                    if (tq < L) {
                        int sl = s0;
                        for (int h = 0; h < tq; ++h) sl = meta_next(pool.meta(sl));
                        k = pool.key(sl);
                        g = pool.gen(sl);
                    }
#pragma unroll
                    for (int kk = 2; kk <= kMidRun; kk <<= 1) {
#pragma unroll
                        for (int j = kk >> 1; j > 0; j >>= 1) {
                            const double ok = __shfl_xor_sync(full, k, j);
                            const uint32_t og = __shfl_xor_sync(full, g, j);
                            const bool lower = (tq & j) == 0;
                            const bool desc = (tq & kk) == 0;
                            const bool mine_first = before(k, g, ok, og);
                            const bool keep = (lower == desc) ? mine_first : !mine_first;
                            if (!keep) {
                                k = ok;
                                g = og;
                            }
                        }
                    }
                    bool alive = tq < L;
                    unsigned bal = __ballot_sync(full, alive);
                    double score = 0.0;
                    int mt = 0;
                    while (bal) {
                        const unsigned mine = (bal >> (seg * 8)) & 0xFFu;
                        const int leader = mine ? seg * 8 + __ffs(mine) - 1 : lane;
                        const uint32_t lg = __shfl_sync(full, g, leader);
                        const double lk = __shfl_sync(full, k, leader);
                        if (mine) {
                            score = __dadd_rn(score, lk);
                            ++mt;
                            if (lane == leader || gen_p1<MODIFIED>(g) == gen_p1<MODIFIED>(lg) ||
                                ((g & 0xFFFFu) == (lg & 0xFFFFu)))
                                alive = false;
                        }
                        bal = __ballot_sync(full, alive);
                    }
                    if (valid && tq == 0)
                        store_result(b_begin + range_lo + meta_query(pool.meta(s0)), score, mt);
                }
                // runs of 9..32 candidates, one at a time on the whole warp
                for (int r = 0; r < n_big; ++r) {
                    const unsigned e = long_runs[kLongRuns - 1 - r];
                    const int s0 = (int)(e & 0xFFFu);
                    const int L = (int)(e >> 12);
                    double k = -INFINITY;
                    uint32_t g = 0;
                    if (lane < L) {
                        int sl = s0;
                        for (int h = 0; h < lane; ++h) sl = meta_next(pool.meta(sl));
                        k = pool.key(sl);
                        g = pool.gen(sl);
                    }
#pragma unroll
                    for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
                        for (int j = kk >> 1; j > 0; j >>= 1) {
                            const double ok = __shfl_xor_sync(full, k, j);
                            const uint32_t og = __shfl_xor_sync(full, g, j);
                            const bool lower = (lane & j) == 0;
                            const bool desc = (lane & kk) == 0;
                            // the lower lane of a descending pair keeps the larger
                            const bool mine_first = before(k, g, ok, og);
                            const bool keep = (lower == desc) ? mine_first : !mine_first;
                            if (!keep) {
                                k = ok;
                                g = og;
                            }
                        }
                    }
                    bool alive = lane < L;
                    unsigned bal = __ballot_sync(full, alive);
                    double score = 0.0;
                    int mt = 0;
                    while (bal) {
                        const int leader = __ffs(bal) - 1;
                        const uint32_t lg = __shfl_sync(full, g, leader);
                        const double lk = __shfl_sync(full, k, leader);
                        score = __dadd_rn(score, lk);
                        ++mt;
                        if (lane == leader || gen_p1<MODIFIED>(g) == gen_p1<MODIFIED>(lg) ||
                            ((g & 0xFFFFu) == (lg & 0xFFFFu)))
                            alive = false;
                        bal = __ballot_sync(full, alive);
                    }
                    if (lane == 0)
                        store_result(b_begin + range_lo + meta_query(pool.meta(s0)), score, mt);
                }
                __syncwarp();
                n_mid = 0;
                n_big = 0;
            };
            for (int c = 0; c < n; c += 32) {
                const int s = c + lane;
                bool own = false;
                int L = 0, qr = 0;
                double snB_own = 0.0;
                double k0 = 0.0, k1 = 0.0, k2 = 0.0;
                uint32_t g0 = 0, g1 = 0, g2 = 0;
                if (s < n) {
                    const uint32_t m0 = pool.meta(s);
                    qr = meta_query(m0);
                    const unsigned h = (head[qr >> 1] >> ((qr & 1) * 16)) & 0xFFFu;
                    own = h == (unsigned)s;
                    if (own) {
                        // the query norm's load starts before the chain walk
                        snB_own = P.snB[b_begin + range_lo + qr];
                        k0 = pool.key(s);
                        g0 = pool.gen(s);
                        L = 1;
                        if (m0 & kHasNext) {
                            const int s1 = meta_next(m0);
                            const uint32_t m1 = pool.meta(s1);
                            k1 = pool.key(s1);
                            g1 = pool.gen(s1);
                            L = 2;
                            if (m1 & kHasNext) {
                                const int s2 = meta_next(m1);
                                uint32_t m2 = pool.meta(s2);
                                k2 = pool.key(s2);
                                g2 = pool.gen(s2);
                                L = 3;
                                // longer runs: count the rest (up to kLongRun + 1)
                                while ((m2 & kHasNext) && L <= kLongRun) {
                                    m2 = pool.meta(meta_next(m2));
                                    ++L;
                                }
                            }
                        }
                    }
                }
                const bool is_long = own && L > 3 && L <= kLongRun && L < P.match_limit;
                const bool is_mid = is_long && L <= kMidRun;
                const unsigned mb = __ballot_sync(full, is_mid);
                const unsigned bb = __ballot_sync(full, is_long && !is_mid);
                if (n_mid + n_big + __popc(mb) + __popc(bb) > kLongRuns) flush_long();
                const unsigned run = (unsigned)s | ((unsigned)L << 12);
                if (is_mid)
                    long_runs[n_mid + __popc(mb & below)] = run;
                else if (is_long)
                    long_runs[kLongRuns - 1 - (n_big + __popc(bb & below))] = run;
                n_mid += __popc(mb);
                n_big += __popc(bb);
                if (own && !is_long) {
                    const int bq = b_begin + range_lo + qr;
                    if (L >= P.match_limit || L > kLongRun) {
                        spill_push(P.spill, A_IS_REF ? a : bq, A_IS_REF ? bq : a, P.err);
                        if (!SPARSE) put_dense(bq, __int_as_float(0x7fc00000), -1);
                    } else {
                        // one to three candidates: sorting network, then greedy
                        double score = k0;
                        int mt = 1;
                        if (L >= 2) {
                            auto order = [](double& ka, uint32_t& ga, double& kb, uint32_t& gb) {
                                if (before(kb, gb, ka, ga)) {
                                    const double tk = ka;
                                    ka = kb;
                                    kb = tk;
                                    const uint32_t tg = ga;
                                    ga = gb;
                                    gb = tg;
                                }
                            };
                            auto clash = [](uint32_t ga, uint32_t gb) {
                                return gen_p1<MODIFIED>(ga) == gen_p1<MODIFIED>(gb) ||
                                       (ga & 0xFFFFu) == (gb & 0xFFFFu);
                            };
                            order(k0, g0, k1, g1);
                            if (L == 3) {
                                order(k1, g1, k2, g2);
                                order(k0, g0, k1, g1);
                            }
                            score = k0;
                            const bool take1 = !clash(g0, g1);
                            if (take1) {
                                score = __dadd_rn(score, k1);
                                mt = 2;
                            }
                            if (L == 3 && !clash(g0, g2) && !(take1 && clash(g1, g2))) {
                                score = __dadd_rn(score, k2);
                                ++mt;
                            }
                        }
                        store_result_n(bq, score, mt, snB_own);
                    }
                }
            }
            __syncwarp();
            flush_long();
            __syncwarp();
            range_lo = range_hi;
            if (n < pool_max / 4) width = min(tn, width * 2);
        }
        __syncwarp();
        if (P.trace.rec && lane == 0) {
            const unsigned long long k = atomicAdd(P.trace.count, 1ull);
            if ((long long)k < P.trace.cap) {
                unsigned int smid;
                asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
                unsigned long long* r = P.trace.rec + 4 * k;
                r[0] = (unsigned long long)P.trace.tag | ((unsigned long long)smid << 32);
                r[1] = base + (unsigned long long)f;
                r[2] = *s_t0;
                r[3] = global_ns();
            }
        }
        }
    }
    if (P.slots) {  // give the global-pool slice back
        __syncthreads();
        if (threadIdx.x == 0 && pslot >= 0) {
            atomicAnd(&P.slots[pslot >> 5], ~(1u << (pslot & 31)));
            __threadfence();
        }
    }
}

// ---------------------------------------------------------------------------
// 6. pair kernel: one CTA per pair
// ---------------------------------------------------------------------------
struct PairParams {
    SpecSet R;
    SpecSet Q;
    const double* snR;
    const double* snQ;
    double tol;
    double shift;
    int match_limit;
    int cap;  // power of two >= match_limit
    // work: either the spill list (pairs != nullptr) or every pair of R x Q
    const int2* pairs;
    const unsigned int* n_pairs;
    unsigned int pairs_cap;
    unsigned long long* work;
    DenseOut dense;
    SparseOut sparse;
    uint32_t* err;
    const uint32_t* bad;
    int sym;  // only pairs (reference i, query j) with i <= j
    // test hook (CMS_TEST_STALL=pair): the pipelined kernel's greedy warp
    // leaves at once, so the producers' bounded waits run out
    int test_stall;
};

// Register-blocked bitonic sort of m = 8 * blockDim.x candidates, descending by
// (order key, gen), for the pair kernel: each thread holds the 8 consecutive
// elements 8t..8t+7 in registers.  Exchange distance j < 8: inside the
// thread; 8 <= j < 256: with lane t ^ (j / 8) of the same warp by shuffle;
// j >= 256: with thread t ^ (j / 8) of another warp through shared memory
// (element-major staging, so those accesses have no bank conflicts).  The
// network and the result are those of the plain shared-memory bitonic sort.
struct Cand {
    unsigned long long k;
    uint32_t g;
};
__device__ __forceinline__ bool cand_gt(const Cand& a, const Cand& b) {
    return a.k > b.k || (a.k == b.k && a.g > b.g);
}
// keep the larger of the pair (i, i ^ j) at the lower index when the block
// of kk elements containing i sorts descending
template <int J>
__device__ __forceinline__ void sort8_local(Cand (&c)[8], int base, int kk) {
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        if (e & J) continue;
        const int f = e | J;
        const bool desc = ((base + e) & kk) == 0;
        const bool gt = cand_gt(c[e], c[f]);
        if (desc ? !gt : gt) {
            const Cand t = c[e];
            c[e] = c[f];
            c[f] = t;
        }
    }
}
// Barriers of the threads that generate and sort a pair's candidates: the
// whole block, or (pipelined pair kernel) the producer warps only, on named
// barrier 1.
struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct GroupSync {
    int n;  // participating threads (a multiple of 32)
    __device__ __forceinline__ void operator()() const {
        asm volatile("bar.sync 1, %0;" ::"r"(n) : "memory");
    }
};

// nt threads (tid 0..nt-1) sort okey/cgen[0, m), m = 8 * nt, in registers.
template <typename Sync>
__device__ void sort8_block(unsigned long long* okey, uint32_t* cgen, int m, int nt, int tid,
                            Sync sync) {
    const int base = 8 * tid;
    const unsigned full = 0xffffffffu;
    Cand c[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        c[e].k = okey[base + e];
        c[e].g = cgen[base + e];
    }
    for (int kk = 2; kk <= m; kk <<= 1) {
        for (int j = kk >> 1; j > 0; j >>= 1) {
            if (j >= 8) {
                const int pt = tid ^ (j >> 3);
                const bool lower = (base & j) == 0;
                const bool desc = (base & kk) == 0;  // kk >= 16: the same for all e
                Cand o[8];
                if (j >= 256) {
                    sync();
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        okey[e * nt + tid] = c[e].k;
                        cgen[e * nt + tid] = c[e].g;
                    }
                    sync();
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        o[e].k = okey[e * nt + pt];
                        o[e].g = cgen[e * nt + pt];
                    }
                } else {
                    const int d = j >> 3;
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        o[e].k = __shfl_xor_sync(full, c[e].k, d);
                        o[e].g = __shfl_xor_sync(full, c[e].g, d);
                    }
                }
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const bool gt = cand_gt(c[e], o[e]);
                    if ((lower == desc) ? !gt : gt) c[e] = o[e];
                }
            } else if (j == 4) {
                sort8_local<4>(c, base, kk);
            } else if (j == 2) {
                sort8_local<2>(c, base, kk);
            } else {
                sort8_local<1>(c, base, kk);
            }
        }
    }
    sync();
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        okey[base + e] = c[e].k;
        cgen[base + e] = c[e].g;
    }
    sync();
}

// Candidates of pair (ri, qi) in generation order, truncated at match_limit,
// into okey/cgen, by nt threads (tid 0..nt-1, whole warps) with barrier
// `sync`; s_scan holds one int per warp.  Returns the number generated
// before truncation stopped it (>= match_limit means overflow).
template <bool MODIFIED, typename Sync>
__device__ int gen_pair(const PairParams& P, int64_t ri, int64_t qi, unsigned long long* okey,
                        uint32_t* cgen, int nt, int tid, int* s_scan, Sync sync) {
    const int lane = tid & 31, wid = tid >> 5, nwarps = nt >> 5;
    const unsigned full = 0xffffffffu;
    const int64_t r0 = P.R.off[ri], q0 = P.Q.off[qi];
    const int nr = (int)(P.R.off[ri + 1] - r0), nq = (int)(P.Q.off[qi + 1] - q0);
    const float* qmz = P.Q.mz + q0;
    int total = 0;
    bool overflow = false;
    // modified cosine generates twice: at shift 0, then at the pair's
    // precursor difference, continuing the same candidate list
#pragma unroll 1
    for (int pass = 0; pass < (MODIFIED ? 2 : 1) && !overflow && nr > 0 && nq > 0; ++pass) {
        const double shift = (MODIFIED && pass) ? __dsub_rn(P.R.prec[ri], P.Q.prec[qi]) : P.shift;
        for (int pc = 0; pc < nr && !overflow; pc += nt) {
            const int p1 = pc + tid;
            int start = 0, cnt = 0;
            double lo = 0.0, hi = 0.0, w1 = 0.0;
            if (p1 < nr) {
                const double mz1 = (double)P.R.mz[r0 + p1];
                lo = __dsub_rn(mz1, P.tol);
                hi = __dadd_rn(mz1, P.tol);
                // first p2 with mz_q + shift >= lo
                int L = 0, H = nq;
                while (L < H) {
                    const int M = (L + H) >> 1;
                    if (__dadd_rn((double)qmz[M], shift) < lo)
                        L = M + 1;
                    else
                        H = M;
                }
                start = L;
                int k = L;
                while (k < nq && !(__dadd_rn((double)qmz[k], shift) > hi)) ++k;
                cnt = k - L;
            }
            // exclusive scan of cnt over the nt threads
            int incl = cnt;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int v = __shfl_up_sync(full, incl, d);
                if (lane >= d) incl += v;
            }
            if (lane == 31) s_scan[wid] = incl;
            sync();
            if (wid == 0) {
                int v = lane < nwarps ? s_scan[lane] : 0;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int u = __shfl_up_sync(full, v, d);
                    if (lane >= d) v += u;
                }
                if (lane < nwarps) s_scan[lane] = v;
            }
            sync();
            const int excl = incl - cnt + (wid > 0 ? s_scan[wid - 1] : 0);
            const int chunk_total = s_scan[nwarps - 1];
            if (cnt > 0) {
                w1 = __dmul_rn(peak_a(P.R.a, r0 + p1), P.R.b[r0 + p1]);
                for (int i = 0; i < cnt; ++i) {
                    const int rank = total + excl + i;
                    if (rank >= P.match_limit) break;
                    const int p2 = start + i;
                    const double key =
                        __dmul_rn(__dmul_rn(w1, peak_a(P.Q.a, q0 + p2)), P.Q.b[q0 + p2]);
                    okey[rank] = order_key(key);
                    cgen[rank] = ((uint32_t)pass << 31) | ((uint32_t)p1 << 16) | (uint32_t)p2;
                }
            }
            total += chunk_total;
            if (total >= P.match_limit) overflow = true;
            sync();
        }
    }
    return total;
}

// the in-thread stages of sort8_words (exchange distance J < 8)
template <int J>
__device__ __forceinline__ void words_local(unsigned long long (&c)[8], int base, int kk) {
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        if (e & J) continue;
        const int f = e | J;
        const bool desc = ((base + e) & kk) == 0;
        const bool gt = c[e] > c[f];
        if (desc ? !gt : gt) {
            const unsigned long long t = c[e];
            c[e] = c[f];
            c[f] = t;
        }
    }
}

// Register-blocked bitonic sort, descending, of m = 8 * nt single 64-bit words
// (thread t holds network positions 8t..8t+7), exchanging through `scratch`
// (m words) for distances of 256 and more; the sorted words end in the
// threads' registers, position 8t + e in c[e] of thread t.
template <typename Sync>
__device__ void sort8_words(unsigned long long* scratch, unsigned long long (&c)[8], int m,
                            int nt, int tid, Sync sync) {
    const int base = 8 * tid;
    const unsigned full = 0xffffffffu;
    for (int kk = 2; kk <= m; kk <<= 1) {
        for (int j = kk >> 1; j > 0; j >>= 1) {
            if (j >= 8) {
                const int pt = tid ^ (j >> 3);
                const bool lower = (base & j) == 0;
                const bool desc = (base & kk) == 0;
                unsigned long long o[8];
                if (j >= 256) {
                    sync();
#pragma unroll
                    for (int e = 0; e < 8; ++e) scratch[e * nt + tid] = c[e];
                    sync();
#pragma unroll
                    for (int e = 0; e < 8; ++e) o[e] = scratch[e * nt + pt];
                } else {
#pragma unroll
                    for (int e = 0; e < 8; ++e) o[e] = __shfl_xor_sync(full, c[e], j >> 3);
                }
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const bool gt = c[e] > o[e];
                    if ((lower == desc) ? !gt : gt) c[e] = o[e];
                }
            } else if (j == 4) {
                words_local<4>(c, base, kk);
            } else if (j == 2) {
                words_local<2>(c, base, kk);
            } else {
                words_local<1>(c, base, kk);
            }
        }
    }
}

// Sorts the m = 8 * nt candidates of okey/cgen (padded past n with zeros)
// into greedy order by sorting one 64-bit word per candidate: the order key
// without its top bit (set for every key >= +0.0) and without its low R + 1
// bits, then a "real candidate" bit, then the R-bit index (m = 2^R), so
// equal words' order is the index order, i.e. generation order, and padding
// sorts last.  Keys that agree in every kept bit but differ in a dropped one
// would be misordered: the pass checks every pair of neighbours for that
// (and for a key below +0.0) and returns false, leaving okey/cgen untouched,
// if it finds one; the caller then sorts the pairs themselves.  On success
// okey/cgen hold the candidates in greedy order.
template <typename Sync>
__device__ bool sort8_by_word(unsigned long long* okey, uint32_t* cgen,
                              unsigned long long* scratch, int* s_flag, int n, int m, int nt,
                              int tid, Sync sync) {
    const int rb = 31 - __clz(m);  // index bits
    const unsigned long long imask = (1ull << rb) - 1ull;
    const unsigned long long real = 1ull << rb;
    const unsigned long long kmask = ~((real << 1) - 1ull);
    if (tid == 0) *s_flag = 0;
    sync();
    unsigned long long c[8];
    bool bad = false;
    // which candidate starts at which network position is free (every word
    // carries its index): thread tid takes candidates e * nt + tid, so that
    // the loads of consecutive threads are consecutive words
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int i = e * nt + tid;
        if (i < n) {
            const unsigned long long k = okey[i];
            bad |= (k >> 63) == 0ull;
            c[e] = ((k << 1) & kmask) | real | (unsigned long long)i;
        } else {
            c[e] = (unsigned long long)i;  // padding: below every real word
        }
    }
    if (bad) atomicOr(s_flag, 1);
    sort8_words(scratch, c, m, nt, tid, sync);
    // neighbours that tie in the kept bits must have equal keys; the word
    // after this thread's last is the next thread's first
    sync();
    scratch[tid] = c[0];
    sync();
    const unsigned long long after = tid + 1 < nt ? scratch[tid + 1] : 0ull;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int i = 8 * tid + e;
        if (i + 1 < m && (c[e] & real)) {
            const unsigned long long nx = e < 7 ? c[e + 1] : after;
            if ((nx & real) && ((nx ^ c[e]) & kmask) == 0ull &&
                okey[nx & imask] != okey[c[e] & imask])
                bad = true;
        }
    }
    if (bad) atomicOr(s_flag, 1);
    sync();
    if (*s_flag) return false;
    // the sorted words to scratch, position p at p + p / 8 (the stores of
    // positions 8 * tid + e, nine words apart, fall in different banks), then
    // each thread gathers positions e * nt + tid, so that the final stores of
    // consecutive threads are consecutive
#pragma unroll
    for (int e = 0; e < 8; ++e) scratch[9 * tid + e] = c[e];
    sync();
    unsigned long long k[8];
    uint32_t g[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int pos = e * nt + tid;
        const unsigned long long w = scratch[pos + (pos >> 3)];
        const bool r = (w & real) != 0ull;
        const int src = (int)(w & imask);
        k[e] = r ? okey[src] : 0ull;
        g[e] = r ? cgen[src] : 0u;
    }
    sync();
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        okey[e * nt + tid] = k[e];
        cgen[e * nt + tid] = g[e];
    }
    sync();
    return true;
}

// Pads okey/cgen[n, m) and sorts [0, m) descending by (okey, gen), m the
// power of two >= n: in registers when m = 8 * nt, else in shared memory.
template <typename Sync>
__device__ void sort_pair(unsigned long long* okey, uint32_t* cgen, int n, int m, int nt, int tid,
                          Sync sync) {
    for (int i = n + tid; i < m; i += nt) {
        okey[i] = 0ull;
        cgen[i] = 0u;
    }
    sync();
    if (m == 8 * nt) {
        sort8_block(okey, cgen, m, nt, tid, sync);
        return;
    }
    for (int k = 2; k <= m; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < m; i += nt) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long ka = okey[i], kb = okey[ixj];
                    const uint32_t ga = cgen[i], gb = cgen[ixj];
                    const bool a_gt_b = ka > kb || (ka == kb && ga > gb);
                    const bool desc = (i & k) == 0;
                    if (desc ? !a_gt_b : a_gt_b) {
                        okey[i] = kb;
                        okey[ixj] = ka;
                        cgen[i] = gb;
                        cgen[ixj] = ga;
                    }
                }
            }
            sync();
        }
    }
}

// Greedy by one warp over chunks of 32 sorted candidates (used_r / used_q
// zeroed for the pair's peaks).  Within a chunk a live candidate is accepted
// iff no earlier accepted one shares its reference or query peak: conflict
// masks come from __match_any_sync, and lanes decide in rounds, each lane as
// soon as every earlier conflicting lane has decided (the lowest undecided
// lane always can, so this ends; usually after one or two rounds).  Accepted
// keys are summed in sorted order, as the sequential greedy; every lane ends
// with the same score and match count.
template <bool MODIFIED>
__device__ void greedy_pair(const unsigned long long* okey, const uint32_t* cgen,
                            uint32_t* used_r, uint32_t* used_q, int n, double& score,
                            int& matches) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    // the next chunk's candidates are loaded while this one is resolved
    // (they do not depend on the used-peak bits)
    uint32_t g_nx = lane < n ? cgen[lane] : 0u;
    unsigned long long k_nx = lane < n ? okey[lane] : 0ull;
    for (int c = 0; c < n; c += 32) {
        const int i = c + lane;
        const uint32_t g = g_nx;
        const unsigned long long ok = k_nx;
        if (i + 32 < n) {
            g_nx = cgen[i + 32];
            k_nx = okey[i + 32];
        }
        bool alive = false;
        if (i < n) {
            const int p1 = (int)gen_p1<MODIFIED>(g), p2 = g & 0xFFFF;
            alive = !((used_r[p1 >> 5] >> (p1 & 31)) & 1u) &&
                    !((used_q[p2 >> 5] >> (p2 & 31)) & 1u);
        }
        const unsigned live = __ballot_sync(full, alive);
        if (live == 0u) continue;
        // dead lanes get values no peak index takes, so they match only
        // themselves
        const unsigned m1 = __match_any_sync(full, alive ? gen_p1<MODIFIED>(g) : 0x10000u + lane);
        const unsigned m2 = __match_any_sync(full, alive ? (g & 0xFFFFu) : 0x10000u + lane);
        const unsigned earlier = (m1 | m2) & live & below;
        unsigned dec = ~live, acc = 0u;
        while (dec != full) {
            bool my_dec = (dec >> lane) & 1u, my_acc = (acc >> lane) & 1u;
            if (!my_dec && (earlier & ~dec) == 0u) {
                my_dec = true;
                my_acc = (earlier & acc) == 0u;
            }
            dec = __ballot_sync(full, my_dec);
            acc = __ballot_sync(full, my_acc);
        }
        if ((acc >> lane) & 1u) {
            const int p1 = (int)gen_p1<MODIFIED>(g), p2 = g & 0xFFFF;
            atomicOr(&used_r[p1 >> 5], 1u << (p1 & 31));
            atomicOr(&used_q[p2 >> 5], 1u << (p2 & 31));
        }
        const double kk = (i < n) ? key_from_order(ok) : 0.0;
        for (unsigned a = acc; a; a &= a - 1u) {
            const double k = __shfl_sync(full, kk, __ffs(a) - 1);
            score = __dadd_rn(score, k);
        }
        matches += __popc(acc);
        __syncwarp();
    }
}

// The pair's outputs (dense, or a sparse hit above the threshold).
template <bool SPARSE>
__device__ void write_pair(const PairParams& P, int64_t ri, int64_t qi, int n, double score,
                           int matches, bool overflow) {
    float sc = 0.f;
    if (matches > 0 || n > 0) {
        const double denom = __dmul_rn(P.snR[ri], P.snQ[qi]);
        sc = (n > 0) ? (float)__ddiv_rn(score, denom) : 0.f;
    }
    if (!SPARSE) {
        const int64_t o = ri * P.dense.ld + qi;
        P.dense.score[o] = sc;
        P.dense.matches[o] = matches;
        P.dense.overflow[o] = overflow ? 1 : 0;
    } else if (n > 0 && sc >= P.sparse.threshold) {
        emit_hit(P.sparse, (int)ri, (int)qi, sc, matches, overflow ? 1 : 0);
    }
}

// item -> pair (reference ri, query qi); false for pairs under the diagonal
// of a symmetric whole-matrix launch (copied afterwards)
__device__ __forceinline__ bool pair_of(const PairParams& P, int64_t item, int64_t& ri,
                                        int64_t& qi) {
    if (P.pairs) {
        const int2 pr = P.pairs[item];
        ri = pr.x;
        qi = pr.y;
        return true;
    }
    ri = item / P.Q.n;
    qi = item - ri * P.Q.n;
    return !(P.sym && ri > qi);
}

template <bool SPARSE, bool MODIFIED>
__global__ void pair_kernel(PairParams P) {
    if (*P.bad) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned long long* okey = reinterpret_cast<unsigned long long*>(smem_raw);
    uint32_t* cgen = reinterpret_cast<uint32_t*>(okey + P.cap);
    uint32_t* used_r = cgen + P.cap;          // 2048 words: 65536 peaks
    uint32_t* used_q = used_r + 2048;
    __shared__ int s_scan[32];
    __shared__ unsigned long long s_item;

    const int tid = threadIdx.x, wid = tid >> 5;
    const int64_t n_items = P.pairs ? (int64_t)min(*P.n_pairs, P.pairs_cap) : P.R.n * P.Q.n;
    const BlockSync sync;

    for (int64_t iter = 0;; ++iter) {
        // spill list: dynamic (pairs differ widely in cost); whole matrix:
        // static stride (uniform pairs, no contention on one counter)
        __syncthreads();
        if (tid == 0) s_item = P.pairs ? atomicAdd(P.work, 1ull)
                                       : (unsigned long long)(blockIdx.x + iter * gridDim.x);
        __syncthreads();
        const int64_t item = (int64_t)s_item;
        if (item >= n_items) break;
        int64_t ri, qi;
        if (!pair_of(P, item, ri, qi)) continue;
        const int total = gen_pair<MODIFIED>(P, ri, qi, okey, cgen, blockDim.x, tid, s_scan, sync);
        const int n = min(total, P.match_limit);
        double score = 0.0;
        int matches = 0;
        if (n > 0) {
            const int nr = (int)(P.R.off[ri + 1] - P.R.off[ri]);
            const int nq = (int)(P.Q.off[qi + 1] - P.Q.off[qi]);
            for (int i = tid; i < (nr + 31) / 32; i += blockDim.x) used_r[i] = 0u;
            for (int i = tid; i < (nq + 31) / 32; i += blockDim.x) used_q[i] = 0u;
            int m = 1;
            while (m < n) m <<= 1;
            sort_pair(okey, cgen, n, m, blockDim.x, tid, sync);
            if (wid == 0) greedy_pair<MODIFIED>(okey, cgen, used_r, used_q, n, score, matches);
        }
        if (tid == 0) write_pair<SPARSE>(P, ri, qi, n, score, matches, total >= P.match_limit);
    }
}

// ---- pipelined pair kernel ----
// Warps 0..G-1 (the producers, G = blockDim.x / 32 - 1) generate and sort the
// candidates of the next pair into one of two buffers while warp G (the
// consumer) runs the greedy of the previous pair from the other buffer, so the
// producers never wait at a barrier while one warp resolves.  The hand-off
// is two mbarriers per buffer: `full` (every producer thread arrives after
// its writes) and `empty` (the consumer, after reading).  Every wait is
// bounded by %globaltimer (kPipeWaitNs); on expiry the waiting side sets
// kErrPipelineTimeout, raises the CTA's stop flag and leaves, and the other
// side leaves at its next (bounded) wait.  The producers of a CTA take every
// decision together (one thread decides, a producer barrier publishes it),
// so their named barrier is never left half-joined.
constexpr unsigned long long kPipeWaitNs = 2000000000ull;

__device__ __forceinline__ unsigned long long pipe_clock() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void pipe_bar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(bar)),
                 "r"(count));
}
__device__ __forceinline__ void pipe_bar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(bar))
                 : "memory");
}
// true once the phase of `parity` has completed; false after kPipeWaitNs or
// when *stop is raised
__device__ __forceinline__ bool pipe_bar_wait(uint64_t* bar, uint32_t parity,
                                              volatile int* stop) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    const unsigned long long t0 = pipe_clock();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if (*stop) return false;
        if (pipe_clock() - t0 > kPipeWaitNs) return false;
    }
}

template <bool SPARSE, bool MODIFIED>
__global__ void pair_kernel_pipe(PairParams P) {
    if (*P.bad) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // two candidate buffers, then the consumer's used-peak bitmaps
    unsigned long long* okey0 = reinterpret_cast<unsigned long long*>(smem_raw);
    uint32_t* cgen0 = reinterpret_cast<uint32_t*>(okey0 + 2 * P.cap);
    uint32_t* used_r = cgen0 + 2 * P.cap;  // 2048 words: 65536 peaks
    uint32_t* used_q = used_r + 2048;
    // the producers' sort scratch: one 64-bit word per candidate slot, and one
    // more per eight (the padded layout of the sorted words)
    unsigned long long* scratch = reinterpret_cast<unsigned long long*>(used_q + 2048);
    __shared__ int s_scan[32];
    __shared__ int s_flag;
    __shared__ unsigned long long s_item;
    __shared__ __align__(8) uint64_t s_full[2], s_empty[2];
    __shared__ long long s_ri[2], s_qi[2];
    __shared__ int s_total[2];  // candidates generated; -1: no more pairs
    __shared__ int s_go;        // producers: 1 to continue
    __shared__ volatile int s_stop;

    const int tid = threadIdx.x;
    const int np = (int)blockDim.x - 32;  // producer threads
    const bool producer = tid < np;
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            pipe_bar_init(&s_full[b], (uint32_t)np);
            pipe_bar_init(&s_empty[b], 1u);
        }
        s_stop = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int64_t n_items = P.pairs ? (int64_t)min(*P.n_pairs, P.pairs_cap) : P.R.n * P.Q.n;

    if (producer) {
        const GroupSync sync{np};
        int b = 0;
        uint32_t ph = 0;  // parity of buffer b's current use
        for (int64_t iter = 0;; ++iter) {
            if (tid == 0) s_item = P.pairs ? atomicAdd(P.work, 1ull)
                                           : (unsigned long long)(blockIdx.x + iter * gridDim.x);
            sync();
            const int64_t item = (int64_t)s_item;
            int64_t ri = 0, qi = 0;
            const bool more = item < n_items;
            if (more && !pair_of(P, item, ri, qi)) {
                sync();  // s_item is rewritten by the next fetch
                continue;
            }
            // buffer b free (the consumer is done with its previous pair)?
            if (tid == 0) s_go = pipe_bar_wait(&s_empty[b], ph ^ 1u, &s_stop) ? 1 : 0;
            sync();
            if (!s_go) {
                if (tid == 0 && !s_stop) {
                    atomicOr(P.err, kErrPipelineTimeout);
                    s_stop = 1;
                }
                break;
            }
            unsigned long long* okey = okey0 + (size_t)b * P.cap;
            uint32_t* cgen = cgen0 + (size_t)b * P.cap;
            int total = -1;
            if (more) {
                total = gen_pair<MODIFIED>(P, ri, qi, okey, cgen, np, tid, s_scan, sync);
                const int n = min(total, P.match_limit);
                if (n > 0) {
                    int m = 1;
                    while (m < n) m <<= 1;
                    // one word per candidate when the pair fills the register
                    // sort; the (key, gen) pairs themselves otherwise
                    if (!(m == 8 * np &&
                          sort8_by_word(okey, cgen, scratch, &s_flag, n, m, np, tid, sync)))
                        sort_pair(okey, cgen, n, m, np, tid, sync);
                }
            }
            if (tid == 0) {
                s_ri[b] = ri;
                s_qi[b] = qi;
                s_total[b] = total;
            }
            sync();
            pipe_bar_arrive(&s_full[b]);
            if (!more) break;
            if (++b == 2) {
                b = 0;
                ph ^= 1u;
            }
        }
    } else if (!P.test_stall) {
        // consumer warp
        const int lane = tid & 31;
        int b = 0;
        uint32_t ph = 0;
        for (;;) {
            int ok = 0;
            if (lane == 0) ok = pipe_bar_wait(&s_full[b], ph, &s_stop) ? 1 : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) {
                if (lane == 0 && !s_stop) {
                    atomicOr(P.err, kErrPipelineTimeout);
                    s_stop = 1;
                }
                break;
            }
            const int total = s_total[b];
            if (total < 0) break;  // no more pairs
            const int64_t ri = s_ri[b], qi = s_qi[b];
            const int n = min(total, P.match_limit);
            double score = 0.0;
            int matches = 0;
            if (n > 0) {
                const int nr = (int)(P.R.off[ri + 1] - P.R.off[ri]);
                const int nq = (int)(P.Q.off[qi + 1] - P.Q.off[qi]);
                for (int i = lane; i < (nr + 31) / 32; i += 32) used_r[i] = 0u;
                for (int i = lane; i < (nq + 31) / 32; i += 32) used_q[i] = 0u;
                __syncwarp();
                greedy_pair<MODIFIED>(okey0 + (size_t)b * P.cap, cgen0 + (size_t)b * P.cap,
                                      used_r, used_q, n, score, matches);
            }
            __syncwarp();
            if (lane == 0) {
                pipe_bar_arrive(&s_empty[b]);
                write_pair<SPARSE>(P, ri, qi, n, score, matches, total >= P.match_limit);
            }
            if (++b == 2) {
                b = 0;
                ph ^= 1u;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
inline int next_pow2(long long x) {
    int p = 1;
    while (p < x && p < (1 << 30)) p <<= 1;
    return p;
}

struct Plan {
    int mode;
    int tile;
    int n_tiles;
    int nb;
    double width;
    int pair_threads;
    int cap;
    unsigned int spill_cap;
    int sym;               // cms_cosine_config.symmetric
    double cand_per_pair;  // cms_cosine_config.cand_per_pair (0: unknown)
    int width_by_class[kOrderClasses];  // cms_cosine_config.width_by_class
};

int make_plan(const CosineArgs& args, const cms_cosine_config* cfg, bool sparse, Plan& p) {
    p.mode = (cfg && cfg->mode) ? cfg->mode : 1;
    if (p.mode != 1 && p.mode != 2) {
        set_error("cms_cosine_greedy: mode must be 0, 1 or 2");
        return CMS_ERR_INVALID;
    }
    if (cfg && cfg->tile_spectra > 0) {
        p.tile = cfg->tile_spectra;
    } else {
        // about 200 expected candidates per work item (reference x tile) when
        // the caller gives candidates per pair, else 1024 queries; at most one
        // item per 100000 pairs so that every resident warp gets tens of items
        const long long pairs = (long long)args.ref.n * (long long)args.qry.n;
        long long t = 1024;
        if (cfg && cfg->cand_per_pair > 0.0)
            t = (long long)std::min(2048.0, 200.0 / cfg->cand_per_pair);
        t = std::min(t, pairs / 100000);
        t = std::max<long long>(32, std::min<long long>(2048, t));
        p.tile = (int)((t + 31) / 32 * 32);
    }
    if (p.tile > kMaxTile) {
        set_error("cms_cosine_greedy: tile_spectra must be <= %d", kMaxTile);
        return CMS_ERR_UNSUPPORTED;
    }
    p.tile = (int)std::min<int64_t>(p.tile, std::max<int64_t>(1, args.qry.n));
    p.n_tiles = (int)((args.qry.n + p.tile - 1) / p.tile);
    // bucket width: tol by default (a window spans two or three buckets);
    // any width is correct, narrower ones want more buckets per tile
    double w = (cfg && cfg->bucket_width > 0.0) ? cfg->bucket_width : args.tol;
    if (w < 0.25 * args.tol) w = 0.25 * args.tol;
    if (!(w > 0.0)) w = 1e-3;
    p.width = w;
    const double avg_tile_peaks =
        args.qry.n > 0 ? (double)args.qry.n_peaks * p.tile / (double)args.qry.n : 1.0;
    p.nb = (cfg && cfg->n_buckets > 0) ? next_pow2(cfg->n_buckets)
                                       : next_pow2((long long)std::max(1024.0, avg_tile_peaks));
    p.nb = std::min(p.nb, 1 << 22);
    p.cap = next_pow2(std::max(2, args.match_limit));
    // whole-matrix pair kernel (mode 2): pairs usually fill match_limit, and
    // eight candidates a thread sort in registers; spilled pairs vary in size
    p.pair_threads = (cfg && cfg->pair_threads > 0)
                         ? cfg->pair_threads
                         : (p.mode == 2 ? std::max(64, std::min(512, p.cap / 8)) : 128);
    if (p.pair_threads < 64 || p.pair_threads > 512 || p.pair_threads % 32) {
        set_error("cms_cosine_greedy: pair_threads must be a multiple of 32 in [64, 512]");
        return CMS_ERR_INVALID;
    }
    const long long pairs = (long long)args.ref.n * (long long)args.qry.n;
    long long sc = std::max<long long>(1 << 20, pairs / 64);
    sc = std::min<long long>(sc, std::min<long long>(pairs, 1LL << 28));
    p.spill_cap = (unsigned int)std::max<long long>(sc, 1);
    for (int c = 0; c < kOrderClasses; ++c) {
        const int w = cfg ? cfg->width_by_class[c] : 0;
        if (w < 0) {
            set_error("cms_cosine_greedy: width_by_class entries must be >= 0");
            return CMS_ERR_INVALID;
        }
        p.width_by_class[c] = w;
    }
    (void)sparse;
    return CMS_OK;
}

template <typename T>
int set_func_smem(T* f, size_t bytes) {
    return raise_func_smem(reinterpret_cast<const void*>(f), bytes);
}

// Launch the join.  Persistent (waves == 0): one resident CTA per slot, each
// warp pulling work until none is left; CTA b owns global-pool slices
// 8b..8b+7, so the grid may not exceed the resident CTAs.  Bounded
// (waves > 0): `waves` times the resident CTAs, each warp exiting after an
// equal share of fetches, so that the SMs free up CTA by CTA and concurrent
// launches on other streams are scheduled in between while every wave stays
// full; each CTA claims a global-pool slice from jp.slots (zeroed by the
// caller) for its lifetime.
template <bool A_IS_REF, bool SPARSE, bool NOSHIFT, bool MODIFIED>
int launch_join(cms_ctx* ctx, JoinParams jp, size_t smem, size_t gpool_warps, int64_t n_items,
                cudaStream_t s, int waves = 0) {
    auto* kern = join_kernel<A_IS_REF, SPARSE, NOSHIFT, MODIFIED>;
    if (const int rc = set_func_smem(kern, smem)) return rc;
    jp.trace = TraceOut{ctx->trace_rec, ctx->trace_count, ctx->trace_cap, ctx->trace_tag};
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kJoinThreads, smem);
    const int64_t resident = (int64_t)ctx->sm_count * std::max(1, per_sm);
    int64_t grid;
    if (waves > 0) {
        const int64_t fetches = std::max<int64_t>(1, (n_items + kFetch - 1) / kFetch);
        grid = std::min<int64_t>(resident * waves, (fetches + kJoinWarps - 1) / kJoinWarps);
        grid = std::max<int64_t>(1, grid);
        const int64_t per_warp = (fetches + grid * kJoinWarps - 1) / (grid * kJoinWarps);
        if (per_warp > INT32_MAX) {
            set_error("cms_cosine_greedy: too many work items for one launch");
            return CMS_ERR_UNSUPPORTED;
        }
        jp.max_fetch = (int)per_warp;
        if (!jp.slots) jp.gpool = nullptr;
        jp.n_slots = (int)std::min<int64_t>(resident, (int64_t)(gpool_warps / kJoinWarps));
        if (jp.n_slots <= 0) jp.gpool = nullptr;
        if (!jp.gpool) jp.pool_max = kPool;
    } else {
        jp.max_fetch = 0;
        jp.slots = nullptr;
        grid = resident;
        if (jp.gpool && (size_t)grid * kJoinWarps > gpool_warps) {
            set_error("cms_cosine_greedy: join grid larger than its scratch");
            return CMS_ERR_CUDA;
        }
    }
    kern<<<(unsigned)grid, kJoinThreads, smem, s>>>(jp);
    CMS_CUDA_TRY(cudaGetLastError());
    return CMS_OK;
}

int enqueue_cosine(cms_ctx* ctx, const CosineArgs& args, const DenseOut* dense,
                   const SparseOut* sparse, const Plan& p, cudaStream_t s);
int run_cosine_graph(cms_ctx* ctx, const CosineArgs& args, const DenseOut* dense,
                     const SparseOut* sparse, const Plan& p, cudaStream_t s);

int run_cosine(cms_ctx* ctx, const CosineArgs& args, const DenseOut* dense,
               const SparseOut* sparse, const cms_cosine_config* cfg, cudaStream_t s) {
    Plan p;
    int rc = make_plan(args, cfg, sparse != nullptr, p);
    if (rc) return rc;
    const int sym = (cfg && cfg->symmetric) ? 1 : 0;
    p.sym = sym;
    p.cand_per_pair = (cfg && cfg->cand_per_pair > 0.0) ? cfg->cand_per_pair : 0.0;
    if (sym && args.ref.n != args.qry.n) {
        set_error("cms_cosine_greedy: symmetric needs as many queries as references "
                  "(%lld != %lld)", (long long)args.ref.n, (long long)args.qry.n);
        return CMS_ERR_INVALID;
    }
    const size_t pair_smem = (size_t)p.cap * 12 + 2 * 2048 * 4;
    if (pair_smem > ctx->smem_optin) {
        set_error("cms_cosine_greedy: match_limit %d needs %zu B shared memory (> %zu)",
                  args.match_limit, pair_smem, ctx->smem_optin);
        return CMS_ERR_UNSUPPORTED;
    }

    // ---- scratch layout ----
    const int64_t nR = args.ref.n, nQ = args.qry.n;
    // global pool extension for every warp the join grid can hold (at most
    // 64 warps per SM are resident)
    const size_t gpool_warps = (size_t)ctx->sm_count * 64;
    const size_t gpool_bytes = gpool_warps * (size_t)kGPool * 16;
    size_t need = 0;
    need += bump_size(64 * sizeof(uint64_t));            // flags, counters
    need += bump_size(nR * sizeof(double)) + bump_size(nQ * sizeof(double));
    if (p.mode == 1) {
        need += bump_size(nR * sizeof(int32_t));
        need += bump_size((size_t)p.n_tiles * (p.nb + 1) * sizeof(uint32_t));
        need += bump_size((size_t)p.n_tiles * p.nb * sizeof(uint32_t));
        need += bump_size((size_t)std::max<int64_t>(1, args.qry.n_peaks) * sizeof(Entry));
        if (args.modified) {  // the neutral-loss index
            need += bump_size((size_t)p.n_tiles * (p.nb + 1) * sizeof(uint32_t));
            need += bump_size((size_t)p.n_tiles * p.nb * sizeof(uint32_t));
            need += bump_size((size_t)std::max<int64_t>(1, args.qry.n_peaks) * sizeof(Entry));
        }
        need += bump_size((size_t)p.spill_cap * sizeof(int2));
        need += bump_size(gpool_bytes);
    }
    need += 4096;
    rc = arena_reserve(ctx, ctx->scratch, need, s);
    if (rc) return rc;
    if (!ctx->graphs) return enqueue_cosine(ctx, args, dense, sparse, p, s);
    return run_cosine_graph(ctx, args, dense, sparse, p, s);
}

// The launch sequence of one call, into scratch already reserved for plan p
// (no allocation or synchronisation inside, so that it can be captured).
int enqueue_cosine(cms_ctx* ctx, const CosineArgs& args, const DenseOut* dense,
                   const SparseOut* sparse, const Plan& p, cudaStream_t s) {
    int rc = CMS_OK;
    const int sym = p.sym;
    const size_t pair_smem = (size_t)p.cap * 12 + 2 * 2048 * 4;
    const int64_t nR = args.ref.n, nQ = args.qry.n;
    const size_t gpool_warps = (size_t)ctx->sm_count * 64;
    const size_t gpool_bytes = gpool_warps * (size_t)kGPool * 16;
    Bump bp{(char*)ctx->scratch.ptr, 0, ctx->scratch.bytes};
    uint64_t* small = bp.take<uint64_t>(64);
    uint32_t* bad = reinterpret_cast<uint32_t*>(small);            // word 0
    uint32_t* cls_count = reinterpret_cast<uint32_t*>(small + 1);  // 17 words
    uint32_t* cls_cursor = reinterpret_cast<uint32_t*>(small + 10);  // 17 words
    unsigned int* spill_count = reinterpret_cast<unsigned int*>(small + 20);
    unsigned long long* work_join = reinterpret_cast<unsigned long long*>(small + 21);
    unsigned long long* work_pair = reinterpret_cast<unsigned long long*>(small + 22);
    double* snR = bp.take<double>(nR);
    double* snQ = bp.take<double>(nQ);
    CMS_CUDA_TRY(cudaMemsetAsync(small, 0, 64 * sizeof(uint64_t), s));

    const int threads = 256;
    auto grid_for = [&](int64_t n, int per_block) {
        int64_t g = (n + per_block - 1) / per_block;
        return (int)std::max<int64_t>(1, std::min<int64_t>(g, (int64_t)ctx->sm_count * 32));
    };
    {
        StageScope sc(ctx, 0, 4, s);
        const int max_peaks = args.modified ? kModifiedMaxPeaks : CMS_MAX_PEAKS;
        validate_kernel<<<grid_for(nR, threads), threads, 0, s>>>(args.ref, bad, ctx->err_word,
                                                                 max_peaks);
        validate_kernel<<<grid_for(nQ, threads), threads, 0, s>>>(args.qry, bad, ctx->err_word,
                                                                 max_peaks);
        norms_kernel<<<grid_for(nR, threads), threads, 0, s>>>(args.ref, snR, bad);
        norms_kernel<<<grid_for(nQ, threads), threads, 0, s>>>(args.qry, snQ, bad);
    }
    CMS_CUDA_TRY(cudaGetLastError());

    if (sparse) CMS_CUDA_TRY(cudaMemsetAsync(sparse->count, 0, sizeof(unsigned long long), s));

    PairParams pp{};
    pp.R = args.ref;
    pp.Q = args.qry;
    pp.snR = snR;
    pp.snQ = snQ;
    pp.tol = args.tol;
    pp.shift = args.shift;
    pp.match_limit = args.match_limit;
    pp.cap = p.cap;
    pp.pairs = nullptr;
    pp.n_pairs = nullptr;
    pp.pairs_cap = 0;
    pp.work = work_pair;
    pp.dense = dense ? *dense : DenseOut{nullptr, nullptr, nullptr, 0};
    pp.sparse = sparse ? *sparse : SparseOut{};
    pp.sparse.mirror = sym;
    pp.err = ctx->err_word;
    pp.bad = bad;
    pp.sym = sym;
    // dense symmetric output: the lower triangle is copied from the upper
    // one once every pair kernel has written it
    auto mirror = [&]() -> int {
        if (!sym || sparse) return CMS_OK;
        return launch_mirror(pp.dense, nR, bad, ctx->sm_count, s);
    };

    void (*pair_k)(PairParams) =
        sparse ? (args.modified ? pair_kernel<true, true> : pair_kernel<true, false>)
               : (args.modified ? pair_kernel<false, true> : pair_kernel<false, false>);
    int pair_blocks_per_sm = 1;
    if ((rc = set_func_smem(pair_k, pair_smem))) return rc;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pair_blocks_per_sm, pair_k, p.pair_threads,
                                                  pair_smem);
    pair_blocks_per_sm = std::max(1, pair_blocks_per_sm);
    const int pair_grid = ctx->sm_count * pair_blocks_per_sm;

    if (p.mode == 2 &&
        pair_smem + (size_t)p.cap * 12 + (size_t)p.pair_threads * 72 <= ctx->smem_optin) {
        // whole matrix: the pipelined pair kernel (pair_threads producers
        // plus a consumer warp, two candidate buffers)
        void (*pipe_k)(PairParams) =
            sparse ? (args.modified ? pair_kernel_pipe<true, true> : pair_kernel_pipe<true, false>)
                   : (args.modified ? pair_kernel_pipe<false, true>
                                    : pair_kernel_pipe<false, false>);
        // two candidate buffers and the sort's word scratch (8 per producer)
        const size_t pipe_smem = pair_smem + (size_t)p.cap * 12 + (size_t)p.pair_threads * 72;
        const int pipe_threads = p.pair_threads + 32;
        pp.test_stall = test_stall("pair");
        if ((rc = set_func_smem(pipe_k, pipe_smem))) return rc;
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pipe_k, pipe_threads, pipe_smem);
        StageScope sc(ctx, 4, 1, s);
        pipe_k<<<ctx->sm_count * std::max(1, per_sm), pipe_threads, pipe_smem, s>>>(pp);
        CMS_CUDA_TRY(cudaGetLastError());
        return mirror();
    }
    if (p.mode == 2) {  // one candidate buffer only fits
        StageScope sc(ctx, 4, 1, s);
        pair_k<<<pair_grid, p.pair_threads, pair_smem, s>>>(pp);
        CMS_CUDA_TRY(cudaGetLastError());
        return mirror();
    }

    // ---- mode 1: order, index, join, spill ----
    int32_t* order = bp.take<int32_t>(nR);
    uint32_t* tab = bp.take<uint32_t>((size_t)p.n_tiles * (p.nb + 1));
    uint32_t* cur = bp.take<uint32_t>((size_t)p.n_tiles * p.nb);
    Entry* ent = bp.take<Entry>((size_t)std::max<int64_t>(1, args.qry.n_peaks));
    uint32_t* tab2 = nullptr;
    uint32_t* cur2 = nullptr;
    Entry* ent2 = nullptr;
    if (args.modified) {
        tab2 = bp.take<uint32_t>((size_t)p.n_tiles * (p.nb + 1));
        cur2 = bp.take<uint32_t>((size_t)p.n_tiles * p.nb);
        ent2 = bp.take<Entry>((size_t)std::max<int64_t>(1, args.qry.n_peaks));
    }
    int2* spill = bp.take<int2>(p.spill_cap);
    unsigned char* gpool = bp.take<unsigned char>(gpool_bytes);

    {
        StageScope sc(ctx, 1, 2, s);
        order_count_kernel<<<grid_for(nR, threads), threads, 0, s>>>(args.ref, cls_count, bad);
        order_scatter_kernel<<<grid_for(nR, threads), threads, 0, s>>>(args.ref, cls_count,
                                                                       cls_cursor, order, bad);
    }
    IndexGeom g{p.tile, p.n_tiles, p.nb, 1.0 / p.width};
    {
        StageScope sc(ctx, 2, 3, s);
        CMS_CUDA_TRY(cudaMemsetAsync(cur, 0, (size_t)p.n_tiles * p.nb * sizeof(uint32_t), s));
        index_count_kernel<false><<<grid_for(nQ * 32, threads), threads, 0, s>>>(args.qry, g, cur, bad);
        index_scan_kernel<<<p.n_tiles, 1024, 0, s>>>(g, cur, tab, bad);
        index_scatter_kernel<false><<<grid_for(nQ * 32, threads), threads, 0, s>>>(args.qry, g, cur,
                                                                            ent, bad);
    }
    if (args.modified) {  // neutral-loss index: m/z - precursor, same geometry
        StageScope sc(ctx, 2, 3, s);
        CMS_CUDA_TRY(cudaMemsetAsync(cur2, 0, (size_t)p.n_tiles * p.nb * sizeof(uint32_t), s));
        index_count_kernel<true><<<grid_for(nQ * 32, threads), threads, 0, s>>>(args.qry, g, cur2,
                                                                                bad);
        index_scan_kernel<<<p.n_tiles, 1024, 0, s>>>(g, cur2, tab2, bad);
        index_scatter_kernel<true><<<grid_for(nQ * 32, threads), threads, 0, s>>>(args.qry, g, cur2,
                                                                                  ent2, bad);
    }
    CMS_CUDA_TRY(cudaGetLastError());

    JoinParams jp{};
    jp.A = args.ref;
    jp.B = args.qry;
    jp.snA = snR;
    jp.snB = snQ;
    jp.a_order = order;
    jp.tab = tab;
    jp.ent = ent;
    jp.tab2 = tab2;
    jp.ent2 = ent2;
    jp.g = g;
    jp.tol = args.tol;
    jp.shift = args.shift;
    jp.match_limit = args.match_limit;
    jp.init_width_scale = 0.f;
    for (int c = 0; c < kOrderClasses; ++c) jp.width_by_class[c] = p.width_by_class[c];
    if (p.cand_per_pair > 0.0 && args.ref.n > 0) {
        // expected candidates of (A spectrum with n peaks, w queries) ~ n*w*lambda
        const double mean_na = (double)args.ref.n_peaks / (double)args.ref.n;
        const double lambda = p.cand_per_pair / std::max(1.0, mean_na);
        jp.init_width_scale = (float)(0.5 * kPoolMax / lambda);
    }
    jp.warp_smem_bytes = warp_slice_bytes(p.tile);
    jp.pool_max = kPoolMax;
    jp.max_fetch = 0;
    jp.gpool = gpool;
    jp.work = work_join;
    jp.spill = SpillList{spill, spill_count, p.spill_cap};
    jp.dense = pp.dense;
    jp.sparse = pp.sparse;
    jp.err = ctx->err_word;
    jp.bad = bad;
    jp.sym = sym;
    const size_t join_smem = (size_t)warp_slice_bytes(p.tile) * kJoinWarps;
    {
        StageScope sc(ctx, 3, 1, s);
        const bool noshift = args.shift == 0.0;
        const int64_t items = nR * (int64_t)p.n_tiles;
        if (args.modified)  // shift 0 at the first pass; the second takes it per pair
            rc = sparse ? launch_join<true, true, true, true>(ctx, jp, join_smem, gpool_warps, items, s)
                        : launch_join<true, false, true, true>(ctx, jp, join_smem, gpool_warps, items,
                                                                s);
        else
        rc = sparse
                 ? (noshift ? launch_join<true, true, true, false>(ctx, jp, join_smem, gpool_warps,
                                                                   items, s)
                            : launch_join<true, true, false, false>(ctx, jp, join_smem, gpool_warps,
                                                                    items, s))
                 : (noshift ? launch_join<true, false, true, false>(ctx, jp, join_smem, gpool_warps,
                                                                    items, s)
                            : launch_join<true, false, false, false>(ctx, jp, join_smem, gpool_warps,
                                                                     items, s));
        if (rc) return rc;
    }
    CMS_CUDA_TRY(cudaGetLastError());

    pp.pairs = spill;
    pp.n_pairs = spill_count;
    pp.pairs_cap = p.spill_cap;
    {
        StageScope sc(ctx, 4, 1, s);
        pair_k<<<pair_grid, p.pair_threads, pair_smem, s>>>(pp);
        CMS_CUDA_TRY(cudaGetLastError());
    }
    return mirror();
}

// Graph path of run_cosine: replay a captured launch sequence whose key (every
// value the sequence bakes in) equals this call's, else capture it on the
// context's capture stream, instantiate and keep it (most recent first, at
// most kGraphCache per context); graphs are launched on the caller's stream.
constexpr size_t kGraphCache = 8;
int run_cosine_graph(cms_ctx* ctx, const CosineArgs& args, const DenseOut* dense,
                     const SparseOut* sparse, const Plan& p, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CMS_CUDA_TRY(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone)  // the caller is capturing: just enqueue
        return enqueue_cosine(ctx, args, dense, sparse, p, s);
    std::vector<uint64_t> key;
    key.reserve(48);
    auto put = [&](auto v) {
        static_assert(sizeof(v) <= sizeof(uint64_t), "key field too wide");
        uint64_t u = 0;
        std::memcpy(&u, &v, sizeof(v));
        key.push_back(u);
    };
    auto put_set = [&](const SpecSet& x) {
        put((uintptr_t)x.mz);
        put((uintptr_t)x.a);
        put((uintptr_t)x.b);
        put((uintptr_t)x.off);
        put(x.n);
        put(x.n_peaks);
    };
    put_set(args.ref);
    put_set(args.qry);
    put(args.tol);
    put(args.shift);
    put(args.match_limit);
    put((int)args.modified);
    put((uintptr_t)args.ref.prec);
    put((uintptr_t)args.qry.prec);
    put((int)(dense != nullptr));
    if (dense) {
        put((uintptr_t)dense->score);
        put((uintptr_t)dense->matches);
        put((uintptr_t)dense->overflow);
        put(dense->ld);
    }
    put((int)(sparse != nullptr));
    if (sparse) {
        put((uintptr_t)sparse->r);
        put((uintptr_t)sparse->q);
        put((uintptr_t)sparse->score);
        put((uintptr_t)sparse->matches);
        put((uintptr_t)sparse->overflow);
        put((uintptr_t)sparse->count);
        put(sparse->capacity);
        put(sparse->threshold);
        put(sparse->mirror);
    }
    put(p.mode);
    put(p.tile);
    put(p.nb);
    put(p.width);
    put(p.pair_threads);
    put(p.cap);
    put(p.spill_cap);
    put(p.sym);
    put(p.cand_per_pair);
    for (int c = 0; c < kOrderClasses; ++c) put(p.width_by_class[c]);
    put((uintptr_t)ctx->scratch.ptr);
    put(ctx->scratch.bytes);
    put((uintptr_t)ctx->trace_rec);
    put((uintptr_t)ctx->trace_count);
    put(ctx->trace_cap);
    put(ctx->trace_tag);

    auto& cache = ctx->graph_cache;
    for (size_t i = 0; i < cache.size(); ++i) {
        if (cache[i].key != key) continue;
        if (i) std::rotate(cache.begin(), cache.begin() + i, cache.begin() + i + 1);
        for (int k = 0; k < CMS_PROFILE_STAGES; ++k) ctx->launches[k] += cache[0].launches[k];
        CMS_CUDA_TRY(cudaGraphLaunch(cache[0].exec, s));
        return CMS_OK;
    }

    if (!ctx->capture_stream)
        CMS_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->capture_stream, cudaStreamNonBlocking));
    cudaStream_t cs_stream = ctx->capture_stream;
    int64_t before[CMS_PROFILE_STAGES];
    std::memcpy(before, ctx->launches, sizeof(before));
    CMS_CUDA_TRY(cudaStreamBeginCapture(cs_stream, cudaStreamCaptureModeRelaxed));
    ctx->capturing = true;
    const int rc = enqueue_cosine(ctx, args, dense, sparse, p, cs_stream);
    ctx->capturing = false;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(cs_stream, &g);
    if (rc != CMS_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
        if (rc != CMS_OK) return rc;
        return cuda_fail(e, "cudaStreamEndCapture");
    }
    cms_graph_entry entry;
    entry.key = std::move(key);
    const cudaError_t ei = cudaGraphInstantiate(&entry.exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate");
    for (int k = 0; k < CMS_PROFILE_STAGES; ++k) entry.launches[k] = ctx->launches[k] - before[k];
    if (cache.size() >= kGraphCache) {
        cudaGraphExecDestroy(cache.back().exec);
        cache.pop_back();
    }
    cache.insert(cache.begin(), std::move(entry));
    CMS_CUDA_TRY(cudaGraphLaunch(cache[0].exec, s));
    return CMS_OK;
}

bool check_common(const CosineArgs& a, const char* who) {
    if (!check_specset(a.ref, "reference") || !check_specset(a.qry, "query")) return false;
    if (a.match_limit < 1 || !(a.tol >= 0.0) || !std::isfinite(a.tol) || !std::isfinite(a.shift)) {
        set_error("%s: invalid match_limit or tolerance/shift", who);
        return false;
    }
    return true;
}

}  // namespace
}  // namespace cms

extern "C" int cms_cosine_greedy(cms_ctx* ctx, const float* ref_mz, const double* ref_a,
                                 const double* ref_b, const int64_t* ref_off, int64_t n_ref,
                                 int64_t n_ref_peaks, const float* q_mz, const double* q_a,
                                 const double* q_b, const int64_t* q_off, int64_t n_q,
                                 int64_t n_q_peaks, double tolerance, double shift,
                                 int match_limit, float* score, int32_t* matches,
                                 uint8_t* overflow, int64_t ld, const cms_cosine_config* cfg,
                                 void* stream) {
    using namespace cms;
    if (!ctx) {
        set_error("cms_cosine_greedy: null context");
        return CMS_ERR_INVALID;
    }
    CosineArgs args{SpecSet{ref_mz, ref_a, ref_b, ref_off, n_ref, n_ref_peaks},
                    SpecSet{q_mz, q_a, q_b, q_off, n_q, n_q_peaks}, tolerance, shift,
                    match_limit};
    if (!check_common(args, "cms_cosine_greedy")) return CMS_ERR_INVALID;
    if (ld < n_q) {
        set_error("cms_cosine_greedy: ld < n_q");
        return CMS_ERR_INVALID;
    }
    if (n_ref == 0 || n_q == 0) return CMS_OK;
    if (!score || !matches || !overflow) {
        set_error("cms_cosine_greedy: null output pointer");
        return CMS_ERR_INVALID;
    }
    CMS_CUDA_TRY(cudaSetDevice(ctx->device));
    DenseOut out{score, matches, overflow, ld};
    return run_cosine(ctx, args, &out, nullptr, cfg, (cudaStream_t)stream);
}

extern "C" int cms_cosine_greedy_sparse(cms_ctx* ctx, const float* ref_mz, const double* ref_a,
                                        const double* ref_b, const int64_t* ref_off, int64_t n_ref,
                                        int64_t n_ref_peaks, const float* q_mz,
                                        const double* q_a, const double* q_b,
                                        const int64_t* q_off, int64_t n_q, int64_t n_q_peaks,
                                        double tolerance, double shift, int match_limit,
                                        float threshold, int32_t* hit_ref, int32_t* hit_query,
                                        float* hit_score, int32_t* hit_matches,
                                        uint8_t* hit_overflow, int64_t capacity,
                                        int64_t* hit_count, const cms_cosine_config* cfg,
                                        void* stream) {
    using namespace cms;
    if (!ctx) {
        set_error("cms_cosine_greedy_sparse: null context");
        return CMS_ERR_INVALID;
    }
    CosineArgs args{SpecSet{ref_mz, ref_a, ref_b, ref_off, n_ref, n_ref_peaks},
                    SpecSet{q_mz, q_a, q_b, q_off, n_q, n_q_peaks}, tolerance, shift,
                    match_limit};
    if (!check_common(args, "cms_cosine_greedy_sparse")) return CMS_ERR_INVALID;
    if (!(threshold > 0.0f)) {
        set_error("cms_cosine_greedy_sparse: threshold must be > 0 (every pair scores >= 0)");
        return CMS_ERR_INVALID;
    }
    if (capacity < 0 || !hit_count || (capacity > 0 && (!hit_ref || !hit_query || !hit_score ||
                                                        !hit_matches || !hit_overflow))) {
        set_error("cms_cosine_greedy_sparse: invalid hit buffers");
        return CMS_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    CMS_CUDA_TRY(cudaSetDevice(ctx->device));
    if (n_ref == 0 || n_q == 0) {
        CMS_CUDA_TRY(cudaMemsetAsync(hit_count, 0, sizeof(int64_t), s));
        return CMS_OK;
    }
    SparseOut out{hit_ref, hit_query, hit_score, hit_matches, hit_overflow, capacity,
                  reinterpret_cast<unsigned long long*>(hit_count), threshold};
    return run_cosine(ctx, args, nullptr, &out, cfg, s);
}

extern "C" int cms_modified_cosine(cms_ctx* ctx, const float* ref_mz, const double* ref_a,
                                   const double* ref_b, const int64_t* ref_off,
                                   const double* ref_precursor, int64_t n_ref, int64_t n_ref_peaks,
                                   const float* q_mz, const double* q_a, const double* q_b,
                                   const int64_t* q_off, const double* q_precursor, int64_t n_q,
                                   int64_t n_q_peaks, double tolerance, int match_limit,
                                   float* score, int32_t* matches, uint8_t* overflow, int64_t ld,
                                   const cms_cosine_config* cfg, void* stream) {
    using namespace cms;
    if (!ctx) {
        set_error("cms_modified_cosine: null context");
        return CMS_ERR_INVALID;
    }
    CosineArgs args{SpecSet{ref_mz, ref_a, ref_b, ref_off, n_ref, n_ref_peaks, ref_precursor},
                    SpecSet{q_mz, q_a, q_b, q_off, n_q, n_q_peaks, q_precursor}, tolerance, 0.0,
                    match_limit, true};
    if (!check_common(args, "cms_modified_cosine")) return CMS_ERR_INVALID;
    if (ld < n_q) {
        set_error("cms_modified_cosine: ld < n_q");
        return CMS_ERR_INVALID;
    }
    if (n_ref == 0 || n_q == 0) return CMS_OK;
    if (!score || !matches || !overflow || !ref_precursor || !q_precursor) {
        set_error("cms_modified_cosine: null output or precursor pointer");
        return CMS_ERR_INVALID;
    }
    CMS_CUDA_TRY(cudaSetDevice(ctx->device));
    DenseOut out{score, matches, overflow, ld};
    return run_cosine(ctx, args, &out, nullptr, cfg, (cudaStream_t)stream);
}

extern "C" int cms_modified_cosine_sparse(
    cms_ctx* ctx, const float* ref_mz, const double* ref_a, const double* ref_b,
    const int64_t* ref_off, const double* ref_precursor, int64_t n_ref, int64_t n_ref_peaks,
    const float* q_mz, const double* q_a, const double* q_b, const int64_t* q_off,
    const double* q_precursor, int64_t n_q, int64_t n_q_peaks, double tolerance, int match_limit,
    float threshold, int32_t* hit_ref, int32_t* hit_query, float* hit_score, int32_t* hit_matches,
    uint8_t* hit_overflow, int64_t capacity, int64_t* hit_count, const cms_cosine_config* cfg,
    void* stream) {
    using namespace cms;
    if (!ctx) {
        set_error("cms_modified_cosine_sparse: null context");
        return CMS_ERR_INVALID;
    }
    CosineArgs args{SpecSet{ref_mz, ref_a, ref_b, ref_off, n_ref, n_ref_peaks, ref_precursor},
                    SpecSet{q_mz, q_a, q_b, q_off, n_q, n_q_peaks, q_precursor}, tolerance, 0.0,
                    match_limit, true};
    if (!check_common(args, "cms_modified_cosine_sparse")) return CMS_ERR_INVALID;
    if (!(threshold > 0.0f)) {
        set_error("cms_modified_cosine_sparse: threshold must be > 0 (every pair scores >= 0)");
        return CMS_ERR_INVALID;
    }
    if (capacity < 0 || !hit_count || (capacity > 0 && (!hit_ref || !hit_query || !hit_score ||
                                                        !hit_matches || !hit_overflow))) {
        set_error("cms_modified_cosine_sparse: invalid hit buffers");
        return CMS_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    CMS_CUDA_TRY(cudaSetDevice(ctx->device));
    if (n_ref == 0 || n_q == 0) {
        CMS_CUDA_TRY(cudaMemsetAsync(hit_count, 0, sizeof(int64_t), s));
        return CMS_OK;
    }
    if (!ref_precursor || !q_precursor) {
        set_error("cms_modified_cosine_sparse: null precursor pointer");
        return CMS_ERR_INVALID;
    }
    SparseOut out{hit_ref, hit_query, hit_score, hit_matches, hit_overflow, capacity,
                  reinterpret_cast<unsigned long long*>(hit_count), threshold};
    return run_cosine(ctx, args, nullptr, &out, cfg, s);
}

// ---------------------------------------------------------------------------
// Allocation-free variant (cms_cosine_greedy_noalloc)
//
// Some callers cannot let a library call cudaMalloc: an application whose
// device memory is already reserved by its own allocator (a framework's
// caching pool that owns almost all of the GPU), a latency-critical loop that
// cannot afford the device-wide synchronisation cudaMalloc/cudaFree may
// imply, or a plugin host that forbids libraries to allocate behind its back.
// For them this entry point runs the dense greedy cosine with the pair kernel
// over every pair, and keeps its only scratch -- validity flags and the two
// per-spectrum norm arrays -- in the fixed device array below instead of a
// context's arena.  The array is part of the library's device image: every
// GPU that loads the library holds it until the process exits.
// ---------------------------------------------------------------------------
namespace cms {
namespace {

constexpr int64_t kNoAllocMaxSpectra = int64_t(1) << 20;  // n_ref + n_q
constexpr size_t kNoAllocHeader = 256;                     // flags and error word
constexpr size_t kNoAllocBytes = kNoAllocHeader + 8 * (size_t)kNoAllocMaxSpectra + 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device, with that device current, and cached.
int noalloc_scratch(unsigned char** out) {
    int dev = 0;
    CMS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("cms_cosine_greedy_noalloc: device ordinal %d out of range", dev);
        return CMS_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return CMS_OK;
}

}  // namespace
}  // namespace cms

extern "C" int cms_cosine_greedy_noalloc(const float* ref_mz, const double* ref_a,
                                         const double* ref_b, const int64_t* ref_off,
                                         int64_t n_ref, int64_t n_ref_peaks, const float* q_mz,
                                         const double* q_a, const double* q_b,
                                         const int64_t* q_off, int64_t n_q, int64_t n_q_peaks,
                                         double tolerance, double shift, int match_limit,
                                         float* score, int32_t* matches, uint8_t* overflow,
                                         int64_t ld, uint32_t* device_error, void* stream) {
    using namespace cms;
    CosineArgs args{SpecSet{ref_mz, ref_a, ref_b, ref_off, n_ref, n_ref_peaks},
                    SpecSet{q_mz, q_a, q_b, q_off, n_q, n_q_peaks}, tolerance, shift,
                    match_limit};
    if (!check_common(args, "cms_cosine_greedy_noalloc")) return CMS_ERR_INVALID;
    if (ld < n_q) {
        set_error("cms_cosine_greedy_noalloc: ld < n_q");
        return CMS_ERR_INVALID;
    }
    if (n_ref + n_q > kNoAllocMaxSpectra) {
        set_error("cms_cosine_greedy_noalloc: n_ref + n_q = %lld exceeds the fixed scratch "
                  "capacity of %lld spectra; split the call or use cms_cosine_greedy",
                  (long long)(n_ref + n_q), (long long)kNoAllocMaxSpectra);
        return CMS_ERR_UNSUPPORTED;
    }
    if (match_limit > 4096) {
        set_error("cms_cosine_greedy_noalloc: match_limit must be <= 4096");
        return CMS_ERR_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (n_ref == 0 || n_q == 0) {
        if (device_error) CMS_CUDA_TRY(cudaMemsetAsync(device_error, 0, sizeof(uint32_t), s));
        return CMS_OK;
    }
    if (!score || !matches || !overflow) {
        set_error("cms_cosine_greedy_noalloc: null output pointer");
        return CMS_ERR_INVALID;
    }
    // Every buffer must be memory of the current device: the scratch address
    // below is the current device's, and a kernel handed another GPU's (or
    // host) memory would read or write out of bounds.  Nothing is launched
    // before these checks.
    const char* who = "cms_cosine_greedy_noalloc";
    const std::pair<const void*, const char*> bufs[] = {
        {ref_mz, "ref_mz"}, {ref_a, "ref_a"}, {ref_b, "ref_b"}, {ref_off, "ref_off"},
        {q_mz, "q_mz"},     {q_a, "q_a"},     {q_b, "q_b"},     {q_off, "q_off"},
        {score, "score"},   {matches, "matches"}, {overflow, "overflow"},
        {device_error, "device_error"}};
    int rc = CMS_OK;
    for (const auto& bf : bufs)
        if (bf.first && (rc = check_device_ptr(bf.first, who, bf.second))) return rc;
    if (s) {
        int sdev = -1, dev = 0;
        CMS_CUDA_TRY(cudaStreamGetDevice(s, &sdev));
        CMS_CUDA_TRY(cudaGetDevice(&dev));
        if (sdev != dev) {
            set_error("%s: stream belongs to device %d, not the current device %d", who, sdev,
                      dev);
            return CMS_ERR_INVALID;
        }
    }
    unsigned char* base = nullptr;
    rc = noalloc_scratch(&base);
    if (rc) return rc;
    uint32_t* bad = reinterpret_cast<uint32_t*>(base);
    uint32_t* err = reinterpret_cast<uint32_t*>(base + 4);
    double* snR = reinterpret_cast<double*>(base + kNoAllocHeader);
    double* snQ = snR + n_ref;
    // the array keeps the previous call's contents: reset the flags
    CMS_CUDA_TRY(cudaMemsetAsync(base, 0, kNoAllocHeader, s));

    int dev = 0, sms = 0;
    CMS_CUDA_TRY(cudaGetDevice(&dev));
    CMS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int threads = 256;
    auto grid_for = [&](int64_t n) {
        return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads,
                                                           (int64_t)sms * 32));
    };
    validate_kernel<<<grid_for(n_ref), threads, 0, s>>>(args.ref, bad, err);
    validate_kernel<<<grid_for(n_q), threads, 0, s>>>(args.qry, bad, err);
    norms_kernel<<<grid_for(n_ref), threads, 0, s>>>(args.ref, snR, bad);
    norms_kernel<<<grid_for(n_q), threads, 0, s>>>(args.qry, snQ, bad);
    CMS_CUDA_TRY(cudaGetLastError());

    PairParams pp{};
    pp.R = args.ref;
    pp.Q = args.qry;
    pp.snR = snR;
    pp.snQ = snQ;
    pp.tol = tolerance;
    pp.shift = shift;
    pp.match_limit = match_limit;
    int cap = 2;
    while (cap < match_limit) cap <<= 1;
    pp.cap = cap;
    pp.pairs = nullptr;  // every pair of R x Q, statically strided
    pp.n_pairs = nullptr;
    pp.pairs_cap = 0;
    pp.work = reinterpret_cast<unsigned long long*>(base + 8);
    pp.dense = DenseOut{score, matches, overflow, ld};
    pp.sparse = SparseOut{};
    pp.err = err;
    pp.bad = bad;
    const int pair_threads = 128;
    const size_t pair_smem = (size_t)cap * 12 + 2 * 2048 * 4;
    if ((rc = set_func_smem(pair_kernel<false, false>, pair_smem))) return rc;
    int per_sm = 1;
    CMS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pair_kernel<false, false>,
                                                               pair_threads, pair_smem));
    pair_kernel<false, false><<<sms * std::max(1, per_sm), pair_threads, pair_smem, s>>>(pp);
    CMS_CUDA_TRY(cudaGetLastError());
    if (device_error)
        CMS_CUDA_TRY(cudaMemcpyAsync(device_error, err, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    return CMS_OK;
}


// ---------------------------------------------------------------------------
// Resident library (cms_library_*): the indexed side built once, searched by
// many query batches.
// ---------------------------------------------------------------------------
struct cms_library {
    int device = 0;
    cms::SpecSet spec{};  // caller-owned device arrays; must outlive the library
    double tol = 0.0, shift = 0.0, cand_per_pair = 0.0;
    int match_limit = 1;
    cms::IndexGeom g{};
    double* sn = nullptr;
    uint32_t* tab = nullptr;
    cms::Entry* ent = nullptr;
    uint32_t* bad = nullptr;
};

namespace {
void library_free(cms_library* L) {
    if (!L) return;
    cudaFree(L->sn);
    cudaFree(L->tab);
    cudaFree(L->ent);
    cudaFree(L->bad);
    delete L;
}
}  // namespace

extern "C" int cms_library_create(cms_ctx* ctx, const float* mz, const double* a, const double* b,
                                  const int64_t* off, int64_t n, int64_t n_peaks,
                                  double tolerance, double shift, int match_limit,
                                  const cms_cosine_config* cfg, cms_library** out, void* stream) {
    using namespace cms;
    if (!ctx || !out) {
        set_error("cms_library_create: null context or output");
        return CMS_ERR_INVALID;
    }
    *out = nullptr;
    CosineArgs args{SpecSet{mz, a, b, off, n, n_peaks}, SpecSet{mz, a, b, off, n, n_peaks},
                    tolerance, shift, match_limit};
    if (!check_common(args, "cms_library_create")) return CMS_ERR_INVALID;
    if (n <= 0) {
        set_error("cms_library_create: empty library");
        return CMS_ERR_INVALID;
    }
    CMS_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    cms_library* L = new cms_library();
    L->device = ctx->device;
    L->spec = args.ref;
    L->tol = tolerance;
    L->shift = shift;
    L->match_limit = match_limit;
    L->cand_per_pair = (cfg && cfg->cand_per_pair > 0.0) ? cfg->cand_per_pair : 0.0;
    const int tile = (int)std::min<int64_t>((cfg && cfg->tile_spectra > 0) ? cfg->tile_spectra
                                                                            : 1024, n);
    if (tile > kMaxTile) {
        delete L;
        set_error("cms_library_create: tile_spectra must be <= %d", kMaxTile);
        return CMS_ERR_UNSUPPORTED;
    }
    double w = (cfg && cfg->bucket_width > 0.0) ? cfg->bucket_width : 2.0 * tolerance;
    if (w < tolerance) w = tolerance;
    if (!(w > 0.0)) w = 1e-3;
    const double avg_tile_peaks = (double)n_peaks * tile / (double)n;
    int nb = (cfg && cfg->n_buckets > 0) ? next_pow2(cfg->n_buckets)
                                         : next_pow2((long long)std::max(1024.0, avg_tile_peaks));
    nb = std::min(nb, 1 << 22);
    L->g = IndexGeom{tile, (int)((n + tile - 1) / tile), nb, 1.0 / w};
    const size_t n_tab = (size_t)L->g.n_tiles * (nb + 1), n_cur = (size_t)L->g.n_tiles * nb;
    uint32_t* cur = nullptr;
    cudaError_t e = cudaMalloc(&L->bad, 64);
    if (e == cudaSuccess) e = cudaMalloc(&L->sn, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&L->tab, sizeof(uint32_t) * n_tab);
    if (e == cudaSuccess) e = cudaMalloc(&L->ent, sizeof(Entry) * std::max<int64_t>(1, n_peaks));
    if (e == cudaSuccess) e = cudaMalloc(&cur, sizeof(uint32_t) * n_cur);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        cudaFree(cur);
        library_free(L);
        set_error("cms_library_create: device allocation failed (%s)", cudaGetErrorString(e));
        return CMS_ERR_NOMEM;
    }
    const int threads = 256;
    auto grid_for = [&](int64_t cnt) {
        return (int)std::max<int64_t>(1, std::min<int64_t>((cnt + threads - 1) / threads,
                                                           (int64_t)ctx->sm_count * 32));
    };
    e = cudaMemsetAsync(L->bad, 0, 64, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cur, 0, sizeof(uint32_t) * n_cur, s);
    if (e == cudaSuccess) {
        validate_kernel<<<grid_for(n), threads, 0, s>>>(L->spec, L->bad, ctx->err_word);
        norms_kernel<<<grid_for(n), threads, 0, s>>>(L->spec, L->sn, L->bad);
        index_count_kernel<false><<<grid_for(n * 32), threads, 0, s>>>(L->spec, L->g, cur, L->bad);
        index_scan_kernel<<<L->g.n_tiles, 1024, 0, s>>>(L->g, cur, L->tab, L->bad);
        index_scatter_kernel<false><<<grid_for(n * 32), threads, 0, s>>>(L->spec, L->g, cur, L->ent,
                                                                  L->bad);
        e = cudaGetLastError();
    }
    uint32_t hbad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, L->bad, sizeof(uint32_t),
                                              cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(cur);
    if (e != cudaSuccess) {
        library_free(L);
        return cuda_fail(e, "cms_library_create");
    }
    if (hbad) {
        library_free(L);
        set_error("cms_library_create: invalid library spectra (offsets or peak counts)");
        return CMS_ERR_DEVICE;
    }
    *out = L;
    return CMS_OK;
}

extern "C" int cms_library_destroy(cms_library* lib) {
    if (!lib) return CMS_OK;
    cudaSetDevice(lib->device);
    cudaDeviceSynchronize();
    library_free(lib);
    return CMS_OK;
}

extern "C" int cms_library_search(cms_ctx* ctx, const cms_library* lib, const float* q_mz,
                                  const double* q_a, const double* q_b, const int64_t* q_off,
                                  int64_t n_q, int64_t n_q_peaks, float threshold,
                                  int32_t* hit_ref, int32_t* hit_query, float* hit_score,
                                  int32_t* hit_matches, uint8_t* hit_overflow, int64_t capacity,
                                  int64_t* hit_count, void* stream) {
    using namespace cms;
    if (!ctx || !lib) {
        set_error("cms_library_search: null context or library");
        return CMS_ERR_INVALID;
    }
    if (ctx->device != lib->device) {
        set_error("cms_library_search: context and library are on different devices");
        return CMS_ERR_INVALID;
    }
    const SpecSet Q{q_mz, q_a, q_b, q_off, n_q, n_q_peaks};
    if (!check_specset(Q, "query")) return CMS_ERR_INVALID;
    if (!(threshold > 0.0f)) {
        set_error("cms_library_search: threshold must be > 0");
        return CMS_ERR_INVALID;
    }
    if (capacity < 0 || !hit_count || (capacity > 0 && (!hit_ref || !hit_query || !hit_score ||
                                                        !hit_matches || !hit_overflow))) {
        set_error("cms_library_search: invalid hit buffers");
        return CMS_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    CMS_CUDA_TRY(cudaSetDevice(ctx->device));
    CMS_CUDA_TRY(cudaMemsetAsync(hit_count, 0, sizeof(int64_t), s));
    if (n_q == 0) return CMS_OK;

    const int cap = next_pow2(std::max(2, lib->match_limit));
    const size_t pair_smem = (size_t)cap * 12 + 2 * 2048 * 4;
    if (pair_smem > ctx->smem_optin) {
        set_error("cms_library_search: match_limit too large for shared memory");
        return CMS_ERR_UNSUPPORTED;
    }
    const long long items = (long long)n_q * lib->g.n_tiles;
    const unsigned int spill_cap =
        (unsigned int)std::min<long long>(std::max<long long>(1 << 16, items), 1 << 24);
    // global-pool slices for up to four resident CTAs per SM (more CTAs per
    // SM run with the shared-memory pool only)
    const size_t gpool_warps =
        (size_t)std::min(ctx->sm_count * 4, kSlotWords * 32) * kJoinWarps;
    const size_t gpool_bytes = gpool_warps * (size_t)kGPool * 16;
    size_t need = bump_size(64 * sizeof(uint64_t)) + bump_size(n_q * sizeof(double)) +
                  bump_size(n_q * sizeof(int32_t)) + bump_size((size_t)spill_cap * sizeof(int2)) +
                  bump_size(kSlotWords * sizeof(uint32_t)) + bump_size(gpool_bytes) + 4096;
    int rc = arena_reserve(ctx, ctx->scratch, need, s);
    if (rc) return rc;
    Bump bp{(char*)ctx->scratch.ptr, 0, ctx->scratch.bytes};
    uint64_t* small = bp.take<uint64_t>(64);
    uint32_t* bad = reinterpret_cast<uint32_t*>(small);
    uint32_t* cls_count = reinterpret_cast<uint32_t*>(small + 1);
    uint32_t* cls_cursor = reinterpret_cast<uint32_t*>(small + 10);
    unsigned int* spill_count = reinterpret_cast<unsigned int*>(small + 20);
    unsigned long long* work_join = reinterpret_cast<unsigned long long*>(small + 21);
    unsigned long long* work_pair = reinterpret_cast<unsigned long long*>(small + 22);
    double* snQ = bp.take<double>(n_q);
    int32_t* order = bp.take<int32_t>(n_q);
    int2* spill = bp.take<int2>(spill_cap);
    uint32_t* slots = bp.take<uint32_t>(kSlotWords);
    unsigned char* gpool = bp.take<unsigned char>(gpool_bytes);
    CMS_CUDA_TRY(cudaMemsetAsync(small, 0, 64 * sizeof(uint64_t), s));
    CMS_CUDA_TRY(cudaMemsetAsync(slots, 0, kSlotWords * sizeof(uint32_t), s));

    const int threads = 256;
    auto grid_for = [&](int64_t cnt) {
        return (int)std::max<int64_t>(1, std::min<int64_t>((cnt + threads - 1) / threads,
                                                           (int64_t)ctx->sm_count * 32));
    };
    {
        StageScope sc(ctx, 0, 2, s);
        validate_kernel<<<grid_for(n_q), threads, 0, s>>>(Q, bad, ctx->err_word);
        norms_kernel<<<grid_for(n_q), threads, 0, s>>>(Q, snQ, bad);
    }
    {
        StageScope sc(ctx, 1, 2, s);
        order_count_kernel<<<grid_for(n_q), threads, 0, s>>>(Q, cls_count, bad);
        order_scatter_kernel<<<grid_for(n_q), threads, 0, s>>>(Q, cls_count, cls_cursor, order,
                                                               bad);
    }
    CMS_CUDA_TRY(cudaGetLastError());

    SparseOut so{hit_ref, hit_query, hit_score, hit_matches, hit_overflow, capacity,
                 reinterpret_cast<unsigned long long*>(hit_count), threshold};
    JoinParams jp{};  // width_by_class zero: widths from cand_per_pair
    jp.A = Q;
    jp.B = lib->spec;
    jp.snA = snQ;
    jp.snB = lib->sn;
    jp.a_order = order;
    jp.tab = lib->tab;
    jp.ent = lib->ent;
    jp.g = lib->g;
    jp.tol = lib->tol;
    jp.shift = lib->shift;
    jp.match_limit = lib->match_limit;
    // A search runs as kSearchWaves waves of short-lived CTAs (an equal share
    // of fetches per warp) so that searches on other streams interleave with
    // it on the device; each CTA claims a global-pool slice while it lives.
    jp.pool_max = kPoolMax;
    jp.gpool = gpool;
    jp.slots = slots;
    jp.init_width_scale = 0.f;
    if (lib->cand_per_pair > 0.0 && n_q > 0) {
        const double mean_na = (double)n_q_peaks / (double)n_q;
        const double lambda = lib->cand_per_pair / std::max(1.0, mean_na);
        jp.init_width_scale = (float)(0.5 * jp.pool_max / lambda);
    }
    jp.warp_smem_bytes = warp_slice_bytes(lib->g.tile);
    jp.work = work_join;
    jp.spill = SpillList{spill, spill_count, spill_cap};
    jp.dense = DenseOut{nullptr, nullptr, nullptr, 0};
    jp.sparse = so;
    jp.err = ctx->err_word;
    jp.bad = bad;
    {
        StageScope sc(ctx, 3, 1, s);
        rc = launch_join<false, true, false, false>(ctx, jp,
                                                    (size_t)jp.warp_smem_bytes * kJoinWarps,
                                                    gpool_warps, items, s, kSearchWaves);
        if (rc) return rc;
    }
    PairParams pp{};
    pp.R = lib->spec;
    pp.Q = Q;
    pp.snR = lib->sn;
    pp.snQ = snQ;
    pp.tol = lib->tol;
    pp.shift = lib->shift;
    pp.match_limit = lib->match_limit;
    pp.cap = cap;
    pp.pairs = spill;
    pp.n_pairs = spill_count;
    pp.pairs_cap = spill_cap;
    pp.work = work_pair;
    pp.dense = DenseOut{nullptr, nullptr, nullptr, 0};
    pp.sparse = so;
    pp.err = ctx->err_word;
    pp.bad = bad;
    {
        StageScope sc(ctx, 4, 1, s);
        if ((rc = set_func_smem(pair_kernel<true, false>, pair_smem))) return rc;
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pair_kernel<true, false>, 128,
                                                      pair_smem);
        pair_kernel<true, false><<<std::max(1, std::min(ctx->sm_count * std::max(1, per_sm),
                                                  (int)std::min<long long>(spill_cap, 1 << 20))),
                            128, pair_smem, s>>>(pp);
    }
    CMS_CUDA_TRY(cudaGetLastError());
    return CMS_OK;
}
