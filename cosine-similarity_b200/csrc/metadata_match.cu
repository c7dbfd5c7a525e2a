// matchms' metadata and m/z-set similarities that the reference prototypes
// beside its CUDA classes (notebooks/prototyping/other_similarities.ipynb
// imports matchms' ParentMassMatch, PrecursorMzMatch and IntersectMz next to
// CosineGreedy, ModifiedCosine and FingerprintSimilarity):
//
//   mass_match_kernel      ParentMassMatch / PrecursorMzMatch: one value per
//                          spectrum (parent mass or precursor m/z, float64);
//                          a pair matches when |r - q| <= tolerance (Dalton)
//                          or |r - q| / ((r + q) / 2) * 1e6 <= tolerance
//                          (ppm), in IEEE float64 in that order of
//                          operations.  Output: one byte (0/1) per pair.
//                          Pure output bandwidth: a CTA takes a tile of 64
//                          rows x 4096 columns, each thread 16 columns whose
//                          query values stay in registers over the 64 rows,
//                          one 16-byte store per row when the row is aligned.
//   intersect_mz_kernel    IntersectMz: |set(mz_r) & set(mz_q)| / |set(mz_r)
//                          | set(mz_q)| * scaling on the exact float64 m/z
//                          values (0 when both are empty), through a hashed
//                          index of the queries' distinct values: per
//                          (reference, 8192-query tile) the reference's
//                          distinct values find their (value, query) entries
//                          and count them per query in shared memory; then
//                          scaling * inter / union in float64 for the whole
//                          tile row.
#include <algorithm>
#include <cstdint>

#include "cms_internal.cuh"

namespace cms {
namespace {

constexpr int kMassThreads = 256;
constexpr int kMassCols = 16;                              // columns per thread
constexpr int kMassTileCols = kMassThreads * kMassCols;    // 4096
constexpr int kMassTileRows = 64;
constexpr int kIxThreads = 256;

__device__ __forceinline__ bool mass_ok(double r, double q, double tol, int ppm) {
    const double d = fabs(__dsub_rn(r, q));
    if (!ppm) return d <= tol;
    // (r + q) / 2: halving is exact scaling, the same rounding as division
    const double mean = __dmul_rn(__dadd_rn(r, q), 0.5);
    return __dmul_rn(__ddiv_rn(d, mean), 1e6) <= tol;
}

__global__ void __launch_bounds__(kMassThreads) mass_match_kernel(const double* __restrict__ ref,
                                                                  int64_t n_ref,
                                                                  const double* __restrict__ q,
                                                                  int64_t n_q, double tol, int ppm,
                                                                  uint8_t* __restrict__ out,
                                                                  int64_t ld, int vec) {
    const int64_t col_tiles = (n_q + kMassTileCols - 1) / kMassTileCols;
    const int64_t tiles = col_tiles * ((n_ref + kMassTileRows - 1) / kMassTileRows);
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int64_t rt = t / col_tiles, ct = t - rt * col_tiles;
        const int64_t j0 = ct * kMassTileCols + (int64_t)threadIdx.x * kMassCols;
        const int64_t i0 = rt * kMassTileRows, i1 = min(n_ref, i0 + kMassTileRows);
        if (j0 >= n_q) continue;
        const int nc = (int)min((int64_t)kMassCols, n_q - j0);
        double qv[kMassCols];
#pragma unroll
        for (int k = 0; k < kMassCols; ++k) qv[k] = k < nc ? q[j0 + k] : 0.0;
        for (int64_t i = i0; i < i1; ++i) {
            const double r = ref[i];
            uint8_t* o = out + i * ld + j0;
            if (vec && nc == kMassCols) {
                uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
                for (int k = 0; k < kMassCols; ++k)
                    w[k >> 2] |= (uint32_t)mass_ok(r, qv[k], tol, ppm) << (8 * (k & 3));
                __stcs(reinterpret_cast<uint4*>(o), make_uint4(w[0], w[1], w[2], w[3]));
            } else {
#pragma unroll
                for (int k = 0; k < kMassCols; ++k)
                    if (k < nc) o[k] = (uint8_t)mass_ok(r, qv[k], tol, ppm);
            }
        }
    }
}

// [a0, a1) of spectrum i, clamped to [0, total]; a clamp sets the error word
__device__ __forceinline__ void spectrum_range(const int64_t* off, int64_t i, int64_t total,
                                               int64_t& a0, int64_t& a1, uint32_t* err) {
    a0 = off[i];
    a1 = off[i + 1];
    if (a0 < 0 || a1 < a0 || a1 > total) {
        if (err) atomicOr(err, kErrBadOffsets);
        a0 = a1 = 0;
    }
}

// ---- IntersectMz through an index of the queries' distinct m/z values ----
// Pairs sharing a value are few against R x Q, so instead of merging every
// pair's peak lists, the queries' distinct (value, query) entries are hashed
// into buckets (count, scan, scatter), and each (reference, query tile) CTA
// walks the buckets of its reference's distinct values, counting shared
// values per query in shared memory, then writes the tile's dense row.
constexpr int kIxTile = 8192;  // queries per CTA pass (32 KB of counters)

struct IxEntry {
    double v;
    uint32_t q;
    uint32_t pad;
};

// bucket of an m/z value: its bit pattern (+0 and -0 folded) mixed by the
// splitmix64 finalizer
__device__ __forceinline__ uint32_t ix_bucket(double v, uint32_t mask) {
    unsigned long long z = v == 0.0 ? 0ull : (unsigned long long)__double_as_longlong(v);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (uint32_t)z & mask;
}

// one warp per query spectrum: its distinct values (sorted peaks: a value
// differing from its predecessor) counted per bucket (SCATTER = false) or
// placed (SCATTER = true); ub[j] = distinct values of query j
template <bool SCATTER>
__global__ void ix_index_kernel(const double* __restrict__ qmz, const int64_t* __restrict__ qoff,
                                int64_t n_q, int64_t n_q_peaks, uint32_t mask, uint32_t* cnt_cur,
                                IxEntry* ent, uint32_t* ub, uint32_t* err) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; j < n_q; j += warps) {
        int64_t b0, b1;
        spectrum_range(qoff, j, n_q_peaks, b0, b1, (!SCATTER && lane == 0) ? err : nullptr);
        uint32_t distinct = 0;
        for (int64_t k = b0 + lane; k < b1; k += 32) {
            const double v = qmz[k];
            if (k > b0 && qmz[k - 1] == v) continue;
            ++distinct;
            const uint32_t h = ix_bucket(v, mask);
            if (SCATTER) {
                const uint32_t pos = atomicAdd(&cnt_cur[h], 1u);
                ent[pos] = IxEntry{v, (uint32_t)j, 0u};
            } else {
                atomicAdd(&cnt_cur[h], 1u);
            }
        }
        if (!SCATTER) {
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) distinct += __shfl_xor_sync(0xffffffffu, distinct, d);
            if (lane == 0) ub[j] = distinct;
        }
    }
}

// Exclusive scan of the bucket counts into tab[0..nb] (cnt_cur becomes the
// scatter cursor), in three coalesced passes over chunks of kScanChunk
// buckets: chunk sums, a scan of the sums (one CTA), the chunks' own scans.
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 8;
constexpr int kScanChunk = kScanThreads * kScanPer;  // 8192 buckets

// block-wide exclusive scan of one value per thread; *total gets the sum
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t x, uint32_t* warp_sums,
                                                    uint32_t* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
    }
    __syncthreads();  // warp_sums free from an earlier use
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t v = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, v, d);
            if (lane >= d) v += u;
        }
        if (lane < (int)(blockDim.x >> 5)) warp_sums[lane] = v;
    }
    __syncthreads();
    if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
    return incl - x + (wid > 0 ? warp_sums[wid - 1] : 0u);
}

__global__ void __launch_bounds__(kScanThreads) ix_chunk_sums(const uint32_t* cnt, uint32_t nb,
                                                              uint32_t* sums) {
    const uint32_t c0 = blockIdx.x * (uint32_t)kScanChunk;
    uint32_t x = 0;
#pragma unroll
    for (int r = 0; r < kScanPer; ++r) {
        const uint32_t k = c0 + r * kScanThreads + threadIdx.x;
        if (k < nb) x += cnt[k];
    }
    __shared__ uint32_t ws[32];
    uint32_t total;
    block_excl_scan(x, ws, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// exclusive scan of the chunk sums in place (n_chunks <= kScanChunk), and
// tab[nb] = the grand total
__global__ void __launch_bounds__(kScanThreads) ix_scan_sums(uint32_t* sums, int n_chunks,
                                                             uint32_t* tab, uint32_t nb) {
    uint32_t v[kScanPer], x = 0;
#pragma unroll
    for (int r = 0; r < kScanPer; ++r) {
        const int k = threadIdx.x * kScanPer + r;
        v[r] = k < n_chunks ? sums[k] : 0u;
        x += v[r];
    }
    __shared__ uint32_t ws[32];
    uint32_t total;
    uint32_t run = block_excl_scan(x, ws, &total);
#pragma unroll
    for (int r = 0; r < kScanPer; ++r) {
        const int k = threadIdx.x * kScanPer + r;
        if (k < n_chunks) sums[k] = run;
        run += v[r];
    }
    if (threadIdx.x == 0) tab[nb] = total;
}

__global__ void __launch_bounds__(kScanThreads) ix_chunk_scan(uint32_t* cnt_cur, uint32_t* tab,
                                                              uint32_t nb,
                                                              const uint32_t* chunk_base) {
    const uint32_t k0 = blockIdx.x * (uint32_t)kScanChunk + threadIdx.x * kScanPer;
    uint32_t v[kScanPer], x = 0;
#pragma unroll
    for (int r = 0; r < kScanPer; ++r) {
        v[r] = k0 + r < nb ? cnt_cur[k0 + r] : 0u;
        x += v[r];
    }
    __shared__ uint32_t ws[32];
    uint32_t run = chunk_base[blockIdx.x] + block_excl_scan(x, ws, nullptr);
#pragma unroll
    for (int r = 0; r < kScanPer; ++r) {
        if (k0 + r < nb) {
            tab[k0 + r] = run;
            cnt_cur[k0 + r] = run;
        }
        run += v[r];
    }
}

__global__ void __launch_bounds__(kIxThreads) intersect_mz_kernel(
    const double* __restrict__ rmz, const int64_t* __restrict__ roff, int64_t n_ref,
    int64_t n_ref_peaks, int64_t n_q, const uint32_t* __restrict__ tab,
    const IxEntry* __restrict__ ent, const uint32_t* __restrict__ ub, uint32_t mask,
    double scaling, double* __restrict__ out, int64_t ld, uint32_t* err) {
    __shared__ uint32_t s_cnt[kIxTile];
    __shared__ uint32_t s_ua[kIxThreads / 32];
    const int64_t tiles = (n_q + kIxTile - 1) / kIxTile;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int64_t u = blockIdx.x; u < n_ref * tiles; u += gridDim.x) {
        const int64_t i = u / tiles, j0 = (u - i * tiles) * kIxTile;
        const int tw = (int)min((int64_t)kIxTile, n_q - j0);
        __syncthreads();  // the previous unit's readers are done with s_cnt
        for (int k = threadIdx.x; k < tw; k += blockDim.x) s_cnt[k] = 0u;
        __syncthreads();
        int64_t a0, a1;
        spectrum_range(roff, i, n_ref_peaks, a0, a1,
                       (threadIdx.x == 0 && j0 == 0) ? err : nullptr);
        // four threads per distinct reference value, each walking every
        // fourth entry of its bucket with two loads in flight
        uint32_t distinct = 0;
        const int sub = threadIdx.x & 3;
        for (int64_t k = a0 + (threadIdx.x >> 2); k < a1; k += kIxThreads / 4) {
            const double v = rmz[k];
            if (k > a0 && rmz[k - 1] == v) continue;
            if (sub == 0) ++distinct;
            const uint32_t h = ix_bucket(v, mask);
            const uint32_t e1 = tab[h + 1];
            for (uint32_t e = tab[h] + sub; e < e1; e += 8) {
                const IxEntry x0 = ent[e];
                const bool two = e + 4 < e1;
                IxEntry x1 = x0;
                if (two) x1 = ent[e + 4];
                const int64_t c0 = (int64_t)x0.q - j0, c1 = (int64_t)x1.q - j0;
                if (x0.v == v && c0 >= 0 && c0 < tw) atomicAdd(&s_cnt[c0], 1u);
                if (two && x1.v == v && c1 >= 0 && c1 < tw) atomicAdd(&s_cnt[c1], 1u);
            }
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) distinct += __shfl_xor_sync(0xffffffffu, distinct, d);
        if (lane == 0) s_ua[wid] = distinct;
        __syncthreads();
        uint32_t ua = 0;
#pragma unroll
        for (int w = 0; w < kIxThreads / 32; ++w) ua += s_ua[w];
        double* orow = out + i * ld + j0;
        for (int k = threadIdx.x; k < tw; k += blockDim.x) {
            const uint32_t inter = s_cnt[k];
            const uint32_t uni = ua + ub[j0 + k] - inter;
            orow[k] = uni == 0u ? 0.0 : __ddiv_rn(__dmul_rn(scaling, (double)inter), (double)uni);
        }
    }
}

int sm_count_of_current() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        sms = 148;
    }
    return sms;
}

}  // namespace
}  // namespace cms

extern "C" int cms_mass_match(const double* ref, int64_t n_ref, const double* q, int64_t n_q,
                              double tolerance, int ppm, uint8_t* out, int64_t ld, void* stream) {
    using namespace cms;
    if (n_ref < 0 || n_q < 0 || ld < n_q || (ppm != 0 && ppm != 1)) {
        set_error("cms_mass_match: invalid sizes or ppm flag (ld >= n_q, ppm 0 or 1)");
        return CMS_ERR_INVALID;
    }
    if (n_ref == 0 || n_q == 0) return CMS_OK;
    if (!ref || !q || !out) {
        set_error("cms_mass_match: null pointer");
        return CMS_ERR_INVALID;
    }
    const int vec = (ld % 16 == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
    const int64_t tiles = ((n_q + kMassTileCols - 1) / kMassTileCols) *
                          ((n_ref + kMassTileRows - 1) / kMassTileRows);
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>(tiles, (int64_t)sm_count_of_current() * 8));
    mass_match_kernel<<<grid, kMassThreads, 0, (cudaStream_t)stream>>>(ref, n_ref, q, n_q,
                                                                       tolerance, ppm, out, ld,
                                                                       vec);
    CMS_CUDA_TRY(cudaGetLastError());
    return CMS_OK;
}

extern "C" int cms_intersect_mz(const double* ref_mz, const int64_t* ref_off, int64_t n_ref,
                                int64_t n_ref_peaks, const double* q_mz, const int64_t* q_off,
                                int64_t n_q, int64_t n_q_peaks, double scaling, double* out,
                                int64_t ld, uint32_t* device_error, void* stream) {
    using namespace cms;
    if (n_ref < 0 || n_q < 0 || n_ref_peaks < 0 || n_q_peaks < 0 || ld < n_q ||
        n_q > 0xFFFFFFFFll || n_q_peaks > 0x7FFFFFFFll) {
        set_error("cms_intersect_mz: invalid sizes (ld >= n_q, n_q < 2^32, n_q_peaks < 2^31)");
        return CMS_ERR_INVALID;
    }
    if (n_ref == 0 || n_q == 0) return CMS_OK;
    if (!ref_off || !q_off || !out || (n_ref_peaks > 0 && !ref_mz) || (n_q_peaks > 0 && !q_mz)) {
        set_error("cms_intersect_mz: null pointer");
        return CMS_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    // buckets: a power of two >= twice the query peaks (load <= 1/2), 2^26 at most
    uint32_t nb = 1024;
    while (nb < (uint64_t)2 * (uint64_t)n_q_peaks && nb < (1u << 26)) nb <<= 1;
    const int sms = sm_count_of_current();
    uint32_t *cnt = nullptr, *tab = nullptr, *ub = nullptr, *sums = nullptr;
    IxEntry* ent = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&cnt), (size_t)nb * 4, s);
    if (e == cudaSuccess)
        e = cudaMallocAsync(reinterpret_cast<void**>(&sums),
                            (size_t)((nb + kScanChunk - 1) / kScanChunk) * 4, s);
    if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void**>(&tab), ((size_t)nb + 1) * 4, s);
    if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void**>(&ub), (size_t)n_q * 4, s);
    if (e == cudaSuccess)
        e = cudaMallocAsync(reinterpret_cast<void**>(&ent),
                            (size_t)std::max<int64_t>(1, n_q_peaks) * sizeof(IxEntry), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, (size_t)nb * 4, s);
    if (e == cudaSuccess) {
        const int igrid = (int)std::max<int64_t>(
            1, std::min<int64_t>((n_q * 32 + 255) / 256, (int64_t)sms * 16));
        ix_index_kernel<false><<<igrid, 256, 0, s>>>(q_mz, q_off, n_q, n_q_peaks, nb - 1, cnt,
                                                     nullptr, ub, device_error);
        const int n_chunks = (int)((nb + kScanChunk - 1) / kScanChunk);
        ix_chunk_sums<<<n_chunks, kScanThreads, 0, s>>>(cnt, nb, sums);
        ix_scan_sums<<<1, kScanThreads, 0, s>>>(sums, n_chunks, tab, nb);
        ix_chunk_scan<<<n_chunks, kScanThreads, 0, s>>>(cnt, tab, nb, sums);
        ix_index_kernel<true><<<igrid, 256, 0, s>>>(q_mz, q_off, n_q, n_q_peaks, nb - 1, cnt, ent,
                                                    nullptr, nullptr);
        const int64_t units = n_ref * ((n_q + kIxTile - 1) / kIxTile);
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(units, (int64_t)sms * 8));
        intersect_mz_kernel<<<grid, kIxThreads, 0, s>>>(ref_mz, ref_off, n_ref, n_ref_peaks, n_q,
                                                        tab, ent, ub, nb - 1, scaling, out, ld,
                                                        device_error);
        e = cudaGetLastError();
    }
    // stream-ordered frees: after the kernels above
    if (ent) cudaFreeAsync(ent, s);
    if (ub) cudaFreeAsync(ub, s);
    if (tab) cudaFreeAsync(tab, s);
    if (cnt) cudaFreeAsync(cnt, s);
    if (sums) cudaFreeAsync(sums, s);
    CMS_CUDA_TRY(e);
    return CMS_OK;
}
