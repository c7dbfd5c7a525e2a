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
//                          values (0 when both are empty).  One CTA per
//                          (reference, 256 queries); the reference's m/z in
//                          shared memory; each thread merges its query's
//                          sorted m/z against them, counting distinct values
//                          only (the set semantics), and forms
//                          scaling * inter / union in float64.
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
constexpr int kIxSmemPeaks = 4096;  // reference m/z staged in shared memory up to this many

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

// Distinct values of sorted x[0, n) from position k on (k at the first of a run)
__device__ __forceinline__ int64_t skip_run(const double* x, int64_t k, int64_t n) {
    const double v = x[k];
    do {
        ++k;
    } while (k < n && x[k] == v);
    return k;
}

__global__ void __launch_bounds__(kIxThreads) intersect_mz_kernel(
    const double* __restrict__ rmz, const int64_t* __restrict__ roff, int64_t n_ref,
    int64_t n_ref_peaks, const double* __restrict__ qmz, const int64_t* __restrict__ qoff,
    int64_t n_q, int64_t n_q_peaks, double scaling, double* __restrict__ out, int64_t ld,
    uint32_t* err) {
    __shared__ double s_r[kIxSmemPeaks];
    const int64_t qblocks = (n_q + kIxThreads - 1) / kIxThreads;
    for (int64_t blk = blockIdx.x; blk < n_ref * qblocks; blk += gridDim.x) {
        const int64_t i = blk / qblocks, j = (blk - i * qblocks) * kIxThreads + threadIdx.x;
        int64_t a0, a1;
        spectrum_range(roff, i, n_ref_peaks, a0, a1, threadIdx.x == 0 ? err : nullptr);
        const int64_t na = a1 - a0;
        const bool staged = na <= kIxSmemPeaks;
        __syncthreads();  // the previous unit's readers are done with s_r
        if (staged)
            for (int64_t k = threadIdx.x; k < na; k += blockDim.x) s_r[k] = rmz[a0 + k];
        __syncthreads();
        if (j >= n_q) continue;
        const double* A = staged ? s_r : rmz + a0;
        int64_t b0, b1;
        spectrum_range(qoff, j, n_q_peaks, b0, b1, err);
        const double* B = qmz + b0;
        const int64_t nb = b1 - b0;
        // merge of the two sorted lists, one step per distinct value
        int64_t ia = 0, ib = 0, inter = 0, uni = 0;
        while (ia < na && ib < nb) {
            const double x = A[ia], y = B[ib];
            if (x < y) {
                ia = skip_run(A, ia, na);
            } else if (y < x) {
                ib = skip_run(B, ib, nb);
            } else {
                ia = skip_run(A, ia, na);
                ib = skip_run(B, ib, nb);
                ++inter;
            }
            ++uni;
        }
        while (ia < na) {
            ia = skip_run(A, ia, na);
            ++uni;
        }
        while (ib < nb) {
            ib = skip_run(B, ib, nb);
            ++uni;
        }
        out[i * ld + j] = uni == 0 ? 0.0 : __ddiv_rn(__dmul_rn(scaling, (double)inter), (double)uni);
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
    if (n_ref < 0 || n_q < 0 || n_ref_peaks < 0 || n_q_peaks < 0 || ld < n_q) {
        set_error("cms_intersect_mz: invalid sizes (ld >= n_q)");
        return CMS_ERR_INVALID;
    }
    if (n_ref == 0 || n_q == 0) return CMS_OK;
    if (!ref_off || !q_off || !out || (n_ref_peaks > 0 && !ref_mz) || (n_q_peaks > 0 && !q_mz)) {
        set_error("cms_intersect_mz: null pointer");
        return CMS_ERR_INVALID;
    }
    const int64_t units = n_ref * ((n_q + kIxThreads - 1) / kIxThreads);
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>(units, (int64_t)sm_count_of_current() * 8));
    intersect_mz_kernel<<<grid, kIxThreads, 0, (cudaStream_t)stream>>>(
        ref_mz, ref_off, n_ref, n_ref_peaks, q_mz, q_off, n_q, n_q_peaks, scaling, out, ld,
        device_error);
    CMS_CUDA_TRY(cudaGetLastError());
    return CMS_OK;
}
