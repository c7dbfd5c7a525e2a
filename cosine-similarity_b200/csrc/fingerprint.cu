// Fingerprint similarity (Jaccard / Dice / cosine) on bit-packed fingerprints.
//
// Replaces cudams/similarity/vector_similarity_functions.py:12-119, which
// computes I = R @ Q^T as a dense float32 GEMM over 0/1 values and then runs
// four elementwise passes.  Here each 128 x 128 output tile is one CTA:
//   - the 128 reference and 128 query rows of one K-chunk (up to 32 64-bit
//     words = 2048 bits) are staged in shared memory (rows padded to 33 words
//     so the column-strided reads of a warp hit 32 distinct banks);
//   - each thread owns an 8 x 8 micro-tile: per 64-bit word it loads 8 + 8
//     words and issues 64 AND + POPC pairs into integer accumulators (the
//     popcount runs on the integer pipe; there is no floating point until
//     the epilogue);
//   - the epilogue forms the measure in IEEE float32 in the reference's
//     order of operations and maps 0/0 to 0 (nan_to_num), or writes `fill`
//     for rows/columns without a fingerprint.
#include <algorithm>

#include "cms_internal.cuh"

namespace cms {
namespace {

constexpr int kBM = 128;
constexpr int kBN = 128;
constexpr int kKC = 32;          // 64-bit words per K chunk
constexpr int kLd = kKC + 1;     // padded row stride (words)
constexpr int kFpThreads = 256;  // 16 x 16 threads, 8 x 8 pairs each

struct FpParams {
    const uint32_t* r;
    const uint8_t* r_valid;
    int64_t n_r;
    const uint32_t* q;
    const uint8_t* q_valid;
    int64_t n_q;
    int n_words;  // uint32 words per row
    float fill;
    float* out;
    int64_t ld;
    int sym;  // only outputs (i, j) with i <= j (n_r == n_q)
};

__device__ __forceinline__ uint64_t load_word64(const uint32_t* row, int w64, int n_words) {
    const int w = 2 * w64;
    const uint32_t lo = w < n_words ? row[w] : 0u;
    const uint32_t hi = (w + 1) < n_words ? row[w + 1] : 0u;
    return (uint64_t)lo | ((uint64_t)hi << 32);
}

template <int MEASURE>
__device__ __forceinline__ float measure_of(int inter, int a, int b) {
    const float fi = (float)inter, fa = (float)a, fb = (float)b;
    float v;
    if (MEASURE == CMS_FP_JACCARD) {
        v = __fdiv_rn(fi, __fsub_rn(__fadd_rn(fa, fb), fi));
    } else if (MEASURE == CMS_FP_DICE) {
        v = __fmul_rn(2.0f, __fdiv_rn(fi, __fadd_rn(fa, fb)));
    } else {
        v = __fdiv_rn(fi, __fsqrt_rn(__fmul_rn(fa, fb)));
    }
    return v != v ? 0.0f : v;
}

template <int MEASURE>
__global__ void __launch_bounds__(kFpThreads)
fingerprint_kernel(FpParams P) {
    // symmetric: tiles wholly below the diagonal are copied afterwards
    if (P.sym && blockIdx.y > blockIdx.x) return;
    extern __shared__ __align__(16) uint64_t fp_smem[];
    uint64_t* sR = fp_smem;
    uint64_t* sQ = fp_smem + kBM * kLd;
    __shared__ int pa[kBM];
    __shared__ int pb[kBN];

    const int tid = threadIdx.x;
    const int tr = tid >> 4, tc = tid & 15;
    const int64_t row0 = (int64_t)blockIdx.y * kBM;
    const int64_t col0 = (int64_t)blockIdx.x * kBN;
    const int n64 = (P.n_words + 1) >> 1;

    int acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0;
    if (tid < kBM) pa[tid] = 0;
    if (tid >= kBM && tid < kBM + kBN) pb[tid - kBM] = 0;

    for (int k0 = 0; k0 < n64; k0 += kKC) {
        const int kc = min(kKC, n64 - k0);
        __syncthreads();
        // stage rows of this K chunk (zeros beyond the matrix edge)
        for (int e = tid; e < kBM * kKC; e += kFpThreads) {
            const int rr = e / kKC, k = e - rr * kKC;
            const int64_t gr = row0 + rr;
            uint64_t v = 0;
            if (gr < P.n_r && k < kc) v = load_word64(P.r + gr * P.n_words, k0 + k, P.n_words);
            sR[rr * kLd + k] = v;
        }
        for (int e = tid; e < kBN * kKC; e += kFpThreads) {
            const int cc = e / kKC, k = e - cc * kKC;
            const int64_t gc = col0 + cc;
            uint64_t v = 0;
            if (gc < P.n_q && k < kc) v = load_word64(P.q + gc * P.n_words, k0 + k, P.n_words);
            sQ[cc * kLd + k] = v;
        }
        __syncthreads();
        // row popcounts of this chunk
        if (tid < kBM) {
            int c = 0;
            for (int k = 0; k < kc; ++k) c += __popcll(sR[tid * kLd + k]);
            pa[tid] += c;
        } else if (tid < kBM + kBN) {
            const int cc = tid - kBM;
            int c = 0;
            for (int k = 0; k < kc; ++k) c += __popcll(sQ[cc * kLd + k]);
            pb[cc] += c;
        }
        // AND + POPC over the chunk
        for (int k = 0; k < kc; ++k) {
            uint64_t rw[8], qw[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) rw[i] = sR[(tr + 16 * i) * kLd + k];
#pragma unroll
            for (int j = 0; j < 8; ++j) qw[j] = sQ[(tc + 16 * j) * kLd + k];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] += __popcll(rw[i] & qw[j]);
        }
    }
    __syncthreads();

    // epilogue
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int rr = tr + 16 * i;
        const int64_t gr = row0 + rr;
        if (gr >= P.n_r) continue;
        const bool rv = P.r_valid ? P.r_valid[gr] != 0 : true;
        float* orow = P.out + gr * P.ld;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int cc = tc + 16 * j;
            const int64_t gc = col0 + cc;
            if (gc >= P.n_q || (P.sym && gr > gc)) continue;
            const bool qv = P.q_valid ? P.q_valid[gc] != 0 : true;
            orow[gc] = (rv && qv) ? measure_of<MEASURE>(acc[i][j], pa[rr], pb[cc]) : P.fill;
        }
    }
}

template <int MEASURE>
int launch_fp(dim3 grid, size_t smem, cudaStream_t s, const FpParams& P) {
    if (const int rc = raise_func_smem(reinterpret_cast<const void*>(fingerprint_kernel<MEASURE>),
                                       smem))
        return rc;
    fingerprint_kernel<MEASURE><<<grid, kFpThreads, smem, s>>>(P);
    return CMS_OK;
}

}  // namespace
}  // namespace cms

namespace cms {
namespace {

int fingerprint_impl(const char* who, int measure, const uint32_t* ref_bits,
                     const uint8_t* ref_valid, int64_t n_ref, const uint32_t* q_bits,
                     const uint8_t* q_valid, int64_t n_q, int n_words, float fill, float* out,
                     int64_t ld, int sym, void* stream) {
    if (measure < CMS_FP_JACCARD || measure > CMS_FP_COSINE) {
        set_error("%s: unknown measure %d", who, measure);
        return CMS_ERR_INVALID;
    }
    if (n_ref < 0 || n_q < 0 || n_words < 0 || n_words > 1024 || ld < n_q) {
        set_error("%s: invalid sizes (n_words must be in [0, 1024], ld >= n_q)", who);
        return CMS_ERR_INVALID;
    }
    if (n_ref == 0 || n_q == 0) return CMS_OK;
    if (!out || (n_words > 0 && (!ref_bits || !q_bits))) {
        set_error("%s: null pointer", who);
        return CMS_ERR_INVALID;
    }
    const int64_t gy = (n_ref + kBM - 1) / kBM, gx = (n_q + kBN - 1) / kBN;
    if (gy > 65535 || gx > 2147483647LL) {
        set_error("%s: too many rows for one launch (split the reference side)", who);
        return CMS_ERR_UNSUPPORTED;
    }
    FpParams P{ref_bits, ref_valid, n_ref, q_bits, q_valid, n_q, n_words, fill, out, ld, sym};
    dim3 grid((unsigned)gx, (unsigned)gy);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t smem = (size_t)(kBM + kBN) * kLd * sizeof(uint64_t);
    int rc = CMS_OK;
    switch (measure) {
        case CMS_FP_JACCARD:
            rc = launch_fp<CMS_FP_JACCARD>(grid, smem, s, P);
            break;
        case CMS_FP_DICE:
            rc = launch_fp<CMS_FP_DICE>(grid, smem, s, P);
            break;
        default:
            rc = launch_fp<CMS_FP_COSINE>(grid, smem, s, P);
            break;
    }
    if (rc) return rc;
    CMS_CUDA_TRY(cudaGetLastError());
    if (sym) {
        int dev = 0, sms = 148;
        CMS_CUDA_TRY(cudaGetDevice(&dev));
        CMS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        return launch_mirror(DenseOut{out, nullptr, nullptr, ld}, n_ref, nullptr, sms, s);
    }
    return CMS_OK;
}

}  // namespace
}  // namespace cms

extern "C" int cms_fingerprint(int measure, const uint32_t* ref_bits, const uint8_t* ref_valid,
                               int64_t n_ref, const uint32_t* q_bits, const uint8_t* q_valid,
                               int64_t n_q, int n_words, float fill, float* out, int64_t ld,
                               void* stream) {
    return cms::fingerprint_impl("cms_fingerprint", measure, ref_bits, ref_valid, n_ref, q_bits,
                                 q_valid, n_q, n_words, fill, out, ld, 0, stream);
}

extern "C" int cms_fingerprint_symmetric(int measure, const uint32_t* ref_bits,
                                         const uint8_t* ref_valid, const uint32_t* q_bits,
                                         const uint8_t* q_valid, int64_t n, int n_words,
                                         float fill, float* out, int64_t ld, void* stream) {
    return cms::fingerprint_impl("cms_fingerprint_symmetric", measure, ref_bits, ref_valid, n,
                                 q_bits, q_valid, n, n_words, fill, out, ld, 1, stream);
}
