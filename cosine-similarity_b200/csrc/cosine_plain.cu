// Plain greedy cosine: one (reference, query) pair per thread.
//
// This is the reference kernel's design (cudams/similarity/
// spectrum_similarity_functions.py:39-262) written in CUDA C++ for sm_100a,
// kept as the "plain" comparator of the benchmark:
//   - grid (n_ref, ceil(n_q/512)), 512 query threads per block sharing one
//     reference spectrum (:28-37);
//   - the reference norm is computed once per block, the query norm again by
//     every thread (:79-110);
//   - the candidate sweep writes into per-thread local arrays of match_limit
//     entries and stops at match_limit, setting overflow (:116-151);
//   - a bottom-up merge sort with a strict '>' merge, so equal keys keep the
//     later-generated candidate first (:161-198);
//   - per-thread used-peak arrays cleared for every pair, then the greedy
//     walk (:201-218).
// Numerics follow matchms (float64 window test and keys, see the public
// header) so that its outputs are bit-identical to cms_cosine_greedy's.
#include "cms_internal.cuh"

namespace cms {
namespace {

constexpr int kPlainThreads = 512;

__device__ __forceinline__ double peak_a(const double* a, int64_t i) { return a ? a[i] : 1.0; }

// Sequential float64 sum of (a*b)^2 over [lo, hi), rounding every product and
// sum separately (no contraction), the order the oracle uses.
__device__ double norm2_seq(const double* a, const double* b, int64_t lo, int64_t hi) {
    double s = 0.0;
    for (int64_t k = lo; k < hi; ++k) {
        double w = __dmul_rn(peak_a(a, k), b[k]);
        s = __dadd_rn(s, __dmul_rn(w, w));
    }
    return s;
}

template <int ML_CAP, int NMAX_CAP>
__global__ void __launch_bounds__(kPlainThreads)
cosine_plain_kernel(CosineArgs args, DenseOut out, int n_max_peaks, uint32_t* err) {
    const int64_t i = blockIdx.x;
    const int64_t j = (int64_t)blockIdx.y * kPlainThreads + threadIdx.x;
    const SpecSet& R = args.ref;
    const SpecSet& Q = args.qry;

    const int64_t r0 = R.off[i];
    const int64_t nr = R.off[i + 1] - r0;
    const bool r_bad = nr < 0 || nr > n_max_peaks || nr > CMS_MAX_PEAKS;

    __shared__ double s_norm2_r;
    if (threadIdx.x == 0) s_norm2_r = (nr > 0 && !r_bad) ? norm2_seq(R.a, R.b, r0, r0 + nr) : 0.0;
    __syncthreads();
    if (j >= Q.n) return;

    const int64_t o = i * out.ld + j;
    out.score[o] = 0.0f;
    out.matches[o] = 0;
    out.overflow[o] = 0;

    const int64_t q0 = Q.off[j];
    const int64_t nq = Q.off[j + 1] - q0;
    if (r_bad || nq < 0 || nq > n_max_peaks || nq > CMS_MAX_PEAKS) {
        atomicOr(err, kErrSpectrumTooLong);
        out.score[o] = __int_as_float(0x7fc00000);
        return;
    }
    if (nr == 0 || nq == 0) return;

    const double norm2_q = norm2_seq(Q.a, Q.b, q0, q0 + nq);

    // ---- candidate sweep (generation order: p1 ascending, p2 ascending) ----
    uint32_t gen[ML_CAP];
    double val[ML_CAP];
    int n = 0;
    int lowest = 0;
    bool overflow = false;
    const int ml = args.match_limit;
    for (int p1 = 0; p1 < nr && !overflow; ++p1) {
        const double mz1 = (double)R.mz[r0 + p1];
        const double lo = __dsub_rn(mz1, args.tol);
        const double hi = __dadd_rn(mz1, args.tol);
        const double w1 = __dmul_rn(peak_a(R.a, r0 + p1), R.b[r0 + p1]);
        for (int p2 = lowest; p2 < nq; ++p2) {
            const double mz2 = __dadd_rn((double)Q.mz[q0 + p2], args.shift);
            if (mz2 > hi) break;
            if (mz2 < lo) {
                lowest = p2 + 1;
                continue;
            }
            val[n] = __dmul_rn(__dmul_rn(w1, peak_a(Q.a, q0 + p2)), Q.b[q0 + p2]);
            gen[n] = ((uint32_t)p1 << 16) | (uint32_t)p2;
            ++n;
            if (n >= ml) {
                overflow = true;
                break;
            }
        }
    }
    out.overflow[o] = overflow ? 1 : 0;
    if (n == 0) return;

    // ---- bottom-up merge sort, key descending; '>' keeps the right run first on ties ----
    uint32_t tgen[ML_CAP];
    double tval[ML_CAP];
    for (int width = 1; width < n; width *= 2) {
        for (int left = 0; left < n - width; left += 2 * width) {
            const int mid = left + width;
            const int end = min(mid + width, n);
            int x = left, y = mid, k = left;
            while (x < mid && y < end) {
                if (val[x] > val[y]) {
                    tval[k] = val[x];
                    tgen[k++] = gen[x++];
                } else {
                    tval[k] = val[y];
                    tgen[k++] = gen[y++];
                }
            }
            while (x < mid) {
                tval[k] = val[x];
                tgen[k++] = gen[x++];
            }
            while (y < end) {
                tval[k] = val[y];
                tgen[k++] = gen[y++];
            }
            for (int m = left; m < end; ++m) {
                val[m] = tval[m];
                gen[m] = tgen[m];
            }
        }
    }

    // ---- greedy assignment ----
    bool used_r[NMAX_CAP];
    bool used_q[NMAX_CAP];
    for (int m = 0; m < n_max_peaks; ++m) {
        used_r[m] = false;
        used_q[m] = false;
    }
    double score = 0.0;
    int matches = 0;
    for (int m = 0; m < n; ++m) {
        const int p1 = gen[m] >> 16;
        const int p2 = gen[m] & 0xFFFF;
        if (!used_r[p1] && !used_q[p2]) {
            used_r[p1] = true;
            used_q[p2] = true;
            score = __dadd_rn(score, val[m]);
            ++matches;
        }
    }
    const double denom = __dmul_rn(sqrt(s_norm2_r), sqrt(norm2_q));
    out.score[o] = (float)__ddiv_rn(score, denom);
    out.matches[o] = matches;
}

template <int ML_CAP, int NMAX_CAP>
cudaError_t launch_plain(const CosineArgs& args, const DenseOut& out, int n_max_peaks,
                         uint32_t* err, cudaStream_t s) {
    dim3 grid((unsigned)args.ref.n, (unsigned)((args.qry.n + kPlainThreads - 1) / kPlainThreads));
    cosine_plain_kernel<ML_CAP, NMAX_CAP><<<grid, kPlainThreads, 0, s>>>(args, out, n_max_peaks, err);
    return cudaGetLastError();
}

template <int ML_CAP>
cudaError_t dispatch_nmax(const CosineArgs& args, const DenseOut& out, int n_max_peaks,
                          uint32_t* err, cudaStream_t s) {
    if (n_max_peaks <= 1024) return launch_plain<ML_CAP, 1024>(args, out, n_max_peaks, err, s);
    if (n_max_peaks <= 2048) return launch_plain<ML_CAP, 2048>(args, out, n_max_peaks, err, s);
    return launch_plain<ML_CAP, 4096>(args, out, n_max_peaks, err, s);
}

// Error word for callers without a context (plain path): one per process.
__device__ uint32_t g_plain_err;

}  // namespace
}  // namespace cms

extern "C" int cms_cosine_greedy_plain(const float* ref_mz, const double* ref_a,
                                       const double* ref_b, const int64_t* ref_off, int64_t n_ref,
                                       const float* q_mz, const double* q_a, const double* q_b,
                                       const int64_t* q_off, int64_t n_q, double tolerance,
                                       double shift, int match_limit, int n_max_peaks,
                                       float* score, int32_t* matches, uint8_t* overflow,
                                       int64_t ld, void* stream) {
    using namespace cms;
    CosineArgs args;
    args.ref = SpecSet{ref_mz, ref_a, ref_b, ref_off, n_ref, 0};
    args.qry = SpecSet{q_mz, q_a, q_b, q_off, n_q, 0};
    args.tol = tolerance;
    args.shift = shift;
    args.match_limit = match_limit;
    if (!check_specset(args.ref, "reference") || !check_specset(args.qry, "query"))
        return CMS_ERR_INVALID;
    if (match_limit < 1 || !(tolerance >= 0.0) || n_max_peaks < 1 || ld < n_q) {
        set_error("cms_cosine_greedy_plain: invalid match_limit/tolerance/n_max_peaks/ld");
        return CMS_ERR_INVALID;
    }
    if (match_limit > 4096 || n_max_peaks > 4096) {
        set_error("cms_cosine_greedy_plain: match_limit and n_max_peaks must be <= 4096 "
                  "(per-thread local arrays)");
        return CMS_ERR_UNSUPPORTED;
    }
    if (n_q > 65535LL * kPlainThreads) {
        set_error("cms_cosine_greedy_plain: too many queries for one launch");
        return CMS_ERR_UNSUPPORTED;
    }
    if (n_ref == 0 || n_q == 0) return CMS_OK;
    if (!score || !matches || !overflow) {
        set_error("cms_cosine_greedy_plain: null output pointer");
        return CMS_ERR_INVALID;
    }
    DenseOut out{score, matches, overflow, ld};
    uint32_t* err = nullptr;
    CMS_CUDA_TRY(cudaGetSymbolAddress((void**)&err, g_plain_err));
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (match_limit <= 256)
        e = dispatch_nmax<256>(args, out, n_max_peaks, err, s);
    else if (match_limit <= 1024)
        e = dispatch_nmax<1024>(args, out, n_max_peaks, err, s);
    else if (match_limit <= 2048)
        e = dispatch_nmax<2048>(args, out, n_max_peaks, err, s);
    else
        e = dispatch_nmax<4096>(args, out, n_max_peaks, err, s);
    if (e != cudaSuccess) return cuda_fail(e, "cosine_plain_kernel launch");
    return CMS_OK;
}
