/*
 * cudams_b200.h -- C ABI of the B200 (sm_100a) pairwise mass-spectrum
 * similarity library, libcudams_b200.so.
 *
 * The reference (tornikeo/cosine-similarity, package `cudams`) has no native
 * library: its GPU work is one Numba-CUDA kernel and three PyTorch
 * expressions called from two matchms plug-in classes.  This header is the
 * boundary that replaces those device calls; the Python classes
 * cudams.similarity.CudaCosineGreedy / CudaFingerprintSimilarity bind it with
 * ctypes (cudams/_native.py).  Each entry point names the reference code it
 * replaces.
 *
 * Conventions
 *  - Every function returns CMS_OK (0) or a CMS_ERR_* code; the message of
 *    the last failure on the calling thread is cms_last_error().  Nothing
 *    throws across this boundary.
 *  - All array arguments are DEVICE pointers owned by the caller, except
 *    where a comment says "host".  `stream` is a cudaStream_t (NULL = legacy
 *    default stream); work is enqueued asynchronously on it.
 *  - Spectra are passed as CSR ("spectrum set"):
 *        mz   float32 [n_peaks]   m/z, ascending within each spectrum
 *        a    float64 [n_peaks]   mz^mz_power per peak, or NULL when
 *                                 mz_power == 0 (then a == 1.0)
 *        b    float64 [n_peaks]   intensity^intensity_power per peak
 *        off  int64   [n + 1]     spectrum s owns peaks [off[s], off[s+1])
 *    with at most CMS_MAX_PEAKS peaks per spectrum (peak indices are packed
 *    in 16 bits, as the reference kernel packs them,
 *    cudams/similarity/spectrum_similarity_functions.py:146).  The caller
 *    applies the n_max_peaks truncation and the float32 rounding of m/z
 *    (cudams/similarity/CudaCosineGreedy.py:74-85); cudams/packing.py does
 *    both.
 *  - Greedy-cosine outputs are three row-major [n_ref, ld] arrays, the three
 *    planes of the reference's out[3, R, Q] (spectrum_similarity_functions.py
 *    :59-61, :151, :261-262): score float32, matches int32, overflow uint8.
 *  - A context (cms_ctx) owns the library's device scratch, tuning state and
 *    error word.  One context per host thread; calls on one context must not
 *    overlap in time on different streams.
 */
#ifndef CUDAMS_B200_H
#define CUDAMS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CMS_OK 0
#define CMS_ERR_INVALID 1     /* bad argument (null pointer, size, value)   */
#define CMS_ERR_CUDA 2        /* a CUDA runtime call failed                  */
#define CMS_ERR_UNSUPPORTED 3 /* valid but outside what this build supports  */
#define CMS_ERR_NOMEM 4       /* device allocation failed                    */
#define CMS_ERR_CAPACITY 5    /* sparse output buffer too small (see below)  */
#define CMS_ERR_DEVICE 6      /* a kernel reported bad input (error word)    */

#define CMS_MAX_PEAKS 65535

#define CMS_FP_JACCARD 0
#define CMS_FP_DICE 1
#define CMS_FP_COSINE 2

typedef struct cms_ctx cms_ctx;
typedef struct cms_library cms_library;

/* Library version as 10000*major + 100*minor + patch. */
int cms_version(void);

/* Message of the last failed call on this host thread ("" if none). */
const char* cms_last_error(void);

/* Create / destroy a context bound to CUDA device `device`. */
int cms_create(cms_ctx** out, int device);
int cms_destroy(cms_ctx* ctx);

/*
 * Read and clear the context's device error word (synchronises `stream`).
 * Kernels set bits in it instead of faulting when they meet input that
 * breaks a precondition: 1 a spectrum longer than CMS_MAX_PEAKS, 2 a sparse
 * spill list overrun, 4 bad offsets; and 8 when a bounded wait between the
 * pipelined pair kernel's warps ran out (2 s; the kernel then stops early
 * and its results are incomplete).  *bits receives the word (host pointer).
 */
int cms_take_device_error(cms_ctx* ctx, uint32_t* bits, void* stream);

/*
 * CUDA graphs for repeated calls (no reference counterpart; the reference
 * relaunches its Numba kernel per batch pair).  When enabled, cms_cosine_greedy
 * and cms_cosine_greedy_sparse capture their whole launch sequence (validation,
 * norms, ordering, index build, join, pair kernel, mirror) into a graph on the
 * first call and replay it on later calls with identical arguments (pointers,
 * sizes, parameters and config; the stream may differ), keeping the 8 most
 * recent graphs per context.  A replay reads the current contents of the caller's buffers.
 * While graphs are on, profiling events are not recorded; launch counts are.
 * Disabling synchronises the device and frees the graphs.
 */
int cms_graph_enable(cms_ctx* ctx, int enable);

/*
 * Per-stage timing of the tiled path, for benchmarks.  When enabled, every
 * cms_cosine_greedy* call records a CUDA event pair on its stream around each
 * stage; cms_profile_read synchronises those events and returns, per stage,
 * the summed device milliseconds and the number of kernel launches since the
 * last reset (host arrays of CMS_PROFILE_STAGES entries; either may be NULL).
 * Launch counts are kept even when timing is disabled.
 * Stages: 0 validate+norms, 1 reference order, 2 query index, 3 join,
 * 4 pair kernel.
 */
#define CMS_PROFILE_STAGES 5
int cms_profile_enable(cms_ctx* ctx, int enable);
int cms_profile_read(cms_ctx* ctx, double* stage_ms, int64_t* stage_launches, int reset);

/*
 * Work-item trace of the join kernel, for tests and studies of scheduling
 * (no reference counterpart).  While enabled on a context, every join launch
 * of that context (cms_cosine_greedy*, cms_library_search) appends one record
 * per work item (a spectrum of the sweeping side against one indexed tile)
 * to `records` (device, 4 uint64 each): tag | (SM id << 32), the item index,
 * and the device's %globaltimer (ns) when the item started and ended.
 * *count (device) is advanced atomically and may exceed `capacity` (records
 * beyond it are dropped); the caller zeroes it.  records == NULL disables.
 */
int cms_trace_enable(cms_ctx* ctx, uint64_t* records, int64_t capacity, uint64_t* count,
                     uint32_t tag);

/*
 * Plain greedy cosine: one (reference, query) pair per thread, the
 * reference's own kernel design restated in CUDA C++ for sm_100a -- 512
 * query threads per block over one reference spectrum, per-thread candidate
 * arrays of match_limit entries, bottom-up merge sort, per-thread used-peak
 * arrays cleared for every pair, query norm recomputed per pair.  Replaces
 * cosine_greedy_kernel()/_kernel (spectrum_similarity_functions.py:12-278)
 * as launched by CudaCosineGreedy.matrix (CudaCosineGreedy.py:149-181).
 * It is the "plain" comparator of the benchmark and has the same numerics
 * as cms_cosine_greedy (float64 keys, matchms ordering).
 * match_limit <= 4096 and n_max_peaks <= 4096 (compile-time array sizes).
 */
int cms_cosine_greedy_plain(const float* ref_mz, const double* ref_a, const double* ref_b,
                            const int64_t* ref_off, int64_t n_ref, const float* q_mz,
                            const double* q_a, const double* q_b, const int64_t* q_off,
                            int64_t n_q, double tolerance, double shift, int match_limit,
                            int n_max_peaks, float* score, int32_t* matches, uint8_t* overflow,
                            int64_t ld, void* stream);

/*
 * Tuning of the tiled path.  Zero in a field means "choose automatically".
 *   tile_spectra   query spectra per indexed tile (<= 4096)
 *   bucket_width   m/z width of one index bucket (default: the tolerance;
 *                  at least a quarter of it)
 *   n_buckets      buckets per tile (power of two; default: the tile's peak
 *                  count rounded up, at least 1024)
 *   mode           0 auto, 1 indexed join with pair spill, 2 pair kernel only
 *   pair_threads   threads per CTA of the pair kernel (64..512, multiple of 32)
 *   cand_per_pair  expected candidates per pair (e.g. sampled on the host);
 *                  sizes the first query sub-range of large spectra so the
 *                  join's candidate pool rarely overflows (0: unknown)
 *   width_by_class first query sub-range width (queries swept per pool fill)
 *                  for reference spectra of length class c = bit length of
 *                  the peak count (c = 0..16); 0: derived from cand_per_pair.
 *                  Set by cudams.autotune from timed trials per class.
 * One field changes the result rather than the speed:
 *   symmetric      nonzero: matchms' is_symmetric=True (matchms
 *                  BaseSimilarity.matrix; accepted but ignored by the
 *                  reference, CudaCosineGreedy.py:131-132).  Needs
 *                  n_ref == n_q.  Only the pairs (i, j) with i <= j are
 *                  computed, as (reference i, query j); the dense output
 *                  copies each to (j, i), the sparse output emits both
 *                  (i, j) and (j, i) for i != j.
 */
typedef struct {
    int32_t tile_spectra;
    double bucket_width;
    int32_t n_buckets;
    int32_t mode;
    int32_t pair_threads;
    double cand_per_pair;
    int32_t symmetric;
    int32_t width_by_class[17];
} cms_cosine_config;

/*
 * Tiled greedy cosine, dense output.  Same contract and numerics as the
 * reference's CudaCosineGreedy.matrix(array_type="numpy")
 * (CudaCosineGreedy.py:107-205): for every (reference i, query j) writes
 * score[i*ld+j], matches[i*ld+j], overflow[i*ld+j].
 *   - window:  query peak matches reference peak iff
 *              !(mz_q+shift > mz_r+tol) && !(mz_q+shift < mz_r-tol) (float64)
 *   - key:     ((a_r*b_r)*a_q)*b_q (float64), sorted descending, ties to the
 *              later-generated candidate (p_ref-major, p_query ascending)
 *   - overflow = 1 when match_limit candidates were generated; only the
 *              first match_limit (in generation order) take part.
 * n_ref_peaks / n_q_peaks are the lengths of the peak arrays.  cfg may be
 * NULL (automatic).  Internally: per-call query index (m/z buckets per tile
 * of query spectra), a persistent warp-per-(reference, tile) join, and a
 * CTA-per-pair kernel for pairs with many candidates.
 */
int cms_cosine_greedy(cms_ctx* ctx, const float* ref_mz, const double* ref_a, const double* ref_b,
                      const int64_t* ref_off, int64_t n_ref, int64_t n_ref_peaks,
                      const float* q_mz, const double* q_a, const double* q_b,
                      const int64_t* q_off, int64_t n_q, int64_t n_q_peaks, double tolerance,
                      double shift, int match_limit, float* score, int32_t* matches,
                      uint8_t* overflow, int64_t ld, const cms_cosine_config* cfg, void* stream);

/*
 * Tiled greedy cosine, sparse output: every pair with score >= threshold
 * (threshold > 0) is appended, in no particular order, to the hit arrays
 * (hit_ref, hit_query int32; hit_score float32; hit_matches int32;
 * hit_overflow uint8), at most `capacity` of them.  *hit_count (device
 * int64, zeroed by the call) receives the number of qualifying pairs, which
 * may exceed capacity: then only `capacity` hits were stored and the caller
 * must retry with a larger buffer.  Replaces the array_type="sparse" branch
 * of CudaCosineGreedy.matrix (CudaCosineGreedy.py:186-226), which builds the
 * same (row, col, score, matches, overflow) tuples from `out[0] >= threshold`.
 */
int cms_cosine_greedy_sparse(cms_ctx* ctx, const float* ref_mz, const double* ref_a,
                             const double* ref_b, const int64_t* ref_off, int64_t n_ref,
                             int64_t n_ref_peaks, const float* q_mz, const double* q_a,
                             const double* q_b, const int64_t* q_off, int64_t n_q,
                             int64_t n_q_peaks, double tolerance, double shift, int match_limit,
                             float threshold, int32_t* hit_ref, int32_t* hit_query,
                             float* hit_score, int32_t* hit_matches, uint8_t* hit_overflow,
                             int64_t capacity, int64_t* hit_count, const cms_cosine_config* cfg,
                             void* stream);

/*
 * Modified cosine (matchms ModifiedCosine): greedy cosine over the union of
 * the matches at shift 0 and the matches at the pair's precursor difference
 * shift = ref_precursor[i] - q_precursor[j] (precursor m/z per spectrum,
 * device float64), in matchms' order -- the unshifted candidates, then the
 * shifted ones, each generated reference-peak-major; one stable descending
 * sort of the keys over that concatenation, one greedy.  No CUDA counterpart
 * in the reference: it prototypes ModifiedCosine beside its CUDA classes
 * (notebooks/prototyping/other_similarities.ipynb) and carries the shift it
 * needs in its kernel (spectrum_similarity_functions.py:14,133).  Outputs,
 * match_limit (counted over the concatenation), overflow, cfg and the sparse
 * form follow cms_cosine_greedy / cms_cosine_greedy_sparse; spectra may have
 * at most 32767 peaks (more sets CMS_ERR_DEVICE's spectrum-too-long bit).
 * The join runs a second sweep per reference chunk through a neutral-loss
 * index (m/z - precursor of each query peak) and confirms each of its
 * candidates with matchms' float64 shifted-window test.
 */
int cms_modified_cosine(cms_ctx* ctx, const float* ref_mz, const double* ref_a,
                        const double* ref_b, const int64_t* ref_off, const double* ref_precursor,
                        int64_t n_ref, int64_t n_ref_peaks, const float* q_mz, const double* q_a,
                        const double* q_b, const int64_t* q_off, const double* q_precursor,
                        int64_t n_q, int64_t n_q_peaks, double tolerance, int match_limit,
                        float* score, int32_t* matches, uint8_t* overflow, int64_t ld,
                        const cms_cosine_config* cfg, void* stream);
int cms_modified_cosine_sparse(cms_ctx* ctx, const float* ref_mz, const double* ref_a,
                               const double* ref_b, const int64_t* ref_off,
                               const double* ref_precursor, int64_t n_ref, int64_t n_ref_peaks,
                               const float* q_mz, const double* q_a, const double* q_b,
                               const int64_t* q_off, const double* q_precursor, int64_t n_q,
                               int64_t n_q_peaks, double tolerance, int match_limit,
                               float threshold, int32_t* hit_ref, int32_t* hit_query,
                               float* hit_score, int32_t* hit_matches, uint8_t* hit_overflow,
                               int64_t capacity, int64_t* hit_count, const cms_cosine_config* cfg,
                               void* stream);

/*
 * Resident library: a spectrum set indexed once on the device (the "reference"
 * side of matchms, e.g. a spectral library) and searched by many query
 * batches.  This is the served form of CudaCosineGreedy.matrix(library,
 * queries, array_type="sparse") (CudaCosineGreedy.py:186-226): each search
 * returns every (library spectrum, query) pair with score >= threshold, with
 * the same numerics as cms_cosine_greedy.  The library's spectrum arrays stay
 * owned by the caller and must outlive the library object; the index and the
 * library norms are allocated by cms_library_create (which synchronises
 * `stream`) and freed by cms_library_destroy.  cfg (may be NULL) sets the
 * library tile size / bucket width and the expected candidates per pair.
 * Searches on different contexts and streams may run concurrently against
 * one library (it is read-only after creation).  A search launches four
 * waves of short-lived CTAs (each warp takes an equal share of the work items
 * and exits; each CTA borrows a slice of the context's candidate pool while
 * it lives), so that the SMs free up continuously and searches on other
 * streams -- give urgent ones a higher stream priority -- are scheduled in
 * between: concurrent searches overlap on the device.  Hit buffers and hit_count
 * follow cms_cosine_greedy_sparse (hit_ref = library index, hit_query =
 * query index).
 */
int cms_library_create(cms_ctx* ctx, const float* mz, const double* a, const double* b,
                       const int64_t* off, int64_t n, int64_t n_peaks, double tolerance,
                       double shift, int match_limit, const cms_cosine_config* cfg,
                       cms_library** out, void* stream);
int cms_library_search(cms_ctx* ctx, const cms_library* lib, const float* q_mz,
                       const double* q_a, const double* q_b, const int64_t* q_off, int64_t n_q,
                       int64_t n_q_peaks, float threshold, int32_t* hit_ref, int32_t* hit_query,
                       float* hit_score, int32_t* hit_matches, uint8_t* hit_overflow,
                       int64_t capacity, int64_t* hit_count, void* stream);
int cms_library_destroy(cms_library* lib);

/*
 * Allocation-free greedy cosine, dense output.  No counterpart in the
 * reference: this entry point exists for callers that must not have a
 * library allocate device memory -- an application whose GPU memory is
 * already reserved by its own allocator, a latency-critical loop that cannot
 * take the device-wide synchronisation cudaMalloc / cudaFree may imply, or a
 * plugin host that forbids allocations behind its back.  It needs no context,
 * calls no cudaMalloc, cudaFree or other allocating routine, and computes the
 * same results as cms_cosine_greedy (same arguments and numerics) with the
 * pair kernel over every pair, which is exact for any input but slower than
 * the indexed join when most pairs have no candidates.
 *   - Scratch: a fixed device array of the library, about 8 MiB (flags plus
 *     one float64 norm per spectrum); every GPU that loads the library holds
 *     it until the process exits.  Limit: n_ref + n_q <= 1048576 spectra and
 *     match_limit <= 4096; larger calls fail with CMS_ERR_UNSUPPORTED.
 *   - Device: every pointer argument must be memory of the CURRENT device
 *     (cudaSetDevice before the call; managed memory is accepted) and the
 *     stream, when not NULL, must belong to it.  Otherwise the call returns
 *     CMS_ERR_INVALID before launching anything.
 *   - The first call on each device looks up the array's device address
 *     (cudaGetSymbolAddress) and caches it; make that first call before any
 *     stream capture begins.  The cache assumes that the device's primary
 *     context lives for the whole process: after cudaDeviceReset the cached
 *     address is stale, so do not call this entry point again after a reset.
 *   - All calls share the one array, and it keeps the last call's contents
 *     (the call clears the flags it needs): calls that overlap on the GPU,
 *     from different streams or host threads, race and corrupt each other.
 *     Serialise them.
 *   - device_error (device uint32, may be NULL) receives the error bits of
 *     this call (see cms_take_device_error); 0 means the results are valid.
 */
int cms_cosine_greedy_noalloc(const float* ref_mz, const double* ref_a, const double* ref_b,
                              const int64_t* ref_off, int64_t n_ref, int64_t n_ref_peaks,
                              const float* q_mz, const double* q_a, const double* q_b,
                              const int64_t* q_off, int64_t n_q, int64_t n_q_peaks,
                              double tolerance, double shift, int match_limit, float* score,
                              int32_t* matches, uint8_t* overflow, int64_t ld,
                              uint32_t* device_error, void* stream);

/*
 * Fingerprint similarity on bit-packed fingerprints: n_words uint32 per
 * row, bit k in word k/32 at bit k%32, unused high bits zero.  The
 * intersection counts I = R . Q^T run on the tensor cores (tcgen05
 * kind::mxf4: 4-bit float operands of value 0 or 1 expanded from the bits in
 * shared memory, block scale factors 1, exact float32 accumulation).  Writes
 * out[i*ld + j] (float32) for every (reference i, query j):
 *   CMS_FP_JACCARD  I / (a + b - I)      vector_similarity_functions.py:42-46
 *   CMS_FP_DICE     2 * (I / (a + b))    vector_similarity_functions.py:87-90
 *   CMS_FP_COSINE   I / sqrt(a * b)      vector_similarity_functions.py:116-118
 * with I = popcount(r & q), a = popcount(r), b = popcount(q), each division
 * and square root in IEEE float32, and 0/0 -> 0 (nan_to_num).  Rows whose
 * valid flag is 0 (no fingerprint) give `fill` in all their pairs
 * (CudaFingerprintSimilarity.py:147-177); valid arrays may be NULL (all
 * valid).  n_words <= 1024.
 */
int cms_fingerprint(int measure, const uint32_t* ref_bits, const uint8_t* ref_valid,
                    int64_t n_ref, const uint32_t* q_bits, const uint8_t* q_valid, int64_t n_q,
                    int n_words, float fill, float* out, int64_t ld, void* stream);

/*
 * Read and clear the error bits of the fingerprint kernels (synchronises
 * `stream`; *bits is a host pointer).  No reference counterpart.  The
 * fingerprint kernels run a multi-stage pipeline whose internal waits are
 * bounded in time; a nonzero word means one ran out of time and the results
 * of the calls since the last read are not valid.
 */
int cms_fingerprint_take_error(uint32_t* bits, void* stream);

/*
 * Self-check of the fingerprint epilogue's branch-free float32 division and
 * square root against CUDA's IEEE operations, bit for bit, on the device.
 * No reference counterpart.  Writes five mismatch counts to the host array
 * `mismatches` (synchronises `stream`): [0] n / d for all integers
 * 0 <= n <= d <= 65536; [1] sqrt(p) and [2] the reciprocal of sqrt(p) for
 * every float p in [1, 2^30]; [3] the cosine I / sqrt(a * b) for every
 * a, b <= 2048 and I <= min(a, b); [4] the same for 2^30 pseudo-random
 * triples with a, b <= 32768.  All five are 0 on a correct device.
 */
int cms_fingerprint_arith_check(uint64_t* mismatches, void* stream);

/*
 * cms_fingerprint with matchms' is_symmetric=True (the reference's
 * CudaFingerprintSimilarity.matrix accepts the flag and ignores it,
 * CudaFingerprintSimilarity.py:113-119): n references and n queries; only the
 * pairs (i, j) with i <= j are computed, as (reference i, query j), and
 * (j, i) receives the same value.  For one set against itself the result is
 * bit-identical to cms_fingerprint (every measure is symmetric in I, a and
 * b); when both sides are the same arrays (ref_bits == q_bits and ref_valid
 * == q_valid) the full matrix is computed directly, which is faster than the
 * upper triangle plus the mirror copy.
 */
int cms_fingerprint_symmetric(int measure, const uint32_t* ref_bits, const uint8_t* ref_valid,
                              const uint32_t* q_bits, const uint8_t* q_valid, int64_t n,
                              int n_words, float fill, float* out, int64_t ld, void* stream);

/*
 * matchms ParentMassMatch / PrecursorMzMatch on the device (the reference
 * prototypes both beside its CUDA classes: notebooks/prototyping/
 * other_similarities.ipynb; matchms >= 0.24.0 is its requirement).  ref[i]
 * and q[j] are the spectra's parent masses or precursor m/z (float64,
 * device memory).  Writes out[i*ld + j] = 1 if
 *   ppm == 0:  |ref[i] - q[j]| <= tolerance                   (Dalton)
 *   ppm == 1:  |ref[i] - q[j]| / ((ref[i] + q[j]) / 2) * 1e6 <= tolerance
 * in IEEE float64 in that order of operations, else 0 (NaN never matches).
 */
int cms_mass_match(const double* ref, int64_t n_ref, const double* q, int64_t n_q,
                   double tolerance, int ppm, uint8_t* out, int64_t ld, void* stream);

/*
 * matchms IntersectMz on the device: for every (reference i, query j)
 * out[i*ld + j] = scaling * |A & B| / |A | B| (float64, 0.0 when both sets
 * are empty), A and B the sets of exact float64 m/z values of the two
 * spectra (CSR: *_off[n+1] into *_mz, peaks sorted by m/z as matchms keeps
 * them; repeated values count once).  Offsets outside [0, n_*_peaks] set
 * bit 2 of *device_error (device memory, may be NULL) and the spectrum reads
 * as empty.
 */
int cms_intersect_mz(const double* ref_mz, const int64_t* ref_off, int64_t n_ref,
                     int64_t n_ref_peaks, const double* q_mz, const int64_t* q_off, int64_t n_q,
                     int64_t n_q_peaks, double scaling, double* out, int64_t ld,
                     uint32_t* device_error, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CUDAMS_B200_H */
