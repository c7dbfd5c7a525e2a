/*
 * CPU oracle for greedy cosine and fingerprint similarity.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product imports, links or calls
 * this file; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * / reference arm use it, as the checker or as the timed CPU baseline.
 *
 * What it restates
 * ----------------
 * Greedy cosine, two key modes:
 *
 *   key_mode 0 ("f64", matchms semantics).  The reference pins its scores to
 *     matchms CosineGreedy (matchms >= 0.24.0, requirements.txt:1), which is a
 *     third-party dependency not vendored in the reference.  Its call sites in
 *     the reference are cudams/similarity/spectrum_similarity_functions.py:
 *     306-317 (collect_peak_pairs -> argsort(kind="mergesort")[::-1] ->
 *     score_best_matches) and tests/utils.py:14-18.  Restated here:
 *       - window:  peak p2 of the query matches peak p1 of the reference iff
 *                  !(mz2 > mz1 + tol) && !(mz2 < mz1 - tol) in float64, with
 *                  mz2 = mz_q + shift (matchms find_matches).
 *       - key:     ((mz1^p * int1^q) * mz2^p) * int2^q in float64, left to
 *                  right as matchms collect_peak_pairs writes it.  The caller
 *                  passes a = mz^p and b = int^q per peak (a == NULL: 1.0).
 *       - order:   key descending, ties -> later-generated candidate first
 *                  (argsort mergesort reversed, spectrum_similarity_functions
 *                  .py:314; equal to the strict-'>' merge at :178).
 *       - greedy:  accept a candidate iff neither peak is used (:210-218).
 *       - score:   sum(keys of accepted, in sorted order) /
 *                  (sqrt(sum w1^2) * sqrt(sum w2^2)), w = a*b, sums taken
 *                  sequentially in peak order (tests/similarity/
 *                  test_cosine_greedy.py:9-24 gives the closed form).
 *
 *   key_mode 1 ("f32", the reference CUDA kernel's own arithmetic,
 *     spectrum_similarity_functions.py:39-262): the window test is
 *     delta = (mz_q + shift) - mz_r against +-tol (:133-137), keys are the
 *     float64 product (a1*b1)*(a2*b2) rounded to float32 (:141-147), norms
 *     are float32 running sums (:92-110).  Used to check this oracle against
 *     outputs of the reference kernel itself (tests/golden).
 *
 *   Both modes: spectra are given as already truncated to n_max_peaks and
 *   with m/z rounded to float32 (CudaCosineGreedy.py:74-85); candidates are
 *   generated p1-major, p2 ascending (:123-149) and generation stops once
 *   match_limit candidates exist, which sets overflow = 1 (:149, an exact fill
 *   counts); an empty spectrum on either side gives (0, 0, 0) (:70, :100); no
 *   candidates gives score 0, matches 0 (:153).
 *
 * Modified cosine (matchms ModifiedCosine, the published algorithm of the
 *   same third-party package; the reference prototypes it beside its CUDA
 *   classes, notebooks/prototyping/other_similarities.ipynb cells 5 and 8, and
 *   carries the shift it needs into its kernel, spectrum_similarity_functions
 *   .py:14,133): the candidates are the matches at shift 0 followed by the
 *   matches at shift = precursor_mz(reference) - precursor_mz(query) (both
 *   float64, the matchms metadata), each list generated as above (p1-major,
 *   p2 ascending); keys, the stable descending sort over the concatenation
 *   (ties -> later position first, so a shifted candidate precedes an
 *   unshifted one of equal key), the greedy and the norms are those of mode 0.
 *   matchms has no candidate limit; here, as for greedy cosine, generation
 *   stops once match_limit candidates exist in the concatenated order and
 *   overflow is set, so a match_limit above every pair's count gives matchms'
 *   result exactly.
 *
 * Fingerprints: cudams/similarity/vector_similarity_functions.py:42-46
 *   (jaccard I/(a+b-I)), :87-90 (dice 2*(I/(a+b))), :116-118 (cosine
 *   I/sqrt(a*b)), each in IEEE float32 with nan_to_num (0/0 -> 0).
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).  Floating
 * point contraction is off so that every product and sum rounds exactly as
 * written, matching the CUDA kernels, which use explicitly rounded
 * intrinsics in the same places.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    double key;   /* float64 key (mode 0) or float32 key widened (mode 1) */
    uint32_t gen; /* generation rank, p1-major */
    uint16_t p1, p2;
} cand_t;

/* key descending, ties: later generation first */
static int cand_cmp(const void* x, const void* y) {
    const cand_t* a = (const cand_t*)x;
    const cand_t* b = (const cand_t*)y;
    if (a->key > b->key) return -1;
    if (a->key < b->key) return 1;
    if (a->gen > b->gen) return -1;
    if (a->gen < b->gen) return 1;
    return 0;
}

static inline double peak_a(const double* a, int64_t i) { return a ? a[i] : 1.0; }

/* sequential sum of squares of w = a*b, float64 (mode 0) */
static double norm2_f64(const double* a, const double* b, int64_t lo, int64_t hi) {
    double s = 0.0;
    for (int64_t i = lo; i < hi; ++i) {
        double w = peak_a(a, i) * b[i];
        double w2 = w * w;
        s = s + w2;
    }
    return s;
}

/* float32 running sum as the reference kernel's query-norm loop (mode 1) */
static float norm2_f32(const double* a, const double* b, int64_t lo, int64_t hi) {
    float s = 0.0f;
    for (int64_t i = lo; i < hi; ++i) {
        double w = peak_a(a, i) * b[i];
        s = (float)((double)s + w * w);
    }
    return s;
}

/* Append the f64-mode candidates of one pair at `shift` (matchms find_matches
 * + collect_peak_pairs) to cands[*n..]; returns 1 when match_limit is reached
 * (overflow). */
static int gen_f64(const float* rmz, const double* ra, const double* rb, int64_t r0, int64_t nr,
                   const float* qmz, const double* qa, const double* qb, int64_t q0, int64_t nq,
                   double tol, double shift, int match_limit, cand_t* cands, int* n) {
    int64_t lowest = 0;
    for (int64_t p1 = 0; p1 < nr; ++p1) {
        double mz1 = (double)rmz[r0 + p1];
        double lo = mz1 - tol, hi = mz1 + tol;
        double w1 = peak_a(ra, r0 + p1) * rb[r0 + p1];
        for (int64_t p2 = lowest; p2 < nq; ++p2) {
            double mz2 = (double)qmz[q0 + p2] + shift;
            if (mz2 > hi) break;
            if (mz2 < lo) {
                lowest = p2 + 1;
                continue;
            }
            double key = (w1 * peak_a(qa, q0 + p2)) * qb[q0 + p2];
            cands[*n].key = key;
            cands[*n].gen = (uint32_t)*n;
            cands[*n].p1 = (uint16_t)p1;
            cands[*n].p2 = (uint16_t)p2;
            if (++*n >= match_limit) return 1;
        }
    }
    return 0;
}

/* greedy over sorted candidates; score and matches (f64 mode) */
static void greedy_f64(cand_t* cands, int n, int64_t nr, int64_t nq, uint8_t* used_r,
                       uint8_t* used_q, double n2r, double n2q, float* out_score,
                       int32_t* out_matches) {
    qsort(cands, (size_t)n, sizeof(cand_t), cand_cmp);
    memset(used_r, 0, (size_t)nr);
    memset(used_q, 0, (size_t)nq);
    double score = 0.0;
    int matches = 0;
    for (int m = 0; m < n; ++m) {
        int p1 = cands[m].p1, p2 = cands[m].p2;
        if (!used_r[p1] && !used_q[p2]) {
            used_r[p1] = 1;
            used_q[p2] = 1;
            score = score + cands[m].key;
            ++matches;
        }
    }
    *out_score = (float)(score / (sqrt(n2r) * sqrt(n2q)));
    *out_matches = matches;
}

static void one_pair(const float* rmz, const double* ra, const double* rb, int64_t r0, int64_t nr,
                     const float* qmz, const double* qa, const double* qb, int64_t q0, int64_t nq,
                     double tol, double shift, int match_limit, int key_mode, double n2r, double n2q,
                     cand_t* cands, uint8_t* used_r, uint8_t* used_q,
                     float* out_score, int32_t* out_matches, uint8_t* out_overflow) {
    *out_score = 0.0f;
    *out_matches = 0;
    *out_overflow = 0;
    if (nr == 0 || nq == 0) return;

    int n = 0;
    int overflow = 0;
    int64_t lowest = 0;
    for (int64_t p1 = 0; p1 < nr && !overflow; ++p1) {
        double mz1 = (double)rmz[r0 + p1];
        double lo = mz1 - tol, hi = mz1 + tol;
        double w1 = peak_a(ra, r0 + p1) * rb[r0 + p1];
        for (int64_t p2 = lowest; p2 < nq; ++p2) {
            double mzq = (double)qmz[q0 + p2];
            int above, below;
            if (key_mode == 0) {
                double mz2 = mzq + shift;
                above = mz2 > hi;
                below = mz2 < lo;
            } else {
                double delta = (mzq + shift) - mz1;
                above = delta > tol;
                below = delta < -tol;
            }
            if (above) break;
            if (below) {
                lowest = p2 + 1;
                continue;
            }
            double a2 = peak_a(qa, q0 + p2), b2 = qb[q0 + p2];
            double key;
            if (key_mode == 0) {
                key = (w1 * a2) * b2;
            } else {
                key = (double)(float)(w1 * (a2 * b2));
            }
            cands[n].key = key;
            cands[n].gen = (uint32_t)n;
            cands[n].p1 = (uint16_t)p1;
            cands[n].p2 = (uint16_t)p2;
            ++n;
            if (n >= match_limit) {
                overflow = 1;
                break;
            }
        }
    }
    *out_overflow = (uint8_t)overflow;
    if (n == 0) return;

    qsort(cands, (size_t)n, sizeof(cand_t), cand_cmp);
    memset(used_r, 0, (size_t)nr);
    memset(used_q, 0, (size_t)nq);
    double score = 0.0;
    int matches = 0;
    for (int m = 0; m < n; ++m) {
        int p1 = cands[m].p1, p2 = cands[m].p2;
        if (!used_r[p1] && !used_q[p2]) {
            used_r[p1] = 1;
            used_q[p2] = 1;
            score = score + cands[m].key;
            ++matches;
        }
    }
    double s;
    if (key_mode == 0) {
        s = score / (sqrt(n2r) * sqrt(n2q));
    } else {
        float nr32 = sqrtf((float)n2r), nq32 = sqrtf((float)n2q);
        s = score / (double)(nr32 * nq32);
    }
    *out_score = (float)s;
    *out_matches = matches;
}

/*
 * Dense greedy cosine over all (reference i, query j) pairs.
 * Spectra are CSR: peaks [off[i], off[i+1]) with m/z ascending.
 * Outputs are row-major with leading dimension ld (>= n_q).
 * n_threads <= 0 uses the OpenMP default.
 * Returns 0, or -1 on bad arguments / allocation failure.
 */
int oracle_cosine_greedy(const float* rmz, const double* ra, const double* rb, const int64_t* roff,
                         int64_t n_ref, const float* qmz, const double* qa, const double* qb,
                         const int64_t* qoff, int64_t n_q, double tol, double shift,
                         int match_limit, int key_mode, float* out_score, int32_t* out_matches,
                         uint8_t* out_overflow, int64_t ld, int n_threads) {
    if (match_limit < 1 || ld < n_q || (key_mode != 0 && key_mode != 1)) return -1;
    int64_t max_nr = 0, max_nq = 0;
    for (int64_t i = 0; i < n_ref; ++i)
        if (roff[i + 1] - roff[i] > max_nr) max_nr = roff[i + 1] - roff[i];
    for (int64_t j = 0; j < n_q; ++j)
        if (qoff[j + 1] - qoff[j] > max_nq) max_nq = qoff[j + 1] - qoff[j];
    if (max_nr > 65536 || max_nq > 65536) return -1;

    double* n2r = (double*)malloc(sizeof(double) * (size_t)(n_ref > 0 ? n_ref : 1));
    double* n2q = (double*)malloc(sizeof(double) * (size_t)(n_q > 0 ? n_q : 1));
    if (!n2r || !n2q) {
        free(n2r);
        free(n2q);
        return -1;
    }
    for (int64_t i = 0; i < n_ref; ++i)
        n2r[i] = key_mode == 0 ? norm2_f64(ra, rb, roff[i], roff[i + 1])
                               : (double)norm2_f32(ra, rb, roff[i], roff[i + 1]);
    for (int64_t j = 0; j < n_q; ++j)
        n2q[j] = key_mode == 0 ? norm2_f64(qa, qb, qoff[j], qoff[j + 1])
                               : (double)norm2_f32(qa, qb, qoff[j], qoff[j + 1]);

    int failed = 0;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel
#endif
    {
        cand_t* cands = (cand_t*)malloc(sizeof(cand_t) * (size_t)match_limit);
        uint8_t* used_r = (uint8_t*)malloc((size_t)max_nr + 1);
        uint8_t* used_q = (uint8_t*)malloc((size_t)max_nq + 1);
        if (!cands || !used_r || !used_q) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
            failed = 1;
        } else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
            for (int64_t i = 0; i < n_ref; ++i) {
                for (int64_t j = 0; j < n_q; ++j) {
                    int64_t o = i * ld + j;
                    one_pair(rmz, ra, rb, roff[i], roff[i + 1] - roff[i], qmz, qa, qb, qoff[j],
                             qoff[j + 1] - qoff[j], tol, shift, match_limit, key_mode, n2r[i],
                             n2q[j], cands, used_r, used_q, &out_score[o], &out_matches[o],
                             &out_overflow[o]);
                }
            }
        }
        free(cands);
        free(used_r);
        free(used_q);
    }
    free(n2r);
    free(n2q);
    return failed ? -1 : 0;
}

/*
 * Dense modified cosine over all (reference i, query j) pairs (f64 mode; see
 * the header).  rprec / qprec: precursor m/z per spectrum.  Returns 0, or -1
 * on bad arguments / allocation failure.
 */
int oracle_modified_cosine(const float* rmz, const double* ra, const double* rb,
                           const int64_t* roff, const double* rprec, int64_t n_ref,
                           const float* qmz, const double* qa, const double* qb,
                           const int64_t* qoff, const double* qprec, int64_t n_q, double tol,
                           int match_limit, float* out_score, int32_t* out_matches,
                           uint8_t* out_overflow, int64_t ld, int n_threads) {
    if (match_limit < 1 || ld < n_q) return -1;
    int64_t max_nr = 0, max_nq = 0;
    for (int64_t i = 0; i < n_ref; ++i)
        if (roff[i + 1] - roff[i] > max_nr) max_nr = roff[i + 1] - roff[i];
    for (int64_t j = 0; j < n_q; ++j)
        if (qoff[j + 1] - qoff[j] > max_nq) max_nq = qoff[j + 1] - qoff[j];
    if (max_nr > 65536 || max_nq > 65536) return -1;
    int failed = 0;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel
#endif
    {
        cand_t* cands = (cand_t*)malloc(sizeof(cand_t) * (size_t)match_limit);
        uint8_t* used_r = (uint8_t*)malloc((size_t)max_nr + 1);
        uint8_t* used_q = (uint8_t*)malloc((size_t)max_nq + 1);
        if (!cands || !used_r || !used_q) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
            failed = 1;
        } else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
            for (int64_t i = 0; i < n_ref; ++i) {
                const int64_t r0 = roff[i], nr = roff[i + 1] - roff[i];
                const double n2r = norm2_f64(ra, rb, roff[i], roff[i + 1]);
                for (int64_t j = 0; j < n_q; ++j) {
                    const int64_t o = i * ld + j;
                    const int64_t q0 = qoff[j], nq = qoff[j + 1] - qoff[j];
                    out_score[o] = 0.0f;
                    out_matches[o] = 0;
                    out_overflow[o] = 0;
                    if (nr == 0 || nq == 0) continue;
                    const double mass_shift = rprec[i] - qprec[j];
                    int n = 0;
                    int ovf = gen_f64(rmz, ra, rb, r0, nr, qmz, qa, qb, q0, nq, tol, 0.0,
                                      match_limit, cands, &n);
                    if (!ovf)
                        ovf = gen_f64(rmz, ra, rb, r0, nr, qmz, qa, qb, q0, nq, tol, mass_shift,
                                      match_limit, cands, &n);
                    out_overflow[o] = (uint8_t)ovf;
                    if (n == 0) continue;
                    greedy_f64(cands, n, nr, nq, used_r, used_q, n2r,
                               norm2_f64(qa, qb, qoff[j], qoff[j + 1]), &out_score[o],
                               &out_matches[o]);
                }
            }
        }
        free(cands);
        free(used_r);
        free(used_q);
    }
    return failed ? -1 : 0;
}

/*
 * Greedy cosine over an explicit list of pairs (ref index, query index); used
 * to check large runs on sampled pairs.
 */
int oracle_cosine_greedy_pairs(const float* rmz, const double* ra, const double* rb,
                               const int64_t* roff, const float* qmz, const double* qa,
                               const double* qb, const int64_t* qoff, const int64_t* pair_r,
                               const int64_t* pair_q, int64_t n_pairs, double tol, double shift,
                               int match_limit, int key_mode, float* out_score,
                               int32_t* out_matches, uint8_t* out_overflow, int n_threads) {
    if (match_limit < 1 || (key_mode != 0 && key_mode != 1)) return -1;
    int failed = 0;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel
#endif
    {
        cand_t* cands = (cand_t*)malloc(sizeof(cand_t) * (size_t)match_limit);
        uint8_t* used_r = (uint8_t*)malloc(65537);
        uint8_t* used_q = (uint8_t*)malloc(65537);
        if (!cands || !used_r || !used_q) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
            failed = 1;
        } else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
            for (int64_t k = 0; k < n_pairs; ++k) {
                int64_t i = pair_r[k], j = pair_q[k];
                int64_t nr = roff[i + 1] - roff[i], nq = qoff[j + 1] - qoff[j];
                if (nr > 65536 || nq > 65536) {
                    out_score[k] = NAN;
                    out_matches[k] = -1;
                    out_overflow[k] = 0;
                    continue;
                }
                double n2r = key_mode == 0 ? norm2_f64(ra, rb, roff[i], roff[i + 1])
                                           : (double)norm2_f32(ra, rb, roff[i], roff[i + 1]);
                double n2q = key_mode == 0 ? norm2_f64(qa, qb, qoff[j], qoff[j + 1])
                                           : (double)norm2_f32(qa, qb, qoff[j], qoff[j + 1]);
                one_pair(rmz, ra, rb, roff[i], nr, qmz, qa, qb, qoff[j], nq, tol, shift,
                         match_limit, key_mode, n2r, n2q, cands, used_r, used_q, &out_score[k],
                         &out_matches[k], &out_overflow[k]);
            }
        }
        free(cands);
        free(used_r);
        free(used_q);
    }
    return failed ? -1 : 0;
}

/*
 * Fingerprint similarity on bit-packed rows (n_words uint32 per row, bit k of
 * the fingerprint in word k/32, bit k%32).  measure: 0 jaccard, 1 dice,
 * 2 cosine.  Rows whose valid flag is 0 (fingerprint missing) produce `fill`
 * in every pair they take part in (CudaFingerprintSimilarity.py:147-177).
 * valid == NULL means all rows are valid.
 */
int oracle_fingerprint(int measure, const uint32_t* rbits, const uint8_t* rvalid, int64_t n_ref,
                       const uint32_t* qbits, const uint8_t* qvalid, int64_t n_q, int n_words,
                       float fill, float* out, int64_t ld, int n_threads) {
    if (measure < 0 || measure > 2 || ld < n_q || n_words < 0) return -1;
    int32_t* pr = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n_ref > 0 ? n_ref : 1));
    int32_t* pq = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n_q > 0 ? n_q : 1));
    if (!pr || !pq) {
        free(pr);
        free(pq);
        return -1;
    }
    for (int64_t i = 0; i < n_ref; ++i) {
        int c = 0;
        for (int w = 0; w < n_words; ++w) c += __builtin_popcount(rbits[i * n_words + w]);
        pr[i] = c;
    }
    for (int64_t j = 0; j < n_q; ++j) {
        int c = 0;
        for (int w = 0; w < n_words; ++w) c += __builtin_popcount(qbits[j * n_words + w]);
        pq[j] = c;
    }
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < n_ref; ++i) {
        for (int64_t j = 0; j < n_q; ++j) {
            float v;
            if ((rvalid && !rvalid[i]) || (qvalid && !qvalid[j])) {
                v = fill;
            } else {
                int inter = 0;
                for (int w = 0; w < n_words; ++w)
                    inter += __builtin_popcount(rbits[i * n_words + w] & qbits[j * n_words + w]);
                float fi = (float)inter, fa = (float)pr[i], fb = (float)pq[j];
                if (measure == 0) {
                    float uni = (fa + fb) - fi;
                    v = fi / uni;
                } else if (measure == 1) {
                    v = 2.0f * (fi / (fa + fb));
                } else {
                    v = fi / sqrtf(fa * fb);
                }
                if (isnan(v)) v = 0.0f;
            }
            out[i * ld + j] = v;
        }
    }
    free(pr);
    free(pq);
    return 0;
}
