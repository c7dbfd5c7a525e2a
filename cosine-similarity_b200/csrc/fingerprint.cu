// Fingerprint similarity (Jaccard / Dice / cosine) on bit-packed fingerprints.
//
// Replaces cudams/similarity/vector_similarity_functions.py:12-119, which
// computes I = R @ Q^T as a dense float32 GEMM over 0/1 values and then runs
// four elementwise passes.  Here the intersection counts I come from the
// tensor cores as an exact 4-bit float GEMM over 0/1 values (tcgen05
// kind::mxf4, float32 accumulators in TMEM), the row bit counts from
// popcounts of the packed words, and the epilogue forms the measure in IEEE float32 in the
// reference's order of operations, mapping 0/0 to 0 (nan_to_num), or writes
// `fill` for rows/columns without a fingerprint.  The kernel is described
// below, above namespace umma.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "cms_internal.cuh"

namespace cms {
namespace {

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
    // test hook (environment variable CMS_TEST_STALL=mma): the MMA issuer
    // issues nothing, so the producers' and the epilogue's bounded waits run
    // out and the error path (abort flag, error bit, TMEM release) is taken
    int test_stall;
};

// Branch-free IEEE float32 division and square root for the operands the
// measures produce.  Both follow the published Newton-Raphson/FMA schemes
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990; J.-M. Muller et al.,
// Handbook of Floating-Point Arithmetic, 2nd ed., 2018, sections 4.7-4.8):
// the hardware approximation, one Newton step, and one FMA correction of the
// result.  They carry no special-case branch, so the 32 elements of a lane's
// chunk interleave freely.  Correct rounding is established by exhaustive
// comparison with CUDA's __fdiv_rn / __fsqrt_rn / __frcp_rn on the device
// (cms_fingerprint_arith_check) over every operand that can occur: n / d for
// integers 0 <= n <= d <= 65536 (Jaccard, Dice: 32768-bit fingerprints at
// most), sqrt(p) for every float p in [1, 2^30] (p = a * b rounded), the
// reciprocal of every such sqrt(p) (which makes the quotient correctly
// rounded for every numerator, by Markstein's theorem), and every cosine
// triple of fingerprints up to 2048 bits.  d = 0 or p = 0 give NaN (0/0
// only), which the measure maps to 0.
__device__ __forceinline__ float rcp_fp(float d) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(d));
    return __fmaf_rn(__fmaf_rn(-d, y, 1.0f), y, y);
}
__device__ __forceinline__ float div_fp(float n, float d) {
    const float y = rcp_fp(d);
    const float q = __fmul_rn(n, y);
    return __fmaf_rn(__fmaf_rn(-q, d, n), y, q);
}
__device__ __forceinline__ float sqrt_fp(float p) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(p));
    float g = __fmul_rn(p, r), h = __fmul_rn(0.5f, r);
    const float e = __fmaf_rn(-g, h, 0.5f);
    g = __fmaf_rn(g, e, g);
    h = __fmaf_rn(h, e, h);
    return __fmaf_rn(__fmaf_rn(-g, g, p), h, g);
}

// The measure from the intersection count fi and the row bit counts fa, fb
// (all exact integers in float32), in the reference's order of operations.
// Only 0/0 is NaN here (fi > 0 implies a nonzero denominator), and fmaxf maps
// it to 0 while keeping every other value, which is >= 0.
template <int MEASURE>
__device__ __forceinline__ float measure_of(float fi, float fa, float fb) {
    float v;
    if (MEASURE == CMS_FP_JACCARD) {
        v = div_fp(fi, __fsub_rn(__fadd_rn(fa, fb), fi));
    } else if (MEASURE == CMS_FP_DICE) {
        v = __fmul_rn(2.0f, div_fp(fi, __fadd_rn(fa, fb)));
    } else {
        v = div_fp(fi, sqrt_fp(__fmul_rn(fa, fb)));
    }
    return fmaxf(v, 0.0f);
}

// ---------------------------------------------------------------------------
// Tensor-core path: I = R . Q^T on tcgen05 (kind::mxf4, exact in float32)
// ---------------------------------------------------------------------------
// The bit-packed rows are expanded on the fly, straight into the
// shared-memory operand stages (no expanded copy in global memory), to packed
// 4-bit floats (E2M1) of value 0 or 1: nibble 0x2 is 1.0.  Every block scale
// factor is 1.0 (E8M0 0x7F), so a dot product over K = n_words * 32 is the
// intersection count, exact in the float32 accumulator (counts <= 32768 are
// integers far below 2^24).  The K order inside a 32-bit word is permuted by
// the expansion -- nibble t of output word v_s holds bit 4t + s -- identically
// for both operands, which leaves every dot product unchanged.  Against 0/1
// bytes (kind::i8) this halves the expansion work, the shared-memory operand
// bytes and the MMA instructions per K bit.
//
// One persistent CTA per SM, warp-specialised:
//   warps 0-7   epilogue: TMEM -> registers (tcgen05.ld 32x32b), measure in
//               IEEE float32, 32 x 32 chunks staged in shared memory and
//               written by 2-D tensor stores.  Warps w and w+4 share TMEM
//               lanes 32*(w%4)..+31 (rows) and take alternate 32-column
//               chunks of the 224 columns.
//   warps 8-11  producers: per 256-bit K block, take the 32 bytes of each of
//               the tile's 128 reference and 224 query rows from the ring,
//               expand them to 128 bytes each in the canonical K-major
//               SWIZZLE_128B layout, make the writes visible to the tensor
//               core (fence.proxy.async), and count the rows' bits (popcounts
//               of the whole row per tile).
//   warp 12     MMA issuer: one thread issues 4 x tcgen05.mma (M=128, N=224,
//               K=64) per stage and commits stage release / accumulator ready.
//   warp 13     loader: one thread brings each K block of the tile's packed
//               rows into a 4-deep shared-memory ring with two 2-D tensor
//               loads (4 KB + 7 KB), so that the producers' reads are
//               shared-memory reads instead of 16-byte global loads from 352
//               rows 256 bytes apart.  When the rows do not meet the
//               tensor-load rules the producers load them themselves.
// Two 128 x 224 float32 accumulators (TMEM columns 0 and 256): the epilogue
// of one tile overlaps the MMAs of the next.  The block scale factors sit in
// columns 224-255, all 1.0: A's at column 224 (four columns for 128 rows),
// B's at column 232 (seven columns for 224 rows); filling the whole range
// with 0x7F bytes makes every factor 1.0 whatever byte of it an MMA reads.  Every mbarrier wait is bounded in
// time; on expiry the kernel sets an error bit, every role stops, and TMEM is
// released before exit.
namespace umma {

constexpr int kBM = 128;           // reference rows per tile (TMEM lanes)
constexpr int kBN = 224;           // query rows per tile (accumulator columns)
constexpr int kAccStride = 256;    // TMEM columns between the two accumulators
constexpr int kSfCol = 224;        // scale factors: columns 224..255
constexpr int kSfaCol = kSfCol, kSfbCol = kSfCol + 8;
constexpr int kBKBytes = 128;      // expanded K bytes per stage (one 128B swizzle row)
constexpr int kBKWords = kBKBytes / 16;  // packed uint32 words per row per stage (256 bits)
constexpr int kStages = 3;
constexpr int kABytes = kBM * kBKBytes;  // 16 KB
constexpr int kBBytes = kBN * kBKBytes;  // 28 KB
constexpr int kStageBytes = kABytes + kBBytes;
constexpr int kEpiWarps = 8;      // a multiple of 4 (one set per TMEM lane quarter)
constexpr int kEpiSets = kEpiWarps / 4;
constexpr int kProdWarps = 4;
constexpr int kMmaWarp = kEpiWarps + kProdWarps;
constexpr int kLoadWarp = kMmaWarp + 1;
constexpr int kThreads = (kEpiWarps + kProdWarps + 2) * 32;
constexpr int kProdThreads = kProdWarps * 32;
constexpr int kTmemCols = 512;
constexpr unsigned long long kWaitNs = 2000000000ull;  // bounded waits: 2 s

// shared-memory layout (offsets from a 1024-byte aligned base)
constexpr int kOffStages = 0;
// per epilogue warp: one 32 x 32 float chunk of the output, staged for a
// tensor store (128-byte swizzle: 16-byte piece j of row r at j ^ (r % 8))
constexpr int kStgBytes = 32 * 32 * 4;
constexpr int kOffStg = kStages * kStageBytes;
// ring of packed K blocks brought by 2-D tensor loads: kBM + kBN rows of
// kBKWords words (32 bytes) each, row-major, 32-byte swizzle (the 16-byte
// halves of row r swapped when r & 4)
constexpr int kIn = 4;
constexpr int kInABytes = kBM * kBKWords * 4;  // 4 KB
constexpr int kInBytes = (kBM + kBN) * kBKWords * 4;  // 11 KB
constexpr int kOffIn = kOffStg + kEpiWarps * kStgBytes;
constexpr int kOffPop = kOffIn + kIn * kInBytes;  // float pa[2][kBM], pb[2][kBN]
constexpr int kOffBar = kOffPop + 2 * (kBM + kBN) * 4;
// barriers: full[S], empty[S], tfull[2], tempty[2], pfull[2], pempty[2], done,
// in_full[kIn], in_empty[kIn]
constexpr int kNumBars = 2 * kStages + 9 + 2 * kIn;
constexpr int kOffTmemSlot = kOffBar + kNumBars * 8;
constexpr int kOffAbort = kOffTmemSlot + 4;
constexpr int kSmemBytes = kOffAbort + 4 + 1024;  // + alignment slack

// Block-scaled UMMA instruction descriptor: A and B E2M1 (bits 7-9, 10-12:
// 1), both K-major, N >> 3 at bits 17-22, scale factors E8M0 (bit 23), M >> 4
// at bits 24-28, scale-factor byte 0 of A and B (bits 29-30, 4-5), K = 64
// (bit 31 clear); the accumulator is float32.
constexpr uint32_t kIdesc = (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) | (1u << 23) |
                            ((uint32_t)(kBM >> 4) << 24);
static_assert(kBN % 32 == 0 && kBN <= kSfCol && kSfbCol + kBN / 32 <= kAccStride,
              "accumulator and scale-factor columns overlap");
static_assert(kSmemBytes <= 227 * 1024, "shared memory");
static_assert(kInABytes % 1024 == 0 && kInBytes % 1024 == 0 && kOffIn % 1024 == 0,
              "tensor-load destinations 1024-byte aligned");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase of `parity` to complete, for at most kWaitNs; on expiry
// (or, unless `drain`, when another role already gave up) raise the CTA's
// abort flag and return false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                          bool drain = false) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (!drain && *abort_flag) return false;
        if (globaltimer() - t0 > kWaitNs) {
            *abort_flag = 1;
            return false;
        }
    }
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// SWIZZLE_128B K-major shared-memory matrix descriptor (8-row atoms of
// 128-byte rows, atoms 1024 bytes apart; Blackwell descriptor version 1)
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) |
           ((uint64_t)(1024u >> 4) << 32) | ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}
__device__ __forceinline__ void umma_mxf4(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t sfa, uint32_t sfb, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::mxf4.block_scale.block32 [%0], %1, %2, %3, [%5], [%6], "
        "p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(sfa), "r"(sfb));
}
// Fill 32 TMEM columns of this warp's 32 lanes with one 32-bit value
__device__ __forceinline__ void tmem_fill32(uint32_t taddr, uint32_t x) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
        "{%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
        "%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1};" ::"r"(taddr),
        "r"(x)
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}
// Load 32 TMEM columns of this warp's 32 lanes (lane i: row i, r[j]: column
// j) without waiting; tmem_wait_ld completes it.  The wait names the
// destination registers as read-write operands, so the compiler can neither
// read nor move them before the data has arrived, and the load overlaps
// whatever the warp does in between.
__device__ __forceinline__ void tmem_ld32_async(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
          "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                   "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                   "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]),
                   "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]),
                   "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]),
                   "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    tmem_ld32_async(taddr, r);
    tmem_wait_ld(r);
}

// 2-D tensor store of one staged chunk (box 32 x 32 floats at column x, row
// y; elements outside the output are not written), and its completion
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, uint32_t src, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(x), "r"(y), "r"(src)
        : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// 2-D tensor load of one box into shared memory, completing on `bar` (no
// multicast: the source is this GPU's own memory and one CTA reads it)
__device__ __forceinline__ void tma_load_2d(const CUtensorMap* map, uint32_t dst, uint64_t* bar,
                                            int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
        "{%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tma_store_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void tma_store_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

struct Geometry {
    int n_tm, n_tn;       // tiles along the reference / query side
    int64_t n_tiles;
    int kb;               // K blocks of kBKWords packed words (>= 1)
};

// Tile t -> (tm, tn); under `sym`, tiles wholly below the diagonal are skipped
// by every role alike.
__device__ __forceinline__ bool tile_live(const FpParams& P, const Geometry& G, int64_t t, int& tm,
                                          int& tn) {
    tm = (int)(t / G.n_tn);
    tn = (int)(t - (int64_t)tm * G.n_tn);
    if (!P.sym) return true;
    return (int64_t)tm * kBM <= (int64_t)tn * kBN + (kBN - 1);
}

// 32 packed bytes (8 words) of one row's K block kb, zero beyond the matrix
struct Bits {
    uint4 lo, hi;
};
__device__ __forceinline__ Bits load_bits(const uint32_t* base, int64_t row, int64_t n_rows,
                                          int n_words, int kb, bool vec) {
    Bits v{make_uint4(0u, 0u, 0u, 0u), make_uint4(0u, 0u, 0u, 0u)};
    if (row >= n_rows) return v;
    const uint32_t* p = base + row * (int64_t)n_words + kb * kBKWords;
    const int w0 = kb * kBKWords;
    if (vec && w0 + kBKWords <= n_words) {
        v.lo = __ldg(reinterpret_cast<const uint4*>(p));
        v.hi = __ldg(reinterpret_cast<const uint4*>(p) + 1);
        return v;
    }
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) w[i] = w0 + i < n_words ? __ldg(p + i) : 0u;
    v.lo = make_uint4(w[0], w[1], w[2], w[3]);
    v.hi = make_uint4(w[4], w[5], w[6], w[7]);
    return v;
}
__device__ __forceinline__ int popc_bits(const Bits& b) {
    return __popc(b.lo.x) + __popc(b.lo.y) + __popc(b.lo.z) + __popc(b.lo.w) + __popc(b.hi.x) +
           __popc(b.hi.y) + __popc(b.hi.z) + __popc(b.hi.w);
}

// Expand one row's 256 bits into 128 bytes of E2M1 nibbles (0x2 = 1.0 where
// the bit is set) at row r of an operand stage (SWIZZLE_128B: 16-byte chunk c
// of row r sits at chunk c ^ (r % 8)).  Word q goes to chunk q; its output
// word s holds bits 4t + s at bit 1 of nibble t.
__device__ __forceinline__ void expand_row(unsigned char* stage, int r, const Bits& bits) {
    unsigned char* row = stage + (r >> 3) * 1024 + (r & 7) * 128;
    const uint32_t w[8] = {bits.lo.x, bits.lo.y, bits.lo.z, bits.lo.w,
                           bits.hi.x, bits.hi.y, bits.hi.z, bits.hi.w};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const uint32_t m = 0x22222222u;
        *reinterpret_cast<uint4*>(row + ((q ^ (r & 7)) << 4)) =
            make_uint4((w[q] << 1) & m, w[q] & m, (w[q] >> 1) & m, (w[q] >> 2) & m);
    }
}

// use_in: the packed rows come through the shared-memory ring by tensor
// loads (in_r, in_q); else each producer thread loads its rows itself
template <int MEASURE>
__global__ void __launch_bounds__(kThreads, 1)
    fp_umma_kernel(FpParams P, Geometry G, uint32_t* err,
                   const __grid_constant__ CUtensorMap out_map, int use_map,
                   const __grid_constant__ CUtensorMap in_r, const __grid_constant__ CUtensorMap in_q,
                   int use_in) {
    extern __shared__ unsigned char smem_dyn[];
    unsigned char* sm = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~uintptr_t(1023));
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kOffBar);
    uint64_t* full = bars;                    // [kStages] producers -> MMA
    uint64_t* empty = bars + kStages;         // [kStages] MMA -> producers
    uint64_t* tfull = bars + 2 * kStages;     // [2] MMA -> epilogue
    uint64_t* tempty = tfull + 2;             // [2] epilogue -> MMA
    uint64_t* pfull = tempty + 2;             // [2] producers -> epilogue (popcounts)
    uint64_t* pempty = pfull + 2;             // [2] epilogue -> producers
    uint64_t* done = pempty + 2;              // MMA completion before TMEM release
    uint64_t* in_full = done + 1;             // [kIn] tensor loads -> producers
    uint64_t* in_empty = in_full + kIn;       // [kIn] producers -> loader
    // row bit counts of the tile (float; -1: no fingerprint)
    float* pa = reinterpret_cast<float*>(sm + kOffPop);  // [2][kBM]
    float* pb = pa + 2 * kBM;                            // [2][kBN]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kOffTmemSlot);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + kOffAbort);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], kProdThreads);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], kEpiWarps * 32);
            mbar_init(&pfull[a], kProdThreads);
            mbar_init(&pempty[a], kEpiWarps * 32);
        }
        mbar_init(done, 1);
        for (int s = 0; s < kIn; ++s) {
            mbar_init(&in_full[s], 1);
            mbar_init(&in_empty[s], kProdThreads);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {  // TMEM: all 512 columns, two accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    if (warp < 4) {  // every block scale factor 1.0 (lanes 32*warp..+31)
        tmem_fill32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)kSfCol, 0x7F7F7F7Fu);
        tc_fence_before();
    }
    __syncthreads();
    tc_fence_after();

    if (warp >= kEpiWarps && warp < kEpiWarps + kProdWarps) {
        // ------------------------------ producers ------------------------------
        const int pt = threadIdx.x - kEpiWarps * 32;  // 0..127
        const bool vec = (P.n_words % kBKWords) == 0 &&
                         (reinterpret_cast<uintptr_t>(P.r) & 15) == 0 &&
                         (reinterpret_cast<uintptr_t>(P.q) & 15) == 0;
        int stage = 0, islot = 0;
        uint32_t phase = 0, iph = 0;
        int64_t it = 0;  // tiles taken by this CTA
        bool ok = true;
        for (int64_t t = blockIdx.x; t < G.n_tiles && ok; t += gridDim.x) {
            int tm, tn;
            if (!tile_live(P, G, t, tm, tn)) continue;
            const int acc = (int)(it & 1);
            const uint32_t acc_phase = (uint32_t)((it >> 1) & 1);
            ++it;
            const int64_t ra = (int64_t)tm * kBM + pt;
            // query rows pt and (for pt < kBN - 128) pt + 128 of the tile
            const bool two_b = pt + 128 < kBN;
            const int64_t qb0 = (int64_t)tn * kBN + pt;
            const int64_t qb1 = two_b ? qb0 + 128 : P.n_q;  // past the end: zero bits
            int ca = 0, cb0 = 0, cb1 = 0;
            Bits xa{}, xb0{}, xb1{};
            if (!use_in) {
                xa = load_bits(P.r, ra, P.n_r, P.n_words, 0, vec);
                xb0 = load_bits(P.q, qb0, P.n_q, P.n_words, 0, vec);
                xb1 = load_bits(P.q, qb1, P.n_q, P.n_words, 0, vec);
            }
            for (int kb = 0; kb < G.kb; ++kb) {
                Bits a = xa, b0 = xb0, b1 = xb1;
                if (use_in) {  // this block's rows from the ring
                    if (!mbar_wait(&in_full[islot], iph, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const uint4* in = reinterpret_cast<const uint4*>(sm + kOffIn + islot * kInBytes);
                    // 32-byte swizzle: the two 16-byte halves of row r are
                    // swapped when bit 2 of r is set (the same for all three
                    // rows of this thread), so that eight lanes read eight
                    // different bank groups
                    const int sw = (pt >> 2) & 1;
                    a = Bits{in[2 * pt + sw], in[2 * pt + (sw ^ 1)]};
                    b0 = Bits{in[2 * (kBM + pt) + sw], in[2 * (kBM + pt) + (sw ^ 1)]};
                    if (two_b)
                        b1 = Bits{in[2 * (kBM + pt + 128) + sw], in[2 * (kBM + pt + 128) + (sw ^ 1)]};
                    mbar_arrive(&in_empty[islot]);
                    if (++islot == kIn) {
                        islot = 0;
                        iph ^= 1u;
                    }
                } else if (kb + 1 < G.kb) {  // next block's bits load while this one expands
                    xa = load_bits(P.r, ra, P.n_r, P.n_words, kb + 1, vec);
                    xb0 = load_bits(P.q, qb0, P.n_q, P.n_words, kb + 1, vec);
                    xb1 = load_bits(P.q, qb1, P.n_q, P.n_words, kb + 1, vec);
                }
                if (!mbar_wait(&empty[stage], phase ^ 1u, abort_flag)) {
                    ok = false;
                    break;
                }
                unsigned char* sa = sm + kOffStages + stage * kStageBytes;
                unsigned char* sb = sa + kABytes;
                expand_row(sa, pt, a);
                expand_row(sb, pt, b0);
                if (two_b) expand_row(sb, pt + 128, b1);
                ca += popc_bits(a);
                cb0 += popc_bits(b0);
                cb1 += popc_bits(b1);
                fence_proxy_async_smem();
                mbar_arrive(&full[stage]);
                if (++stage == kStages) {
                    stage = 0;
                    phase ^= 1u;
                }
            }
            if (!ok) break;
            // the tile's row popcounts (-1: no fingerprint) for its epilogue
            if (!mbar_wait(&pempty[acc], acc_phase ^ 1u, abort_flag)) break;
            const bool va = ra < P.n_r && (P.r_valid ? P.r_valid[ra] != 0 : true);
            const bool vb0 = qb0 < P.n_q && (P.q_valid ? P.q_valid[qb0] != 0 : true);
            const bool vb1 = qb1 < P.n_q && (P.q_valid ? P.q_valid[qb1] != 0 : true);
            pa[acc * kBM + pt] = va ? (float)ca : -1.0f;
            pb[acc * kBN + pt] = vb0 ? (float)cb0 : -1.0f;
            if (two_b) pb[acc * kBN + pt + 128] = vb1 ? (float)cb1 : -1.0f;
            mbar_arrive(&pfull[acc]);
        }
    } else if (warp == kLoadWarp) {
        // ------------------------------ loader ------------------------------
        // one thread brings each K block of the tile's packed rows into the
        // ring (rows and words past the end read as zero), up to kIn blocks
        // ahead of the producers
        if (lane == 0 && use_in) {
            int slot = 0;
            uint32_t ph = 0;
            uint32_t issued = 0, issued_ph = 0;  // per slot: a load was issued / its phase
            bool ok = true;
            for (int64_t t = blockIdx.x; t < G.n_tiles && ok; t += gridDim.x) {
                int tm, tn;
                if (!tile_live(P, G, t, tm, tn)) continue;
                for (int kb = 0; kb < G.kb; ++kb) {
                    if (!mbar_wait(&in_empty[slot], ph ^ 1u, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const uint32_t dst = smem_u32(sm + kOffIn + slot * kInBytes);
                    mbar_expect_tx(&in_full[slot], (uint32_t)kInBytes);
                    tma_load_2d(&in_r, dst, &in_full[slot], kb * kBKWords, tm * kBM);
                    tma_load_2d(&in_q, dst + kInABytes, &in_full[slot], kb * kBKWords, tn * kBN);
                    issued |= 1u << slot;
                    issued_ph = (issued_ph & ~(1u << slot)) | (ph << slot);
                    if (++slot == kIn) {
                        slot = 0;
                        ph ^= 1u;
                    }
                }
            }
            // every load issued has landed before the CTA may exit (no later
            // load went to the same slot, so its phase is the last one)
            for (int s = 0; s < kIn; ++s)
                if (issued & (1u << s)) mbar_wait(&in_full[s], (issued_ph >> s) & 1u, abort_flag, true);
        }
        __syncwarp();
    } else if (warp == kMmaWarp) {
        // ------------------------------ MMA issuer ------------------------------
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int64_t it = 0;
            bool ok = !P.test_stall;
            for (int64_t t = blockIdx.x; t < G.n_tiles && ok; t += gridDim.x) {
                int tm, tn;
                if (!tile_live(P, G, t, tm, tn)) continue;
                const int acc = (int)(it & 1);
                const uint32_t acc_phase = (uint32_t)((it >> 1) & 1);
                ++it;
                if (!mbar_wait(&tempty[acc], acc_phase ^ 1u, abort_flag)) break;
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(acc * kAccStride);
                for (int kb = 0; kb < G.kb; ++kb) {
                    if (!mbar_wait(&full[stage], phase, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(sm + kOffStages + stage * kStageBytes);
                    const uint32_t sb = sa + kABytes;
#pragma unroll
                    for (int k = 0; k < kBKBytes / 32; ++k)
                        umma_mxf4(d, smem_desc(sa + 32 * k), smem_desc(sb + 32 * k),
                                  tmem + (uint32_t)kSfaCol, tmem + (uint32_t)kSfbCol,
                                  (kb > 0 || k > 0) ? 1u : 0u);
                    umma_commit(&empty[stage]);  // stage free once these MMAs have read it
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) break;
                umma_commit(&tfull[acc]);  // accumulator ready
            }
            // every MMA issued by this thread completes before TMEM is released
            umma_commit(done);
            mbar_wait(done, 0, abort_flag, true);
        }
        __syncwarp();
    } else {
        // ------------------------------ epilogue ------------------------------
        const int quarter = warp & 3;        // TMEM lanes 32*quarter .. +31
        const int set = warp >> 2;           // which of the kEpiSets warps of this quarter
        const bool vec_out = (P.ld & 3) == 0 && (reinterpret_cast<uintptr_t>(P.out) & 15) == 0;
        unsigned char* stg = sm + kOffStg + warp * kStgBytes;
        int64_t it = 0;
        for (int64_t t = blockIdx.x; t < G.n_tiles; t += gridDim.x) {
            int tm, tn;
            if (!tile_live(P, G, t, tm, tn)) continue;
            const int acc = (int)(it & 1);
            const uint32_t acc_phase = (uint32_t)((it >> 1) & 1);
            ++it;
            // warp-uniform exits: the TMEM loads below are warp-collective
            if (!__all_sync(0xFFFFFFFFu, mbar_wait(&tfull[acc], acc_phase, abort_flag))) break;
            tc_fence_after();
            if (!__all_sync(0xFFFFFFFFu, mbar_wait(&pfull[acc], acc_phase, abort_flag))) break;
            const int row_l = quarter * 32 + lane;
            const float fa = pa[acc * kBM + row_l];
            const int64_t gr = (int64_t)tm * kBM + row_l;  // this lane's output row
            float* orow = P.out + gr * P.ld;
            // the quarter's warps take every kEpiSets-th 32-column chunk,
            // starting one further on each tile, so that the odd chunk of
            // the 224 columns goes to each warp in turn
            // chunk c's accumulator columns are read (into vn) while chunk
            // c - kEpiSets is computed and stored
            uint32_t vn[32];
            const uint32_t tbase =
                tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * kAccStride);
            const int c0 = (int)((set + it) % kEpiSets);
            __syncwarp();
            if (c0 < kBN / 32) tmem_ld32(tbase + (uint32_t)(c0 * 32), vn);
            for (int c = c0; c < kBN / 32; c += kEpiSets) {
                const int col_l = c * 32;  // first column of this chunk in the tile
                const int64_t gc0 = (int64_t)tn * kBN + col_l;
                uint32_t v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = vn[j];
                __syncwarp();
                if (c + kEpiSets < kBN / 32)
                    tmem_ld32_async(tbase + (uint32_t)((c + kEpiSets) * 32), vn);
                const float* pbc = pb + acc * kBN + col_l;
                // every row and column of the chunk has a fingerprint: no
                // per-element fill test
                const bool whole = __all_sync(0xFFFFFFFFu, fa >= 0.0f && pbc[lane] >= 0.0f);
                // a chunk inside the tensor map's columns is stored by the
                // warp (rows past the end hold the fill value and are clipped
                // by the store); the others lane by lane
                const bool tma_chunk = use_map && gc0 + 32 <= (P.n_q & ~int64_t(3));
                const bool live = tma_chunk ? (int64_t)tm * kBM + quarter * 32 < P.n_r
                                            : (gr < P.n_r && gc0 < P.n_q);
                if (live) {
                    float o[32];
                    const float4* pbv = reinterpret_cast<const float4*>(pbc);
                    if (whole) {
#pragma unroll
                        for (int j4 = 0; j4 < 8; ++j4) {
                            const float4 b4 = pbv[j4];
                            const float fb[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
                            for (int u = 0; u < 4; ++u)
                                o[4 * j4 + u] =
                                    measure_of<MEASURE>(__uint_as_float(v[4 * j4 + u]), fa, fb[u]);
                        }
                    } else {
#pragma unroll
                        for (int j4 = 0; j4 < 8; ++j4) {
                            const float4 b4 = pbv[j4];
                            const float fb[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const int j = 4 * j4 + u;
                                o[j] = (fa >= 0.0f && fb[u] >= 0.0f)
                                           ? measure_of<MEASURE>(__uint_as_float(v[j]), fa, fb[u])
                                           : P.fill;
                            }
                        }
                    }
                    // with the output's tensor map: the warp stages its 32 x 32
                    // chunk and one lane stores it (under sym, elements below
                    // the diagonal are rewritten by the mirror pass anyway).
                    // Else a lane writes 32 consecutive floats of its row:
                    // eight 16-byte streaming stores when the chunk is whole,
                    // aligned and (under sym) on or above the diagonal, else
                    // one by one.
                    if (tma_chunk) {
                        if (lane == 0) tma_store_wait_read();  // the previous chunk left stg
                        __syncwarp();
#pragma unroll
                        for (int j4 = 0; j4 < 8; ++j4)
                            *reinterpret_cast<float4*>(stg + lane * 128 + ((j4 ^ (lane & 7)) << 4)) =
                                make_float4(o[4 * j4], o[4 * j4 + 1], o[4 * j4 + 2], o[4 * j4 + 3]);
                        fence_proxy_async_smem();
                        __syncwarp();
                        if (lane == 0)
                            tma_store_2d(&out_map, smem_u32(stg), (int)gc0,
                                         (int)((int64_t)tm * kBM + quarter * 32));
                    } else if (vec_out && gc0 + 32 <= P.n_q && !(P.sym && gr > gc0)) {
#pragma unroll
                        for (int j4 = 0; j4 < 8; ++j4)
                            __stcs(reinterpret_cast<float4*>(orow + gc0) + j4,
                                   make_float4(o[4 * j4], o[4 * j4 + 1], o[4 * j4 + 2],
                                               o[4 * j4 + 3]));
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const int64_t gc = gc0 + j;
                            if (gc < P.n_q && !(P.sym && gr > gc)) __stcs(orow + gc, o[j]);
                        }
                    }
                }
                tmem_wait_ld(vn);
            }
            __syncwarp();
            tc_fence_before();
            mbar_arrive(&tempty[acc]);
            mbar_arrive(&pempty[acc]);
        }
        if (use_map && lane == 0) tma_store_wait_all();
        __syncwarp();
    }

    __syncthreads();
    if (*abort_flag && threadIdx.x == 0) atomicOr(err, 1u);
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols));
    }
}

}  // namespace umma

// Error bits of the tensor-core kernel (a pipeline wait that ran out of
// time); read and cleared by cms_fingerprint_take_error.
__device__ uint32_t g_fp_error;

template <int MEASURE>
int launch_umma(int grid, cudaStream_t s, const FpParams& P, const umma::Geometry& G,
                uint32_t* err, const CUtensorMap& out_map, int use_map, const CUtensorMap& in_r,
                const CUtensorMap& in_q, int use_in) {
    auto* k = umma::fp_umma_kernel<MEASURE>;
    if (const int rc = raise_func_smem(reinterpret_cast<const void*>(k), umma::kSmemBytes))
        return rc;
    k<<<grid, umma::kThreads, umma::kSmemBytes, s>>>(P, G, err, out_map, use_map, in_r, in_q,
                                                     use_in);
    return CMS_OK;
}

// cuTensorMapEncodeTiled from the driver (through the runtime, so that the
// library needs no link against libcuda); null when the driver lacks it
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    });
    return fn;
}

// Tensor map of the float output for the epilogue's 32 x 32 tensor stores:
// n_r rows, row pitch ld, and the first n_q rounded down to a multiple of four
// columns (a tensor store clips rows at the end, but columns only to whole 16
// bytes, so the last partial group is stored lane by lane).  False when the
// output does not meet the tensor-store rules (16-byte aligned base and
// pitch), is narrower than four columns, or the driver has no encoder; the
// epilogue then stores from registers.
bool output_tensor_map(float* out, int64_t n_r, int64_t n_q, int64_t ld, CUtensorMap& map) {
    std::memset(&map, 0, sizeof(map));
    const int64_t n_q4 = n_q & ~int64_t(3);
    if ((reinterpret_cast<uintptr_t>(out) & 15) || (ld & 3) || n_q4 == 0 ||
        n_q > (1LL << 31) || n_r > (1LL << 31))
        return false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)n_q4, (cuuint64_t)n_r};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
    const cuuint32_t box[2] = {32, 32};
    const cuuint32_t estr[2] = {1, 1};
    return enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, out, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
               CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

// Tensor map of packed fingerprints for the producers' ring: n_rows rows of
// n_words uint32 words, boxes of one K block (kBKWords words = 32 bytes) by
// box_rows rows, 32-byte swizzle.  False when the rows do not meet the tensor-load rules (16-byte
// aligned base, row pitch a multiple of 16 bytes) or the driver has no
// encoder; the producers then load the rows themselves.
bool input_tensor_map(const uint32_t* bits, int64_t n_rows, int n_words, int box_rows,
                      CUtensorMap& map) {
    std::memset(&map, 0, sizeof(map));
    if (!bits || (reinterpret_cast<uintptr_t>(bits) & 15) || n_words <= 0 || (n_words & 3) ||
        n_rows <= 0 || n_rows > (1LL << 31))
        return false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)n_words, (cuuint64_t)n_rows};
    const cuuint64_t strides[1] = {(cuuint64_t)n_words * 4};
    const cuuint32_t box[2] = {(cuuint32_t)umma::kBKWords, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<uint32_t*>(bits), dims, strides,
               box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
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
    // one set against itself (the same rows and flags): every measure is
    // symmetric in (I, a, b), so the full matrix is the mirrored one bit for
    // bit, and computing it costs less than half the tiles plus the mirror
    // pass's transposed copy of the lower triangle
    if (sym && ref_bits == q_bits && ref_valid == q_valid) sym = 0;
    FpParams P{ref_bits, ref_valid, n_ref, q_bits, q_valid, n_q, n_words, fill, out, ld, sym,
               test_stall("mma")};
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0, sms = 148;
    CMS_CUDA_TRY(cudaGetDevice(&dev));
    CMS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    umma::Geometry G;
    G.n_tm = (int)((n_ref + umma::kBM - 1) / umma::kBM);
    G.n_tn = (int)((n_q + umma::kBN - 1) / umma::kBN);
    G.n_tiles = (int64_t)G.n_tm * G.n_tn;
    G.kb = std::max(1, (n_words + umma::kBKWords - 1) / umma::kBKWords);
    uint32_t* err = nullptr;
    CMS_CUDA_TRY(cudaGetSymbolAddress(reinterpret_cast<void**>(&err), g_fp_error));
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(sms, G.n_tiles));
    CUtensorMap out_map;
    const int use_map = output_tensor_map(out, n_ref, n_q, ld, out_map) ? 1 : 0;
    CUtensorMap in_r, in_q;
    const int use_in = input_tensor_map(ref_bits, n_ref, n_words, umma::kBM, in_r) &&
                               input_tensor_map(q_bits, n_q, n_words, umma::kBN, in_q)
                           ? 1
                           : 0;
    int rc = CMS_OK;
    switch (measure) {
        case CMS_FP_JACCARD:
            rc = launch_umma<CMS_FP_JACCARD>(grid, s, P, G, err, out_map, use_map, in_r, in_q, use_in);
            break;
        case CMS_FP_DICE:
            rc = launch_umma<CMS_FP_DICE>(grid, s, P, G, err, out_map, use_map, in_r, in_q, use_in);
            break;
        default:
            rc = launch_umma<CMS_FP_COSINE>(grid, s, P, G, err, out_map, use_map, in_r, in_q, use_in);
            break;
    }
    if (rc) return rc;
    CMS_CUDA_TRY(cudaGetLastError());
    if (sym) return launch_mirror(DenseOut{out, nullptr, nullptr, ld}, n_ref, nullptr, sms, s);
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

namespace cms {
namespace {

// Exhaustive comparison of the epilogue's branch-free arithmetic with CUDA's
// IEEE operations (bit patterns), over the operands the measures can produce.
__global__ void arith_div_check(unsigned long long* bad) {  // n / d, 0 <= n <= d <= 65536
    const int d = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (d > 65536) return;
    const float fd = (float)d;
    unsigned long long b = 0;
    for (int n = 0; n <= d; ++n)
        b += __float_as_uint(div_fp((float)n, fd)) != __float_as_uint(__fdiv_rn((float)n, fd));
    if (b) atomicAdd(bad, b);
}
__global__ void arith_sqrt_check(unsigned long long* bad_sqrt, unsigned long long* bad_rcp) {
    const uint32_t lo = 0x3F800000u, hi = 0x4E800000u;  // every float in [1, 2^30]
    unsigned long long bs = 0, br = 0;
    for (uint32_t u = lo + blockIdx.x * blockDim.x + threadIdx.x; u <= hi;
         u += gridDim.x * blockDim.x) {
        const float p = __uint_as_float(u), root = __fsqrt_rn(p);
        bs += __float_as_uint(sqrt_fp(p)) != __float_as_uint(root);
        br += __float_as_uint(rcp_fp(root)) != __float_as_uint(__frcp_rn(root));
    }
    if (bs) atomicAdd(bad_sqrt, bs);
    if (br) atomicAdd(bad_rcp, br);
}
__device__ __forceinline__ unsigned long long cosine_mismatch(int i, int a, int b) {
    const float p = __fmul_rn((float)a, (float)b), fi = (float)i;
    return __float_as_uint(div_fp(fi, sqrt_fp(p))) != __float_as_uint(__fdiv_rn(fi, __fsqrt_rn(p)));
}
__global__ void arith_cos_check(unsigned long long* bad) {  // a, b <= 2048, every i <= min(a, b)
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2048 * 2048) return;
    const int a = t / 2048 + 1, b = t % 2048 + 1, m = a < b ? a : b;
    unsigned long long c = 0;
    for (int i = 0; i <= m; ++i) c += cosine_mismatch(i, a, b);
    if (c) atomicAdd(bad, c);
}
__global__ void arith_cos_sample(unsigned long long* bad, unsigned long long n) {
    // triples with a, b <= 32768 drawn by a counter-based generator (splitmix64)
    unsigned long long c = 0;
    for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < n;
         k += (unsigned long long)gridDim.x * blockDim.x) {
        unsigned long long z = (k + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const int a = (int)(z & 32767) + 1, b = (int)((z >> 15) & 32767) + 1;
        const int m = a < b ? a : b;
        c += cosine_mismatch((int)((z >> 30) % (unsigned long long)(m + 1)), a, b);
    }
    if (c) atomicAdd(bad, c);
}

}  // namespace
}  // namespace cms

extern "C" int cms_fingerprint_arith_check(uint64_t* mismatches, void* stream) {
    using namespace cms;
    if (!mismatches) {
        set_error("cms_fingerprint_arith_check: null argument");
        return CMS_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long* d = nullptr;
    CMS_CUDA_TRY(cudaMalloc(&d, 5 * sizeof(unsigned long long)));
    unsigned long long h[5] = {0, 0, 0, 0, 0};
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof(h), s);
    if (e == cudaSuccess) {
        arith_div_check<<<65536 / 256, 256, 0, s>>>(d);
        arith_sqrt_check<<<148 * 8, 256, 0, s>>>(d + 1, d + 2);
        arith_cos_check<<<2048 * 2048 / 256, 256, 0, s>>>(d + 3);
        arith_cos_sample<<<148 * 8, 256, 0, s>>>(d + 4, 1ull << 30);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d);
    CMS_CUDA_TRY(e);
    for (int i = 0; i < 5; ++i) mismatches[i] = h[i];
    return CMS_OK;
}

extern "C" int cms_fingerprint_take_error(uint32_t* bits, void* stream) {
    using namespace cms;
    if (!bits) {
        set_error("cms_fingerprint_take_error: null argument");
        return CMS_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t h = 0;
    const uint32_t zero = 0;
    CMS_CUDA_TRY(cudaMemcpyFromSymbolAsync(&h, g_fp_error, sizeof(h), 0, cudaMemcpyDeviceToHost, s));
    CMS_CUDA_TRY(cudaMemcpyToSymbolAsync(g_fp_error, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, s));
    CMS_CUDA_TRY(cudaStreamSynchronize(s));
    *bits = h;
    return CMS_OK;
}
