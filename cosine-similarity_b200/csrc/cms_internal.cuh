// Internal declarations shared by the CUDA translation units of
// libcudams_b200.so.  Public entry points live in include/cudams_b200.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstddef>
#include <utility>
#include <vector>

#include "../../include/cudams_b200.h"

namespace cms {

// Device error word bits (cms_take_device_error).
enum : uint32_t {
    kErrSpectrumTooLong = 1u << 0,  // a spectrum exceeds CMS_MAX_PEAKS peaks
    kErrSpillOverrun = 1u << 1,     // sparse spill list capacity exceeded
    kErrBadOffsets = 1u << 2,       // offsets not non-decreasing / out of range
    kErrPipelineTimeout = 1u << 3,  // a bounded hand-off wait between warps ran out
};

// One CSR spectrum set on the device (see the header comment of the public API).
struct SpecSet {
    const float* mz;
    const double* a;  // nullptr => 1.0
    const double* b;
    const int64_t* off;
    int64_t n;
    int64_t n_peaks;
    const double* prec = nullptr;  // precursor m/z per spectrum (modified cosine only)
};

struct CosineArgs {
    SpecSet ref;
    SpecSet qry;
    double tol;
    double shift;
    int match_limit;
    // modified cosine: candidates at shift 0 followed by those at the
    // precursor difference prec_ref - prec_query (ref.prec / qry.prec set)
    bool modified = false;
};

struct DenseOut {
    float* score;
    int32_t* matches;
    uint8_t* overflow;
    int64_t ld;
};

struct SparseOut {
    int32_t* r;
    int32_t* q;
    float* score;
    int32_t* matches;
    uint8_t* overflow;
    int64_t capacity;
    unsigned long long* count;  // int64 count, as an atomically updatable word
    float threshold;
    int mirror;                 // nonzero: every hit (r, q) with r != q also as (q, r)
};

// Symmetric dense output: copies element (c, r) to (r, c) for every r > c of
// the n x n matrix (score, and matches/overflow unless null), reading the
// upper triangle and writing the lower one.  `bad` (may be null) is a device
// flag that turns the kernel into a no-op.  Defined in mirror.cu.
int launch_mirror(const DenseOut& d, int64_t n, const uint32_t* bad, int sm_count,
                  cudaStream_t s);

// Thread-local last-error string.
void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);

// Growable device arena owned by a context (never shrinks until destroy).
struct Arena {
    void* ptr = nullptr;
    size_t bytes = 0;
};

}  // namespace cms

// A captured call: the key is every argument the launch sequence bakes in
// (pointers, sizes, parameters, stream, scratch arena), so a replay is valid
// exactly when a later call has the same key.
struct cms_graph_entry {
    std::vector<uint64_t> key;
    cudaGraphExec_t exec = nullptr;
    int64_t launches[CMS_PROFILE_STAGES] = {0, 0, 0, 0, 0};
};

struct cms_ctx {
    int device = 0;
    int sm_count = 0;
    size_t smem_optin = 0;
    cms::Arena scratch;       // per-call scratch (indices, lists, counters)
    uint32_t* err_word = nullptr;  // device, 1 word
    // profiling (cms_profile_*)
    bool profile = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> events;
    std::vector<cudaEvent_t> event_pool;
    int64_t launches[CMS_PROFILE_STAGES] = {0, 0, 0, 0, 0};
    // CUDA graphs (cms_graph_enable): most recently used first
    bool graphs = false;
    bool capturing = false;
    std::vector<cms_graph_entry> graph_cache;
    // graphs are captured on this stream (capture is not allowed on the legacy
    // default stream) and launched on the caller's
    cudaStream_t capture_stream = nullptr;
    // join-kernel work-item trace (cms_trace_enable); rec null: off
    unsigned long long* trace_rec = nullptr;
    unsigned long long* trace_count = nullptr;
    long long trace_cap = 0;
    unsigned int trace_tag = 0;
};

namespace cms {

// Ensure the arena holds at least `bytes`; returns CMS_OK or an error code.
// Growing the arena drops the context's captured graphs (they hold its address).
int arena_reserve(cms_ctx* ctx, Arena& a, size_t bytes, cudaStream_t s);

// Destroy every captured graph of the context.
void graph_cache_clear(cms_ctx* ctx);

// Bump allocator over an arena region (256-byte aligned slices).
struct Bump {
    char* base;
    size_t used;
    size_t cap;
    template <typename T>
    T* take(size_t count) {
        size_t off = (used + 255) & ~size_t(255);
        used = off + count * sizeof(T);
        return reinterpret_cast<T*>(base + off);
    }
};
inline size_t bump_size(size_t bytes) { return (bytes + 255) & ~size_t(255); }

bool check_specset(const SpecSet& s, const char* name);

// Raise a kernel's cudaFuncAttributeMaxDynamicSharedMemorySize on the current
// device to at least `bytes`, never lowering it.  The attribute is process
// wide, so a call that lowered it could make a concurrent call's launch (on
// another host thread, with a larger need) fail between its set and its
// launch; a monotone value under one mutex cannot.
int raise_func_smem(const void* func, size_t bytes);

// CMS_OK when `p` is device (or managed) memory that the current device can
// use in a kernel, else CMS_ERR_INVALID with a message naming `what`.
int check_device_ptr(const void* p, const char* who, const char* what);

// Test hook: nonzero when the environment variable CMS_TEST_STALL names
// `role` ("mma": the fingerprint kernel's MMA issuer, "pair": the pipelined
// pair kernel's greedy warp).  That role then does nothing, so the other
// roles' bounded waits run out and the kernel's error path is exercised.
int test_stall(const char* role);

// Scope that counts `n` launches for a profiling stage and, when profiling
// is on, records an event pair around them on stream `s`.
class StageScope {
  public:
    StageScope(cms_ctx* ctx, int stage, int n, cudaStream_t s);
    ~StageScope();

  private:
    cms_ctx* ctx_;
    int stage_;
    cudaStream_t s_;
    cudaEvent_t stop_ = nullptr;
};

}  // namespace cms

#define CMS_CUDA_TRY(expr)                                         \
    do {                                                           \
        cudaError_t _e = (expr);                                   \
        if (_e != cudaSuccess) return cms::cuda_fail(_e, #expr);   \
    } while (0)
