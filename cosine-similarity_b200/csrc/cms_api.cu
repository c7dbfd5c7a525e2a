// Context, errors and scratch management of libcudams_b200.so.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "cms_internal.cuh"

namespace cms {

static thread_local std::string g_last_error;

int test_stall(const char* role) {
    const char* v = std::getenv("CMS_TEST_STALL");
    return (v && role && std::strcmp(v, role) == 0) ? 1 : 0;
}

void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

int cuda_fail(cudaError_t e, const char* what) {
    set_error("CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), what);
    return e == cudaErrorMemoryAllocation ? CMS_ERR_NOMEM : CMS_ERR_CUDA;
}

void graph_cache_clear(cms_ctx* ctx) {
    for (auto& g : ctx->graph_cache)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    ctx->graph_cache.clear();
}

int arena_reserve(cms_ctx* ctx, Arena& a, size_t bytes, cudaStream_t s) {
    if (bytes <= a.bytes) return CMS_OK;
    // Growing: wait for work that may still use the old block, then replace it.
    if (a.ptr) {
        graph_cache_clear(ctx);
        CMS_CUDA_TRY(cudaStreamSynchronize(s));
        CMS_CUDA_TRY(cudaFree(a.ptr));
        a.ptr = nullptr;
        a.bytes = 0;
    }
    size_t want = bytes + bytes / 4;
    cudaError_t e = cudaMalloc(&a.ptr, want);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        e = cudaMalloc(&a.ptr, bytes);
        want = bytes;
    }
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        a.ptr = nullptr;
        set_error("device allocation of %zu bytes of scratch failed", bytes);
        return CMS_ERR_NOMEM;
    }
    a.bytes = want;
    (void)ctx;
    return CMS_OK;
}

bool check_specset(const SpecSet& s, const char* name) {
    if (s.n < 0 || s.n_peaks < 0) {
        set_error("%s: negative size", name);
        return false;
    }
    if (s.n > 0 && (!s.off || (s.n_peaks > 0 && (!s.mz || !s.b)))) {
        set_error("%s: null device pointer", name);
        return false;
    }
    if (s.n >= (int64_t(1) << 31) || s.n_peaks >= (int64_t(1) << 32)) {
        set_error("%s: too many spectra or peaks for this build", name);
        return false;
    }
    return true;
}

int raise_func_smem(const void* func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> set_to;
    int dev = 0;
    CMS_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = set_to[{dev, func}];
    if (bytes <= cur) return CMS_OK;
    CMS_CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)bytes));
    cur = bytes;
    return CMS_OK;
}

int check_device_ptr(const void* p, const char* who, const char* what) {
    cudaPointerAttributes at{};
    const cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        set_error("%s: %s is not a CUDA pointer (%s)", who, what, cudaGetErrorString(e));
        return CMS_ERR_INVALID;
    }
    if (at.type == cudaMemoryTypeManaged) return CMS_OK;
    int dev = 0;
    CMS_CUDA_TRY(cudaGetDevice(&dev));
    if (at.type != cudaMemoryTypeDevice || at.device != dev) {
        set_error("%s: %s must be device memory of the current device %d (memory type %d, "
                  "device %d)", who, what, dev, (int)at.type, at.device);
        return CMS_ERR_INVALID;
    }
    return CMS_OK;
}

static cudaEvent_t pool_event(cms_ctx* ctx) {
    if (!ctx->event_pool.empty()) {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
        (void)cudaGetLastError();
        return nullptr;
    }
    return e;
}

StageScope::StageScope(cms_ctx* ctx, int stage, int n, cudaStream_t s)
    : ctx_(ctx), stage_(stage), s_(s) {
    ctx->launches[stage] += n;
    if (!ctx->profile || ctx->capturing) return;
    cudaEvent_t start = pool_event(ctx);
    stop_ = pool_event(ctx);
    if (!start || !stop_) {
        stop_ = nullptr;
        return;
    }
    cudaEventRecord(start, s);
    ctx->events.push_back({stage, {start, stop_}});
}

StageScope::~StageScope() {
    if (stop_) cudaEventRecord(stop_, s_);
}

}  // namespace cms

extern "C" {

int cms_profile_enable(cms_ctx* ctx, int enable) {
    if (!ctx) {
        cms::set_error("cms_profile_enable: null context");
        return CMS_ERR_INVALID;
    }
    ctx->profile = enable != 0;
    return CMS_OK;
}

int cms_graph_enable(cms_ctx* ctx, int enable) {
    if (!ctx) {
        cms::set_error("cms_graph_enable: null context");
        return CMS_ERR_INVALID;
    }
    ctx->graphs = enable != 0;
    if (!ctx->graphs) {
        cudaSetDevice(ctx->device);
        cudaDeviceSynchronize();
        cms::graph_cache_clear(ctx);
    }
    return CMS_OK;
}

int cms_trace_enable(cms_ctx* ctx, uint64_t* records, int64_t capacity, uint64_t* count,
                     uint32_t tag) {
    if (!ctx || (records && (!count || capacity < 0))) {
        cms::set_error("cms_trace_enable: null context or invalid trace buffer");
        return CMS_ERR_INVALID;
    }
    ctx->trace_rec = reinterpret_cast<unsigned long long*>(records);
    ctx->trace_count = reinterpret_cast<unsigned long long*>(count);
    ctx->trace_cap = records ? capacity : 0;
    ctx->trace_tag = tag;
    return CMS_OK;
}

int cms_profile_read(cms_ctx* ctx, double* stage_ms, int64_t* stage_launches, int reset) {
    if (!ctx) {
        cms::set_error("cms_profile_read: null context");
        return CMS_ERR_INVALID;
    }
    double ms[CMS_PROFILE_STAGES] = {0, 0, 0, 0, 0};
    for (auto& ev : ctx->events) {
        CMS_CUDA_TRY(cudaEventSynchronize(ev.second.second));
        float t = 0.f;
        CMS_CUDA_TRY(cudaEventElapsedTime(&t, ev.second.first, ev.second.second));
        ms[ev.first] += t;
    }
    for (int i = 0; i < CMS_PROFILE_STAGES; ++i) {
        if (stage_ms) stage_ms[i] = ms[i];
        if (stage_launches) stage_launches[i] = ctx->launches[i];
    }
    if (reset) {
        for (auto& ev : ctx->events) {
            ctx->event_pool.push_back(ev.second.first);
            ctx->event_pool.push_back(ev.second.second);
        }
        ctx->events.clear();
        for (int i = 0; i < CMS_PROFILE_STAGES; ++i) ctx->launches[i] = 0;
    }
    return CMS_OK;
}


int cms_version(void) { return 100; }

const char* cms_last_error(void) { return cms::g_last_error.c_str(); }

int cms_create(cms_ctx** out, int device) {
    if (!out) {
        cms::set_error("cms_create: out is null");
        return CMS_ERR_INVALID;
    }
    *out = nullptr;
    int n = 0;
    CMS_CUDA_TRY(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) {
        cms::set_error("cms_create: device %d not present (%d devices)", device, n);
        return CMS_ERR_INVALID;
    }
    CMS_CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    CMS_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        cms::set_error("cms_create: device %d is sm_%d%d; this library is built for sm_100a only",
                       device, prop.major, prop.minor);
        return CMS_ERR_UNSUPPORTED;
    }
    cms_ctx* c = new cms_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    c->smem_optin = prop.sharedMemPerBlockOptin;
    cudaError_t e = cudaMalloc(&c->err_word, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(c->err_word, 0, sizeof(uint32_t));
    if (e != cudaSuccess) {
        cudaFree(c->err_word);
        delete c;
        return cms::cuda_fail(e, "cms_create: error word");
    }
    *out = c;
    return CMS_OK;
}

int cms_destroy(cms_ctx* ctx) {
    if (!ctx) return CMS_OK;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    cms::graph_cache_clear(ctx);
    if (ctx->capture_stream) cudaStreamDestroy(ctx->capture_stream);
    if (ctx->scratch.ptr) cudaFree(ctx->scratch.ptr);
    for (auto& ev : ctx->events) {
        cudaEventDestroy(ev.second.first);
        cudaEventDestroy(ev.second.second);
    }
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    if (ctx->err_word) cudaFree(ctx->err_word);
    delete ctx;
    return CMS_OK;
}

int cms_take_device_error(cms_ctx* ctx, uint32_t* bits, void* stream) {
    if (!ctx || !bits) {
        cms::set_error("cms_take_device_error: null argument");
        return CMS_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t h = 0;
    CMS_CUDA_TRY(cudaMemcpyAsync(&h, ctx->err_word, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    CMS_CUDA_TRY(cudaMemsetAsync(ctx->err_word, 0, sizeof(uint32_t), s));
    CMS_CUDA_TRY(cudaStreamSynchronize(s));
    *bits = h;
    return CMS_OK;
}

}  // extern "C"
