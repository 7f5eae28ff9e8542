// ctx.cu -- context lifecycle, error reporting and buffer management.
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>

#include <atomic>

#include "pbt_internal.h"

namespace pbt {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
}
void clear_error() { g_last_error.clear(); }
const char *last_error() { return g_last_error.c_str(); }

// pending injected allocation failures (pbt_test_fail_next_alloc)
static std::atomic<int32_t> g_fail_allocs{0};

int DevBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return PBT_OK;
    release();
    size_t want = bytes < 256 ? 256 : bytes;
    int32_t pending = g_fail_allocs.load();
    while (pending > 0 && !g_fail_allocs.compare_exchange_weak(pending, pending - 1)) {
    }
    if (pending > 0) {
        set_error("cudaMalloc(%zu) failed: out of memory (injected by pbt_test_fail_next_alloc)", want);
        return PBT_ENOMEM;
    }
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        cap = 0;
        (void)cudaGetLastError();
        set_error("cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
        return PBT_ENOMEM;
    }
    cap = want;
    return PBT_OK;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

int HostBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return PBT_OK;
    release();
    size_t want = bytes < 4096 ? 4096 : bytes;
    cudaError_t e = cudaMallocHost(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        cap = 0;
        (void)cudaGetLastError();
        set_error("cudaMallocHost(%zu) failed: %s", want, cudaGetErrorString(e));
        return PBT_ENOMEM;
    }
    cap = want;
    return PBT_OK;
}
void HostBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
}

void timing_begin(pbt_ctx *ctx, cudaStream_t st) {
    if (!ctx->timing || ctx->capturing) return;
    if (ctx->ev_used + 2 > ctx->ev.size()) {
        for (int i = 0; i < 2; i++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) {
                (void)cudaGetLastError();
                return;
            }
            ctx->ev.push_back(e);
        }
    }
    cudaEventRecord(ctx->ev[ctx->ev_used], st);
}

void timing_end(pbt_ctx *ctx, cudaStream_t st) {
    if (!ctx->timing || ctx->capturing || ctx->ev_used + 2 > ctx->ev.size()) return;
    cudaEventRecord(ctx->ev[ctx->ev_used + 1], st);
    ctx->ev_used += 2;
}

}  // namespace pbt

using namespace pbt;

extern "C" int pbt_set_kernel_timing(pbt_ctx *ctx, int32_t enable) {
    clear_error();
    if (!ctx) {
        set_error("context is NULL");
        return PBT_EINVAL;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->timing = enable != 0;
    ctx->ev_used = 0;
    return PBT_OK;
}

extern "C" int pbt_set_plan(pbt_ctx *ctx, int32_t variant, int32_t bins_per_thread,
                            int64_t records_per_item) {
    clear_error();
    if (!ctx) {
        set_error("context is NULL");
        return PBT_EINVAL;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (variant < 0) {
        ctx->plan_variant = -1;
        return PBT_OK;
    }
    if (variant > 1 || (bins_per_thread != 1 && bins_per_thread != 2) || records_per_item < 32 ||
        records_per_item > (1 << 22)) {
        set_error("bad plan (variant %d, bins_per_thread %d, records_per_item %lld)", variant,
                  bins_per_thread, (long long)records_per_item);
        return PBT_EINVAL;
    }
    ctx->plan_variant = variant;
    ctx->plan_bpt = bins_per_thread;
    ctx->plan_rpi = records_per_item;
    return PBT_OK;
}

extern "C" int pbt_kernel_time_ms(pbt_ctx *ctx, double *total_ms, int64_t *nlaunch) {
    clear_error();
    if (!ctx || !total_ms || !nlaunch) {
        set_error("NULL argument");
        return PBT_EINVAL;
    }
    DeviceRestore dev_restore;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    double t = 0.0;
    for (size_t i = 0; i + 1 < ctx->ev_used; i += 2) {
        PBT_CUDA_TRY(cudaEventSynchronize(ctx->ev[i + 1]));
        float ms = 0.f;
        PBT_CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev[i], ctx->ev[i + 1]));
        t += ms;
    }
    *total_ms = t;
    *nlaunch = (int64_t)(ctx->ev_used / 2);
    ctx->ev_used = 0;
    return PBT_OK;
}

extern "C" int pbt_version(void) { return 10000; }

extern "C" const char *pbt_last_error_string(void) { return last_error(); }

// The node-local rank that an MPI or torchrun launcher exports (the first of
// these variables set to a non-negative integer), or 0.
static int local_rank_from_env() {
    static const char *const vars[] = {"LOCAL_RANK",      "OMPI_COMM_WORLD_LOCAL_RANK",
                                       "MV2_COMM_WORLD_LOCAL_RANK", "MPI_LOCALRANKID",
                                       "SLURM_LOCALID",   "PMI_LOCAL_RANK"};
    for (const char *v : vars) {
        const char *s = getenv(v);
        if (!s || !*s) continue;
        char *end = nullptr;
        const long r = strtol(s, &end, 10);
        if (*end == '\0' && r >= 0 && r <= 1000000) return (int)r;
    }
    return 0;
}

extern "C" int pbt_ctx_create(int device, pbt_ctx **out) {
    clear_error();
    if (!out) {
        set_error("out must not be NULL");
        return PBT_EINVAL;
    }
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        set_error("no CUDA device: %s", e != cudaSuccess ? cudaGetErrorString(e) : "count is 0");
        return PBT_ENODEV;
    }
    if (device == PBT_DEVICE_LOCAL_RANK) device = local_rank_from_env() % ndev;
    if (device < 0 || device >= ndev) {
        set_error("device %d out of range (have %d)", device, ndev);
        return PBT_EINVAL;
    }
    cudaDeviceProp prop;
    PBT_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        set_error("device %d is sm_%d%d; this library is built for sm_100a", device, prop.major,
                  prop.minor);
        return PBT_ENODEV;
    }
    DeviceRestore dev_restore;
    PBT_CUDA_TRY(cudaSetDevice(device));
    pbt_ctx *c = new pbt_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        set_error("cudaStreamCreate failed: %s", cudaGetErrorString(e));
        return PBT_ECUDA;
    }
    *out = c;
    return PBT_OK;
}

extern "C" int pbt_ctx_device(const pbt_ctx *ctx, int *device) {
    clear_error();
    if (!ctx || !device) {
        set_error("ctx and device must not be NULL");
        return PBT_EINVAL;
    }
    *device = ctx->device;
    return PBT_OK;
}

extern "C" int pbt_ctx_destroy(pbt_ctx *ctx) {
    clear_error();
    if (!ctx) return PBT_OK;
    {
        DeviceRestore dev_restore;
        std::lock_guard<std::mutex> lk(ctx->mu);
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        DevBuf *bufs[] = {&ctx->d_fac, &ctx->d_edge, &ctx->d_out,  &ctx->d_mu,
                          &ctx->d_m1,  &ctx->d_misc, &ctx->d_in,   &ctx->d_rec,
                          &ctx->d_ws,  &ctx->d_scan, &ctx->d_items, &ctx->d_tk, &ctx->d_k1part, &ctx->grid.xyz,
                          &ctx->grid.phitab,
                          &ctx->grid.thtab, &ctx->grid.wbin, &ctx->grid.wphi,
                          &ctx->grid.fast_perm, &ctx->grid.fast_cone};
        for (DevBuf *b : bufs) b->release();
        ctx->tot.release();
        ctx->btot.release();
        ctx->h_stage.release();
        for (cudaEvent_t e : ctx->ev) cudaEventDestroy(e);
        if (ctx->stage_ev) cudaEventDestroy(ctx->stage_ev);
        for (int i = 0; i < 2; i++) {
            if (ctx->up_ev[i]) cudaEventDestroy(ctx->up_ev[i]);
            if (ctx->done_ev[i]) cudaEventDestroy(ctx->done_ev[i]);
        }
        if (ctx->copy_stream) {
            cudaStreamSynchronize(ctx->copy_stream);
            cudaStreamDestroy(ctx->copy_stream);
        }
        cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return PBT_OK;
}

extern "C" int64_t pbt_last_launch_count(pbt_ctx *ctx) { return ctx ? ctx->launches : -1; }

extern "C" int pbt_test_fail_next_alloc(int32_t count) {
    return pbt::g_fail_allocs.exchange(count > 0 ? count : 0);
}
