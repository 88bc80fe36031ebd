// context.cuh — host-side context: device, stream, device pool, error text.
//
// The pool is one device buffer.  Each entry point carves its buffers from
// it front to back (host-side bump, reset at the start of every call), and
// the rest is handed to the device-side Arena for allocations whose sizes are
// only known inside a kernel (cut fragments).  With pool_bytes = 0 the pool
// grows on demand; the reference instead reserves a fixed share of free
// memory at init (csrc/heap.c:171-177).
#pragma once
#include <cstdio>
#include <cstring>
#include <cstdarg>
#include <cuda_runtime.h>
#include "common.cuh"
#include "../../include/cuacd_b200.h"

struct gpu_ctx {
    int            device;
    int            n_sm;               // streaming multiprocessors of the device
    cudaStream_t   stream;
    char*          pool;
    size_t         cap;
    int            fixed;
    size_t         carve;
    size_t         high_water;
    Arena*         d_arena;
    unsigned long long stats[6];
    unsigned long long launches;
    int            profile;            // record stage events in the evaluator
    cudaEvent_t    ev[8];              // stage boundaries of the last evaluation
    int            n_ev;
    int            eval_groups;        // plane groups evaluated concurrently (0: default)
    cudaStream_t   aux[3];             // streams of groups 1..3 (created on first use)
    cudaEvent_t    fork_ev, join_ev[3];
    cudaMemPool_t  parts_pool;         // stream-ordered allocations of search parts; keeps what it
                                       // reserved (release threshold: never), so a search does not
                                       // return memory to the driver at every synchronisation
    char           last_error[256];
};

static int ctx_fail(gpu_ctx* ctx, int code, const char* fmt, ...)
{
    if (ctx) {
        va_list ap; va_start(ap, fmt);
        vsnprintf(ctx->last_error, sizeof(ctx->last_error), fmt, ap);
        va_end(ap);
    }
    return code ? code : -1;
}

#define CK(call) do { cudaError_t _e = (call); if (_e != cudaSuccess) \
    return ctx_fail(ctx, (int)_e, "%s failed at %s:%d: %s", #call, __FILE__, __LINE__, cudaGetErrorString(_e)); } while (0)

static inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// Make sure the pool holds `bytes`; resets the host carve.
static int pool_begin(gpu_ctx* ctx, size_t bytes)
{
    ctx->carve = 0;
    bytes = al256(bytes);
    if (bytes <= ctx->cap) return 0;
    if (ctx->fixed)
        return ctx_fail(ctx, KERR_HEAP_OOM, "device pool too small: need %zu bytes, have %zu", bytes, ctx->cap);
    size_t ncap = ctx->cap * 2;
    if (ncap < bytes) ncap = bytes;
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->pool) CK(cudaFree(ctx->pool));
    ctx->pool = nullptr; ctx->cap = 0;
    CK(cudaMalloc(&ctx->pool, ncap));
    ctx->cap = ncap;
    return 0;
}

template <typename T>
static T* pool_take(gpu_ctx* ctx, size_t count)
{
    size_t b = al256(sizeof(T) * (count > 0 ? count : 1));
    if (ctx->carve + b > ctx->cap) return nullptr;
    T* p = (T*)(ctx->pool + ctx->carve);
    ctx->carve += b;
    if (ctx->carve > ctx->high_water) ctx->high_water = ctx->carve;
    ctx->stats[3] = ctx->carve;
    ctx->stats[4]++;
    return p;
}

// Hand the uncarved rest of the pool to the device arena.
static int arena_reset(gpu_ctx* ctx)
{
    Arena a;
    a.base = ctx->pool + ctx->carve;
    a.capacity = ctx->cap - ctx->carve;
    a.offset = 0;
    a.high_water = 0;
    a.n_allocs = 0;
    a.n_resets = 0;
    CK(cudaMemcpyAsync(ctx->d_arena, &a, sizeof(Arena), cudaMemcpyHostToDevice, ctx->stream));
    ctx->stats[5]++;
    return 0;
}

static int sync_and_check(gpu_ctx* ctx, const char* what)
{
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx_fail(ctx, (int)e, "%s: %s", what, cudaGetErrorString(e));
    e = cudaGetLastError();
    if (e != cudaSuccess) return ctx_fail(ctx, (int)e, "%s: %s", what, cudaGetErrorString(e));
    return 0;
}

// eval.cu: exact evaluation of the planes a selection keeps, the cut of
// every plane overlapping the caller's selection work on stream s.
struct EvalPrecut;
int eval_precut_begin(gpu_ctx* ctx, const float* d_v, int nv, const int* d_t, int nt, const float4* d_planes, int n,
                      EvalPrecut& P, cudaStream_t s);
int eval_precut_finish(gpu_ctx* ctx, EvalPrecut& P, const int* d_pos, int n_sel, int flags, float res, int mins,
                       int total, cuacd_cand_result* d_out, cudaStream_t s);
void eval_precut_release(EvalPrecut& P);      // frees the work set (finish does it too)
