// hull_kernels.cuh — bodies of the batched hull pipeline's kernels
// (set-up, wrap-grid shares, persistent wrapping, output).  hull.cu wraps
// each in its __global__ kernel; keeping the bodies here lets the CTA
// emulator of the tests run the same code on the CPU.
#pragma once
#include "hull.cuh"

// retry_round 0: every cloud, first-attempt capacities (hull_first_cap);
// retry_round 1: only the clouds whose tables overflowed, at h = n.
static __device__ void hull_setup_body(const HullJob* __restrict__ jobs, int n_jobs, Arena* scratch, HullState* states, int* ctl,
                                       int seed_min_n = 1 << 30, int retry_round = 0, int reduce_max_n = 1 << 30)
{
    __shared__ HullSetupShared sh;
    __shared__ char* s_scr;
    __shared__ int s_err;
    const int j = blockIdx.x;
    if (j >= n_jobs) return;
    const HullJob J = jobs[j];
    HullState* S = &states[j];
    if (retry_round && !S->retry) {              // built on the first attempt: nothing to do
        if (threadIdx.x == 0) S->active = 0;
        return;
    }
    const int hcap = retry_round ? J.n : hull_first_cap(J.n, reduce_max_n);
    double mv = 0.0;
    if (J.tris && J.nt > 0 && J.n > 0) mv = block_mesh_signed_volume(J.pts, J.n, J.tris, J.nt, sh.dsh);
    if (threadIdx.x == 0) {
        S->n = J.n; S->n_faces = 0; S->err = 0; S->active = 0; S->q_pending = 0; S->hcap = hcap;
        if (!retry_round) S->retry = 0;
        for (int k = 0; k < 8; k++) { S->stats[k] = 0; S->fail[k] = 0; }
        s_err = 0; s_scr = nullptr;
        if (J.n >= 4) {
            s_scr = (char*)arena_alloc(scratch, hull_attempt_bytes(J.n, hcap), &s_err);
            if (!s_scr) S->err = s_err | KERR_BT_POOL_EXHAUST;
        }
    }
    __syncthreads();
    if (s_scr) hull_setup_cta(J.pts, J.n, s_scr, S, sh, seed_min_n, hcap);
    if (threadIdx.x == 0) {
        S->mesh_vol = fabs(mv);
        if (s_scr && S->active) atomicAdd(&ctl[0], 1);
    }
}
static __device__ void hull_assign_body(HullState* states, int n_jobs, int n_ctas, long long* total)
{
    __shared__ long long part[1024 / 32];
    __shared__ long long carry, s_sum, s_floor;
    __shared__ int s_h;
    if (threadIdx.x == 0) { carry = 0; s_sum = 0; s_h = 0; }
    __syncthreads();
    {
        long long sn = 0; int h = 0;
        for (int j = threadIdx.x; j < n_jobs; j += 1024)
            if (states[j].active) { sn += states[j].n; h++; }
        atomicAdd((unsigned long long*)&s_sum, (unsigned long long)sn);
        atomicAdd(&s_h, h);
    }
    __syncthreads();
    if (threadIdx.x == 0) s_floor = n_ctas > s_h ? (s_sum + (n_ctas - s_h) - 1) / (n_ctas - s_h) : 0;
    __syncthreads();
    const long long floor_w = s_floor;
    for (int base = 0; base < n_jobs; base += 1024) {
        const int j = base + threadIdx.x;
        long long w = (j < n_jobs && states[j].active) ? (long long)states[j].n + floor_w : 0;
        long long x = w;                                  // inclusive warp scan
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(FULL_MASK, x, o);
            if ((threadIdx.x & 31) >= o) x += y;
        }
        if ((threadIdx.x & 31) == 31) part[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            long long p = part[threadIdx.x], q = p;
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                long long y = __shfl_up_sync(FULL_MASK, q, o);
                if (threadIdx.x >= o) q += y;
            }
            part[threadIdx.x] = q - p;                    // exclusive over warps
        }
        __syncthreads();
        if (j < n_jobs) states[j].wbase = carry + part[threadIdx.x >> 5] + x - w;
        __syncthreads();
        if (threadIdx.x == 1023) carry += part[31] + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}
static __device__ void hull_wrap_body(HullState* states, int n_jobs, int* ctl, const long long* total, int* wbuf, int* wsm_dyn)
{
    __shared__ HullWrapShared sh;
    __shared__ int s_h0[HULL_NT / 32], s_go;
    // one reader decides for the whole CTA: other CTAs may finish the last
    // hull while this one starts
    if (threadIdx.x == 0) s_go = *(volatile int*)&ctl[0] > 0;
    // Home hull of each warp: the active hull whose share holds the warp's
    // point.  With at most one hull per CTA the point is the CTA's (all its
    // warps wrap one hull, whose BVH stays in that SM's L1); with more hulls
    // than CTAs it is the warp's own, so many small clouds start at once
    // instead of queueing behind one home hull per CTA.
    if (threadIdx.x < HULL_NT / 32) {
        const long long W = *total;
        const bool per_warp = n_jobs > (int)gridDim.x;
        const long long pos = per_warp ? 2LL * ((long long)blockIdx.x * (HULL_NT / 32) + threadIdx.x) + 1
                                       : 2LL * blockIdx.x + 1;
        const long long den = per_warp ? 2LL * gridDim.x * (HULL_NT / 32) : 2LL * gridDim.x;
        const long long t = (pos * W) / den;
        int lo = 0, hi = n_jobs - 1;
        while (lo < hi) {                                 // last j with wbase[j] <= t
            int mid = (lo + hi + 1) >> 1;
            if (states[mid].wbase <= t) lo = mid; else hi = mid - 1;
        }
        s_h0[threadIdx.x] = lo;
    }
    __syncthreads();
    if (!s_go) return;
    hull_wrap_grid(states, n_jobs, s_h0[threadIdx.x >> 5], ctl, wbuf, sh, wsm_dyn);
}
static __device__ void hull_output_body(const HullJob* __restrict__ jobs, HullState* states, int n_jobs, Arena* out, const int* ctl,
              HullRes* res, unsigned long long* stats, int retry_round = 0)
{
    __shared__ HullOutShared sh;
    __shared__ float* s_ov;
    __shared__ int* s_ot;
    __shared__ int s_mhv, s_mht, s_aerr, s_nv, s_nt, s_oerr, s_skip;
    __shared__ float s_vol;
    const int j = blockIdx.x;
    if (j >= n_jobs) return;
    const HullJob J = jobs[j];
    HullState* S = &states[j];
    if (threadIdx.x == 0) {
        if (J.n >= 4 && S->active) atomicOr(&S->err, ctl[1] ? ctl[1] : KERR_TIMEOUT);   // not finished
        // a first attempt whose tables overflowed (and not for want of
        // arena memory) is built again at full capacity: no output yet
        const int e = S->err;
        s_skip = retry_round ? !S->retry : 0;
        if (!retry_round && J.n >= 4 && S->hcap < J.n && (e & KERR_BT_POOL_EXHAUST) && !(e & KERR_HEAP_OOM)) {
            S->retry = 1;
            s_skip = 1;
        }
        if (retry_round) S->retry = 0;
    }
    __syncthreads();
    if (s_skip) return;
    if (threadIdx.x == 0) {
        s_aerr = 0;
        s_ov = J.out_v; s_ot = J.out_t; s_mhv = J.max_hv; s_mht = J.max_ht;
        if (!J.out_v && J.n >= 4 && S->err == 0) {
            s_ov = (float*)arena_alloc(out, 12ull * J.n, &s_aerr);
            s_ot = (int*)arena_alloc(out, 12ull * (2 * J.n + 4), &s_aerr);
            s_mhv = J.n; s_mht = 2 * J.n + 4;
        }
        s_nv = 0; s_nt = 0; s_vol = 0.f; s_oerr = 0;
    }
    __syncthreads();
    if (s_aerr) {
        if (threadIdx.x == 0) { HullRes r; memset(&r, 0, sizeof(r)); r.mesh_vol = S->mesh_vol; r.err = s_aerr; res[j] = r; }
        return;
    }
    hull_output_cta(J.pts, S, s_ov, s_ot, s_mhv, s_mht, &s_nv, &s_nt, &s_vol, &s_oerr, sh);
    __syncthreads();
    if (threadIdx.x == 0) {
        HullRes r;
        r.hv = s_nv > 0 ? s_ov : nullptr; r.ht = s_nt > 0 ? s_ot : nullptr;
        r.hnv = s_nv; r.hnt = s_nt;
        r.mesh_vol = S->mesh_vol; r.hull_vol = s_vol;
        r.err = s_oerr | S->err;
        res[j] = r;
    }
    if (stats && threadIdx.x < 8) {
        unsigned long long x = threadIdx.x == 2 ? (unsigned long long)S->n_faces : S->stats[threadIdx.x];
        if (S->fail[0] && threadIdx.x >= 4) {       // failed hull: slots 4-7 hold the failure record
            const int k = 2 * ((int)threadIdx.x - 4);
            x = (unsigned long long)(unsigned)S->fail[k] | ((unsigned long long)(unsigned)S->fail[k + 1] << 32);
        }
        stats[8 * (size_t)j + threadIdx.x] = x;
    }
}