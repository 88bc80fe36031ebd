// CTA emulation of the batched Hausdorff distance (test infrastructure
// only): hd_prep_cta (one CTA per surface) and hd_query_body (ONE CTA takes
// every chunk of both directions) from cuacd_b200/csrc/hausdorff.cuh, each
// CTA run by std::threads with the barrier-checking stand-in of
// cuda_runtime.h, the query planned as the library's k_hd_plan plans it.
//
//   emu_hd input.bin
//   input.bin: int32 nv_a, nt_a, nv_b, nt_b, min_samples, total;
//              float32 resolution; float32 verts_a[3nv_a]; int32 tris_a[3nt_a];
//              float32 verts_b[3nv_b]; int32 tris_b[3nt_b]
// Prints the distance (max of both directions) and the sample counts.
// Divergent barriers and warp votes go to stderr as "[emu] ..." lines.
#include <cmath>
#include <unistd.h>
#include "cuda_runtime.h"
struct float3 { float x, y, z; };
inline float3 make_float3(float a, float b, float c) { return {a, b, c}; }
template <class T> T __ldg(const T* p) { return *p; }
inline float __fsqrt_rn(float x) { return std::sqrt(x); }
inline long long __double2ll_rn(double x) { return std::llrint(x); }
#include "../../cuacd_b200/csrc/hausdorff.cuh"

thread_local dim3 threadIdx;
dim3 blockIdx, blockDim, gridDim;
namespace emu {
int NT = 0;
std::barrier<>* cta_bar;
std::barrier<>* warp_bar[64];
int site[1024];
unsigned long long xch[1024];
std::atomic<int> live[64];
std::atomic<long long> clk{0};
static std::mutex report_mutex;
static int n_reports = 0;
static const char* stage = "";
// A divergent vote would leave the query's loops out of step (on the GPU the
// warp hangs), so the first report ends the run.
void report(const char* what, int line)
{
    std::lock_guard<std::mutex> g(report_mutex);
    if (n_reports++ < 50)
        fprintf(stderr, "[emu] %s block %u thread %u: %s at line %d\n", stage, blockIdx.x, threadIdx.x, what, line);
    fflush(stderr);
    _exit(3);
}
}  // namespace emu

// Run `body` as CTA `block` of `grid` CTAs of nt threads.
template <class F> static void run_cta(const char* stage, int nt, int block, int grid, F body)
{
    emu::stage = stage;
    emu::NT = nt;
    blockIdx.x = block; blockDim.x = nt; gridDim.x = grid;
    emu::cta_bar = new std::barrier<>(nt);
    for (int w = 0; w < nt / 32; w++) { emu::warp_bar[w] = new std::barrier<>(32); emu::live[w] = 32; }
    std::vector<std::thread> th;
    for (int k = 0; k < nt; k++)
        th.emplace_back([&, k]() {
            threadIdx.x = k;
            body();
            emu::site[k] = -1;
            emu::live[k >> 5]--;
            emu::warp_bar[k >> 5]->arrive_and_drop();
            emu::cta_bar->arrive_and_drop();
        });
    for (auto& x : th) x.join();
    delete emu::cta_bar;
    for (int w = 0; w < nt / 32; w++) delete emu::warp_bar[w];
}

int main(int argc, char** argv)
{
    if (argc < 2) { fprintf(stderr, "usage: emu_hd input.bin\n"); return 2; }
    FILE* f = fopen(argv[1], "rb");
    if (!f) { perror(argv[1]); return 2; }
    int hdr[6];
    float resolution;
    if (fread(hdr, 4, 6, f) != 6 || fread(&resolution, 4, 1, f) != 1) return 2;
    const int nv[2] = {hdr[0], hdr[2]}, nt[2] = {hdr[1], hdr[3]};
    const int min_samples = hdr[4], total = hdr[5];
    std::vector<float> v[2];
    std::vector<int> t[2];
    for (int s = 0; s < 2; s++) {
        v[s].resize(3 * (size_t)nv[s]); t[s].resize(3 * (size_t)nt[s]);
        if (fread(v[s].data(), 4, v[s].size(), f) != v[s].size() || fread(t[s].data(), 4, t[s].size(), f) != t[s].size())
            return 2;
    }
    fclose(f);
    HDSurf surfs[2];
    HDPrep preps[2];
    std::vector<char*> scratch;
    for (int s = 0; s < 2; s++) {
        surfs[s] = {v[s].data(), t[s].data(), nv[s], nt[s]};
        char* scr = (char*)aligned_alloc(256, (hd_prep_bytes(nt[s]) + 255) & ~(size_t)255);
        memset(scr, 0, hd_prep_bytes(nt[s]));
        scratch.push_back(scr);
        run_cta("prep", HD_PREP_NT, s, 2, [&]() {
            __shared__ HDShared sh;
            hd_prep_cta(surfs[s], scr, resolution, min_samples, total, &preps[s], sh);
        });
    }
    // the library's plan for one pair: direction 0 samples A against B, 1 B against A
    HDDir dirs[2];
    int chunks = 0;
    const bool has = nt[0] > 0 && nt[1] > 0 && preps[0].n_samples > 0 && preps[1].n_samples > 0;
    for (int d = 0; d < 2; d++) {
        dirs[d].src = d; dirs[d].dst = 1 - d; dirs[d].pair = 0;
        dirs[d].n_samples = has ? preps[d].n_samples : 0;
        dirs[d].chunk0 = chunks;
        chunks += (dirs[d].n_samples + HD_CHUNK - 1) / HD_CHUNK;
    }
    int counter = 0;
    float pmax = 0.f;
    run_cta("query", HD_NT, 0, 1, [&]() { hd_query_body(surfs, preps, dirs, 2, &chunks, &counter, &pmax); });
    printf("%.9g %d %d\n", std::sqrt((double)pmax), preps[0].n_samples, preps[1].n_samples);
    for (char* p : scratch) free(p);
    return 0;
}
