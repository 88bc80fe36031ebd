// CTA emulation of the batched hull pipeline (test infrastructure only):
// k_hull_setup (one CTA per cloud), k_hull_assign, k_hull_wrap (ONE
// persistent CTA wraps every cloud) and k_hull_output, each CTA run by
// std::threads with the barrier-checking stand-in of cuda_runtime.h.  The
// bodies are the device code of cuacd_b200/csrc/hull_kernels.cuh.
//
//   emu_hull input.bin
//   input.bin: int32 n_clouds, int32 sizes[n_clouds], float32 xyz of every
//              cloud in order
// Prints per cloud: error word, hull vertex and triangle counts, volume, then
// the hull's vertex coordinates (one line) and triangles (one line).
// Divergent barriers and other warp misuse go to stderr as "[emu] ..." lines.
#include "cuda_runtime.h"
inline void __nanosleep(unsigned) { std::this_thread::yield(); }
#include "../../cuacd_b200/csrc/hull_kernels.cuh"

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
void report(const char* what, int line)
{
    std::lock_guard<std::mutex> g(report_mutex);
    if (n_reports++ < 50)
        fprintf(stderr, "[emu] %s block %u thread %u: %s at line %d\n", stage, blockIdx.x, threadIdx.x, what, line);
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
    if (argc < 2) { fprintf(stderr, "usage: emu_hull input.bin\n"); return 2; }
    FILE* f = fopen(argv[1], "rb");
    if (!f) { perror(argv[1]); return 2; }
    int n_jobs = 0;
    if (fread(&n_jobs, 4, 1, f) != 1) return 2;
    std::vector<int> sizes(n_jobs);
    if (fread(sizes.data(), 4, n_jobs, f) != (size_t)n_jobs) return 2;
    std::vector<std::vector<float>> pts(n_jobs);
    for (int j = 0; j < n_jobs; j++) {
        pts[j].resize(3 * (size_t)sizes[j]);
        if (fread(pts[j].data(), 4, pts[j].size(), f) != pts[j].size()) return 2;
    }
    fclose(f);
    // arenas: scratch for the set-up, outputs for the output CTAs
    size_t scap = 0, ocap = 0;
    for (int j = 0; j < n_jobs; j++) {
        scap += ((hull_scratch_bytes(sizes[j]) + 255) & ~(size_t)255) + 256;
        ocap += 12 * (size_t)sizes[j] + 12 * (2 * (size_t)sizes[j] + 4) + 1024;
    }
    std::vector<char> smem(scap + 4096), omem(ocap + 4096);
    Arena scratch{smem.data(), scap, 0, 0, 0, 0}, out{omem.data(), ocap, 0, 0, 0, 0};
    std::vector<HullJob> jobs(n_jobs);
    for (int j = 0; j < n_jobs; j++) {
        memset(&jobs[j], 0, sizeof(HullJob));
        jobs[j].pts = pts[j].data(); jobs[j].n = sizes[j];
    }
    std::vector<HullState> states(n_jobs);
    memset(states.data(), 0, sizeof(HullState) * n_jobs);
    std::vector<HullRes> res(n_jobs);
    std::vector<int> wbuf((HULL_NT / 32) * 2 * HULL_SGCAP);
    std::vector<int> wsm(HULL_WRAP_DSMEM / sizeof(int));
    // the launcher's two rounds: first-attempt tables, then full-size tables
    // for the clouds whose tables overflowed
    for (int round = 0; round < 2; round++) {
        int ctl[4] = {0, 0, 0, 0};
        long long total = 0;
        for (int j = 0; j < n_jobs; j++)
            run_cta("setup", HULL_NT, j, n_jobs,
                    [&]() { hull_setup_body(jobs.data(), n_jobs, &scratch, states.data(), ctl, 1 << 30, round); });
        run_cta("assign", 1024, 0, 1, [&]() { hull_assign_body(states.data(), n_jobs, 1, &total); });
        run_cta("wrap", HULL_NT, 0, 1,
                [&]() { hull_wrap_body(states.data(), n_jobs, ctl, &total, wbuf.data(), wsm.data()); });
        for (int j = 0; j < n_jobs; j++)
            run_cta("output", HULL_NT, j, n_jobs,
                    [&]() { hull_output_body(jobs.data(), states.data(), n_jobs, &out, ctl, res.data(), nullptr, round); });
    }
    for (int j = 0; j < n_jobs; j++) {
        const HullRes& r = res[j];
        printf("hull %d: err %d nv %d nt %d vol %.9g\n", j, r.err, r.hnv, r.hnt, (double)r.hull_vol);
        for (int i = 0; i < 3 * r.hnv; i++) printf("%.9g ", (double)r.hv[i]);
        printf("\n");
        for (int i = 0; i < 3 * r.hnt; i++) printf("%d ", r.ht[i]);
        printf("\n");
    }
    return 0;
}
