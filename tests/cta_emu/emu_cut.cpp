// CTA emulation of the plane cut (test infrastructure only): runs
// cut_cta (cuacd_b200/csrc/cut.cuh) for each plane of an input file with
// CUT_NT std::threads and the barrier-checking stand-in of cuda_runtime.h.
//
//   emu_cut input.bin [first_plane end_plane]
//   input.bin: int32 nv, nt, n_planes; float32 verts[3nv]; int32 tris[3nt];
//              float32 planes[4 n_planes]
// Prints one line per plane (error word, fragment sizes, cap triangles,
// loops, boundary and crossing counts); divergent barriers and other warp
// misuse go to stderr as "[emu] ..." lines.
#include "cuda_runtime.h"
#include "../../cuacd_b200/csrc/cut.cuh"

thread_local dim3 threadIdx;
dim3 blockIdx, blockDim, gridDim;
namespace emu {
int NT = CUT_NT;
std::barrier<>* cta_bar;
std::barrier<>* warp_bar[64];
int site[1024];
unsigned long long xch[1024];
std::atomic<int> live[64];
std::atomic<long long> clk{0};
static std::mutex report_mutex;
static int n_reports = 0;
void report(const char* what, int line)
{
    std::lock_guard<std::mutex> g(report_mutex);
    if (n_reports++ < 50) fprintf(stderr, "[emu] plane %u thread %u: %s at line %d\n", blockIdx.x, threadIdx.x, what, line);
}
}  // namespace emu

// Scratch one cut may carve (the device launcher's cut_scratch_bytes).
static size_t a256(size_t b) { return (b + 255) & ~(size_t)255; }
static size_t scratch_bytes(int nv, int nt)
{
    size_t occ = 1;
    while (occ < (size_t)2 * nt + 1) occ <<= 1;
    size_t b = 0;
    b += a256(nv) + a256(8 * occ) + 2 * a256(4 * occ) + a256(8 * occ) + 2 * a256(4 * occ);
    b += a256(12 * ((size_t)nv + occ)) + 2 * a256(4 * (size_t)nt);
    b += 2 * a256(12 * ((size_t)2 * nt + 8));
    b += 2 * a256(8 * (occ * 4));
    b += a256(4 * (4 * occ + 6 * (occ * 4 + 64)));
    b += 2 * a256(4 * ((size_t)nv + occ));
    b += 2 * (a256(12 * ((size_t)nv + occ)) + a256(12 * ((size_t)2 * nt + 8 + 4 * occ)));
    return b + 64 * 256;
}

int main(int argc, char** argv)
{
    if (argc < 2) { fprintf(stderr, "usage: emu_cut input.bin [first end]\n"); return 2; }
    FILE* f = fopen(argv[1], "rb");
    if (!f) { perror(argv[1]); return 2; }
    int hdr[3];
    if (fread(hdr, 4, 3, f) != 3) return 2;
    const int nv = hdr[0], nt = hdr[1], np = hdr[2];
    std::vector<float> v(3 * (size_t)nv), pl(4 * (size_t)np);
    std::vector<int> t(3 * (size_t)nt);
    if (fread(v.data(), 4, v.size(), f) != v.size() || fread(t.data(), 4, t.size(), f) != t.size() ||
        fread(pl.data(), 4, pl.size(), f) != pl.size()) return 2;
    fclose(f);
    const int p0 = argc > 2 ? atoi(argv[2]) : 0, p1 = argc > 3 ? atoi(argv[3]) : np;
    const size_t cap = scratch_bytes(nv, nt);
    std::vector<char> arena_mem;
    for (int i = p0; i < p1 && i < np; i++) {
        arena_mem.assign(cap + 4096, 0);
        Arena A{arena_mem.data(), cap, 0, 0, 0, 0};
        CutResult res;
        memset(&res, 0, sizeof(res));
        static CutShared sh;
        blockIdx.x = i; blockDim.x = CUT_NT; gridDim.x = np;
        emu::cta_bar = new std::barrier<>(CUT_NT);
        for (int w = 0; w < CUT_NT / 32; w++) { emu::warp_bar[w] = new std::barrier<>(32); emu::live[w] = 32; }
        std::vector<std::thread> th;
        for (int k = 0; k < CUT_NT; k++)
            th.emplace_back([&, k]() {
                threadIdx.x = k;
                CutFixedOut none;
                memset(&none, 0, sizeof(none));
                cut_cta(v.data(), nv, t.data(), nt, pl[4 * i], pl[4 * i + 1], pl[4 * i + 2], pl[4 * i + 3], &A, none,
                        &res, sh);
                emu::site[k] = -1;
                emu::live[k >> 5]--;
                emu::warp_bar[k >> 5]->arrive_and_drop();
                emu::cta_bar->arrive_and_drop();
            });
        for (auto& x : th) x.join();
        printf("plane %d: err %d npv %d npt %d nnv %d nnt %d cap %d loops %d nb %d cross %d failed %d\n", i, res.err,
               res.npv, res.npt, res.nnv, res.nnt, res.n_cap, res.n_loops, res.n_boundary, res.n_cross,
               res.cap_failed);
        fflush(stdout);
        delete emu::cta_bar;
        for (int w = 0; w < CUT_NT / 32; w++) delete emu::warp_bar[w];
    }
    return 0;
}
