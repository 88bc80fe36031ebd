// Host run of the remesh's device code (cuacd_b200/csrc/remesh.cuh): the
// same per-item functions that remesh.cu's kernels call, in the kernels'
// index order, with atomicMin as a plain minimum and the scans serial.
// Input (binary): int R, nv, nt; float verts[3 nv]; int tris[3 nt].
// Output (binary, stdout): int nv_out, nt_out; float verts; int tris.
// Build with -ffp-contract=off so every FP64 expression rounds as written.
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <vector>
#include "../../cuacd_b200/csrc/remesh.cuh"

static uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

static long long scan(std::vector<int>& a)
{
    long long s = 0;
    for (auto& x : a) { const int v = x; x = (int)s; s += v; }
    return s;
}

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int hdr[3];
    if (std::fread(hdr, 4, 3, f) != 3) return 2;
    const int R = hdr[0], nv = hdr[1], nt = hdr[2];
    std::vector<float> V(3 * (size_t)nv);
    std::vector<int> T(3 * (size_t)nt);
    if (std::fread(V.data(), 4, V.size(), f) != V.size() || std::fread(T.data(), 4, T.size(), f) != T.size()) return 2;
    std::fclose(f);

    RmTable tab;
    rm_build_table(tab);
    RmParams P;
    float vmax[3];
    for (int k = 0; k < 3; k++) { P.vmin[k] = V[k]; vmax[k] = V[k]; }
    for (int i = 1; i < nv; i++)
        for (int k = 0; k < 3; k++) {
            const float p = V[3 * i + k];
            if (p < P.vmin[k]) P.vmin[k] = p;
            if (p > vmax[k]) vmax[k] = p;
        }
    float extent = -1.0f;
    for (int k = 0; k < 3; k++)
        if (vmax[k] - P.vmin[k] > extent) extent = vmax[k] - P.vmin[k];
    P.R = R; P.extent = extent; P.band = 3.0 / R; P.margin = 1.0 + 2.0 * P.band;

    const long long N = (long long)R * R * R;
    std::vector<double> u(3 * (size_t)nv);
    for (long long i = 0; i < 3ll * nv; i++) u[i] = rm_norm(V[i], (int)(i % 3), P);     // k_rm_norm
    std::vector<uint32_t> d2(N, RM_FAR);                                                 // k_rm_init
    std::vector<unsigned char> outside(N), blk(3 * N, 0);
    for (long long n = 0; n < N; n++) {
        const int x = (int)(n % R), y = (int)(n / R % R), z = (int)(n / ((long long)R * R));
        outside[n] = (x == 0 || y == 0 || z == 0 || x == R - 1 || y == R - 1 || z == R - 1) ? 1 : 0;
    }
    for (int t = 0; t < nt; t++) {                                                       // k_rm_tris
        double a[3], b[3], c[3];
        for (int k = 0; k < 3; k++) {
            a[k] = u[3ll * T[3 * t] + k]; b[k] = u[3ll * T[3 * t + 1] + k]; c[k] = u[3ll * T[3 * t + 2] + k];
        }
        int lo[3], hi[3];
        rm_tri_box(a, b, c, R, lo, hi);
        if (hi[0] >= lo[0] && hi[1] >= lo[1] && hi[2] >= lo[2]) {
            const long long nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
            for (long long q = 0; q < nx * ny * nz; q++) {
                const int x = lo[0] + (int)(q % nx), y = lo[1] + (int)(q / nx % ny), z = lo[2] + (int)(q / (nx * ny));
                const double p[3] = {(double)x, (double)y, (double)z};
                const double dd = rm_point_tri_d2(p, a, b, c);
                if (dd <= RM_BAND * RM_BAND) {
                    const uint32_t v = fbits((float)dd);
                    uint32_t& g = d2[rm_lin(x, y, z, R)];
                    if (v < g) g = v;
                }
            }
        }
        for (int k = 0; k < 3; k++) {
            if (rm_tri_area2(a, b, c, k) == 0) continue;
            int llo[2], lhi[2];
            rm_tri_lines(a, b, c, k, R, llo, lhi);
            if (lhi[0] < llo[0] || lhi[1] < llo[1]) continue;
            const long long na = lhi[0] - llo[0] + 1, nb = lhi[1] - llo[1] + 1;
            for (long long q = 0; q < na * nb; q++) {
                const long long node = rm_line_cross(a, b, c, k, llo[0] + (int)(q % na), llo[1] + (int)(q / na), R);
                if (node >= 0) blk[k * N + node] = 1;
            }
        }
    }
    for (long long round = 0;; round++) {                                                // k_rm_sweep
        bool changed = false;
        for (int k = 0; k < 3; k++) {
            const int i = (k + 1) % 3, j = (k + 2) % 3;
            const long long st = k == 0 ? 1 : (k == 1 ? R : (long long)R * R);
            for (long long line = 0; line < (long long)R * R; line++) {
                int q[3];
                q[k] = 0; q[i] = (int)(line % R); q[j] = (int)(line / R);
                const long long base = rm_lin(q[0], q[1], q[2], R);
                const unsigned char* bk = blk.data() + k * N;
                unsigned char prev = outside[base];
                for (int c = 1; c < R; c++) {
                    const long long idx = base + c * st;
                    if (!outside[idx] && prev && !bk[idx - st]) { outside[idx] = 1; changed = true; }
                    prev = outside[idx];
                }
                prev = outside[base + (R - 1) * st];
                for (int c = R - 2; c >= 0; c--) {
                    const long long idx = base + c * st;
                    if (!outside[idx] && prev && !bk[idx]) { outside[idx] = 1; changed = true; }
                    prev = outside[idx];
                }
            }
        }
        if (!changed || round > N) break;
    }
    std::vector<float> sd(N);                                                            // k_rm_field
    for (long long n = 0; n < N; n++) sd[n] = rm_field(d2[n], outside[n] != 0);
    auto crossed = [&](long long n, int x, int y, int z, int k) {
        const int q[3] = {x, y, z};
        if (q[k] > R - 2) return false;
        const long long st = k == 0 ? 1 : (k == 1 ? R : (long long)R * R);
        return (sd[n] < 0.0f) != (sd[n + st] < 0.0f);
    };
    std::vector<int> vid(3 * N);                                                         // k_rm_edge_flags
    for (long long n = 0; n < N; n++) {
        const int x = (int)(n % R), y = (int)(n / R % R), z = (int)(n / ((long long)R * R));
        for (int k = 0; k < 3; k++) vid[3 * n + k] = crossed(n, x, y, z, k) ? 1 : 0;
    }
    const int Rc = R - 1;
    const long long C = (long long)Rc * Rc * Rc;
    std::vector<int> ctri(C), cctr(C);                                                   // k_rm_cell_counts
    for (long long m = 0; m < C; m++) {
        const int x = (int)(m % Rc), y = (int)(m / Rc % Rc), z = (int)(m / ((long long)Rc * Rc));
        const int cs = rm_case(sd.data(), x, y, z, R);
        ctri[m] = tab.ntri[cs]; cctr[m] = tab.nctr[cs];
    }
    const long long nev = scan(vid), ntr = scan(ctri), nct = scan(cctr);
    std::vector<float> ov(3 * (size_t)(nev + nct));
    std::vector<int> ot(3 * (size_t)ntr);
    for (long long n = 0; n < N; n++) {                                                  // k_rm_edge_verts
        const int x = (int)(n % R), y = (int)(n / R % R), z = (int)(n / ((long long)R * R));
        for (int k = 0; k < 3; k++) {
            if (!crossed(n, x, y, z, k)) continue;
            double g[3];
            rm_edge_pos(sd.data(), x, y, z, k, R, g);
            for (int d = 0; d < 3; d++) ov[3 * (size_t)vid[3 * n + k] + d] = rm_denorm(g[d], d, P);
        }
    }
    for (long long m = 0; m < C; m++) {                                                  // k_rm_cells
        const int x = (int)(m % Rc), y = (int)(m / Rc % Rc), z = (int)(m / ((long long)Rc * Rc));
        rm_cell_emit(tab, sd.data(), vid.data(), x, y, z, R, P, (int)nev, ctri[m], cctr[m], ov.data(), ot.data());
    }
    const int out_hdr[2] = {(int)(nev + nct), (int)ntr};
    std::fwrite(out_hdr, 4, 2, stdout);
    std::fwrite(ov.data(), 4, ov.size(), stdout);
    std::fwrite(ot.data(), 4, ot.size(), stdout);
    return 0;
}
