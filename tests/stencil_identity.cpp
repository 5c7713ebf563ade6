// Checks, on random FP32 meshes, that the per-cell divergence brackets of
// coseis_b200/csrc/stencil.cuh (cell_cn_brackets) are bit-identical to the
// per-node diff_cn brackets (brackets_cn) for every corner of the cell.
// Built and run by tests/test_stencil.py.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>

#include "../coseis_b200/csrc/stencil.cuh"

using namespace sordgpu;

int main(int argc, char** argv) {
    int trials = argc > 1 ? atoi(argv[1]) : 20000;
    std::mt19937 rng(7);
    std::uniform_real_distribution<float> U(-1, 1);
    long bad = 0, tot = 0;
    const int ct[8] = {-1, 0, -1, 0, -1, 0, -1, 0}, kt[8] = {-1, -1, -1, -1, 0, 0, 0, 0}, lt[8] = {-1, -1, 0, 0, -1, -1, 0, 0};
    for (int trial = 0; trial < trials; trial++) {
        float base[3] = {U(rng) * 40000, U(rng) * 40000, U(rng) * 20000};
        float sc = trial % 2 ? 50.f : 1e-3f;
        float N[3][27];
        for (int c = 0; c < 3; c++)
            for (int m = 0; m < 27; m++) {
                int d[3] = {m % 3, (m / 3) % 3, m / 9};
                N[c][m] = base[c] + sc * (d[c] + 0.3f * U(rng)) + (trial % 3 == 0 ? 0.f : 5.f * U(rng));
            }
        auto XA = [&](int c, int m) { return N[c][m]; };
        for (int a = 0; a < 3; a++) {
            float Bcn[8];
            brackets_cn(XA, a, Bcn);
            for (int t = 0; t < 8; t++) {
                int cj = 1 + ct[t], ck = 1 + kt[t], cl = 1 + lt[t];
                float X[3][8];
                for (int c = 0; c < 3; c++)
                    for (int n = 0; n < 8; n++)
                        X[c][n] = N[c][(cj + (n & 1)) + 3 * (ck + ((n >> 1) & 1)) + 9 * (cl + (n >> 2))];
                float nc[8], cn[8];
                brackets_nc(X, a, nc);
                cell_cn_brackets(X, a, nc, cn);
                uint32_t bx, by;
                std::memcpy(&bx, &Bcn[t], 4);
                std::memcpy(&by, &cn[t], 4);
                tot++;
                if (bx != by) bad++;
            }
        }
    }
    printf("%ld %ld\n", tot, bad);
    return bad != 0;
}
