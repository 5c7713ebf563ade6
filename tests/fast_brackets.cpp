// Checks, on random FP32 cells, the fast-arithmetic forms of the support-
// operator brackets in coseis_b200/csrc/stencil.cuh against the reference
// forms (brackets_nc_g, cell_cn_brackets_g, restating diff_nc_op.f90 and
// diff_cn_op.f90), evaluated in double:
//   * terrain cells (x = x(j), y = y(k)): terrain_brackets_0 / _1 against
//     brackets_nc_g of directions 0 and 1;
//   * general cells: -nc[cn_of_nc(t)] against the divergence brackets;
//   * hg_term, the inverse of hg_corner;
//   * the hourglass butterflies hg_modes / hg_reader against hg_sum and the
//     signed mode sums of the reading node's term.
// Prints the largest error relative to the largest bracket of each cell for
// both checks.  Built and run by tests/test_stencil.py.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../coseis_b200/csrc/stencil.cuh"

using namespace sordgpu;

int main(int argc, char** argv) {
    const int trials = argc > 1 ? atoi(argv[1]) : 20000;
    std::mt19937 rng(11);
    std::uniform_real_distribution<double> U(-1, 1);
    double eterr = 0, ecn = 0;
    for (int trial = 0; trial < trials; trial++) {
        const double dx = 50 + 40 * U(rng), dy = 50 + 40 * U(rng), x0 = 2e4 * U(rng), y0 = 2e4 * U(rng);
        double X[3][8];
        float z[8];
        for (int n = 0; n < 8; n++) {
            X[0][n] = x0 + (n & 1) * dx;
            X[1][n] = y0 + ((n >> 1) & 1) * dy;
            z[n] = (float)(-3000 + 80 * (n >> 2) + 30 * U(rng));
            X[2][n] = z[n];
        }
        // terrain: reference brackets in double from the float coordinates
        double B0[8], B1[8];
        brackets_nc_g<double>(X[1], X[2], B0);
        brackets_nc_g<double>(X[2], X[0], B1);
        float T0[8], T1[8];
        terrain_brackets_0((float)dy, z, T0);
        terrain_brackets_1((float)dx, z, T1);
        double m0 = 0, m1 = 0;
        for (int t = 0; t < 8; t++) { m0 = fmax(m0, fabs(B0[t])); m1 = fmax(m1, fabs(B1[t])); }
        for (int t = 0; t < 8; t++) {
            eterr = fmax(eterr, fabs(T0[t] - B0[t]) / m0);
            eterr = fmax(eterr, fabs(T1[t] - B1[t]) / m1);
        }
        // general cell: divergence brackets are the negated gradient brackets
        double G[3][8];
        for (int c = 0; c < 3; c++)
            for (int n = 0; n < 8; n++) G[c][n] = 100.0 * (c == 0 ? (n & 1) : c == 1 ? ((n >> 1) & 1) : (n >> 2)) + 30 * U(rng);
        for (int a = 0; a < 3; a++) {
            double nc[8], cn[8], m = 0;
            brackets_nc_g<double>(G[(a + 1) % 3], G[(a + 2) % 3], nc);
            cell_cn_brackets_g<double>(G[(a + 1) % 3], G[(a + 2) % 3], nc, cn, 0.0);
            for (int t = 0; t < 8; t++) m = fmax(m, fabs(nc[t]));
            for (int t = 0; t < 8; t++) ecn = fmax(ecn, fabs(cn[t] + nc[cn_of_nc(t)]) / m);
        }
    }
    // hourglass butterflies: hg_modes against hg_sum over the term order, and
    // hg_reader against the signed mode sums of the reading node's term
    double ehg = 0;
    for (int trial = 0; trial < 2000; trial++) {
        double X[8], W2[8], m[4], r[4];
        for (int n = 0; n < 8; n++) X[n] = U(rng);
        for (int t = 0; t < 8; t++) W2[t] = X[hg_corner(t)];
        hg_modes<double>(X, m);
        for (int iq = 0; iq < 4; iq++) ehg = fmax(ehg, fabs(m[iq] - hg_sum<double>(W2, iq)));
        hg_readers_pre<double>(m, r);
        for (int q = 0; q < 4; q++) {
            const int hu = hg_term(7 - (q + 4)), hl = hg_term(7 - q);
            double yu = hg_neg(0, hu) ? m[0] : -m[0], yl = hg_neg(0, hl) ? m[0] : -m[0];
            for (int iq = 1; iq < 4; iq++) {
                yu = hg_neg(iq, hu) ? yu + m[iq] : yu - m[iq];
                yl = hg_neg(iq, hl) ? yl + m[iq] : yl - m[iq];
            }
            double bu, bl;
            hg_reader<double>(r, q, bu, bl);
            ehg = fmax(ehg, fmax(fabs(bu - yu), fabs(bl - yl)));
        }
    }
    if (ehg > 1e-14) {
        printf("hourglass butterflies differ: %.3e\n", ehg);
        return 1;
    }
    // hg_term inverts hg_corner (the fast kernel finds a cell's hourglass term by its corner)
    for (int t = 0; t < 8; t++)
        if (hg_term(hg_corner(t)) != t) {
            printf("hg_term(hg_corner(%d)) = %d\n", t, hg_term(hg_corner(t)));
            return 1;
        }
    printf("%.3e %.3e\n", eterr, ecn);
    return 0;
}
