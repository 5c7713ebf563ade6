// Bit-identity of the packed f32x2 evaluation (F2 lanes) of the support-
// operator and hourglass templates against their scalar evaluation on the
// same inputs.  Built and run by tests/test_pair_identity.py.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "../coseis_b200/csrc/pair.cuh"
#include "../coseis_b200/csrc/stencil.cuh"

using namespace sordgpu;

// in: per case 8 xb, 8 xc for lane x, 8 xb, 8 xc for lane y, 8 F, 8 F', h
constexpr int IN = 16 * 2 + 16 + 1;

__global__ void k_pair(const float* in, unsigned* bad, int n, float nzf) {
    const unsigned long long nz = f2_pack(nzf, nzf);
    // bad[0]: all, bad[1]: diff_nc brackets, bad[2]: diff_cn brackets, bad[3]: stencil, bad[4]: hourglass
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = in + (size_t)i * IN;
    float xb0[8], xc0[8], xb1[8], xc1[8], F0[8], F1[8];
    for (int t = 0; t < 8; t++) {
        xb0[t] = p[t]; xc0[t] = p[8 + t]; xb1[t] = p[16 + t]; xc1[t] = p[24 + t];
        F0[t] = p[32 + t]; F1[t] = p[40 + t];
    }
    const float h = p[48];
    F2 PB[8], PC[8], PF[8];
    for (int t = 0; t < 8; t++) { PB[t] = f2(xb0[t], xb1[t], nz); PC[t] = f2(xc0[t], xc1[t], nz); PF[t] = f2(F0[t], F1[t], nz); }
    float B0[8], B1[8], N0[8], N1[8];
    brackets_nc_g<float>(xb0, xc0, B0);
    brackets_nc_g<float>(xb1, xc1, B1);
    cell_cn_brackets_g<float>(xb0, xc0, B0, N0, 0.0f);
    cell_cn_brackets_g<float>(xb1, xc1, B1, N1, 0.0f);
    F2 P[8], PN[8];
    brackets_nc_g<F2>(PB, PC, P);
    cell_cn_brackets_g<F2>(PB, PC, P, PN, f2(0.0f, nz));
    unsigned nb[5] = {0, 0, 0, 0, 0};
    for (int t = 0; t < 8; t++) {
        nb[1] += __float_as_uint(P[t].x()) != __float_as_uint(B0[t]);
        nb[1] += __float_as_uint(P[t].y()) != __float_as_uint(B1[t]);
        nb[2] += __float_as_uint(PN[t].x()) != __float_as_uint(N0[t]);
        nb[2] += __float_as_uint(PN[t].y()) != __float_as_uint(N1[t]);
    }
    // stencil on the scalar brackets in both forms, so it is tested alone
    F2 PBs[8];
    for (int t = 0; t < 8; t++) PBs[t] = f2(B0[t], B1[t], nz);
    const F2 s = stencil8<F2>(PF, PBs, f2(h, nz));
    nb[3] += __float_as_uint(s.x()) != __float_as_uint(stencil8<float>(F0, B0, h));
    nb[3] += __float_as_uint(s.y()) != __float_as_uint(stencil8<float>(F1, B1, h));
    for (int iq = 0; iq < 4; iq++) {
        const F2 r = hg_sum<F2>(PF, iq);
        nb[4] += __float_as_uint(r.x()) != __float_as_uint(hg_sum<float>(F0, iq));
        nb[4] += __float_as_uint(r.y()) != __float_as_uint(hg_sum<float>(F1, iq));
    }
    nb[0] = nb[1] + nb[2] + nb[3] + nb[4];
    for (int c = 0; c < 5; c++)
        if (nb[c]) atomicAdd(bad + c, nb[c]);
}

int main(int argc, char** argv) {
    const int n = argc > 1 ? atoi(argv[1]) : 100000;
    std::mt19937 rng(1234);
    std::uniform_real_distribution<float> U(-1.f, 1.f);
    std::vector<float> in((size_t)n * IN);
    for (int i = 0; i < n; i++) {
        float* p = &in[(size_t)i * IN];
        // perturbed unit-cube corners scaled to metres, as in a curvilinear mesh
        for (int lane = 0; lane < 2; lane++)
            for (int c = 0; c < 2; c++)
                for (int t = 0; t < 8; t++) {
                    const float base = (float)((t >> c) & 1) * 100.f + 1000.f * (float)(i % 7);
                    p[16 * lane + 8 * c + t] = base + 15.f * U(rng);
                }
        for (int t = 0; t < 16; t++) p[32 + t] = U(rng) * 1e-3f;
        p[48] = 1.0f / 12.0f;
    }
    float* din;
    unsigned* dbad;
    unsigned bad[5] = {0, 0, 0, 0, 0};
    cudaMalloc(&din, in.size() * sizeof(float));
    cudaMalloc(&dbad, sizeof(bad));
    cudaMemcpy(din, in.data(), in.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(dbad, 0, sizeof(bad));
    k_pair<<<(n + 127) / 128, 128>>>(din, dbad, n, -0.0f);
    cudaError_t e = cudaMemcpy(bad, dbad, sizeof(bad), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { printf("cuda error %s\n", cudaGetErrorString(e)); return 2; }
    printf("%d %u %u %u %u %u\n", n, bad[0], bad[1], bad[2], bad[3], bad[4]);
    cudaFree(din);
    cudaFree(dbad);
    return 0;
}
