// Block-local point-injection lists.
//
// A step's injection list (field-I/O '.' ops, finite sources) holds a few
// dozen entries for the whole mesh, and each entry touches one cell or
// node.  Instead of every thread scanning the global list, warp 0 of each
// block copies, in list order, the entries whose position lies in the
// block's box into shared memory; almost every block ends up with an empty
// list.  Order is kept so that repeated entries on one element apply in the
// same sequence as the reference's loop.  If more than `cap` entries fall in
// the box, the block falls back to the global list (count = -1).
#pragma once

#include "sord.cuh"

namespace sordgpu {

constexpr int kLocalInject = 64;

__device__ __forceinline__ void gather_inject(const InjectList& L, Inject* dst, int* count, const Geom& g, int j1, int j2,
                                              int k1, int k2, int l1, int l2) {
    const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    if (t < 32) {
        int base = 0;
        for (int c = 0; c < L.n; c += 32) {
            const int i = c + t;
            bool in = false;
            Inject e;
            if (i < L.n) {
                e = L.e[i];
                const int j = (int)(e.idx % g.sy) + 1, k = (int)((e.idx / g.sy) % g.nm[1]) + 1, l = (int)(e.idx / g.sz) + 1;
                in = j >= j1 && j <= j2 && k >= k1 && k <= k2 && l >= l1 && l <= l2;
            }
            const unsigned m = __ballot_sync(0xffffffffu, in);
            const int pos = base + __popc(m & ((1u << t) - 1u));
            if (in && pos < kLocalInject) dst[pos] = e;
            base += __popc(m);
        }
        if (t == 0) *count = base <= kLocalInject ? base : -1;
    }
}

// Apply the entries of (local or global) list at element q to a 6-vector.
__device__ __forceinline__ void apply_inject(const Inject* loc, int nloc, const InjectList& L, long long q, float* ed,
                                             float* eo) {
    const Inject* E = nloc >= 0 ? loc : L.e;
    const int n = nloc >= 0 ? nloc : L.n;
    for (int e = 0; e < n; e++)
        if (E[e].idx == q) {
            // constant indices only, so ed / eo stay in registers
            const int c = E[e].comp;
            const float inc = E[e].inc;
            if (c == 0) ed[0] = ed[0] + inc;
            else if (c == 1) ed[1] = ed[1] + inc;
            else if (c == 2) ed[2] = ed[2] + inc;
            else if (c == 3) eo[0] = eo[0] + inc;
            else if (c == 4) eo[1] = eo[1] + inc;
            else eo[2] = eo[2] + inc;
        }
}

}  // namespace sordgpu
