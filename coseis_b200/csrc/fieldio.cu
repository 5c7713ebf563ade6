// Field-I/O engine (sord/input_output.f90:103-591) with device-side data
// movement:
//   non-disk ops  = + * (=~ +~ *~ with the counter hash) @-cubes  -> one
//                 kernel over the strided region; '.' -> point injection
//   disk output   '=>' gathers a strided region into a device record buffer,
//                 '.>' probes (trilinear, <= 8 terms) are batched: one
//                 launch per hook serves every firing probe; records are
//                 copied to the host and appended to the file every nb
//                 samples, at it2 and every itio steps
//   disk input    whole-volume records with unit stride (the setup inputs:
//                 material, coordinates) are read in chunks through pinned
//                 buffers straight into a device record, checked for
//                 NaN / Inf, staged into the volume scratch s1 and applied
//                 on the device; other inputs (sub-cell '.<', strided or
//                 half-dimension records, time-varying inputs) read their
//                 records on the host nb at a time (checked there), and
//                 each record is copied to the device when its step comes
//                 and applied there with the reference's staging,
//                 interpolation and half-dimension fill rules: only the
//                 file's records cross to the device
//   output flush  records are copied into pinned buffers on the stream and
//                 written to disk by a writer thread (write_async)
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <thread>

#include "sord.cuh"
#include "timefn.h"

namespace sordgpu {

#define FCHK(s) do { (s).launches++; SORD_CUDA(cudaGetLastError()); } while (0)

__device__ __forceinline__ unsigned long long f_splitmix(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ float f_urand(unsigned long long call, unsigned long long idx) {
    unsigned long long h = f_splitmix(f_splitmix(call * 0x100000001B3ull + 0x5151) ^ idx);
    return (float)(h >> 40) * (1.0f / 16777216.0f);
}

struct Region {
    int n[3];           // field extents
    int i1[3], i2[3], di[3];
    long long vsy, vsz; // volume strides (random-number index, like s1 of the reference)
};

// op: 0 '=', 1 '+', 2 '*', 3 '=~', 4 '+~', 5 '*~'
__global__ void k_region_op(float* f, Region R, int op, float val, unsigned long long call) {
    long long c0 = (R.i2[0] - R.i1[0]) / R.di[0] + 1, c1 = (R.i2[1] - R.i1[1]) / R.di[1] + 1, c2 = (R.i2[2] - R.i1[2]) / R.di[2] + 1;
    long long n = c0 * c1 * c2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int j = R.i1[0] + R.di[0] * (int)(t % c0), k = R.i1[1] + R.di[1] * (int)((t / c0) % c1), l = R.i1[2] + R.di[2] * (int)(t / (c0 * c1));
        long long q = (j - 1) + (long long)R.n[0] * ((k - 1) + (long long)R.n[1] * (l - 1));
        float F = f[q];
        if (op == 0) F = val;
        else if (op == 1) F = F + val;
        else if (op == 2) F = F * val;
        else {
            float r = f_urand(call, (unsigned long long)((j - 1) + R.vsy * (k - 1) + R.vsz * (l - 1)));
            if (op == 3) F = val * r;
            else if (op == 4) F = F + val * r;
            else F = F * val * r;
        }
        f[q] = F;
    }
}

// '@' cube ops: node fields test node coordinates, cell fields cell centres
__global__ void k_cube(float* f, Region R, const float* x0, const float* x1, const float* x2, Geom g, int cell, int pax,
                       int pidx, int op, float val, float a0, float a1, float a2, float b0, float b1, float b2) {
    long long c0 = (R.i2[0] - R.i1[0]) / R.di[0] + 1, c1 = (R.i2[1] - R.i1[1]) / R.di[1] + 1, c2 = (R.i2[2] - R.i1[2]) / R.di[2] + 1;
    long long n = c0 * c1 * c2;
    const float* X[3] = {x0, x1, x2};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int p[3] = {R.i1[0] + R.di[0] * (int)(t % c0), R.i1[1] + R.di[1] * (int)((t / c0) % c1), R.i1[2] + R.di[2] * (int)(t / (c0 * c1))};
        int v[3] = {p[0], p[1], p[2]};
        if (pax >= 0) v[pax] = pidx;
        long long q = g.idx(v[0], v[1], v[2]);
        float c[3];
        for (int a = 0; a < 3; a++) {
            const float* x = X[a];
            if (cell)
                c[a] = 0.125f * (x[q] + x[q + 1 + g.sy + g.sz] + x[q + g.sy + g.sz] + x[q + 1] + x[q + 1 + g.sz] + x[q + g.sy] +
                                 x[q + 1 + g.sy] + x[q + g.sz]);
            else
                c[a] = x[q];
        }
        if (c[0] >= a0 && c[0] <= b0 && c[1] >= a1 && c[1] <= b1 && c[2] >= a2 && c[2] <= b2) {
            long long fq = (p[0] - 1) + (long long)R.n[0] * ((p[1] - 1) + (long long)R.n[1] * (p[2] - 1));
            float F = f[fq];
            if (op == 0) F = val;
            else if (op == 1) F = F + val;
            else F = F * val;
            f[fq] = F;
        }
    }
}

// '=>' gather of a strided region into one record
__global__ void k_gather(const float* f, Region R, float* dst) {
    long long c0 = (R.i2[0] - R.i1[0]) / R.di[0] + 1, c1 = (R.i2[1] - R.i1[1]) / R.di[1] + 1, c2 = (R.i2[2] - R.i1[2]) / R.di[2] + 1;
    long long n = c0 * c1 * c2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int j = R.i1[0] + R.di[0] * (int)(t % c0), k = R.i1[1] + R.di[1] * (int)((t / c0) % c1), l = R.i1[2] + R.di[2] * (int)(t / (c0 * c1));
        dst[t] = f[(j - 1) + (long long)R.n[0] * ((k - 1) + (long long)R.n[1] * (l - 1))];
    }
}

// '.>' probes: acc = acc + f(j,k,l) * r over <= 8 terms in loop order
struct Probe {
    long long idx[8];
    float r[8];
    int n;
};
struct ProbeBatch {
    int count;
    const Probe* probes;  // device table (all probes)
    int id[128];          // probe ids firing now
    float* dst[128];      // destination of each
};
__global__ void k_probe(const float* f, ProbeBatch b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.count) return;
    const Probe& P = b.probes[b.id[i]];
    float acc = 0.f;
    for (int t = 0; t < P.n; t++) acc = acc + f[P.idx[t]] * P.r[t];
    *b.dst[i] = acc;
}

// Whole-volume input record (unit stride): s1 region = record, and any NaN
// or +Inf flagged (input_output.f90:333-337, 359-369).
__global__ void k_stage_in(float* s1, const float* rec, Region R, unsigned* bad) {
    const long long c0 = R.i2[0] - R.i1[0] + 1, c1 = R.i2[1] - R.i1[1] + 1, c2 = R.i2[2] - R.i1[2] + 1;
    const long long n = c0 * c1 * c2;
    unsigned b = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int j = R.i1[0] + (int)(t % c0), k = R.i1[1] + (int)((t / c0) % c1), l = R.i1[2] + (int)(t / (c0 * c1));
        const float v = rec[t];
        if (v != v || v > 3.402823466e38f) b = 1;
        s1[(j - 1) + (long long)R.n[0] * ((k - 1) + (long long)R.n[1] * (l - 1))] = v;
    }
    if (b) atomicOr(bad, 1u);
}

// f region (op) s1 region: 0 '=<', 1 '+<', 2 '*<' (input_output.f90:392-419)
__global__ void k_apply_in(float* f, const float* s1, Region R, int op) {
    const long long c0 = R.i2[0] - R.i1[0] + 1, c1 = R.i2[1] - R.i1[1] + 1, c2 = R.i2[2] - R.i1[2] + 1;
    const long long n = c0 * c1 * c2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int j = R.i1[0] + (int)(t % c0), k = R.i1[1] + (int)((t / c0) % c1), l = R.i1[2] + (int)(t / (c0 * c1));
        const long long q = (j - 1) + (long long)R.n[0] * ((k - 1) + (long long)R.n[1] * (l - 1));
        const float a = s1[q];
        if (op == 0) f[q] = a;
        else if (op == 1) f[q] = f[q] + a;
        else f[q] = f[q] * a;
    }
}

// One disk-input record (input_output.f90:392-398): the record, j fastest,
// into the strided region of S.
__global__ void k_rec_scatter(float* S, const float* rec, Region R) {
    const long long c0 = (R.i2[0] - R.i1[0]) / R.di[0] + 1, c1 = (R.i2[1] - R.i1[1]) / R.di[1] + 1;
    const long long c2 = (R.i2[2] - R.i1[2]) / R.di[2] + 1, n = c0 * c1 * c2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int j = R.i1[0] + R.di[0] * (int)(t % c0), k = R.i1[1] + R.di[1] * (int)((t / c0) % c1);
        const int l = R.i1[2] + R.di[2] * (int)(t / (c0 * c1));
        S[(j - 1) + (long long)R.n[0] * ((k - 1) + (long long)R.n[1] * (l - 1))] = rec[t];
    }
}

// Linear interpolation between strided samples along one axis
// (utilities.f90:168-220), every i = 1..d-1 at once: positions j + i are
// never samples, so no thread reads what another writes.  The loops, with
// their bounds and steps, are the reference's: axis 0 steps l by di2 and k
// by di1; axis 1 steps l by di0 (sic); axis 2 takes every k and j.
__global__ void k_rec_interp(float* S, int n0, int n1, int axis, int d, int a10, int a11, int a12, int a20, int a21,
                             int a22, int lstep, int kstep) {
    const int jstep = axis == 0 ? d : 1;
    const int kst = axis == 1 ? d : axis == 0 ? kstep : 1, lst = axis == 2 ? d : lstep;
    const int jhi = axis == 0 ? a20 - d : a20, khi = axis == 1 ? a21 - d : a21, lhi = axis == 2 ? a22 - d : a22;
    if (jhi < a10 || khi < a11 || lhi < a12) return;
    const long long cj = (jhi - a10) / jstep + 1, ck = (khi - a11) / kst + 1, cl = (lhi - a12) / lst + 1;
    const long long n = cj * ck * cl * (long long)(d - 1);
    const float rd = 1.0f / (float)d;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = 1 + (int)(t % (d - 1));
        const long long u = t / (d - 1);
        const int j = a10 + jstep * (int)(u % cj), k = a11 + kst * (int)((u / cj) % ck), l = a12 + lst * (int)(u / (cj * ck));
        const float h1 = rd * (float)i, h2 = rd * (float)(d - i);
        auto at = [&](int jj, int kk, int ll) -> float& {
            return S[(jj - 1) + (long long)n0 * ((kk - 1) + (long long)n1 * (ll - 1))];
        };
        if (axis == 0) at(j + i, k, l) = h1 * at(j, k, l) + h2 * at(j + d, k, l);
        else if (axis == 1) at(j, k + i, l) = h1 * at(j, k, l) + h2 * at(j, k + d, l);
        else at(j, k, l + i) = h1 * at(j, k, l) + h2 * at(j, k, l + d);
    }
}

// Half-dimension fill (input_output.f90:399-405): plane 1 of `axis` copied
// along the whole extent of that axis.
__global__ void k_rec_fill(float* S, int n0, int n1, int n2, int axis) {
    const int na = axis == 0 ? n0 : axis == 1 ? n1 : n2;
    const long long plane = (long long)n0 * n1 * n2 / na, n = plane * (na - 1);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int a = 2 + (int)(t / plane);
        const long long r = t % plane;
        long long q, q1;
        if (axis == 0) {
            q1 = r * n0;
            q = q1 + (a - 1);
        } else if (axis == 1) {
            const long long j = r % n0, l = r / n0;
            q1 = j + (long long)n0 * n1 * l;
            q = q1 + (long long)n0 * (a - 1);
        } else {
            q1 = r;
            q = r + (long long)n0 * n1 * (a - 1);
        }
        S[q] = S[q1];
    }
}

// '.<': the record value times each trilinear weight added to the field
// (input_output.f90:378-390); weights from the host, in its order of
// operations
struct PointIn {
    long long idx[8];
    float r[8];
    int n;
};
__global__ void k_point_in(float* f, PointIn P, const float* v) {
    const int t = threadIdx.x;
    if (t < P.n) f[P.idx[t]] = f[P.idx[t]] + P.r[t] * v[0];
}

// ------------------------------------------------------------ host
static unsigned gf(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148LL * 32) b = 148LL * 32;
    return (unsigned)(b < 1 ? 1 : b);
}
static int imod(int a, int b) { int m = a % b; return m < 0 ? m + b : m; }

float host_time_function(const std::string& pulse, float t, float dt, float tau) {
    const float pi = 3.14159265f;
    float f = 0, a, b;
    if (pulse == "const") f = 1;
    else if (pulse == "delta") { if (std::fabs(t) < 0.25f * dt) f = 1.0f / dt; }
    else if (pulse == "step" || pulse == "integral_delta") {
        if (std::fabs(t) < 0.25f * dt) f = 0.5f;
        else if (t >= 0.25f * dt) f = 1;
    } else if (pulse == "brune") {
        if (0.0f < t) { a = 1.0f / tau; f = std::exp(-a * t) * a * a * t; }
    } else if (pulse == "integral_brune") {
        if (0.0f < t) { a = 1.0f / tau; f = 1.0f - std::exp(-a * t) * (a * t + 1.0f); }
    } else if (pulse == "hann") {
        b = pi * tau;
        if (-b < t && t < b) { a = 1.0f / tau; f = 0.5f / pi * a * (1.0f + std::cos(a * t)); }
    } else if (pulse == "integral_hann") {
        b = pi * tau;
        if (-b < t && t < b) { a = 1.0f / tau; f = 0.5f + 0.5f / pi * (a * t + std::sin(a * t)); }
        else if (0.0f < t) f = 1;
    } else if (pulse == "gaussian" || pulse == "integral_ricker1") {
        a = 0.5f / (tau * tau); b = std::sqrt(a / pi); f = std::exp(-a * t * t) * b;
    } else if (pulse == "ricker1" || pulse == "integral_ricker2") {
        a = 0.5f / (tau * tau); b = std::sqrt(a / pi) * 2.0f * a; f = -std::exp(-a * t * t) * b * t;
    } else if (pulse == "ricker2") {
        a = 0.5f / (tau * tau); b = std::sqrt(a / pi) * 4.0f * a; f = std::exp(-a * t * t) * b * (a * t * t - 0.5f);
    } else throw SordError(SORD_E_PARAM, "invalid time func: " + pulse);
    return f;
}

static inline float wgt(float x, int j, bool plane) { return plane ? 1.0f : 1.0f - std::fabs(x - (float)j); }

// as_read: by the op as read from sord.in (the same on every part of a
// partitioned run), not by whether this process holds any of its region
static bool applies(Solver& s, const IoOp& io, const char* field, char pass, bool as_read = false) {
    const std::string& op = as_read ? io.op0 : io.op;
    int it1 = io.ii[3][0], it2 = io.ii[3][1], dit = io.ii[3][2];
    if (s.it > it2) return false;
    if (op[0] == '#') return false;
    if (s.it < it1) return false;
    if (imod(s.it - it1, dit) != 0) return false;
    if (io.field != field) return false;
    char op2 = op.size() > 1 ? op[1] : ' ';
    if (pass == '<' && op2 == '>') return false;
    if (pass == '>' && op2 != '>') return false;
    return true;
}

bool field_active(Solver& s, const char* field, char pass) {
    for (auto& io : s.ops)
        if (applies(s, io, field, pass)) return true;
    return false;
}

// Point-op geometry: i1/i2 (1-based, inclusive), xi and plane flags
struct PointGeom {
    int i1[3], i2[3];
    float xi[3];
    bool plane[3];
};
// probe: a '.>' op of a partitioned run, whose stencil may reach the halo
// planes of the l split (they hold the neighbours' current values); it is
// taken by the part whose core holds the stencil's upper plane
static void point_geom(Solver& s, const IoOp& io, const FieldView& f, PointGeom& P, bool probe = false) {
    const Geom& g = s.g;
    for (int i = 0; i < 3; i++) {
        int i3, i4;
        if (io.reg == 'n') { i3 = g.i1node[i]; i4 = g.i2node[i]; P.xi[i] = io.x1[i] - (float)g.nnoff[i] + 1.0f; }
        else { i3 = g.i1cell[i]; i4 = g.i2cell[i]; P.xi[i] = io.x1[i] - (float)g.nnoff[i] + 0.5f; }
        if (probe && s.nparts > 1 && i == 2) {
            if (s.part > 0) i3 = 1;
            if (s.part < s.nparts - 1) i4 = g.nm[2];
        }
        int fl = (int)std::floor(P.xi[i]);
        P.i1[i] = std::max(i3, fl);
        P.i2[i] = std::min(i4, fl + 1);
        P.plane[i] = f.n[i] == 1 && g.nm[i] != 1;
    }
}

// Injection entries of a '.' op: f(j,k,l) = f(j,k,l) + val*r in loop order.
// Returns false if the op is outside the block (the reference marks it '#').
bool point_injection(Solver& s, IoOp& io, const FieldView& f, int comp, std::vector<Inject>& out) {
    PointGeom P;
    point_geom(s, io, f, P);
    for (int i = 0; i < 3; i++)
        if (P.i2[i] < P.i1[i]) { io.op = "#"; return false; }
    for (int i = 0; i < 3; i++)
        if (P.plane[i]) P.i1[i] = P.i2[i] = 1;
    float val = io.val * host_time_function(io.fname, s.tm, s.g.dt, io.tau);
    for (int l = P.i1[2]; l <= P.i2[2]; l++)
        for (int k = P.i1[1]; k <= P.i2[1]; k++)
            for (int j = P.i1[0]; j <= P.i2[0]; j++) {
                float r = wgt(P.xi[0], j, P.plane[0]) * wgt(P.xi[1], k, P.plane[1]) * wgt(P.xi[2], l, P.plane[2]);
                Inject e;
                e.idx = (long long)(j - 1) + (long long)f.n[0] * ((long long)(k - 1) + (long long)f.n[1] * (long long)(l - 1));
                e.comp = comp;
                e.inc = val * r;
                out.push_back(e);
            }
    return true;
}

// The cells a '.' op touches with their trilinear weights r and dr/dx1
// (x1 in node-index units), in the loop order of point_injection.
bool point_weights(Solver& s, IoOp& io, const FieldView& f, std::vector<PointWeight>& out) {
    PointGeom P;
    point_geom(s, io, f, P);
    for (int i = 0; i < 3; i++)
        if (P.i2[i] < P.i1[i]) return false;
    for (int i = 0; i < 3; i++)
        if (P.plane[i]) P.i1[i] = P.i2[i] = 1;
    for (int l = P.i1[2]; l <= P.i2[2]; l++)
        for (int k = P.i1[1]; k <= P.i2[1]; k++)
            for (int j = P.i1[0]; j <= P.i2[0]; j++) {
                const int c[3] = {j, k, l};
                double w[3], dw[3];
                for (int i = 0; i < 3; i++) {
                    const double d = (double)P.xi[i] - (double)c[i];
                    w[i] = P.plane[i] ? 1.0 : 1.0 - std::fabs(d);
                    dw[i] = P.plane[i] ? 0.0 : (d > 0.0 ? -1.0 : d < 0.0 ? 1.0 : 0.0);
                }
                PointWeight e;
                e.idx = (long long)(j - 1) + (long long)f.n[0] * ((long long)(k - 1) + (long long)f.n[1] * (long long)(l - 1));
                e.r = w[0] * w[1] * w[2];
                e.dr[0] = dw[0] * w[1] * w[2];
                e.dr[1] = w[0] * dw[1] * w[2];
                e.dr[2] = w[0] * w[1] * dw[2];
                out.push_back(e);
            }
    return true;
}

// file-name suffix of a process's own part of a region (mpin / mpout 0)
static std::string part_suffix(const Solver& s) {
    char b[16];
    snprintf(b, sizeof b, "-%06d", s.part);
    return b;
}

static void file_write(Solver& s, IoOp& io, const float* data, int recl, int nrec, const std::string& filename, int m, int o) {
    std::string fn = s.path(filename);
    if (s.nparts > 1 && s.prm.mpout != 0 && io.grecl != (long long)recl) {
        // a partitioned run's shared file: each part writes its part of every
        // record at its offset (the reference writes with MPI-IO,
        // input_output.f90:494-508); no part checks that the file is new
        const int fd = ::open(fn.c_str(), O_WRONLY | O_CREAT, 0644);
        if (fd < 0) throw SordError(SORD_E_IO, "cannot open " + filename);
        for (int r = 0; r < nrec; r++) {
            const size_t bytes = sizeof(float) * (size_t)recl;
            const off_t pos = (off_t)(((size_t)(o + r) * (size_t)io.grecl + (size_t)io.loff) * sizeof(float));
            size_t done = 0;
            while (done < bytes) {
                const ssize_t w = pwrite(fd, reinterpret_cast<const char*>(data + (size_t)r * recl) + done, bytes - done,
                                         pos + (off_t)done);
                if (w <= 0) { ::close(fd); throw SordError(SORD_E_IO, "write failed: " + filename); }
                done += (size_t)w;
            }
        }
        ::close(fd);
        return;
    }
    FILE* fp;
    if (!io.open && o == 0) {
        fp = fopen(fn.c_str(), "rb");
        if (fp) { fclose(fp); throw SordError(SORD_E_IO, "file exists: " + filename); }
        fp = fopen(fn.c_str(), "wb");
    } else {
        fp = fopen(fn.c_str(), "r+b");
    }
    if (!fp) throw SordError(SORD_E_IO, "cannot open " + filename);
    io.open = true;
    fseek(fp, (long)((size_t)recl * sizeof(float) * (size_t)o), SEEK_SET);
    fwrite(data, sizeof(float), (size_t)recl * nrec, fp);
    fclose(fp);
    if (o + nrec == m) io.open = false;
}

static void region_scalar_bc(Solver& s, IoOp& io, FieldView f) {
    const Geom& g = s.g;
    if (io.reg == 'n') launch_scalar_bc(s, f.p, f.n, s.prm.bc1, s.prm.bc2, g.i1bc, g.i2bc);
    if (io.reg == 'c') {
        int t[3] = {g.i2bc[0] - 1, g.i2bc[1] - 1, g.i2bc[2] - 1};
        launch_scalar_bc(s, f.p, f.n, s.prm.bc1, s.prm.bc2, g.i1bc, t);
    }
}

struct ProbeTable {
    std::vector<Probe> host;
    Probe* dev = nullptr;
    std::vector<int> id_of_op;  // op index -> probe id (-1 none)
};
static std::map<const Solver*, ProbeTable> g_probes;  // guarded by g_probes_m
static std::mutex g_probes_m;

static ProbeTable& probe_table(const Solver& s) {
    std::lock_guard<std::mutex> lock(g_probes_m);
    return g_probes[&s];  // element references stay valid while the map changes
}

static int probe_id(Solver& s, size_t opi, const IoOp& io, const FieldView& f) {
    ProbeTable& T = probe_table(s);
    if (T.id_of_op.size() != s.ops.size()) T.id_of_op.assign(s.ops.size(), -1);
    if (T.id_of_op[opi] >= 0) return T.id_of_op[opi];
    PointGeom P;
    point_geom(s, io, f, P, true);
    int i1[3], i2[3];
    for (int i = 0; i < 3; i++) { i1[i] = P.i1[i]; i2[i] = P.i2[i]; if (f.n[i] == 1) { i1[i] = i2[i] = 1; } }
    Probe pr;
    pr.n = 0;
    for (int l = i1[2]; l <= i2[2]; l++)
        for (int k = i1[1]; k <= i2[1]; k++)
            for (int j = i1[0]; j <= i2[0]; j++) {
                if (pr.n >= 8) break;
                pr.idx[pr.n] = (long long)(j - 1) + (long long)f.n[0] * ((long long)(k - 1) + (long long)f.n[1] * (long long)(l - 1));
                pr.r[pr.n] = wgt(P.xi[0], j, P.plane[0]) * wgt(P.xi[1], k, P.plane[1]) * wgt(P.xi[2], l, P.plane[2]);
                pr.n++;
            }
    T.host.push_back(pr);
    dev_free(s, T.dev);
    SORD_CUDA(dev_malloc(s, (void**)&T.dev, sizeof(Probe) * T.host.size()));
    SORD_CUDA(cudaMemcpyAsync(T.dev, T.host.data(), sizeof(Probe) * T.host.size(), cudaMemcpyHostToDevice, s.stream));
    SORD_CUDA(cudaStreamSynchronize(s.stream));
    T.id_of_op[opi] = (int)T.host.size() - 1;
    return T.id_of_op[opi];
}

// Probe of '.>' op opi (recorded when the op first fired): node or cell
// indices and trilinear weights; returns the count, or 0 if the op never fired.
int probe_of_op(const Solver& s, size_t opi, long long* idx, float* r) {
    std::lock_guard<std::mutex> lock(g_probes_m);
    auto it = g_probes.find(&s);
    if (it == g_probes.end() || opi >= it->second.id_of_op.size() || it->second.id_of_op[opi] < 0) return 0;
    const Probe& p = it->second.host[it->second.id_of_op[opi]];
    for (int t = 0; t < p.n; t++) { idx[t] = p.idx[t]; r[t] = p.r[t]; }
    return p.n;
}

void probes_free(Solver& s) {
    std::lock_guard<std::mutex> lock(g_probes_m);
    auto it = g_probes.find(&s);
    if (it != g_probes.end()) {
        dev_free(s, it->second.dev);
        g_probes.erase(it);
    }
}

// Output records go to disk on a writer thread per handle: a flush copies
// the device record buffer into a pinned buffer on the solver's stream and
// queues the write behind an event, so the stream never waits for the
// disk; the writer takes the jobs in order (so each file's records are
// written in order), waits for each copy, writes and returns the buffer.
// Errors are kept and reported by writer_drain.
struct OutJob {
    size_t opi;
    float* pin;
    cudaEvent_t ev;
    int recl, nrec, m, o;
    std::string filename;
};
struct OutWriter {
    std::thread th;
    std::mutex mu;
    std::condition_variable cv, idle;
    std::deque<OutJob> q;
    bool stop = false, busy = false;
    int code = 0;
    std::string msg;
};

static void writer_loop(Solver* s, OutWriter* w) {
    cudaSetDevice(s->device);
    for (;;) {
        OutJob job;
        {
            std::unique_lock<std::mutex> lock(w->mu);
            w->cv.wait(lock, [&] { return w->stop || !w->q.empty(); });
            if (w->q.empty()) return;
            job = std::move(w->q.front());
            w->q.pop_front();
            w->busy = true;
        }
        int code = 0;
        std::string msg;
        try {
            SORD_CUDA(cudaEventSynchronize(job.ev));
            file_write(*s, s->ops[job.opi], job.pin, job.recl, job.nrec, job.filename, job.m, job.o);
        } catch (const SordError& e) {
            code = e.code;
            msg = e.what();
        } catch (const std::exception& e) {
            code = SORD_E_IO;
            msg = e.what();
        }
        cudaEventDestroy(job.ev);
        pinned_put(job.pin);
        std::lock_guard<std::mutex> lock(w->mu);
        if (code && !w->code) { w->code = code; w->msg = msg; }
        w->busy = false;
        if (w->q.empty()) w->idle.notify_all();
    }
}

// Wait until every queued record is on disk; throw the first write error.
void writer_drain(Solver& s) {
    OutWriter* w = s.writer;
    if (!w) return;
    std::unique_lock<std::mutex> lock(w->mu);
    w->idle.wait(lock, [&] { return w->q.empty() && !w->busy; });
    if (w->code) {
        const int c = w->code;
        w->code = 0;
        throw SordError(c, w->msg);
    }
}

void writer_free(Solver& s) {
    OutWriter* w = s.writer;
    if (!w) return;
    {
        std::lock_guard<std::mutex> lock(w->mu);
        w->stop = true;
    }
    w->cv.notify_all();
    if (w->th.joinable()) w->th.join();
    delete w;
    s.writer = nullptr;
}

static void write_async(Solver& s, IoOp& io, int nrec, const std::string& filename, int m, int o) {
    if (!s.writer) {
        s.writer = new OutWriter();
        s.writer->th = std::thread(writer_loop, &s, s.writer);
    }
    OutJob job;
    job.opi = (size_t)(&io - s.ops.data());
    job.recl = io.bufn;
    job.nrec = nrec;
    job.m = m;
    job.o = o;
    job.filename = filename;
    const size_t bytes = sizeof(float) * (size_t)io.bufn * nrec;
    job.pin = (float*)pinned_get(bytes);
    SORD_CUDA(cudaMemcpyAsync(job.pin, io.dbuf, bytes, cudaMemcpyDeviceToHost, s.stream));
    SORD_CUDA(cudaEventCreateWithFlags(&job.ev, cudaEventDisableTiming));
    SORD_CUDA(cudaEventRecord(job.ev, s.stream));
    {
        std::lock_guard<std::mutex> lock(s.writer->mu);
        s.writer->q.push_back(std::move(job));
    }
    s.writer->cv.notify_one();
}

static void flush_output(Solver& s, IoOp& io, int n3[3], int m3[3]) {
    int it1 = io.ii[3][0], it2 = io.ii[3][1], dit = io.ii[3][2];
    int n4 = io.ib;
    int m4 = (it2 - it1) / dit + 1;
    int o4 = (s.it - it1) / dit + 1 - n4;
    std::string filename = io.fname;
    if ((n3[0] != m3[0] || n3[1] != m3[1] || n3[2] != m3[2]) && s.prm.mpout == 0) filename += part_suffix(s);
    if (!(n3[0] < 1 || n3[1] < 1 || n3[2] < 1 || n4 < 1)) write_async(s, io, n4, filename, m4, o4);
    io.ib = 0;
    if (s.it == it2 || n3[0] < 1 || n3[1] < 1 || n3[2] < 1 || n4 < 1) {
        dev_free(s, io.dbuf);
        io.dbuf = nullptr;
        io.op = "#";
    }
}

static void magnitude(Solver& s, const std::string& fl) {
    const Geom& g = s.g;
    int one[3] = {1, 1, 1};
    if (fl == "vm2") dev_vector_norm(s, s.d.s1, s.d.v, g.i1core, g.i2core, one);
    else if (fl == "um2") dev_vector_norm(s, s.d.s1, s.d.u, g.i1core, g.i2core, one);
    else if (fl == "am2") dev_vector_norm(s, s.d.s1, s.d.w1n, g.i1core, g.i2core, one);
    else if (fl == "wm2") dev_tensor_norm(s, s.d.s1, s.d.sd, s.d.so, g.i1core, g.i2core, one);
}

// Read `count` floats of file `fn` from float offset `off` into device
// memory `dst`.  kReaders host threads each read every kReaders-th chunk of
// 8 M floats with pread into their own pinned buffer and copy it to the
// device on the solver's stream; a thread waits for its previous copy before
// reusing its buffer.
static constexpr int kReaders = 8;
static constexpr size_t kChunk = (size_t)8 << 20;
static void read_to_device(Solver& s, const std::string& fn, size_t off, size_t count, float* dst) {
    static_assert(kReaders <= (int)(sizeof(s.pin_io) / sizeof(s.pin_io[0])), "pinned buffers");
    for (int i = 0; i < kReaders; i++)
        if (!s.pin_io[i]) {
            s.pin_io[i] = (float*)pinned_get(sizeof(float) * kChunk);
            SORD_CUDA(cudaEventCreateWithFlags(&s.pin_ev[i], cudaEventDisableTiming));
        }
    const int fd = open(s.path(fn).c_str(), O_RDONLY);
    if (fd < 0) throw SordError(SORD_E_IO, "cannot open " + fn);
    const size_t nchunk = (count + kChunk - 1) / kChunk;
    std::atomic<int> err{0};  // 1 short read, 2 CUDA error
    auto reader = [&](int t) {
        for (size_t c = (size_t)t; c < nchunk && !err.load(); c += kReaders) {
            const size_t want = std::min(kChunk, count - c * kChunk);
            if (cudaEventSynchronize(s.pin_ev[t]) != cudaSuccess) { err = 2; return; }
            char* p = reinterpret_cast<char*>(s.pin_io[t]);
            size_t got = 0;
            const size_t bytes = want * sizeof(float);
            const off_t base = (off_t)((off + c * kChunk) * sizeof(float));
            while (got < bytes) {
                const ssize_t r = pread(fd, p + got, bytes - got, base + (off_t)got);
                if (r <= 0) { err = 1; return; }
                got += (size_t)r;
            }
            if (cudaMemcpyAsync(dst + c * kChunk, p, bytes, cudaMemcpyHostToDevice, s.stream) != cudaSuccess ||
                cudaEventRecord(s.pin_ev[t], s.stream) != cudaSuccess) {
                err = 2;
                return;
            }
        }
    };
    std::thread th[kReaders];
    for (int t = 0; t < kReaders; t++) th[t] = std::thread(reader, t);
    for (int t = 0; t < kReaders; t++) th[t].join();
    close(fd);
    if (err == 1) {
        SORD_CUDA(cudaStreamSynchronize(s.stream));
        throw SordError(SORD_E_IO, "short read " + fn);
    }
    if (err == 2) SORD_CUDA(cudaGetLastError());
}

// Copy `count` floats of host memory to device memory `dst` on the solver's
// stream through the pinned chunk buffers, so that the copy is queued
// behind the stream's work instead of waiting for it (a pageable source
// would); a chunk buffer is refilled once its previous copy has run.
static void upload_record(Solver& s, const float* src, size_t count, float* dst) {
    for (size_t c = 0; c * kChunk < count; c++) {
        const int t = s.rec_slot;
        s.rec_slot = (s.rec_slot + 1) % kReaders;
        if (!s.pin_io[t]) {
            s.pin_io[t] = (float*)pinned_get(sizeof(float) * kChunk);
            SORD_CUDA(cudaEventCreateWithFlags(&s.pin_ev[t], cudaEventDisableTiming));
        }
        SORD_CUDA(cudaEventSynchronize(s.pin_ev[t]));
        const size_t want = std::min(kChunk, count - c * kChunk);
        std::memcpy(s.pin_io[t], src + c * kChunk, sizeof(float) * want);
        SORD_CUDA(cudaMemcpyAsync(dst + c * kChunk, s.pin_io[t], sizeof(float) * want, cudaMemcpyHostToDevice, s.stream));
        SORD_CUDA(cudaEventRecord(s.pin_ev[t], s.stream));
    }
}

// Device path of disk input for one whole-volume record with unit stride
// and no half-dimension fill, read once (static inputs).  Same semantics as
// the host path below: s1 keeps the staged record, f gets the op.
static bool device_volume_input(Solver& s, IoOp& io, FieldView f, const int* i1, const int* i2, const int* di,
                                const int* m, const int* n) {
    const Geom& g = s.g;
    const int it1 = io.ii[3][0], it2 = io.ii[3][1], dit = io.ii[3][2];
    const int code = io.op == "=<" ? 0 : io.op == "+<" ? 1 : io.op == "*<" ? 2 : -1;
    if (code < 0 || io.ib >= 0 || s.it != it2) return false;
    if (code != 0 && f.p == s.d.s1) return false;  // f aliases the staging scratch: host path order
    for (int i = 0; i < 3; i++)
        if (f.n[i] != g.nm[i] || di[i] != 1 || (m[i] != n[i] && !(s.nparts > 1 && i == 2)) || m[i] == 1 || n[i] < 1)
            return false;
    const size_t nsp = (size_t)n[0] * n[1] * n[2];
    if (nsp == 0) return false;
    if (s.stage_cap < nsp) {
        dev_free(s, s.d_stage);
        s.d_stage = nullptr;
        s.stage_cap = 0;
        if (dev_malloc(s, (void**)&s.d_stage, sizeof(float) * (nsp + 1)) != cudaSuccess) {
            cudaGetLastError();
            throw SordError(SORD_E_NOMEM, "cannot allocate the input staging record");
        }
        s.stage_cap = nsp;
    }
    unsigned* bad = reinterpret_cast<unsigned*>(s.d_stage + nsp);
    SORD_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned), s.stream));
    const int o4 = (s.it - it1) / dit;
    read_to_device(s, io.fname, (size_t)io.grecl * (size_t)o4 + (size_t)io.loff, nsp, s.d_stage);
    Region R;
    for (int i = 0; i < 3; i++) { R.n[i] = f.n[i]; R.i1[i] = i1[i]; R.i2[i] = i2[i]; R.di[i] = 1; }
    R.vsy = g.sy;
    R.vsz = g.sz;
    k_stage_in<<<gf((long long)nsp), 256, 0, s.stream>>>(s.d.s1, s.d_stage, R, bad);
    FCHK(s);
    unsigned hbad = 0;
    SORD_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, s.stream));
    SORD_CUDA(cudaStreamSynchronize(s.stream));
    if (hbad) throw SordError(SORD_E_NANINF, "NaN/Inf in " + io.fname);
    k_apply_in<<<gf((long long)nsp), 256, 0, s.stream>>>(f.p, s.d.s1, R, code);
    FCHK(s);
    return true;
}

// disk input (input_output.f90:296-437): records read on the host in
// batches of nb, each applied on the device when its step comes
static void disk_input(Solver& s, IoOp& io, FieldView f, int* i1, int* i2, int* di, int* m, int* n, int* o, const PointGeom* P) {
    const Geom& g = s.g;
    int it1 = io.ii[3][0], it2 = io.ii[3][1], dit = io.ii[3][2];
    if (io.op != ".<")
        for (int i = 0; i < 3; i++)
            if (m[i] == 1) { i1[i] = 1; i2[i] = 1; n[i] = 1; o[i] = 0; }
    if (io.op != ".<" && device_volume_input(s, io, f, i1, i2, di, m, n)) {
        region_scalar_bc(s, io, f);
        io.op = "#";
        return;
    }
    int nsp = n[0] * n[1] * n[2];
    if (io.ib < 0) {
        io.bufn = std::max(nsp, 0);
        io.hbuf.assign((size_t)io.bufn * io.nb, 0.f);
        io.ib = io.nb;
    }
    if (io.ib == io.nb) {
        int n4 = std::min(io.nb, (it2 - s.it) / dit + 1);
        int o4 = (s.it - it1) / dit;
        std::string filename = io.fname;
        if ((n[0] != m[0] || n[1] != m[1] || n[2] != m[2]) && s.prm.mpin == 0) filename += part_suffix(s);
        io.ib = 0;
        if (n[0] < 1 || n[1] < 1 || n[2] < 1 || n4 < 1) { io.hbuf.clear(); io.op = "#"; return; }
        FILE* fp = fopen(s.path(filename).c_str(), "rb");
        if (!fp) throw SordError(SORD_E_IO, "cannot open " + filename);
        size_t recl = (size_t)nsp;
        // records of the whole region, this process's part of each (one
        // read when that is the whole record)
        const bool whole = s.prm.mpin == 0 || (size_t)io.grecl == recl;
        const size_t frecl = whole ? recl : (size_t)io.grecl, foff = whole ? 0 : (size_t)io.loff;
        size_t got = 0;
        if (frecl == recl) {
            fseek(fp, (long)(recl * sizeof(float) * (size_t)o4), SEEK_SET);
            got = fread(io.hbuf.data(), sizeof(float), recl * n4, fp);
        } else {
            for (int r = 0; r < n4; r++) {
                fseek(fp, (long)(((size_t)(o4 + r) * frecl + foff) * sizeof(float)), SEEK_SET);
                got += fread(io.hbuf.data() + (size_t)r * recl, sizeof(float), recl, fp);
            }
        }
        fclose(fp);
        if (got != recl * n4) throw SordError(SORD_E_IO, "short read " + filename);
        for (size_t q = 0; q < recl * n4; q++) {
            float v = io.hbuf[q];
            if (v != v || v > std::numeric_limits<float>::max()) throw SordError(SORD_E_NANINF, "NaN/Inf in " + io.fname);
        }
    }
    io.ib = io.ib + 1;
    const float* buf = io.hbuf.data() + (size_t)io.bufn * (io.ib - 1);
    // on the device: only the record crosses to it
    const size_t fsz = (size_t)f.n[0] * f.n[1] * f.n[2];
    const bool volume = f.n[0] == g.nm[0] && f.n[1] == g.nm[1] && f.n[2] == g.nm[2];
    // S: the volume scratch s1 for volume fields (the reference stages the
    // record there, and s1 keeps it), else a zeroed temporary after the
    // record; a field that is s1 itself also takes the temporary, and ends
    // as its old values op S like the reference's (F op S, then f = F)
    const bool in_s1 = volume && f.p != s.d.s1;
    const size_t need = (size_t)nsp + (in_s1 ? 0 : fsz) + 1;
    if (s.stage_cap < need) {
        dev_free(s, s.d_stage);
        s.d_stage = nullptr;
        s.stage_cap = 0;
        if (dev_malloc(s, (void**)&s.d_stage, sizeof(float) * need) != cudaSuccess) {
            cudaGetLastError();
            throw SordError(SORD_E_NOMEM, "cannot allocate the input staging record");
        }
        s.stage_cap = need;
    }
    upload_record(s, buf, (size_t)nsp, s.d_stage);
    if (io.op == ".<") {
        PointIn pin{};
        for (int l = i1[2]; l <= i2[2]; l++)
            for (int k = i1[1]; k <= i2[1]; k++)
                for (int j = i1[0]; j <= i2[0]; j++) {
                    pin.idx[pin.n] = (long long)(j - 1) + (long long)f.n[0] * ((long long)(k - 1) + (long long)f.n[1] * (long long)(l - 1));
                    pin.r[pin.n] = wgt(P->xi[0], j, P->plane[0]) * wgt(P->xi[1], k, P->plane[1]) * wgt(P->xi[2], l, P->plane[2]);
                    pin.n++;
                }
        k_point_in<<<1, 32, 0, s.stream>>>(f.p, pin, s.d_stage);
        FCHK(s);
    } else {
        float* S = in_s1 ? s.d.s1 : s.d_stage + nsp;
        if (!in_s1) SORD_CUDA(cudaMemsetAsync(S, 0, sizeof(float) * fsz, s.stream));
        Region R;
        for (int i = 0; i < 3; i++) { R.n[i] = f.n[i]; R.i1[i] = i1[i]; R.i2[i] = i2[i]; R.di[i] = di[i]; }
        R.vsy = g.sy;
        R.vsz = g.sz;
        k_rec_scatter<<<gf((long long)nsp), 256, 0, s.stream>>>(S, s.d_stage, R);
        FCHK(s);
        if (di[0] > 1 || di[1] > 1 || di[2] > 1) {
            // utilities.f90:168-220
            int a1[3], a2[3];
            for (int i = 0; i < 3; i++) {
                a1[i] = io.ii[i][0] - g.nnoff[i]; a2[i] = io.ii[i][1] - g.nnoff[i];
                if (a1[i] < 1) a1[i] = a1[i] + (-a1[i] / di[i] + 1) * di[i];
                if (a2[i] > f.n[i]) a2[i] = a1[i] + (f.n[i] - a1[i]) / di[i] * di[i];
            }
            for (int axis = 0; axis < 3; axis++) {
                const int d = di[axis];
                if (d <= 1) continue;
                k_rec_interp<<<gf((long long)fsz), 256, 0, s.stream>>>(S, f.n[0], f.n[1], axis, d, a1[0], a1[1], a1[2],
                                                                       a2[0], a2[1], a2[2], axis == 0 ? di[2] : di[0], di[1]);
                FCHK(s);
            }
        }
        for (int axis = 0; axis < 3; axis++)
            if (m[axis] == 1) {
                i2[axis] = f.n[axis];
                if (f.n[axis] > 1) {
                    k_rec_fill<<<gf((long long)fsz), 256, 0, s.stream>>>(S, f.n[0], f.n[1], f.n[2], axis);
                    FCHK(s);
                }
            }
        const int code = io.op == "=<" ? 0 : io.op == "+<" ? 1 : io.op == "*<" ? 2 : -1;
        if (code < 0) throw SordError(SORD_E_PARAM, "bad i/o op");
        Region A;
        for (int i = 0; i < 3; i++) { A.n[i] = f.n[i]; A.i1[i] = i1[i]; A.i2[i] = i2[i]; A.di[i] = 1; }
        A.vsy = g.sy;
        A.vsz = g.sz;
        const long long na = (long long)(i2[0] - i1[0] + 1) * (i2[1] - i1[1] + 1) * (i2[2] - i1[2] + 1);
        if (na > 0) {
            k_apply_in<<<gf(na), 256, 0, s.stream>>>(f.p, S, A, code);
            FCHK(s);
        }
    }
    region_scalar_bc(s, io, f);
    if (s.it == it2) { io.hbuf.clear(); io.op = "#"; }
}

static void field_io_op(Solver& s, size_t opi, FieldView f, ProbeBatch& batch) {
    IoOp& io = s.ops[opi];
    const Geom& g = s.g;
    int i1[3], i2[3], i3[3], i4[3], di[3], m[4], n[4], o[4];
    char op2 = io.op.size() > 1 ? io.op[1] : ' ';
    PointGeom P;
    point_geom(s, io, f, P, io.op == ".>");
    if (io.op[0] == '.') {
        for (int i = 0; i < 3; i++) { i1[i] = P.i1[i]; i2[i] = P.i2[i]; di[i] = 1; }
    } else {
        for (int i = 0; i < 3; i++) {
            if (io.reg == 'n') { i3[i] = g.i1node[i]; i4[i] = g.i2node[i]; }
            else { i3[i] = g.i1cell[i]; i4[i] = g.i2cell[i]; }
            i1[i] = io.ii[i][0] - g.nnoff[i]; i2[i] = io.ii[i][1] - g.nnoff[i]; di[i] = io.ii[i][2];
            if (i1[i] < i3[i]) i1[i] = i1[i] + ((i3[i] - i1[i] - 1) / di[i] + 1) * di[i];
            if (i2[i] > i4[i]) i2[i] = i1[i] + (i4[i] - i1[i]) / di[i] * di[i];
        }
    }
    // non-disk input
    if (op2 != '<' && op2 != '>') {
        for (int i = 0; i < 3; i++)
            if (i2[i] < i1[i]) { io.op = "#"; return; }
        int pax = -1;
        for (int i = 0; i < 3; i++)
            if (P.plane[i]) { i1[i] = i2[i] = 1; di[i] = 1; pax = i; }
        if (io.op == ".") {
            std::vector<Inject> e;
            point_injection(s, io, f, 0, e);
            if (!e.empty()) {
                float* F6[6] = {f.p, f.p, f.p, f.p, f.p, f.p};
                launch_inject(s, F6, upload_inject(s, 3, e));
            }
        } else {
            float val = io.val * host_time_function(io.fname, s.tm, g.dt, io.tau);
            Region R;
            for (int i = 0; i < 3; i++) { R.n[i] = f.n[i]; R.i1[i] = i1[i]; R.i2[i] = i2[i]; R.di[i] = di[i]; }
            R.vsy = g.sy; R.vsz = g.sz;
            long long cnt = 1;
            for (int i = 0; i < 3; i++) cnt *= (i2[i] - i1[i]) / di[i] + 1;
            const std::string& op = io.op;
            if (op == "=" || op == "+" || op == "*" || op == "=~" || op == "+~" || op == "*~") {
                int code = op == "=" ? 0 : op == "+" ? 1 : op == "*" ? 2 : op == "=~" ? 3 : op == "+~" ? 4 : 5;
                unsigned long long call = code >= 3 ? s.rng_calls++ : 0;
                k_region_op<<<gf(cnt), 256, 0, s.stream>>>(f.p, R, code, val, call);
                FCHK(s);
            } else if (op == "=@" || op == "+@" || op == "*@") {
                int code = op[0] == '=' ? 0 : op[0] == '+' ? 1 : 2;
                int pidx = pax >= 0 ? g.irup : 0;
                k_cube<<<gf(cnt), 256, 0, s.stream>>>(f.p, R, s.d.x[0], s.d.x[1], s.d.x[2], g, io.reg == 'c' ? 1 : 0, pax, pidx,
                                                     code, val, io.x1[0], io.x1[1], io.x1[2], io.x2[0], io.x2[1], io.x2[2]);
                FCHK(s);
            } else {
                throw SordError(SORD_E_PARAM, "bad i/o mode '" + op + "'");
            }
        }
        region_scalar_bc(s, io, f);
        return;
    }
    // spatial indices for disk i/o
    if (io.op[0] == '.') {
        for (int i = 0; i < 4; i++) { m[i] = 1; n[i] = 1; o[i] = 0; }
    } else {
        for (int i = 0; i < 3; i++) {
            i1[i] = io.ii[i][0] - g.nnoff[i]; i2[i] = io.ii[i][1] - g.nnoff[i]; di[i] = io.ii[i][2];
            i3[i] = i1[i]; i4[i] = i2[i];
            if (i1[i] < g.i1core[i]) i1[i] = i1[i] + ((g.i1core[i] - i1[i] - 1) / di[i] + 1) * di[i];
            if (i2[i] > g.i2core[i]) i2[i] = i1[i] + (g.i2core[i] - i1[i]) / di[i] * di[i];
            m[i] = (i4[i] - i3[i]) / di[i] + 1;
            n[i] = (i2[i] - i1[i]) / di[i] + 1;
            o[i] = (i1[i] - i3[i]) / di[i];
            n[i] = std::max(n[i], 0);
        }
        m[3] = n[3] = 1; o[3] = 0;
    }
    for (int i = 0; i < 3; i++)
        if (f.n[i] == 1) {
            if (n[i] < 1) { io.op = "#"; return; }
            i1[i] = 1; i2[i] = 1; m[i] = 1; n[i] = 1; o[i] = 0;
        }
    // this process's part of each file record: contiguous when only l is
    // split (a partitioned run); the whole record otherwise
    io.grecl = (long long)m[0] * m[1] * m[2];
    io.loff = (long long)o[0] + (long long)m[0] * ((long long)o[1] + (long long)m[1] * o[2]);
    if ((n[0] != m[0] || n[1] != m[1]) && n[2] > 1 && n[0] > 0 && n[1] > 0 && n[2] > 0 && s.nparts > 1)
        throw SordError(SORD_E_PARAM, "partitioned run: a disk region split in j or k");
    if (op2 == '<') {
        disk_input(s, io, f, i1, i2, di, m, n, o, &P);
        return;
    }
    if (op2 == '>') {
        if (io.op == ".>")
            for (int i = 0; i < 3; i++)
                if (!P.plane[i] && (i2[i] < g.i1core[i] || i2[i] > g.i2core[i])) { io.op = "#"; return; }
        int nsp = n[0] * n[1] * n[2];
        if (io.ib < 0) {
            io.bufn = std::max(nsp, 0);
            size_t bytes = sizeof(float) * (size_t)std::max(io.bufn * io.nb, 1);
            cudaError_t e = dev_malloc(s, (void**)&io.dbuf, bytes);
            if (e != cudaSuccess) throw SordError(SORD_E_NOMEM, "output buffer: " + std::string(cudaGetErrorString(e)));
            io.ib = 0;
            io.open = false;
        }
        std::string fl = io.field;
        if (fl == "vm2" || fl == "um2" || fl == "wm2" || fl == "am2") magnitude(s, fl);
        io.ib = io.ib + 1;
        float* dst = io.dbuf + (size_t)io.bufn * (io.ib - 1);
        if (io.op == ".>") {
            int id = probe_id(s, opi, io, f);
            if (batch.count == 128) {
                // flush a full batch before adding more
                k_probe<<<1, 128, 0, s.stream>>>(f.p, batch);
                FCHK(s);
                batch.count = 0;
            }
            batch.probes = probe_table(s).dev;
            batch.id[batch.count] = id;
            batch.dst[batch.count] = dst;
            batch.count++;
        } else if (io.op == "=>") {
            Region R;
            for (int i = 0; i < 3; i++) { R.n[i] = f.n[i]; R.i1[i] = i1[i]; R.i2[i] = i2[i]; R.di[i] = di[i]; }
            R.vsy = g.sy; R.vsz = g.sz;
            if (nsp > 0) {
                k_gather<<<gf(nsp), 256, 0, s.stream>>>(f.p, R, dst);
                FCHK(s);
            }
        } else throw SordError(SORD_E_PARAM, "bad i/o op");
        if (io.ib == io.nb || s.it == io.ii[3][1] || imod(s.it, s.prm.itio) == 0) {
            if (batch.count) {
                k_probe<<<1, 128, 0, s.stream>>>(f.p, batch);
                FCHK(s);
                batch.count = 0;
            }
            int n3[3] = {n[0], n[1], n[2]}, m3[3] = {m[0], m[1], m[2]};
            flush_output(s, io, n3, m3);
        }
        return;
    }
    throw SordError(SORD_E_PARAM, "bad i/o op");
}

void field_io(Solver& s, const char* passes, const char* field, FieldView f) {
    for (const char* pp = passes; *pp; pp++) {
        char pass = *pp;
        ProbeBatch batch;
        batch.count = 0;
        batch.probes = nullptr;
        bool any = false;
        for (size_t i = 0; i < s.ops.size(); i++) {
            if (applies(s, s.ops[i], field, pass, true)) any = true;
            if (!applies(s, s.ops[i], field, pass)) continue;
            field_io_op(s, i, f, batch);
        }
        // a partitioned run takes the halo planes of an input volume field
        // from its neighbours (input_output.f90:218-238, 367 swap the staged
        // values); `any` goes by the ops as read, so every part makes the
        // same exchanges
        if (pass == '<' && any && s.nparts > 1 && f.n[0] == s.g.nm[0] && f.n[1] == s.g.nm[1] && f.n[2] == s.g.nm[2])
            halo_exchange(s, &f.p, 1);
        if (batch.count) {
            k_probe<<<1, 128, 0, s.stream>>>(f.p, batch);
            FCHK(s);
        }
    }
}

void field_io_flush_all(Solver& s) { (void)s; }

}  // namespace sordgpu
