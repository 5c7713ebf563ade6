// SORD oracle: CPU restatement of the reference Fortran solver.
//
// TEST INFRASTRUCTURE ONLY.  This program is the parity checker for the
// CUDA solver in coseis_b200/; it is never linked into, loaded by or called
// from the product.  Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / reference arm run it.
//
// It restates, routine by routine and in the same floating-point operation
// order, the serial (process_serial + thread_omp) build of SORD from
// shineusn/coseis:
//   sord/sord.f90:24-47            main program and step loop
//   sord/input_output.f90:21-591   sord.in parser, field_io engine, set_cube
//   sord/setup.f90:6-119           dimensions and index regions
//   sord/grid_generation.f90:6-200 mesh, gridnoise, rexpand, affine, vc
//   sord/material_model.f90:6-171  rho/vp/vs/gam -> lam, mu, yy; CFL
//   sord/boundary_pml.f90:7-82     PML coefficients and memories
//   sord/kinematic_source.f90      finite source files and injection
//   sord/dynamic_rupture.f90       rupture init and step
//   sord/material_resample.f90     mr, 1/vc, gam at nodes
//   sord/time_integration.f90      leapfrog + fault slip bookkeeping
//   sord/stress.f90                strain, PML g memory, Hooke, sources
//   sord/acceleration.f90          divergence, PML p memory, hourglass, BC
//   sord/diff_nc_op.f90, diff_cn_op.f90, hourglass_op.f90
//   sord/boundary_cond.f90, surf_normals.f90, utilities.f90, statistics.f90
//
// Build: oracle/build.py (FP32 -> _build/sord_oracle_f32, FP64 -> _f64).
// Run:   cd <dir containing sord.in> && sord_oracle_f32 [--threads N]
//        [--nt-limit K] [--w1-geometry]  -> writes the same output files as
//        sord.x.  --w1-geometry reproduces the reference's fault normals and
//        hypocentral radius from w1 (see the list of decisions below).
//
// Decisions where the reference is undefined or broken are the same ones the
// CUDA solver makes: the PML bounds from sord.in are converted so that exactly npml node
// and cell layers are damped on PML faces and none elsewhere (the reference
// reads its coefficient arrays one past the end and damps the boundary
// layer of non-PML faces); fault normals and the hypocentral radius use the
// node coordinates xx (the reference passes w1, which then holds cell
// centres); random_number() is replaced by a counter hash; fault-plane
// fields use index 1 in the fault-normal dimension for every op (the
// reference indexes them out of bounds); '.<' uses its own buffer value and
// '.>' on fault fields is not discarded; '@' cube ops test node coordinates
// for node fields and cell centres for cell fields.
//
// Compile with -ffp-contract=off so that no multiply-add is fused: the CUDA
// kernels are compiled with -fmad=false and follow the same operation order.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef SORD_REAL
#define SORD_REAL float
#endif
typedef SORD_REAL real;
#define R(x) ((real)(x))

struct SordStop : std::runtime_error {
    explicit SordStop(const std::string& s) : std::runtime_error(s) {}
};

// ---------------------------------------------------------------- arrays
// Column-major (j fastest) with 1-based indices, like the Fortran arrays.
struct V3 {  // 3-D view
    real* p = nullptr;
    int n[3] = {0, 0, 0};
    real& operator()(int j, int k, int l) const {
        return p[(size_t)(j - 1) + (size_t)n[0] * ((size_t)(k - 1) + (size_t)n[1] * (size_t)(l - 1))];
    }
    size_t size() const { return (size_t)n[0] * n[1] * n[2]; }
};
struct A3 {
    std::vector<real> d;
    int n[3] = {0, 0, 0};
    void alloc(int a, int b, int c) { n[0] = a; n[1] = b; n[2] = c; d.assign((size_t)a * b * c, R(0)); }
    V3 v() { V3 x; x.p = d.data(); x.n[0] = n[0]; x.n[1] = n[1]; x.n[2] = n[2]; return x; }
    real& operator()(int j, int k, int l) { return d[(size_t)(j - 1) + (size_t)n[0] * ((size_t)(k - 1) + (size_t)n[1] * (size_t)(l - 1))]; }
    size_t size() const { return d.size(); }
};
struct A4 {
    std::vector<real> d;
    int n[4] = {0, 0, 0, 0};
    void alloc(int a, int b, int c, int e) { n[0] = a; n[1] = b; n[2] = c; n[3] = e; d.assign((size_t)a * b * c * e, R(0)); }
    real& operator()(int j, int k, int l, int i) {
        return d[(size_t)(j - 1) + (size_t)n[0] * ((size_t)(k - 1) + (size_t)n[1] * ((size_t)(l - 1) + (size_t)n[2] * (size_t)(i - 1)))];
    }
    V3 c(int i) { V3 x; x.p = d.data() + (size_t)n[0] * n[1] * n[2] * (i - 1); x.n[0] = n[0]; x.n[1] = n[1]; x.n[2] = n[2]; return x; }
    bool empty() const { return d.empty(); }
};

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int imod(int a, int b) { int m = a % b; return m < 0 ? m + b : m; }  // Fortran modulo
static inline int ffloor(real x) { return (int)std::floor(x); }
static inline real fsign(real a, real b) { return b >= R(0) ? std::fabs(a) : -std::fabs(a); }

// integer power by binary exponentiation (Fortran real**integer)
static real powi(real x, int n) {
    if (n < 0) return R(1) / powi(x, -n);
    real r = R(1), b = x;
    bool first = true;
    while (n) {
        if (n & 1) { r = first ? b : r * b; first = false; }
        n >>= 1;
        if (n) b = b * b;
    }
    return r;
}
static long ipow(long x, int n) { long r = 1; for (int i = 0; i < n; i++) r *= x; return r; }

// Counter-based uniform [0,1) generator replacing Fortran random_number:
// value = f(call, linear index), identical in the CUDA solver.
static inline uint64_t splitmix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline real urand(uint64_t call, uint64_t idx) {
    uint64_t h = splitmix(splitmix(call * 0x100000001B3ull + 0x5151) ^ idx);
    return (real)((float)(h >> 40) * (1.0f / 16777216.0f));
}

// ---------------------------------------------------------------- io op
struct IoOp {
    std::string field, op, fname;
    char reg = 'n';
    int ii[4][3];  // ii[dim][0..2] = start(1-based), stop, step  (Fortran ii(1:3, dim))
    int nb = 1, ib = -1;
    real x1[3], x2[3], val = 0, tau = 0;
    std::vector<real> buff;  // n*nb
    int bufn = 0;
    bool open = false;  // file handle state (fh /= fio_file_null)
};

// ---------------------------------------------------------------- solver
struct Sord {
    // input parameters (sord/globals.f90:59-68)
    int bc1[3], bc2[3], debug, faultopening, i1pml[3], i2pml[3], itio, itstats, mpin, mpout;
    int n1expand[3], n2expand[3], npml, nproc3[3], nsource, nthread, ppml, shape_[4];
    real affine[9], delta[4], gam_max, gam_min, gridnoise, hourglass[2], hypocenter[3];
    real rcrit, rexpand, rho_max, rho_min, slipvector[3], svtol, tm0, trelax, vdamp;
    real vp_max, vp_min, vpml, vrup, vs_max, vs_min;
    std::string source, faultnormal;
    // misc
    real dt, dx[3], tm = 0;
    int it = 0, nt, ifn, irup;
    int nn[3], nm[3], nhalo[3], i1bc[3], i2bc[3], i1core[3], i2core[3], i1node[3], i2node[3];
    int i1cell[3], i2cell[3], nnoff[3];
    // arrays
    std::vector<real> dn1, dn2, dc1, dc2;  // size npml+1 (entry npml+1: zero damping)
    A4 p1, p2, p3, p4, p5, p6, g1, g2, g3, g4, g5, g6;
    A3 vc, mr, lam, mu, gam, yy, s1, s2;
    A4 xx, vv, uu, w1, w2;
    // fault
    A3 mus, mud, dc, co, area, rhypo, lamf, muf, sl, psv, trup, tarr, tn, ts, f1, f2;
    A4 nhat, t0, t1, t2, t3;
    // statistics module
    real amax = 0, vmax = 0, umax = 0, wmax = 0, samax = 0, svmax = 0, sumax = 0, slmax = 0;
    real tsmax = 0, tnmin = 0, tnmax = 0, tarrmax = 0, efric = 0, estrain = 0, moment = 0;
    // field io
    std::vector<IoOp> io_list;
    uint64_t rng_calls = 0;
    // finite source
    std::vector<int> src_nt;
    std::vector<real> src_xi[3], src_dt, src_t0, src_w1[3], src_w2[3], src_history;
    // stats buffers
    bool stats_init = true;
    int stats_j = 0;
    std::vector<real> maxl, suml;
    std::vector<long long> prof;
    long long timers[4] = {0, 0, 0, 0};
    bool stats_open[20];
    std::chrono::steady_clock::time_point clock0;
    int nt_limit = -1;
    int timed_from = -1;              // report the time of steps timed_from+1 .. nt
    // --w1-geometry: fault normals and the hypocentral radius from w1 as the
    // reference computes them (dynamic_rupture.f90:120,186,197-199): w1 then
    // holds cell centres with a zeroed halo (grid_generation.f90:127-132).
    // Off by default: node coordinates xx.
    bool w1_geometry = false;
    double timed_seconds = 0;

    long long clock_ticks() {
        return (long long)std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - clock0).count();
    }

    // ------------------------------------------------------------ parameters
    // sord/input_output.f90:21-98 (list-directed read of sord.in)
    void read_parameters(const std::string& path) {
        FILE* fp = fopen(path.c_str(), "rb");
        if (!fp) throw SordStop("cannot open " + path);
        std::string str;
        char buf[65536];
        size_t n;
        while ((n = fread(buf, 1, sizeof buf, fp)) > 0) str.append(buf, n);
        fclose(fp);
        size_t nl = str.find('\n');
        std::istringstream h(str.substr(0, nl));
        auto rd = [&](auto& x) { if (!(h >> x)) throw SordStop("Error reading sord.in parameters"); };
        int nfieldio;
        for (auto& a : affine) rd(a);
        for (auto& a : bc1) rd(a);
        for (auto& a : bc2) rd(a);
        rd(debug);
        for (auto& a : delta) rd(a);
        rd(faultnormal); rd(faultopening); rd(gam_max); rd(gam_min); rd(gridnoise);
        for (auto& a : hourglass) rd(a);
        for (auto& a : hypocenter) rd(a);
        for (auto& a : i1pml) rd(a);
        for (auto& a : i2pml) rd(a);
        rd(itio); rd(itstats); rd(mpin); rd(mpout);
        for (auto& a : n1expand) rd(a);
        for (auto& a : n2expand) rd(a);
        rd(nfieldio); rd(npml);
        for (auto& a : nproc3) rd(a);
        rd(nsource); rd(nthread); rd(ppml); rd(rcrit); rd(rexpand); rd(rho_max); rd(rho_min);
        for (auto& a : shape_) rd(a);
        for (auto& a : slipvector) rd(a);
        rd(source); rd(svtol); rd(tm0); rd(trelax); rd(vdamp); rd(vp_max); rd(vp_min); rd(vpml);
        rd(vrup); rd(vs_max); rd(vs_min);
        if (faultnormal.size() > 2) faultnormal = faultnormal.substr(0, 2);  // character(2)
        // i1pml/i2pml arrive as the 0-based Python bounds [i1, i2) of the
        // non-PML region; the loops below treat them as the last near-side and
        // first far-side PML node (1-based).  input_output.f90:62 adds 1 to
        // i1pml only, which shifts both bounds one node inward (defect, see
        // header); the consistent conversion is i1pml = i1, i2pml = i2 + 1.
        for (int i = 0; i < 3; i++) i2pml[i] += 1;
        std::istringstream b(nl == std::string::npos ? std::string() : str.substr(nl + 1));
        io_list.resize(nfieldio);
        for (int j = 0; j < nfieldio; j++) {
            IoOp& io = io_list[j];
            std::string reg;
            if (!(b >> io.field >> reg)) throw SordStop("Error reading sord.in field i/o");
            io.reg = reg[0];
            for (int d = 0; d < 4; d++)
                for (int c = 0; c < 3; c++) b >> io.ii[d][c];
            b >> io.nb;
            for (auto& a : io.x1) b >> a;
            for (auto& a : io.x2) b >> a;
            b >> io.val >> io.tau >> io.op >> io.fname;
            if (!b) throw SordStop("Error reading sord.in field i/o");
            if (io.field.size() > 4) io.field = io.field.substr(0, 4);
            io.ib = -1;
            for (int d = 0; d < 4; d++) io.ii[d][0] += 1;
        }
    }

    // ------------------------------------------------------------ setup
    // sord/setup.f90:6-84 (serial: ip3 = 0)
    void setup_dimensions() {
        for (int i = 0; i < 3; i++) { dx[i] = delta[i]; nn[i] = shape_[i]; }
        dt = delta[3];
        nt = imax(shape_[3], 0);
        if (nt_limit >= 0) nt = imin(nt, nt_limit);
        char c = faultnormal.size() > 1 ? faultnormal[1] : ' ';
        switch (c) {
            case 'o': ifn = 0; break;
            case 'x': ifn = 1; break;
            case 'y': ifn = 2; break;
            case 'z': ifn = 3; break;
            default: throw SordStop("Error in faultnormal");
        }
        if (nproc3[0] * nproc3[1] * nproc3[2] != 1) throw SordStop("MPI build required for multiprocessing");
        int nl3[3];
        for (int i = 0; i < 3; i++) {
            nl3[i] = (nn[i] - 1) / nproc3[i] + 1;
            nhalo[i] = 1;
        }
        if (ifn) nhalo[ifn - 1] = 2;
        for (int i = 0; i < 3; i++) {
            nl3[i] = imax(nl3[i], nhalo[i]);
            nnoff[i] = -nhalo[i];
            int nl = imin(nl3[i], nn[i] - nnoff[i] - nhalo[i]);
            nm[i] = nl + 2 * nhalo[i];
            i1bc[i] = 1 - nnoff[i];
            i2bc[i] = nn[i] - nnoff[i];
            i1core[i] = 1 + nhalo[i];
            i2core[i] = nm[i] - nhalo[i];
            i1node[i] = imax(i1bc[i], 2);
            i2node[i] = imin(i2bc[i], nm[i] - 1);
            i1cell[i] = imax(i1bc[i], 1);
            i2cell[i] = imin(i2bc[i] - 1, nm[i] - 1);
            i1pml[i] -= nnoff[i];
            i2pml[i] -= nnoff[i];
        }
        irup = 0;
        if (ifn) {
            irup = ffloor(hypocenter[ifn - 1] + R(0.000001)) - nnoff[ifn - 1] + 1;
            if (irup + 1 < i1core[ifn - 1] || irup > i2core[ifn - 1]) ifn = 0;
        }
    }

    // sord/arrays.f90:6-34
    void allocate_arrays() {
        int j = nm[0], k = nm[1], l = nm[2];
        xx.alloc(j, k, l, 3); vv.alloc(j, k, l, 3); uu.alloc(j, k, l, 3);
        w1.alloc(j, k, l, 3); w2.alloc(j, k, l, 3);
        vc.alloc(j, k, l); mr.alloc(j, k, l); lam.alloc(j, k, l); mu.alloc(j, k, l);
        gam.alloc(j, k, l); yy.alloc(j, k, l); s1.alloc(j, k, l); s2.alloc(j, k, l);
    }

    // ------------------------------------------------------------ utilities
    // sord/utilities.f90:79-100
    void average(V3 f2_, V3 f1_, const int* a1, const int* a2, int d) {
        for (int i = 0; i < 3; i++)
            if (a1[i] < 1 || a2[i] > f1_.n[i]) throw SordStop("error in average");
#pragma omp parallel for schedule(static)
        for (int l = a1[2]; l <= a2[2]; l++)
            for (int k = a1[1]; k <= a2[1]; k++)
                for (int j = a1[0]; j <= a2[0]; j++)
                    f2_(j, k, l) = R(0.125) *
                        (f1_(j, k, l) + f1_(j + d, k + d, l + d) + f1_(j, k + d, l + d) + f1_(j + d, k, l) +
                         f1_(j + d, k, l + d) + f1_(j, k + d, l) + f1_(j + d, k + d, l) + f1_(j, k, l + d));
        set_halo(f2_, R(0), a1, a2);
    }
    // sord/utilities.f90:103-117
    static void set_halo(V3 f, real r, const int* a1, const int* a2) {
        int i3[3], i4[3];
        for (int i = 0; i < 3; i++) { i3[i] = imin(a1[i], f.n[i] + 1); i4[i] = imax(a2[i], 0); }
        for (int l = 1; l <= f.n[2]; l++)
            for (int k = 1; k <= f.n[1]; k++)
                for (int j = 1; j <= f.n[0]; j++) {
                    bool h = (f.n[0] > 1 && (j < i3[0] || j > i4[0])) || (f.n[1] > 1 && (k < i3[1] || k > i4[1])) ||
                             (f.n[2] > 1 && (l < i3[2] || l > i4[2]));
                    if (h) f(j, k, l) = r;
                }
    }
    static void rinvert(V3 f) {
        size_t n = f.size();
        for (size_t i = 0; i < n; i++)
            if (f.p[i] != R(0)) f.p[i] = R(1) / f.p[i];
    }
    static void rlimits(V3 f, real fmin, real fmax) {
        size_t n = f.size();
        if (fmin > 0 && fmax > 0) { for (size_t i = 0; i < n; i++) f.p[i] = std::max(std::min(f.p[i], fmax), fmin); }
        else if (fmin > 0) { for (size_t i = 0; i < n; i++) f.p[i] = std::max(f.p[i], fmin); }
        else if (fmax > 0) { for (size_t i = 0; i < n; i++) f.p[i] = std::min(f.p[i], fmax); }
    }
    // sord/utilities.f90:120-139
    void vector_norm(V3 f, A4& w, const int* a1, const int* a2, const int* di) {
        for (int i = 0; i < 3; i++)
            if (a1[i] < 1 || a2[i] > f.n[i]) throw SordStop("error in vector_norm");
        V3 w_1 = w.c(1), w_2 = w.c(2), w_3 = w.c(3);
#pragma omp parallel for schedule(static)
        for (int l = a1[2]; l <= a2[2]; l += di[2])
            for (int k = a1[1]; k <= a2[1]; k += di[1])
                for (int j = a1[0]; j <= a2[0]; j += di[0])
                    f(j, k, l) = w_1(j, k, l) * w_1(j, k, l) + w_2(j, k, l) * w_2(j, k, l) + w_3(j, k, l) * w_3(j, k, l);
    }
    // sord/utilities.f90:142-165
    void tensor_norm(V3 f, A4& a, A4& b, const int* a1, const int* a2, const int* di) {
        for (int i = 0; i < 3; i++)
            if (a1[i] < 1 || a2[i] > f.n[i]) throw SordStop("error in tensor_norm");
        V3 a_1 = a.c(1), a_2 = a.c(2), a_3 = a.c(3), b_1 = b.c(1), b_2 = b.c(2), b_3 = b.c(3);
#pragma omp parallel for schedule(static)
        for (int l = a1[2]; l <= a2[2]; l += di[2])
            for (int k = a1[1]; k <= a2[1]; k += di[1])
                for (int j = a1[0]; j <= a2[0]; j += di[0])
                    f(j, k, l) = (a_1(j, k, l) * a_1(j, k, l) + a_2(j, k, l) * a_2(j, k, l) + a_3(j, k, l) * a_3(j, k, l)) +
                                 R(2) * (b_1(j, k, l) * b_1(j, k, l) + b_2(j, k, l) * b_2(j, k, l) + b_3(j, k, l) * b_3(j, k, l));
    }
    // sord/utilities.f90:168-220
    static void interpolate(V3 f, const int* a3, const int* a4, const int* di) {
        int i1[3], i2[3];
        for (int i = 0; i < 3; i++) {
            i1[i] = a3[i]; i2[i] = a4[i];
            if (i1[i] < 1) i1[i] = i1[i] + (-i1[i] / di[i] + 1) * di[i];
            if (i2[i] > f.n[i]) i2[i] = i1[i] + (f.n[i] - i1[i]) / di[i] * di[i];
        }
        int d = di[0];
        for (int i = 1; i <= d - 1; i++) {
            real h1 = R(1) / R(d) * R(i), h2 = R(1) / R(d) * R(d - i);
            for (int l = i1[2]; l <= i2[2]; l += di[2])
                for (int k = i1[1]; k <= i2[1]; k += di[1])
                    for (int j = i1[0]; j <= i2[0] - d; j += d) f(j + i, k, l) = h1 * f(j, k, l) + h2 * f(j + d, k, l);
        }
        d = di[1];
        for (int i = 1; i <= d - 1; i++) {
            real h1 = R(1) / R(d) * R(i), h2 = R(1) / R(d) * R(d - i);
            for (int l = i1[2]; l <= i2[2]; l += di[0])
                for (int k = i1[1]; k <= i2[1] - d; k += d)
                    for (int j = i1[0]; j <= i2[0]; j++) f(j, k + i, l) = h1 * f(j, k, l) + h2 * f(j, k + d, l);
        }
        d = di[2];
        for (int i = 1; i <= d - 1; i++) {
            real h1 = R(1) / R(d) * R(i), h2 = R(1) / R(d) * R(d - i);
            for (int l = i1[2]; l <= i2[2] - d; l += d)
                for (int k = i1[1]; k <= i2[1]; k++)
                    for (int j = i1[0]; j <= i2[0]; j++) f(j, k, l + i) = h1 * f(j, k, l) + h2 * f(j, k, l + d);
        }
    }

    // sord/utilities.f90:223-281
    static real time_function(const std::string& pulse, real t, real dt_, real tau) {
        const real pi = R(3.14159265);
        real f = 0, a, b;
        if (pulse == "const") f = 1;
        else if (pulse == "delta") { if (std::fabs(t) < R(0.25) * dt_) f = R(1) / dt_; }
        else if (pulse == "step" || pulse == "integral_delta") {
            if (std::fabs(t) < R(0.25) * dt_) f = R(0.5);
            else if (t >= R(0.25) * dt_) f = 1;
        } else if (pulse == "brune") {
            if (R(0) < t) { a = R(1) / tau; f = std::exp(-a * t) * a * a * t; }
        } else if (pulse == "integral_brune") {
            if (R(0) < t) { a = R(1) / tau; f = R(1) - std::exp(-a * t) * (a * t + R(1)); }
        } else if (pulse == "hann") {
            b = pi * tau;
            if (-b < t && t < b) { a = R(1) / tau; f = R(0.5) / pi * a * (R(1) + std::cos(a * t)); }
        } else if (pulse == "integral_hann") {
            b = pi * tau;
            if (-b < t && t < b) { a = R(1) / tau; f = R(0.5) + R(0.5) / pi * (a * t + std::sin(a * t)); }
            else if (R(0) < t) f = 1;
        } else if (pulse == "gaussian" || pulse == "integral_ricker1") {
            a = R(0.5) / (tau * tau); b = std::sqrt(a / pi); f = std::exp(-a * t * t) * b;
        } else if (pulse == "ricker1" || pulse == "integral_ricker2") {
            a = R(0.5) / (tau * tau); b = std::sqrt(a / pi) * R(2) * a; f = -std::exp(-a * t * t) * b * t;
        } else if (pulse == "ricker2") {
            a = R(0.5) / (tau * tau); b = std::sqrt(a / pi) * R(4) * a; f = std::exp(-a * t * t) * b * (a * t * t - R(0.5));
        } else throw SordStop("invalid time func: " + pulse);
        return f;
    }

    // ------------------------------------------------------------ operators
    // sord/diff_nc_op.f90:6-73
    void diff_nc(V3 df, A4& f, int i, int a, const int* i1, const int* i2, A4& x) {
        if (i1[0] > i2[0] || i1[1] > i2[1] || i1[2] > i2[2]) return;
        real h = fsign(R(1) / R(12), dx[0] * dx[1] * dx[2]);
        int b = imod(a, 3) + 1, c = imod(a + 1, 3) + 1;
        V3 F = f.c(i), B = x.c(b), C = x.c(c);
#pragma omp parallel for schedule(static)
        for (int l = i1[2]; l <= i2[2]; l++)
            for (int k = i1[1]; k <= i2[1]; k++)
                for (int j = i1[0]; j <= i2[0]; j++) {
                    real d = h * F(j, k, l) *
                        ((B(j, k + 1, l + 1) - B(j + 1, k, l)) * (C(j, k + 1, l) - C(j, k, l + 1)) + B(j + 1, k, l) * (C(j + 1, k, l + 1) - C(j + 1, k + 1, l)) +
                         (B(j + 1, k, l + 1) - B(j, k + 1, l)) * (C(j, k, l + 1) - C(j + 1, k, l)) + B(j, k + 1, l) * (C(j + 1, k + 1, l) - C(j, k + 1, l + 1)) +
                         (B(j + 1, k + 1, l) - B(j, k, l + 1)) * (C(j + 1, k, l) - C(j, k + 1, l)) + B(j, k, l + 1) * (C(j, k + 1, l + 1) - C(j + 1, k, l + 1)));
                    d = d + h * F(j + 1, k, l) *
                        ((B(j + 1, k + 1, l + 1) - B(j, k, l)) * (C(j + 1, k, l + 1) - C(j + 1, k + 1, l)) + B(j, k, l) * (C(j, k + 1, l) - C(j, k, l + 1)) +
                         (B(j, k + 1, l) - B(j + 1, k, l + 1)) * (C(j + 1, k + 1, l) - C(j, k, l)) + B(j + 1, k, l + 1) * (C(j, k, l + 1) - C(j + 1, k + 1, l + 1)) +
                         (B(j, k, l + 1) - B(j + 1, k + 1, l)) * (C(j, k, l) - C(j + 1, k, l + 1)) + B(j + 1, k + 1, l) * (C(j + 1, k + 1, l + 1) - C(j, k + 1, l)));
                    d = d + h * F(j, k + 1, l) *
                        ((B(j + 1, k + 1, l + 1) - B(j, k, l)) * (C(j + 1, k + 1, l) - C(j, k + 1, l + 1)) + B(j, k, l) * (C(j, k, l + 1) - C(j + 1, k, l)) +
                         (B(j + 1, k, l) - B(j, k + 1, l + 1)) * (C(j, k, l) - C(j + 1, k + 1, l)) + B(j, k + 1, l + 1) * (C(j + 1, k + 1, l + 1) - C(j, k, l + 1)) +
                         (B(j, k, l + 1) - B(j + 1, k + 1, l)) * (C(j, k + 1, l + 1) - C(j, k, l)) + B(j + 1, k + 1, l) * (C(j + 1, k, l) - C(j + 1, k + 1, l + 1)));
                    d = d + h * F(j + 1, k + 1, l) *
                        ((B(j, k, l) - B(j + 1, k + 1, l + 1)) * (C(j, k + 1, l) - C(j + 1, k, l)) + B(j + 1, k + 1, l + 1) * (C(j + 1, k, l + 1) - C(j, k + 1, l + 1)) +
                         (B(j, k + 1, l + 1) - B(j + 1, k, l)) * (C(j + 1, k + 1, l + 1) - C(j, k + 1, l)) + B(j + 1, k, l) * (C(j, k, l) - C(j + 1, k, l + 1)) +
                         (B(j + 1, k, l + 1) - B(j, k + 1, l)) * (C(j + 1, k, l) - C(j + 1, k + 1, l + 1)) + B(j, k + 1, l) * (C(j, k + 1, l + 1) - C(j, k, l)));
                    d = d + h * F(j, k, l + 1) *
                        ((B(j + 1, k + 1, l + 1) - B(j, k, l)) * (C(j, k + 1, l + 1) - C(j + 1, k, l + 1)) + B(j, k, l) * (C(j + 1, k, l) - C(j, k + 1, l)) +
                         (B(j + 1, k, l) - B(j, k + 1, l + 1)) * (C(j + 1, k, l + 1) - C(j, k, l)) + B(j, k + 1, l + 1) * (C(j, k + 1, l) - C(j + 1, k + 1, l + 1)) +
                         (B(j, k + 1, l) - B(j + 1, k, l + 1)) * (C(j, k, l) - C(j, k + 1, l + 1)) + B(j + 1, k, l + 1) * (C(j + 1, k + 1, l + 1) - C(j + 1, k, l)));
                    d = d + h * F(j + 1, k, l + 1) *
                        ((B(j, k, l) - B(j + 1, k + 1, l + 1)) * (C(j + 1, k, l) - C(j, k, l + 1)) + B(j + 1, k + 1, l + 1) * (C(j, k + 1, l + 1) - C(j + 1, k + 1, l)) +
                         (B(j, k + 1, l + 1) - B(j + 1, k, l)) * (C(j, k, l + 1) - C(j + 1, k + 1, l + 1)) + B(j + 1, k, l) * (C(j + 1, k + 1, l) - C(j, k, l)) +
                         (B(j + 1, k + 1, l) - B(j, k, l + 1)) * (C(j + 1, k + 1, l + 1) - C(j + 1, k, l)) + B(j, k, l + 1) * (C(j, k, l) - C(j, k + 1, l + 1)));
                    d = d + h * F(j + 1, k + 1, l + 1) *
                        ((B(j + 1, k, l) - B(j, k + 1, l + 1)) * (C(j + 1, k + 1, l) - C(j + 1, k, l + 1)) + B(j, k + 1, l + 1) * (C(j, k, l + 1) - C(j, k + 1, l)) +
                         (B(j, k + 1, l) - B(j + 1, k, l + 1)) * (C(j, k + 1, l + 1) - C(j + 1, k + 1, l)) + B(j + 1, k, l + 1) * (C(j + 1, k, l) - C(j, k, l + 1)) +
                         (B(j, k, l + 1) - B(j + 1, k + 1, l)) * (C(j + 1, k, l + 1) - C(j, k + 1, l + 1)) + B(j + 1, k + 1, l) * (C(j, k + 1, l) - C(j + 1, k, l)));
                    d = d + h * F(j, k + 1, l + 1) *
                        ((B(j, k, l) - B(j + 1, k + 1, l + 1)) * (C(j, k, l + 1) - C(j, k + 1, l)) + B(j + 1, k + 1, l + 1) * (C(j + 1, k + 1, l) - C(j + 1, k, l + 1)) +
                         (B(j + 1, k, l + 1) - B(j, k + 1, l)) * (C(j + 1, k + 1, l + 1) - C(j, k, l + 1)) + B(j, k + 1, l) * (C(j, k, l) - C(j + 1, k + 1, l)) +
                         (B(j + 1, k + 1, l) - B(j, k, l + 1)) * (C(j, k + 1, l) - C(j + 1, k + 1, l + 1)) + B(j, k, l + 1) * (C(j + 1, k, l + 1) - C(j, k, l)));
                    df(j, k, l) = d;
                }
    }

    // sord/diff_cn_op.f90:6-73 (declaration clash of `b` at :10-11 resolved as `real :: h`)
    void diff_cn(V3 df, A4& f, int i, int a, const int* i1, const int* i2, A4& x) {
        if (i1[0] > i2[0] || i1[1] > i2[1] || i1[2] > i2[2]) return;
        real h = fsign(R(1) / R(12), dx[0] * dx[1] * dx[2]);
        int b = imod(a, 3) + 1, c = imod(a + 1, 3) + 1;
        V3 F = f.c(i), B = x.c(b), C = x.c(c);
#pragma omp parallel for schedule(static)
        for (int l = i1[2]; l <= i2[2]; l++)
            for (int k = i1[1]; k <= i2[1]; k++)
                for (int j = i1[0]; j <= i2[0]; j++) {
                    real d = h * F(j - 1, k - 1, l - 1) *
                        ((B(j - 1, k, l) - B(j, k - 1, l - 1)) * (C(j, k, l - 1) - C(j, k - 1, l)) + B(j - 1, k, l) * (C(j - 1, k, l - 1) - C(j - 1, k - 1, l)) +
                         (B(j, k - 1, l) - B(j - 1, k, l - 1)) * (C(j - 1, k, l) - C(j, k, l - 1)) + B(j, k - 1, l) * (C(j - 1, k - 1, l) - C(j, k - 1, l - 1)) +
                         (B(j, k, l - 1) - B(j - 1, k - 1, l)) * (C(j, k - 1, l) - C(j - 1, k, l)) + B(j, k, l - 1) * (C(j, k - 1, l - 1) - C(j - 1, k, l - 1)));
                    d = d + h * F(j, k - 1, l - 1) *
                        ((B(j + 1, k, l) - B(j, k - 1, l - 1)) * (C(j, k - 1, l) - C(j, k, l - 1)) + B(j + 1, k, l) * (C(j + 1, k - 1, l) - C(j + 1, k, l - 1)) +
                         (B(j, k - 1, l) - B(j + 1, k, l - 1)) * (C(j, k, l - 1) - C(j + 1, k, l)) + B(j, k - 1, l) * (C(j, k - 1, l - 1) - C(j + 1, k - 1, l)) +
                         (B(j, k, l - 1) - B(j + 1, k - 1, l)) * (C(j + 1, k, l) - C(j, k - 1, l)) + B(j, k, l - 1) * (C(j + 1, k, l - 1) - C(j, k - 1, l - 1)));
                    d = d + h * F(j - 1, k - 1, l) *
                        ((B(j, k, l + 1) - B(j - 1, k - 1, l)) * (C(j - 1, k, l) - C(j, k - 1, l)) + B(j, k, l + 1) * (C(j - 1, k, l + 1) - C(j, k - 1, l + 1)) +
                         (B(j - 1, k, l) - B(j, k - 1, l + 1)) * (C(j, k - 1, l) - C(j, k, l + 1)) + B(j - 1, k, l) * (C(j - 1, k - 1, l) - C(j - 1, k, l + 1)) +
                         (B(j, k - 1, l) - B(j - 1, k, l + 1)) * (C(j, k, l + 1) - C(j - 1, k, l)) + B(j, k - 1, l) * (C(j, k - 1, l + 1) - C(j - 1, k - 1, l)));
                    d = d + h * F(j, k - 1, l) *
                        ((B(j, k - 1, l) - B(j + 1, k, l + 1)) * (C(j + 1, k, l) - C(j, k, l + 1)) + B(j, k - 1, l) * (C(j + 1, k - 1, l) - C(j, k - 1, l + 1)) +
                         (B(j, k, l + 1) - B(j + 1, k - 1, l)) * (C(j, k - 1, l) - C(j + 1, k, l)) + B(j, k, l + 1) * (C(j, k - 1, l + 1) - C(j + 1, k, l + 1)) +
                         (B(j + 1, k, l) - B(j, k - 1, l + 1)) * (C(j, k, l + 1) - C(j, k - 1, l)) + B(j + 1, k, l) * (C(j + 1, k, l + 1) - C(j + 1, k - 1, l)));
                    d = d + h * F(j - 1, k, l - 1) *
                        ((B(j, k + 1, l) - B(j - 1, k, l - 1)) * (C(j, k, l - 1) - C(j - 1, k, l)) + B(j, k + 1, l) * (C(j, k + 1, l - 1) - C(j - 1, k + 1, l)) +
                         (B(j, k, l - 1) - B(j - 1, k + 1, l)) * (C(j - 1, k, l) - C(j, k + 1, l)) + B(j, k, l - 1) * (C(j - 1, k, l - 1) - C(j, k + 1, l - 1)) +
                         (B(j - 1, k, l) - B(j, k + 1, l - 1)) * (C(j, k + 1, l) - C(j, k, l - 1)) + B(j - 1, k, l) * (C(j - 1, k + 1, l) - C(j - 1, k, l - 1)));
                    d = d + h * F(j, k, l - 1) *
                        ((B(j, k, l - 1) - B(j + 1, k + 1, l)) * (C(j, k + 1, l) - C(j + 1, k, l)) + B(j, k, l - 1) * (C(j, k + 1, l - 1) - C(j + 1, k, l - 1)) +
                         (B(j + 1, k, l) - B(j, k + 1, l - 1)) * (C(j, k, l - 1) - C(j, k + 1, l)) + B(j + 1, k, l) * (C(j + 1, k, l - 1) - C(j + 1, k + 1, l)) +
                         (B(j, k + 1, l) - B(j + 1, k, l - 1)) * (C(j + 1, k, l) - C(j, k, l - 1)) + B(j, k + 1, l) * (C(j + 1, k + 1, l) - C(j, k + 1, l - 1)));
                    d = d + h * F(j - 1, k, l) *
                        ((B(j - 1, k, l) - B(j, k + 1, l + 1)) * (C(j, k, l + 1) - C(j, k + 1, l)) + B(j - 1, k, l) * (C(j - 1, k, l + 1) - C(j - 1, k + 1, l)) +
                         (B(j, k + 1, l) - B(j - 1, k, l + 1)) * (C(j - 1, k, l) - C(j, k, l + 1)) + B(j, k + 1, l) * (C(j - 1, k + 1, l) - C(j, k + 1, l + 1)) +
                         (B(j, k, l + 1) - B(j - 1, k + 1, l)) * (C(j, k + 1, l) - C(j - 1, k, l)) + B(j, k, l + 1) * (C(j, k + 1, l + 1) - C(j - 1, k, l + 1)));
                    d = d + h * F(j, k, l) *
                        ((B(j + 1, k, l) - B(j, k + 1, l + 1)) * (C(j, k + 1, l) - C(j, k, l + 1)) + B(j + 1, k, l) * (C(j + 1, k + 1, l) - C(j + 1, k, l + 1)) +
                         (B(j, k + 1, l) - B(j + 1, k, l + 1)) * (C(j, k, l + 1) - C(j + 1, k, l)) + B(j, k + 1, l) * (C(j, k + 1, l + 1) - C(j + 1, k + 1, l)) +
                         (B(j, k, l + 1) - B(j + 1, k + 1, l)) * (C(j + 1, k, l) - C(j, k + 1, l)) + B(j, k, l + 1) * (C(j + 1, k, l + 1) - C(j, k + 1, l + 1)));
                    df(j, k, l) = d;
                }
    }

    // sord/hourglass_op.f90:7-74
    static void hourglass_nc(V3 df, V3 f, int iq, const int* i1, const int* i2) {
        if (i1[0] > i2[0] || i1[1] > i2[1] || i1[2] > i2[2]) return;
#pragma omp parallel for schedule(static)
        for (int l = i1[2]; l <= i2[2]; l++)
            for (int k = i1[1]; k <= i2[1]; k++)
                for (int j = i1[0]; j <= i2[0]; j++) {
                    real r;
                    switch (iq) {
                        case 1: r = f(j, k, l) + f(j + 1, k + 1, l + 1) + f(j, k + 1, l + 1) + f(j + 1, k, l) - f(j + 1, k, l + 1) - f(j, k + 1, l) - f(j + 1, k + 1, l) - f(j, k, l + 1); break;
                        case 2: r = f(j, k, l) + f(j + 1, k + 1, l + 1) - f(j, k + 1, l + 1) - f(j + 1, k, l) + f(j + 1, k, l + 1) + f(j, k + 1, l) - f(j + 1, k + 1, l) - f(j, k, l + 1); break;
                        case 3: r = f(j, k, l) + f(j + 1, k + 1, l + 1) - f(j, k + 1, l + 1) - f(j + 1, k, l) - f(j + 1, k, l + 1) - f(j, k + 1, l) + f(j + 1, k + 1, l) + f(j, k, l + 1); break;
                        default: r = f(j, k, l) - f(j + 1, k + 1, l + 1) + f(j, k + 1, l + 1) - f(j + 1, k, l) + f(j + 1, k, l + 1) - f(j, k + 1, l) + f(j + 1, k + 1, l) - f(j, k, l + 1); break;
                    }
                    df(j, k, l) = r;
                }
    }
    // sord/hourglass_op.f90:79-146
    static void hourglass_cn(V3 df, V3 f, int iq, const int* i1, const int* i2) {
        if (i1[0] > i2[0] || i1[1] > i2[1] || i1[2] > i2[2]) return;
#pragma omp parallel for schedule(static)
        for (int l = i1[2]; l <= i2[2]; l++)
            for (int k = i1[1]; k <= i2[1]; k++)
                for (int j = i1[0]; j <= i2[0]; j++) {
                    real r;
                    switch (iq) {
                        case 1: r = f(j, k, l) + f(j - 1, k - 1, l - 1) + f(j, k - 1, l - 1) + f(j - 1, k, l) - f(j - 1, k, l - 1) - f(j, k - 1, l) - f(j - 1, k - 1, l) - f(j, k, l - 1); break;
                        case 2: r = f(j, k, l) + f(j - 1, k - 1, l - 1) - f(j, k - 1, l - 1) - f(j - 1, k, l) + f(j - 1, k, l - 1) + f(j, k - 1, l) - f(j - 1, k - 1, l) - f(j, k, l - 1); break;
                        case 3: r = f(j, k, l) + f(j - 1, k - 1, l - 1) - f(j, k - 1, l - 1) - f(j - 1, k, l) - f(j - 1, k, l - 1) - f(j, k - 1, l) + f(j - 1, k - 1, l) + f(j, k, l - 1); break;
                        default: r = f(j, k, l) - f(j - 1, k - 1, l - 1) + f(j, k - 1, l - 1) - f(j - 1, k, l) + f(j - 1, k, l - 1) - f(j, k - 1, l) + f(j - 1, k - 1, l) - f(j, k, l - 1); break;
                    }
                    df(j, k, l) = r;
                }
    }

    // sord/boundary_cond.f90:7-27
    static void scalar_bc(V3 f, const int* bc1_, const int* bc2_, const int* a1, const int* a2) {
        int b1[3], b2[3];
        for (int i = 0; i < 3; i++) {
            b1[i] = std::abs(bc1_[i] % 10); b2[i] = std::abs(bc2_[i] % 10);
            if (b1[i] == 4) b1[i] = 2;
            if (b2[i] == 4) b2[i] = 2;
            if (f.n[i] == 1 || a1[i] < 1 || a1[i] >= f.n[i]) b1[i] = 99;
            if (f.n[i] == 1 || a2[i] <= 1 || a2[i] > f.n[i]) b2[i] = 99;
        }
        int j1 = a1[0], k1 = a1[1], l1 = a1[2], j2 = a2[0], k2 = a2[1], l2 = a2[2];
        if (b1[0] == 2) for (int l = 1; l <= f.n[2]; l++) for (int k = 1; k <= f.n[1]; k++) f(j1, k, l) = f(j1 + 1, k, l);
        if (b1[1] == 2) for (int l = 1; l <= f.n[2]; l++) for (int j = 1; j <= f.n[0]; j++) f(j, k1, l) = f(j, k1 + 1, l);
        if (b1[2] == 2) for (int k = 1; k <= f.n[1]; k++) for (int j = 1; j <= f.n[0]; j++) f(j, k, l1) = f(j, k, l1 + 1);
        if (b2[0] == 2) for (int l = 1; l <= f.n[2]; l++) for (int k = 1; k <= f.n[1]; k++) f(j2, k, l) = f(j2 - 1, k, l);
        if (b2[1] == 2) for (int l = 1; l <= f.n[2]; l++) for (int j = 1; j <= f.n[0]; j++) f(j, k2, l) = f(j, k2 - 1, l);
        if (b2[2] == 2) for (int k = 1; k <= f.n[1]; k++) for (int j = 1; j <= f.n[0]; j++) f(j, k, l2) = f(j, k, l2 - 1);
    }

    // sord/boundary_cond.f90:30-115
    static void vector_bc(A4& f, const int* bc1_, const int* bc2_, const int* a1, const int* a2) {
        int nmm[3] = {f.n[0], f.n[1], f.n[2]};
        int b1[3], b2[3], sg1[3], sg2[3];
        for (int i = 0; i < 3; i++) {
            b1[i] = bc1_[i] % 10; b2[i] = bc2_[i] % 10;
            if (nmm[i] == 1 || a1[i] < 1 || a1[i] > nmm[i]) b1[i] = 99;
            if (nmm[i] == 1 || a2[i] < 1 || a2[i] > nmm[i]) b2[i] = 99;
        }
        // plane setters: dim d, index p, component c (1..3), value via lambda
        auto plane = [&](int d, int p, auto fn) {
            int lo[3] = {1, 1, 1}, hi[3] = {nmm[0], nmm[1], nmm[2]};
            lo[d] = hi[d] = p;
            for (int l = lo[2]; l <= hi[2]; l++)
                for (int k = lo[1]; k <= hi[1]; k++)
                    for (int j = lo[0]; j <= hi[0]; j++) fn(j, k, l);
        };
        const int* a[2] = {a1, a2};
        int* bb[2] = {b1, b2};
        // anti-mirror symmetry at the node: zero the two tangential components
        for (int s = 0; s < 2; s++)
            for (int d = 0; d < 3; d++)
                if (bb[s][d] == -1) {
                    int c1 = (d + 1) % 3 + 1, c2 = (d + 2) % 3 + 1;
                    plane(d, a[s][d], [&](int j, int k, int l) { f(j, k, l, c1) = 0; f(j, k, l, c2) = 0; });
                }
        // mirror symmetry at the node: zero the normal component
        for (int s = 0; s < 2; s++)
            for (int d = 0; d < 3; d++)
                if (bb[s][d] == 1) plane(d, a[s][d], [&](int j, int k, int l) { f(j, k, l, d + 1) = 0; });
        // rigid
        for (int s = 0; s < 2; s++)
            for (int d = 0; d < 3; d++)
                if (bb[s][d] == 3) plane(d, a[s][d], [&](int j, int k, int l) { for (int c = 1; c <= 3; c++) f(j, k, l, c) = 0; });
        for (int i = 0; i < 3; i++) {
            if (a1[i] >= nmm[i]) b1[i] = 99;
            if (a2[i] <= 1) b2[i] = 99;
        }
        // continue
        for (int d = 0; d < 3; d++)
            if (b1[d] == 4) plane(d, a1[d], [&](int j, int k, int l) {
                int o[3] = {0, 0, 0}; o[d] = 1;
                for (int c = 1; c <= 3; c++) f(j, k, l, c) = f(j + o[0], k + o[1], l + o[2], c);
            });
        for (int d = 0; d < 3; d++)
            if (b2[d] == 4) plane(d, a2[d], [&](int j, int k, int l) {
                int o[3] = {0, 0, 0}; o[d] = 1;
                for (int c = 1; c <= 3; c++) f(j, k, l, c) = f(j - o[0], k - o[1], l - o[2], c);
            });
        // symmetry at the cell
        for (int i = 0; i < 3; i++) {
            b1[i] = std::abs(b1[i]); b2[i] = std::abs(b2[i]);
            sg1[i] = bc1_[i] >= 0 ? 1 : -1; sg2[i] = bc2_[i] >= 0 ? 1 : -1;
        }
        for (int d = 0; d < 3; d++)
            if (b1[d] == 2) plane(d, a1[d], [&](int j, int k, int l) {
                int o[3] = {0, 0, 0}; o[d] = 1;
                for (int c = 1; c <= 3; c++) {
                    real s = (real)(c == d + 1 ? -sg1[d] : sg1[d]);
                    f(j, k, l, c) = s * f(j + o[0], k + o[1], l + o[2], c);
                }
            });
        for (int d = 0; d < 3; d++)
            if (b2[d] == 2) plane(d, a2[d], [&](int j, int k, int l) {
                int o[3] = {0, 0, 0}; o[d] = 1;
                for (int c = 1; c <= 3; c++) {
                    real s = (real)(c == d + 1 ? -sg2[d] : sg2[d]);
                    f(j, k, l, c) = s * f(j - o[0], k - o[1], l - o[2], c);
                }
            });
    }

    // sord/surf_normals.f90:53-128
    void node_normals(A4& nh, A4& x, const int* i1, const int* i2, int ihat) {
        std::fill(nh.d.begin(), nh.d.end(), R(0));
        real h = fsign(R(1) / R(12), dx[0] * dx[1] * dx[2]);
        for (int a = 1; a <= 3; a++) {
            int b = imod(a, 3) + 1, c = imod(a + 1, 3) + 1;
            V3 B = x.c(b), C = x.c(c);
            if (ihat == 1) {
                int j = i1[0];
                for (int l = i1[2]; l <= i2[2]; l++)
                    for (int k = i1[1]; k <= i2[1]; k++)
                        nh(1, k, l, a) = h * (B(j, k + 1, l) * (C(j, k, l + 1) + C(j, k + 1, l + 1) - C(j, k, l - 1) - C(j, k + 1, l - 1)) +
                                              B(j, k - 1, l) * (C(j, k, l - 1) + C(j, k - 1, l - 1) - C(j, k, l + 1) - C(j, k - 1, l + 1)) +
                                              B(j, k, l + 1) * (C(j, k - 1, l) + C(j, k - 1, l + 1) - C(j, k + 1, l) - C(j, k + 1, l + 1)) +
                                              B(j, k, l - 1) * (C(j, k + 1, l) + C(j, k + 1, l - 1) - C(j, k - 1, l) - C(j, k - 1, l - 1)) +
                                              B(j, k + 1, l + 1) * (C(j, k, l + 1) - C(j, k + 1, l)) + B(j, k - 1, l - 1) * (C(j, k, l - 1) - C(j, k - 1, l)) +
                                              B(j, k - 1, l + 1) * (C(j, k - 1, l) - C(j, k, l + 1)) + B(j, k + 1, l - 1) * (C(j, k + 1, l) - C(j, k, l - 1)));
            } else if (ihat == 2) {
                int k = i1[1];
                for (int l = i1[2]; l <= i2[2]; l++)
                    for (int j = i1[0]; j <= i2[0]; j++)
                        nh(j, 1, l, a) = h * (B(j, k, l + 1) * (C(j + 1, k, l) + C(j + 1, k, l + 1) - C(j - 1, k, l) - C(j - 1, k, l + 1)) +
                                              B(j, k, l - 1) * (C(j - 1, k, l) + C(j - 1, k, l - 1) - C(j + 1, k, l) - C(j + 1, k, l - 1)) +
                                              B(j + 1, k, l) * (C(j, k, l - 1) + C(j + 1, k, l - 1) - C(j, k, l + 1) - C(j + 1, k, l + 1)) +
                                              B(j - 1, k, l) * (C(j, k, l + 1) + C(j - 1, k, l + 1) - C(j, k, l - 1) - C(j - 1, k, l - 1)) +
                                              B(j + 1, k, l + 1) * (C(j + 1, k, l) - C(j, k, l + 1)) + B(j - 1, k, l - 1) * (C(j - 1, k, l) - C(j, k, l - 1)) +
                                              B(j + 1, k, l - 1) * (C(j, k, l - 1) - C(j + 1, k, l)) + B(j - 1, k, l + 1) * (C(j, k, l + 1) - C(j - 1, k, l)));
            } else if (ihat == 3) {
                int l = i1[2];
                for (int k = i1[1]; k <= i2[1]; k++)
                    for (int j = i1[0]; j <= i2[0]; j++)
                        nh(j, k, 1, a) = h * (B(j + 1, k, l) * (C(j, k + 1, l) + C(j + 1, k + 1, l) - C(j, k - 1, l) - C(j + 1, k - 1, l)) +
                                              B(j - 1, k, l) * (C(j, k - 1, l) + C(j - 1, k - 1, l) - C(j, k + 1, l) - C(j - 1, k + 1, l)) +
                                              B(j, k + 1, l) * (C(j - 1, k, l) + C(j - 1, k + 1, l) - C(j + 1, k, l) - C(j + 1, k + 1, l)) +
                                              B(j, k - 1, l) * (C(j + 1, k, l) + C(j + 1, k - 1, l) - C(j - 1, k, l) - C(j - 1, k - 1, l)) +
                                              B(j + 1, k + 1, l) * (C(j, k + 1, l) - C(j + 1, k, l)) + B(j - 1, k - 1, l) * (C(j, k - 1, l) - C(j - 1, k, l)) +
                                              B(j - 1, k + 1, l) * (C(j - 1, k, l) - C(j, k + 1, l)) + B(j + 1, k - 1, l) * (C(j + 1, k, l) - C(j, k - 1, l)));
            } else throw SordStop("error: surfnormal");
        }
    }

    // ------------------------------------------------------------ file i/o
    // sord/fortran_io.f90:51-92: direct-access records of n values, record o+1..o+n
    void frio2(IoOp* io, bool& opened, real* f2, int recl, int nrec, char mode, const std::string& filename, int m, int o) {
        std::vector<float> tmp;
        const size_t rb = (size_t)recl * sizeof(real);
        FILE* fp;
        if (mode == 'r') {
            fp = fopen(filename.c_str(), "rb");
            if (!fp) throw SordStop("cannot open " + filename);
            fseek(fp, (long)(rb * (size_t)o), SEEK_SET);
            size_t got = fread(f2, sizeof(real), (size_t)recl * nrec, fp);
            fclose(fp);
            if (got != (size_t)recl * nrec) throw SordStop("short read " + filename);
        } else {
            if (!opened && o == 0) {
                fp = fopen(filename.c_str(), "rb");
                if (fp) { fclose(fp); throw SordStop("file exists: " + filename); }
                fp = fopen(filename.c_str(), "wb");
            } else {
                fp = fopen(filename.c_str(), "r+b");
            }
            if (!fp) throw SordStop("cannot open " + filename);
            opened = true;
            fseek(fp, (long)(rb * (size_t)o), SEEK_SET);
            fwrite(f2, sizeof(real), (size_t)recl * nrec, fp);
            fclose(fp);
        }
        if (o + nrec == m) opened = false;
        (void)io;
    }

    // ------------------------------------------------------------ field io
    // sord/input_output.f90:103-542
    void field_io(const char* passes, const char* field, V3 f) {
        for (const char* pp = passes; *pp; pp++) {
            char pass = *pp;
            for (size_t iloop = 0; iloop < io_list.size(); iloop++) {
                IoOp& io = io_list[iloop];
                int it1 = io.ii[3][0], it2 = io.ii[3][1], dit = io.ii[3][2];
                if (it > it2) continue;
                if (io.op[0] == '#') continue;
                if (it < it1) continue;
                if (imod(it - it1, dit) != 0) continue;
                if (io.field != field) continue;
                char op2 = io.op.size() > 1 ? io.op[1] : ' ';
                if (pass == '<' && op2 == '>') continue;
                if (pass == '>' && op2 != '>') continue;
                field_io_op(io, f, field);
            }
        }
    }

    void field_io_op(IoOp& io, V3 f, const char* field) {
        int i1[3], i2[3], i3[3], i4[3], di[3], m[4], n[4], o[4];
        real xi[3];
        int it1 = io.ii[3][0], it2 = io.ii[3][1], dit = io.ii[3][2];
        char op2 = io.op.size() > 1 ? io.op[1] : ' ';
        for (int i = 0; i < 3; i++) {
            if (io.reg == 'n') { i3[i] = i1node[i]; i4[i] = i2node[i]; xi[i] = io.x1[i] - R(nnoff[i]) + R(1); }
            else { i3[i] = i1cell[i]; i4[i] = i2cell[i]; xi[i] = io.x1[i] - R(nnoff[i]) + R(0.5); }
        }
        if (io.op[0] == '.') {
            for (int i = 0; i < 3; i++) { i1[i] = imax(i3[i], ffloor(xi[i])); i2[i] = imin(i4[i], ffloor(xi[i]) + 1); di[i] = 1; }
        } else {
            for (int i = 0; i < 3; i++) {
                i1[i] = io.ii[i][0] - nnoff[i]; i2[i] = io.ii[i][1] - nnoff[i]; di[i] = io.ii[i][2];
                if (i1[i] < i3[i]) i1[i] = i1[i] + ((i3[i] - i1[i] - 1) / di[i] + 1) * di[i];
                if (i2[i] > i4[i]) i2[i] = i1[i] + (i4[i] - i1[i]) / di[i] * di[i];
            }
        }
        // fault-plane arrays: the fault-normal dimension has extent 1 (defect fix,
        // see header): every op addresses index 1 there with weight 1.
        bool plane[3];
        for (int i = 0; i < 3; i++) plane[i] = (f.n[i] == 1 && nm[i] != 1);
        // non-disk input
        if (op2 != '<' && op2 != '>') {
            for (int i = 0; i < 3; i++)
                if (i2[i] < i1[i]) { io.op = "#"; return; }
            for (int i = 0; i < 3; i++)
                if (plane[i]) { i1[i] = i2[i] = 1; di[i] = 1; }
            real val = io.val * time_function(io.fname, tm, dt, io.tau);
            const std::string& op = io.op;
            if (op == ".") {
                for (int l = i1[2]; l <= i2[2]; l++)
                    for (int k = i1[1]; k <= i2[1]; k++)
                        for (int j = i1[0]; j <= i2[0]; j++) {
                            real r = wgt(xi[0], j, plane[0]) * wgt(xi[1], k, plane[1]) * wgt(xi[2], l, plane[2]);
                            f(j, k, l) = f(j, k, l) + val * r;
                        }
            } else if (op == "=" || op == "+" || op == "*" || op == "=~" || op == "+~" || op == "*~") {
                bool rnd = op.size() > 1;
                if (rnd) {  // random_number(s1): counter hash over the whole s1 array
                    uint64_t call = rng_calls++;
                    for (size_t q = 0; q < s1.size(); q++) s1.d[q] = urand(call, q);
                }
                for (int l = i1[2]; l <= i2[2]; l += di[2])
                    for (int k = i1[1]; k <= i2[1]; k += di[1])
                        for (int j = i1[0]; j <= i2[0]; j += di[0]) {
                            real& F = f(j, k, l);
                            if (op == "=") F = val;
                            else if (op == "+") F = F + val;
                            else if (op == "*") F = F * val;
                            else {
                                real r = s1(j, k, l);
                                if (op == "=~") F = val * r;
                                else if (op == "+~") F = F + val * r;
                                else F = F * val * r;
                            }
                        }
            } else if (op == "=@" || op == "+@" || op == "*@") {
                set_cube(f, io, i1, i2, di, val);
            } else {
                throw SordStop("bad i/o mode '" + op + "'");
            }
            if (io.reg == 'n') scalar_bc(f, bc1, bc2, i1bc, i2bc);
            if (io.reg == 'c') { int t[3] = {i2bc[0] - 1, i2bc[1] - 1, i2bc[2] - 1}; scalar_bc(f, bc1, bc2, i1bc, t); }
            return;
        }
        // spatial indices for disk i/o
        if (io.op[0] == '.') {
            for (int i = 0; i < 4; i++) { m[i] = 1; n[i] = 1; o[i] = 0; }
        } else {
            for (int i = 0; i < 3; i++) {
                i1[i] = io.ii[i][0] - nnoff[i]; i2[i] = io.ii[i][1] - nnoff[i]; di[i] = io.ii[i][2];
                i3[i] = i1[i]; i4[i] = i2[i];
                if (i1[i] < i1core[i]) i1[i] = i1[i] + ((i1core[i] - i1[i] - 1) / di[i] + 1) * di[i];
                if (i2[i] > i2core[i]) i2[i] = i1[i] + (i2core[i] - i1[i]) / di[i] * di[i];
                m[i] = (i4[i] - i3[i]) / di[i] + 1;
                n[i] = (i2[i] - i1[i]) / di[i] + 1;
                o[i] = (i1[i] - i3[i]) / di[i];
                n[i] = imax(n[i], 0);
            }
            m[3] = n[3] = 1; o[3] = 0;
        }
        // array dimensionality
        for (int i = 0; i < 3; i++)
            if (f.n[i] == 1) {
                if (n[i] < 1) { io.op = "#"; return; }
                i1[i] = 1; i2[i] = 1; m[i] = 1; n[i] = 1; o[i] = 0;
            }
        // disk input
        if (op2 == '<') {
            if (io.op != ".<")
                for (int i = 0; i < 3; i++)
                    if (m[i] == 1) { i1[i] = 1; i2[i] = 1; n[i] = 1; o[i] = 0; }
            int nsp = n[0] * n[1] * n[2];
            if (io.ib < 0) {
                io.bufn = imax(nsp, 0);
                io.buff.assign((size_t)io.bufn * io.nb, R(0));
                io.ib = io.nb;
                io.open = false;
            }
            if (io.ib == io.nb) {
                n[3] = imin(io.nb, (it2 - it) / dit + 1);
                m[3] = (it2 - it1) / dit + 1;
                o[3] = (it - it1) / dit;
                std::string filename = io.fname;
                if ((n[0] != m[0] || n[1] != m[1] || n[2] != m[2]) && mpin == 0) filename += "-000000";
                io.ib = 0;
                if (n[0] < 1 || n[1] < 1 || n[2] < 1 || n[3] < 1) { io.buff.clear(); io.op = "#"; return; }
                read_subarray(io, filename, m, n, o);
                for (size_t q = 0; q < (size_t)nsp * n[3]; q++) {
                    real v = io.buff[q];
                    if (v != v || v > std::numeric_limits<real>::max())
                        throw SordStop("NaN/Inf in " + io.fname);
                }
            }
            io.ib = io.ib + 1;
            real* buf = io.buff.data() + (size_t)io.bufn * (io.ib - 1);
            if (io.op == ".<") {
                for (int l = i1[2]; l <= i2[2]; l++)
                    for (int k = i1[1]; k <= i2[1]; k++)
                        for (int j = i1[0]; j <= i2[0]; j++) {
                            real r = wgt(xi[0], j, plane[0]) * wgt(xi[1], k, plane[1]) * wgt(xi[2], l, plane[2]);
                            f(j, k, l) = f(j, k, l) + r * buf[0];
                        }
            } else {
                // copy buffer to the scratch array s1 (the field's own shape)
                V3 S;
                std::vector<real> sp;
                if (f.n[0] == nm[0] && f.n[1] == nm[1] && f.n[2] == nm[2]) S = s1.v();
                else { sp.assign(f.size(), R(0)); S.p = sp.data(); for (int i = 0; i < 3; i++) S.n[i] = f.n[i]; }
                size_t q = 0;
                for (int l = i1[2]; l <= i2[2]; l += di[2])
                    for (int k = i1[1]; k <= i2[1]; k += di[1])
                        for (int j = i1[0]; j <= i2[0]; j += di[0]) S(j, k, l) = buf[q++];
                if (di[0] > 1 || di[1] > 1 || di[2] > 1) {
                    int a3[3], a4[3];
                    for (int i = 0; i < 3; i++) { a3[i] = io.ii[i][0] - nnoff[i]; a4[i] = io.ii[i][1] - nnoff[i]; }
                    interpolate(S, a3, a4, di);
                }
                if (m[0] == 1) { i2[0] = f.n[0]; for (int l = 1; l <= S.n[2]; l++) for (int k = 1; k <= S.n[1]; k++) for (int j = 2; j <= i2[0]; j++) S(j, k, l) = S(1, k, l); }
                if (m[1] == 1) { i2[1] = f.n[1]; for (int l = 1; l <= S.n[2]; l++) for (int k = 2; k <= i2[1]; k++) for (int j = 1; j <= S.n[0]; j++) S(j, k, l) = S(j, 1, l); }
                if (m[2] == 1) { i2[2] = f.n[2]; for (int l = 2; l <= i2[2]; l++) for (int k = 1; k <= S.n[1]; k++) for (int j = 1; j <= S.n[0]; j++) S(j, k, l) = S(j, k, 1); }
                for (int l = i1[2]; l <= i2[2]; l++)
                    for (int k = i1[1]; k <= i2[1]; k++)
                        for (int j = i1[0]; j <= i2[0]; j++) {
                            if (io.op == "=<") f(j, k, l) = S(j, k, l);
                            else if (io.op == "+<") f(j, k, l) = f(j, k, l) + S(j, k, l);
                            else if (io.op == "*<") f(j, k, l) = f(j, k, l) * S(j, k, l);
                            else throw SordStop("bad i/o op");
                        }
            }
            if (io.reg == 'n') scalar_bc(f, bc1, bc2, i1bc, i2bc);
            if (io.reg == 'c') { int t[3] = {i2bc[0] - 1, i2bc[1] - 1, i2bc[2] - 1}; scalar_bc(f, bc1, bc2, i1bc, t); }
            if (it == it2) { io.buff.clear(); io.op = "#"; }
            return;
        }
        // disk output
        if (op2 == '>') {
            if (io.op == ".>") {
                for (int i = 0; i < 3; i++)
                    if (!plane[i] && (i2[i] < i1core[i] || i2[i] > i2core[i])) { io.op = "#"; return; }
            }
            int nsp = n[0] * n[1] * n[2];
            if (io.ib < 0) {
                io.bufn = imax(nsp, 0);
                io.buff.assign((size_t)io.bufn * io.nb, R(0));
                io.ib = 0;
                io.open = false;
            }
            if (imod(it, itstats) != 0) {
                std::string fl = io.field;
                if (fl == "vm2") vector_norm(f, vv, i1, i2, di);
                else if (fl == "um2") vector_norm(f, uu, i1, i2, di);
                else if (fl == "wm2") tensor_norm(f, w1, w2, i1, i2, di);
                else if (fl == "am2") vector_norm(f, w1, i1, i2, di);
            }
            io.ib = io.ib + 1;
            real* buf = io.buff.data() + (size_t)io.bufn * (io.ib - 1);
            if (io.op == ".>") {
                real acc = 0;
                for (int l = i1[2]; l <= i2[2]; l++)
                    for (int k = i1[1]; k <= i2[1]; k++)
                        for (int j = i1[0]; j <= i2[0]; j++) {
                            real r = wgt(xi[0], j, plane[0]) * wgt(xi[1], k, plane[1]) * wgt(xi[2], l, plane[2]);
                            acc = acc + f(j, k, l) * r;
                        }
                buf[0] = acc;
            } else if (io.op == "=>") {
                size_t q = 0;
                for (int l = i1[2]; l <= i2[2]; l += di[2])
                    for (int k = i1[1]; k <= i2[1]; k += di[1])
                        for (int j = i1[0]; j <= i2[0]; j += di[0]) buf[q++] = f(j, k, l);
            } else throw SordStop("bad i/o op");
            if (io.ib == io.nb || it == it2 || imod(it, itio) == 0) {
                n[3] = io.ib;
                m[3] = (it2 - it1) / dit + 1;
                o[3] = (it - it1) / dit + 1 - n[3];
                std::string filename = io.fname;
                if ((n[0] != m[0] || n[1] != m[1] || n[2] != m[2]) && mpout == 0) filename += "-000000";
                if (!(n[0] < 1 || n[1] < 1 || n[2] < 1 || n[3] < 1))
                    frio2(&io, io.open, io.buff.data(), io.bufn, n[3], 'w', filename, m[3], o[3]);
                io.ib = 0;
                if (it == it2 || n[0] < 1 || n[1] < 1 || n[2] < 1 || n[3] < 1) { io.buff.clear(); io.op = "#"; }
            }
            return;
        }
        throw SordStop("bad i/o op");
        (void)field;
    }

    static real wgt(real x, int j, bool plane) {
        if (plane) return R(1);
        return R(1) - std::fabs(x - R(j));
    }

    // rio2 read of the sub-array n(1:3) at offset o(1:3) of a file of m(1:3) per record
    void read_subarray(IoOp& io, const std::string& filename, const int* m, const int* n, const int* o) {
        // serial build: n == m except for clipped ops, which read the "-000000" file
        // holding exactly n(1:3) values per record (rank-local file).
        FILE* fp = fopen(filename.c_str(), "rb");
        if (!fp) throw SordStop("cannot open " + filename);
        size_t recl = (size_t)n[0] * n[1] * n[2];
        fseek(fp, (long)(recl * sizeof(real) * (size_t)o[3]), SEEK_SET);
        size_t got = fread(io.buff.data(), sizeof(real), recl * n[3], fp);
        fclose(fp);
        if (got != recl * n[3]) throw SordStop("short read " + filename);
        (void)m;
    }

    // sord/input_output.f90:546-591 with node coordinates for node fields and
    // cell centres for cell fields (the reference passes w1/w2 here).
    void set_cube(V3 f, IoOp& io, const int* i1, const int* i2, const int* di, real r) {
        int o[3];
        for (int i = 0; i < 3; i++) o[i] = f.n[i] == 1 ? 1 - i1[i] : 0;
        char c = io.op[0];
        for (int l = i1[2]; l <= i2[2]; l += di[2])
            for (int k = i1[1]; k <= i2[1]; k += di[1])
                for (int j = i1[0]; j <= i2[0]; j += di[0]) {
                    real X[3];
                    for (int a = 1; a <= 3; a++) {
                        if (io.reg == 'c') X[a - 1] = R(0.125) * (xx(j, k, l, a) + xx(j + 1, k + 1, l + 1, a) + xx(j, k + 1, l + 1, a) + xx(j + 1, k, l, a) +
                                                               xx(j + 1, k, l + 1, a) + xx(j, k + 1, l, a) + xx(j + 1, k + 1, l, a) + xx(j, k, l + 1, a));
                        else X[a - 1] = xx(j, k, l, a);
                    }
                    if (X[0] >= io.x1[0] && X[0] <= io.x2[0] && X[1] >= io.x1[1] && X[1] <= io.x2[1] && X[2] >= io.x1[2] && X[2] <= io.x2[2]) {
                        real& F = f(j + o[0], k + o[1], l + o[2]);
                        if (c == '=') F = r;
                        else if (c == '+') F = F + r;
                        else if (c == '*') F = F * r;
                        else throw SordStop("error in cube");
                    }
                }
    }

    // ------------------------------------------------------------ init
    // sord/grid_generation.f90:6-200
    void init_grid() {
        int i1[3], i2[3];
        std::fill(xx.d.begin(), xx.d.end(), R(0));
        for (int i = 0; i < 3; i++) { i1[i] = i1node[i]; i2[i] = i2node[i]; }
        for (int i = i1[0]; i <= i2[0]; i++) for (int l = 1; l <= nm[2]; l++) for (int k = 1; k <= nm[1]; k++) xx(i, k, l, 1) = dx[0] * R(i + nnoff[0] - 1);
        for (int i = i1[1]; i <= i2[1]; i++) for (int l = 1; l <= nm[2]; l++) for (int j = 1; j <= nm[0]; j++) xx(j, i, l, 2) = dx[1] * R(i + nnoff[1] - 1);
        for (int i = i1[2]; i <= i2[2]; i++) for (int k = 1; k <= nm[1]; k++) for (int j = 1; j <= nm[0]; j++) xx(j, k, i, 3) = dx[2] * R(i + nnoff[2] - 1);
        for (int i = 0; i < 3; i++) i1[i] = imax(i1core[i], irup + 1);
        char fc = faultnormal.size() > 1 ? faultnormal[1] : ' ';
        if (fc == 'x') for (int i = i1[0]; i <= i2[0]; i++) for (int l = 1; l <= nm[2]; l++) for (int k = 1; k <= nm[1]; k++) xx(i, k, l, 1) = dx[0] * R(i + nnoff[0] - 2);
        if (fc == 'y') for (int i = i1[1]; i <= i2[1]; i++) for (int l = 1; l <= nm[2]; l++) for (int j = 1; j <= nm[0]; j++) xx(j, i, l, 2) = dx[1] * R(i + nnoff[1] - 2);
        if (fc == 'z') for (int i = i1[2]; i <= i2[2]; i++) for (int k = 1; k <= nm[1]; k++) for (int j = 1; j <= nm[0]; j++) xx(j, k, i, 3) = dx[2] * R(i + nnoff[2] - 2);
        field_io("<", "x", xx.c(1));
        field_io("<", "y", xx.c(2));
        field_io("<", "z", xx.c(3));
        if (gridnoise > R(0)) {
            uint64_t call = rng_calls++;
            for (size_t q = 0; q < w1.d.size(); q++) w1.d[q] = urand(call, q);
            real amp = std::sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]) * gridnoise;
            for (size_t q = 0; q < w1.d.size(); q++) w1.d[q] = amp * (w1.d[q] - R(0.5));
            int a1[3], a2[3];
            for (int i = 0; i < 3; i++) { a1[i] = i1pml[i] + 1; a2[i] = i2pml[i] - 1; }
            for (int c = 1; c <= 3; c++) set_halo(w1.c(c), R(0), a1, a2);
            for (int i = 0; i < 3; i++) { a1[i] = i1bc[i] + 1; a2[i] = i2bc[i] - 1; }
            for (int c = 1; c <= 3; c++) set_halo(w1.c(c), R(0), a1, a2);
            for (int i = 0; i < 3; i++) { a1[i] = imax(i1core[i], irup); a2[i] = imin(i2core[i], irup + 1); }
            int d = fc == 'x' ? 0 : fc == 'y' ? 1 : fc == 'z' ? 2 : -1;
            if (d >= 0)
                for (int c = 1; c <= 3; c++)
                    for (int l = 1; l <= nm[2]; l++)
                        for (int k = 1; k <= nm[1]; k++)
                            for (int j = 1; j <= nm[0]; j++) {
                                int p = d == 0 ? j : d == 1 ? k : l;
                                if (p >= a1[d] && p <= a2[d]) w1(j, k, l, c) = 0;
                            }
            for (size_t q = 0; q < xx.d.size(); q++) xx.d[q] = xx.d[q] + w1.d[q];
        }
        if (rexpand > R(1)) {
            int e1[3], e2[3];
            for (int i = 0; i < 3; i++) { e1[i] = n1expand[i] - nnoff[i]; e2[i] = nn[i] - n2expand[i] + 1 - nnoff[i]; }
            for (int d = 0; d < 3; d++) {
                for (int p = i1node[d]; p <= imin(i2node[d], e1[d]); p++) {
                    int i = e1[d] - p;
                    real s = dx[d] * (R(i + 1) - (powi(rexpand, i + 1) - R(1)) / (rexpand - R(1)));
                    plane_add(d, p, s);
                }
                for (int p = imax(i1node[d], e2[d]); p <= i2node[d]; p++) {
                    int i = p - e2[d];
                    real s = dx[d] * (R(i + 1) - (powi(rexpand, i + 1) - R(1)) / (rexpand - R(1)));
                    plane_add(d, p, -s);
                }
            }
        }
        const real* mm = affine;
#pragma omp parallel for schedule(static)
        for (int l = 1; l <= nm[2]; l++)
            for (int k = 1; k <= nm[1]; k++)
                for (int j = 1; j <= nm[0]; j++) {
                    real a = xx(j, k, l, 1), b = xx(j, k, l, 2), c = xx(j, k, l, 3);
                    real x = mm[0] * a + mm[1] * b + mm[2] * c;
                    real y = mm[3] * a + mm[4] * b + mm[5] * c;
                    real z = mm[6] * a + mm[7] * b + mm[8] * c;
                    xx(j, k, l, 1) = x; xx(j, k, l, 2) = y; xx(j, k, l, 3) = z;
                }
        {
            int bc[3] = {4, 4, 4}, a1[3], a2[3];
            for (int i = 0; i < 3; i++) { a1[i] = i1bc[i] - 1; a2[i] = i2bc[i] + 1; }
            vector_bc(xx, bc, bc, a1, a2);
        }
        for (int c = 1; c <= 3; c++) {
            average(w1.c(c), xx.c(c), i1cell, i2cell, 1);
            set_halo(w1.c(c), R(0), i1cell, i2cell);
        }
        field_io(">", "x", xx.c(1));
        field_io(">", "y", xx.c(2));
        field_io(">", "z", xx.c(3));
        field_io(">", "xc", w1.c(1));
        field_io(">", "yc", w1.c(2));
        field_io(">", "zc", w1.c(3));
        set_halo(vc.v(), R(0), i1cell, i2cell);
        bool err = false;
        for (int i = 1; i <= 3; i++) {
            diff_nc(vc.v(), xx, i, i, i1cell, i2cell, xx);
            if (ifn) zero_plane(vc.v(), ifn - 1, irup);
            real mn = vc.d[0];
            for (real v : vc.d) mn = std::min(mn, v);
            err = mn < R(0);
        }
        field_io(">", "vc", vc.v());
        if (err) throw SordStop("Negative cell volume. Wrong sign in dx or problem with mesh.");
    }
    void plane_add(int d, int p, real s) {
        for (int l = 1; l <= nm[2]; l++)
            for (int k = 1; k <= nm[1]; k++)
                for (int j = 1; j <= nm[0]; j++) {
                    int q = d == 0 ? j : d == 1 ? k : l;
                    if (q == p) xx(j, k, l, d + 1) = xx(j, k, l, d + 1) + s;
                }
    }
    static void zero_plane(V3 f, int d, int p) {
        for (int l = 1; l <= f.n[2]; l++)
            for (int k = 1; k <= f.n[1]; k++)
                for (int j = 1; j <= f.n[0]; j++) {
                    int q = d == 0 ? j : d == 1 ? k : l;
                    if (q == p) f(j, k, l) = 0;
                }
    }

    // sord/material_model.f90:6-171
    void init_material() {
        std::fill(mr.d.begin(), mr.d.end(), R(0));
        std::fill(lam.d.begin(), lam.d.end(), R(0));
        std::fill(mu.d.begin(), mu.d.end(), R(0));
        std::fill(gam.d.begin(), gam.d.end(), R(0));
        field_io("<", "rho", mr.v());
        field_io("<", "vp", lam.v());
        field_io("<", "vs", mu.v());
        field_io("<", "gam", gam.v());
        s1.d = lam.d;
        s2.d = mu.d;
        rlimits(mr.v(), rho_min, rho_max);
        rlimits(s1.v(), vp_min, vp_max);
        rlimits(s2.v(), vs_min, vs_max);
        if (vdamp > R(0))
            for (size_t q = 0; q < gam.size(); q++) gam.d[q] = s2.d[q] == R(0) ? R(0) : vdamp / s2.d[q];
        rlimits(gam.v(), gam_min, gam_max);
        set_halo(mr.v(), R(0), i1cell, i2cell);
        set_halo(s1.v(), R(0), i1cell, i2cell);
        set_halo(s2.v(), R(0), i1cell, i2cell);
        set_halo(gam.v(), R(0), i1cell, i2cell);
        for (size_t q = 0; q < mu.size(); q++) {
            mu.d[q] = mr.d[q] * s2.d[q] * s2.d[q];
            lam.d[q] = mr.d[q] * s1.d[q] * s1.d[q] - R(2) * mu.d[q];
            real r = lam.d[q] + mu.d[q];
            yy.d[q] = r == R(0) ? R(0) : R(0.5) * lam.d[q] / r;
        }
        int a1[3], a2[3];
        for (int i = 0; i < 3; i++) { a1[i] = imax(i1core[i], i1bc[i]); a2[i] = imin(i2core[i], i2bc[i] - 1); }
        real maxg[14];
        A3* arrs[7] = {&mr, &s1, &s2, &gam, &lam, &mu, &yy};
        for (int q = 0; q < 7; q++) {
            real mn = std::numeric_limits<real>::max(), mx = -std::numeric_limits<real>::max();
            for (int l = a1[2]; l <= a2[2]; l++)
                for (int k = a1[1]; k <= a2[1]; k++)
                    for (int j = a1[0]; j <= a2[0]; j++) { real v = (*arrs[q])(j, k, l); mn = std::min(mn, v); mx = std::max(mx, v); }
            maxg[q] = -mn;
            maxg[q + 7] = mx;
        }
        field_io(">", "rho", mr.v());
        field_io(">", "vp", s1.v());
        field_io(">", "vs", s2.v());
        field_io(">", "gam", gam.v());
        field_io(">", "lam", lam.v());
        field_io(">", "mu", mu.v());
        field_io(">", "nu", yy.v());
        real s = std::sqrt((dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]) / R(3)) / R(12);
        for (size_t q = 0; q < yy.size(); q++) {
            real r = lam.d[q] + R(2) * mu.d[q];
            yy.d[q] = r == R(0) ? R(0) : mu.d[q] * (lam.d[q] + mu.d[q]) * s / r;
        }
        if (vpml <= R(0)) {
            real vmn = -maxg[2], vmx = maxg[8];
            vpml = R(2) * vmn * vmx / (vmn + vmx);
        }
        real vmx = maxg[8];
        real r = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        real cfl1 = dt * vmx * std::sqrt(R(3) / r);
        real cfl2 = dt * vmx * R(3) / std::sqrt(r);
        FILE* fp = fopen("material.json", "w");
        if (fp) {
            fprintf(fp, "{\n");
            fprintf(fp, "    \"cfl\": [%.9g, %.9g],\n", (double)cfl1, (double)cfl2);
            const char* nm_[7] = {"rho", "vp", "vs", "gam", "lam", "mu", "nu"};
            for (int q = 0; q < 7; q++)
                fprintf(fp, "    \"%s\": [%.9g, %.9g]%s\n", nm_[q], (double)-maxg[q], (double)maxg[q + 7], q < 6 ? "," : "");
            fprintf(fp, "}\n");
            fclose(fp);
        }
        for (int q = 0; q < 7; q++)
            if (maxg[q] > R(0)) throw SordStop("negative moduli");
        if (cfl2 > R(1)) throw SordStop("Courant condition not satisfied!");
    }

    // sord/boundary_pml.f90:7-82
    void init_pml() {
        if (npml < 1) return;
        dn1.assign(npml, R(0)); dn2.assign(npml, R(0)); dc1.assign(npml, R(0)); dc2.assign(npml, R(0));
        real c1 = R(8) / R(15), c2 = R(-3) / R(100), c3 = R(1) / R(1500), tune = R(3.5);
        real r = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        real damp = tune * vpml / std::sqrt(r / R(3)) * (c1 + (c2 + c3 * R(npml)) * R(npml)) / R(ipow(npml, ppml));
        for (int i = 1; i <= npml; i++) {
            real dampn = damp * R(ipow(i, ppml));
            real dampc = damp * R(ipow(i, ppml) + ipow(i - 1, ppml)) * R(0.5);
            int p = npml - i;  // 0-based slot of dn1(npml-i+1)
            dn1[p] = -(R(2) * dampn) / (R(2) + dt * dampn);
            dc1[p] = (R(2) - dt * dampc) / (R(2) + dt * dampc);
            dn2[p] = R(2) / (R(2) + dt * dampn);
            dc2[p] = R(2) * dt / (R(2) + dt * dampc);
        }
        int a1[3], a2[3];
        for (int i = 0; i < 3; i++) { a1[i] = imin(i2node[i], i1pml[i]) - i1node[i] + 1; a2[i] = i2node[i] - imax(i1node[i], i2pml[i]) + 1; }
        p1.alloc(imax(a1[0], 0), nm[1], nm[2], 3); p2.alloc(nm[0], imax(a1[1], 0), nm[2], 3); p3.alloc(nm[0], nm[1], imax(a1[2], 0), 3);
        p4.alloc(imax(a2[0], 0), nm[1], nm[2], 3); p5.alloc(nm[0], imax(a2[1], 0), nm[2], 3); p6.alloc(nm[0], nm[1], imax(a2[2], 0), 3);
        for (int i = 0; i < 3; i++) { a1[i] = imin(i2cell[i], i1pml[i]) - i1cell[i] + 1; a2[i] = i2cell[i] - imax(i1cell[i], i2pml[i] - 1) + 1; }
        g1.alloc(imax(a1[0], 0), nm[1], nm[2], 3); g2.alloc(nm[0], imax(a1[1], 0), nm[2], 3); g3.alloc(nm[0], nm[1], imax(a1[2], 0), 3);
        g4.alloc(imax(a2[0], 0), nm[1], nm[2], 3); g5.alloc(nm[0], imax(a2[1], 0), nm[2], 3); g6.alloc(nm[0], nm[1], imax(a2[2], 0), 3);
    }
    real DN1(int p) const { return dn1[p - 1]; }
    real DN2(int p) const { return dn2[p - 1]; }
    real DC1(int p) const { return dc1[p - 1]; }
    real DC2(int p) const { return dc2[p - 1]; }

    // sord/kinematic_source.f90:10-63
    void init_finite_source() {
        if (nsource == 0) return;
        int n = std::abs(nsource);
        auto rd = [&](std::vector<real>& v, const char* fn) {
            v.assign(n, R(0));
            FILE* fp = fopen(fn, "rb");
            if (!fp) throw SordStop(std::string("cannot open ") + fn);
            if (fread(v.data(), sizeof(real), n, fp) != (size_t)n) { fclose(fp); throw SordStop(std::string("short read ") + fn); }
            fclose(fp);
        };
        rd(src_xi[0], "source-xi1.bin"); rd(src_xi[1], "source-xi2.bin"); rd(src_xi[2], "source-xi3.bin");
        if (source == "force") {
            for (int i = 0; i < 3; i++) {
                for (auto& x : src_xi[i]) x = x - R(nnoff[i]);
                bool lo = true, hi = true;
                for (auto x : src_xi[i]) { lo = lo && x < R(-1 + i1node[i]); hi = hi && x > R(1 + i2node[i]); }
                if (lo || hi) { nsource = 0; return; }
            }
            rd(src_w1[0], "source-w11.bin"); rd(src_w1[1], "source-w12.bin"); rd(src_w1[2], "source-w13.bin");
        } else {
            for (int i = 0; i < 3; i++) {
                for (auto& x : src_xi[i]) x = x - R(0.5) - R(nnoff[i]);
                bool lo = true, hi = true;
                for (auto x : src_xi[i]) { lo = lo && x < R(-1 + i1cell[i]); hi = hi && x > R(1 + i2cell[i]); }
                if (lo || hi) { nsource = 0; return; }
            }
            rd(src_w1[0], "source-w11.bin"); rd(src_w1[1], "source-w22.bin"); rd(src_w1[2], "source-w33.bin");
            rd(src_w2[0], "source-w23.bin"); rd(src_w2[1], "source-w31.bin"); rd(src_w2[2], "source-w12.bin");
        }
        rd(src_t0, "source-t0.bin");
        rd(src_dt, "source-dt.bin");
        {
            src_nt.assign(n, 0);
            FILE* fp = fopen("source-nt.bin", "rb");
            if (!fp) throw SordStop("cannot open source-nt.bin");
            if (fread(src_nt.data(), sizeof(int), n, fp) != (size_t)n) { fclose(fp); throw SordStop("short read source-nt.bin"); }
            fclose(fp);
        }
        long tot = 0;
        for (int v : src_nt) tot += v;
        std::vector<real> hist;
        src_history.assign(tot, R(0));
        if (tot) {
            FILE* fp = fopen("source-history.bin", "rb");
            if (!fp) throw SordStop("cannot open source-history.bin");
            if (fread(src_history.data(), sizeof(real), tot, fp) != (size_t)tot) { fclose(fp); throw SordStop("short read source-history.bin"); }
            fclose(fp);
        }
    }

    // sord/kinematic_source.f90:66-118
    void finite_source() {
        if (nsource == 0) return;
        long itoff = 0;
        for (int isrc = 0; isrc < std::abs(nsource); isrc++) {
            int i = ffloor((tm - src_t0[isrc]) / src_dt[isrc]) + 1;
            real xi[3] = {src_xi[0][isrc], src_xi[1][isrc], src_xi[2][isrc]};
            int i1[3], i2[3];
            for (int d = 0; d < 3; d++) {
                if (source == "force") { i1[d] = imax(i1node[d], ffloor(xi[d])); i2[d] = imin(i2node[d], ffloor(xi[d]) + 1); }
                else { i1[d] = imax(i1cell[d], ffloor(xi[d])); i2[d] = imin(i2cell[d], ffloor(xi[d]) + 1); }
            }
            if (i >= 0 && i2[0] >= i1[0] && i2[1] >= i1[1] && i2[2] >= i1[2]) {
                i = imin(i, src_nt[isrc] - 1);
                real t = src_t0[isrc] + src_dt[isrc] * R(i - 1);
                real h = std::min(R(1), (tm - t) / src_dt[isrc]);
                if (i == 0) h = h * src_history[itoff];
                else h = (R(1) - h) * src_history[itoff + i - 1] + h * src_history[itoff + i];
                for (int l = i1[2]; l <= i2[2]; l++)
                    for (int k = i1[1]; k <= i2[1]; k++)
                        for (int j = i1[0]; j <= i2[0]; j++) {
                            real w = h * ((R(1) - std::fabs(xi[0] - R(j))) * (R(1) - std::fabs(xi[1] - R(k))) * (R(1) - std::fabs(xi[2] - R(l))));
                            for (int c = 1; c <= 3; c++) {
                                if (source == "force") w1(j, k, l, c) = w1(j, k, l, c) + w * src_w1[c - 1][isrc];
                                else {
                                    w1(j, k, l, c) = w1(j, k, l, c) - w * src_w1[c - 1][isrc];
                                    w2(j, k, l, c) = w2(j, k, l, c) - w * src_w2[c - 1][isrc];
                                }
                            }
                        }
            }
            itoff += src_nt[isrc];
        }
    }

    // fault-plane view helpers: array f(nm with extent 1 along ifn)
    int fn3[3];
    V3 fv(A3& a) { return a.v(); }
    // volume value at fault side `side` (irup or irup+1) for fault plane index (j,k,l)
    size_t vol_index(int j, int k, int l, int side) const {
        int p[3] = {j, k, l};
        p[ifn - 1] = side;
        return (size_t)(p[0] - 1) + (size_t)nm[0] * ((size_t)(p[1] - 1) + (size_t)nm[1] * (size_t)(p[2] - 1));
    }

    // sord/dynamic_rupture.f90:7-238
    void init_rupture() {
        if (faultnormal == "no") return;
        if (ifn == 0) return;
        for (int i = 0; i < 3; i++) fn3[i] = nm[i];
        fn3[ifn - 1] = 1;
        int j = fn3[0], k = fn3[1], l = fn3[2];
        nhat.alloc(j, k, l, 3); t0.alloc(j, k, l, 3); t1.alloc(j, k, l, 3); t2.alloc(j, k, l, 3); t3.alloc(j, k, l, 3);
        A3* sc[] = {&mus, &mud, &dc, &co, &area, &rhypo, &lamf, &muf, &sl, &psv, &trup, &tarr, &tn, &ts, &f1, &f2};
        for (A3* a : sc) a->alloc(j, k, l);
        field_io("<>", "mus", mus.v());
        field_io("<>", "mud", mud.v());
        field_io("<>", "dc", dc.v());
        field_io("<>", "co", co.v());
        field_io("<>", "sxx", t1.c(1));
        field_io("<>", "syy", t1.c(2));
        field_io("<>", "szz", t1.c(3));
        field_io("<>", "syz", t2.c(1));
        field_io("<>", "szx", t2.c(2));
        field_io("<>", "sxy", t2.c(3));
        field_io("<>", "ts", t3.c(1));
        field_io("<>", "td", t3.c(2));
        field_io("<>", "tn", t3.c(3));
        {
            real rr = -std::numeric_limits<real>::max();
            for (real v : t3.c(3).p ? std::vector<real>(t3.c(3).p, t3.c(3).p + t3.c(3).size()) : std::vector<real>()) rr = std::max(rr, v);
            if (rr > R(0)) fprintf(stderr, "Warning: positive normal traction: %g\n", (double)rr);
        }
        {
            int a1[3], a2[3];
            for (int i = 0; i < 3; i++) { a1[i] = i1pml[i] + 1; a2[i] = i2pml[i] - 1; }
            set_halo(co.v(), R(1e20), a1, a2);
        }
        {
            int a1[3], a2[3];
            for (int i = 0; i < 3; i++) { a1[i] = i1core[i]; a2[i] = i2core[i]; }
            a1[ifn - 1] = irup; a2[ifn - 1] = irup;
            node_normals(nhat, w1_geometry ? w1 : xx, a1, a2, ifn);
        }
        size_t np = area.size();
        for (size_t q = 0; q < np; q++) {
            real s = nhat.d[q] * nhat.d[q] + nhat.d[q + np] * nhat.d[q + np] + nhat.d[q + 2 * np] * nhat.d[q + 2 * np];
            area.d[q] = faultnormal[0] == '+' ? std::sqrt(s) : -std::sqrt(s);
        }
        f1.d = area.d;
        rinvert(f1.v());
        for (int c = 0; c < 3; c++)
            for (size_t q = 0; q < np; q++) nhat.d[q + c * np] = nhat.d[q + c * np] * f1.d[q];
        field_io(">", "nsx", nhat.c(1));
        field_io(">", "nsy", nhat.c(2));
        field_io(">", "nsz", nhat.c(3));
        for (int i = 1; i <= 3; i++) {
            int jj = imod(i, 3) + 1, kk = imod(i + 1, 3) + 1;
            for (size_t q = 0; q < np; q++)
                t0.d[q + (i - 1) * np] = t1.d[q + (i - 1) * np] * nhat.d[q + (i - 1) * np] + t2.d[q + (jj - 1) * np] * nhat.d[q + (kk - 1) * np] +
                                         t2.d[q + (kk - 1) * np] * nhat.d[q + (jj - 1) * np];
        }
        for (size_t q = 0; q < np; q++) {
            real n1 = nhat.d[q], n2 = nhat.d[q + np], n3 = nhat.d[q + 2 * np];
            t2.d[q] = n2 * slipvector[2] - n3 * slipvector[1];
            t2.d[q + np] = n3 * slipvector[0] - n1 * slipvector[2];
            t2.d[q + 2 * np] = n1 * slipvector[1] - n2 * slipvector[0];
            real s = t2.d[q] * t2.d[q] + t2.d[q + np] * t2.d[q + np] + t2.d[q + 2 * np] * t2.d[q + 2 * np];
            f1.d[q] = std::sqrt(s);
        }
        rinvert(f1.v());
        for (int c = 0; c < 3; c++) for (size_t q = 0; q < np; q++) t2.d[q + c * np] = t2.d[q + c * np] * f1.d[q];
        for (size_t q = 0; q < np; q++) {
            real a1 = t2.d[q], a2 = t2.d[q + np], a3 = t2.d[q + 2 * np];
            real n1 = nhat.d[q], n2 = nhat.d[q + np], n3 = nhat.d[q + 2 * np];
            t1.d[q] = a2 * n3 - a3 * n2;
            t1.d[q + np] = a3 * n1 - a1 * n3;
            t1.d[q + 2 * np] = a1 * n2 - a2 * n1;
            real s = t1.d[q] * t1.d[q] + t1.d[q + np] * t1.d[q + np] + t1.d[q + 2 * np] * t1.d[q + 2 * np];
            f1.d[q] = std::sqrt(s);
        }
        rinvert(f1.v());
        for (int c = 0; c < 3; c++) for (size_t q = 0; q < np; q++) t1.d[q + c * np] = t1.d[q + c * np] * f1.d[q];
        for (int c = 0; c < 3; c++)
            for (size_t q = 0; q < np; q++)
                t0.d[q + c * np] = t0.d[q + c * np] + t3.d[q] * t1.d[q + c * np] + t3.d[q + np] * t2.d[q + c * np] + t3.d[q + 2 * np] * nhat.d[q + c * np];
        if (rcrit > R(0) && vrup > R(0)) {
            A4& geo = w1_geometry ? w1 : xx;
            real xhypo[3] = {0, 0, 0}, xi[3];
            int i1[3];
            for (int i = 0; i < 3; i++) { xi[i] = hypocenter[i] - R(nnoff[i]) + R(1); i1[i] = ffloor(xi[i]); }
            if (i1[0] >= 1 && i1[0] < nm[0] && i1[1] >= 1 && i1[1] < nm[1] && i1[2] >= 1 && i1[2] < nm[2]) {
                for (int l = i1[2]; l <= i1[2] + 1; l++)
                    for (int k = i1[1]; k <= i1[1] + 1; k++)
                        for (int j2 = i1[0]; j2 <= i1[0] + 1; j2++) {
                            real w = (R(1) - std::fabs(xi[0] - R(j2))) * (R(1) - std::fabs(xi[1] - R(k))) * (R(1) - std::fabs(xi[2] - R(l)));
                            for (int i = 1; i <= 3; i++) xhypo[i - 1] = xhypo[i - 1] + w * geo(j2, k, l, i);
                        }
            }
            for (int ll = 1; ll <= fn3[2]; ll++)
                for (int kk = 1; kk <= fn3[1]; kk++)
                    for (int jj = 1; jj <= fn3[0]; jj++) {
                        size_t q = (size_t)(jj - 1) + (size_t)fn3[0] * ((size_t)(kk - 1) + (size_t)fn3[1] * (size_t)(ll - 1));
                        size_t vq = vol_index(jj, kk, ll, irup);
                        size_t nv = (size_t)nm[0] * nm[1] * nm[2];
                        for (int i = 0; i < 3; i++) t2.d[q + i * np] = geo.d[vq + i * nv] - xhypo[i];
                        rhypo.d[q] = std::sqrt(t2.d[q] * t2.d[q] + t2.d[q + np] * t2.d[q + np] + t2.d[q + 2 * np] * t2.d[q + 2 * np]);
                    }
        }
        for (int ll = 1; ll <= fn3[2]; ll++)
            for (int kk = 1; kk <= fn3[1]; kk++)
                for (int jj = 1; jj <= fn3[0]; jj++) {
                    size_t q = (size_t)(jj - 1) + (size_t)fn3[0] * ((size_t)(kk - 1) + (size_t)fn3[1] * (size_t)(ll - 1));
                    size_t vq = vol_index(jj, kk, ll, irup);
                    lamf.d[q] = lam.d[vq];
                    muf.d[q] = mu.d[vq];
                }
        rinvert(lamf.v());
        rinvert(muf.v());
        // 2-point averages along the in-plane dimensions (array sections, evaluated
        // from the right-hand side before assignment)
        for (A3* a : {&lamf, &muf}) {
            for (int d = 0; d < 3; d++) {
                if (d == ifn - 1) continue;
                std::vector<real> src = a->d;
                int e = nm[d] - 1;
                for (int ll = 1; ll <= fn3[2]; ll++)
                    for (int kk = 1; kk <= fn3[1]; kk++)
                        for (int jj = 1; jj <= fn3[0]; jj++) {
                            int p[3] = {jj, kk, ll};
                            if (p[d] < 2 || p[d] > e) continue;
                            size_t q = (size_t)(jj - 1) + (size_t)fn3[0] * ((size_t)(kk - 1) + (size_t)fn3[1] * (size_t)(ll - 1));
                            size_t stride = d == 0 ? 1 : d == 1 ? (size_t)fn3[0] : (size_t)fn3[0] * fn3[1];
                            a->d[q] = R(0.5) * (src[q] + src[q - stride]);
                        }
            }
        }
        rinvert(muf.v());
        std::fill(psv.d.begin(), psv.d.end(), R(0));
        std::fill(trup.d.begin(), trup.d.end(), R(1e9));
        std::fill(tarr.d.begin(), tarr.d.end(), R(0));
        efric = 0;
    }

    // sord/dynamic_rupture.f90:243-384
    void step_rupture() {
        if (ifn == 0) return;
        size_t np = area.size(), nv = (size_t)nm[0] * nm[1] * nm[2];
        std::vector<size_t> q1(np), q2(np);
        for (int ll = 1; ll <= fn3[2]; ll++)
            for (int kk = 1; kk <= fn3[1]; kk++)
                for (int jj = 1; jj <= fn3[0]; jj++) {
                    size_t q = (size_t)(jj - 1) + (size_t)fn3[0] * ((size_t)(kk - 1) + (size_t)fn3[1] * (size_t)(ll - 1));
                    q1[q] = vol_index(jj, kk, ll, irup);
                    q2[q] = vol_index(jj, kk, ll, irup + 1);
                }
        for (size_t q = 0; q < np; q++) f1.d[q] = dt * dt * area.d[q] * (mr.d[q1[q]] + mr.d[q2[q]]);
        rinvert(f1.v());
        for (int i = 0; i < 3; i++)
            for (size_t q = 0; q < np; q++) {
                size_t a = q1[q] + i * nv, b = q2[q] + i * nv;
                t1.d[q + i * np] = t0.d[q + i * np] + f1.d[q] * dt * (vv.d[b] - vv.d[a] + w1.d[b] * mr.d[q2[q]] * dt - w1.d[a] * mr.d[q1[q]] * dt);
                t2.d[q + i * np] = t1.d[q + i * np] + f1.d[q] * (uu.d[b] - uu.d[a]);
            }
        for (size_t q = 0; q < np; q++) {
            tn.d[q] = t1.d[q] * nhat.d[q] + t1.d[q + np] * nhat.d[q + np] + t1.d[q + 2 * np] * nhat.d[q + 2 * np];
            for (int i = 0; i < 3; i++) t3.d[q + i * np] = t1.d[q + i * np] - tn.d[q] * nhat.d[q + i * np];
            ts.d[q] = std::sqrt(t3.d[q] * t3.d[q] + t3.d[q + np] * t3.d[q + np] + t3.d[q + 2 * np] * t3.d[q + 2 * np]);
        }
        if (it > 1) {
            for (size_t q = 0; q < np; q++) {
                tn.d[q] = t2.d[q] * nhat.d[q] + t2.d[q + np] * nhat.d[q + np] + t2.d[q + 2 * np] * nhat.d[q + 2 * np];
                if (faultopening == 1) tn.d[q] = std::min(R(0), tn.d[q]);
            }
            for (int i = 0; i < 3; i++)
                for (size_t q = 0; q < np; q++) t2.d[q + i * np] = vv.d[q2[q] + i * nv] - vv.d[q1[q] + i * nv];
            for (size_t q = 0; q < np; q++) f2.d[q] = t2.d[q] * t2.d[q] + t2.d[q + np] * t2.d[q + np] + t2.d[q + 2 * np] * t2.d[q + 2 * np];
            for (size_t q = 0; q < np; q++) {
                real v = mud.d[q];
                if (sl.d[q] < dc.d[q]) v = v + (R(1) - sl.d[q] / dc.d[q]) * (mus.d[q] - mud.d[q]);
                f1.d[q] = -std::min(R(0), tn.d[q]) * v + co.d[q];
            }
            if (rcrit > R(0) && vrup > R(0)) {
                for (size_t q = 0; q < np; q++) {
                    real g = 1;
                    if (trelax > R(0)) g = std::min((tm - rhypo.d[q] / vrup) / trelax, R(1));
                    g = (R(1) - g) * ts.d[q] + g * (-tn.d[q] * mud.d[q] + co.d[q]);
                    f2.d[q] = g;
                    if (rhypo.d[q] < std::min(rcrit, tm * vrup) && f2.d[q] < f1.d[q]) f1.d[q] = f2.d[q];
                }
            }
            for (size_t q = 0; q < np; q++) {
                real g = 1;
                if (ts.d[q] > f1.d[q]) g = f1.d[q] / ts.d[q];
                f2.d[q] = g;
                for (int i = 0; i < 3; i++) t3.d[q + i * np] = g * t3.d[q + i * np];
                ts.d[q] = std::min(ts.d[q], f1.d[q]);
                for (int i = 0; i < 3; i++) t1.d[q + i * np] = t3.d[q + i * np] + tn.d[q] * nhat.d[q + i * np];
            }
        }
        for (int i = 0; i < 3; i++)
            for (size_t q = 0; q < np; q++) {
                real g = area.d[q] * (t1.d[q + i * np] - t0.d[q + i * np]);
                f2.d[q] = g;
                w1.d[q1[q] + i * nv] = w1.d[q1[q] + i * nv] + g;
                w1.d[q2[q] + i * nv] = w1.d[q2[q] + i * nv] - g;
            }
        vector_bc(w1, bc1, bc2, i1bc, i2bc);
        field_io(">", "tx", t1.c(1));
        field_io(">", "ty", t1.c(2));
        field_io(">", "tz", t1.c(3));
        field_io(">", "tsx", t3.c(1));
        field_io(">", "tsy", t3.c(2));
        field_io(">", "tsz", t3.c(3));
        field_io(">", "tsm", ts.v());
        field_io(">", "tnm", tn.v());
        field_io(">", "fr", f1.v());
        set_halo(ts.v(), R(-1), i1core, i2core);
        tsmax = maxval(ts.v());
        set_halo(tn.v(), std::numeric_limits<real>::max(), i1core, i2core);
        tnmin = minval(tn.v());
        set_halo(tn.v(), -std::numeric_limits<real>::max(), i1core, i2core);
        tnmax = maxval(tn.v());
        set_halo(tn.v(), R(0), i1core, i2core);
        for (int i = 0; i < 3; i++) for (size_t q = 0; q < np; q++) t2.d[q + i * np] = vv.d[q2[q] + i * nv] - vv.d[q1[q] + i * nv];
        for (size_t q = 0; q < np; q++) f2.d[q] = (t1.d[q] * t2.d[q] + t1.d[q + np] * t2.d[q + np] + t1.d[q + 2 * np] * t2.d[q + 2 * np]) * area.d[q];
        set_halo(f2.v(), R(0), i1core, i2core);
        efric = efric + dt * sumval(f2.v());
        for (int i = 0; i < 3; i++) for (size_t q = 0; q < np; q++) t2.d[q + i * np] = uu.d[q2[q] + i * nv] - uu.d[q1[q] + i * nv];
        for (size_t q = 0; q < np; q++)
            f2.d[q] = ((t0.d[q] + t1.d[q]) * t2.d[q] + (t0.d[q + np] + t1.d[q + np]) * t2.d[q + np] + (t0.d[q + 2 * np] + t1.d[q + 2 * np]) * t2.d[q + 2 * np]) * area.d[q];
        set_halo(f2.v(), R(0), i1core, i2core);
        estrain = R(0.5) * sumval(f2.v());
        for (size_t q = 0; q < np; q++) f2.d[q] = muf.d[q] * area.d[q] * std::sqrt(t2.d[q] * t2.d[q] + t2.d[q + np] * t2.d[q + np] + t2.d[q + 2 * np] * t2.d[q + 2 * np]);
        set_halo(f2.v(), R(0), i1core, i2core);
        moment = sumval(f2.v());
        for (int i = 0; i < 3; i++)
            for (size_t q = 0; q < np; q++)
                t2.d[q + i * np] = w1.d[q2[q] + i * nv] * mr.d[q2[q]] - w1.d[q1[q] + i * nv] * mr.d[q1[q]];
        for (size_t q = 0; q < np; q++) f2.d[q] = std::sqrt(t2.d[q] * t2.d[q] + t2.d[q + np] * t2.d[q + np] + t2.d[q + 2 * np] * t2.d[q + 2 * np]);
        field_io(">", "sax", t2.c(1));
        field_io(">", "say", t2.c(2));
        field_io(">", "saz", t2.c(3));
        field_io(">", "sam", f2.v());
        set_halo(f2.v(), R(-1), i1core, i2core);
        samax = maxval(f2.v());
    }
    static real maxval(V3 f) { real m = -std::numeric_limits<real>::max(); size_t n = f.size(); for (size_t q = 0; q < n; q++) m = std::max(m, f.p[q]); return m; }
    static real minval(V3 f) { real m = std::numeric_limits<real>::max(); size_t n = f.size(); for (size_t q = 0; q < n; q++) m = std::min(m, f.p[q]); return m; }
    static real sumval(V3 f) { real s = 0; size_t n = f.size(); for (size_t q = 0; q < n; q++) s = s + f.p[q]; return s; }

    // sord/material_resample.f90:6-55
    void resample_material() {
        for (size_t q = 0; q < s2.size(); q++) s2.d[q] = mr.d[q] * vc.d[q];
        average(mr.v(), s2.v(), i1node, i2node, -1);
        rinvert(mr.v());
        scalar_bc(mr.v(), bc1, bc2, i1bc, i2bc);
        rinvert(vc.v());
        int bc[3] = {4, 4, 4}, a1[3], a2[3];
        for (int i = 0; i < 3; i++) { a1[i] = i1bc[i] - 1; a2[i] = i2bc[i]; }
        scalar_bc(gam.v(), bc, bc, a1, a2);
        for (size_t q = 0; q < s2.size(); q++) s2.d[q] = gam.d[q] * dt;
        average(gam.v(), s2.v(), i1node, i2node, -1);
        set_halo(gam.v(), R(0), i1bc, i2bc);
        scalar_bc(gam.v(), bc1, bc2, i1bc, i2bc);
        for (int i = 0; i < 3; i++) { a1[i] = i1bc[i]; a2[i] = i2bc[i] - 1; }
        set_halo(yy.v(), R(0), a1, a2);
        if (ifn) zero_plane(yy.v(), ifn - 1, irup);
        std::fill(vv.d.begin(), vv.d.end(), R(0));
        std::fill(uu.d.begin(), uu.d.end(), R(0));
        std::fill(w1.d.begin(), w1.d.end(), R(0));
        std::fill(w2.d.begin(), w2.d.end(), R(0));
        std::fill(s1.d.begin(), s1.d.end(), R(0));
        std::fill(s2.d.begin(), s2.d.end(), R(0));
    }

    // ------------------------------------------------------------ step
    // sord/time_integration.f90:6-115
    void step_time() {
        size_t nv = (size_t)nm[0] * nm[1] * nm[2];
        size_t np = ifn ? area.size() : 0;
        std::vector<size_t> q1, q2;
        if (ifn) {
            q1.resize(np); q2.resize(np);
            for (int ll = 1; ll <= fn3[2]; ll++)
                for (int kk = 1; kk <= fn3[1]; kk++)
                    for (int jj = 1; jj <= fn3[0]; jj++) {
                        size_t q = (size_t)(jj - 1) + (size_t)fn3[0] * ((size_t)(kk - 1) + (size_t)fn3[1] * (size_t)(ll - 1));
                        q1[q] = vol_index(jj, kk, ll, irup);
                        q2[q] = vol_index(jj, kk, ll, irup + 1);
                    }
            for (int i = 0; i < 3; i++) for (size_t q = 0; q < np; q++) t2.d[q + i * np] = vv.d[q2[q] + i * nv] - vv.d[q1[q] + i * nv];
            for (size_t q = 0; q < np; q++) f2.d[q] = std::sqrt(t2.d[q] * t2.d[q] + t2.d[q + np] * t2.d[q + np] + t2.d[q + 2 * np] * t2.d[q + 2 * np]);
        }
        tm = tm0 + dt * R(it - 1);
        for (int i = 0; i < 3; i++) {
            real* V = vv.d.data() + i * nv;
            real* U = uu.d.data() + i * nv;
            real* W = w1.d.data() + i * nv;
            const real* G = gam.d.data();
#pragma omp parallel for schedule(static)
            for (long q = 0; q < (long)nv; q++) {
                real v = V[q] + dt * W[q];
                real u = U[q] + dt * v;
                V[q] = v;
                U[q] = u;
                W[q] = u + G[q] * v;
            }
        }
        int ones[3] = {1, 1, 1};
        field_io("<>", "vx", vv.c(1));
        field_io("<>", "vy", vv.c(2));
        field_io("<>", "vz", vv.c(3));
        if (imod(it, itstats) == 0) {
            vector_norm(s1.v(), vv, i1core, i2core, ones);
            set_halo(s1.v(), R(-1), i1core, i2core);
            vmax = maxval(s1.v());
        }
        field_io(">", "vm2", s1.v());
        field_io("<>", "ux", uu.c(1));
        field_io("<>", "uy", uu.c(2));
        field_io("<>", "uz", uu.c(3));
        if (imod(it, itstats) == 0) {
            vector_norm(s1.v(), uu, i1core, i2core, ones);
            set_halo(s1.v(), R(-1), i1core, i2core);
            umax = maxval(s1.v());
        }
        field_io(">", "um2", s1.v());
        if (ifn) {
            for (int i = 0; i < 3; i++) for (size_t q = 0; q < np; q++) t1.d[q + i * np] = vv.d[q2[q] + i * nv] - vv.d[q1[q] + i * nv];
            for (size_t q = 0; q < np; q++) {
                f1.d[q] = std::sqrt(t1.d[q] * t1.d[q] + t1.d[q + np] * t1.d[q + np] + t1.d[q + 2 * np] * t1.d[q + 2 * np]);
                sl.d[q] = sl.d[q] + dt * f1.d[q];
                psv.d[q] = std::max(psv.d[q], f1.d[q]);
            }
            if (svtol > R(0)) {
                for (size_t q = 0; q < np; q++) {
                    real a = f1.d[q], b = f2.d[q];
                    if (a >= svtol && trup.d[q] > R(1e8)) trup.d[q] = tm - dt * (R(0.5) + (svtol - a) / (b - a));
                    if (a >= svtol) tarr.d[q] = R(1e9);
                    if (a < svtol && b >= svtol) tarr.d[q] = tm - dt * (R(0.5) + (svtol - a) / (b - a));
                }
            }
            for (int i = 0; i < 3; i++) for (size_t q = 0; q < np; q++) t2.d[q + i * np] = uu.d[q2[q] + i * nv] - uu.d[q1[q] + i * nv];
            for (size_t q = 0; q < np; q++) f2.d[q] = std::sqrt(t2.d[q] * t2.d[q] + t2.d[q + np] * t2.d[q + np] + t2.d[q + 2 * np] * t2.d[q + 2 * np]);
            field_io(">", "svx", t1.c(1));
            field_io(">", "svy", t1.c(2));
            field_io(">", "svz", t1.c(3));
            field_io(">", "svm", f1.v());
            field_io(">", "psv", psv.v());
            field_io(">", "sux", t2.c(1));
            field_io(">", "suy", t2.c(2));
            field_io(">", "suz", t2.c(3));
            field_io(">", "sum", f2.v());
            field_io(">", "sl", sl.v());
            field_io(">", "trup", trup.v());
            field_io(">", "tarr", tarr.v());
            set_halo(f1.v(), R(-1), i1core, i2core);
            set_halo(f2.v(), R(-1), i1core, i2core);
            set_halo(tarr.v(), R(-1), i1core, i2core);
            svmax = maxval(f1.v());
            sumax = maxval(f2.v());
            slmax = maxval(sl.v());
            tarrmax = maxval(tarr.v());
        }
    }

    // PML slab memory element: slab s (0..5 -> g1..g6 / p1..p6), position (j,k,l), comp ic
    // sord/stress.f90:6-255
    void step_stress() {
        set_halo(s1.v(), R(0), i1cell, i2cell);
        size_t nv = (size_t)nm[0] * nm[1] * nm[2];
        for (int ic = 1; ic <= 3; ic++)
            for (int iid = 1; iid <= 3; iid++) {
                int id = imod(ic + iid - 1, 3) + 1;
                int i1[3], i2[3];
                for (int i = 0; i < 3; i++) { i1[i] = imax(i1pml[i] + 1, i1cell[i]); i2[i] = imin(i2pml[i] - 2, i2cell[i]); }
                diff_nc(s1.v(), w1, ic, id, i1, i2, xx);
                if (npml > 0) {
                    for (int i = 0; i < 3; i++) {
                        if (id == i + 1) continue;
                        for (int d = 0; d < 3; d++) { i1[d] = i1cell[d]; i2[d] = i2cell[d]; }
                        i2[i] = imin(i2[i], i1pml[i]);
                        diff_nc(s1.v(), uu, ic, id, i1, i2, xx);
                        for (int d = 0; d < 3; d++) { i1[d] = i1cell[d]; i2[d] = i2cell[d]; }
                        i1[i] = imax(i1[i], i2pml[i] - 1);
                        diff_nc(s1.v(), uu, ic, id, i1, i2, xx);
                    }
                    int d = id - 1;
                    A4* gn[3] = {&g1, &g2, &g3};
                    A4* gf[3] = {&g4, &g5, &g6};
                    for (int q = 0; q < 3; q++) { i1[q] = i1cell[q]; i2[q] = i2cell[q]; }
                    i2[d] = imin(i2[d], i1pml[d]);
                    diff_nc(s1.v(), vv, ic, id, i1, i2, xx);
                    if (i1[0] <= i2[0] && i1[1] <= i2[1] && i1[2] <= i2[2])
                        for (int l = i1[2]; l <= i2[2]; l++)
                            for (int k = i1[1]; k <= i2[1]; k++)
                                for (int j = i1[0]; j <= i2[0]; j++) {
                                    int pos[3] = {j, k, l};
                                    int ii = pos[d] - i1[d] + 1;
                                    int p = pos[d] + nnoff[d];
                                    int gp[3] = {j, k, l}; gp[d] = ii;
                                    real& G = (*gn[d])(gp[0], gp[1], gp[2], ic);
                                    s1(j, k, l) = DC2(p) * s1(j, k, l) + DC1(p) * G;
                                    G = s1(j, k, l);
                                }
                    for (int q = 0; q < 3; q++) { i1[q] = i1cell[q]; i2[q] = i2cell[q]; }
                    i1[d] = imax(i1[d], i2pml[d] - 1);
                    diff_nc(s1.v(), vv, ic, id, i1, i2, xx);
                    if (i1[0] <= i2[0] && i1[1] <= i2[1] && i1[2] <= i2[2])
                        for (int l = i1[2]; l <= i2[2]; l++)
                            for (int k = i1[1]; k <= i2[1]; k++)
                                for (int j = i1[0]; j <= i2[0]; j++) {
                                    int pos[3] = {j, k, l};
                                    int ii = i2[d] - pos[d] + 1;
                                    int p = nn[d] - pos[d] - nnoff[d];
                                    int gp[3] = {j, k, l}; gp[d] = ii;
                                    real& G = (*gf[d])(gp[0], gp[1], gp[2], ic);
                                    s1(j, k, l) = DC2(p) * s1(j, k, l) + DC1(p) * G;
                                    G = s1(j, k, l);
                                }
                }
                int i = 6 - ic - id;
                real* S = s1.d.data();
                if (ic < id) { real* W = w2.d.data() + (i - 1) * nv; for (size_t q = 0; q < nv; q++) W[q] = R(0.5) * S[q]; }
                else if (ic > id) { real* W = w2.d.data() + (i - 1) * nv; for (size_t q = 0; q < nv; q++) W[q] = W[q] + R(0.5) * S[q]; }
                else { real* W = w1.d.data() + (ic - 1) * nv; for (size_t q = 0; q < nv; q++) W[q] = S[q]; }
            }
        if (source == "potency") finite_source();
        field_io("<>", "pxx", w1.c(1));
        field_io("<>", "pyy", w1.c(2));
        field_io("<>", "pzz", w1.c(3));
        field_io("<>", "pyz", w2.c(1));
        field_io("<>", "pzx", w2.c(2));
        field_io("<>", "pxy", w2.c(3));
        for (size_t q = 0; q < nv; q++) s1.d[q] = lam.d[q] * (w1.d[q] + w1.d[q + nv] + w1.d[q + 2 * nv]);
        for (int i = 0; i < 3; i++)
            for (size_t q = 0; q < nv; q++) {
                w1.d[q + i * nv] = R(2) * mu.d[q] * w1.d[q + i * nv] + s1.d[q];
                w2.d[q + i * nv] = R(2) * mu.d[q] * w2.d[q + i * nv];
            }
        if (source == "moment") finite_source();
        field_io("<>", "mxx", w1.c(1));
        field_io("<>", "myy", w1.c(2));
        field_io("<>", "mzz", w1.c(3));
        field_io("<>", "myz", w2.c(1));
        field_io("<>", "mzx", w2.c(2));
        field_io("<>", "mxy", w2.c(3));
        for (int i = 0; i < 3; i++)
            for (size_t q = 0; q < nv; q++) {
                w1.d[q + i * nv] = w1.d[q + i * nv] * vc.d[q];
                w2.d[q + i * nv] = w2.d[q + i * nv] * vc.d[q];
            }
        field_io("<>", "wxx", w1.c(1));
        field_io("<>", "wyy", w1.c(2));
        field_io("<>", "wzz", w1.c(3));
        field_io("<>", "wyz", w2.c(1));
        field_io("<>", "wzx", w2.c(2));
        field_io("<>", "wxy", w2.c(3));
        if (imod(it, itstats) == 0) {
            int ones[3] = {1, 1, 1};
            tensor_norm(s1.v(), w1, w2, i1core, i2core, ones);
            set_halo(s1.v(), R(-1), i1core, i2core);
            wmax = maxval(s1.v());
        }
        field_io(">", "wm2", s1.v());
    }

    // sord/acceleration.f90:6-265
    void step_accel() {
        set_halo(s1.v(), R(0), i1node, i2node);
        size_t nv = (size_t)nm[0] * nm[1] * nm[2];
        for (int ic = 1; ic <= 3; ic++)
            for (int iid = 1; iid <= 3; iid++) {
                int id = imod(ic + iid - 2, 3) + 1;
                int i1[3], i2[3];
                for (int i = 0; i < 3; i++) { i1[i] = i1node[i]; i2[i] = i2node[i]; }
                if (ic == id) diff_cn(s1.v(), w1, ic, id, i1, i2, xx);
                else diff_cn(s1.v(), w2, 6 - ic - id, id, i1, i2, xx);
                if (npml > 0) {
                    int d = id - 1;
                    A4* pn[3] = {&p1, &p2, &p3};
                    A4* pf[3] = {&p4, &p5, &p6};
                    int lo = i1[d], hi = imin(i2[d], i1pml[d]);
                    for (int pd = lo; pd <= hi; pd++) {
                        int ii = pd - i1[d] + 1, p = pd + nnoff[d];
                        slab_loop(d, pd, i1, i2, [&](int j, int k, int l) {
                            int gp[3] = {j, k, l}; gp[d] = ii;
                            real& P = (*pn[d])(gp[0], gp[1], gp[2], ic);
                            s1(j, k, l) = DN2(p) * s1(j, k, l) + DN1(p) * P;
                            P = P + dt * s1(j, k, l);
                        });
                    }
                    lo = imax(i1[d], i2pml[d]); hi = i2[d];
                    for (int pd = lo; pd <= hi; pd++) {
                        int ii = i2[d] - pd + 1, p = nn[d] - pd - nnoff[d] + 1;
                        slab_loop(d, pd, i1, i2, [&](int j, int k, int l) {
                            int gp[3] = {j, k, l}; gp[d] = ii;
                            real& P = (*pf[d])(gp[0], gp[1], gp[2], ic);
                            s1(j, k, l) = DN2(p) * s1(j, k, l) + DN1(p) * P;
                            P = P + dt * s1(j, k, l);
                        });
                    }
                }
                real* W = w1.d.data() + (ic - 1) * nv;
                const real* S = s1.d.data();
                if (ic == id) for (size_t q = 0; q < nv; q++) W[q] = S[q];
                else for (size_t q = 0; q < nv; q++) W[q] = W[q] + S[q];
            }
        if (hourglass[0] > R(0) || hourglass[1] > R(0)) {
            set_halo(s1.v(), R(0), i1cell, i2cell);
            set_halo(s2.v(), R(0), i1node, i2node);
            real dh2 = dt * hourglass[1];
            for (int i = 0; i < 3; i++)
                for (size_t q = 0; q < nv; q++) w2.d[q + i * nv] = hourglass[0] * uu.d[q + i * nv] + dh2 * vv.d[q + i * nv];
            for (int iq = 1; iq <= 4; iq++)
                for (int ic = 1; ic <= 3; ic++) {
                    int i1[3], i2[3];
                    for (int i = 0; i < 3; i++) { i1[i] = imax(i1pml[i], i1cell[i]); i2[i] = imin(i2pml[i] - 1, i2cell[i]); }
                    hourglass_nc(s1.v(), w2.c(ic), iq, i1, i2);
                    for (size_t q = 0; q < nv; q++) s1.d[q] = s1.d[q] * yy.d[q];
                    for (int i = 0; i < 3; i++) { i1[i] = imax(i1pml[i] + 1, i1node[i]); i2[i] = imin(i2pml[i] - 1, i2node[i]); }
                    hourglass_cn(s2.v(), s1.v(), iq, i1, i2);
                    if (hourglass[1] > R(0) && npml > 0) {
                        for (int i = 0; i < 3; i++) {
                            for (int q = 0; q < 3; q++) { i1[q] = i1cell[q]; i2[q] = i2cell[q]; }
                            i2[i] = imin(i2[i], i1pml[i]);
                            hourglass_nc(s1.v(), vv.c(ic), iq, i1, i2);
                            scale_region(i1, i2);
                            for (int q = 0; q < 3; q++) { i1[q] = i1cell[q]; i2[q] = i2cell[q]; }
                            i1[i] = imax(i1[i], i2pml[i] - 1);
                            hourglass_nc(s1.v(), vv.c(ic), iq, i1, i2);
                            scale_region(i1, i2);
                        }
                        for (int i = 0; i < 3; i++) {
                            for (int q = 0; q < 3; q++) { i1[q] = i1node[q]; i2[q] = i2node[q]; }
                            i2[i] = imin(i2[i], i1pml[i]);
                            hourglass_cn(s2.v(), s1.v(), iq, i1, i2);
                            for (int q = 0; q < 3; q++) { i1[q] = i1node[q]; i2[q] = i2node[q]; }
                            i1[i] = imax(i1[i], i2pml[i]);
                            hourglass_cn(s2.v(), s1.v(), iq, i1, i2);
                        }
                    }
                    real* W = w1.d.data() + (ic - 1) * nv;
                    for (size_t q = 0; q < nv; q++) W[q] = W[q] - s2.d[q];
                }
        }
        if (source == "force") finite_source();
        field_io("<", "fx", w1.c(1));
        field_io("<", "fy", w1.c(2));
        field_io("<", "fz", w1.c(3));
        vector_bc(w1, bc1, bc2, i1bc, i2bc);
        step_rupture();
        field_io(">", "fx", w1.c(1));
        field_io(">", "fy", w1.c(2));
        field_io(">", "fz", w1.c(3));
        for (int i = 0; i < 3; i++)
            for (size_t q = 0; q < nv; q++) w1.d[q + i * nv] = w1.d[q + i * nv] * mr.d[q];
        field_io("<>", "ax", w1.c(1));
        field_io("<>", "ay", w1.c(2));
        field_io("<>", "az", w1.c(3));
        if (imod(it, itstats) == 0) {
            int ones[3] = {1, 1, 1};
            vector_norm(s1.v(), w1, i1core, i2core, ones);
            set_halo(s1.v(), R(-1), i1core, i2core);
            amax = maxval(s1.v());
        }
        field_io(">", "am2", s1.v());
    }
    template <class F>
    void slab_loop(int d, int pd, const int* i1, const int* i2, F fn) {
        int lo[3] = {i1[0], i1[1], i1[2]}, hi[3] = {i2[0], i2[1], i2[2]};
        lo[d] = hi[d] = pd;
        for (int l = lo[2]; l <= hi[2]; l++)
            for (int k = lo[1]; k <= hi[1]; k++)
                for (int j = lo[0]; j <= hi[0]; j++) fn(j, k, l);
    }
    void scale_region(const int* i1, const int* i2) {
        real dh2 = dt * hourglass[1];
        for (int l = i1[2]; l <= i2[2]; l++)
            for (int k = i1[1]; k <= i2[1]; k++)
                for (int j = i1[0]; j <= i2[0]; j++) s1(j, k, l) = dh2 * yy(j, k, l) * s1(j, k, l);
    }

    // sord/statistics.f90:13-131
    void stats() {
        long long t3 = clock_ticks();
        bool fault = faultnormal != "no";
        int nq = fault ? 12 : 4;
        if (stats_init) {
            stats_init = false;
            prof.assign((size_t)4 * itio, 0);
            maxl.assign((size_t)nq * itio, R(0));
            if (fault) suml.assign((size_t)3 * itio, R(0));
            for (bool& b : stats_open) b = false;
        }
        if (imod(it, itstats) == 0) {
            stats_j++;
            int j = stats_j;
            real* M = maxl.data() + (size_t)nq * (j - 1);
            M[0] = amax; M[1] = vmax; M[2] = umax; M[3] = wmax;
            real val = -std::numeric_limits<real>::max();
            for (real v : maxl) val = std::max(val, v);
            for (int q = 0; q < 4; q++)
                if (M[q] != M[q]) val = M[q];
            if (val != val || val > std::numeric_limits<real>::max()) throw SordStop("NaN/Inf!");
            if (fault) {
                M[4] = samax; M[5] = svmax; M[6] = sumax; M[7] = slmax; M[8] = tsmax; M[9] = -tnmin; M[10] = tnmax; M[11] = tarrmax;
                real* S = suml.data() + (size_t)3 * (j - 1);
                S[0] = efric; S[1] = estrain; S[2] = moment;
            }
        }
        if (stats_j > 0 && (imod(it, itio) == 0 || it == nt)) {
            int j = stats_j;
            int m = nt / itstats, o = it / itstats - j;
            static const char* nmax[12] = {"amax", "vmax", "umax", "wmax", "samax", "svmax", "sumax", "slmax", "tsmax", "tnmin", "tnmax", "tarrmax"};
            std::vector<real> col(j);
            for (int q = 0; q < nq; q++) {
                for (int r = 0; r < j; r++) {
                    real v = maxl[(size_t)nq * r + q];
                    if (q < 4) v = std::sqrt(v);
                    if (q == 9) v = -v;
                    col[r] = v;
                }
                frio2(nullptr, stats_open[q], col.data(), 1, j, 'w', std::string("stats-") + nmax[q] + ".bin", m, o);
            }
            if (fault) {
                static const char* nsum[3] = {"efric", "estrain", "moment"};
                for (int q = 0; q < 3; q++) {
                    for (int r = 0; r < j; r++) col[r] = suml[(size_t)3 * r + q];
                    frio2(nullptr, stats_open[12 + q], col.data(), 1, j, 'w', std::string("stats-") + nsum[q] + ".bin", m, o);
                }
                for (int r = 0; r < j; r++) {
                    real v = suml[(size_t)3 * r + 2];
                    col[r] = v > R(0) ? (std::log10(v) - R(9.05)) / R(1.5) : R(-999);
                }
                frio2(nullptr, stats_open[15], col.data(), 1, j, 'w', "stats-mw.bin", m, o);
            }
            stats_j = 0;
        }
        timers[2] = clock_ticks() - t3;
        timers[3] = clock_ticks();
        int i = imod(it - 1, itio) + 1;
        for (int q = 0; q < 4; q++) prof[(size_t)4 * (i - 1) + q] = timers[q];
        if (i == itio || it == nt) {
            static const char* np_[4] = {"prof-halo.bin", "prof-io.bin", "prof-stats.bin", "prof-step.bin"};
            for (int q = 0; q < 4; q++) {
                std::vector<int32_t> col(i);
                for (int r = 0; r < i; r++) col[r] = (int32_t)prof[(size_t)4 * r + q];
                write_int_records(np_[q], col, nt, it - i, stats_open[16 + q]);
            }
        }
    }
    void write_int_records(const char* fn, const std::vector<int32_t>& v, int m, int o, bool& opened) {
        FILE* fp = (!opened && o == 0) ? fopen(fn, "wb") : fopen(fn, "r+b");
        if (!fp) throw SordStop(std::string("cannot open ") + fn);
        opened = true;
        fseek(fp, (long)(sizeof(int32_t) * (size_t)o), SEEK_SET);
        fwrite(v.data(), sizeof(int32_t), v.size(), fp);
        fclose(fp);
        if (o + (int)v.size() == m) opened = false;
    }

    // sord/sord.f90:24-47
    void run(const std::string& path) {
        clock0 = std::chrono::steady_clock::now();
        read_parameters(path);
        setup_dimensions();
        allocate_arrays();
        init_grid();
        init_material();
        init_pml();
        init_finite_source();
        init_rupture();
        resample_material();
        std::chrono::steady_clock::time_point tw = std::chrono::steady_clock::now();
        for (it = 1; it <= nt; it++) {
            if (it == timed_from + 1) tw = std::chrono::steady_clock::now();
            timers[0] = timers[1] = timers[2] = timers[3] = 0;
            step_time();
            step_stress();
            step_accel();
            stats();
        }
        if (timed_from >= 0) timed_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tw).count();
    }
};

int main(int argc, char** argv) {
    std::string path = "sord.in";
    int threads = 1, ntl = -1, tfrom = -1;
    bool w1g = false;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        if (a == "--threads" && i + 1 < argc) threads = atoi(argv[++i]);
        else if (a == "--nt-limit" && i + 1 < argc) ntl = atoi(argv[++i]);
        else if (a == "--timed-from" && i + 1 < argc) tfrom = atoi(argv[++i]);
        else if (a == "--w1-geometry") w1g = true;
        else path = a;
    }
#ifdef _OPENMP
    omp_set_num_threads(threads > 0 ? threads : 1);
#else
    (void)threads;
#endif
    Sord* s = new Sord();
    s->nt_limit = ntl;
    s->timed_from = tfrom;
    s->w1_geometry = w1g;
    try {
        auto t0 = std::chrono::steady_clock::now();
        s->run(path);
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        fprintf(stdout, "{\"oracle\": \"%s\", \"nt\": %d, \"nodes\": %lld, \"seconds\": %.6f, \"timed_from\": %d, \"timed_seconds\": %.6f, \"threads\": %d}\n",
                sizeof(real) == 4 ? "f32" : "f64", s->nt, (long long)s->nn[0] * s->nn[1] * s->nn[2], el, s->timed_from,
                s->timed_seconds, threads);
    } catch (SordStop& e) {
        fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
