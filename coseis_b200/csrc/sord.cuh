// Internal declarations of the B200 SORD solver (libsordgpu.so).
//
// Layout: every volume field is one FP32 array over the local block including
// its halo, nm = nn + 2*nhalo nodes per axis, j fastest (the Fortran
// column-major order of sord/globals.f90, so .bin slices need no transpose).
// Indices in kernels are 1-based like the Fortran so that every index range
// can be checked against the reference line it restates.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sordgpu.h"

namespace sordgpu {

struct SordError : std::runtime_error {
    int code;
    SordError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define SORD_CUDA(x)                                                                                  \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            throw ::sordgpu::SordError(SORD_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ----------------------------------------------------------------- params
// Values of sord.in (sord/globals.f90:59-68, input_output.f90:51-59).
struct Params {
    int bc1[3], bc2[3], debug, faultopening, i1pml[3], i2pml[3], itio, itstats, mpin, mpout;
    int n1expand[3], n2expand[3], nfieldio, npml, nproc3[3], nsource, nthread, ppml, shape[4];
    float affine[9], delta[4], gam_max, gam_min, gridnoise, hourglass[2], hypocenter[3];
    float rcrit, rexpand, rho_max, rho_min, slipvector[3], svtol, tm0, trelax, vdamp;
    float vp_max, vp_min, vpml, vrup, vs_max, vs_min;
    std::string source, faultnormal;
};

// One field-I/O operation (sord/input_output.f90:4-12, type t_io).
struct IoOp {
    std::string field, op, fname;
    char reg = 'n';
    int ii[4][3];  // [dim][start(1-based), stop, step]
    int nb = 1, ib = -1;
    float x1[3], x2[3], val = 0, tau = 0;
    int bufn = 0;
    float* dbuf = nullptr;     // device output buffer (bufn * nb)
    std::vector<float> hbuf;   // host staging of input / output records
    bool open = false;         // output file created (direct-access append state)
    // disk ops: floats per record in the file (the whole region) and the
    // offset of this process's part of it (nonzero in a partitioned run)
    long long grecl = 0, loff = 0;
    // the op as read from sord.in: `op` becomes "#" where this process holds
    // none of the region, op0 is the same on every part of a partitioned run
    std::string op0;
};

Params parse_sord_in(const std::string& text, std::vector<IoOp>& ops);

// ----------------------------------------------------------------- geometry
// Index regions of setup.f90:56-84 for the serial block (nnoff = -nhalo),
// passed by value to kernels.
struct Geom {
    int nn[3], nm[3], nhalo[3], nnoff[3];
    int i1bc[3], i2bc[3], i1core[3], i2core[3], i1node[3], i2node[3], i1cell[3], i2cell[3];
    int i1pml[3], i2pml[3];
    int npml;
    long long nv;   // nm0*nm1*nm2
    long long sy;   // nm0
    long long sz;   // nm0*nm1
    float dt, dx[3];
    float h;        // sign(1/12, product(dx))
    int ifn, irup;  // fault normal (1..3, 0 none) and fault index (local)
    __host__ __device__ long long idx(int j, int k, int l) const {
        return (long long)(j - 1) + sy * (long long)(k - 1) + sz * (long long)(l - 1);
    }
};

// PML slab memories (boundary_pml.f90:40-80): slab s = 0..2 near side of
// axis s (p1..p3 / g1..g3), 3..5 far side (p4..p6 / g4..g6).  Extents equal
// nm except thickness t along the slab axis; 3 components.
struct Slabs {
    float* p[6];
    float* g[6];
    int tp[6];  // node-slab thickness
    int tg[6];  // cell-slab thickness
};

// Rectilinear support-operator brackets (diff_nc_op.f90 / diff_cn_op.f90):
// bnc[a][t] = bracket of term t for direction a, identical at every real cell
// when the mesh is a tensor product (verified on the device at setup).
struct Brackets {
    float bnc[3][8];
    float bcn[3][8];
};

// Point injections into the strain/stress tensor (field_io '.' ops on
// p**/m** fields, finite sources) or into the force: applied in list order.
struct Inject {
    long long idx;  // linear index
    int comp;       // 0..2 diagonal / force component, 3..5 off-diagonal (yz, zx, xy)
    float inc;      // value added (val * trilinear weight, or -w*src)
};
static const int kMaxInject = 256;
static const int kInjectSlots = 4;  // 0 potency, 1 moment, 2 force, 3 field-I/O '.' ops
static const int kInjectRing = 16;  // uploads in flight per slot (the host runs that far ahead)
inline size_t inj_off(int slot, int r) { return ((size_t)slot * kInjectRing + (size_t)r) * kMaxInject; }

// Layout of the reduction scratch Device::red (16384 floats):
static const int kRedBad = 15;        // unsigned index: rectilinear check flag
static const int kRedRef = 32;        // float index: 48 reference brackets
static const int kRedReduce = 64;     // double index: region-reduction partials (2 x 1024)
static const int kRedEnergy = 2112;   // double index: efric, estrain, moment
static const int kRedPart = 2176;     // double index: fault energy partials (3 x 1024)
static const long long kRedFloats = 16384;

struct InjectList {
    const Inject* e;
    int n;
};

// Mesh classes of the fused step kernel: rectilinear (all support-operator
// brackets equal at every real cell), terrain (x = x(j), y = y(k), and the
// z-free direction's brackets constant), general.
enum { GEOM_RECT = 0, GEOM_TERRAIN = 1, GEOM_GENERAL = 2 };

struct StepArgs {
    Geom g;
    Brackets br;
    Brackets brh;      // br scaled by h (fast arithmetic)
    const float* x1d;  // terrain: x at nodes j = 1..nm0
    const float* y1d;  // terrain: y at nodes k = 1..nm1
    const float* x[3];
    const float* vin[3];
    const float* uin[3];
    float* vout[3];
    float* uout[3];
    float* aout[3];
    const float *gam, *mr, *lam, *mu, *vc, *yy;
    const float* pmlc;
    Slabs sl;
    float* gout[6];
    InjectList pot, mom, force;
    float hg1, dh2;
    int hourglass, hgvisc, fold, stats;
    unsigned* red;
    int segl;
    // interior kernel: tiles from node (jf, kf), output nodes up to
    // (jend, kend), node planes lf0..lf1; shell kernel: work items of six
    // ints (j0, k0, last j, last k, first plane, last plane)
    int jf, kf, jend, kend, lf0, lf1;
    const int* items;
    float negzero;  // -0.0, the addend of packed products (pair.cuh)
    // double-node fault: normal axis (0..2, -1 without a fault) and the
    // minus-side node index; nodes of planes firup and firup + 1 keep their
    // force in fout, unscaled, and their v, u are copied by the fold
    int fax, firup;
    float* fout[3];
};

#ifdef __CUDACC__
// 4-byte asynchronous global -> shared copies (cp.async) and their groups
__device__ __forceinline__ void cp_async4(float* smem, const float* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
#endif

// Device state of one handle.
struct Device {
    float* x[3] = {};
    float* v[3] = {};
    float* u[3] = {};
    float* w1n[3] = {};  // node role of w1: u + gam*v, then force, then acceleration
    float* sd[3] = {};   // cell role of w1: strain / stress diagonal
    float* so[3] = {};   // cell role of w2: strain / stress off-diagonal (yz, zx, xy)
    float *vc = nullptr, *mr = nullptr, *lam = nullptr, *mu = nullptr, *gam = nullptr, *yy = nullptr;
    float *s1 = nullptr, *s2 = nullptr;  // volume scratch (field-I/O, setup, magnitudes)
    float* pmlc = nullptr;               // dn1, dn2, dc1, dc2 (npml each)
    Slabs slabs{};
    float* vb[3] = {};                   // second v / u buffers of the fused step
    float* ub[3] = {};
    float* gb[6] = {};                   // second PML g buffers
    float* x1d = nullptr;                // terrain meshes: x(j), y(k)
    float* y1d = nullptr;
    float* red = nullptr;                // reduction scratch (uint bit patterns / doubles)
    Inject* inj = nullptr;               // device injection lists (3 * kMaxInject)
    // fault plane (nm with extent 1 along ifn)
    long long np = 0;
    float* fp = nullptr;                 // all fault arrays in one allocation
    // the 32 volume fields (x .. ub above) are carved from one block; from
    // 4 GiB up a plain cudaMalloc (vol_plain): growing the stream-ordered
    // pool by 26 GB took about 0.16 s and returning it as long again, a
    // cudaMalloc of the same size about 2 ms; smaller blocks come from the
    // pool, which concurrent handles reuse without synchronising the device
    void* vol = nullptr;
    bool vol_plain = false;
};

// Fault-plane arrays (dynamic_rupture.f90:22-63), offsets into Device::fp.
enum FaultArr {
    F_MUS, F_MUD, F_DC, F_CO, F_AREA, F_RHYPO, F_LAMF, F_MUF, F_SL, F_PSV, F_TRUP, F_TARR, F_TN, F_TS, F_F1, F_F2,
    F_NHAT, F_T0 = F_NHAT + 3, F_T1 = F_T0 + 3, F_T2 = F_T1 + 3, F_T3 = F_T2 + 3, F_COUNT = F_T3 + 3
};

struct Solver;

// kernel classes for sord_kernel_times
enum { KC_TIME = 0, KC_STRESS = 1, KC_ACCEL = 2, KC_MASS = 3, KC_FAULT = 4, KC_IO = 5, KC_OTHER = 6, KC_FUSED = 7 };

// kernels.cu entry points
void launch_time_update(Solver& s, bool stats);
void launch_stress(Solver& s, const InjectList& pot, const InjectList& mom, bool hooke);
void launch_hooke(Solver& s);
void launch_volume_scale(Solver& s);
void launch_accel(Solver& s, bool mass, bool stats, const InjectList& force);
void launch_mass(Solver& s, bool stats);
void launch_vector_bc(Solver& s, float* const f[3], const int* bc1, const int* bc2, const int* i1, const int* i2);
void launch_scalar_bc(Solver& s, float* f, const int* fn, const int* bc1, const int* bc2, const int* i1, const int* i2);
void launch_inject(Solver& s, float* const f[6], const InjectList& l);
struct FusedPlan;
void fused_free(Solver& s);
void launch_fused(Solver& s, const InjectList& pot, const InjectList& mom, const InjectList& force,
                  const std::vector<Inject>& hpot, const std::vector<Inject>& hmom, const std::vector<Inject>& hforce,
                  bool fold, bool write_a,
                  bool stats);

// setup.cu
void setup_all(Solver& s);
// fault.cu
void fault_time_pre(Solver& s);
void fault_time_post(Solver& s);
void fault_rupture(Solver& s);
void fault_rupture_fused(Solver& s);
void fault_fold(Solver& s);
// fieldio.cu
struct FieldView {
    float* p;
    int n[3];
};
void field_io(Solver& s, const char* passes, const char* field, FieldView f);
void field_io_flush_all(Solver& s);
InjectList upload_inject(Solver& s, int slot, const std::vector<Inject>& e);  // through the slot's ring (api.cu)
void halo_exchange(Solver& s, float* const* fields, int nf);  // halo planes along l from the neighbouring parts
void all_reduce(Solver& s, double* vals, int n, int op);      // over the parts: op 0 max, 1 sum
void writer_drain(Solver& s);  // every queued output record on disk; throws the first write error
void writer_free(Solver& s);
bool field_active(Solver& s, const char* field, char pass);
// cells (or nodes) of a '.' op with their trilinear weights and the
// weights' derivatives with respect to the op's position (adjoint)
struct PointWeight {
    long long idx;  // index into the field
    double r;       // trilinear weight
    double dr[3];   // d r / d x1, x1 in node-index units
};
bool point_weights(Solver& s, IoOp& io, const FieldView& f, std::vector<PointWeight>& out);
float host_time_function(const std::string& pulse, float t, float dt, float tau);

// misc device helpers (util.cu)
void dev_fill(Solver& s, float* p, long long n, float v);
void dev_copy(Solver& s, float* dst, const float* src, long long n);
void dev_set_halo(Solver& s, FieldView f, float r, const int* i1, const int* i2);
float dev_reduce_max(Solver& s, FieldView f, const int* i1, const int* i2);  // max over region
float dev_reduce_min(Solver& s, FieldView f, const int* i1, const int* i2);
double dev_reduce_sum_d(Solver& s, FieldView f, const int* i1, const int* i2);
void dev_vector_norm(Solver& s, float* dst, float* const w[3], const int* i1, const int* i2, const int* di);
void dev_tensor_norm(Solver& s, float* dst, float* const a[3], float* const b[3], const int* i1, const int* i2, const int* di);
void dev_rinvert(Solver& s, float* p, long long n);

struct Solver {
    Params prm;
    std::vector<IoOp> ops;
    Geom g{};
    Device d{};
    Brackets br{};
    bool rect = false;        // rectilinear fast path verified
    int geom = GEOM_GENERAL;  // mesh class of the fused kernel
    bool use_fused = true;    // fused step kernel allowed (SORD_FUSED=0 disables)
    int arith = 0;            // interior step arithmetic: 0 reference order, 1 fast (SORD_ARITHMETIC=fast)
    bool folded = false;      // previous step already applied this step's leapfrog update
    std::string workdir;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_step_ms = 0;
    long long launches = 0;
    // optional per-kernel device timing (sord_set_profiling): class id per
    // launch, events recorded around the launch on the solver stream
    bool profiling = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_ev;
    double kernel_ms[8] = {};
    long long kernel_n[8] = {};
    void prof_begin(int cls, cudaEvent_t* e0);
    void prof_end(int cls, cudaEvent_t e0);
    void prof_collect();
    // time
    float tm = 0;
    int it = 0, nt = 0;
    uint64_t rng_calls = 0;
    // statistics module (statistics.f90:124-130)
    float amax = 0, vmax = 0, umax = 0, wmax = 0, samax = 0, svmax = 0, sumax = 0, slmax = 0;
    float tsmax = 0, tnmin = 0, tnmax = 0, tarrmax = 0;
    double efric = 0, estrain = 0, moment = 0;
    bool stats_init = true;
    int stats_j = 0;
    std::vector<double> maxl, suml;
    std::vector<int32_t> prof;
    long long timers[4] = {0, 0, 0, 0};
    bool stats_open[20] = {};
    double last_stats[16] = {};
    // PML coefficients on the host (boundary_pml.f90:20-33)
    std::vector<float> dn1, dn2, dc1, dc2;
    // finite source (kinematic_source.f90:4-6)
    std::vector<int> src_nt;
    std::vector<float> src_xi[3], src_dt, src_t0, src_w1[3], src_w2[3], src_history;
    // injection staging (pinned): one slot per list
    Inject* hinj = nullptr;
    // volume file input on the device (fieldio.cu): staging record and two
    // pinned chunk buffers for the file reads
    float* d_stage = nullptr;
    size_t stage_cap = 0;
    float* pin_io[8] = {};     // pinned chunks of the whole-volume input readers
    cudaEvent_t pin_ev[8] = {};
    int rec_slot = 0;          // next chunk buffer for a time-varying input record
    // work decomposition of the fused step kernels (fused.cu)
    FusedPlan* fplan = nullptr;
    struct AdjointState* adj = nullptr;  // checkpoints and adjoint fields (adjoint.cu)
    struct OutWriter* writer = nullptr;  // output-record writer thread (fieldio.cu)
    // partitioned run (sord_create_part): part `part` of `nparts` slabs along
    // l, the caller's halo-exchange and reduction callbacks, and the device
    // buffers of the exchange (send / receive planes below and above)
    int part = 0, nparts = 1;
    sord_halo_fn halo_fn = nullptr;
    sord_reduce_fn reduce_fn = nullptr;
    void* cb_ctx = nullptr;
    float* xbuf = nullptr;
    size_t xcap = 0;
    bool mem_attached = false;  // holds a reference on the device's memory pool
    cudaEvent_t inj_done[kInjectSlots][kInjectRing] = {};
    int inj_ring[kInjectSlots] = {};
    // fault bookkeeping
    int fn3[3] = {0, 0, 0};
    float* fa(int a) const { return d.fp + (long long)a * d.np; }
    std::string err;

    long long clock0_us = 0;
    long long clock_us() const;
    std::string path(const std::string& f) const;

    void step(bool last_in_call = true);
    void step_general(bool st);
    bool fusable(int step) const;
    void stats();
    void write_stats(const std::string& name, const std::vector<float>& col, int m, int o, bool& opened);
    void destroy();
};

void smem_limit(const void* func, int bytes);
void adjoint_free(Solver& s);
int adjoint_segment(Solver& s, int seg);
void adjoint_begin(Solver& s, int seg, int snaps);
const std::vector<int>& adjoint_stops(Solver& s);
long long binomial_cost(int l, int s);
void adjoint_checkpoint(Solver& s);
void adjoint_backward(Solver& s, int nrec, const char* const* files, const float* const* dtrace, const int* ntrace,
                      float* glam, float* gmu, float* gyy, float* gmr, double* gmom, int nmom);
void adjoint_source_gradients(Solver& s, double* gx, double* gt, int nmom);
void mem_attach(int device);
void mem_detach(int device);
void mem_trim(int device);
cudaError_t dev_malloc(Solver& s, void** p, size_t bytes);
void dev_free(Solver& s, void* p);
void* pinned_get(size_t bytes);
void pinned_put(void* p);

// cell / node counts for launches
inline unsigned div_up(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace sordgpu
