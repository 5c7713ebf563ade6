// C ABI (include/sordgpu.h), sord.in parser and the per-step orchestration
// (sord/sord.f90:39-47, statistics.f90:13-131).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <sstream>
#include <thread>
#include <vector>
#include <atomic>
#include <mutex>
#include <algorithm>

#include "sord.cuh"

namespace sordgpu {

float host_time_function(const std::string& pulse, float t, float dt, float tau);
bool point_injection(Solver& s, IoOp& io, const FieldView& f, int comp, std::vector<Inject>& out);
void probes_free(Solver& s);

// sord.in: the first line holds the values of the sorted parameter keys, one
// field-I/O op per following line (cst/sord.py:538-544,
// input_output.f90:51-92).  i1pml/i2pml arrive as the Python bounds [i1, i2)
// of the non-PML region; they are stored as the last near-side and the first
// far-side PML node (1-based), i.e. i1pml = i1 and i2pml = i2 + 1, which is
// the convention the PML loops of stress.f90 / acceleration.f90 index with
// (input_output.f90:62 converts i1pml only, so every face would get one
// extra damped layer read from past the end of the coefficient arrays).
Params parse_sord_in(const std::string& str, std::vector<IoOp>& ops) {
    Params P;
    size_t nl = str.find('\n');
    std::istringstream h(str.substr(0, nl));
    auto rd = [&](auto& x) {
        if (!(h >> x)) throw SordError(SORD_E_PARAM, "Error reading sord.in parameters");
    };
    for (auto& a : P.affine) rd(a);
    for (auto& a : P.bc1) rd(a);
    for (auto& a : P.bc2) rd(a);
    rd(P.debug);
    for (auto& a : P.delta) rd(a);
    rd(P.faultnormal); rd(P.faultopening); rd(P.gam_max); rd(P.gam_min); rd(P.gridnoise);
    for (auto& a : P.hourglass) rd(a);
    for (auto& a : P.hypocenter) rd(a);
    for (auto& a : P.i1pml) rd(a);
    for (auto& a : P.i2pml) rd(a);
    rd(P.itio); rd(P.itstats); rd(P.mpin); rd(P.mpout);
    for (auto& a : P.n1expand) rd(a);
    for (auto& a : P.n2expand) rd(a);
    rd(P.nfieldio); rd(P.npml);
    for (auto& a : P.nproc3) rd(a);
    rd(P.nsource); rd(P.nthread); rd(P.ppml); rd(P.rcrit); rd(P.rexpand); rd(P.rho_max); rd(P.rho_min);
    for (auto& a : P.shape) rd(a);
    for (auto& a : P.slipvector) rd(a);
    rd(P.source); rd(P.svtol); rd(P.tm0); rd(P.trelax); rd(P.vdamp); rd(P.vp_max); rd(P.vp_min); rd(P.vpml);
    rd(P.vrup); rd(P.vs_max); rd(P.vs_min);
    if (P.faultnormal.size() > 2) P.faultnormal = P.faultnormal.substr(0, 2);
    for (int i = 0; i < 3; i++) P.i2pml[i] += 1;
    if (P.itstats < 1 || P.itio < 1) throw SordError(SORD_E_PARAM, "Error in itstats / itio");
    std::istringstream b(nl == std::string::npos ? std::string() : str.substr(nl + 1));
    ops.resize(P.nfieldio);
    for (int j = 0; j < P.nfieldio; j++) {
        IoOp& io = ops[j];
        std::string reg;
        if (!(b >> io.field >> reg)) throw SordError(SORD_E_PARAM, "Error reading sord.in field i/o");
        io.reg = reg[0];
        for (int d = 0; d < 4; d++)
            for (int c = 0; c < 3; c++) b >> io.ii[d][c];
        b >> io.nb;
        for (auto& a : io.x1) b >> a;
        for (auto& a : io.x2) b >> a;
        b >> io.val >> io.tau >> io.op >> io.fname;
        if (!b) throw SordError(SORD_E_PARAM, "Error reading sord.in field i/o");
        if (io.field.size() > 4) io.field = io.field.substr(0, 4);
        for (int d = 0; d < 4; d++) {
            io.ii[d][0] += 1;
            if (io.ii[d][2] < 1) throw SordError(SORD_E_PARAM, "Error in i/o step");
        }
        if (io.nb < 1) io.nb = 1;
        io.ib = -1;
        io.op0 = io.op;
    }
    return P;
}

long long Solver::clock_us() const {
    return (long long)std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now().time_since_epoch()).count() -
           clock0_us;
}

std::string Solver::path(const std::string& f) const {
    if (f.empty() || f[0] == '/' || workdir.empty()) return f;
    return workdir + "/" + f;
}

static FieldView vol(Solver& s, float* p) {
    FieldView f;
    f.p = p;
    for (int i = 0; i < 3; i++) f.n[i] = s.g.nm[i];
    return f;
}

static bool any_pass(Solver& s, const char* const* names, int n, char pass) {
    for (int i = 0; i < n; i++)
        if (field_active(s, names[i], pass)) return true;
    return false;
}

static bool bc_noop(const Params& P) {
    for (int i = 0; i < 3; i++)
        if (P.bc1[i] % 10 != 0 || P.bc2[i] % 10 != 0) return false;
    return true;
}
static bool bc_cells_noop(const Params& P) {
    for (int i = 0; i < 3; i++) {
        int a = std::abs(P.bc1[i] % 10), b = std::abs(P.bc2[i] % 10);
        if (a == 2 || a == 4 || b == 2 || b == 4) return false;
    }
    return true;
}

// Finite-source entries (kinematic_source.f90:66-118) for this step.
static void finite_source_entries(Solver& s, std::vector<Inject>& out) {
    const Params& P = s.prm;
    const Geom& g = s.g;
    if (P.nsource == 0) return;
    long itoff = 0;
    bool force = P.source == "force";
    for (int isrc = 0; isrc < std::abs(P.nsource); isrc++) {
        int i = (int)std::floor((s.tm - s.src_t0[isrc]) / s.src_dt[isrc]) + 1;
        float xi[3] = {s.src_xi[0][isrc], s.src_xi[1][isrc], s.src_xi[2][isrc]};
        int i1[3], i2[3];
        for (int d = 0; d < 3; d++) {
            int fl = (int)std::floor(xi[d]);
            if (force) { i1[d] = std::max(g.i1node[d], fl); i2[d] = std::min(g.i2node[d], fl + 1); }
            else { i1[d] = std::max(g.i1cell[d], fl); i2[d] = std::min(g.i2cell[d], fl + 1); }
        }
        if (i >= 0 && i2[0] >= i1[0] && i2[1] >= i1[1] && i2[2] >= i1[2]) {
            i = std::min(i, s.src_nt[isrc] - 1);
            float t = s.src_t0[isrc] + s.src_dt[isrc] * (float)(i - 1);
            float hh = std::min(1.0f, (s.tm - t) / s.src_dt[isrc]);
            if (i == 0) hh = hh * s.src_history[itoff];
            else hh = (1.0f - hh) * s.src_history[itoff + i - 1] + hh * s.src_history[itoff + i];
            for (int l = i1[2]; l <= i2[2]; l++)
                for (int k = i1[1]; k <= i2[1]; k++)
                    for (int j = i1[0]; j <= i2[0]; j++) {
                        float w = hh * ((1.0f - std::fabs(xi[0] - (float)j)) * (1.0f - std::fabs(xi[1] - (float)k)) * (1.0f - std::fabs(xi[2] - (float)l)));
                        for (int c = 0; c < 3; c++) {
                            Inject e;
                            e.idx = g.idx(j, k, l);
                            if (force) {
                                e.comp = c; e.inc = w * s.src_w1[c][isrc]; out.push_back(e);
                            } else {
                                e.comp = c; e.inc = -(w * s.src_w1[c][isrc]); out.push_back(e);
                                e.comp = 3 + c; e.inc = -(w * s.src_w2[c][isrc]); out.push_back(e);
                            }
                        }
                    }
        }
        itoff += s.src_nt[isrc];
    }
}

static const char* kPot[6] = {"pxx", "pyy", "pzz", "pyz", "pzx", "pxy"};
static const char* kMom[6] = {"mxx", "myy", "mzz", "myz", "mzx", "mxy"};
static const char* kStr[6] = {"wxx", "wyy", "wzz", "wyz", "wzx", "wxy"};
static const char* kForce[3] = {"fx", "fy", "fz"};
static const char* kAcc[3] = {"ax", "ay", "az"};
static const char* kVel[3] = {"vx", "vy", "vz"};
static const char* kDis[3] = {"ux", "uy", "uz"};

// Are all ops firing now on these six tensor fields '.' injections that a
// fused kernel can apply?  Collect them in hook order if so.
static bool tensor_point_ops(Solver& s, const char* const* names, std::vector<Inject>& out) {
    for (int c = 0; c < 6; c++)
        for (auto& io : s.ops) {
            int it1 = io.ii[3][0], it2 = io.ii[3][1], dit = io.ii[3][2];
            if (s.it > it2 || io.op[0] == '#' || s.it < it1 || ((s.it - it1) % dit) != 0 || io.field != names[c]) continue;
            if (io.op != ".") return false;
        }
    if (!bc_cells_noop(s.prm)) return false;
    for (int c = 0; c < 6; c++)
        for (auto& io : s.ops) {
            int it1 = io.ii[3][0], it2 = io.ii[3][1], dit = io.ii[3][2];
            if (s.it > it2 || io.op[0] == '#' || s.it < it1 || ((s.it - it1) % dit) != 0 || io.field != names[c]) continue;
            point_injection(s, io, vol(s, s.d.sd[0]), c, out);
        }
    return true;
}

InjectList upload_inject(Solver& s, int slot, const std::vector<Inject>& e) {
    if ((int)e.size() > kMaxInject) throw SordError(SORD_E_PARAM, "too many point injections in one step");
    if (e.empty()) return InjectList{s.d.inj + inj_off(slot, 0), 0};
    // a ring of staging buffers per slot: the copy that last used buffer r
    // (kInjectRing uploads ago) must have completed before it is refilled
    const int r = s.inj_ring[slot];
    s.inj_ring[slot] = (r + 1) % kInjectRing;
    Inject* h = s.hinj + inj_off(slot, r);
    SORD_CUDA(cudaEventSynchronize(s.inj_done[slot][r]));
    std::memcpy(h, e.data(), sizeof(Inject) * e.size());
    SORD_CUDA(cudaMemcpyAsync(s.d.inj + inj_off(slot, r), h, sizeof(Inject) * e.size(), cudaMemcpyHostToDevice, s.stream));
    SORD_CUDA(cudaEventRecord(s.inj_done[slot][r], s.stream));
    return InjectList{s.d.inj + inj_off(slot, r), (int)e.size()};
}

// One forward step n with no field-I/O hook: leapfrog update (unless the
// caller has done it), then the fused stress/force/acceleration step with
// the point sources of step n, so that u, v and w1n = a are the state after
// step n; folded, the step also writes u, v of step n + 1 into ub, vb (which
// launch_fused then swaps in).  The
// adjoint recomputes checkpointed segments with it; every step of such a run
// is fusable, and the arithmetic is that of Solver::step.
void bare_step(Solver& s, int n, bool update, bool fold) {
    s.it = n;
    s.tm = s.prm.tm0 + s.g.dt * (float)(n - 1);
    if (update) launch_time_update(s, false);
    std::vector<Inject> pot, mom, frc;
    tensor_point_ops(s, kPot, pot);
    tensor_point_ops(s, kMom, mom);
    InjectList lp = upload_inject(s, 0, pot), lm = upload_inject(s, 1, mom), lf = upload_inject(s, 2, frc);
    launch_fused(s, lp, lm, lf, pot, mom, frc, fold, true, false);
    s.folded = fold;
}

// Injection entries of '.' moment op opi at step s.it (none if it does not fire).
void moment_entries(Solver& s, int opi, std::vector<Inject>& out) {
    IoOp& io = s.ops[opi];
    int it1 = io.ii[3][0], it2 = io.ii[3][1], dit = io.ii[3][2];
    if (io.op != "." || s.it > it2 || s.it < it1 || ((s.it - it1) % dit) != 0) return;
    for (int c = 0; c < 6; c++)
        if (io.field == kMom[c]) point_injection(s, io, vol(s, s.d.sd[0]), c, out);
}

static float read_max(Solver& s, int slot) {
    unsigned b;
    SORD_CUDA(cudaMemcpyAsync(&b, (unsigned*)s.d.red + slot, sizeof(unsigned), cudaMemcpyDeviceToHost, s.stream));
    SORD_CUDA(cudaStreamSynchronize(s.stream));
    float f;
    std::memcpy(&f, &b, sizeof f);
    return f;
}

static float norm_max(Solver& s, float* const w[3]) {
    int one[3] = {1, 1, 1};
    dev_vector_norm(s, s.d.s1, w, s.g.i1core, s.g.i2core, one);
    return dev_reduce_max(s, vol(s, s.d.s1), s.g.i1core, s.g.i2core);
}

// Fault-plane fields (the 'f' class of cst/sord.py:59-163): their outputs
// are read between the fault kernels, which run beside the fused kernel.
static bool fault_field(const std::string& f) {
    static const char* const names[] = {"mus", "mud", "dc", "co", "tn", "ts", "td", "sxx", "syy", "szz", "syz",
                                        "szx", "sxy", "nsx", "nsy", "nsz", "tx", "ty", "tz", "tsx", "tsy", "tsz",
                                        "tnm", "tsm", "fr", "sax", "say", "saz", "sam", "svx", "svy", "svz", "svm",
                                        "psv", "sux", "suy", "suz", "sum", "sl", "trup", "tarr"};
    for (const char* n : names)
        if (f == n) return true;
    return false;
}

// Can step `n` run as one fused kernel?  Every field-I/O op firing at that
// step must be an output of v, u, a or their magnitudes or of a fault-plane
// field (read between kernels) or a '.' point op on the potency / moment
// tensor (applied inside the kernel), and no boundary condition may copy
// planes.  A fault is finished by its own kernels around the fused one.
bool Solver::fusable(int n) const {
    if (!use_fused || !bc_noop(prm)) return false;
    for (auto& io : ops) {
        // the parts of a partitioned run decide alike: by the ops as read
        const std::string& op = nparts > 1 ? io.op0 : io.op;
        int it1 = io.ii[3][0], it2 = io.ii[3][1], dit = io.ii[3][2];
        if (n > it2 || op[0] == '#' || n < it1 || ((n - it1) % dit) != 0) continue;
        const std::string& f = io.field;
        char op2 = op.size() > 1 ? op[1] : ' ';
        bool out = op2 == '>';
        if (out) {
            bool ok = f == "vx" || f == "vy" || f == "vz" || f == "ux" || f == "uy" || f == "uz" || f == "ax" ||
                      f == "ay" || f == "az" || f == "vm2" || f == "um2" || f == "am2" || (g.ifn && fault_field(f));
            if (!ok) return false;
        } else {
            bool tensor = f[0] == 'p' || f[0] == 'm';
            if (!(tensor && op == "." && bc_cells_noop(prm))) return false;
        }
    }
    return true;
}

void Solver::step(bool last_in_call) {
    it++;
    for (auto& t : timers) t = 0;
    long long t_step = clock_us();
    const bool st = it % prm.itstats == 0;
    if (st) SORD_CUDA(cudaMemsetAsync(d.red, 0, sizeof(unsigned) * 8, stream));
    if (!fusable(it)) {
        folded = false;
        step_general(st);
        timers[3] = clock_us() - t_step;
        stats();
        return;
    }
    long long tio = 0;
    auto io = [&](const char* passes, const char* field, FieldView f) {
        long long t0 = clock_us();
        field_io(*this, passes, field, f);
        tio += clock_us() - t0;
    };
    // leapfrog update of this step, unless the previous fused step did it
    // (for all nodes but the fault's, which fault_fold advances)
    tm = prm.tm0 + g.dt * (float)(it - 1);
    if (!folded) {
        if (g.ifn) fault_time_pre(*this);
        launch_time_update(*this, false);
    } else if (g.ifn) {
        fault_fold(*this);
    }
    for (int i = 0; i < 3; i++) io("<>", kVel[i], vol(*this, d.v[i]));
    io(">", "vm2", vol(*this, d.s1));
    for (int i = 0; i < 3; i++) io("<>", kDis[i], vol(*this, d.u[i]));
    io(">", "um2", vol(*this, d.s1));
    if (g.ifn && !folded) fault_time_post(*this);
    std::vector<Inject> pot, mom, frc;
    if (prm.source == "potency") finite_source_entries(*this, pot);
    if (prm.source == "moment") finite_source_entries(*this, mom);
    if (prm.source == "force") finite_source_entries(*this, frc);
    tensor_point_ops(*this, kPot, pot);
    tensor_point_ops(*this, kMom, mom);
    // never fold across the end of a sord_step call: the state it leaves is
    // the state after its last step
    const bool fold = !last_in_call && it < nt && fusable(it + 1);
    const bool write_a = any_pass(*this, kAcc, 3, '>') || field_active(*this, "am2", '>') || it == nt;
    InjectList lp = upload_inject(*this, 0, pot), lm = upload_inject(*this, 1, mom), lf = upload_inject(*this, 2, frc);
    launch_fused(*this, lp, lm, lf, pot, mom, frc, fold, write_a, st);
    if (g.ifn) fault_rupture_fused(*this);
    folded = fold;
    if (nparts > 1) {
        // the halo planes of the state the step leaves: v, u of the next
        // step (folded) and a (the start of an unfolded next step advances
        // every plane with it) -- the reference's swap of w1 at
        // acceleration.f90:232, taken after the update
        float* F[9] = {d.v[0], d.v[1], d.v[2], d.u[0], d.u[1], d.u[2], d.w1n[0], d.w1n[1], d.w1n[2]};
        halo_exchange(*this, F, 9);
    }
    for (int i = 0; i < 3; i++) io("<>", kAcc[i], vol(*this, d.w1n[i]));
    io(">", "am2", vol(*this, d.s1));
    if (st) {
        amax = read_max(*this, 0);
        vmax = read_max(*this, 1);
        umax = read_max(*this, 2);
        wmax = read_max(*this, 3);
    }
    timers[1] = tio;
    timers[3] = clock_us() - t_step;
    stats();
}

// One step with separate kernels and every field-I/O hook of
// time_integration.f90, stress.f90 and acceleration.f90 in place.
void Solver::step_general(bool st) {
    Geom& G = g;
    long long tio = 0;
    auto io = [&](const char* passes, const char* field, FieldView f) {
        long long t0 = clock_us();
        field_io(*this, passes, field, f);
        tio += clock_us() - t0;
    };
    // ---- step_time (time_integration.f90:6-115)
    if (G.ifn) fault_time_pre(*this);
    tm = prm.tm0 + G.dt * (float)(it - 1);
    const bool vin = any_pass(*this, kVel, 3, '<') || any_pass(*this, kDis, 3, '<');
    launch_time_update(*this, st && !vin);
    for (int i = 0; i < 3; i++) io("<>", kVel[i], vol(*this, d.v[i]));
    if (st) vmax = vin ? norm_max(*this, d.v) : read_max(*this, 1);
    io(">", "vm2", vol(*this, d.s1));
    for (int i = 0; i < 3; i++) io("<>", kDis[i], vol(*this, d.u[i]));
    if (st) umax = vin ? norm_max(*this, d.u) : read_max(*this, 2);
    io(">", "um2", vol(*this, d.s1));
    if (G.ifn) fault_time_post(*this);
    // ---- step_stress (stress.f90:123-372)
    std::vector<Inject> pot, mom;
    if (prm.source == "potency") finite_source_entries(*this, pot);
    if (prm.source == "moment") finite_source_entries(*this, mom);
    bool fuse = tensor_point_ops(*this, kPot, pot) && tensor_point_ops(*this, kMom, mom) && !any_pass(*this, kStr, 6, '<');
    float* sdso[6] = {d.sd[0], d.sd[1], d.sd[2], d.so[0], d.so[1], d.so[2]};
    if (fuse) {
        InjectList lp = upload_inject(*this, 0, pot), lm = upload_inject(*this, 1, mom);
        launch_stress(*this, lp, lm, true);
        for (int i = 0; i < 6; i++) io("<>", kStr[i], vol(*this, sdso[i]));
        if (st) wmax = read_max(*this, 3);
    } else {
        InjectList none{d.inj, 0};
        launch_stress(*this, none, none, false);
        pot.clear();
        mom.clear();
        if (prm.source == "potency") { finite_source_entries(*this, pot); launch_inject(*this, sdso, upload_inject(*this, 0, pot)); }
        for (int i = 0; i < 6; i++) io("<>", kPot[i], vol(*this, sdso[i]));
        launch_hooke(*this);
        if (prm.source == "moment") { finite_source_entries(*this, mom); launch_inject(*this, sdso, upload_inject(*this, 1, mom)); }
        for (int i = 0; i < 6; i++) io("<>", kMom[i], vol(*this, sdso[i]));
        launch_volume_scale(*this);
        for (int i = 0; i < 6; i++) io("<>", kStr[i], vol(*this, sdso[i]));
        if (st) {
            int one[3] = {1, 1, 1};
            dev_tensor_norm(*this, d.s1, d.sd, d.so, G.i1core, G.i2core, one);
            wmax = dev_reduce_max(*this, vol(*this, d.s1), G.i1core, G.i2core);
        }
    }
    io(">", "wm2", vol(*this, d.s1));
    // ---- step_accel (acceleration.f90:6-265)
    std::vector<Inject> frc;
    if (prm.source == "force") finite_source_entries(*this, frc);
    const bool ain = any_pass(*this, kAcc, 3, '<');
    const bool fuse_a = G.ifn == 0 && bc_noop(prm) && !any_pass(*this, kForce, 3, '<') && !any_pass(*this, kForce, 3, '>');
    if (fuse_a) {
        launch_accel(*this, true, st && !ain, upload_inject(*this, 2, frc));
        // the halo of a = f m (pointwise from the force halo the reference
        // swaps, acceleration.f90:229-233; the mass halo came at setup)
        halo_exchange(*this, d.w1n, 3);
    } else {
        InjectList none{d.inj, 0};
        launch_accel(*this, false, false, none);
        float* w6[6] = {d.w1n[0], d.w1n[1], d.w1n[2], d.w1n[0], d.w1n[1], d.w1n[2]};
        if (!frc.empty()) launch_inject(*this, w6, upload_inject(*this, 2, frc));
        for (int i = 0; i < 3; i++) io("<", kForce[i], vol(*this, d.w1n[i]));
        launch_vector_bc(*this, d.w1n, prm.bc1, prm.bc2, G.i1bc, G.i2bc);
        if (G.ifn) fault_rupture(*this);
        halo_exchange(*this, d.w1n, 3);  // acceleration.f90:229-233
        for (int i = 0; i < 3; i++) io(">", kForce[i], vol(*this, d.w1n[i]));
        launch_mass(*this, st && !ain);
    }
    for (int i = 0; i < 3; i++) io("<>", kAcc[i], vol(*this, d.w1n[i]));
    if (st) amax = ain ? norm_max(*this, d.w1n) : read_max(*this, 0);
    io(">", "am2", vol(*this, d.s1));
    timers[1] = tio;
}

// statistics.f90:13-131 (maxima exact in FP32; energy sums in FP64)
void Solver::stats() {
    long long t3 = clock_us();
    bool fault = prm.faultnormal != "no";
    int nq = fault ? 12 : 4;
    if (stats_init) {
        stats_init = false;
        prof.assign((size_t)4 * prm.itio, 0);
        maxl.assign((size_t)nq * prm.itio, 0.0);
        if (fault) suml.assign((size_t)3 * prm.itio, 0.0);
    }
    if (it % prm.itstats == 0) {
        stats_j++;
        int j = stats_j;
        double* M = maxl.data() + (size_t)nq * (j - 1);
        M[0] = amax; M[1] = vmax; M[2] = umax; M[3] = wmax;
        all_reduce(*this, M, 4, 0);  // statistics.f90:78 over the parts
        bool bad = false;
        for (int q = 0; q < 4; q++)
            if (!(M[q] == M[q]) || M[q] > (double)std::numeric_limits<float>::max()) bad = true;
        if (bad) {
            char msg[256];
            snprintf(msg, sizeof msg, "NaN/Inf! amax %g vmax %g umax %g wmax %g", M[0], M[1], M[2], M[3]);
            throw SordError(SORD_E_NANINF, msg);
        }
        if (fault) {
            M[4] = samax; M[5] = svmax; M[6] = sumax; M[7] = slmax; M[8] = tsmax; M[9] = -tnmin; M[10] = tnmax; M[11] = tarrmax;
            double* S = suml.data() + (size_t)3 * (j - 1);
            S[0] = efric; S[1] = estrain; S[2] = moment;
        }
        for (int q = 0; q < 16; q++) last_stats[q] = 0;
        for (int q = 0; q < 4; q++) last_stats[q] = std::sqrt(M[q]);
        if (fault) {
            for (int q = 4; q < 12; q++) last_stats[q] = M[q];
            last_stats[9] = -M[9];
            last_stats[12] = efric; last_stats[13] = estrain; last_stats[14] = moment;
            last_stats[15] = moment > 0 ? (std::log10(moment) - 9.05) / 1.5 : -999;
        }
    }
    if (stats_j > 0 && (it % prm.itio == 0 || it == nt)) {
        int j = stats_j;
        int m = nt / prm.itstats, o = it / prm.itstats - j;
        static const char* nmax[12] = {"amax", "vmax", "umax", "wmax", "samax", "svmax", "sumax", "slmax", "tsmax", "tnmin", "tnmax", "tarrmax"};
        std::vector<float> col(j);
        IoOp dummy;
        for (int q = 0; q < nq; q++) {
            for (int r = 0; r < j; r++) {
                double v = maxl[(size_t)nq * r + q];
                float fv = (float)v;
                if (q < 4) fv = std::sqrt(fv);
                if (q == 9) fv = -fv;
                col[r] = fv;
            }
            write_stats(std::string("stats-") + nmax[q] + ".bin", col, m, o, stats_open[q]);
        }
        if (fault) {
            static const char* nsum[3] = {"efric", "estrain", "moment"};
            for (int q = 0; q < 3; q++) {
                for (int r = 0; r < j; r++) col[r] = (float)suml[(size_t)3 * r + q];
                write_stats(std::string("stats-") + nsum[q] + ".bin", col, m, o, stats_open[12 + q]);
            }
            for (int r = 0; r < j; r++) {
                double v = suml[(size_t)3 * r + 2];
                col[r] = v > 0 ? (float)((std::log10(v) - 9.05) / 1.5) : -999.0f;
            }
            write_stats("stats-mw.bin", col, m, o, stats_open[15]);
        }
        stats_j = 0;
    }
    timers[2] = clock_us() - t3;
    int i = (it - 1) % prm.itio + 1;
    for (int q = 0; q < 4; q++) prof[(size_t)4 * (i - 1) + q] = (int32_t)timers[q];
    if ((i == prm.itio || it == nt) && part == 0) {
        static const char* np_[4] = {"prof-halo.bin", "prof-io.bin", "prof-stats.bin", "prof-step.bin"};
        for (int q = 0; q < 4; q++) {
            std::vector<int32_t> col(i);
            for (int r = 0; r < i; r++) col[r] = prof[(size_t)4 * r + q];
            std::string fn = path(np_[q]);
            int o = it - i;
            FILE* fp = (!stats_open[16 + q] && o == 0) ? fopen(fn.c_str(), "wb") : fopen(fn.c_str(), "r+b");
            if (!fp) throw SordError(SORD_E_IO, std::string("cannot open ") + np_[q]);
            stats_open[16 + q] = true;
            fseek(fp, (long)(sizeof(int32_t) * (size_t)o), SEEK_SET);
            fwrite(col.data(), sizeof(int32_t), col.size(), fp);
            fclose(fp);
            if (o + i == nt) stats_open[16 + q] = false;
        }
    }
}

void Solver::write_stats(const std::string& name, const std::vector<float>& col, int m, int o, bool& opened) {
    if (part != 0) return;  // the master writes the statistics of all parts (statistics.f90:82)
    std::string fn = path(name);
    FILE* fp;
    if (!opened && o == 0) {
        fp = fopen(fn.c_str(), "rb");
        if (fp) { fclose(fp); throw SordError(SORD_E_IO, "file exists: " + name); }
        fp = fopen(fn.c_str(), "wb");
    } else {
        fp = fopen(fn.c_str(), "r+b");
    }
    if (!fp) throw SordError(SORD_E_IO, "cannot open " + name);
    opened = true;
    fseek(fp, (long)(sizeof(float) * (size_t)o), SEEK_SET);
    fwrite(col.data(), sizeof(float), col.size(), fp);
    fclose(fp);
    if (o + (int)col.size() == m) opened = false;
}

void Solver::prof_begin(int cls, cudaEvent_t* e0) {
    (void)cls;
    if (!profiling) return;
    SORD_CUDA(cudaEventCreate(e0));
    SORD_CUDA(cudaEventRecord(*e0, stream));
}
void Solver::prof_end(int cls, cudaEvent_t e0) {
    if (!profiling || !e0) return;
    cudaEvent_t e1;
    SORD_CUDA(cudaEventCreate(&e1));
    SORD_CUDA(cudaEventRecord(e1, stream));
    prof_ev.push_back({cls, {e0, e1}});
}
void Solver::prof_collect() {
    if (prof_ev.empty()) return;
    SORD_CUDA(cudaStreamSynchronize(stream));
    for (auto& p : prof_ev) {
        float ms = 0;
        SORD_CUDA(cudaEventElapsedTime(&ms, p.second.first, p.second.second));
        kernel_ms[p.first] += ms;
        kernel_n[p.first] += 1;
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    prof_ev.clear();
}

void Solver::destroy() {
    if (device >= 0) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    writer_free(*this);
    auto fr = [this](void* p) { dev_free(*this, p); };
    // the volume fields live in d.vol
    if (!d.vol_plain) fr(d.vol);
    fr(d.pmlc); fr(d.red); fr(d.inj); fr(d.fp);
    for (int i = 0; i < 6; i++) { fr(d.slabs.p[i]); fr(d.slabs.g[i]); fr(d.gb[i]); }
    fr(d.x1d); fr(d.y1d); fr(xbuf);
    for (auto& io : ops) fr(io.dbuf);
    probes_free(*this);
    fused_free(*this);
    adjoint_free(*this);
    for (auto& p : prof_ev) { cudaEventDestroy(p.second.first); cudaEventDestroy(p.second.second); }
    prof_ev.clear();
    pinned_put(hinj);
    fr(d_stage);
    for (int i = 0; i < (int)(sizeof(pin_io) / sizeof(pin_io[0])); i++) {
        pinned_put(pin_io[i]);
        if (pin_ev[i]) cudaEventDestroy(pin_ev[i]);
    }
    for (auto& row : inj_done)
        for (auto& e : row) if (e) cudaEventDestroy(e);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) {
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
    }
    if (d.vol && d.vol_plain) cudaFree(d.vol);
    d.vol = nullptr;
    if (mem_attached) mem_detach(device);
    mem_attached = false;
    hinj = nullptr;
    d_stage = nullptr;
    for (auto& p : pin_io) p = nullptr;
    d = Device{};
    stream = nullptr;
}

}  // namespace sordgpu

using namespace sordgpu;

struct sord_handle {
    Solver s;
};

// last error of a call without a handle, per host thread
static thread_local std::string g_create_error;

namespace sordgpu {
void set_global_error(const char* msg) { g_create_error = msg; }
}  // namespace sordgpu

static int fail(sord_handle* h, const std::exception& e) {
    const SordError* se = dynamic_cast<const SordError*>(&e);
    int code = se ? se->code : SORD_E_PARAM;
    if (h) h->s.err = e.what();
    else g_create_error = e.what();
    return code;
}

namespace sordgpu {

// Halo planes along l of a partitioned run (the reference's
// scalar_swap_halo / vector_swap_halo, process_mpi.f90:179-246, for the l
// direction): the first and last core planes of each field are copied into
// contiguous device send buffers, the caller's callback moves them between
// neighbouring parts, and the received planes are copied into the halo
// planes.  Planes are contiguous in the j-fastest layout.
void halo_exchange(Solver& s, float* const* fields, int nf) {
    if (s.nparts <= 1) return;
    const Geom& g = s.g;
    const size_t sz = (size_t)g.sz, n = sz * (size_t)nf;
    if (s.xcap < n) {
        dev_free(s, s.xbuf);
        s.xbuf = nullptr;
        s.xcap = 0;
        SORD_CUDA(dev_malloc(s, (void**)&s.xbuf, sizeof(float) * 4 * n));
        s.xcap = n;
    }
    float *send_lo = s.xbuf, *recv_lo = s.xbuf + n, *send_hi = s.xbuf + 2 * n, *recv_hi = s.xbuf + 3 * n;
    const bool lo = s.part > 0, hi = s.part < s.nparts - 1;
    const size_t core1 = (size_t)(g.i1core[2] - 1) * sz, core2 = (size_t)(g.i2core[2] - 1) * sz;
    const size_t halo1 = (size_t)(g.i1core[2] - 2) * sz, halo2 = (size_t)g.i2core[2] * sz;
    for (int i = 0; i < nf; i++) {
        if (lo) SORD_CUDA(cudaMemcpyAsync(send_lo + i * sz, fields[i] + core1, sizeof(float) * sz, cudaMemcpyDeviceToDevice, s.stream));
        if (hi) SORD_CUDA(cudaMemcpyAsync(send_hi + i * sz, fields[i] + core2, sizeof(float) * sz, cudaMemcpyDeviceToDevice, s.stream));
    }
    SORD_CUDA(cudaStreamSynchronize(s.stream));
    if (!s.halo_fn) throw SordError(SORD_E_PARAM, "partitioned run without a halo-exchange callback");
    const int rc = s.halo_fn(s.cb_ctx, s.part, lo ? send_lo : nullptr, lo ? recv_lo : nullptr, hi ? send_hi : nullptr,
                             hi ? recv_hi : nullptr, (long long)n);
    if (rc) throw SordError(SORD_E_STATE, "halo exchange failed (" + std::to_string(rc) + ")");
    for (int i = 0; i < nf; i++) {
        if (lo) SORD_CUDA(cudaMemcpyAsync(fields[i] + halo1, recv_lo + i * sz, sizeof(float) * sz, cudaMemcpyDeviceToDevice, s.stream));
        if (hi) SORD_CUDA(cudaMemcpyAsync(fields[i] + halo2, recv_hi + i * sz, sizeof(float) * sz, cudaMemcpyDeviceToDevice, s.stream));
    }
}

void all_reduce(Solver& s, double* vals, int n, int op) {
    if (s.nparts <= 1) return;
    if (!s.reduce_fn) throw SordError(SORD_E_PARAM, "partitioned run without a reduction callback");
    const int rc = s.reduce_fn(s.cb_ctx, s.part, vals, n, op);
    if (rc) throw SordError(SORD_E_STATE, "reduction failed (" + std::to_string(rc) + ")");
}

}  // namespace sordgpu

extern "C" {

static int create(const char* workdir, const char* sord_in_text, int device, int part, sord_halo_fn halo,
                  sord_reduce_fn reduce, void* ctx, bool partitioned, sord_handle** out) {
    if (!out || !sord_in_text) return SORD_E_PARAM;
    *out = nullptr;
    sord_handle* h = new sord_handle();
    Solver& s = h->s;
    try {
        if (partitioned) {
            if (part < 0 || !halo || !reduce) throw SordError(SORD_E_PARAM, "bad part index or missing callbacks");
            s.part = part;
            s.nparts = -1;  // set from nproc3 by setup
            s.halo_fn = halo;
            s.reduce_fn = reduce;
            s.cb_ctx = ctx;
        }
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) throw SordError(SORD_E_CUDA, "no CUDA device available");
        if (device < 0 || device >= n) throw SordError(SORD_E_CUDA, "bad device index");
        s.device = device;
        SORD_CUDA(cudaSetDevice(device));
        s.workdir = workdir ? workdir : "";
        s.clock0_us = 0;
        s.clock0_us = s.clock_us();
        SORD_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
        mem_attach(device);
        s.mem_attached = true;
        SORD_CUDA(cudaEventCreate(&s.ev0));
        SORD_CUDA(cudaEventCreate(&s.ev1));
        for (auto& row : s.inj_done)
            for (auto& e : row) SORD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        s.prm = parse_sord_in(sord_in_text, s.ops);
        setup_all(s);
    } catch (const std::exception& e) {
        int c = fail(nullptr, e);
        s.destroy();
        delete h;
        return c;
    }
    *out = h;
    return SORD_OK;
}

int sord_create(const char* workdir, const char* sord_in_text, int device, sord_handle** out) {
    return create(workdir, sord_in_text, device, 0, nullptr, nullptr, nullptr, false, out);
}

int sord_create_part(const char* workdir, const char* sord_in_text, int device, int part, sord_halo_fn halo,
                     sord_reduce_fn reduce, void* ctx, sord_handle** out) {
    return create(workdir, sord_in_text, device, part, halo, reduce, ctx, true, out);
}

int sord_step(sord_handle* h, int nsteps) {
    if (!h) return SORD_E_PARAM;
    Solver& s = h->s;
    try {
        SORD_CUDA(cudaSetDevice(s.device));
        if (nsteps < 0 || s.it + nsteps > s.nt) throw SordError(SORD_E_STATE, "step past nt");
        SORD_CUDA(cudaEventRecord(s.ev0, s.stream));
        for (int i = 0; i < nsteps; i++) s.step(i == nsteps - 1);
        SORD_CUDA(cudaEventRecord(s.ev1, s.stream));
        SORD_CUDA(cudaEventSynchronize(s.ev1));
        float ms = 0;
        SORD_CUDA(cudaEventElapsedTime(&ms, s.ev0, s.ev1));
        s.last_step_ms = ms;
        writer_drain(s);
    } catch (const std::exception& e) {
        return fail(h, e);
    }
    return SORD_OK;
}

static int adjoint_forward(sord_handle* h, int segment, int snapshots) {
    if (!h) return SORD_E_PARAM;
    Solver& s = h->s;
    try {
        SORD_CUDA(cudaSetDevice(s.device));
        if (s.nparts > 1) throw SordError(SORD_E_PARAM, "not available on a part of a partitioned run");
        if (snapshots < 0) throw SordError(SORD_E_PARAM, "adjoint: snapshots must be positive");
        adjoint_begin(s, snapshots > 0 ? 0 : adjoint_segment(s, segment), snapshots);
        SORD_CUDA(cudaEventRecord(s.ev0, s.stream));
        // run to each step whose state is kept; the last step before a
        // checkpoint is not folded, so the state it leaves is that step's
        for (int stop : adjoint_stops(s)) {
            const int n = stop - s.it;
            for (int i = 0; i < n; i++) s.step(i == n - 1);
            adjoint_checkpoint(s);
        }
        SORD_CUDA(cudaEventRecord(s.ev1, s.stream));
        SORD_CUDA(cudaEventSynchronize(s.ev1));
        float ms = 0;
        SORD_CUDA(cudaEventElapsedTime(&ms, s.ev0, s.ev1));
        s.last_step_ms = ms;
        writer_drain(s);
    } catch (const std::exception& e) {
        return fail(h, e);
    }
    return SORD_OK;
}

int sord_adjoint_forward(sord_handle* h, int segment) { return adjoint_forward(h, segment, 0); }

int sord_adjoint_forward_binomial(sord_handle* h, int snapshots) {
    if (snapshots < 1) return h ? fail(h, SordError(SORD_E_PARAM, "adjoint: snapshots must be at least 1")) : SORD_E_PARAM;
    return adjoint_forward(h, 0, snapshots);
}

int sord_adjoint_binomial_cost(int nt, int snapshots, long long* steps) {
    if (nt < 0 || snapshots < 1 || !steps) return SORD_E_PARAM;
    *steps = sordgpu::binomial_cost(nt, snapshots);
    return SORD_OK;
}

int sord_adjoint_backward(sord_handle* h, int nrec, const char* const* files, const float* const* dtrace,
                          const int* ntrace, float* grad_lam, float* grad_mu, float* grad_yy, float* grad_mr,
                          double* grad_moment, int nmoment) {
    if (!h || nrec < 0 || (nrec > 0 && (!files || !dtrace || !ntrace))) return SORD_E_PARAM;
    Solver& s = h->s;
    try {
        SORD_CUDA(cudaSetDevice(s.device));
        adjoint_backward(s, nrec, files, dtrace, ntrace, grad_lam, grad_mu, grad_yy, grad_mr, grad_moment, nmoment);
    } catch (const std::exception& e) {
        return fail(h, e);
    }
    return SORD_OK;
}

int sord_adjoint_source_gradients(sord_handle* h, double* grad_x0, double* grad_t0, int nmoment) {
    if (!h || nmoment < 0) return SORD_E_PARAM;
    try {
        adjoint_source_gradients(h->s, grad_x0, grad_t0, nmoment);
    } catch (const std::exception& e) {
        return fail(h, e);
    }
    return SORD_OK;
}

int sord_run(sord_handle* h) {
    if (!h) return SORD_E_PARAM;
    return sord_step(h, h->s.nt - h->s.it);
}

int sord_run_directory(const char* workdir, int device) {
    std::string dir = workdir ? workdir : ".";
    std::string fn = dir + "/sord.in";
    FILE* fp = fopen(fn.c_str(), "rb");
    if (!fp) { g_create_error = "cannot open " + fn; return SORD_E_IO; }
    std::string text;
    char buf[65536];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, n);
    fclose(fp);
    sord_handle* h = nullptr;
    int rc = sord_create(dir.c_str(), text.c_str(), device, &h);
    if (rc) return rc;
    rc = sord_run(h);
    if (rc) g_create_error = h->s.err;
    sord_destroy(h);
    return rc;
}

int sord_run_ensemble(const char* const* workdirs, int n, int device, int nthreads, int* status) {
    if (!workdirs || n < 0 || nthreads < 1) {
        g_create_error = "bad ensemble arguments";
        return SORD_E_PARAM;
    }
    std::atomic<int> next{0};
    std::mutex m;
    int first = SORD_OK;
    std::string msg;
    // each worker runs whole scenarios; every scenario has its own handle and
    // stream, so the device overlaps the kernels of different scenarios
    auto worker = [&]() {
        for (;;) {
            const int i = next++;
            if (i >= n) return;
            const int rc = workdirs[i] ? sord_run_directory(workdirs[i], device) : SORD_E_PARAM;
            if (status) status[i] = rc;
            if (rc != SORD_OK) {
                std::lock_guard<std::mutex> lock(m);
                if (first == SORD_OK) {
                    first = rc;
                    msg = std::string(workdirs[i] ? workdirs[i] : "(null)") + ": " + g_create_error;
                }
            }
        }
    };
    const int nt = std::min(nthreads, std::max(n, 1));
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    if (first != SORD_OK) g_create_error = msg;
    return first;
}

int sord_get_field(sord_handle* h, const char* name, float* host, size_t n) {
    if (!h || !name || !host) return SORD_E_PARAM;
    Solver& s = h->s;
    try {
        SORD_CUDA(cudaSetDevice(s.device));
        if (s.nparts > 1) throw SordError(SORD_E_PARAM, "not available on a part of a partitioned run");
        std::string f = name;
        float* src = nullptr;
        bool cell = false;
        const char* vn[9] = {"vx", "vy", "vz", "ux", "uy", "uz", "ax", "ay", "az"};
        for (int i = 0; i < 9; i++)
            if (f == vn[i]) src = i < 3 ? s.d.v[i] : i < 6 ? s.d.u[i - 3] : s.d.w1n[i - 6];
        if (f == "lam") { src = s.d.lam; cell = true; }
        if (f == "mu") { src = s.d.mu; cell = true; }
        if (f == "yy") { src = s.d.yy; cell = true; }
        if (f == "vc") { src = s.d.vc; cell = true; }
        if (!src) throw SordError(SORD_E_PARAM, "unknown field " + f);
        int c[3];
        for (int i = 0; i < 3; i++) c[i] = cell ? s.g.nn[i] - 1 : s.g.nn[i];
        size_t need = (size_t)c[0] * c[1] * c[2];
        if (n < need) throw SordError(SORD_E_PARAM, "host buffer too small");
        std::vector<float> all((size_t)s.g.nv);
        SORD_CUDA(cudaMemcpyAsync(all.data(), src, sizeof(float) * (size_t)s.g.nv, cudaMemcpyDeviceToHost, s.stream));
        SORD_CUDA(cudaStreamSynchronize(s.stream));
        size_t q = 0;
        for (int l = 0; l < c[2]; l++)
            for (int k = 0; k < c[1]; k++)
                for (int j = 0; j < c[0]; j++)
                    host[q++] = all[(size_t)s.g.idx(s.g.i1core[0] + j, s.g.i1core[1] + k, s.g.i1core[2] + l)];
    } catch (const std::exception& e) {
        return fail(h, e);
    }
    return SORD_OK;
}

int sord_set_field(sord_handle* h, const char* name, const float* host, size_t n) {
    if (!h || !name || !host) return SORD_E_PARAM;
    Solver& s = h->s;
    try {
        SORD_CUDA(cudaSetDevice(s.device));
        if (s.nparts > 1) throw SordError(SORD_E_PARAM, "not available on a part of a partitioned run");
        std::string f = name;
        float* dst = nullptr;
        bool cell = false;
        const char* vn[6] = {"vx", "vy", "vz", "ux", "uy", "uz"};
        for (int i = 0; i < 6; i++)
            if (f == vn[i]) dst = i < 3 ? s.d.v[i] : s.d.u[i - 3];
        if (f == "lam") { dst = s.d.lam; cell = true; }
        if (f == "mu") { dst = s.d.mu; cell = true; }
        if (f == "yy") { dst = s.d.yy; cell = true; }
        if (!dst) throw SordError(SORD_E_PARAM, "field cannot be set: " + f);
        // a fault's moduli (lamf, muf) and the zeroed hourglass constant of
        // its cell layer are derived from lam, mu and yy at setup
        if (cell && s.g.ifn != 0)
            throw SordError(SORD_E_PARAM, "field cannot be set on a run with a fault (its fault-plane moduli are "
                                          "derived from lam and mu at setup): " + f);
        int c[3];
        for (int i = 0; i < 3; i++) c[i] = cell ? s.g.nn[i] - 1 : s.g.nn[i];
        size_t need = (size_t)c[0] * c[1] * c[2];
        if (n != need) throw SordError(SORD_E_PARAM, "host array has " + std::to_string(n) + " values, the field " +
                                                     std::to_string(need));
        // read-modify-write of the whole array keeps the halo as it is
        std::vector<float> all((size_t)s.g.nv);
        SORD_CUDA(cudaMemcpyAsync(all.data(), dst, sizeof(float) * (size_t)s.g.nv, cudaMemcpyDeviceToHost, s.stream));
        SORD_CUDA(cudaStreamSynchronize(s.stream));
        size_t q = 0;
        for (int l = 0; l < c[2]; l++)
            for (int k = 0; k < c[1]; k++)
                for (int j = 0; j < c[0]; j++)
                    all[(size_t)s.g.idx(s.g.i1core[0] + j, s.g.i1core[1] + k, s.g.i1core[2] + l)] = host[q++];
        SORD_CUDA(cudaMemcpyAsync(dst, all.data(), sizeof(float) * (size_t)s.g.nv, cudaMemcpyHostToDevice, s.stream));
        SORD_CUDA(cudaStreamSynchronize(s.stream));
    } catch (const std::exception& e) {
        return fail(h, e);
    }
    return SORD_OK;
}

int sord_info(const sord_handle* h, int* nn3, int* it, int* nt) {
    if (!h) return SORD_E_PARAM;
    if (nn3) for (int i = 0; i < 3; i++) nn3[i] = h->s.g.nn[i];
    if (it) *it = h->s.it;
    if (nt) *nt = h->s.nt;
    return SORD_OK;
}

int sord_stats(const sord_handle* h, double* out, int n) {
    if (!h || !out) return SORD_E_PARAM;
    int m = n < 16 ? n : 16;
    for (int i = 0; i < m; i++) out[i] = h->s.last_stats[i];
    return m;
}

double sord_last_step_ms(const sord_handle* h) { return h ? h->s.last_step_ms : 0.0; }

int sord_set_profiling(sord_handle* h, int on) {
    if (!h) return SORD_E_PARAM;
    try {
        h->s.prof_collect();
        h->s.profiling = on != 0;
        for (int i = 0; i < 8; i++) { h->s.kernel_ms[i] = 0; h->s.kernel_n[i] = 0; }
    } catch (const std::exception& e) {
        return fail(h, e);
    }
    return SORD_OK;
}

int sord_set_arithmetic(sord_handle* h, int mode) {
    if (!h) return SORD_E_PARAM;
    if (mode != 0 && mode != 1) {
        h->s.err = "sord_set_arithmetic: mode must be 0 or 1";
        return SORD_E_PARAM;
    }
    h->s.arith = mode;
    return SORD_OK;
}

int sord_get_arithmetic(const sord_handle* h) { return h ? h->s.arith : SORD_E_PARAM; }

int sord_trim_memory(int device) {
    try {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
            throw SordError(SORD_E_CUDA, "sord_trim_memory: no CUDA device " + std::to_string(device));
        SORD_CUDA(cudaSetDevice(device));
        mem_trim(device);
    } catch (const std::exception& e) {
        return fail(nullptr, e);
    }
    return SORD_OK;
}

int sord_kernel_times(sord_handle* h, double* ms, long long* count, int n) {
    if (!h) return SORD_E_PARAM;
    try {
        h->s.prof_collect();
    } catch (const std::exception& e) {
        return fail(h, e);
    }
    int m = n < 8 ? n : 8;
    for (int i = 0; i < m; i++) {
        if (ms) ms[i] = h->s.kernel_ms[i];
        if (count) count[i] = h->s.kernel_n[i];
    }
    return m;
}

long long sord_kernel_launches(const sord_handle* h) { return h ? h->s.launches : 0; }

const char* sord_last_error(const sord_handle* h) { return h ? h->s.err.c_str() : g_create_error.c_str(); }

const char* sord_error_string(int code) {
    switch (code) {
        case SORD_OK: return "SORD_OK";
        case SORD_E_PARAM: return "SORD_E_PARAM";
        case SORD_E_CFL: return "SORD_E_CFL";
        case SORD_E_NEGVOL: return "SORD_E_NEGVOL";
        case SORD_E_NANINF: return "SORD_E_NANINF";
        case SORD_E_IO: return "SORD_E_IO";
        case SORD_E_CUDA: return "SORD_E_CUDA";
        case SORD_E_STATE: return "SORD_E_STATE";
        case SORD_E_NOMEM: return "SORD_E_NOMEM";
        default: return "SORD_E_UNKNOWN";
    }
}

void sord_destroy(sord_handle* h) {
    if (!h) return;
    h->s.destroy();
    delete h;
}

}  // extern "C"
