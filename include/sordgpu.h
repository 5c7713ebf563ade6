/*
 * sordgpu.h - C ABI of the B200-native SORD time-stepper (libsordgpu.so).
 *
 * The reference has no library interface: cst/sord.py:stage() writes the
 * text deck `sord.in` (cst/sord.py:538-544) and cst/job.py:launch()
 * (cst/job.py:176-195) runs the Fortran executable `sord.x` as a separate
 * process, which reads `sord.in` (sord/input_output.f90:21-98), runs the
 * setup and step loop (sord/sord.f90:24-47) and writes `.bin`, `stats-*.bin`,
 * `prof-*.bin` and `material.json` into the working directory.
 *
 * This ABI replaces that process boundary with in-process calls that take
 * the same `sord.in` text and write the same files.  All arguments are plain
 * C types; the library owns all device memory.  Every call returns SORD_OK
 * (0) or a negative SORD_E_* code; sord_last_error() gives the message (the
 * text the Fortran `stop` would have printed).  A handle is used by one host
 * thread at a time; each handle runs on its own CUDA stream.
 */
#ifndef SORDGPU_H
#define SORDGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sord_handle sord_handle;

enum {
    SORD_OK = 0,
    SORD_E_PARAM = -1,   /* bad sord.in / bad i/o op        (input_output.f90:253,423,514) */
    SORD_E_CFL = -2,     /* Courant condition / negative moduli (material_model.f90:167-168) */
    SORD_E_NEGVOL = -3,  /* negative cell volume            (grid_generation.f90:195-198) */
    SORD_E_NANINF = -4,  /* NaN/Inf in stats or input file  (statistics.f90:53-59, input_output.f90:333-337) */
    SORD_E_IO = -5,      /* file open/read/write failure */
    SORD_E_CUDA = -6,    /* CUDA runtime error or no device */
    SORD_E_STATE = -7,   /* call out of order (e.g. step past nt) */
    SORD_E_NOMEM = -8    /* device allocation failed */
};

/* Parse `sord_in_text` (the sord.in wire format) and run the whole setup
 * (sord/sord.f90:27-36: dimensions, grid, material, PML, finite source,
 * rupture, resample) on CUDA device `device`.  Input files named by the I/O
 * ops and all outputs are resolved relative to `workdir`.
 * Replaces: the start of `sord.x` (sord/sord.f90:24-37). */
int sord_create(const char* workdir, const char* sord_in_text, int device, sord_handle** out);

/* Halo exchange of a partitioned run.  The part's halo planes along l are
 * filled from its neighbours: recv_lo (the plane below the part's first
 * plane) from part - 1's send_hi, recv_hi from part + 1's send_lo.  Each
 * buffer holds n floats of device memory, NULL where the part has no such
 * neighbour.  Called with the part's stream idle; the transfer must be
 * complete when it returns.  Returns 0 on success.
 * Replaces: vector_swap_halo / scalar_swap_halo (sord/process_mpi.f90:179-246). */
typedef int (*sord_halo_fn)(void* ctx, int part, const float* send_lo, float* recv_lo, const float* send_hi,
                            float* recv_hi, long long n);

/* All-reduce of n host doubles in place over the parts of a run: op 0 the
 * maximum, op 1 the sum.  Returns 0 on success.
 * Replaces: rreduce1 / rreduce2 (sord/process_mpi.f90:137-177). */
typedef int (*sord_reduce_fn)(void* ctx, int part, double* vals, int n, int op);

/* Create part `part` of a run split along l into nproc3[2] parts of the
 * sord.in parameter nproc3 (= [1, 1, P]): the planes of each part, its
 * global offset and its index ranges follow sord/setup.f90:33-84 (nl3 =
 * (nn - 1) / P + 1 planes per part).  Each part runs setup and steps on its
 * own device; `halo` and `reduce` carry the communication (the halo planes
 * of coordinates, mass and viscosity at setup, of v, u and a after every
 * step; material extrema and statistics).  Output files are shared: each
 * part writes its planes at their offsets (mpout = 1); part 0 writes the
 * statistics files and material.json.  Rejected (SORD_E_PARAM): nproc3
 * splitting j or k, a fault, gridnoise or random ('~') field ops (the
 * reference seeds these per process, setup.f90:41-44, so they depend on
 * the split), and a first or last part that does not hold the PML of
 * its l face and one plane more.  Every step exchanges the halo planes of the acceleration (the
 * reference's force-halo swap, acceleration.f90:229-233) and, after a fused
 * step that also advanced v and u, of v and u.
 * Replaces: one MPI rank of sord.x built with process_mpi.f90. */
int sord_create_part(const char* workdir, const char* sord_in_text, int device, int part, sord_halo_fn halo,
                     sord_reduce_fn reduce, void* ctx, sord_handle** out);

/* Advance `nsteps` time steps (sord/sord.f90:39-47: step_time, step_stress,
 * step_accel, stats), including every field-I/O hook of those steps. */
int sord_step(sord_handle* h, int nsteps);

/* Run all remaining steps and flush every output.  Replaces the remainder of
 * `sord.x` after setup (sord/sord.f90:39-50). */
int sord_run(sord_handle* h);

/* Convenience: sord_create on `workdir`/sord.in, sord_run, sord_destroy.
 * This is the whole of `sord.x` (cst/job.py:193-194 `subprocess.check_call`). */
int sord_run_directory(const char* workdir, int device);

/* Run `n` staged directories (each with its sord.in) to completion on CUDA
 * device `device`, up to `nthreads` at a time: host threads take scenarios in
 * turn, each scenario with its own handle and stream, so the device overlaps
 * the kernels of different scenarios (ensembles of small runs are bound by
 * launch latency when run one at a time).  Each scenario's outputs are those
 * of sord_run_directory on its own.  status[i] (if not NULL) receives each
 * scenario's return code; the call returns the first failure, whose message
 * sord_last_error(NULL) gives.  Replaces: one `sord.x` process per scenario
 * (cst/job.py:176-195), which the reference runs one job at a time. */
int sord_run_ensemble(const char* const* workdirs, int n, int device, int nthreads, int* status);

/* Adjoint (no reference counterpart: the reference computes no
 * derivatives).  Gradients of a misfit of '.>' velocity or displacement
 * receivers with respect to the per-cell moduli and node masses and to the
 * value of every '.' moment op, for runs on a rectilinear mesh without
 * fault whose every step is a plain fused step (field-I/O outputs and '.'
 * moment/potency ops only).  PML faces are supported (their cell and node
 * memories are part of the state and have adjoints of their own) unless
 * the bands of opposite faces meet; the damping profile is held fixed (set
 * vpml, or it follows the material's extremes, which are not
 * differentiated).
 *
 * sord_adjoint_forward runs the whole forward run of a fresh handle (it must
 * be at step 0), writing its outputs as sord_run does, and keeps the state
 * (u, v, a), and with PML the memories, every `segment` steps on the
 * device.  Memory: about 36 B x (nt / segment + 2 segment) per node, plus
 * the PML memories per state.  segment 1 keeps every state
 * and the backward pass recomputes nothing; segment 0 chooses 1 when all
 * states fit in half of the free device memory, else about sqrt(nt).  sord_last_step_ms gives the
 * device time of the call (and of sord_adjoint_backward after that one). */
int sord_adjoint_forward(sord_handle* h, int segment);

/* sord_adjoint_forward with binomial checkpointing (the revolve schedule)
 * instead of uniform segments: at most `snapshots` states are kept on the
 * device at any time, besides the last state and three work states, and
 * the backward pass recomputes the others from them with the fewest
 * forward steps that storage allows.  sord_adjoint_binomial_cost gives the
 * forward steps the schedule takes for nt steps, counting the chain of
 * kept states that the forward run itself provides.  With snapshots >= nt
 * nothing is recomputed.  The backward pass is sord_adjoint_backward, once
 * per forward run (the records are reused as it goes); it runs on one
 * stream (no overlap of recomputation and adjoint steps). */
int sord_adjoint_forward_binomial(sord_handle* h, int snapshots);
int sord_adjoint_binomial_cost(int nt, int snapshots, long long* steps);

/* Backward pass after sord_adjoint_forward: files[i] names the output file
 * of a '.>' receiver op on vx/vy/vz/ux/uy/uz and dtrace[i] holds dL/d(sample)
 * for its ntrace[i] samples (the file's layout).  Each segment is recomputed
 * from its checkpoint and the transposed step kernels run backwards through
 * it.  Outputs (any may be NULL): grad_lam, grad_mu, grad_yy per real cell
 * ((nx-1)(ny-1)(nz-1), j fastest) = dL/d(lambda), dL/d(mu), dL/d(hourglass
 * modulus yy); grad_mr per node (nx ny nz) = dL/d(mr), mr being the inverse
 * nodal mass; grad_moment[m] = dL/d(value) of the m-th '.' moment op in
 * sord.in order (nmoment must equal their count). */
int sord_adjoint_backward(sord_handle* h, int nrec, const char* const* files, const float* const* dtrace,
                          const int* ntrace, float* grad_lam, float* grad_mu, float* grad_yy, float* grad_mr,
                          double* grad_moment, int nmoment);

/* Device memory of the handles comes from the device's default memory
 * pool; when the last handle on a device is destroyed the pool's memory is
 * returned to the driver on a helper thread, so sord_destroy and
 * sord_run_directory return without waiting for it.  sord_trim_memory
 * waits for that, and with no live handle on `device` returns the pool's
 * unused memory now: call it before allocating the memory elsewhere in the
 * same process.  No reference counterpart (the reference frees its arrays
 * at process exit). */
int sord_trim_memory(int device);

/* After sord_adjoint_backward: the gradients with respect to the position
 * and the delay of each '.' moment op (sord.in order), which the backward
 * pass computes with the moment values.  An op injects val tf(t - t0) r(x)
 * with r its trilinear weights: grad_x0[3 m + d] = dL/dx_d of op m (per
 * metre; the weights are piecewise linear, so this is the derivative inside
 * the current cell), grad_t0[m] = dL/dt0 (per second, t0 a delay of the
 * time function).  Either pointer may be NULL; nmoment as for
 * sord_adjoint_backward. */
int sord_adjoint_source_gradients(sord_handle* h, double* grad_x0, double* grad_t0, int nmoment);

/* Copy a node or cell volume field to host memory (core region only, j
 * fastest; nn or nn-1 values per axis).  Names: vx vy vz ux uy uz ax ay az
 * (nodes; `a` holds the last acceleration) and lam mu yy vc (cells).
 * `n` is the capacity of `host` in floats. */
int sord_get_field(sord_handle* h, const char* name, float* host, size_t n);

/* Overwrite a field between steps from host memory (the layout of
 * sord_get_field; `n` must equal the field's core size): the state vx vy vz
 * ux uy uz (initial conditions, perturbations) or the cell moduli lam mu yy,
 * where yy is the hourglass coefficient as sord_get_field returns it (the
 * material setup's mu (lam + mu) / (lam + 2 mu) times the cell-size factor,
 * sord/material_model.f90:120-131, zero outside the cell region,
 * sord/material_resample.f90:40).  No consistency with the other material
 * arrays or the Courant condition is checked, and on a run with a fault the
 * moduli cannot be set (SORD_E_PARAM): the fault-plane moduli are derived
 * from them at setup.  Halo values are kept.  Replaces: fields read by '=<' ops
 * (sord/input_output.f90:392-419), from memory and between any two steps. */
int sord_set_field(sord_handle* h, const char* name, const float* host, size_t n);

/* Query dimensions and progress: nn[3] global nodes, it (steps done), nt. */
int sord_info(const sord_handle* h, int* nn3, int* it, int* nt);

/* Latest statistics (statistics.f90:13-131): out[0..15] = amax vmax umax wmax
 * samax svmax sumax slmax tsmax tnmin tnmax tarrmax efric estrain moment mw
 * of the last stats step (maxima as magnitudes).  Returns the count written. */
int sord_stats(const sord_handle* h, double* out, int n);

/* Device time of the last sord_step call in milliseconds (CUDA events on the
 * handle's stream, step kernels and I/O hooks included). */
double sord_last_step_ms(const sord_handle* h);

/* Arithmetic of the interior fused step kernel (no reference counterpart).
 * Mode 0 (the default): every operation of the reference in its order and
 * without fused multiply-adds, so outputs are bit-identical to a serial FP32
 * build of the reference's arithmetic (sord/diff_nc_op.f90, diff_cn_op.f90,
 * stress.f90, acceleration.f90, time_integration.f90).  Mode 1 (fast): fused
 * multiply-adds, the support-operator brackets scaled by h once per cell,
 * each divergence bracket taken as the negated gradient bracket of the same
 * cell and corner, and on terrain meshes (x = x(j), y = y(k)) the closed
 * form of the two z-dependent bracket sets; equal to mode 0 in exact
 * arithmetic, FP32 rounding apart.  The PML shell, fault, source and
 * separate-kernel paths keep mode 0.  New handles start in mode 1 when the
 * environment variable SORD_ARITHMETIC is "fast".  May be called between any
 * two steps.  sord_get_arithmetic returns the mode. */
int sord_set_arithmetic(sord_handle* h, int mode);
int sord_get_arithmetic(const sord_handle* h);

/* Per-kernel device timing for performance reports.  With profiling on,
 * CUDA events are recorded around each step kernel on the handle's stream
 * and accumulated per class: 0 time update, 1 stress, 2 acceleration,
 * 3 mass, 4 fault, 5 field I/O, 6 other, 7 fused step kernel (one whole
 * time step).  Turning it on or off resets the
 * sums.  sord_kernel_times writes min(n, 8) totals (ms) and launch counts
 * and returns that number.  No reference counterpart (the reference writes
 * host timers to prof-*.bin, statistics.f90:116-129; those files are
 * written here too). */
int sord_set_profiling(sord_handle* h, int on);
int sord_kernel_times(sord_handle* h, double* ms, long long* count, int n);

/* Maximum of w0^2 + w1^2 + w2^2 over the region [i1, i2] (1-based,
 * inclusive) of a caller-owned FP32 device field of extents nm[3] (j
 * fastest) -- the statistic behind the |v|, |u|, |a| maxima of
 * sord_stats -- written to the device float `out`, enqueued on CUDA stream
 * `stream` (NULL for the default stream) on the current device.
 *
 * No counterpart in the reference.  It allocates nothing (no cudaMalloc,
 * cudaFree or allocating library call), for callers that cannot allocate
 * device memory where they need the reduction (a frozen or exhausted memory
 * pool, allocation-free sections of a host framework).  Its partial results
 * live in a 4 KiB file-scope device array (1024 block maxima) that every GPU
 * loading this library keeps until the process exits; regions of 2^31
 * elements or more are rejected with SORD_E_PARAM.  All calls share that
 * array, so calls that overlap on the GPU race and must be serialised by the
 * caller.  The first call on each device looks up the array's address with
 * that device current; make it before any stream capture.  On error,
 * sord_last_error(NULL) gives the message. */
int sord_vector_max_noalloc(const float* w0, const float* w1, const float* w2, const int* nm, const int* i1,
                            const int* i2, float* out, void* stream);

/* Number of kernels this library launched since the handle was created. */
long long sord_kernel_launches(const sord_handle* h);

/* Message for the last error on `h` (or the last create failure if h is NULL). */
const char* sord_last_error(const sord_handle* h);

/* Static name of an error code. */
const char* sord_error_string(int code);

/* Free all device memory of the handle and flush pending output. */
void sord_destroy(sord_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* SORDGPU_H */
