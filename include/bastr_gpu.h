/*
 * bastr_gpu.h -- C ABI of the B200 (sm_100a) pseudo-spectral Burgers time step.
 *
 * The library replaces the FFTW-MPI hot path of Bastr (lcs27/Bastr).  A Fortran driver
 * binds these entry points with iso_c_binding; every function returns an int status
 * (0 = ok, < 0 = error, message via bastr_last_error), plain pointers and sizes only.
 *
 * Entry point                 replaces (reference file:line)
 * --------------------------  ---------------------------------------------------------------
 * bastr_create                readinput derivations (readwrite.F90:69-83), mpisizedis_fftw
 *                             (fftwlink.F90:34-153), allocation (fftwlink.F90:370-467),
 *                             prepareplan_fftw_plan (fftwlink.F90:284-303), quantity_prepare
 *                             (solution.F90:1288-1313)
 * bastr_set_state             the initial dealias of mainloop2D/3D (solution.F90:41-52,
 *                             106-122) applied to u1,u2[,u3] after read_initial_field /
 *                             read_continue_field (readwrite.F90:114-220)
 * bastr_set_counters          nstep/time restored by read_continue_field (readwrite.F90:211-218)
 * bastr_step                  n iterations of the `do while(nstep<=maxstep)` body of
 *                             mainloop2D/3D (solution.F90:54-97, 124-169): spectra_compute,
 *                             velgrad_calculate, nstep/time advance, RK3 or CN, forcing
 * bastr_get_state             the physical u1,u2[,u3] that writeflfed dumps (readwrite.F90:222-257)
 * bastr_spectra               spectra_compute2D/3D shell arrays (solution.F90:930-1108)
 * bastr_fft                   fft2d/fft3d/ifft2d/ifft3d (fftwlink.F90:324-368), in place on a
 *                             full complex(8) grid, for Bastrpp-style callers
 * bastr_destroy               deallocation (fftwlink.F90:469-490)
 * bastr_transfer              Bastrpp transfer2d/transfer3d (Bastrpp.F90:174-305, 418-599)
 * bastr_hitgen                Bastrpp hitgen2d/hitgen2dbis/hitgen3d (Bastrpp.F90:601-1005)
 * bastr_profile, bastr_info,  no reference counterpart: per-kernel timing and introspection
 *   bastr_step_async/records,  for measurement; asynchronous stepping and stream control
 *   bastr_set_stream, bastr_sync
 * bastr_last_error            the reference's `stop 'message'` text, as a return value
 *
 * Layout: fields are real(8) arrays in Fortran order u(1:ia,1:ja[,1:ka]), x fastest,
 * which is C order [ka][ja][ia].
 *
 * A handle owns one stream on one GPU and is not thread-safe; use one handle per GPU.
 */
#ifndef BASTR_GPU_H
#define BASTR_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define BASTR_API __attribute__((visibility("default")))
#else
#define BASTR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define BASTR_OK 0
#define BASTR_E_INVALID (-1)     /* bad argument or parameter */
#define BASTR_E_UNSUPPORTED (-2) /* valid for the reference, not built here (e.g. grid size) */
#define BASTR_E_CUDA (-3)        /* CUDA runtime error */
#define BASTR_E_NAN (-4)         /* Es+Ed became NaN (solution.F90:81): stepping stopped */
#define BASTR_E_STATE (-5)       /* call order: no state set yet */

#define BASTR_FP64 0             /* FP64 fields and transforms: parity form */
#define BASTR_FP32 1             /* FP32 fields/transforms/product, FP64 state and reductions */

/* The datin/input.dat values the time step reads (readwrite.F90:35-44), plus GPU knobs. */
typedef struct bastr_params {
    int32_t ia, ja, ka;          /* grid; ka == 0 selects 2D */
    double ref_tem, reynolds;    /* nu = miucal(1)/reynolds = 1/reynolds; reynolds == 0 -> nu = 0 */
    double deltat;
    int32_t kmax;                /* allkmax = min(ia/3, kmax) */
    int32_t timemethod;          /* 1 = RK3 (Kutta), 2 = Crank-Nicolson 6-sweep fixed point */
    int32_t forcemethod;         /* 0 none, 1 linear, 2 band, 3/4 random-phase band, 5 band to target */
    int32_t forcek;
    double target_energy;
    int32_t lprojectd;           /* project the right-hand side on its dilatational part */
    int32_t precision;           /* BASTR_FP64 or BASTR_FP32 */
    int32_t device;              /* CUDA device ordinal */
    int32_t velgrad_every;       /* velocity-gradient statistics every n steps (1 = reference; 0 = never) */
} bastr_params;

/* One iteration of the main loop.  nstep/time are the values the reference logs with the
 * spectra and velgrad lines (before the increment); the forcing line uses nstep+1, time+dt. */
typedef struct bastr_step_out {
    int64_t nstep;
    double time;
    double Esspe, Edspe, k2Edspe, kMEdspe;      /* log/stat{2,3}d_specall.dat */
    double velgrad[8];                          /* umumtheta2 umumijji u2theta dissp etamin Tay ReTay Kol */
    double factor, E;                           /* log/factor_output.dat (NaN when not written) */
    double energy, Fen;                         /* forcing 3 and 4 also log these (else NaN) */
} bastr_step_out;

typedef struct bastr_handle bastr_handle;

BASTR_API int bastr_create(const bastr_params* p, bastr_handle** out);
BASTR_API int bastr_destroy(bastr_handle* h);

/* Host arrays, x fastest; u3 ignored in 2D. */
BASTR_API int bastr_set_state(bastr_handle* h, const double* u1, const double* u2, const double* u3);
BASTR_API int bastr_get_state(bastr_handle* h, double* u1, double* u2, double* u3);
BASTR_API int bastr_set_counters(bastr_handle* h, int64_t nstep, double time);
BASTR_API int bastr_get_counters(bastr_handle* h, int64_t* nstep, double* time);

/* Runs nsteps iterations; out[nsteps] (may be NULL); shells (may be NULL) receives, per step,
 * Es[0..allkmax] then Ed[0..allkmax].  Returns BASTR_E_NAN at the first step whose Es+Ed is NaN,
 * as the reference stops there (solution.F90:69-81), also when out is NULL: that step's record is
 * filled, the records and shells of the later steps are NaN, no kernel of a later step runs, and
 * the state and the counters (bastr_get_state, bastr_get_counters) are those of the NaN step, the
 * state the reference dumps before it stops.  Returns BASTR_E_CUDA, with a message, when a kernel
 * of the batch reported an internal error instead of faulting: a bounded wait for its TMA staging
 * that gave up, or (libbastr_gpu_checked.so) an access outside the handle's buffers. */
BASTR_API int bastr_step(bastr_handle* h, int32_t nsteps, bastr_step_out* out, double* shells);

/* Enqueues nsteps iterations on the handle's stream and returns without synchronising;
 * per-step records stay on the device (bastr_step_records copies the last batch, and returns
 * BASTR_E_NAN with the counters wound back to the NaN step when the batch stopped at one). */
BASTR_API int bastr_step_async(bastr_handle* h, int32_t nsteps);
BASTR_API int bastr_step_records(bastr_handle* h, int32_t nsteps, bastr_step_out* out, double* shells);

/* Shell spectra of the current state: arrays of allkmax+1 entries (shell 0..allkmax). */
BASTR_API int bastr_spectra(bastr_handle* h, double* kn, double* Es, double* Ed, int64_t* Ecount);

/* Energy transfer spectra of the current state, Bastrpp's transfer2d/transfer3d
 * (Bastrpp.F90:174-305, 418-599): T (advective form), T1 (conservative form) and T2 (the
 * u_i div(u) part) per shell nint(|k|) = 0..allkmax (host arrays of allkmax+1; any may be NULL).
 * Allocates its full-grid work buffers on the first call (about (2d + 2d^2) complex grids). */
BASTR_API int bastr_transfer(bastr_handle* h, double* T, double* T1, double* T2);

/* Initial-field generators of Bastrpp: variant 0 = hitgen2d / hitgen3d (create_initial_field_2d
 * Bastrpp.F90:601-696, create_initial_field_3d :698-808, by the handle's dimension), variant 1 =
 * hitgen2dbis (create_initial_field_2d_bis :810-1005, 2D only).  A dilatational field with the
 * generators' spectrum (the handle's forcek) and random phases, scaled to mean(|u|^2) = the
 * handle's target_energy.  The phases are atan2 of the FFT of a uniform (0,1) field drawn from
 * Philox-4x32-10 keyed by `seed` (not gfortran's random_number).  Host outputs, x fastest (any may
 * be NULL): u1, u2[, u3] and random_angle (the phase of every mode; the uniform value at k = 0).
 * stats[8] (may be NULL): energy before scaling, factor, alpha (NaN for variant 0), the cubic's
 * residual at alpha, QX, QY, QZ, QW.  The handle's state is not changed; pass the result to
 * bastr_set_state to start from it.  Uses the work buffers of bastr_transfer. */
BASTR_API int bastr_hitgen(bastr_handle* h, int32_t variant, uint64_t seed, double* u1, double* u2, double* u3,
                           double* angle, double* stats);

/* In-place c2c transform of a full complex(8) grid (interleaved re,im; x fastest):
 * dir = -1 forward scaled by 1/N (fft2d/fft3d), dir = +1 backward unscaled (ifft2d/ifft3d). */
BASTR_API int bastr_fft(bastr_handle* h, double* array, int32_t dir);

/* Stream control for callers that time or order work around the library. */
BASTR_API int bastr_set_stream(bastr_handle* h, void* cuda_stream);
BASTR_API int bastr_sync(bastr_handle* h);

/* Introspection: allkmax, kernels launched per step, device bytes held. */
BASTR_API int bastr_info(bastr_handle* h, int32_t* allkmax, int32_t* launches_per_step, int64_t* device_bytes);

/* Per-kernel timing: runs nsteps (1..256) iterations with CUDA events around every launch and
 * returns, per kernel, launches, total device time and algorithmic bytes per launch (unique
 * global reads plus writes of its inputs and outputs).  The state advances by nsteps. */
typedef struct bastr_kernel_stat {
    char name[48];
    int32_t launches;
    double total_ms;
    double bytes_per_launch;
} bastr_kernel_stat;
BASTR_API int bastr_profile(bastr_handle* h, int32_t nsteps, bastr_kernel_stat* stats, int32_t max_stats,
                            int32_t* n_stats);

/* Shell spectra of a caller-owned spectrum, allocating nothing.  No counterpart in the reference:
 * it serves callers that keep their spectra in their own device memory and cannot let a library
 * call cudaMalloc (GPU memory owned by CUDA Fortran / OpenACC data regions of a post-processing
 * driver, or a memory-capped pool), so they cannot create a handle, which allocates.
 *   d_u1spe, d_u2spe[, d_u3spe]: device arrays of ia*ja*max(ka,1) complex(8) values (re, im
 *       interleaved, x fastest), the forward-normalised spectra that fft2d/fft3d produce;
 *   d_Es, d_Ed: device arrays of allkmax+1 doubles (allkmax = min(ia/3, kmax)), shells 0..allkmax;
 *   d_totals (may be NULL): 4 doubles Esspe, Edspe, k2Edspe, kMEdspe over every mode.
 * The only workspace is a fixed 128 KiB device array inside the library (BASTR_NOALLOC_MAX_SHELLS
 * shells x 4 doubles), held by every GPU that loads the library until the process exits; grids
 * with nint(|k|max) + 1 > BASTR_NOALLOC_MAX_SHELLS are rejected with BASTR_E_TOO_LARGE.  The first
 * call in a CUDA context looks up that array's device address in that context (the address is
 * cached per context id, so a context made current by the caller, or the primary context created
 * anew after a cudaDeviceReset, gets its own lookup); make that first call before any stream
 * capture.
 * All calls share the array: calls that overlap on the GPU (other streams or host threads) race
 * and must be serialised by the caller.  Each call writes every slot it reads, so no clearing is
 * needed between calls.  Runs on `stream` (NULL: legacy default stream), does not synchronise. */
#define BASTR_NOALLOC_MAX_SHELLS 4096
#define BASTR_E_TOO_LARGE (-6)
BASTR_API int bastr_spectra_noalloc(int32_t ia, int32_t ja, int32_t ka, int32_t kmax,
                                    const double* d_u1spe, const double* d_u2spe, const double* d_u3spe,
                                    double* d_Es, double* d_Ed, double* d_totals, void* stream);

/* Copies the message of the last failed call into buf (NUL-terminated); returns its length. */
BASTR_API int bastr_last_error(bastr_handle* h, char* buf, int32_t n);

/* ------------------------------------------------------------------------------------------
 * Field files without libhdf5: the subset of HDF5 the reference's field files use, read and
 * written from the HDF5 file format specification (host code only; no GPU, no handle).
 * Replaces, for a caller without libhdf5, hdf5io.F90's h5io_init/h5write/h5read/h5srite/h5io_end
 * as readwrite.F90 uses them: writeflfed (readwrite.F90:222-257; hdf5io.F90:752-802 h5wa3d_r8_struct,
 * 1009-1184 h5_write1int/h5_write1rl8), read_initial_field / read_continue_field
 * (readwrite.F90:114-220; hdf5io.F90:204-256 h5ra3d_r8_struct, 404-452 h5r_int4/h5r_real8).
 * Files: HDF5 superblock version 0, root group as a symbol table, datasets of IEEE little-endian
 * binary64 (H5T_NATIVE_DOUBLE) or signed 32-bit integers (H5T_NATIVE_INTEGER) with contiguous
 * storage, the format libhdf5 writes by default; the reader also takes version 1 superblocks,
 * object-header continuation blocks and compact storage.  Dimensions are in C order (slowest
 * first), the reverse of Fortran's.
 *
 *   bastr_h5_write        a file holding the n datasets in its root group (replaced if it exists)
 *   bastr_h5_read         one dataset: its rank and dims (dims[4], C order), and its values into
 *                         data when data is not NULL (capacity in bytes; BASTR_E_INVALID if short)
 *   bastr_h5_write_field  the reference's field file: u1, u2[, u3] as (ia+1, ja+1, ka+1) Fortran
 *                         arrays holding the grid values in [0:ia, 0:ja, 0:max(ka,1)) and zero in
 *                         the padding, plus nstep (int32) and time when nstep >= 0; u* host arrays
 *                         x fastest, as bastr_set_state takes them
 *   bastr_h5_read_field   the grid values of u1, u2[, u3] and, when the pointers are not NULL,
 *                         nstep and time (flowini files have no counters: pass NULL)
 *   bastr_h5_last_error   message of the calling thread's last failed bastr_h5_* call
 * ------------------------------------------------------------------------------------------ */
#define BASTR_H5_F64 0
#define BASTR_H5_I32 1
typedef struct bastr_h5_dataset {
    const char* name;
    int32_t type;                /* BASTR_H5_F64 or BASTR_H5_I32 */
    int32_t rank;                /* 1..4 */
    int64_t dims[4];             /* C order, slowest first */
    const void* data;
} bastr_h5_dataset;
BASTR_API int bastr_h5_write(const char* path, const bastr_h5_dataset* sets, int32_t n);
BASTR_API int bastr_h5_read(const char* path, const char* name, int32_t type, int32_t* rank, int64_t* dims,
                            void* data, int64_t capacity);
BASTR_API int bastr_h5_write_field(const char* path, int32_t ia, int32_t ja, int32_t ka, const double* u1,
                                   const double* u2, const double* u3, int64_t nstep, double time);
BASTR_API int bastr_h5_read_field(const char* path, int32_t ia, int32_t ja, int32_t ka, double* u1, double* u2,
                                  double* u3, int64_t* nstep, double* time);
BASTR_API int bastr_h5_last_error(char* buf, int32_t n);


/* ------------------------------------------------------------------------------------------
 * Plan of a handle: its persistent grids use 1/2^share_log2 of the blocks that fit on the GPU
 * (0 = all, the default).  No reference counterpart (execution plan only; results depend on
 * it only through the order of the per-block partial sums).
 * ------------------------------------------------------------------------------------------ */
BASTR_API int bastr_set_plan(bastr_handle* h, int32_t share_log2);

/* ------------------------------------------------------------------------------------------
 * Batched ensemble: n independent realizations (each with its own bastr_params: grid size,
 * forcing, precision; one device for all) advanced together.  No reference counterpart: the
 * reference runs one field per job.  A batch of nsteps (<= 256) steps of every realization is
 * one CUDA-graph launch whose branches (one per realization) run concurrently.
 *
 *   bastr_ensemble_step    out: [n][nsteps] records, realization-major; BASTR_E_NAN if some
 *                          realization's Es+Ed became NaN (message names it)
 *   bastr_ensemble_tune    autotuner of the plans (per grid-size class), timing nsteps steps
 *                          of the graph best of reps, shares 0..max_share_log2; state restored
 *   bastr_ensemble_set_plan realization i (-1: all)
 * ------------------------------------------------------------------------------------------ */
typedef struct bastr_ensemble bastr_ensemble;
BASTR_API int bastr_ensemble_create(const bastr_params* params, int32_t n, bastr_ensemble** out);
BASTR_API int bastr_ensemble_destroy(bastr_ensemble* e);
BASTR_API int bastr_ensemble_size(bastr_ensemble* e, int32_t* n);
BASTR_API int bastr_ensemble_set_state(bastr_ensemble* e, int32_t i, const double* u1, const double* u2,
                                       const double* u3);
BASTR_API int bastr_ensemble_get_state(bastr_ensemble* e, int32_t i, double* u1, double* u2, double* u3);
BASTR_API int bastr_ensemble_step(bastr_ensemble* e, int32_t nsteps, bastr_step_out* out);
BASTR_API int bastr_ensemble_set_plan(bastr_ensemble* e, int32_t i, int32_t share_log2);
BASTR_API int bastr_ensemble_get_plan(bastr_ensemble* e, int32_t* share_log2);
BASTR_API int bastr_ensemble_tune(bastr_ensemble* e, int32_t nsteps, int32_t reps, int32_t max_share_log2,
                                  double* best_ms);
BASTR_API int bastr_ensemble_last_error(bastr_ensemble* e, char* buf, int32_t n);
/* nsteps = k * batch steps as k replays of the batch graph, device time (events on the ensemble's
 * stream around all k) in *device_ms; the records of the last batch are kept. */
BASTR_API int bastr_ensemble_run(bastr_ensemble* e, int32_t nsteps, int32_t batch, double* device_ms);

/* ------------------------------------------------------------------------------------------
 * Learned subgrid closure for a coarse 3D solve (no reference counterpart).  A local network
 * (3x3x3 stencil 3->32, then 1x1x1 32->32, 32->32, 32->3; GELU; BF16 weights and layer
 * inputs, FP32 sums) maps the velocity u [3][nz][ny][nx] to the subgrid term tau.  Device
 * pointers; weights are bastr_net_nparams() BF16 values (uint16_t bit patterns) with FP32 master
 * copies for training.  Grids of 3 nx ny nz >= 2^31 points return BASTR_E_UNSUPPORTED.
 *
 *   bastr_net_forward   out = scale * net(u), the four layers as tensor-core (tcgen05) GEMMs
 *   bastr_net_grad      loss = mean((net(u) - tau)^2) and its gradient; d_part: workspace of
 *                       nblk * (nparams + 1) floats (nblk: e.g. bastr_net_grad_blocks()); the
 *                       result is deterministic for a given nblk
 *   bastr_net_adam      one Adam step on the FP32 weights; refreshes the BF16 copy
 *   bastr_closure_apply one sub-step u <- u - dt * scale * net(u) on a 3D handle's state
 *                       (physical space, then back to the dealiased spectral state)
 * ------------------------------------------------------------------------------------------ */
BASTR_API int bastr_net_nparams(void);
BASTR_API int bastr_net_grad_blocks(void);
BASTR_API int bastr_net_forward(int32_t nx, int32_t ny, int32_t nz, const float* d_u, const uint16_t* d_w,
                                float* d_out, float scale, void* stream);
BASTR_API int bastr_net_grad(int32_t nx, int32_t ny, int32_t nz, const float* d_u, const float* d_tau,
                             const uint16_t* d_w, float* d_part, int32_t nblk, float* d_grad, double* d_loss,
                             void* stream);
BASTR_API int bastr_net_adam(float* d_w, uint16_t* d_wb, float* d_m, float* d_v, const float* d_g, int32_t t,
                             float lr, float b1, float b2, float eps, void* stream);
BASTR_API int bastr_closure_apply(bastr_handle* h, const uint16_t* d_w, float scale, double dt);

/* Closure training data from a handle's current state, on the device (no reference counterpart):
 * the box filter of width r (mean over r^d cells, decimation r) of the velocity, ub, and the
 * subgrid term tau_i = filter(u_j d_j u_i) - ub_j d_j ub_i, spectral derivatives on the fine and
 * the coarse grid, FP64 arithmetic.  d_ubar, d_tau (either may be NULL): device arrays of
 * d * (ia/r)(ja/r)(ka/r) floats, [component][coarse grid], x fastest.  r is a power of two that
 * divides every extent, leaving coarse extents of at least 16.  Allocates its work buffers (three
 * fine real grids' worth) on the first call.  bastr_ensemble_subgrid does the same for
 * realization i of an ensemble: the batched solver's output as the closure's training data. */
BASTR_API int bastr_subgrid(bastr_handle* h, int32_t r, float* d_ubar, float* d_tau);
BASTR_API int bastr_ensemble_subgrid(bastr_ensemble* e, int32_t i, int32_t r, float* d_ubar, float* d_tau);

/* ------------------------------------------------------------------------------------------
 * Slab-decomposed 3D transforms over several GPUs: the reference distributes its grid in z-slabs
 * over MPI ranks and transforms it with FFTW-MPI (decomposition fftwlink.F90:63-77, transforms
 * fftwlink.F90:324-368); these are the per-GPU pieces, on caller-owned device arrays, between
 * which the caller runs one all-to-all of equal blocks per transform (bastr_b200/slabfft.py:
 * NCCL).  Complex FP64 arrays [nz][ny][nx] (x fastest), device pointers, the caller's stream.
 *
 *   bastr_fft_lines    every line along `axis` (0 x, 1 y, 2 z) transformed in place: dir -1
 *                      e^{-ikx}, dir +1 e^{+ikx}, times `scale`; line lengths powers of two in
 *                      [16, 2048]; the first call per (device, length) makes a twiddle table
 *                      (cudaMalloc) kept until exit
 *   bastr_slab_pack    d_blocks[q][zl][yl][x] = d_slab[zl][q*nyl + yl][x], nyl = ny/nparts
 *   bastr_slab_unpack  its inverse
 * ------------------------------------------------------------------------------------------ */
BASTR_API int bastr_fft_lines(double* d_a, int32_t nx, int32_t ny, int32_t nz, int32_t axis, int32_t dir,
                              double scale, void* stream);
BASTR_API int bastr_slab_pack(const double* d_slab, double* d_blocks, int32_t nx, int32_t ny, int32_t nzl,
                              int32_t nparts, void* stream);
BASTR_API int bastr_slab_unpack(const double* d_blocks, double* d_slab, int32_t nx, int32_t ny, int32_t nzl,
                                int32_t nparts, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BASTR_GPU_H */
