/*
 * pfc_b200.h -- C ABI of the B200-native conserved phase-field-crystal stepper.
 *
 * Every entry point replaces one host interface of mcstar-libs' header API (paths
 * relative to the mcstar-libs root are cited beside each declaration).  The
 * reference-name C++ headers shipped with this library (include/mcstar/)
 * forward to these functions, so a driver written against mcstar-libs compiles
 * unchanged against this library; other languages bind the functions directly
 * (plain pointers, sizes and scalars; no C++ or torch types).
 *
 * Conventions
 *  - A context (pfc_ctx) is made for one grid shape (nx, ny, nz) and one precision.
 *    It owns every workspace (FFT twiddles and scratch, reduction and peak scratch,
 *    the FP64 k=0 slot of the fused stepper); no entry point allocates device
 *    memory after pfc_create, except that pfc_bond_order and pfc_bond_reserve grow
 *    the bond-order scratch.  Field buffers belong to the caller.
 *  - Layouts are the reference's (cuda/array_abstraction.hpp:37-70): x fastest,
 *    real field F[nz][ny][nx], half spectrum {F re, F im}[nz][ny][nx/2+1].  All
 *    field pointers are DEVICE pointers.  F = float (PFC_F32) or double (PFC_F64).
 *  - Work is enqueued on the context's stream (pfc_set_stream; default the legacy
 *    stream).  Entry points that return a host value synchronise that stream.
 *  - Errors are returned as pfc_status; nothing calls exit() or aborts.  The
 *    message of the last failure is pfc_last_error(ctx).  A context is not
 *    thread-safe: use one per host thread.
 */
#ifndef PFC_B200_H
#define PFC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pfc_status {
    PFC_OK = 0,
    PFC_ERR_INVALID = 1,      /* bad argument or shape                                */
    PFC_ERR_UNSUPPORTED = 2,  /* valid but not implemented (e.g. a prime FFT length)  */
    PFC_ERR_CUDA = 3,         /* a CUDA runtime error; see pfc_last_error            */
    PFC_ERR_NOMEM = 4,        /* a device allocation failed (pfc_create, bond order)  */
    PFC_ERR_CAPACITY = 5,     /* an output buffer was too small (count still set)    */
    PFC_ERR_NONFINITE = 6     /* the stepper's watchdog saw NaN/Inf in the state     */
} pfc_status;

typedef enum pfc_dtype { PFC_F32 = 0, PFC_F64 = 1 } pfc_dtype;

typedef struct pfc_desc {
    int nx, ny, nz;   /* real extents; 2D fields have nz = 1, 1D fields ny = nz = 1 */
    int dtype;        /* pfc_dtype                                                  */
} pfc_desc;

typedef struct pfc_ctx pfc_ctx;

/* Replaces: the implicit set-up of the reference's typedef'd GPUArray/CufftPlan
 * (cuda/array_abstraction.hpp:74-96, cuda/cufft_wrapper.hpp:68-77).  Every length
 * must have prime factors <= 31 (PFC_ERR_UNSUPPORTED otherwise); the reference's own
 * drivers keep to 2, 3, 5 (cufft_unittest/main.cu:32-36, cuda/math.hpp:125-149). */
pfc_status  pfc_create(const pfc_desc* desc, pfc_ctx** out);
pfc_status  pfc_destroy(pfc_ctx* ctx);

/* ---- kernel schedules and their autotuner (no counterpart in mcstar-libs, which leaves
 * every choice to cuFFT's planner: cuda/cufft_wrapper.hpp:68-77; its only related code
 * is the 2-3-5 size rounding of cuda/math.hpp:125-149).
 * pfc_options selects, per context, among schedules that compute the same step:
 *   z_carry      the state the stepper's z pass carries between steps: 0 A = IFFT_z(psi^)/nz
 *                (three z transforms, three field sweeps), 1 psi^ itself (two transforms,
 *                four sweeps); -1 the library's choice
 *   x_kernel     the register x pass of the kx-tiled layout: 0 one row per transform over
 *                16 lanes per row and 16 rows per CTA with a shared-memory row stage, 1 row
 *                pairs packed into one complex transform (nx = 128, 512), 2 one row per
 *                half-warp straight from and to global memory (nx = 512); -1 the library's
 *                choice
 *   tiled        the register passes' field layout: 0 the reference layout, 1 kx tiles of
 *                8 columns (contiguous z and y column blocks); -1 the library's choice
 *   radix_order  the general (mixed-radix Stockham) passes: 0 radix 8 first, 1 radices 4
 *                and 2 only, 2 the odd radices first
 *   tile_shift   the general passes' lines per CTA halved this many times (0..4), for the
 *                x rows, the y columns, the z columns and the stepper's z pass
 *   y_kernel     the register y pass between the kx-tiled layouts (ny = 512): 0 per-thread
 *                loads and stores, 1 the TMA unit moving whole tiles (bulk copies of the
 *                row-tiled blocks, tensor-map tile copies of the z-tiled pieces); -1 the
 *                library's choice
 * A choice the shape has no kernel for is PFC_ERR_UNSUPPORTED at creation.
 * pfc_tune times the step (pfc_step, FP32 or FP64 per desc) under candidate options on
 * the current device -- a coordinate search, one option at a time from the library's
 * choice -- and returns the fastest in *best (and its time per step in *ms_per_step, may
 * be NULL).  With a cache_path, results are kept in that JSON file keyed by shape,
 * precision and device, and a cached entry is returned without timing.  Tuning creates
 * and destroys contexts and allocates device memory (setup time, not the step). */
typedef struct pfc_options {
    int z_carry;
    int x_kernel;
    int tiled;
    int radix_order;
    int tile_shift[4];
    int y_kernel;
} pfc_options;
pfc_status  pfc_default_options(pfc_options* opts);
pfc_status  pfc_create_with(const pfc_desc* desc, const pfc_options* opts, pfc_ctx** out);
pfc_status  pfc_get_options(const pfc_ctx* ctx, pfc_options* opts);
pfc_status  pfc_tune(const pfc_desc* desc, const char* cache_path, pfc_options* best, double* ms_per_step);
pfc_status  pfc_set_stream(pfc_ctx* ctx, void* cuda_stream);
const char* pfc_last_error(const pfc_ctx* ctx);
const char* pfc_status_string(pfc_status s);
/* bytes of one half-spectrum buffer, (nx/2+1)*ny*nz*2*sizeof(F) -- Array::m_bytes,
 * cuda/array_abstraction.hpp:53 */
size_t      pfc_state_bytes(const pfc_ctx* ctx);
size_t      pfc_workspace_bytes(const pfc_ctx* ctx);

/* ---- FFT: replaces FFT::CufftPlan<F, R2C/C2R>::execute (cuda/cufft_wrapper.hpp:61-86).
 * Unnormalised; a round trip multiplies by nx*ny*nz.  in and out must not alias;
 * the input is preserved (cuFFT's C2R may overwrite its input; this one does not). */
pfc_status pfc_fft_r2c(pfc_ctx* ctx, const void* real_in, void* cmpl_out);
pfc_status pfc_fft_c2r(pfc_ctx* ctx, const void* cmpl_in, void* real_out);

/* ---- pointwise kernels: replace the call_kernel_ functions of cuda/kernels/ ------------ */
/* call_kernel_update_eom (cuda/kernels/eom.hpp:73-86); knoise may be NULL (eom.hpp:80) */
pfc_status pfc_update_eom(pfc_ctx* ctx, void* kpsi, const void* knonlin, const void* knoise,
                          double namp, double dt, double eps, double lx, double ly, double lz);
/* call_kernel_update_eom_with_fen (eom.hpp:103-109): also overwrites knoise with L^psi^_old */
pfc_status pfc_update_eom_with_fen(pfc_ctx* ctx, void* kpsi, const void* knonlin, void* knoise,
                                   double namp, double dt, double eps, double lx, double ly, double lz);
/* call_kernel_psi3_split (cuda/kernels/psi3_split.hpp:15-26); pot may be NULL */
pfc_status pfc_psi3_split(pfc_ctx* ctx, void* arr, const void* pot, double mu, int norm);
/* call_kernel_norm (cuda/kernels/norm.hpp:5-10) */
pfc_status pfc_norm(pfc_ctx* ctx, void* arr);
/* call_kernel_calc_fen (eom.hpp:130-141): writes the density f into lpsi like the
 * reference and returns h^3 * sum(f) in *out, summed in FP64 in a fixed order
 * (deterministic; the reference sums float atomics). */
pfc_status pfc_calc_fen(pfc_ctx* ctx, const void* psi, void* lpsi,
                        double hx, double hy, double hz, double* out);

/* ---- the reference's other propagators, pointwise on the half spectrum ---------------
 * pfc_init_eom_op: kop = {exp(-L dt), (exp(-L dt) - 1)/L}, L = k^2 ((1 - k^2)^2 + 1 - eps)
 *   (-dt where L = 0) -- kernel_init_eom_op, cuda/kernels/eom-exp.hpp:3-16.
 * pfc_update_eom_exp(_with_fen): psi^ <- kop.x psi^ + k^2 kop.y N^ - namp sqrt(N) |k| kop.y xi^
 *   (knoise may be NULL; _with_fen also writes L^ psi^_old into knoise) -- eom-exp.hpp:18-60.
 * pfc_update_el: non-conserved relaxation psi^ <- (psi^ - dt N^)/(1 + dt((1-k^2)^2 + 1 - eps)),
 *   *max_change = max_k |psi^'_k - psi^_k| -- el.hpp:3-45.
 * pfc_init_el_op / pfc_update_el_exp: its exponential form, kop = {exp(-L dt), (exp(-L dt)-1)/L},
 *   L = (1-k^2)^2 + 1 - eps; psi^ <- kop.x psi^ + kop.y N^ -- el-exp.hpp:3-60.
 * pfc_update_eom_py: the conserved update with the polynomial P(k^2) of eom.hpp:143-180,
 *   denominator 1 + dt k^2 (1 - eps - P(k^2)).
 * pfc_update_eom_hpfcnoise: the 2D conserved update with the anisotropic noise built from
 *   three noise fields, cut off above |k| = 0.25 -- eom.hpp:16-58; PFC_ERR_INVALID on 3D grids
 *   (the reference exits). */
pfc_status pfc_init_eom_op(pfc_ctx* ctx, void* kop, double dt, double eps, double lx, double ly, double lz);
pfc_status pfc_update_eom_exp(pfc_ctx* ctx, const void* kop, void* kpsi, const void* knonlin, const void* knoise,
                              double namp, double eps, double lx, double ly, double lz);
pfc_status pfc_update_eom_exp_with_fen(pfc_ctx* ctx, const void* kop, void* kpsi, const void* knonlin, void* knoise,
                                       double namp, double eps, double lx, double ly, double lz);
pfc_status pfc_update_el(pfc_ctx* ctx, void* kpsi, const void* knonlin, double dt, double eps,
                         double lx, double ly, double lz, double* max_change);
pfc_status pfc_init_el_op(pfc_ctx* ctx, void* kop, double dt, double eps, double lx, double ly, double lz);
pfc_status pfc_update_el_exp(pfc_ctx* ctx, const void* kop, void* kpsi, const void* knonlin, double* max_change);
pfc_status pfc_update_eom_py(pfc_ctx* ctx, void* kpsi, const void* knonlin, const void* knoise,
                             double namp, double dt, double eps, double lx, double ly, double lz);
pfc_status pfc_update_eom_hpfcnoise(pfc_ctx* ctx, void* kpsi, const void* knonlin, const void* knoise1,
                                    const void* knoise2, const void* knoise3, double namp, double dt, double eps,
                                    double lx, double ly, double lz);

/* ---- spectral low-pass post-processing: replaces cuda/kernels/gaussian.hpp and
 * cuda/kernels/lowpass.hpp --------------------------------------------------------------
 * pfc_gaussian_init: kgauss_k = (e, 1 - e), e = exp(-1/2 sum_a (1.1 d h_a K_a)^2), d =
 *   divs_per_sigma, h the grid spacings -- call_kernel_gaussian_init, gaussian.hpp:23-39.
 * pfc_kmult_real / pfc_kmult_imag: karr_k *= Re / Im kgauss_k -- call_kernel_kmult_real /
 *   _imag (gaussian.hpp:41-67) and _call_kernel_multassign_cmpl_with_real / _imag
 *   (lowpass.hpp:1-35).
 * pfc_square: psi <- psi^2 on the real field -- _call_kernel_square, lowpass.hpp:37-52.
 * pfc_write_lowpass_2d: spectrum *= Re kgauss (in place), then the gzip-compressed LOWPASS
 *   text dump of the low-passed half spectrum (the reference's byte format) to path --
 *   write_lowpass_2d, lowpass.hpp:54-77.  2D grids only (PFC_ERR_INVALID otherwise: the
 *   reference asserts); PFC_ERR_INVALID with a message when the file cannot be written.
 * pfc_amplitude_lowpass: the local amplitude of a 2D field -- calc_amplitude_lowpass,
 *   lowpass.hpp:78-93: spectrum *= Im kgauss (the high-pass), C2R into aux, normalise and
 *   square, R2C into spectrum, the LOWPASS dump as pfc_write_lowpass_2d (skipped when path is
 *   NULL), C2R into aux, normalise.  On return aux holds the amplitude field (real layout) and
 *   spectrum the low-passed spectrum of the squared high-pass field. */
pfc_status pfc_gaussian_init(pfc_ctx* ctx, void* kgauss, double lx, double ly, double lz, double hx, double hy,
                             double hz, double divs_per_sigma);
pfc_status pfc_kmult_real(pfc_ctx* ctx, void* karr, const void* kgauss);
pfc_status pfc_kmult_imag(pfc_ctx* ctx, void* karr, const void* kgauss);
pfc_status pfc_square(pfc_ctx* ctx, void* arr);
pfc_status pfc_write_lowpass_2d(pfc_ctx* ctx, void* spectrum, const void* kgauss, double lx, double ly,
                                const char* path);
pfc_status pfc_amplitude_lowpass(pfc_ctx* ctx, void* spectrum, void* aux, const void* kgauss, double lx, double ly,
                                 const char* path);

/* ---- noise: replaces NoiseHostApi<F> (cuda/noise.hpp:93-150) -------------------------
 * Counter-based Philox4x32-10: (seed, counter) selects the draw, so a run resumes
 * bit-exactly.  fill_kspace: complex normal, E|xi|^2 = 1, Hermitian on the i0 = 0 and
 * i0 = nx/2 planes, self-conjugate modes real with unit variance (noise.hpp:110-142).
 * fill: real N(0, sigma^2) per element (noise.hpp:108-109). */
pfc_status pfc_noise_fill_kspace(pfc_ctx* ctx, void* arr, uint64_t seed, uint64_t counter);
pfc_status pfc_noise_fill(pfc_ctx* ctx, void* arr, double sigma, uint64_t seed, uint64_t counter);

/* ---- peaks: replaces call_kernel_findpeaks / call_kernel_findpeaks_2d
 * (cuda/kernels/findpeaks.hpp:31-63, findpeaks_2d.hpp:29-56).  Cells strictly greater
 * than all 26 (3D) or 8 (nz == 1) periodic neighbours and >= ths.  Output records
 * have the layout of Maximum<F> (common/maximum_struct.hpp:3-6): {F i0, i1, i2; float
 * field} -- 16 bytes for F32, 32 for F64 -- written to DEVICE memory, sorted by linear
 * index (deterministic; the reference's order is that of racing atomics).
 * *n_found receives the total count; if it exceeds capacity, capacity records are
 * written and PFC_ERR_CAPACITY is returned. */
pfc_status pfc_findpeaks(pfc_ctx* ctx, const void* psi, double ths,
                         void* out_maxima, int capacity, int* n_found);

/* The peak finder with its records going straight to host memory while the caller keeps
 * stepping -- the overlap of findpeaks.hpp:37-53's copy and text output with the run.  The
 * search starts when the work already queued on the context's stream is done (psi is
 * ready), runs on the context's copy stream, writes the records into host_out (pinned host
 * memory mapped into the device's address space, e.g. cudaHostAlloc / cudaMallocHost; else
 * PFC_ERR_INVALID) and the count into *host_count, and the call returns at once.  psi, the
 * records and the count belong to the search until pfc_findpeaks_wait(ctx, &n) returns it
 * (n: the count; PFC_ERR_CAPACITY if it exceeded capacity, as pfc_findpeaks).  One search in
 * flight per context; a pfc_findpeaks call on the context waits for it on the device. */
pfc_status pfc_findpeaks_async(pfc_ctx* ctx, const void* psi, double ths, void* host_out, int capacity,
                               int* host_count);
pfc_status pfc_findpeaks_wait(pfc_ctx* ctx, int* n_found);

/* The same peak finder for callers that must not allocate device memory -- no
 * counterpart in mcstar-libs.  A simulation whose device memory is reserved up front
 * by its own pool, or a driver that cannot afford the device-wide synchronisation a
 * cudaMalloc may bring, cannot create a context (pfc_create allocates workspaces).
 * This entry point takes the shape, precision and stream directly, allocates
 * nothing, and keeps its scratch (block counts and their scan) in a static device
 * array of 4 MiB that every GPU loading the library holds until exit; grids of more
 * than 2^27 cells (512^3) are refused with PFC_ERR_CAPACITY and a message on stderr.
 * The first call on a device looks up the array's address (make that first call
 * before any stream capture); after a cudaDeviceReset the next call looks it up
 * again.  All calls share the array: calls whose work overlaps on the GPU race.  A
 * CUDA error already pending when the call starts is returned as PFC_ERR_CUDA (with
 * a message on stderr) and left pending.  Output, ordering, counts and errors
 * otherwise as pfc_findpeaks. */
pfc_status pfc_findpeaks_static(const void* psi, int nx, int ny, int nz, int dtype, double ths,
                                void* out_maxima, int capacity, int* n_found, void* cuda_stream);

/* ---- bond order: replaces bond_order_analysis<T> (bond-order-analysis/bond-order.hpp:4,
 * bond-order.cpp:289-349) on the GPU.  Input: n device Maximum<F> records (as written
 * by pfc_findpeaks).  Atoms with field > ths are kept; neighbours are atoms within
 * rlim under the minimum image of a cubic box of side boxsize.  For every kept atom
 * with at least one neighbour, one row of PFC_BOND_NCOL doubles is written to
 * out_rows (device), in input order, with the columns
 *   x y z nb xi q4 q6 q8 w4 q4b q6b q8b w4b w6
 * (the reference's table, bond-order.cpp:333-338, plus w6).  *n_rows receives the
 * row count; PFC_ERR_CAPACITY if it exceeds row_capacity.  Like the reference there is
 * no limit on the atom count or on the neighbours of an atom: the context's bond-order
 * scratch (about 700 bytes per atom plus 4 bytes per neighbour entry) grows inside this
 * call when an input needs more -- the one entry point that may allocate device memory
 * after pfc_create (PFC_ERR_NOMEM when that fails).  pfc_bond_reserve makes that
 * allocation up front (for max_atoms input records and max_pairs neighbour entries in
 * total); a context starts with room for 4096 atoms and 262144 entries. */
#define PFC_BOND_NCOL 14
pfc_status pfc_bond_order(pfc_ctx* ctx, const void* maxima, int n,
                          double h0, double h1, double h2, double ths, double boxsize, double rlim,
                          double* out_rows, int row_capacity, int* n_rows);
pfc_status pfc_bond_reserve(pfc_ctx* ctx, int max_atoms, long long max_pairs);

/* ---- fused stepper (no reference counterpart as one call: it is the driver loop of
 * copy, C2R, psi3_split(norm), R2C, [fill_kspace], update_eom that every mcstar-libs
 * driver runs, eom.hpp:60-86 + psi3_split.hpp + cufft_wrapper.hpp).
 * Advances kpsi (device, half spectrum, in place) by nsteps conserved semi-implicit
 * steps  psi^ <- (psi^ - dt k^2 FFT((psi^3 - C psi - mu)) + dt namp sqrt(N) |k| xi^) /
 *               (1 + dt k^2 ((1-k^2)^2 + C - eps)).
 * C = 1 is the reference's split; the k = 0 mode is carried in FP64 and is invariant.
 * Noise (namp != 0) of step t uses (seed, counter + t). */
typedef struct pfc_step_params {
    double dt, eps, mu, C;
    double namp;
    double lx, ly, lz;
    uint64_t seed, counter;
} pfc_step_params;
pfc_status pfc_step(pfc_ctx* ctx, void* kpsi, int nsteps, const pfc_step_params* params);

/* The same fused step with the reference's other update kernels in the propagator slot
 * (the driver loops of eom-exp.hpp, el.hpp and el-exp.hpp run as one call):
 *   PFC_PROP_CONSERVED      the semi-implicit conserved update above (= pfc_step)
 *   PFC_PROP_CONSERVED_EXP  exponential time differencing of the same equation,
 *                           psi^' = E psi^ + k^2 Q N^ - namp sqrt(N) |k| Q xi^ with
 *                           L = k^2 ((1 - k^2)^2 + C - eps), E = exp(-L dt), Q = (E - 1)/L
 *                           (-dt where L = 0) -- kernel_init_eom_op / kernel_update_eom,
 *                           eom-exp.hpp:3-40
 *   PFC_PROP_RELAX          non-conserved relaxation psi^' = (psi^ - dt N^) / (1 + dt
 *                           ((1 - k^2)^2 + C - eps)) -- kernel_update_el, el.hpp:3-45
 *   PFC_PROP_RELAX_EXP      its exponential form psi^' = E psi^ + Q N^, L = (1 - k^2)^2 +
 *                           C - eps -- el-exp.hpp:3-60
 *   PFC_PROP_CONSERVED_POLY the conserved update with the polynomial correlation function,
 *                           D = 1 + dt k^2 (C - eps - P(k^2)), P the degree-6 polynomial in
 *                           k^2 of kernel_update_eom_py (eom.hpp:143-180)
 *   PFC_PROP_CONSERVED_HPFC the conserved update with the anisotropic noise of
 *                           kernel_update_eom_hpfcnoise (eom.hpp:16-58): three noise fields
 *                           weighted by the wavevector, cut off above |k| = 1/4; 2D fields only
 *                           (nz = 1, PFC_ERR_INVALID otherwise, as the reference exits)
 * The relaxations move the k = 0 mode and take no noise (namp must be 0); for them
 * *max_change (may be NULL) receives max_k |psi^'_k - psi^_k| of the last step, the value
 * call_kernel_update_el returns (el.hpp:23-45), as a float.  The exponentials are
 * evaluated in the field's precision. */
typedef enum pfc_propagator {
    PFC_PROP_CONSERVED = 0,
    PFC_PROP_CONSERVED_EXP = 1,
    PFC_PROP_RELAX = 2,
    PFC_PROP_RELAX_EXP = 3,
    PFC_PROP_CONSERVED_POLY = 4,
    PFC_PROP_CONSERVED_HPFC = 5
} pfc_propagator;
pfc_status pfc_step_prop(pfc_ctx* ctx, void* kpsi, int nsteps, const pfc_step_params* params, int propagator,
                         double* max_change);
/* pfc_step with the field in host memory: the driver's `d_arr << h_arr`, the steps and
 * `h_arr << d_arr` (the copies of cuda/array_abstraction.hpp:86-96) as one call.  host_in
 * holds psi^ (state layout, pfc_state_bytes(ctx) bytes; pinned memory for the copies to
 * overlap), kpsi is the device state buffer (it holds psi^ at the end, as after pfc_step),
 * host_out receives the final psi^ (may be host_in).  The copy in runs by ky chunks
 * overlapped with the step's entry pass.  Returns when host_out is written. */
pfc_status pfc_step_host(pfc_ctx* ctx, const void* host_in, void* host_out, void* kpsi, int nsteps,
                         const pfc_step_params* params);

/* ---- ensembles (no counterpart in mcstar-libs, whose drivers run one field per process):
 * n independent fields, each with its own context (contexts and buffers must not be
 * shared between members), shape, precision and parameters, advanced together.
 * pfc_ensemble_create sorts the members into classes -- same shape, precision, kernel
 * schedules and shared parameters (dt, C, mu, box lengths, noise on or off) -- and steps the
 * members of a class as one batch: every pass of the step is one launch over all of them
 * (per-member eps, noise amplitude, seed and counter in a device table).  It captures
 * steps_per_graph steps of every class into one CUDA graph, one branch per class, so
 * classes of different sizes run concurrently;
 * pfc_ensemble_run(e, nsteps, stream) converts every member into the stepper's carried
 * form, replays the graph nsteps / steps_per_graph times (nsteps must be a multiple) and
 * converts back, then checks every member's non-finite watchdog.  Each member's noise
 * counter lives on the device and advances by one per step, so replays draw fresh noise
 * and a run resumes exactly where the last one stopped. */
typedef struct pfc_ensemble pfc_ensemble;
pfc_status  pfc_ensemble_create(int n, pfc_ctx* const* ctxs, void* const* kpsis, const pfc_step_params* params,
                                int steps_per_graph, pfc_ensemble** out);
pfc_status  pfc_ensemble_run(pfc_ensemble* e, int nsteps, void* cuda_stream);
pfc_status  pfc_ensemble_destroy(pfc_ensemble* e);
const char* pfc_ensemble_last_error(const pfc_ensemble* e);

/* ---- slab-decomposed steps (no counterpart in mcstar-libs, whose drivers run one field per
 * GPU through cuFFT): a field of nx x NY x NZ spread over G processes, each holding a
 * ky-slab of NY / G rows between steps and a z-slab of NZ / G planes inside a step.  Rank r
 * makes a ky-slab context of shape (nx, NY / G, NZ) and a z-slab context of shape
 * (nx, NY, NZ / G), both of the field's precision, and steps its ky-slab A with
 *   once:      pfc_slab_zinv(ky_ctx, kpsi_slab, A, ky0)        A = IFFT_z(psi^) / NZ
 *   per step:  all-to-all A: ky-slabs -> z-slabs (the caller, e.g. NCCL all-to-all)
 *              pfc_slab_xy(z_ctx, A_z, B_z, C, mu)              B = FFT_xy(cubic(IFFT_xy(A) / (nx NY)))
 *              all-to-all B: z-slabs -> ky-slabs
 *              pfc_slab_zpass(ky_ctx, A, B, p, ky0, NY, last)   N^ = FFT_z(B), the update with the
 *                                                               field's wavenumbers and noise keys,
 *                                                               A' = IFFT_z(psi^')/NZ, or psi^' in A
 *                                                               on the last step (then synchronises)
 * ky0 is the rank's first global ky row; p carries the field's lengths.  Slab buffers are
 * standard-layout half spectra of the slab shape (pfc_state_bytes of its context).  The
 * result equals pfc_step on the whole field up to rounding; the noise of mode k is the
 * whole field's (keys of global indices).  The z pass runs the general kernels. */
pfc_status pfc_slab_zinv(pfc_ctx* ky_ctx, const void* kpsi, void* A, int ky0);
pfc_status pfc_slab_xy(pfc_ctx* z_ctx, const void* A, void* B, double C, double mu);
pfc_status pfc_slab_zpass(pfc_ctx* ky_ctx, void* A, const void* B, const pfc_step_params* params, int ky0,
                          int ny_global, int final_step);

/* Free energy F = h^3 sum 1/2 psi ((1+lap)^2 - eps) psi + 1/4 psi^4 of the state kpsi,
 * computed as the reference does (eom.hpp:88-141: L^psi^, C2R, norm, calc_fen) with an
 * FP64 deterministic sum.  Does not modify kpsi. */
pfc_status pfc_free_energy(pfc_ctx* ctx, const void* kpsi, double eps,
                           double lx, double ly, double lz,
                           double hx, double hy, double hz, double* out);

/* ---- reverse mode of pfc_step (no counterpart in mcstar-libs) ------------------------
 * The step maps psi^ -> psi^' = D^-1 (psi^ - dt k^2 F[psi^3 - C psi - mu]) + D^-1 noise,
 * D = 1 + dt k^2 (C - eps + (1 - k^2)^2), on the real field psi = C2R(psi^)/N.  The
 * adjoint variable lam is a REAL field in a state-sized buffer: lam = dL/dpsi.
 *
 * pfc_sf_loss: L = sum over the full spectrum of (|psi^_k|^2 / N - s_k)^2, s given on
 *   the half spectrum (n_cmpl reals of the context's precision, even in k); writes
 *   lam_T = dL/dpsi to lam_out and L (FP64 sum) to *loss.
 * pfc_adjoint_step: from lam_{n+1} (in lam) and the states psi^_n, psi^_{n+1} of that
 *   step (p: the step's dt, eps, C, lengths; noise and mu do not enter), writes
 *   lam_n = dL/dpsi_n to lam and adds the step's dL/deps to *deps (may be NULL).
 *   workspace: pfc_adjoint_workspace_bytes(ctx) bytes of device memory (2 states).
 * A whole run: forward with checkpoints, then adjoint steps from the last step back,
 * recomputing the states between checkpoints (mcstar_b200.adjoint).  dL/dpsi0 of the
 * initial mean density is the sum of lam_0. */
size_t     pfc_adjoint_workspace_bytes(const pfc_ctx* ctx);
pfc_status pfc_sf_loss(pfc_ctx* ctx, const void* kpsi, const void* s_target, void* lam_out, double* loss);
pfc_status pfc_adjoint_step(pfc_ctx* ctx, const void* kpsi_n, const void* kpsi_np1, void* lam,
                            const pfc_step_params* p, void* workspace, double* deps);

/* ---- tracing (the role of TimeAcc, cuda/cutiming.hpp:5-25, inside the library) ------
 * While enabled, pfc_step brackets each kernel family with CUDA events on the
 * context's stream and counts every kernel the library launches.  Families:
 *   0 = entry/exit passes, 1 = the xy part of a step (one plane kernel, or the
 *   y/x/y passes), 2 = the z pass with the propagator, 3 = each register y pass and
 *   4 = the register x pass (3 and 4 only when those passes run on the whole field;
 *   their time is also inside family 1).
 * pfc_profile_read synchronises the stream and returns the totals since enabling. */
#define PFC_PROFILE_FAMILIES 5
typedef struct pfc_profile {
    long long launches;                          /* kernels launched by the library  */
    long long calls[PFC_PROFILE_FAMILIES];       /* bracketed launches per family    */
    double ms[PFC_PROFILE_FAMILIES];             /* summed device time per family    */
    int xy_variant;                              /* 0: general y/x/y passes; else the
                                                    fused plane kernel in use        */
    int xy_mode;                                 /* 0 general passes, 1 cluster plane
                                                    kernel, 2 register y/x/y passes  */
    int z_mode;                                  /* 0 general z pass carrying A =
                                                    IFFT_z(psi^)/nz, 1 register z pass
                                                    carrying A, 2 register z pass
                                                    carrying psi^, 3 register z pass
                                                    carrying A in the kx-tiled layout,
                                                    4 carrying psi^ in the kx-tiled
                                                    layout, 5 general z pass carrying
                                                    psi^                             */
    int z_variant;                               /* register z kernel (0: none): 1-4
                                                    square split for nz 512, 256, 128,
                                                    64; 5: 16-column tiles; 6: 16
                                                    values per thread (nz 512)       */
    int y_variant;                               /* register y kernel (0: none): 1-4
                                                    32 / 16 / 16 / 8 values per thread
                                                    for ny 512, 256, 128, 64; 5: 16
                                                    columns; 6, 7: 16 values per
                                                    thread over 32 threads (ny 512)  */
} pfc_profile;
pfc_status pfc_profile_enable(pfc_ctx* ctx, int on);
pfc_status pfc_profile_read(pfc_ctx* ctx, pfc_profile* out);

#ifdef __cplusplus
}
#endif
#endif /* PFC_B200_H */
