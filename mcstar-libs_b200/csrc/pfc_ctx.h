// The context behind the C ABI and the host launchers of every kernel family.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>
#include "pfc_internal.cuh"
#include "../../include/pfc_b200.h"

namespace pfc {

// Bytes of dynamic shared memory any general kernel may ask for (B200: 227 KB per CTA).
constexpr size_t kMaxDynSmem = 200 * 1024;
constexpr int kRedBlocks = 1184;        // 8 x 148 SMs: fixed grid of the FP64 reductions
constexpr int kPeakBlock = 256;         // cells per block of the peak finder

struct AxisPlan {
    LinePlan plan;
    int tile;          // lines per CTA (columns) or rows per CTA (x axis)
    size_t smem;       // dynamic shared memory of the kernel using this plan
};

}  // namespace pfc

struct pfc_ctx {
    int nx, ny, nz, nxh;
    int dtype;
    size_t fsize;                 // sizeof(F)
    size_t n_real, n_cmpl;        // element counts
    size_t state_bytes;           // n_cmpl * 2 * fsize
    cudaStream_t stream;
    std::string err;
    pfc_options opt;              // the options in effect (pfc_get_options)

    pfc::AxisPlan px;             // x: complex length nx/2 (even nx) or nx (odd nx)
    pfc::AxisPlan py, pz;         // y, z: complex length ny, nz
    pfc::AxisPlan pzprop;         // the stepper's z pass (two fields per tile)
    pfc::AxisPlan pxnl;           // the stepper's fused x pass
    int post_off;                 // twiddle offset of W_nx^k, k = 0..nx/2 (even nx)
    void* tw;                     // device twiddles, cx<F>
    void* work;                   // state_bytes: C2R scratch and the stepper's second field
    void* work2;                  // state_bytes: free-energy real field
    double* red;                  // kRedBlocks partial sums + 4 results
    double2* k0;                  // FP64 k = 0 mode carried by the stepper
    int* flag;                    // device status word of the stepper (non-finite watchdog)
    uint32_t* peak_mask;          // one bit per cell (peak finder)
    int* peak_counts;             // set bits per chunk of the mask
    int* peak_offsets;            // exclusive scan of peak_counts (+ total)
    int n_peak_blocks;            // chunks
    // bond order: per-atom scratch for max_atoms atoms and the neighbour lists (max_pairs
    // entries), both grown by pfc_bond_order / pfc_bond_reserve when a call needs more
    int max_atoms;
    void* bond_scratch;
    size_t bond_scratch_bytes;
    int64_t max_pairs;
    int* bond_pairs;
    int fused_z;                  // 0: general z pass; otherwise the register z kernel variant id
    int z_carry;                  // carry psi^ itself instead of A: standard layout, A = IFFT_z(psi^)/nz
                                  // in work2; tiled, psi^ z-tiled in work2 and A in the psi^ buffer
    int tiled;                    // register passes on kx-tiled fields (col_addr): A z-tiled in work2,
                                  // the x pass field row-tiled in work, the z pass input B z-tiled
                                  // in the caller's psi^ buffer
    int num_sms;                  // multiprocessors of the device the context was made on
    // batched fields (ensembles): the step's kernels run over `batch` fields of this shape
    // stored mstride complex elements apart (grid z = field); 1 and 0 for a single field
    int batch = 1;
    int64_t mstride = 0;
    int zcol_tw_off;              // twiddles of the register z kernel: W_nz^m
    int fused_y, fused_x;         // register y / x pass variants (0: none)
    int fused_zfft;               // register column kernel variant for plain z transforms (0: none)
    int zfft_tw_off;              // W_nz^m of the plain z transforms
    int ypass_tw_off;             // W_ny^m
    int xpass_tw_off;             // W_{nx/2}^m, then W_nx^k (k <= nx/2)
    int xkern;                    // the row-tiled x pass: 0 k_xrow, 1 k_xpair (row pairs), 2 k_xlane
    int ykern;                    // the y pass between the tiled layouts: 0 k_ycol3, 1 k_ybulk (TMA)
    int xpair_tw_off;             // W_nx^m, m < nx
    int xy_mode;                  // 0 general passes, 2 register y/x/y passes
    // tracing (pfc_profile_enable / pfc_profile_read)
    bool prof_on = false;
    long long launches = 0;
    long long prof_calls[PFC_PROFILE_FAMILIES] = {};
    double prof_ms[PFC_PROFILE_FAMILIES] = {};
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    struct Span { int family; size_t from, to; };     // elapsed time between two pool events
    std::vector<Span> ev_pending;
    // pfc_step_host: the copy stream and the events that order the field's ky chunks between
    // it and the context's stream (created by the first call)
    static constexpr int kHostChunks = 8;
    // the z pass of the tiled psi^-carrying schedule: the last kx tile (one column) runs on
    // this stream beside the bulk-copy kernel of the whole tiles (forked and joined by events)
    cudaStream_t side_stream = nullptr;
    cudaEvent_t side_fork = nullptr, side_join = nullptr;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t host_ev[2 * kHostChunks + 2] = {};
    // pfc_findpeaks_async: its completion event (on the copy stream), the caller's count and
    // capacity; pending until pfc_findpeaks_wait
    cudaEvent_t peaks_done = nullptr;
    int* async_count = nullptr;
    int async_capacity = 0;
    bool async_pending = false;
};

namespace pfc {

// Resident CTAs per SM of a kernel launch shape (at least 1).
template <class K>
int resident_ctas(K kernel, int threads, size_t smem) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess) {
        (void)cudaGetLastError();
        n = 1;
    }
    return n > 0 ? n : 1;
}

// ---- general FFT passes (kern_fft.cu) ----
cudaError_t set_fft_attributes(const pfc_ctx* c);
// complex FFT along y or z of a half-spectrum-shaped buffer (in may equal out)
cudaError_t launch_cols(const pfc_ctx* c, int axis, int dir, const void* in, void* out, double scale);
cudaError_t launch_rows_r2c(const pfc_ctx* c, const void* in_real, void* out_cmpl);
cudaError_t launch_rows_c2r(const pfc_ctx* c, const void* in_cmpl, void* out_real);
cudaError_t launch_rows_nonlin(const pfc_ctx* c, void* buf, const void* pot, double mul, double C, double mu);
struct ZPropArgs {
    double dt, eps, C, namp_eff, lx, ly, lz;
    uint64_t seed, counter;
    // when set, the noise counter is read from device memory (graph-replayed steps, whose
    // kernel arguments are fixed at capture, advance it on the device)
    const unsigned long long* dev_counter;
    int use_noise;
    int final_step;
    int prop;        // kPropConserved, kPropConservedExp, kPropRelax, kPropRelaxExp (pfc_internal.cuh)
    unsigned* maxc;  // relaxations: the largest |psi^' - psi^| of the step (float bits), or null
    // batched fields: per-field eps, noise amplitude and seed (null: the values above for
    // every field); k0 and dev_counter then hold one entry per field
    const MemberArgs* margs;
    // a ky-slab of a larger field (slab-decomposed steps; the general z pass only): this
    // context's ky = 0 is the field's ky0, of ny_global rows (0, 0: the context's own field)
    int ky0, ny_global;
};
cudaError_t launch_zprop(const pfc_ctx* c, void* A, const void* B, const ZPropArgs& a);
// the general z pass over the kx columns [col0, col0 + ncols); carry: A holds psi^ itself
// (updated in place) and A' = IFFT_z(psi^')/nz goes to anext (not on the final step)
cudaError_t launch_zprop_cols(const pfc_ctx* c, void* A, const void* B, const ZPropArgs& a, int col0, int ncols,
                              void* anext = nullptr, bool carry = false);
// the psi^-carrying general z pass over the whole field (nz > 1)
cudaError_t launch_zprop_carry(const pfc_ctx* c, void* kpsi, const void* B, void* anext, const ZPropArgs& a);

// ---- register-resident y and x passes (kern_passes.cu) ----
int fused_y_variant(int ny, int dtype);
int fused_x_variant(int nx, int dtype);
// the row-tiled x kernels this nx has (bit i: x kernel i; bit 0 always) and the default among them
int xkernel_variants(int nx, int dtype);
// whether the y pass has its TMA kernel for this context's y length (and the driver offers
// tensor maps)
bool ybulk_available(const pfc_ctx* c);
int default_xkernel(int variants);
cudaError_t set_pass_attributes(const pfc_ctx* c);
// y FFT of nzs consecutive planes starting at in / out (in may equal out); lay & 3 / lay
// >> 2: the layouts of in / out (col_addr; tiled: whole fields only, not in place)
cudaError_t launch_ypass(const pfc_ctx* c, int dir, const void* in, void* out, double scale, int nzs, int lay = 0);
// C2R, cubic term, R2C on the rows of nzs consecutive planes starting at b, in place;
// pot (real field, or null) starts at the same first plane; lay: 0 standard, 2 row-tiled
// (col_addr; whole fields only)
cudaError_t launch_xpass(const pfc_ctx* c, void* b, const void* pot, double mul, double C, double mu, int nzs,
                         int lay = 0);
// unnormalised real transforms of every x row (register kernels; out of place)
cudaError_t launch_xrows_r2c(const pfc_ctx* c, const void* in_real, void* out_cmpl);
cudaError_t launch_xrows_c2r(const pfc_ctx* c, const void* in_cmpl, void* out_real);
// complex FFT along z of a half-spectrum-shaped field with the register column kernel
int fused_zfft_variant(int nz, int dtype);
cudaError_t set_zfft_attributes(const pfc_ctx* c);
// (lay as launch_ypass)
// (ky0, nky: the z columns of ky in [ky0, ky0 + nky) only; nky < 0: to ny; copy, or null:
// the input columns as read, written in the output's layout -- a relayout fused with the FFT)
cudaError_t launch_zfft(const pfc_ctx* c, int dir, const void* in, void* out, double scale, int lay = 0, int ky0 = 0,
                        int nky = -1, void* copy = nullptr);

// ---- spectral low-pass post-processing (kern_lowpass.cu) ----
cudaError_t launch_gaussian_init(const pfc_ctx* c, void* g, double lx, double ly, double lz, double hx, double hy,
                                 double hz, double dps);
// a_k *= Re g_k (imag 0) or Im g_k (imag 1)
cudaError_t launch_kmult(const pfc_ctx* c, void* a, const void* g, int imag);
// real field: psi <- (psi / N)^2 (norm 1) or psi^2 (norm 0)
cudaError_t launch_norm_square(const pfc_ctx* c, void* a, int norm);
// LOWPASS dump of a device spectrum: 0 ok, 1 CUDA error (cuda_err), 2 file not written
int write_lowpass_file(const pfc_ctx* c, const void* spectrum, double lx, double ly, const char* path,
                       cudaError_t* cuda_err);

// ---- register-resident z pass (kern_zcol.cu) ----
bool zcarry_available(int fused_z);
int fused_z_variant(int nx, int nz, int dtype);
cudaError_t set_zcol_attributes(const pfc_ctx* c);
cudaError_t set_peak_attributes();
// reads A and B, writes A' (or psi^' on the last step) to O; lay bits 0, 1, 2: A, B, O
// z-tiled (col_addr layout 1; standard otherwise).  O may be A or B when it has the same
// layout.
cudaError_t launch_zcol(const pfc_ctx* c, const void* A, const void* B, void* O, const ZPropArgs& a, int lay = 0);
// the z pass that carries psi^: reads psi^ (kpsi) and B, writes psi^' and (unless last) A'
cudaError_t launch_zcarry(const pfc_ctx* c, void* kpsi, void* A, const void* B, const ZPropArgs& a);
// the same on the z-tiled layout (nz = 512): psi^ z-tiled (psi_out may be psi_in); B and A
// z-tiled (A may be B), or on the last step B and psi_out standard (psi_out may be B), no A
cudaError_t launch_zcarry_tiled(const pfc_ctx* c, const void* psi_in, const void* B, void* psi_out, void* A,
                                const ZPropArgs& a);
// FP32 field copy between the standard and the z-tiled layout (out of place)
cudaError_t launch_relayout(const pfc_ctx* c, const void* in, void* out, int to_tiled, int ky0 = 0, int nky = -1);

// ---- pointwise kernels, noise and reductions (kern_point.cu) ----
cudaError_t launch_update_eom(const pfc_ctx* c, void* kpsi, const void* knl, const void* knoise,
                              double namp, double dt, double eps, double lx, double ly, double lz,
                              int with_fen, double C);
cudaError_t launch_psi3(const pfc_ctx* c, void* arr, const void* pot, double mu, int norm, double C);
cudaError_t launch_norm(const pfc_ctx* c, void* arr);
cudaError_t launch_calc_fen(const pfc_ctx* c, const void* psi, void* lpsi, double scale);
cudaError_t launch_fen_spectral(const pfc_ctx* c, const void* kpsi, double eps, double lx, double ly, double lz);
cudaError_t launch_quartic_sum(const pfc_ctx* c, const void* psi_unnorm, double mul);
cudaError_t launch_noise_kspace(const pfc_ctx* c, void* arr, uint64_t seed, uint64_t counter);
cudaError_t launch_noise_real(const pfc_ctx* c, void* arr, double sigma, uint64_t seed, uint64_t counter);
cudaError_t launch_k0_save(const pfc_ctx* c, const void* kpsi);
cudaError_t launch_k0_restore(const pfc_ctx* c, void* kpsi);
// set (set != 0) or increment n device-side step counters
cudaError_t launch_counter(cudaStream_t st, unsigned long long* ctr, unsigned long long value, int set, int n = 1);
// reduce the kRedBlocks partials in c->red into c->red[kRedBlocks + slot]
cudaError_t launch_reduce_final(const pfc_ctx* c, int slot, double scale);

// ---- peaks (kern_peaks.cu) ----
int64_t peak_mask_words(int nx, int ny, int nz);
int peak_chunks(int nx, int ny, int nz);
// (on stream st: the context's, or the copy stream of pfc_findpeaks_async)
cudaError_t launch_findpeaks(const pfc_ctx* c, const void* psi, double ths, void* out, int capacity,
                             cudaStream_t st);

// ---- bond order (kern_bond.cu) ----
size_t bond_scratch_bytes(int max_atoms);
// grows the bond-order scratch to `atoms` atoms and `pairs` neighbour entries
cudaError_t bond_reserve(pfc_ctx* c, int atoms, int64_t pairs);
cudaError_t launch_bond_order(pfc_ctx* c, const void* maxima, int n, double h0, double h1, double h2,
                              double ths, double boxsize, double rlim, double* out_rows, int row_capacity,
                              int* n_rows_host);

// ---- the reference's other propagators (kern_variants.cu) ----
cudaError_t launch_init_eom_op(const pfc_ctx* c, void* kop, double dt, double eps, double lx, double ly, double lz);
cudaError_t launch_update_eom_exp(const pfc_ctx* c, const void* kop, void* kpsi, const void* knl, void* knoise,
                                  double namp, double eps, double lx, double ly, double lz, int with_fen);
cudaError_t launch_init_el_op(const pfc_ctx* c, void* kop, double dt, double eps, double lx, double ly, double lz);
cudaError_t launch_update_el(const pfc_ctx* c, const void* kop, void* kpsi, const void* knl, double dt, double eps,
                             double lx, double ly, double lz, double* max_change);
cudaError_t launch_update_eom_py(const pfc_ctx* c, void* kpsi, const void* knl, const void* knoise, double namp,
                                 double dt, double eps, double lx, double ly, double lz);
cudaError_t launch_update_eom_hpfcnoise(const pfc_ctx* c, void* kpsi, const void* knl, const void* n1, const void* n2,
                                        const void* n3, double namp, double dt, double eps, double lx, double ly,
                                        double lz);

// ---- adjoint of the step (kern_adjoint.cu); the sums land in red slot 3 ----
cudaError_t launch_adj_mul(const pfc_ctx* c, const void* in, void* out, const pfc_step_params* p, int mode);
cudaError_t launch_adj_eps(const pfc_ctx* c, const void* lam_hat, const void* kpsi_np1, const pfc_step_params* p);
cudaError_t launch_adj_combine(const pfc_ctx* c, void* lam, const void* psi_u, const void* b, double C);
cudaError_t launch_sf_loss(const pfc_ctx* c, const void* kpsi, const void* s_target, void* out);

}  // namespace pfc
