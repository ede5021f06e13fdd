// extern "C" entry points of libpfc_b200 (declared in include/pfc_b200.h).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include "bulk.cuh"
#include "pfc_ctx.h"

using namespace pfc;

namespace {

// The radices of an n-point Stockham plan, in stage order.  order 0: radix 8 first, then
// 4, 2, 3, 5 and the other primes up to kMaxOddRadix; 1: radices 4 and 2 only for the
// power of two; 2: the odd radices first, then 8, 4, 2.
bool factor_radices(int n, std::vector<int>& rs, int order = 0) {
    rs.clear();
    if (n < 1) return false;
    std::vector<int> pow2, odd;
    if (order == 1) {
        while (n % 4 == 0) { pow2.push_back(4); n /= 4; }
    } else {
        while (n % 8 == 0) { pow2.push_back(8); n /= 8; }
        while (n % 4 == 0) { pow2.push_back(4); n /= 4; }
    }
    while (n % 2 == 0) { pow2.push_back(2); n /= 2; }
    while (n % 3 == 0) { odd.push_back(3); n /= 3; }
    while (n % 5 == 0) { odd.push_back(5); n /= 5; }
    for (int p = 7; p <= kMaxOddRadix; p += 2) {
        bool prime = true;
        for (int d = 3; d * d <= p; d += 2) prime = prime && (p % d != 0);
        if (!prime) continue;
        while (n % p == 0) { odd.push_back(p); n /= p; }
    }
    if (order == 2) {
        rs = odd;
        rs.insert(rs.end(), pow2.begin(), pow2.end());
    } else {
        rs = pow2;
        rs.insert(rs.end(), odd.begin(), odd.end());
    }
    return n == 1 && (int)rs.size() <= kMaxStages;
}

// Appends the Stockham twiddles of an n-point plan to tab (forward sign, FP64).
bool make_plan(int n, LinePlan& p, std::vector<std::complex<double>>& tab, int order) {
    std::vector<int> rs;
    if (!factor_radices(n, rs, order)) return false;
    std::memset(&p, 0, sizeof(p));
    p.n = n;
    p.nst = (int)rs.size();
    p.by_n = make_fastdiv(n);
    int Ns = 1;
    for (int s = 0; s < p.nst; ++s) {
        const int R = rs[s];
        p.radix[s] = R;
        p.ns[s] = Ns;
        p.twoff[s] = (int)tab.size();
        for (int jj = 0; jj < Ns; ++jj)
            for (int r = 1; r < R; ++r) {
                const long long num = ((long long)r * jj) % ((long long)Ns * R);
                const double ang = -2.0 * M_PI * (double)num / (double)(Ns * R);
                tab.emplace_back(std::cos(ang), std::sin(ang));
            }
        p.rtoff[s] = (int)tab.size();
        p.by_m[s] = make_fastdiv(n / R);
        p.by_ns[s] = make_fastdiv(Ns);
        if (R > 5)
            for (int q = 0; q < R; ++q) {
                const double ang = -2.0 * M_PI * (double)q / (double)R;
                tab.emplace_back(std::cos(ang), std::sin(ang));
            }
        Ns *= R;
    }
    return true;
}

int pow2_floor(size_t v, int cap) {
    int t = 1;
    while (t * 2 <= cap && (size_t)(t * 2) <= v) t *= 2;
    return t;
}

pfc_status fail(pfc_ctx* c, pfc_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}

pfc_status cuda_fail(pfc_ctx* c, cudaError_t e, const char* where) {
    return fail(c, PFC_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define PFC_CUDA(call, where)                       \
    do {                                            \
        cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
    } while (0)

#define PFC_CHECK_CTX()                                                      \
    do {                                                                     \
        if (!ctx) return PFC_ERR_INVALID;                                    \
    } while (0)

void free_ctx(pfc_ctx* c) {
    if (!c) return;
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : c->host_ev)
        if (e) cudaEventDestroy(e);
    if (c->peaks_done) cudaEventDestroy(c->peaks_done);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->side_fork) cudaEventDestroy(c->side_fork);
    if (c->side_join) cudaEventDestroy(c->side_join);
    if (c->side_stream) cudaStreamDestroy(c->side_stream);
    void* ptrs[] = {c->tw,          c->work,         c->work2,        c->red,       c->k0,
                    c->flag,        c->peak_counts,  c->peak_offsets, c->bond_scratch, c->bond_pairs,
                    c->peak_mask};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete c;
}

// Accumulates the device time of every bracketed launch recorded so far.
cudaError_t prof_resolve(pfc_ctx* c) {
    if (c->ev_pending.empty()) { c->ev_used = 0; return cudaSuccess; }
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e) return e;
    for (auto& p : c->ev_pending) {
        float ms = 0.f;
        if ((e = cudaEventElapsedTime(&ms, c->ev_pool[p.from], c->ev_pool[p.to]))) return e;
        c->prof_ms[p.family] += ms;
        c->prof_calls[p.family] += 1;
    }
    c->ev_pending.clear();
    c->ev_used = 0;
    return cudaSuccess;
}

// Runs launch() (which enqueues `n` kernels) bracketed by events when tracing is on.
template <typename F>
cudaError_t traced(pfc_ctx* c, int family, int n, F&& launch) {
    c->launches += n;
    if (!c->prof_on) return launch();
    if (c->ev_used + 2 > c->ev_pool.size()) {
        cudaError_t e = prof_resolve(c);
        if (e) return e;
    }
    const size_t i = c->ev_used;
    c->ev_used += 2;
    cudaError_t e = cudaEventRecord(c->ev_pool[i], c->stream);
    if (e) return e;
    if ((e = launch())) return e;
    if ((e = cudaEventRecord(c->ev_pool[i + 1], c->stream))) return e;
    c->ev_pending.push_back({family, i, i + 1});
    return cudaSuccess;
}

// The register xy part (y-inverse, x, y-forward passes) with each pass bracketed too:
// family 1 gets the whole part, 3 each y pass and 4 the x pass.
template <typename FY1, typename FX, typename FY2>
cudaError_t traced_xy3(pfc_ctx* c, FY1&& y1, FX&& x, FY2&& y2) {
    c->launches += 3;
    if (!c->prof_on) {
        cudaError_t e = y1();
        if (!e) e = x();
        if (!e) e = y2();
        return e;
    }
    if (c->ev_used + 4 > c->ev_pool.size()) {
        cudaError_t e = prof_resolve(c);
        if (e) return e;
    }
    const size_t i = c->ev_used;
    c->ev_used += 4;
    cudaError_t e;
    if ((e = cudaEventRecord(c->ev_pool[i], c->stream)) || (e = y1()) ||
        (e = cudaEventRecord(c->ev_pool[i + 1], c->stream)) || (e = x()) ||
        (e = cudaEventRecord(c->ev_pool[i + 2], c->stream)) || (e = y2()) ||
        (e = cudaEventRecord(c->ev_pool[i + 3], c->stream)))
        return e;
    c->ev_pending.push_back({1, i, i + 3});
    c->ev_pending.push_back({3, i, i + 1});
    c->ev_pending.push_back({4, i + 1, i + 2});
    c->ev_pending.push_back({3, i + 2, i + 3});
    return cudaSuccess;
}

// ---- the pieces of a step (enqueue only; capturable in a CUDA graph) -----------------------
ZPropArgs zargs(const pfc_ctx* c, const pfc_step_params* p) {
    ZPropArgs za;
    za.dt = p->dt; za.eps = p->eps; za.C = p->C;
    za.namp_eff = p->namp * std::sqrt((double)c->n_real);
    za.lx = p->lx; za.ly = p->ly; za.lz = p->lz;
    za.seed = p->seed;
    za.counter = p->counter;
    za.dev_counter = nullptr;
    za.use_noise = p->namp != 0.0;
    za.final_step = 0;
    za.prop = PFC_PROP_CONSERVED;
    za.maxc = nullptr;
    za.margs = nullptr;
    za.ky0 = 0;
    za.ny_global = 0;
    return za;
}

// Layout codes of col_addr (kx-tiled fields of the tiled stepper)
constexpr int kLayZ = 1, kLayRow = 2;

// Where the stepper's mixed-grid field A = IFFT_z(psi^)/nz lives: in work2 beside the
// carried psi^ (z_carry) or z-tiled (tiled), in work when tiled with psi^ carried z-tiled in
// work2 (the psi^ buffer then holds the row-tiled field of the x pass), else in place of
// psi^.
void* carried_A(pfc_ctx* ctx, void* kpsi) {
    if (ctx->tiled) return ctx->z_carry ? ctx->work : ctx->work2;
    return ctx->z_carry ? ctx->work2 : kpsi;
}
// The row-tiled field of the x pass (tiled schedules): the psi^ buffer when psi^ is carried
// in work2 and A in work, else work.
void* row_field(pfc_ctx* ctx, void* kpsi) { return ctx->z_carry ? kpsi : ctx->work; }

// psi^ -> A = IFFT_z(psi^)/nz; the k = 0 mode is kept in FP64
// complex FFT along z of a half-spectrum field: the register column kernel where the
// length has one, else the general column pass
cudaError_t zcols(const pfc_ctx* ctx, int dir, const void* in, void* out, double scale, int lay = 0) {
    if (ctx->fused_zfft) return launch_zfft(ctx, dir, in, out, scale, lay);
    if (lay) return cudaErrorNotSupported;
    return launch_cols(ctx, 2, dir, in, out, scale);
}
// the same along y (register kernel only together with the register x rows)
cudaError_t ycols(const pfc_ctx* ctx, int dir, const void* in, void* out) {
    if (ctx->fused_y && ctx->fused_x) return launch_ypass(ctx, dir, in, out, 1.0, ctx->nz);
    return launch_cols(ctx, 1, dir, in, out, 1.0);
}

cudaError_t step_entry(pfc_ctx* ctx, void* kpsi) {
    if (ctx->tiled && ctx->z_carry)
        // one pass: the z columns of psi^ (standard layout) read once, A = IFFT_z/nz into work
        // and psi^ itself into work2, both z-tiled
        return traced(ctx, 0, 2, [&] {
            cudaError_t e = launch_k0_save(ctx, kpsi);
            if (!e) e = launch_zfft(ctx, 1, kpsi, ctx->work, 1.0 / ctx->nz, kLayZ << 2, 0, -1, ctx->work2);
            return e;
        });
    return traced(ctx, 0, ctx->nz > 1 ? 2 : 1, [&] {
        cudaError_t e = launch_k0_save(ctx, kpsi);
        if (e || ctx->nz == 1) return e;
        return zcols(ctx, 1, kpsi, carried_A(ctx, kpsi), 1.0 / ctx->nz, ctx->tiled ? kLayZ << 2 : 0);
    });
}

// back to psi^ after non-final steps: FFT_z(A) with the k = 0 mode restored from FP64
// (nothing to do when psi^ is carried)
cudaError_t step_exit(pfc_ctx* ctx, void* kpsi) {
    if (ctx->tiled && ctx->z_carry) return traced(ctx, 0, 1, [&] { return launch_relayout(ctx, ctx->work2, kpsi, 0); });
    if (ctx->z_carry) return cudaSuccess;
    return traced(ctx, 0, ctx->nz > 1 ? 2 : 1, [&] {
        cudaError_t e = ctx->nz > 1 ? zcols(ctx, -1, carried_A(ctx, kpsi), kpsi, 1.0, ctx->tiled ? kLayZ : 0)
                                    : cudaSuccess;
        if (e) return e;
        return launch_k0_restore(ctx, kpsi);
    });
}

// B = FFT_xy(cubic term of IFFT_xy(A)) on the mixed grid.  Tiled: A (z-tiled) -> the
// row-tiled field, the x pass in place, then B z-tiled (or, on the last step, in the
// standard layout): with psi^ carried, A and B in work and the row-tiled field in the psi^
// buffer; with A carried (in work2), the row-tiled field in work and B in the psi^ buffer,
// where the last z pass then writes psi^' in place.
cudaError_t step_xy(pfc_ctx* ctx, void* kpsi, const pfc_step_params* p, bool last) {
    const void* A = carried_A(ctx, kpsi);
    void* B = ctx->work;
    const double mul = 1.0 / ((double)ctx->nx * (double)ctx->ny);
    if (ctx->tiled) {
        void* R = row_field(ctx, kpsi);
        void* Bt = ctx->z_carry ? ctx->work : kpsi;
        return traced_xy3(
            ctx, [&] { return launch_ypass(ctx, 1, A, R, 1.0, ctx->nz, kLayZ | kLayRow << 2); },
            [&] { return launch_xpass(ctx, R, nullptr, mul, p->C, p->mu, ctx->nz, kLayRow); },
            [&] { return launch_ypass(ctx, -1, R, Bt, 1.0, ctx->nz, kLayRow | (last ? 0 : kLayZ << 2)); });
    }
    if (ctx->xy_mode == 2)
        return traced_xy3(
            ctx, [&] { return launch_ypass(ctx, 1, A, B, 1.0, ctx->nz); },
            [&] { return launch_xpass(ctx, B, nullptr, mul, p->C, p->mu, ctx->nz); },
            [&] { return launch_ypass(ctx, -1, B, B, 1.0, ctx->nz); });
    return traced(ctx, 1, ctx->ny > 1 ? 3 : 1, [&] {
        cudaError_t e;
        if (ctx->ny > 1) e = launch_cols(ctx, 1, 1, A, B, 1.0);
        else e = cudaMemcpyAsync(B, A, ctx->state_bytes * ctx->batch, cudaMemcpyDeviceToDevice, ctx->stream);
        if (e) return e;
        if ((e = launch_rows_nonlin(ctx, B, nullptr, mul, p->C, p->mu))) return e;
        return ctx->ny > 1 ? launch_cols(ctx, 1, -1, B, B, 1.0) : cudaSuccess;
    });
}

// the z pass with the semi-implicit update.  Tiled, psi^ carried: psi^ in work2 and B in
// work -> psi^' (work2) and A' (work); the last step writes psi^' into the psi^ buffer
// (standard layout).  Tiled, A carried: B is in the psi^ buffer; A' stays z-tiled in work2,
// and the last step writes psi^' over B (standard layout, in place).
cudaError_t step_z(pfc_ctx* ctx, void* kpsi, const ZPropArgs& za) {
    void* B = ctx->work;
    if (ctx->tiled && ctx->z_carry)
        return traced(ctx, 2, 1, [&] {
            return launch_zcarry_tiled(ctx, ctx->work2, ctx->work, za.final_step ? kpsi : ctx->work2,
                                       za.final_step ? nullptr : ctx->work, za);
        });
    if (ctx->tiled) {
        void* A = ctx->work2;
        if (za.final_step) return traced(ctx, 2, 1, [&] { return launch_zcol(ctx, A, kpsi, kpsi, za, 1); });
        return traced(ctx, 2, 1, [&] { return launch_zcol(ctx, A, kpsi, A, za, 7); });
    }
    if (ctx->z_carry && !ctx->fused_z)
        return traced(ctx, 2, 1, [&] { return launch_zprop_carry(ctx, kpsi, B, ctx->work2, za); });
    if (ctx->z_carry) return traced(ctx, 2, 1, [&] { return launch_zcarry(ctx, kpsi, ctx->work2, B, za); });
    if (ctx->fused_z) return traced(ctx, 2, 1, [&] { return launch_zcol(ctx, kpsi, B, kpsi, za); });
    return traced(ctx, 2, 1, [&] { return launch_zprop(ctx, kpsi, B, za); });
}

}  // namespace

// ---- ensembles: many independent fields advanced by one CUDA graph launch -------------------
// Members are grouped into classes of equal shape, precision, kernel schedules and shared
// step parameters (dt, C, mu, lengths, noise on or off).  A class steps all of its members
// with one launch per pass: its context has the members' shape with batch = members, and
// its buffers hold every member's state and workspaces one field apart (the kernels take
// the field from grid z).  eps, the noise amplitude, the seed and the noise counter are per
// member (a device table).  The graph holds one branch per class.
struct pfc_ensemble {
    std::vector<pfc_ctx*> ctx;
    std::vector<void*> kpsi;
    std::vector<pfc_step_params> p;
    struct Class {
        pfc_ctx* cc = nullptr;              // the class context (batch = members)
        std::vector<int> members;           // member indices, in batch order
        void* state = nullptr;              // the members' psi^ buffers (the kpsi role), one field apart
        MemberArgs* margs = nullptr;        // per-member eps, noise amplitude, seed (device)
        unsigned long long* ctr = nullptr;  // per-member noise counters (device)
        cudaStream_t st = nullptr;
        cudaEvent_t join = nullptr;
    };
    std::vector<Class> cls;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int steps_per_graph = 1;
    std::string err;
};

namespace {
void free_ensemble(pfc_ensemble* e) {
    if (!e) return;
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    for (auto& k : e->cls) {
        if (k.join) cudaEventDestroy(k.join);
        if (k.st) cudaStreamDestroy(k.st);
        if (k.state) cudaFree(k.state);
        if (k.margs) cudaFree(k.margs);
        if (k.ctr) cudaFree(k.ctr);
        if (k.cc) free_ctx(k.cc);
    }
    if (e->fork) cudaEventDestroy(e->fork);
    delete e;
}

// Members that may share a class: same shape, precision, schedules and shared parameters.
bool same_class(const pfc_ctx* a, const pfc_step_params& pa, const pfc_ctx* b, const pfc_step_params& pb) {
    const pfc_options &oa = a->opt, &ob = b->opt;
    return a->nx == b->nx && a->ny == b->ny && a->nz == b->nz && a->dtype == b->dtype && oa.z_carry == ob.z_carry &&
           oa.x_kernel == ob.x_kernel && oa.tiled == ob.tiled && oa.radix_order == ob.radix_order &&
           std::memcmp(oa.tile_shift, ob.tile_shift, sizeof(oa.tile_shift)) == 0 && oa.y_kernel == ob.y_kernel &&
           pa.dt == pb.dt && pa.C == pb.C &&
           pa.mu == pb.mu && pa.lx == pb.lx && pa.ly == pb.ly && pa.lz == pb.lz && (pa.namp != 0.0) == (pb.namp != 0.0);
}

// A context of the shape and schedules of `like` holding m fields (batch = m).
cudaError_t make_class_context(const pfc_ctx* like, int m, pfc_ctx** out) {
    pfc_desc d{like->nx, like->ny, like->nz, like->dtype};
    pfc_ctx* c = nullptr;
    if (pfc_create_with(&d, &like->opt, &c) != PFC_OK) return cudaErrorMemoryAllocation;
    cudaFree(c->work);
    cudaFree(c->work2);
    cudaFree(c->k0);
    c->work = c->work2 = nullptr;
    c->k0 = nullptr;
    cudaError_t e = cudaMalloc(&c->work, c->state_bytes * m);
    if (!e) e = cudaMalloc(&c->work2, c->state_bytes * m);
    if (!e) e = cudaMalloc((void**)&c->k0, sizeof(double2) * m);
    if (e) {
        free_ctx(c);
        return e;
    }
    c->batch = m;
    c->mstride = (int64_t)c->n_cmpl;
    *out = c;
    return cudaSuccess;
}
}  // namespace

extern "C" {

const char* pfc_status_string(pfc_status s) {
    switch (s) {
        case PFC_OK: return "ok";
        case PFC_ERR_INVALID: return "invalid argument";
        case PFC_ERR_UNSUPPORTED: return "unsupported";
        case PFC_ERR_CUDA: return "CUDA error";
        case PFC_ERR_NOMEM: return "out of device memory";
        case PFC_ERR_CAPACITY: return "output capacity exceeded";
        case PFC_ERR_NONFINITE: return "non-finite value in the state";
    }
    return "unknown status";
}

const char* pfc_last_error(const pfc_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

pfc_status pfc_default_options(pfc_options* o) {
    if (!o) return PFC_ERR_INVALID;
    o->z_carry = -1;
    o->x_kernel = -1;
    o->tiled = -1;
    o->radix_order = 0;
    for (int i = 0; i < 4; ++i) o->tile_shift[i] = 0;
    o->y_kernel = -1;
    return PFC_OK;
}

pfc_status pfc_create(const pfc_desc* d, pfc_ctx** out) { return pfc_create_with(d, nullptr, out); }

pfc_status pfc_get_options(const pfc_ctx* ctx, pfc_options* o) {
    if (!ctx || !o) return PFC_ERR_INVALID;
    *o = ctx->opt;
    return PFC_OK;
}

pfc_status pfc_create_with(const pfc_desc* d, const pfc_options* opts, pfc_ctx** out) {
    if (!d || !out) return PFC_ERR_INVALID;
    *out = nullptr;
    pfc_options o;
    pfc_default_options(&o);
    if (opts) o = *opts;
    if (o.z_carry < -1 || o.z_carry > 1 || o.x_kernel < -1 || o.x_kernel > 2 || o.tiled < -1 || o.tiled > 1 ||
        o.radix_order < 0 || o.radix_order > 2 || o.y_kernel < -1 || o.y_kernel > 1)
        return PFC_ERR_INVALID;
    for (int i = 0; i < 4; ++i)
        if (o.tile_shift[i] < 0 || o.tile_shift[i] > 4) return PFC_ERR_INVALID;
    if (d->nx < 1 || d->ny < 1 || d->nz < 1) return PFC_ERR_INVALID;
    // the reference plans a 1D transform of the first row for (nx, 1, nz > 1)
    // (technicalities.hpp:16-32 with cufft_wrapper.hpp:72-75); such shapes are refused.
    if (d->ny == 1 && d->nz > 1) return PFC_ERR_INVALID;
    if (d->dtype != PFC_F32 && d->dtype != PFC_F64) return PFC_ERR_INVALID;
    pfc_ctx* c = new (std::nothrow) pfc_ctx();
    if (!c) return PFC_ERR_NOMEM;
    c->nx = d->nx; c->ny = d->ny; c->nz = d->nz;
    c->nxh = d->nx / 2 + 1;
    c->dtype = d->dtype;
    c->fsize = d->dtype == PFC_F64 ? 8 : 4;
    c->n_real = (size_t)d->nx * d->ny * d->nz;
    c->n_cmpl = (size_t)c->nxh * d->ny * d->nz;
    c->state_bytes = c->n_cmpl * 2 * c->fsize;
    c->stream = 0;
    const size_t csz = 2 * c->fsize;

    std::vector<std::complex<double>> tab;
    const bool even = (c->nx % 2) == 0;
    const int lx = even ? c->nx / 2 : c->nx;
    if (!make_plan(lx, c->px.plan, tab, o.radix_order) || !make_plan(c->ny, c->py.plan, tab, o.radix_order) ||
        !make_plan(c->nz, c->pz.plan, tab, o.radix_order)) {
        free_ctx(c);
        return PFC_ERR_UNSUPPORTED;
    }
    c->post_off = (int)tab.size();
    for (int k = 0; k <= c->nx / 2; ++k) {
        const double ang = -2.0 * M_PI * (double)k / (double)c->nx;
        tab.emplace_back(std::cos(ang), std::sin(ang));
    }
    auto roots = [&](int n, int count) {
        for (int m = 0; m < count; ++m) {
            const double ang = -2.0 * M_PI * (double)m / (double)n;
            tab.emplace_back(std::cos(ang), std::sin(ang));
        }
    };
    c->fused_z = fused_z_variant(c->nx, c->nz, c->dtype);
    c->zcol_tw_off = (int)tab.size();
    if (c->fused_z) roots(c->nz, c->nz);
    c->fused_y = fused_y_variant(c->ny, c->dtype);
    c->fused_x = fused_x_variant(c->nx, c->dtype);
    if (!(c->fused_y && c->fused_x)) c->fused_y = c->fused_x = 0;
    c->ypass_tw_off = (int)tab.size();
    if (c->fused_y) roots(c->ny, c->ny);
    c->xpass_tw_off = (int)tab.size();
    if (c->fused_x) {
        roots(c->nx / 2, c->nx / 2);
        roots(c->nx, c->nx / 2 + 1);
    }
    // the kernel of the row-tiled x pass: rows (0), row pairs (1) or a row per half-warp (2),
    // among those the length has
    {
        const int have = c->fused_x ? xkernel_variants(c->nx, c->dtype) : 1;
        if (o.x_kernel > 0 && !((have >> o.x_kernel) & 1)) {
            free_ctx(c);
            return PFC_ERR_UNSUPPORTED;
        }
        c->xkern = o.x_kernel >= 0 ? o.x_kernel : default_xkernel(have);
    }
    c->xpair_tw_off = (int)tab.size();
    if (c->xkern == 1) roots(c->nx, c->nx);
    // (its line stride ny (nx/2+1) is a 32-bit int)
    c->fused_zfft = c->nz > 1 && c->n_cmpl < (1ull << 31) ? fused_zfft_variant(c->nz, c->dtype) : 0;
    c->zfft_tw_off = (int)tab.size();
    if (c->fused_zfft) roots(c->nz, c->nz);
    // xy part of a step: the register y/x/y passes where the y and x lengths have them,
    // else the general passes
    c->xy_mode = c->fused_y ? 2 : 0;
    // the z pass carries A = IFFT_z(psi^)/nz (three z transforms, three field sweeps) or
    // psi^ itself (two transforms, four sweeps); a field with nz = 1 has no z transforms
    if (o.z_carry == 1 && !c->fused_z && c->nz == 1) {
        free_ctx(c);
        return PFC_ERR_UNSUPPORTED;
    }
    // kx-tiled fields (measured faster: whole-block z and y columns); tiled = 0 keeps the
    // standard layout.  Needs the register y, x, z passes, whole fields, and the register
    // column kernel for the entry / exit z transforms.
    c->tiled = c->fused_z && c->fused_zfft && c->xy_mode == 2 && c->fused_y;
    if (o.tiled == 1 && !c->tiled) {
        free_ctx(c);
        return PFC_ERR_UNSUPPORTED;
    }
    if (o.tiled == 0) c->tiled = 0;
    // The library carries psi^ where the tiled bulk-copy z kernel exists (nz = 512): faster
    // (two z transforms; 0.344 against 0.447 ms at 512^3) and no FP32 round trip of the state
    // through IFFT_z / FFT_z each step (its FP32 error against FP64 is the reference cuFFT
    // path's or lower at 1, 10, 100, 1000 steps); elsewhere A.
    // The general (Stockham) z pass carries psi^ too unless the options ask for A: one
    // transform fewer per column, the kernels being issue-bound at the lengths they serve.
    const bool gen_carry = !c->fused_z && c->nz > 1 && o.z_carry != 0;
    const bool carry =
        gen_carry || (c->fused_z && (o.z_carry == 1 || (o.z_carry == -1 && c->tiled && c->fused_z == 6)));
    // psi^ carried: tiled, with the 16-values-per-thread kernel (nz 512); standard layout,
    // with the square split.  A tiled context whose z length has no tiled psi^-carrying
    // kernel carries A unless the options ask for psi^ (then the layout is standard).
    if (carry && c->tiled && c->fused_z != 6) {
        if (o.z_carry == 1 && o.tiled == 1) {
            free_ctx(c);
            return PFC_ERR_UNSUPPORTED;
        }
        if (o.z_carry == 1) c->tiled = 0;
    }
    c->z_carry = carry && (!c->tiled || c->fused_z == 6);
    if (!c->tiled && c->z_carry && c->fused_z == 6) c->fused_z = 1;
    // the reference-layout psi^-carrying register z pass exists for nz = 64, 128, 256, 512
    if (c->z_carry && !c->tiled && c->fused_z && !zcarry_available(c->fused_z)) {
        free_ctx(c);
        return PFC_ERR_UNSUPPORTED;
    }
    // the y pass between the tiled layouts: per-thread accesses (0) or the TMA unit (1),
    // for the y lengths that have the latter (used when the layout is tiled)
    {
        const bool tma = ybulk_available(c);
        if (o.y_kernel == 1 && !tma) {
            free_ctx(c);
            return PFC_ERR_UNSUPPORTED;
        }
        c->ykern = o.y_kernel >= 0 ? o.y_kernel : (tma ? 1 : 0);
    }
    {
        int dev = 0;
        c->num_sms = 148;
        if (cudaGetDevice(&dev) == cudaSuccess)
            cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev);
        cudaGetLastError();
    }
    // tiles: two ping-pong buffers of `tile` lines per CTA, halved tile_shift times; a pass
    // with few lines takes smaller tiles, so that it still has two CTAs per SM
    auto shifted = [](int t, int sh) { return std::max(1, t >> sh); };
    auto fit = [&](int t, int64_t lines) {
        while (t > 1 && (lines + t - 1) / t < 2 * (int64_t)c->num_sms) t >>= 1;
        return t;
    };
    const int64_t nyz = (int64_t)c->ny * c->nz;
    c->px.tile = shifted(fit(pow2_floor((64 * 1024) / (2 * (size_t)lx * csz), 16), nyz), o.tile_shift[0]);
    c->px.smem = 2 * (size_t)c->px.tile * line_stride(lx) * csz;
    c->py.tile = shifted(fit(pow2_floor((64 * 1024) / (2 * (size_t)c->ny * csz), 16), (int64_t)c->nxh * c->nz),
                         o.tile_shift[1]);
    c->py.smem = 2 * (size_t)c->py.tile * line_stride(c->ny) * csz;
    c->pz.tile = shifted(fit(pow2_floor((64 * 1024) / (2 * (size_t)c->nz * csz), 16), (int64_t)c->nxh * c->ny),
                         o.tile_shift[2]);
    c->pz.smem = 2 * (size_t)c->pz.tile * line_stride(c->nz) * csz;
    c->pzprop.tile = shifted(fit(pow2_floor((96 * 1024) / (4 * (size_t)c->nz * csz), 8), (int64_t)c->nxh * c->ny),
                             o.tile_shift[3]);
    c->pzprop.smem = 4 * (size_t)c->pzprop.tile * line_stride(c->nz) * csz;
    if (c->px.smem > kMaxDynSmem || c->py.smem > kMaxDynSmem || c->pz.smem > kMaxDynSmem ||
        c->pzprop.smem > kMaxDynSmem) {
        free_ctx(c);
        return PFC_ERR_UNSUPPORTED;
    }
    c->n_peak_blocks = peak_chunks(c->nx, c->ny, c->nz);
    // bond order starts with room for 4096 atoms and 64 neighbours each; pfc_bond_order
    // grows both when a call needs more (pfc_bond_reserve does it up front)
    c->max_atoms = 4096;
    c->bond_scratch_bytes = bond_scratch_bytes(c->max_atoms);
    c->max_pairs = 64 * 4096;

    cudaError_t e = cudaSuccess;
    auto alloc = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    alloc(&c->tw, tab.size() * csz);
    alloc(&c->work, c->state_bytes);
    alloc(&c->work2, c->state_bytes);
    alloc((void**)&c->red, sizeof(double) * (kRedBlocks + 8));
    alloc((void**)&c->k0, sizeof(double2));
    alloc((void**)&c->flag, sizeof(int) * 4);
    alloc((void**)&c->peak_mask, sizeof(uint32_t) * (size_t)peak_mask_words(c->nx, c->ny, c->nz));
    alloc((void**)&c->peak_counts, sizeof(int) * c->n_peak_blocks);
    alloc((void**)&c->peak_offsets, sizeof(int) * (c->n_peak_blocks + 1));
    alloc(&c->bond_scratch, c->bond_scratch_bytes);
    alloc((void**)&c->bond_pairs, sizeof(int) * (size_t)c->max_pairs);
    if (e != cudaSuccess) {
        cudaGetLastError();
        free_ctx(c);
        return e == cudaErrorMemoryAllocation ? PFC_ERR_NOMEM : PFC_ERR_CUDA;
    }
    if (c->dtype == PFC_F64) {
        e = cudaMemcpy(c->tw, tab.data(), tab.size() * csz, cudaMemcpyHostToDevice);
    } else {
        std::vector<float2> t32(tab.size());
        for (size_t i = 0; i < tab.size(); ++i) t32[i] = make_float2((float)tab[i].real(), (float)tab[i].imag());
        e = cudaMemcpy(c->tw, t32.data(), tab.size() * csz, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemset(c->flag, 0, sizeof(int) * 4);
    if (e == cudaSuccess) e = set_fft_attributes(c);
    if (e == cudaSuccess && c->fused_z) e = set_zcol_attributes(c);
    if (e == cudaSuccess && c->fused_y) e = set_pass_attributes(c);
    if (e == cudaSuccess && c->fused_zfft) e = set_zfft_attributes(c);
    if (e == cudaSuccess) e = set_peak_attributes();
    if (e == cudaSuccess && c->tiled && c->z_carry) {
        e = cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking);
        if (!e) e = cudaEventCreateWithFlags(&c->side_fork, cudaEventDisableTiming);
        if (!e) e = cudaEventCreateWithFlags(&c->side_join, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        free_ctx(c);
        return PFC_ERR_CUDA;
    }
    // the options in effect (the library's choices filled in)
    c->opt = o;
    c->opt.z_carry = c->z_carry ? 1 : 0;
    c->opt.x_kernel = c->xkern;
    c->opt.y_kernel = c->ykern;
    c->opt.tiled = c->tiled ? 1 : 0;
    *out = c;
    return PFC_OK;
}

pfc_status pfc_destroy(pfc_ctx* ctx) {
    PFC_CHECK_CTX();
    free_ctx(ctx);
    return PFC_OK;
}

pfc_status pfc_set_stream(pfc_ctx* ctx, void* stream) {
    PFC_CHECK_CTX();
    ctx->stream = (cudaStream_t)stream;
    return PFC_OK;
}

size_t pfc_state_bytes(const pfc_ctx* ctx) { return ctx ? ctx->state_bytes : 0; }

size_t pfc_workspace_bytes(const pfc_ctx* ctx) {
    if (!ctx) return 0;
    return 2 * ctx->state_bytes + ctx->bond_scratch_bytes + sizeof(int) * (size_t)ctx->max_pairs +
           sizeof(double) * (kRedBlocks + 8) + sizeof(int) * (2 * ctx->n_peak_blocks + 1) +
           sizeof(uint32_t) * (size_t)peak_mask_words(ctx->nx, ctx->ny, ctx->nz);
}

// ---- FFT ------------------------------------------------------------------------------
pfc_status pfc_fft_r2c(pfc_ctx* ctx, const void* in, void* out) {
    PFC_CHECK_CTX();
    if (!in || !out) return fail(ctx, PFC_ERR_INVALID, "pfc_fft_r2c: null buffer");
    const bool reg_xy = ctx->fused_x && ctx->fused_y;
    if (reg_xy) PFC_CUDA(launch_xrows_r2c(ctx, in, out), "pfc_fft_r2c rows");
    else PFC_CUDA(launch_rows_r2c(ctx, in, out), "pfc_fft_r2c rows");
    if (ctx->ny > 1) PFC_CUDA(ycols(ctx, -1, out, out), "pfc_fft_r2c y");
    if (ctx->nz > 1) PFC_CUDA(zcols(ctx, -1, out, out, 1.0), "pfc_fft_r2c z");
    ctx->launches += 1 + (ctx->ny > 1) + (ctx->nz > 1);
    return PFC_OK;
}

pfc_status pfc_fft_c2r(pfc_ctx* ctx, const void* in, void* out) {
    PFC_CHECK_CTX();
    if (!in || !out) return fail(ctx, PFC_ERR_INVALID, "pfc_fft_c2r: null buffer");
    const void* src = in;  // the input is left unchanged: the passes run in the workspace
    if (ctx->nz > 1) { PFC_CUDA(zcols(ctx, 1, src, ctx->work, 1.0), "pfc_fft_c2r z"); src = ctx->work; }
    if (ctx->ny > 1) { PFC_CUDA(ycols(ctx, 1, src, ctx->work), "pfc_fft_c2r y"); src = ctx->work; }
    if (ctx->fused_x && ctx->fused_y) PFC_CUDA(launch_xrows_c2r(ctx, src, out), "pfc_fft_c2r rows");
    else PFC_CUDA(launch_rows_c2r(ctx, src, out), "pfc_fft_c2r rows");
    ctx->launches += 1 + (ctx->ny > 1) + (ctx->nz > 1);
    return PFC_OK;
}

// ---- pointwise ------------------------------------------------------------------------
pfc_status pfc_update_eom(pfc_ctx* ctx, void* kpsi, const void* knl, const void* knoise, double namp, double dt,
                          double eps, double lx, double ly, double lz) {
    PFC_CHECK_CTX();
    if (!kpsi || !knl) return fail(ctx, PFC_ERR_INVALID, "pfc_update_eom: null buffer");
    PFC_CUDA(launch_update_eom(ctx, kpsi, knl, knoise, namp, dt, eps, lx, ly, lz, 0, 1.0), "pfc_update_eom");
    return PFC_OK;
}

pfc_status pfc_update_eom_with_fen(pfc_ctx* ctx, void* kpsi, const void* knl, void* knoise, double namp, double dt,
                                   double eps, double lx, double ly, double lz) {
    PFC_CHECK_CTX();
    if (!kpsi || !knl || !knoise) return fail(ctx, PFC_ERR_INVALID, "pfc_update_eom_with_fen: null buffer");
    PFC_CUDA(launch_update_eom(ctx, kpsi, knl, knoise, namp, dt, eps, lx, ly, lz, 1, 1.0), "pfc_update_eom_with_fen");
    return PFC_OK;
}

pfc_status pfc_psi3_split(pfc_ctx* ctx, void* arr, const void* pot, double mu, int norm) {
    PFC_CHECK_CTX();
    if (!arr) return fail(ctx, PFC_ERR_INVALID, "pfc_psi3_split: null buffer");
    PFC_CUDA(launch_psi3(ctx, arr, pot, mu, norm, 1.0), "pfc_psi3_split");
    return PFC_OK;
}

pfc_status pfc_norm(pfc_ctx* ctx, void* arr) {
    PFC_CHECK_CTX();
    if (!arr) return fail(ctx, PFC_ERR_INVALID, "pfc_norm: null buffer");
    PFC_CUDA(launch_norm(ctx, arr), "pfc_norm");
    return PFC_OK;
}

pfc_status pfc_calc_fen(pfc_ctx* ctx, const void* psi, void* lpsi, double hx, double hy, double hz, double* out) {
    PFC_CHECK_CTX();
    if (!psi || !lpsi || !out) return fail(ctx, PFC_ERR_INVALID, "pfc_calc_fen: null buffer");
    PFC_CUDA(launch_calc_fen(ctx, psi, lpsi, hx * hy * hz), "pfc_calc_fen");
    PFC_CUDA(cudaMemcpyAsync(out, ctx->red + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
             "pfc_calc_fen copy");
    PFC_CUDA(cudaStreamSynchronize(ctx->stream), "pfc_calc_fen sync");
    return PFC_OK;
}

pfc_status pfc_noise_fill_kspace(pfc_ctx* ctx, void* arr, uint64_t seed, uint64_t counter) {
    PFC_CHECK_CTX();
    if (!arr) return fail(ctx, PFC_ERR_INVALID, "pfc_noise_fill_kspace: null buffer");
    PFC_CUDA(launch_noise_kspace(ctx, arr, seed, counter), "pfc_noise_fill_kspace");
    return PFC_OK;
}

pfc_status pfc_noise_fill(pfc_ctx* ctx, void* arr, double sigma, uint64_t seed, uint64_t counter) {
    PFC_CHECK_CTX();
    if (!arr) return fail(ctx, PFC_ERR_INVALID, "pfc_noise_fill: null buffer");
    PFC_CUDA(launch_noise_real(ctx, arr, sigma, seed, counter), "pfc_noise_fill");
    return PFC_OK;
}

// ---- peaks and bond order ---------------------------------------------------------------
pfc_status pfc_findpeaks(pfc_ctx* ctx, const void* psi, double ths, void* out, int capacity, int* n_found) {
    PFC_CHECK_CTX();
    if (!psi || !n_found || capacity < 0 || (capacity > 0 && !out))
        return fail(ctx, PFC_ERR_INVALID, "pfc_findpeaks: bad arguments");
    if (ctx->nz == 1 && !(ctx->nx > 1 && ctx->ny > 1))
        return fail(ctx, PFC_ERR_INVALID, "pfc_findpeaks: input not a 2d array");
    if (ctx->async_pending)  // the scratch of a search still in flight on the copy stream
        PFC_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->peaks_done, 0), "pfc_findpeaks wait");
    PFC_CUDA(launch_findpeaks(ctx, psi, ths, out, capacity, ctx->stream), "pfc_findpeaks");
    int total = 0;
    PFC_CUDA(cudaMemcpyAsync(&total, ctx->peak_offsets + ctx->n_peak_blocks, sizeof(int), cudaMemcpyDeviceToHost,
                             ctx->stream), "pfc_findpeaks copy");
    PFC_CUDA(cudaStreamSynchronize(ctx->stream), "pfc_findpeaks sync");
    *n_found = total;
    if (total > capacity) return fail(ctx, PFC_ERR_CAPACITY, "pfc_findpeaks: more peaks than capacity");
    return PFC_OK;
}

namespace {
// the copy stream and its events (created by the first call that needs them)
cudaError_t ensure_copy_stream(pfc_ctx* ctx) {
    if (ctx->copy_stream) return cudaSuccess;
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
    for (cudaEvent_t& ev : ctx->host_ev)
        if (!e) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (!e) e = cudaEventCreateWithFlags(&ctx->peaks_done, cudaEventDisableTiming);
    return e;
}
}  // namespace

pfc_status pfc_findpeaks_async(pfc_ctx* ctx, const void* psi, double ths, void* host_out, int capacity,
                               int* host_count) {
    PFC_CHECK_CTX();
    if (!psi || !host_count || capacity < 0 || (capacity > 0 && !host_out))
        return fail(ctx, PFC_ERR_INVALID, "pfc_findpeaks_async: bad arguments");
    if (ctx->nz == 1 && !(ctx->nx > 1 && ctx->ny > 1))
        return fail(ctx, PFC_ERR_INVALID, "pfc_findpeaks_async: input not a 2d array");
    void* dout = nullptr;
    if (capacity > 0 && cudaHostGetDevicePointer(&dout, host_out, 0) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, PFC_ERR_INVALID, "pfc_findpeaks_async: host_out is not pinned host memory mapped to the device");
    }
    PFC_CUDA(ensure_copy_stream(ctx), "pfc_findpeaks_async stream");
    // the search starts when the work queued on the context's stream (which wrote psi) is done
    cudaEvent_t ready = ctx->host_ev[2 * pfc_ctx::kHostChunks];
    PFC_CUDA(cudaEventRecord(ready, ctx->stream), "pfc_findpeaks_async event");
    PFC_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ready, 0), "pfc_findpeaks_async wait");
    PFC_CUDA(launch_findpeaks(ctx, psi, ths, dout, capacity, ctx->copy_stream), "pfc_findpeaks_async");
    PFC_CUDA(cudaMemcpyAsync(host_count, ctx->peak_offsets + ctx->n_peak_blocks, sizeof(int), cudaMemcpyDeviceToHost,
                             ctx->copy_stream),
             "pfc_findpeaks_async count");
    PFC_CUDA(cudaEventRecord(ctx->peaks_done, ctx->copy_stream), "pfc_findpeaks_async event");
    ctx->async_count = host_count;
    ctx->async_capacity = capacity;
    ctx->async_pending = true;
    return PFC_OK;
}

pfc_status pfc_findpeaks_wait(pfc_ctx* ctx, int* n_found) {
    PFC_CHECK_CTX();
    if (!ctx->async_pending) return fail(ctx, PFC_ERR_INVALID, "pfc_findpeaks_wait: no search in flight");
    PFC_CUDA(cudaEventSynchronize(ctx->peaks_done), "pfc_findpeaks_wait");
    ctx->async_pending = false;
    const int total = *ctx->async_count;
    if (n_found) *n_found = total;
    if (total > ctx->async_capacity) return fail(ctx, PFC_ERR_CAPACITY, "pfc_findpeaks_async: more peaks than capacity");
    return PFC_OK;
}

pfc_status pfc_bond_order(pfc_ctx* ctx, const void* maxima, int n, double h0, double h1, double h2, double ths,
                          double boxsize, double rlim, double* out_rows, int row_capacity, int* n_rows) {
    PFC_CHECK_CTX();
    if (!n_rows || n < 0 || (n > 0 && !maxima) || row_capacity < 0 || (row_capacity > 0 && !out_rows) ||
        !(boxsize > 0.0))
        return fail(ctx, PFC_ERR_INVALID, "pfc_bond_order: bad arguments");
    int rows = 0;
    cudaError_t e = launch_bond_order(ctx, maxima, n, h0, h1, h2, ths, boxsize, rlim, out_rows, row_capacity, &rows);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(ctx, PFC_ERR_NOMEM, "pfc_bond_order: cannot grow the bond-order scratch");
    }
    PFC_CUDA(e, "pfc_bond_order");
    *n_rows = rows;
    if (rows > row_capacity) return fail(ctx, PFC_ERR_CAPACITY, "pfc_bond_order: more rows than capacity");
    return PFC_OK;
}

pfc_status pfc_bond_reserve(pfc_ctx* ctx, int max_atoms, long long max_pairs) {
    PFC_CHECK_CTX();
    if (max_atoms < 0 || max_pairs < 0) return fail(ctx, PFC_ERR_INVALID, "pfc_bond_reserve: negative size");
    if (max_pairs > INT32_MAX)
        return fail(ctx, PFC_ERR_UNSUPPORTED, "pfc_bond_reserve: more than 2^31 - 1 neighbour entries");
    cudaError_t e = bond_reserve(ctx, max_atoms, max_pairs);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(ctx, PFC_ERR_NOMEM, "pfc_bond_reserve: out of device memory");
    }
    PFC_CUDA(e, "pfc_bond_reserve");
    return PFC_OK;
}

// ---- stepper ------------------------------------------------------------------------------
pfc_status pfc_step(pfc_ctx* ctx, void* kpsi, int nsteps, const pfc_step_params* p) {
    return pfc_step_prop(ctx, kpsi, nsteps, p, PFC_PROP_CONSERVED, nullptr);
}

pfc_status pfc_step_prop(pfc_ctx* ctx, void* kpsi, int nsteps, const pfc_step_params* p, int propagator,
                         double* max_change) {
    PFC_CHECK_CTX();
    if (!kpsi || !p || nsteps < 0) return fail(ctx, PFC_ERR_INVALID, "pfc_step: bad arguments");
    if (propagator < PFC_PROP_CONSERVED || propagator > PFC_PROP_CONSERVED_HPFC)
        return fail(ctx, PFC_ERR_INVALID, "pfc_step_prop: unknown propagator");
    if (propagator == PFC_PROP_CONSERVED_HPFC && ctx->nz != 1)
        return fail(ctx, PFC_ERR_INVALID, "pfc_step_prop: the hpfc noise is for 2D fields only (eom.hpp:16-58)");
    const bool relax = propagator == PFC_PROP_RELAX || propagator == PFC_PROP_RELAX_EXP;
    if (relax && p->namp != 0.0)
        return fail(ctx, PFC_ERR_INVALID, "pfc_step_prop: the relaxation propagators take no noise (el.hpp)");
    if (max_change) *max_change = 0.0;
    if (nsteps == 0) return PFC_OK;
    ZPropArgs za = zargs(ctx, p);
    za.prop = propagator;
    // flag[0]: the watchdog and wait status; flag[2]: the last step's largest mode change
    PFC_CUDA(cudaMemsetAsync(ctx->flag, 0, 3 * sizeof(int), ctx->stream), "pfc_step flag");
    PFC_CUDA(step_entry(ctx, kpsi), "pfc_step entry");
    for (int t = 0; t < nsteps; ++t) {
        PFC_CUDA(step_xy(ctx, kpsi, p, t == nsteps - 1), "pfc_step xy");
        za.counter = p->counter + (uint64_t)t;
        za.final_step = (t == nsteps - 1);  // the last step writes psi^ itself
        za.maxc = relax && za.final_step ? reinterpret_cast<unsigned*>(ctx->flag + 2) : nullptr;
        PFC_CUDA(step_z(ctx, kpsi, za), "pfc_step z");
    }
    int flag[3] = {0, 0, 0};
    PFC_CUDA(cudaMemcpyAsync(flag, ctx->flag, sizeof(flag), cudaMemcpyDeviceToHost, ctx->stream), "pfc_step copy flag");
    PFC_CUDA(cudaStreamSynchronize(ctx->stream), "pfc_step sync");
    if (flag[0] & kFlagWaitTimeout) return fail(ctx, PFC_ERR_CUDA, "pfc_step: a device wait timed out");
    if (flag[0]) return fail(ctx, PFC_ERR_NONFINITE, "pfc_step: non-finite value in the state");
    if (max_change) {
        float m;
        std::memcpy(&m, &flag[2], sizeof(float));
        *max_change = (double)m;
    }
    return PFC_OK;
}

// ---- the step with the field in host memory ---------------------------------------------------
// The field comes in by ky chunks (nz rows of nky (nx/2+1) modes each, one strided copy per
// chunk on the copy stream) into the psi^ buffer, and the entry pass (psi^ -> z-tiled psi^
// and A) runs on each chunk as soon as it has arrived; the final psi^ goes back in one copy.  Only the
// schedule that carries psi^ z-tiled has a chunked entry pass; others copy, step and copy
// back in order.
pfc_status pfc_step_host(pfc_ctx* ctx, const void* host_in, void* host_out, void* kpsi, int nsteps,
                         const pfc_step_params* p) {
    PFC_CHECK_CTX();
    if (!host_in || !host_out || !kpsi || !p || nsteps < 0)
        return fail(ctx, PFC_ERR_INVALID, "pfc_step_host: bad arguments");
    const size_t S = ctx->state_bytes * ctx->batch;
    constexpr int G = pfc_ctx::kHostChunks;
    const bool chunked = ctx->tiled && ctx->z_carry && ctx->batch == 1 && nsteps >= 1 && ctx->ny % G == 0;
    if (!chunked) {
        PFC_CUDA(cudaMemcpyAsync(kpsi, host_in, S, cudaMemcpyHostToDevice, ctx->stream), "pfc_step_host copy in");
        pfc_status st = pfc_step(ctx, kpsi, nsteps, p);
        if (st != PFC_OK) return st;
        PFC_CUDA(cudaMemcpyAsync(host_out, kpsi, S, cudaMemcpyDeviceToHost, ctx->stream), "pfc_step_host copy out");
        PFC_CUDA(cudaStreamSynchronize(ctx->stream), "pfc_step_host sync");
        return PFC_OK;
    }
    PFC_CUDA(ensure_copy_stream(ctx), "pfc_step_host stream");
    cudaStream_t cs = ctx->copy_stream;
    cudaEvent_t* ev_in = ctx->host_ev;  // chunk g has arrived
    cudaEvent_t ev_start = ctx->host_ev[2 * G];
    const int cky = ctx->ny / G;
    const size_t pitch = (size_t)ctx->nxh * ctx->ny * sizeof(float2), width = (size_t)ctx->nxh * cky * sizeof(float2);
    ZPropArgs za = zargs(ctx, p);
    PFC_CUDA(cudaMemsetAsync(ctx->flag, 0, 3 * sizeof(int), ctx->stream), "pfc_step_host flag");
    // the copies start after the work already queued on the context's stream (work is free)
    PFC_CUDA(cudaEventRecord(ev_start, ctx->stream), "pfc_step_host event");
    PFC_CUDA(cudaStreamWaitEvent(cs, ev_start, 0), "pfc_step_host wait");
    for (int g = 0; g < G; ++g) {
        PFC_CUDA(cudaMemcpy2DAsync((char*)kpsi + g * width, pitch, (const char*)host_in + g * width, pitch, width,
                                   ctx->nz, cudaMemcpyHostToDevice, cs),
                 "pfc_step_host copy in");
        PFC_CUDA(cudaEventRecord(ev_in[g], cs), "pfc_step_host event");
    }
    for (int g = 0; g < G; ++g) {
        PFC_CUDA(cudaStreamWaitEvent(ctx->stream, ev_in[g], 0), "pfc_step_host wait");
        PFC_CUDA(traced(ctx, 0, g == 0 ? 2 : 1,
                        [&] {
                            cudaError_t e = g == 0 ? launch_k0_save(ctx, kpsi) : cudaSuccess;
                            if (!e)
                                e = launch_zfft(ctx, 1, kpsi, ctx->work, 1.0 / ctx->nz, kLayZ << 2, g * cky, cky,
                                                ctx->work2);
                            return e;
                        }),
                 "pfc_step_host entry");
    }
    for (int t = 0; t < nsteps; ++t) {
        const bool last = t == nsteps - 1;
        PFC_CUDA(step_xy(ctx, kpsi, p, last), "pfc_step_host xy");
        za.counter = p->counter + (uint64_t)t;
        za.final_step = last;
        PFC_CUDA(step_z(ctx, kpsi, za), "pfc_step_host z");
    }
    // the copy out in one piece: strided device-to-host copies by ky chunk measured slower than
    // one contiguous copy (10.1 against 9.6 ms for the 539 MB field), more than the last z
    // pass they would hide
    PFC_CUDA(cudaMemcpyAsync(host_out, kpsi, S, cudaMemcpyDeviceToHost, ctx->stream), "pfc_step_host copy out");
    int flag[3] = {0, 0, 0};
    PFC_CUDA(cudaMemcpyAsync(flag, ctx->flag, sizeof(flag), cudaMemcpyDeviceToHost, ctx->stream), "pfc_step_host flag");
    PFC_CUDA(cudaStreamSynchronize(ctx->stream), "pfc_step_host sync");
    if (flag[0] & kFlagWaitTimeout) return fail(ctx, PFC_ERR_CUDA, "pfc_step_host: a device wait timed out");
    if (flag[0]) return fail(ctx, PFC_ERR_NONFINITE, "pfc_step_host: non-finite value in the state");
    return PFC_OK;
}

// ---- slab-decomposed steps of fields spread over several processes --------------------------
pfc_status pfc_slab_zinv(pfc_ctx* ctx, const void* kpsi, void* A, int ky0) {
    PFC_CHECK_CTX();
    if (!kpsi || !A || kpsi == A || ky0 < 0) return fail(ctx, PFC_ERR_INVALID, "pfc_slab_zinv: bad arguments");
    if (ky0 == 0) PFC_CUDA(launch_k0_save(ctx, kpsi), "pfc_slab_zinv k0");
    if (ctx->nz > 1) {
        PFC_CUDA(zcols(ctx, 1, kpsi, A, 1.0 / ctx->nz), "pfc_slab_zinv");
    } else {
        PFC_CUDA(cudaMemcpyAsync(A, kpsi, ctx->state_bytes, cudaMemcpyDeviceToDevice, ctx->stream), "pfc_slab_zinv");
    }
    return PFC_OK;
}

pfc_status pfc_slab_xy(pfc_ctx* ctx, const void* A, void* B, double C, double mu) {
    PFC_CHECK_CTX();
    if (!A || !B || A == B) return fail(ctx, PFC_ERR_INVALID, "pfc_slab_xy: bad arguments");
    const double mul = 1.0 / ((double)ctx->nx * (double)ctx->ny);
    if (ctx->xy_mode == 2) {
        PFC_CUDA(launch_ypass(ctx, 1, A, B, 1.0, ctx->nz), "pfc_slab_xy y");
        PFC_CUDA(launch_xpass(ctx, B, nullptr, mul, C, mu, ctx->nz), "pfc_slab_xy x");
        PFC_CUDA(launch_ypass(ctx, -1, B, B, 1.0, ctx->nz), "pfc_slab_xy y");
    } else {
        if (ctx->ny > 1) PFC_CUDA(launch_cols(ctx, 1, 1, A, B, 1.0), "pfc_slab_xy y");
        else PFC_CUDA(cudaMemcpyAsync(B, A, ctx->state_bytes, cudaMemcpyDeviceToDevice, ctx->stream), "pfc_slab_xy");
        PFC_CUDA(launch_rows_nonlin(ctx, B, nullptr, mul, C, mu), "pfc_slab_xy x");
        if (ctx->ny > 1) PFC_CUDA(launch_cols(ctx, 1, -1, B, B, 1.0), "pfc_slab_xy y");
    }
    ctx->launches += 3;
    return PFC_OK;
}

pfc_status pfc_slab_zpass(pfc_ctx* ctx, void* A, const void* B, const pfc_step_params* p, int ky0, int ny_global,
                          int final_step) {
    PFC_CHECK_CTX();
    if (!A || !B || !p || ky0 < 0 || ny_global < ctx->ny || ky0 + ctx->ny > ny_global)
        return fail(ctx, PFC_ERR_INVALID, "pfc_slab_zpass: bad arguments");
    ZPropArgs za = zargs(ctx, p);
    // the noise amplitude of the whole field: sqrt(N) of its nx ny_global nz cells
    za.namp_eff = p->namp * std::sqrt((double)ctx->nx * (double)ny_global * (double)ctx->nz);
    za.ky0 = ky0;
    za.ny_global = ny_global;
    za.final_step = final_step != 0;
    PFC_CUDA(launch_zprop(ctx, A, B, za), "pfc_slab_zpass");
    ctx->launches += 1;
    if (!final_step) return PFC_OK;
    int flag = 0;
    PFC_CUDA(cudaMemcpyAsync(&flag, ctx->flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "pfc_slab_zpass");
    PFC_CUDA(cudaStreamSynchronize(ctx->stream), "pfc_slab_zpass sync");
    if (flag) return fail(ctx, PFC_ERR_NONFINITE, "pfc_slab_zpass: non-finite value in the state");
    return PFC_OK;
}

pfc_status pfc_free_energy(pfc_ctx* ctx, const void* kpsi, double eps, double lx, double ly, double lz, double hx,
                           double hy, double hz, double* out) {
    PFC_CHECK_CTX();
    if (!kpsi || !out) return fail(ctx, PFC_ERR_INVALID, "pfc_free_energy: bad arguments");
    const double N = (double)ctx->n_real;
    PFC_CUDA(launch_fen_spectral(ctx, kpsi, eps, lx, ly, lz), "pfc_free_energy spectral");
    PFC_CUDA(launch_reduce_final(ctx, 1, 1.0), "pfc_free_energy reduce");
    pfc_status s = pfc_fft_c2r(ctx, kpsi, ctx->work2);
    if (s != PFC_OK) return s;
    PFC_CUDA(launch_quartic_sum(ctx, ctx->work2, 1.0 / N), "pfc_free_energy quartic");
    PFC_CUDA(launch_reduce_final(ctx, 2, 1.0), "pfc_free_energy reduce");
    double h[2] = {0.0, 0.0};
    PFC_CUDA(cudaMemcpyAsync(h, ctx->red + kRedBlocks + 1, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
             "pfc_free_energy copy");
    PFC_CUDA(cudaStreamSynchronize(ctx->stream), "pfc_free_energy sync");
    *out = hx * hy * hz * (h[0] / (2.0 * N) + 0.25 * h[1]);
    return PFC_OK;
}

// ---- spectral low-pass post-processing ---------------------------------------------------------
pfc_status pfc_gaussian_init(pfc_ctx* ctx, void* kgauss, double lx, double ly, double lz, double hx, double hy,
                             double hz, double divs_per_sigma) {
    PFC_CHECK_CTX();
    if (!kgauss) return fail(ctx, PFC_ERR_INVALID, "pfc_gaussian_init: null buffer");
    PFC_CUDA(launch_gaussian_init(ctx, kgauss, lx, ly, lz, hx, hy, hz, divs_per_sigma), "pfc_gaussian_init");
    return PFC_OK;
}

pfc_status pfc_kmult_real(pfc_ctx* ctx, void* karr, const void* kgauss) {
    PFC_CHECK_CTX();
    if (!karr || !kgauss) return fail(ctx, PFC_ERR_INVALID, "pfc_kmult_real: null buffer");
    PFC_CUDA(launch_kmult(ctx, karr, kgauss, 0), "pfc_kmult_real");
    return PFC_OK;
}

pfc_status pfc_kmult_imag(pfc_ctx* ctx, void* karr, const void* kgauss) {
    PFC_CHECK_CTX();
    if (!karr || !kgauss) return fail(ctx, PFC_ERR_INVALID, "pfc_kmult_imag: null buffer");
    PFC_CUDA(launch_kmult(ctx, karr, kgauss, 1), "pfc_kmult_imag");
    return PFC_OK;
}

pfc_status pfc_square(pfc_ctx* ctx, void* arr) {
    PFC_CHECK_CTX();
    if (!arr) return fail(ctx, PFC_ERR_INVALID, "pfc_square: null buffer");
    PFC_CUDA(launch_norm_square(ctx, arr, 0), "pfc_square");
    return PFC_OK;
}

namespace {
bool is_2d(const pfc_ctx* c) { return c->nz == 1 && c->ny > 1 && c->nx > 1; }
pfc_status lowpass_dump(pfc_ctx* ctx, const void* spectrum, double lx, double ly, const char* path) {
    cudaError_t ce = cudaSuccess;
    const int r = write_lowpass_file(ctx, spectrum, lx, ly, path, &ce);
    if (r == 1) return fail(ctx, PFC_ERR_CUDA, std::string("LOWPASS dump: ") + cudaGetErrorString(ce));
    if (r == 2) return fail(ctx, PFC_ERR_INVALID, std::string("LOWPASS dump: cannot write ") + path);
    return PFC_OK;
}
}  // namespace

pfc_status pfc_write_lowpass_2d(pfc_ctx* ctx, void* spectrum, const void* kgauss, double lx, double ly,
                                const char* path) {
    PFC_CHECK_CTX();
    if (!spectrum || !kgauss || !path) return fail(ctx, PFC_ERR_INVALID, "pfc_write_lowpass_2d: null argument");
    if (!is_2d(ctx)) return fail(ctx, PFC_ERR_INVALID, "pfc_write_lowpass_2d: the grid is not 2D");
    PFC_CUDA(launch_kmult(ctx, spectrum, kgauss, 0), "pfc_write_lowpass_2d");
    return lowpass_dump(ctx, spectrum, lx, ly, path);
}

pfc_status pfc_amplitude_lowpass(pfc_ctx* ctx, void* spectrum, void* aux, const void* kgauss, double lx, double ly,
                                 const char* path) {
    PFC_CHECK_CTX();
    if (!spectrum || !aux || !kgauss) return fail(ctx, PFC_ERR_INVALID, "pfc_amplitude_lowpass: null buffer");
    if (!is_2d(ctx)) return fail(ctx, PFC_ERR_INVALID, "pfc_amplitude_lowpass: the grid is not 2D");
    PFC_CUDA(launch_kmult(ctx, spectrum, kgauss, 1), "pfc_amplitude_lowpass high-pass");
    pfc_status s = pfc_fft_c2r(ctx, spectrum, aux);
    if (s != PFC_OK) return s;
    PFC_CUDA(launch_norm_square(ctx, aux, 1), "pfc_amplitude_lowpass square");
    if ((s = pfc_fft_r2c(ctx, aux, spectrum)) != PFC_OK) return s;
    PFC_CUDA(launch_kmult(ctx, spectrum, kgauss, 0), "pfc_amplitude_lowpass low-pass");
    if (path && (s = lowpass_dump(ctx, spectrum, lx, ly, path)) != PFC_OK) return s;
    if ((s = pfc_fft_c2r(ctx, spectrum, aux)) != PFC_OK) return s;
    PFC_CUDA(launch_norm(ctx, aux), "pfc_amplitude_lowpass norm");
    return PFC_OK;
}

// ---- the reference's other propagators ------------------------------------------------------
pfc_status pfc_init_eom_op(pfc_ctx* ctx, void* kop, double dt, double eps, double lx, double ly, double lz) {
    PFC_CHECK_CTX();
    if (!kop) return fail(ctx, PFC_ERR_INVALID, "pfc_init_eom_op: null buffer");
    PFC_CUDA(launch_init_eom_op(ctx, kop, dt, eps, lx, ly, lz), "pfc_init_eom_op");
    return PFC_OK;
}

pfc_status pfc_update_eom_exp(pfc_ctx* ctx, const void* kop, void* kpsi, const void* knonlin, const void* knoise,
                              double namp, double eps, double lx, double ly, double lz) {
    PFC_CHECK_CTX();
    if (!kop || !kpsi || !knonlin) return fail(ctx, PFC_ERR_INVALID, "pfc_update_eom_exp: null buffer");
    PFC_CUDA(launch_update_eom_exp(ctx, kop, kpsi, knonlin, const_cast<void*>(knoise), namp, eps, lx, ly, lz, 0),
             "pfc_update_eom_exp");
    return PFC_OK;
}

pfc_status pfc_update_eom_exp_with_fen(pfc_ctx* ctx, const void* kop, void* kpsi, const void* knonlin, void* knoise,
                                       double namp, double eps, double lx, double ly, double lz) {
    PFC_CHECK_CTX();
    if (!kop || !kpsi || !knonlin || !knoise)
        return fail(ctx, PFC_ERR_INVALID, "pfc_update_eom_exp_with_fen: null buffer");
    PFC_CUDA(launch_update_eom_exp(ctx, kop, kpsi, knonlin, knoise, namp, eps, lx, ly, lz, 1),
             "pfc_update_eom_exp_with_fen");
    return PFC_OK;
}

pfc_status pfc_update_el(pfc_ctx* ctx, void* kpsi, const void* knonlin, double dt, double eps, double lx, double ly,
                         double lz, double* max_change) {
    PFC_CHECK_CTX();
    if (!kpsi || !knonlin || !max_change) return fail(ctx, PFC_ERR_INVALID, "pfc_update_el: null argument");
    PFC_CUDA(launch_update_el(ctx, nullptr, kpsi, knonlin, dt, eps, lx, ly, lz, max_change), "pfc_update_el");
    return PFC_OK;
}

pfc_status pfc_init_el_op(pfc_ctx* ctx, void* kop, double dt, double eps, double lx, double ly, double lz) {
    PFC_CHECK_CTX();
    if (!kop) return fail(ctx, PFC_ERR_INVALID, "pfc_init_el_op: null buffer");
    PFC_CUDA(launch_init_el_op(ctx, kop, dt, eps, lx, ly, lz), "pfc_init_el_op");
    return PFC_OK;
}

pfc_status pfc_update_el_exp(pfc_ctx* ctx, const void* kop, void* kpsi, const void* knonlin, double* max_change) {
    PFC_CHECK_CTX();
    if (!kop || !kpsi || !knonlin || !max_change)
        return fail(ctx, PFC_ERR_INVALID, "pfc_update_el_exp: null argument");
    PFC_CUDA(launch_update_el(ctx, kop, kpsi, knonlin, 0.0, 0.0, 1.0, 1.0, 1.0, max_change), "pfc_update_el_exp");
    return PFC_OK;
}

pfc_status pfc_update_eom_py(pfc_ctx* ctx, void* kpsi, const void* knonlin, const void* knoise, double namp,
                             double dt, double eps, double lx, double ly, double lz) {
    PFC_CHECK_CTX();
    if (!kpsi || !knonlin) return fail(ctx, PFC_ERR_INVALID, "pfc_update_eom_py: null buffer");
    PFC_CUDA(launch_update_eom_py(ctx, kpsi, knonlin, knoise, namp, dt, eps, lx, ly, lz), "pfc_update_eom_py");
    return PFC_OK;
}

pfc_status pfc_update_eom_hpfcnoise(pfc_ctx* ctx, void* kpsi, const void* knonlin, const void* knoise1,
                                    const void* knoise2, const void* knoise3, double namp, double dt, double eps,
                                    double lx, double ly, double lz) {
    PFC_CHECK_CTX();
    if (!kpsi || !knonlin || !knoise1 || !knoise2 || !knoise3)
        return fail(ctx, PFC_ERR_INVALID, "pfc_update_eom_hpfcnoise: null buffer");
    if (ctx->nz != 1) return fail(ctx, PFC_ERR_INVALID, "pfc_update_eom_hpfcnoise: 2D grids only (nz = 1)");
    PFC_CUDA(launch_update_eom_hpfcnoise(ctx, kpsi, knonlin, knoise1, knoise2, knoise3, namp, dt, eps, lx, ly, lz),
             "pfc_update_eom_hpfcnoise");
    return PFC_OK;
}

// ---- reverse mode ------------------------------------------------------------------------
size_t pfc_adjoint_workspace_bytes(const pfc_ctx* ctx) { return ctx ? 2 * ctx->state_bytes : 0; }

pfc_status pfc_sf_loss(pfc_ctx* ctx, const void* kpsi, const void* s_target, void* lam_out, double* loss) {
    PFC_CHECK_CTX();
    if (!kpsi || !s_target || !lam_out || !loss) return fail(ctx, PFC_ERR_INVALID, "pfc_sf_loss: null argument");
    // (4/N) r psi^ into work2, then its C2R (which runs in work) into lam_out
    PFC_CUDA(launch_sf_loss(ctx, kpsi, s_target, ctx->work2), "pfc_sf_loss");
    PFC_CUDA(cudaMemcpyAsync(loss, ctx->red + kRedBlocks + 3, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
             "pfc_sf_loss copy");
    PFC_CUDA(cudaStreamSynchronize(ctx->stream), "pfc_sf_loss sync");
    return pfc_fft_c2r(ctx, ctx->work2, lam_out);
}

pfc_status pfc_adjoint_step(pfc_ctx* ctx, const void* kpsi_n, const void* kpsi_np1, void* lam,
                            const pfc_step_params* p, void* workspace, double* deps) {
    PFC_CHECK_CTX();
    if (!kpsi_n || !kpsi_np1 || !lam || !p || !workspace)
        return fail(ctx, PFC_ERR_INVALID, "pfc_adjoint_step: null argument");
    // w1: lam^ then D^-1 lam^; w2 (work2): (dt k^2/D) lam^ then psi_n; w3: B.  The
    // transforms use work for their intermediates.
    void* w1 = workspace;
    void* w3 = (char*)workspace + ctx->state_bytes;
    void* w2 = ctx->work2;
    pfc_status s = pfc_fft_r2c(ctx, lam, w1);
    if (s != PFC_OK) return s;
    if (deps) {
        PFC_CUDA(launch_adj_eps(ctx, w1, kpsi_np1, p), "pfc_adjoint_step eps");
        double v = 0.0;
        PFC_CUDA(cudaMemcpyAsync(&v, ctx->red + kRedBlocks + 3, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
                 "pfc_adjoint_step copy");
        PFC_CUDA(cudaStreamSynchronize(ctx->stream), "pfc_adjoint_step sync");
        *deps += v;
    }
    PFC_CUDA(launch_adj_mul(ctx, w1, w2, p, 1), "pfc_adjoint_step K");
    if ((s = pfc_fft_c2r(ctx, w2, w3)) != PFC_OK) return s;
    PFC_CUDA(launch_adj_mul(ctx, w1, w1, p, 0), "pfc_adjoint_step M");
    if ((s = pfc_fft_c2r(ctx, w1, lam)) != PFC_OK) return s;
    if ((s = pfc_fft_c2r(ctx, kpsi_n, w2)) != PFC_OK) return s;
    PFC_CUDA(launch_adj_combine(ctx, lam, w2, w3, p->C), "pfc_adjoint_step combine");
    ctx->launches += 4;
    return PFC_OK;
}

pfc_status pfc_ensemble_create(int n, pfc_ctx* const* ctxs, void* const* kpsis, const pfc_step_params* params,
                                int steps_per_graph, pfc_ensemble** out) {
    if (!out || n < 1 || !ctxs || !kpsis || !params || steps_per_graph < 1) return PFC_ERR_INVALID;
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (!ctxs[i] || !kpsis[i]) return PFC_ERR_INVALID;
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == ctxs[i] || kpsis[j] == kpsis[i]) return PFC_ERR_INVALID;  // members run concurrently
    }
    pfc_ensemble* e = new (std::nothrow) pfc_ensemble();
    if (!e) return PFC_ERR_NOMEM;
    e->ctx.assign(ctxs, ctxs + n);
    e->kpsi.assign(kpsis, kpsis + n);
    e->p.assign(params, params + n);
    e->steps_per_graph = steps_per_graph;
    for (int i = 0; i < n; ++i) {
        bool placed = false;
        for (auto& k : e->cls) {
            const int j = k.members[0];
            if (same_class(e->ctx[j], e->p[j], e->ctx[i], e->p[i])) {
                k.members.push_back(i);
                placed = true;
                break;
            }
        }
        if (!placed) {
            e->cls.emplace_back();
            e->cls.back().members.push_back(i);
        }
    }
    cudaError_t ce = cudaSuccess;
    for (auto& k : e->cls) {
        if (ce) break;
        const int m = (int)k.members.size();
        const pfc_ctx* like = e->ctx[k.members[0]];
        ce = make_class_context(like, m, &k.cc);
        if (!ce) ce = cudaMalloc(&k.state, like->state_bytes * m);
        if (!ce) ce = cudaMalloc((void**)&k.margs, sizeof(MemberArgs) * m);
        if (!ce) ce = cudaMalloc((void**)&k.ctr, sizeof(unsigned long long) * m);
        if (!ce) {
            std::vector<MemberArgs> h(m);
            for (int q = 0; q < m; ++q) {
                const int i = k.members[q];
                const ZPropArgs za = zargs(e->ctx[i], &e->p[i]);
                h[q] = MemberArgs{za.eps, za.namp_eff, za.seed};
            }
            ce = cudaMemcpy(k.margs, h.data(), sizeof(MemberArgs) * m, cudaMemcpyHostToDevice);
        }
        if (!ce) ce = cudaStreamCreateWithFlags(&k.st, cudaStreamNonBlocking);
        if (!ce) ce = cudaEventCreateWithFlags(&k.join, cudaEventDisableTiming);
    }
    if (!ce) ce = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
    cudaStream_t cap = nullptr;
    if (!ce) ce = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    // One graph: a fork, steps_per_graph steps of every class on its own branch (one launch
    // per pass for all of the class's members), a join.
    if (!ce) ce = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (!ce) {
        cudaError_t ie = cudaEventRecord(e->fork, cap);
        for (auto& k : e->cls) {
            if (ie) break;
            pfc_ctx* c = k.cc;
            c->stream = k.st;
            ie = cudaStreamWaitEvent(k.st, e->fork, 0);
            const pfc_step_params& p0 = e->p[k.members[0]];
            ZPropArgs za = zargs(c, &p0);
            za.dev_counter = k.ctr;
            za.margs = k.margs;
            for (int s = 0; s < steps_per_graph && !ie; ++s) {
                ie = step_xy(c, k.state, &p0, false);
                if (!ie) ie = step_z(c, k.state, za);
                if (!ie) ie = launch_counter(k.st, k.ctr, 0, 0, (int)k.members.size());
            }
            if (!ie) ie = cudaEventRecord(k.join, k.st);
            if (!ie) ie = cudaStreamWaitEvent(cap, k.join, 0);
        }
        ce = cudaStreamEndCapture(cap, &e->graph);
        if (!ce) ce = ie;
    }
    if (!ce) ce = cudaGraphInstantiate(&e->exec, e->graph, 0);
    if (cap) cudaStreamDestroy(cap);
    if (ce) {
        cudaGetLastError();
        free_ensemble(e);
        return ce == cudaErrorMemoryAllocation ? PFC_ERR_NOMEM : PFC_ERR_CUDA;
    }
    *out = e;
    return PFC_OK;
}

pfc_status pfc_ensemble_run(pfc_ensemble* e, int nsteps, void* stream) {
    if (!e) return PFC_ERR_INVALID;
    if (nsteps < 0 || nsteps % e->steps_per_graph) {
        e->err = "pfc_ensemble_run: nsteps must be a multiple of steps_per_graph";
        return PFC_ERR_INVALID;
    }
    if (nsteps == 0) return PFC_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int n = (int)e->ctx.size();
    std::vector<cudaStream_t> saved(n);
    for (int i = 0; i < n; ++i) saved[i] = e->ctx[i]->stream;
    cudaError_t ce = cudaSuccess;
    // each member to its carried form (its own context), then into its class's slot: the
    // psi^ buffer, work2 (the carried field of the tiled and psi^-carrying schedules) and k0
    for (auto& k : e->cls) {
        if (ce) break;
        const size_t S = k.cc->state_bytes;
        ce = cudaMemsetAsync(k.cc->flag, 0, sizeof(int), st);
        for (int q = 0; q < (int)k.members.size() && !ce; ++q) {
            const int i = k.members[q];
            pfc_ctx* c = e->ctx[i];
            c->stream = st;
            ce = step_entry(c, e->kpsi[i]);
            // A: in the psi^ buffer, or in work for the tiled psi^-carrying schedule
            const bool awork = c->tiled && c->z_carry;
            if (!ce)
                ce = cudaMemcpyAsync((char*)(awork ? k.cc->work : k.state) + q * S, awork ? c->work : e->kpsi[i], S,
                                     cudaMemcpyDeviceToDevice, st);
            if (!ce) ce = cudaMemcpyAsync((char*)k.cc->work2 + q * S, c->work2, S, cudaMemcpyDeviceToDevice, st);
            if (!ce) ce = cudaMemcpyAsync(k.cc->k0 + q, c->k0, sizeof(double2), cudaMemcpyDeviceToDevice, st);
            if (!ce) ce = launch_counter(st, k.ctr + q, e->p[i].counter, 1);
        }
    }
    for (int r = 0; r < nsteps / e->steps_per_graph && !ce; ++r) ce = cudaGraphLaunch(e->exec, st);
    // back from the class slots, then each member to psi^
    for (auto& k : e->cls) {
        if (ce) break;
        const size_t S = k.cc->state_bytes;
        for (int q = 0; q < (int)k.members.size() && !ce; ++q) {
            const int i = k.members[q];
            pfc_ctx* c = e->ctx[i];
            const bool awork = c->tiled && c->z_carry;  // (psi^ is in work2 then: A is not needed)
            ce = awork ? cudaSuccess
                       : cudaMemcpyAsync(e->kpsi[i], (char*)k.state + q * S, S, cudaMemcpyDeviceToDevice, st);
            if (!ce) ce = cudaMemcpyAsync(c->work2, (char*)k.cc->work2 + q * S, S, cudaMemcpyDeviceToDevice, st);
            if (!ce) ce = step_exit(c, e->kpsi[i]);
        }
    }
    std::vector<int> flags(e->cls.size(), 0);
    for (size_t k = 0; k < e->cls.size() && !ce; ++k)
        ce = cudaMemcpyAsync(&flags[k], e->cls[k].cc->flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (!ce) ce = cudaStreamSynchronize(st);
    for (int i = 0; i < n; ++i) e->ctx[i]->stream = saved[i];
    if (ce) {
        e->err = std::string("pfc_ensemble_run: ") + cudaGetErrorString(ce);
        return PFC_ERR_CUDA;
    }
    for (int i = 0; i < n; ++i) e->p[i].counter += (uint64_t)nsteps;
    for (size_t k = 0; k < e->cls.size(); ++k)
        if (flags[k]) {
            e->err = "pfc_ensemble_run: non-finite value in member " + std::to_string(e->cls[k].members[0]) +
                     (e->cls[k].members.size() > 1 ? " or another member of its shape" : "");
            return PFC_ERR_NONFINITE;
        }
    return PFC_OK;
}

pfc_status pfc_ensemble_destroy(pfc_ensemble* e) {
    if (!e) return PFC_ERR_INVALID;
    free_ensemble(e);
    return PFC_OK;
}

const char* pfc_ensemble_last_error(const pfc_ensemble* e) { return e ? e->err.c_str() : "null ensemble"; }

pfc_status pfc_profile_enable(pfc_ctx* ctx, int on) {
    PFC_CHECK_CTX();
    if (on && ctx->ev_pool.empty()) {
        ctx->ev_pool.resize(4096);
        for (auto& e : ctx->ev_pool) PFC_CUDA(cudaEventCreate(&e), "pfc_profile_enable");
    }
    ctx->ev_pending.clear();
    ctx->ev_used = 0;
    ctx->launches = 0;
    for (int f = 0; f < PFC_PROFILE_FAMILIES; ++f) { ctx->prof_calls[f] = 0; ctx->prof_ms[f] = 0.0; }
    ctx->prof_on = on != 0;
    return PFC_OK;
}

pfc_status pfc_profile_read(pfc_ctx* ctx, pfc_profile* out) {
    PFC_CHECK_CTX();
    if (!out) return fail(ctx, PFC_ERR_INVALID, "pfc_profile_read: null output");
    PFC_CUDA(prof_resolve(ctx), "pfc_profile_read");
    out->launches = ctx->launches;
    out->xy_variant = 0;
    out->xy_mode = ctx->xy_mode;
    out->z_mode = ctx->z_carry ? (ctx->tiled ? 4 : (ctx->fused_z ? 2 : 5)) : (ctx->tiled ? 3 : (ctx->fused_z ? 1 : 0));
    out->z_variant = ctx->fused_z;
    out->y_variant = ctx->xy_mode == 2 ? ctx->fused_y : 0;
    for (int f = 0; f < PFC_PROFILE_FAMILIES; ++f) { out->calls[f] = ctx->prof_calls[f]; out->ms[f] = ctx->prof_ms[f]; }
    return PFC_OK;
}

}  // extern "C"
