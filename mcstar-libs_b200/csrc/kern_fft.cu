// General-size FFT passes over the reference layout (x fastest; half spectrum of
// nx/2+1 complex per row).  Each CTA stages a tile of whole lines in shared memory
// and runs the Stockham engine of pfc_internal.cuh on them.  These kernels serve the
// reference-shaped primitives (R2C, C2R) and the stepper for every grid the fused
// plane kernels do not cover.
#include "pfc_ctx.h"

namespace pfc {
namespace {

// ---------------------------------------------------------------------------------
// complex FFT along a strided axis: element (line o, inner i, position k) at
// base + o*os + i + k*es.  A CTA owns `tile` consecutive inner lines of one o.
// ---------------------------------------------------------------------------------
template <typename T, int DIR>
__global__ void __launch_bounds__(256) k_cols(const cx<T>* __restrict__ in, cx<T>* out, int ni, int64_t es,
                                              int64_t os, LinePlan p, const cx<T>* __restrict__ tw, int tile,
                                              T scale, int64_t ms) {
    in += blockIdx.z * ms;  // fields of a batch (grid z)
    out += blockIdx.z * ms;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
    const int n = p.n;
    const int ld = line_stride(n);
    cx<T>* b1 = b0 + (size_t)tile * ld;
    const int tile_lg = __ffs(tile) - 1;  // tile: a power of two
    const int i0 = blockIdx.x * tile;
    const int nt = min(tile, ni - i0);
    const int64_t base = (int64_t)blockIdx.y * os + i0;
    for (int e = threadIdx.x; e < tile * n; e += blockDim.x) {
        const int i = e & (tile - 1), k = e >> tile_lg;
        if (i < nt) b0[i * ld + lpad(k)] = in[base + i + k * es];
    }
    __syncthreads();
    cx<T>* r = stockham_lines<T, DIR>(b0, b1, nt, ld, p, tw);
    for (int e = threadIdx.x; e < tile * n; e += blockDim.x) {
        const int i = e & (tile - 1), k = e >> tile_lg;
        if (i < nt) out[base + i + k * es] = r[i * ld + lpad(k)] * scale;
    }
}

// ---------------------------------------------------------------------------------
// rows: real <-> half spectrum along x.  Even nx packs x[2m], x[2m+1] into one
// complex and runs an nx/2-point FFT with the split/merge twiddles W_nx^k; odd nx
// runs the full nx-point complex FFT.
// ---------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ cx<T> r2c_post(cx<T> zk, cx<T> zm, cx<T> w) {
    // X[k] = 1/2 (Z[k] + conj Z[M-k]) - i/2 W^k (Z[k] - conj Z[M-k])
    const cx<T> s = mkc<T>(zk.x + zm.x, zk.y - zm.y);
    const cx<T> d = mkc<T>(zk.x - zm.x, zk.y + zm.y);
    const cx<T> wd = cmul(w, d);
    return mkc<T>(T(0.5) * (s.x + wd.y), T(0.5) * (s.y - wd.x));
}
template <typename T>
__device__ __forceinline__ cx<T> c2r_pre(cx<T> xk, cx<T> xm, cx<T> w) {
    // Z[k] = (X[k] + conj X[M-k]) + i W^-k (X[k] - conj X[M-k]); IFFT_M(Z) = nx * (x[2m] + i x[2m+1])
    const cx<T> e = mkc<T>(xk.x + xm.x, xk.y - xm.y);
    const cx<T> o = cmul(mkc<T>(xk.x - xm.x, xk.y + xm.y), cconj(w));
    return mkc<T>(e.x - o.y, e.y + o.x);
}

template <typename T>
__global__ void __launch_bounds__(256) k_rows_r2c(const T* __restrict__ in, cx<T>* __restrict__ out, int nrows,
                                                  int nx, LinePlan p, const cx<T>* __restrict__ tw,
                                                  const cx<T>* __restrict__ post, int rpc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
    const int L = p.n, ld = line_stride(L);
    cx<T>* b1 = b0 + (size_t)rpc * ld;
    const int row0 = blockIdx.x * rpc;
    const int nr = min(rpc, nrows - row0);
    const int nxh = nx / 2 + 1;
    const FastDiv by_nxh = make_fastdiv(nxh);
    const bool even = (nx & 1) == 0;
    for (int e = threadIdx.x; e < nr * L; e += blockDim.x) {
        const int r = fdiv(e, p.by_n), m = e - r * L;
        const T* row = in + (int64_t)(row0 + r) * nx;
        b0[r * ld + lpad(m)] = even ? reinterpret_cast<const cx<T>*>(row)[m] : mkc<T>(row[m], T(0));
    }
    __syncthreads();
    cx<T>* z = stockham_lines<T, -1>(b0, b1, nr, ld, p, tw);
    for (int e = threadIdx.x; e < nr * nxh; e += blockDim.x) {
        const int r = fdiv(e, by_nxh), k = e - r * nxh;
        const cx<T>* zr = z + (size_t)r * ld;
        cx<T> v;
        if (even) v = r2c_post<T>(zr[lpad(k % L)], zr[lpad((L - k) % L)], post[k]);
        else v = zr[lpad(k)];
        out[(int64_t)(row0 + r) * nxh + k] = v;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_rows_c2r(const cx<T>* __restrict__ in, T* __restrict__ out, int nrows,
                                                  int nx, LinePlan p, const cx<T>* __restrict__ tw,
                                                  const cx<T>* __restrict__ post, int rpc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
    const int L = p.n, ld = line_stride(L);
    cx<T>* b1 = b0 + (size_t)rpc * ld;
    const int row0 = blockIdx.x * rpc;
    const int nr = min(rpc, nrows - row0);
    const int nxh = nx / 2 + 1;
    const bool even = (nx & 1) == 0;
    for (int e = threadIdx.x; e < nr * L; e += blockDim.x) {
        const int r = fdiv(e, p.by_n), k = e - r * L;
        const cx<T>* row = in + (int64_t)(row0 + r) * nxh;
        cx<T> v;
        if (even) v = c2r_pre<T>(row[k], row[L - k], post[k]);
        else v = k < nxh ? row[k] : cconj(row[nx - k]);
        b0[r * ld + lpad(k)] = v;
    }
    __syncthreads();
    cx<T>* z = stockham_lines<T, 1>(b0, b1, nr, ld, p, tw);
    for (int e = threadIdx.x; e < nr * L; e += blockDim.x) {
        const int r = fdiv(e, p.by_n), m = e - r * L;
        T* row = out + (int64_t)(row0 + r) * nx;
        if (even) reinterpret_cast<cx<T>*>(row)[m] = z[r * ld + lpad(m)];
        else row[m] = z[r * ld + lpad(m)].x;
    }
}

// The stepper's x pass: C2R, the cubic nonlinearity (psi3_split.hpp:8-13 with the
// stabilisation constant C), R2C -- in place on rows of the mixed (kx, y, z) field.
template <typename T>
__device__ __forceinline__ T cubic(T v, T mul, T C, T mu) {
    const T t = v * mul;
    return t * t * t - C * t - mu;
}

template <typename T>
__global__ void __launch_bounds__(256) k_rows_nonlin(cx<T>* buf, const T* __restrict__ pot, int nrows, int nx,
                                                     LinePlan p, const cx<T>* __restrict__ tw,
                                                     const cx<T>* __restrict__ post, int rpc, T mul, T C, T mu,
                                                     int64_t ms) {
    buf += blockIdx.z * ms;  // fields of a batch (grid z; no potential then)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
    const int L = p.n, ld = line_stride(L);
    cx<T>* b1 = b0 + (size_t)rpc * ld;
    const int row0 = blockIdx.x * rpc;
    const int nr = min(rpc, nrows - row0);
    const int nxh = nx / 2 + 1;
    const FastDiv by_nxh = make_fastdiv(nxh);
    const bool even = (nx & 1) == 0;
    for (int e = threadIdx.x; e < nr * L; e += blockDim.x) {
        const int r = fdiv(e, p.by_n), k = e - r * L;
        const cx<T>* row = buf + (int64_t)(row0 + r) * nxh;
        cx<T> v;
        if (even) v = c2r_pre<T>(row[k], row[L - k], post[k]);
        else v = k < nxh ? row[k] : cconj(row[nx - k]);
        b0[r * ld + lpad(k)] = v;
    }
    __syncthreads();
    cx<T>* z = stockham_lines<T, 1>(b0, b1, nr, ld, p, tw);
    cx<T>* other = (z == b0) ? b1 : b0;
    for (int e = threadIdx.x; e < nr * L; e += blockDim.x) {
        const int r = fdiv(e, p.by_n), m = e - r * L;
        const int64_t rowi = (int64_t)(row0 + r) * nx;
        cx<T> v = z[r * ld + lpad(m)];
        if (even) {
            T a = cubic<T>(v.x, mul, C, mu), b = cubic<T>(v.y, mul, C, mu);
            if (pot) { a += pot[rowi + 2 * m]; b += pot[rowi + 2 * m + 1]; }
            v = mkc<T>(a, b);
        } else {
            T a = cubic<T>(v.x, mul, C, mu);
            if (pot) a += pot[rowi + m];
            v = mkc<T>(a, T(0));
        }
        z[r * ld + lpad(m)] = v;
    }
    __syncthreads();
    cx<T>* y = stockham_lines<T, -1>(z, other, nr, ld, p, tw);
    for (int e = threadIdx.x; e < nr * nxh; e += blockDim.x) {
        const int r = fdiv(e, by_nxh), k = e - r * nxh;
        const cx<T>* yr = y + (size_t)r * ld;
        cx<T> v;
        if (even) v = r2c_post<T>(yr[lpad(k % L)], yr[lpad((L - k) % L)], post[k]);
        else v = yr[lpad(k)];
        buf[(int64_t)(row0 + r) * nxh + k] = v;
    }
}

// ---------------------------------------------------------------------------------
// The stepper's z pass.  The state is carried as A = IFFT_z(psi^)/nz (k-space in x
// and y, real space in z) and B = FFT_xy of the nonlinear term on the same mixed
// grid.  Per tile of kx columns at one ky: FFT_z(A) = psi^, FFT_z(B) = N^, the
// semi-implicit update (eom.hpp:60-72 with stabilisation C), conserved noise, the
// FP64 k = 0 mode, then IFFT_z/nz back into A (or psi^ itself on the last step).
// ---------------------------------------------------------------------------------
template <typename T>
struct ZArgsT {
    T dt, eps, C, namp_eff, lx, ly, lz;
    uint64_t seed, counter;
    const unsigned long long* dev_counter;  // read instead of counter when set
    int use_noise, final_step;
    unsigned* maxc;                         // relaxations: max |psi^' - psi^| (float bits), or null
    const MemberArgs* margs;                // batched fields: per-field eps, noise amplitude, seed
    int ky0, nyg;                           // a ky-slab: the field's first row here and its row count
};

// The field of a batch this CTA steps (grid z): its noise counter and parameters.
template <typename T>
__device__ __forceinline__ void zmember(ZArgsT<T>& a) {
    if (a.dev_counter) a.dev_counter += blockIdx.z;
    if (a.margs) {
        const MemberArgs m = a.margs[blockIdx.z];
        a.eps = (T)m.eps;
        a.namp_eff = (T)m.namp_eff;
        a.seed = m.seed;
    }
}

// The update of mode (kx, kyg, kz) from psi^ and N^ (the propagator PROP, conserved noise,
// the FP64 k = 0 mode); k1 = the ky wavenumber, deps = 1 + C - eps.  The relaxations fold
// |psi^' - psi^| into mc.
template <typename T, int PROP>
__device__ __forceinline__ cx<T> zmode(cx<T> psi, cx<T> nl, int kx, int kyg, int kz, int nx, int nz, T k1, T deps,
                                       const ZArgsT<T>& a, const double2* __restrict__ k0, float& mc) {
    const T kk0 = kwave<T>(kx, nx, a.lx), kk2 = kwave<T>(kz, nz, a.lz);
    const T dopx = -kk0 * kk0 - k1 * k1 - kk2 * kk2;
    cx<T> v;
    if constexpr (PROP == kPropConserved) {
        const T dopy = dopx * dopx;
        const T denom = T(1) - a.dt * (deps * dopx + T(2) * dopy + dopx * dopy);
        if (kx == 0 && kyg == 0 && kz == 0) psi = mkc<T>((T)k0->x, (T)k0->y);
        const T f = a.dt * dopx;
        cx<T> num = mkc<T>(psi.x + f * nl.x, psi.y + f * nl.y);
        if (a.use_noise) {
            const T kabs = sqrt(-dopx);
            const uint64_t ctr = a.dev_counter ? *a.dev_counter : a.counter;
            const cx<T> xi = kspace_noise<T>(kx, kyg, kz, nx, a.nyg, nz, a.seed, ctr);
            const T g = a.dt * a.namp_eff * kabs;
            num.x += g * xi.x;
            num.y += g * xi.y;
        }
        v = mkc<T>(num.x / denom, num.y / denom);
    } else {
        if (prop_conserved<PROP>() && kx == 0 && kyg == 0 && kz == 0) psi = mkc<T>((T)k0->x, (T)k0->y);
        T ca, cb, cg;
        prop_coef<PROP, T>(dopx, a.dt, deps, ca, cb, cg);
        v = mkc<T>(ca * psi.x + cb * nl.x, ca * psi.y + cb * nl.y);
        if (prop_conserved<PROP>() && a.use_noise) {
            const uint64_t ctr = a.dev_counter ? *a.dev_counter : a.counter;
            const cx<T> xi = PROP == kPropConservedHpfc
                                 ? hpfc_noise<T>(kx, kyg, nx, a.nyg, kk0, k1, sqrt(-dopx), a.seed, ctr)
                                 : kspace_noise<T>(kx, kyg, kz, nx, a.nyg, nz, a.seed, ctr);
            v.x += a.namp_eff * cg * xi.x;
            v.y += a.namp_eff * cg * xi.y;
        }
        if (!prop_conserved<PROP>()) {
            const T dx = v.x - psi.x, dy = v.y - psi.y;
            mc = fmaxf(mc, (float)sqrt(dx * dx + dy * dy));
        }
    }
    return v;
}

// The z pass of a field with nz = 1 (2D): no z transform, so the update of every mode in
// place, one thread per mode of the columns [col0, col0 + ncols) of every ky row.
template <typename T, int PROP>
__global__ void __launch_bounds__(256) k_zflat(cx<T>* A, const cx<T>* __restrict__ B, int nx, int ny, ZArgsT<T> a,
                                               const double2* __restrict__ k0, int* flag, int col0, int ncols,
                                               int64_t ms) {
    A += blockIdx.z * ms;
    B += blockIdx.z * ms;
    k0 += blockIdx.z;
    zmember(a);
    const int nxh = nx / 2 + 1;
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = m < (int64_t)ncols * ny;
    float mc = 0.f;
    bool bad = false;
    if (valid) {
        const int ky = (int)(m / ncols), kx = col0 + (int)(m - (int64_t)ky * ncols);
        const int64_t off = (int64_t)ky * nxh + kx;
        const int kyg = ky + a.ky0;
        const T k1 = kwave<T>(kyg, a.nyg, a.ly);
        const cx<T> v = zmode<T, PROP>(A[off], B[off], kx, kyg, 0, nx, 1, k1, T(1) + a.C - a.eps, a, k0, mc);
        bad = !isfinite(v.x) || !isfinite(v.y);
        A[off] = v;
    }
    if (!prop_conserved<PROP>() && a.maxc) fold_max_change(mc, a.maxc);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// The z pass of the general-length stepper over the reference layout, a tile of z columns
// per CTA.  CARRY false: A = IFFT_z(psi^)/nz is carried; psi^ = FFT_z(A) and N^ = FFT_z(B),
// the update, A' = IFFT_z(psi^')/nz over A (three transforms).  CARRY true: psi^ itself is
// carried in A; N^ = FFT_z(B), the update writes psi^' over psi^, and A' = IFFT_z(psi^')/nz
// goes to anext (two transforms; none after the update on the final step).
template <typename T, int PROP, bool CARRY>
__global__ void __launch_bounds__(256) k_zprop(cx<T>* A, const cx<T>* __restrict__ B, int nx, int ny, int nz,
                                               LinePlan p, const cx<T>* __restrict__ tw, int tile, ZArgsT<T> a,
                                               const double2* __restrict__ k0, int* flag, int col0, int col_end,
                                               int64_t ms, cx<T>* anext) {
    // fields of a batch (grid z): their own state, k0, noise counter and parameters
    A += blockIdx.z * ms;
    B += blockIdx.z * ms;
    if (CARRY && anext) anext += blockIdx.z * ms;
    k0 += blockIdx.z;
    zmember(a);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int bad;
    cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
    const int n = nz;
    const int ld = line_stride(n);
    cx<T>* b1 = b0 + (size_t)2 * tile * ld;
    const int tile_lg = __ffs(tile) - 1;  // tile: a power of two
    const int nxh = nx / 2 + 1;
    const int i0 = col0 + blockIdx.x * tile;
    const int ky = blockIdx.y;
    const int nt = min(tile, col_end - i0);
    if (threadIdx.x == 0) bad = 0;
    for (int e = threadIdx.x; e < tile * n; e += blockDim.x) {
        const int i = e & (tile - 1), k = e >> tile_lg;
        if (i < nt) {
            const int64_t off = ((int64_t)k * ny + ky) * nxh + i0 + i;
            b0[i * ld + lpad(k)] = A[off];
            b0[(tile + i) * ld + lpad(k)] = B[off];
        }
    }
    __syncthreads();
    // CARRY: only the B lines are transformed (lines tile.. of both buffers); psi^ stays in b0
    cx<T>* rb = stockham_lines<T, -1>(CARRY ? b0 + (size_t)tile * ld : b0, CARRY ? b1 + (size_t)tile * ld : b1,
                                      CARRY ? tile : 2 * tile, ld, p, tw);
    cx<T>* r = CARRY ? b0 : rb;
    cx<T>* nl = CARRY ? rb : rb + (size_t)tile * ld;
    cx<T>* other = (r == b0) ? b1 : b0;
    // a ky-slab of a larger field: wavenumbers, the k = 0 mode and the noise keys of the field
    const int kyg = ky + a.ky0;
    const T k1 = kwave<T>(kyg, a.nyg, a.ly);
    const T deps = T(1) + a.C - a.eps;
    float mc = 0.f;
    for (int e = threadIdx.x; e < nt * n; e += blockDim.x) {
        const int i = fdiv(e, p.by_n), kz = e - i * n;
        const int kx = i0 + i;
        const cx<T> v =
            zmode<T, PROP>(r[i * ld + lpad(kz)], nl[i * ld + lpad(kz)], kx, kyg, kz, nx, nz, k1, deps, a, k0, mc);
        if (!isfinite(v.x) || !isfinite(v.y)) bad = 1;
        r[i * ld + lpad(kz)] = v;
    }
    if (!prop_conserved<PROP>() && a.maxc) fold_max_change(mc, a.maxc);
    __syncthreads();
    if (threadIdx.x == 0 && bad) atomicOr(flag, 1);
    if (CARRY) {
        // psi^' over psi^; A' = IFFT_z(psi^')/nz into anext unless this is the last step
        for (int e = threadIdx.x; e < tile * n; e += blockDim.x) {
            const int i = e & (tile - 1), k = e >> tile_lg;
            if (i < nt) A[((int64_t)k * ny + ky) * nxh + i0 + i] = r[i * ld + lpad(k)];
        }
        if (a.final_step || !anext) return;
    }
    cx<T>* outb = r;
    T scale = T(1);
    if (!a.final_step) {
        // (CARRY: the b1 lines below tile held nothing)
        outb = stockham_lines<T, 1>(r, other, nt, ld, p, tw);
        scale = T(1) / T(nz);
    }
    cx<T>* dst = CARRY ? anext : A;
    for (int e = threadIdx.x; e < tile * n; e += blockDim.x) {
        const int i = e & (tile - 1), k = e >> tile_lg;
        if (i < nt) dst[((int64_t)k * ny + ky) * nxh + i0 + i] = outb[i * ld + lpad(k)] * scale;
    }
}

// f(std::integral_constant<int, PROP>) for a run-time propagator
template <class F>
cudaError_t by_zprop(int prop, F&& f) {
    switch (prop) {
        case kPropConservedExp: return f(std::integral_constant<int, kPropConservedExp>{});
        case kPropRelax: return f(std::integral_constant<int, kPropRelax>{});
        case kPropRelaxExp: return f(std::integral_constant<int, kPropRelaxExp>{});
        case kPropConservedPoly: return f(std::integral_constant<int, kPropConservedPoly>{});
        case kPropConservedHpfc: return f(std::integral_constant<int, kPropConservedHpfc>{});
        default: return f(std::integral_constant<int, kPropConserved>{});
    }
}

template <typename T>
cudaError_t set_attrs_T(const pfc_ctx* c) {
    const int m = (int)kMaxDynSmem;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_cols<T, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, m))) return e;
    if ((e = cudaFuncSetAttribute(k_cols<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, m))) return e;
    if ((e = cudaFuncSetAttribute(k_rows_r2c<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, m))) return e;
    if ((e = cudaFuncSetAttribute(k_rows_c2r<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, m))) return e;
    if ((e = cudaFuncSetAttribute(k_rows_nonlin<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, m))) return e;
    for (int prop = 0; prop <= kPropConservedHpfc && !e; ++prop)
        e = by_zprop(prop, [&](auto P) {
            cudaError_t r = cudaFuncSetAttribute(k_zprop<T, P.value, false>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, m);
            if (!r) r = cudaFuncSetAttribute(k_zprop<T, P.value, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, m);
            return r;
        });
    if (e) return e;
    (void)c;
    return cudaSuccess;
}

template <typename T>
cudaError_t cols_T(const pfc_ctx* c, int axis, int dir, const void* in, void* out, double scale) {
    const AxisPlan& ap = axis == 1 ? c->py : c->pz;
    const int n = ap.plan.n;
    if (n == 1 && in == out && scale == 1.0) return cudaSuccess;
    int64_t es, os;
    int no;
    if (axis == 1) { es = c->nxh; os = (int64_t)c->ny * c->nxh; no = c->nz; }
    else { es = (int64_t)c->ny * c->nxh; os = c->nxh; no = c->ny; }
    dim3 grid((c->nxh + ap.tile - 1) / ap.tile, no, c->batch);
    const cx<T>* tw = reinterpret_cast<const cx<T>*>(c->tw);
    if (dir < 0)
        k_cols<T, -1><<<grid, 256, ap.smem, c->stream>>>((const cx<T>*)in, (cx<T>*)out, c->nxh, es, os, ap.plan, tw,
                                                           ap.tile, (T)scale, c->mstride);
    else
        k_cols<T, 1><<<grid, 256, ap.smem, c->stream>>>((const cx<T>*)in, (cx<T>*)out, c->nxh, es, os, ap.plan, tw,
                                                          ap.tile, (T)scale, c->mstride);
    return cudaGetLastError();
}

}  // namespace

cudaError_t set_fft_attributes(const pfc_ctx* c) {
    return c->dtype == PFC_F64 ? set_attrs_T<double>(c) : set_attrs_T<float>(c);
}

cudaError_t launch_cols(const pfc_ctx* c, int axis, int dir, const void* in, void* out, double scale) {
    return c->dtype == PFC_F64 ? cols_T<double>(c, axis, dir, in, out, scale)
                               : cols_T<float>(c, axis, dir, in, out, scale);
}

cudaError_t launch_rows_r2c(const pfc_ctx* c, const void* in, void* out) {
    const int nrows = c->ny * c->nz;
    dim3 grid((nrows + c->px.tile - 1) / c->px.tile);
    if (c->dtype == PFC_F64) {
        const cx<double>* tw = (const cx<double>*)c->tw;
        k_rows_r2c<double><<<grid, 256, c->px.smem, c->stream>>>((const double*)in, (cx<double>*)out, nrows, c->nx,
                                                                  c->px.plan, tw, tw + c->post_off, c->px.tile);
    } else {
        const cx<float>* tw = (const cx<float>*)c->tw;
        k_rows_r2c<float><<<grid, 256, c->px.smem, c->stream>>>((const float*)in, (cx<float>*)out, nrows, c->nx,
                                                                 c->px.plan, tw, tw + c->post_off, c->px.tile);
    }
    return cudaGetLastError();
}

cudaError_t launch_rows_c2r(const pfc_ctx* c, const void* in, void* out) {
    const int nrows = c->ny * c->nz;
    dim3 grid((nrows + c->px.tile - 1) / c->px.tile);
    if (c->dtype == PFC_F64) {
        const cx<double>* tw = (const cx<double>*)c->tw;
        k_rows_c2r<double><<<grid, 256, c->px.smem, c->stream>>>((const cx<double>*)in, (double*)out, nrows, c->nx,
                                                                  c->px.plan, tw, tw + c->post_off, c->px.tile);
    } else {
        const cx<float>* tw = (const cx<float>*)c->tw;
        k_rows_c2r<float><<<grid, 256, c->px.smem, c->stream>>>((const cx<float>*)in, (float*)out, nrows, c->nx,
                                                                 c->px.plan, tw, tw + c->post_off, c->px.tile);
    }
    return cudaGetLastError();
}

cudaError_t launch_rows_nonlin(const pfc_ctx* c, void* buf, const void* pot, double mul, double C, double mu) {
    const int nrows = c->ny * c->nz;
    dim3 grid((nrows + c->px.tile - 1) / c->px.tile, 1, c->batch);
    if (pot && c->batch > 1) return cudaErrorNotSupported;
    if (c->dtype == PFC_F64) {
        const cx<double>* tw = (const cx<double>*)c->tw;
        k_rows_nonlin<double><<<grid, 256, c->px.smem, c->stream>>>((cx<double>*)buf, (const double*)pot, nrows,
                                                                     c->nx, c->px.plan, tw, tw + c->post_off,
                                                                     c->px.tile, mul, C, mu, c->mstride);
    } else {
        const cx<float>* tw = (const cx<float>*)c->tw;
        k_rows_nonlin<float><<<grid, 256, c->px.smem, c->stream>>>((cx<float>*)buf, (const float*)pot, nrows, c->nx,
                                                                    c->px.plan, tw, tw + c->post_off, c->px.tile,
                                                                    (float)mul, (float)C, (float)mu, c->mstride);
    }
    return cudaGetLastError();
}

template <typename T, int PROP>
void zprop_T(const pfc_ctx* c, void* A, const void* B, const ZPropArgs& a, int col0, int ncols, void* anext,
             bool carry) {
    const int tile = c->pzprop.tile;
    dim3 grid((ncols + tile - 1) / tile, c->ny, c->batch);
    ZArgsT<T> t{(T)a.dt,      (T)a.eps,    (T)a.C,      (T)a.namp_eff,
                (T)a.lx,      (T)a.ly,     (T)a.lz,     a.seed,
                a.counter,    a.dev_counter, a.use_noise, a.final_step,
                a.maxc,       a.margs,     a.ky0,       a.ny_global > 0 ? a.ny_global : c->ny};
    if (c->nz == 1) {
        const int64_t modes = (int64_t)ncols * c->ny;
        k_zflat<T, PROP><<<dim3((unsigned)((modes + 255) / 256), 1, c->batch), 256, 0, c->stream>>>(
            (cx<T>*)A, (const cx<T>*)B, c->nx, c->ny, t, c->k0, c->flag, col0, ncols, c->mstride);
        return;
    }
    if (carry)
        k_zprop<T, PROP, true><<<grid, 256, c->pzprop.smem, c->stream>>>(
            (cx<T>*)A, (const cx<T>*)B, c->nx, c->ny, c->nz, c->pz.plan, (const cx<T>*)c->tw, tile, t, c->k0, c->flag,
            col0, col0 + ncols, c->mstride, (cx<T>*)anext);
    else
        k_zprop<T, PROP, false><<<grid, 256, c->pzprop.smem, c->stream>>>(
            (cx<T>*)A, (const cx<T>*)B, c->nx, c->ny, c->nz, c->pz.plan, (const cx<T>*)c->tw, tile, t, c->k0, c->flag,
            col0, col0 + ncols, c->mstride, nullptr);
}

cudaError_t launch_zprop_cols(const pfc_ctx* c, void* A, const void* B, const ZPropArgs& a, int col0, int ncols,
                              void* anext, bool carry) {
    if (carry && c->nz == 1) return cudaErrorNotSupported;
    by_zprop(a.prop, [&](auto P) {
        if (c->dtype == PFC_F64) zprop_T<double, P.value>(c, A, B, a, col0, ncols, anext, carry);
        else zprop_T<float, P.value>(c, A, B, a, col0, ncols, anext, carry);
        return cudaSuccess;
    });
    return cudaGetLastError();
}

cudaError_t launch_zprop(const pfc_ctx* c, void* A, const void* B, const ZPropArgs& a) {
    return launch_zprop_cols(c, A, B, a, 0, c->nxh);
}

cudaError_t launch_zprop_carry(const pfc_ctx* c, void* kpsi, const void* B, void* anext, const ZPropArgs& a) {
    return launch_zprop_cols(c, kpsi, B, a, 0, c->nxh, anext, true);
}

}  // namespace pfc
