// Internal building blocks of libpfc_b200: complex helpers, small-radix DFTs, the
// shared-memory Stockham line FFT used by the general-size kernels, the wavenumber
// of the reference, Philox4x32-10 and the noise draw.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

namespace pfc {

template <typename T> struct CxOf;
template <> struct CxOf<float> { using type = float2; };
template <> struct CxOf<double> { using type = double2; };
template <typename T> using cx = typename CxOf<T>::type;

template <typename T> __host__ __device__ __forceinline__ cx<T> mkc(T a, T b) { cx<T> r; r.x = a; r.y = b; return r; }
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
// DIR * i * a  (DIR = -1 forward transform, +1 inverse)
template <int DIR, typename C> __host__ __device__ __forceinline__ C rot(C a) {
    C r;
    if (DIR > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
    return r;
}

// ---------------------------------------------------------------------------------
// small DFTs, X[k] = sum_n x[n] exp(DIR 2 pi i n k / R), in place, natural order.
// Constants are the exact values of cos/sin at multiples of 2 pi / R.
// ---------------------------------------------------------------------------------
template <typename T, int DIR, int R> struct Dft;

template <typename T, int DIR> struct Dft<T, DIR, 2> {
    __device__ __forceinline__ static void run(cx<T>* v) {
        cx<T> a = v[0], b = v[1]; v[0] = a + b; v[1] = a - b;
    }
};
template <typename T, int DIR> struct Dft<T, DIR, 4> {
    __device__ __forceinline__ static void run(cx<T>* v) {
        cx<T> s02 = v[0] + v[2], d02 = v[0] - v[2], s13 = v[1] + v[3], d13 = rot<DIR>(v[1] - v[3]);
        v[0] = s02 + s13; v[2] = s02 - s13; v[1] = d02 + d13; v[3] = d02 - d13;
    }
};
template <typename T, int DIR> struct Dft<T, DIR, 8> {
    __device__ __forceinline__ static void run(cx<T>* v) {
        const T h = T(0.70710678118654752440);
        cx<T> e[4] = {v[0], v[2], v[4], v[6]};
        cx<T> o[4] = {v[1], v[3], v[5], v[7]};
        Dft<T, DIR, 4>::run(e);
        Dft<T, DIR, 4>::run(o);
        // W8^1 = h (1 + DIR i), W8^2 = DIR i, W8^3 = h (-1 + DIR i)
        cx<T> o1 = mkc<T>(h * (o[1].x - T(DIR) * o[1].y), h * (o[1].y + T(DIR) * o[1].x));
        cx<T> o2 = rot<DIR>(o[2]);
        cx<T> o3 = mkc<T>(h * (-o[3].x - T(DIR) * o[3].y), h * (-o[3].y + T(DIR) * o[3].x));
        v[0] = e[0] + o[0]; v[4] = e[0] - o[0];
        v[1] = e[1] + o1;   v[5] = e[1] - o1;
        v[2] = e[2] + o2;   v[6] = e[2] - o2;
        v[3] = e[3] + o3;   v[7] = e[3] - o3;
    }
};
template <typename T, int DIR> struct Dft<T, DIR, 3> {
    __device__ __forceinline__ static void run(cx<T>* v) {
        const T s3 = T(0.86602540378443864676);
        cx<T> t1 = v[1] + v[2];
        cx<T> t2 = v[0] - t1 * T(0.5);
        cx<T> t3 = rot<DIR>(v[1] - v[2]) * s3;
        v[0] = v[0] + t1; v[1] = t2 + t3; v[2] = t2 - t3;
    }
};
template <typename T, int DIR> struct Dft<T, DIR, 5> {
    __device__ __forceinline__ static void run(cx<T>* v) {
        const T c1 = T(0.30901699437494742410), c2 = T(-0.80901699437494742410);
        const T s1 = T(0.95105651629515357212), s2 = T(0.58778525229247312917);
        cx<T> a14 = v[1] + v[4], d14 = v[1] - v[4], a23 = v[2] + v[3], d23 = v[2] - v[3];
        cx<T> A1 = v[0] + a14 * c1 + a23 * c2;
        cx<T> A2 = v[0] + a14 * c2 + a23 * c1;
        cx<T> B1 = rot<DIR>(d14 * s1 + d23 * s2);
        cx<T> B2 = rot<DIR>(d14 * s2 - d23 * s1);
        v[0] = v[0] + a14 + a23;
        v[1] = A1 + B1; v[4] = A1 - B1; v[2] = A2 + B2; v[3] = A2 - B2;
    }
};

// ---------------------------------------------------------------------------------
// Stockham autosort FFT over lines held in shared memory (general 2^a 3^b 5^c).
// Stage s has radix R_s and span Ns = R_0 ... R_{s-1}: butterfly j reads
// x[j + r n/R], applies exp(DIR 2 pi i r (j mod Ns) / (Ns R)), runs the R-point DFT
// and writes to (j - j mod Ns) R + j mod Ns + r Ns.  Twiddles are precomputed on
// the host in FP64 (forward sign; the inverse uses their conjugates).
// ---------------------------------------------------------------------------------
constexpr int kMaxStages = 16;
constexpr int kMaxOddRadix = 31;  // largest prime radix of the general stage

// Division of a non-negative 31-bit n by a fixed d >= 1 as a multiply-high, an add and a
// shift: with l = ceil(log2 d) and mul = floor(2^32 (2^l - d) / d) + 1 (below 2^32),
// n / d = (umulhi(n, mul) + n) >> l for every n < 2^31 (the round-up method of Granlund and
// Montgomery, "Division by invariant integers using multiplication", PLDI 1994).
struct FastDiv {
    uint32_t mul;
    int shift;
};
__host__ __device__ inline FastDiv make_fastdiv(int d) {
    int l = 0;
    while ((1ll << l) < d) ++l;
    const unsigned long long m = ((1ull << 32) * (((1ull << l) - (unsigned long long)d))) / (unsigned long long)d + 1;
    return FastDiv{(uint32_t)m, l};
}
__device__ __forceinline__ int fdiv(int n, FastDiv f) {
    return (int)((__umulhi((uint32_t)n, f.mul) + (uint32_t)n) >> f.shift);
}

// Lines of the Stockham engine in shared memory: element k of a line sits at lpad(k) (one
// pad element after every 32), so that the strided writes of the early stages (R apart) and
// the reads of later ones spread over the banks; lines are line_stride(n) elements apart, an
// odd number, so that the lanes of a warp moving one element of each of consecutive lines
// hit distinct banks too.
__host__ __device__ __forceinline__ constexpr int lpad(int k) { return k + (k >> 5); }
__host__ __device__ constexpr int line_stride(int n) { return (n + (n >> 5) + 1) | 1; }

struct LinePlan {
    int n;
    int nst;
    int radix[kMaxStages];
    int ns[kMaxStages];
    int twoff[kMaxStages];
    int rtoff[kMaxStages];     // W_R^q, q < R, for radices without a hand-written DFT
    FastDiv by_n;              // division by n
    FastDiv by_m[kMaxStages];  // by n / R_s
    FastDiv by_ns[kMaxStages]; // by Ns
};

// Stage of a prime radix R (7 <= R <= kMaxOddRadix): direct R-point DFT with the
// roots of unity W_R^q from the plan's table.
template <typename T, int DIR>
__device__ __forceinline__ void stockham_bfly_gen(const cx<T>* __restrict__ sl, cx<T>* __restrict__ dl, int j,
                                                  int m, int Ns, int R, const cx<T>* __restrict__ tws,
                                                  const cx<T>* __restrict__ wr, FastDiv by_ns) {
    cx<T> v[kMaxOddRadix];
    const int jj = j - fdiv(j, by_ns) * Ns;
    for (int r = 0; r < R; ++r) {
        cx<T> a = sl[lpad(j + r * m)];
        if (Ns > 1 && r > 0) {
            cx<T> w = tws[jj * (R - 1) + r - 1];
            if (DIR > 0) w.y = -w.y;
            a = cmul(a, w);
        }
        v[r] = a;
    }
    const int od = (j - jj) * R + jj;
    for (int k = 0; k < R; ++k) {
        cx<T> acc = v[0];
        int q = 0;
        for (int r = 1; r < R; ++r) {
            q += k;
            if (q >= R) q -= R;
            cx<T> w = wr[q];
            if (DIR > 0) w.y = -w.y;
            const cx<T> p = cmul(v[r], w);
            acc.x += p.x;
            acc.y += p.y;
        }
        dl[lpad(od + k * Ns)] = acc;
    }
}

template <typename T, int DIR, int R>
__device__ __forceinline__ void stockham_bfly(const cx<T>* __restrict__ sl, cx<T>* __restrict__ dl,
                                              int j, int m, int Ns, const cx<T>* __restrict__ tws,
                                              FastDiv by_ns) {
    cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = sl[lpad(j + r * m)];
    const int jj = j - fdiv(j, by_ns) * Ns;
    if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
            cx<T> w = tws[jj * (R - 1) + r - 1];
            if (DIR > 0) w.y = -w.y;
            v[r] = cmul(v[r], w);
        }
    }
    Dft<T, DIR, R>::run(v);
    const int od = (j - jj) * R + jj;
#pragma unroll
    for (int r = 0; r < R; ++r) dl[lpad(od + r * Ns)] = v[r];
}

// FFT of nlines lines, line l at a[l*ld .. l*ld+n).  Ping-pongs between a and b and
// returns the buffer holding the result.  All threads of the block must call it.
template <typename T, int DIR>
__device__ cx<T>* stockham_lines(cx<T>* a, cx<T>* b, int nlines, int ld, const LinePlan& p,
                                 const cx<T>* __restrict__ tw) {
    cx<T>* src = a;
    cx<T>* dst = b;
    for (int s = 0; s < p.nst; ++s) {
        const int R = p.radix[s], Ns = p.ns[s], m = p.n / R;
        const FastDiv by_m = p.by_m[s], by_ns = p.by_ns[s];
        const cx<T>* tws = tw + p.twoff[s];
        const int total = nlines * m;
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
            const int line = fdiv(e, by_m), j = e - line * m;
            const cx<T>* sl = src + (size_t)line * ld;
            cx<T>* dl = dst + (size_t)line * ld;
            switch (R) {
                case 8: stockham_bfly<T, DIR, 8>(sl, dl, j, m, Ns, tws, by_ns); break;
                case 4: stockham_bfly<T, DIR, 4>(sl, dl, j, m, Ns, tws, by_ns); break;
                case 2: stockham_bfly<T, DIR, 2>(sl, dl, j, m, Ns, tws, by_ns); break;
                case 3: stockham_bfly<T, DIR, 3>(sl, dl, j, m, Ns, tws, by_ns); break;
                case 5: stockham_bfly<T, DIR, 5>(sl, dl, j, m, Ns, tws, by_ns); break;
                default: stockham_bfly_gen<T, DIR>(sl, dl, j, m, Ns, R, tws, tw + p.rtoff[s], by_ns); break;
            }
        }
        __syncthreads();
        cx<T>* t = src; src = dst; dst = t;
    }
    return src;
}

// ---------------------------------------------------------------------------------
// The reference's wavenumber, K(i, n, len) = (i < n/2+1 ? i : i-n) * 2pi / len
// (cuda/kernels/common.hpp:27-28), evaluated in the field's precision.
// ---------------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T kwave(int i, int n, T len) {
    return T(i < n / 2 + 1 ? i : i - n) * T(6.283185307179586232) / len;
}

// ---------------------------------------------------------------------------------
// The stepper's propagators: the reference's update kernels as the per-mode map
// psi^' = a psi^ + b N^ + g namp_eff xi^, with dopx = -k^2, dopy = k^4 and the split
// deps = 1 + C - eps (C = 1 is the reference's split: psi3_split.hpp subtracts psi):
//  kPropConserved     semi-implicit conserved (eom.hpp:60-72): D = 1 - dt (deps dopx + 2 dopy
//                     + dopx dopy); a = 1/D, b = dt dopx / D, g = dt |k| / D
//  kPropConservedExp  exponential time differencing (eom-exp.hpp:3-60): L = -dopx (deps +
//                     2 dopx + dopy), E = exp(-L dt), Q = (E - 1)/L (-dt where L = 0, as
//                     kernel_init_eom_op); a = E, b = -dopx Q, g = -|k| Q
//  kPropRelax         non-conserved relaxation (el.hpp:3-45): D = 1 + dt (deps + 2 dopx +
//                     dopy); a = 1/D, b = -dt / D; no noise
//  kPropRelaxExp      its exponential form (el-exp.hpp:3-60): L = deps + 2 dopx + dopy,
//                     E = exp(-L dt), Q = (E - 1)/L (-dt where L = 0); a = E, b = Q; no noise
//  kPropConservedPoly the conserved update with the polynomial correlation function
//                     (eom.hpp:143-180): D = 1 - dt dopx (deps - 1 - P(k^2)), P the model's
//                     degree-6 polynomial in k^2; a = 1/D, b = dt dopx / D, g = dt |k| / D
//  kPropConservedHpfc the conserved update with the anisotropic 2D noise of eom.hpp:16-58:
//                     D as kPropConserved; a = 1/D, b = dt dopx / D, g = dt / D multiplies
//                     (c1 kx^2 + c2 ky^2) xi1 + (c2 kx^2 + c1 ky^2) xi2 + 2 kx ky xi3 for
//                     |k| <= 1/4, three independent noise fields (hpfc_noise)
// The conserved propagators leave the k = 0 mode unchanged (the stepper restores it from
// FP64); the relaxations move it.
enum {
    kPropConserved = 0,
    kPropConservedExp = 1,
    kPropRelax = 2,
    kPropRelaxExp = 3,
    kPropConservedPoly = 4,
    kPropConservedHpfc = 5
};
template <int PROP> __host__ __device__ constexpr bool prop_conserved() {
    return PROP == kPropConserved || PROP == kPropConservedExp || PROP == kPropConservedPoly ||
           PROP == kPropConservedHpfc;
}

// the polynomial P(k^2) of eom.hpp:143-149 (the model's coefficients c12 .. c0, Horner)
template <typename T> __host__ __device__ __forceinline__ T py_poly(T k2) {
    T d = T(-0.293423255328944);
    d = d * k2 + T(4.678065276755401);
    d = d * k2 + T(-30.20985042718309);
    d = d * k2 + T(100.6942650417575);
    d = d * k2 + T(-181.1481995196213);
    d = d * k2 + T(164.4074088310241);
    d = d * k2 + T(-57.94636917114257);
    return d;
}

// Per-field parameters of a batch of fields stepped by one launch (grid z = field).
struct MemberArgs {
    double eps, namp_eff;
    uint64_t seed;
};

template <typename T> __device__ __forceinline__ T dev_exp(T x);
template <> __device__ __forceinline__ float dev_exp<float>(float x) { return expf(x); }
template <> __device__ __forceinline__ double dev_exp<double>(double x) { return exp(x); }

// a, b and g (see above) of the propagators other than kPropConserved, whose kernels keep
// their own arithmetic
template <int PROP, typename T>
__device__ __forceinline__ void prop_coef(T dopx, T dt, T deps, T& a, T& b, T& g) {
    const T dopy = dopx * dopx;
    if constexpr (PROP == kPropConservedExp) {
        const T lin = -dopx * (deps + T(2) * dopx + dopy);
        const T e = dev_exp<T>(-lin * dt);
        T q = (e - T(1)) / lin;
        if (q != q) q = -dt;
        a = e;
        b = -dopx * q;
        g = -sqrt(-dopx) * q;
    } else if constexpr (PROP == kPropRelax) {
        const T inv = T(1) / (T(1) + dt * (deps + T(2) * dopx + dopy));
        a = inv;
        b = -dt * inv;
        g = T(0);
    } else if constexpr (PROP == kPropConservedPoly) {
        // the polynomial and D in FP64: near the maximum of P (k^2 ~ 1.2 .. 4) its terms cancel
        // to a few parts in 10^3 of their size, which costs an FP32 evaluation ~1e-3 of D
        const double dd = 1.0 - (double)dt * (double)dopx * ((double)deps - 1.0 - py_poly<double>(-(double)dopx));
        const T inv = T(1.0 / dd);
        a = inv;
        b = dt * dopx * inv;
        g = dt * sqrt(-dopx) * inv;
    } else if constexpr (PROP == kPropConservedHpfc) {
        const T inv = T(1) / (T(1) - dt * (deps * dopx + T(2) * dopy + dopx * dopy));
        a = inv;
        b = dt * dopx * inv;
        g = dt * inv;
    } else {
        const T lin = deps + T(2) * dopx + dopy;
        const T e = dev_exp<T>(-lin * dt);
        T q = (e - T(1)) / lin;
        if (q != q) q = -dt;
        a = e;
        b = q;
        g = T(0);
    }
}

// The largest |psi^' - psi^| of a relaxation step: a warp's maximum, folded into *out
// (float bits of a non-negative value: their integer order is the value order).  Every
// lane of the warp calls it.
__device__ __forceinline__ void fold_max_change(float m, unsigned* out) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(out, __float_as_uint(m));
}

// ---------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with Weyl key bumps.
// ---------------------------------------------------------------------------------
struct U4 { uint32_t x, y, z, w; };
__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
        U4 n;
        n.x = (uint32_t)(p1 >> 32) ^ c.y ^ k0;
        n.y = (uint32_t)p1;
        n.z = (uint32_t)(p0 >> 32) ^ c.w ^ k1;
        n.w = (uint32_t)p0;
        c = n;
    }
    return c;
}

constexpr uint32_t kKspaceDomain = 0x0u;
constexpr uint32_t kRealDomain = 0x52454131u;
constexpr uint32_t kHpfcDomain = 0x48504600u;  // + 1, 2, 3: the three fields of the hpfc noise


// Two standard normals from counter (idx, counter) under key (seed, domain),
// Box-Muller on uniforms strictly inside (0, 1) that are exact in T.
template <typename T> __device__ __forceinline__ void philox_normal2(uint64_t idx, uint64_t seed, uint64_t counter,
                                                                     uint32_t domain, T& g1, T& g2);
template <> __device__ __forceinline__ void philox_normal2<float>(uint64_t idx, uint64_t seed, uint64_t counter,
                                                                  uint32_t domain, float& g1, float& g2) {
    U4 c{(uint32_t)idx, (uint32_t)(idx >> 32), (uint32_t)counter, (uint32_t)(counter >> 32)};
    U4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32) ^ domain);
    const float u1 = (float)((r.x >> 9) * 2u + 1u) * 5.9604644775390625e-08f;  // 2^-24
    const float u2 = (float)((r.y >> 9) * 2u + 1u) * 5.9604644775390625e-08f;
    const float rad = sqrtf(-2.0f * logf(u1));
    float s, co;
    sincospif(2.0f * u2, &s, &co);
    g1 = rad * co; g2 = rad * s;
}
template <> __device__ __forceinline__ void philox_normal2<double>(uint64_t idx, uint64_t seed, uint64_t counter,
                                                                   uint32_t domain, double& g1, double& g2) {
    U4 c{(uint32_t)idx, (uint32_t)(idx >> 32), (uint32_t)counter, (uint32_t)(counter >> 32)};
    U4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32) ^ domain);
    const uint64_t a = ((((uint64_t)r.x << 32) | r.y) >> 12) * 2u + 1u;
    const uint64_t b = ((((uint64_t)r.z << 32) | r.w) >> 12) * 2u + 1u;
    const double u1 = (double)a * 1.1102230246251565404e-16;  // 2^-53
    const double u2 = (double)b * 1.1102230246251565404e-16;
    const double rad = sqrt(-2.0 * log(u1));
    double s, co;
    sincospi(2.0 * u2, &s, &co);
    g1 = rad * co; g2 = rad * s;
}

// k-space noise of half-spectrum mode (i0, i1, i2): modes on the i0 = 0 and
// i0 = nx/2 planes are keyed by the canonical (lower linear index) member of their
// +-k pair and conjugated on the other member; self-conjugate modes are real.
template <typename T>
__device__ __forceinline__ cx<T> kspace_noise(int i0, int i1, int i2, int nx, int ny, int nz,
                                              uint64_t seed, uint64_t counter, uint32_t domain = kKspaceDomain) {
    const int nxh = nx / 2 + 1;
    const int64_t lin = ((int64_t)i2 * ny + i1) * nxh + i0;
    int64_t canon = lin;
    bool conj = false, selfc = false;
    if (i0 == 0 || ((nx & 1) == 0 && i0 == nx / 2)) {
        const int j1 = i1 == 0 ? 0 : ny - i1;
        const int j2 = i2 == 0 ? 0 : nz - i2;
        const int64_t part = ((int64_t)j2 * ny + j1) * nxh + i0;
        if (part < lin) { canon = part; conj = true; }
        selfc = (part == lin);
    }
    T g1, g2;
    philox_normal2<T>((uint64_t)canon, seed, counter, domain, g1, g2);
    const T s = T(0.70710678118654752440);
    if (selfc) return mkc<T>(g1, T(0));
    return mkc<T>(g1 * s, conj ? -g2 * s : g2 * s);
}

// The anisotropic 2D noise of eom.hpp:16-58 at wavenumbers (k0, k1), |k| = kabs: the three
// Hermitian-consistent fields (keyed like kspace_noise, domains kHpfcDomain + 1..3) weighted
// by c1 = kappa / (2 c2), c2 = sqrt(1 + kappa/2 + sqrt(1 + kappa)), kappa = 4/3, and cut off
// above |k| = 1/4.
template <typename T>
__device__ __forceinline__ cx<T> hpfc_noise(int i0, int i1, int nx, int ny, T k0, T k1, T kabs, uint64_t seed,
                                            uint64_t counter) {
    if (!(kabs <= T(0.25))) return mkc<T>(T(0), T(0));
    const T kappa = T(4) / T(3);
    const T c2 = sqrt(T(1) + kappa / T(2) + sqrt(T(1) + kappa));
    const T c1 = kappa / c2 / T(2);
    const cx<T> a = kspace_noise<T>(i0, i1, 0, nx, ny, 1, seed, counter, kHpfcDomain + 1u);
    const cx<T> b = kspace_noise<T>(i0, i1, 0, nx, ny, 1, seed, counter, kHpfcDomain + 2u);
    const cx<T> c = kspace_noise<T>(i0, i1, 0, nx, ny, 1, seed, counter, kHpfcDomain + 3u);
    const T fa = c1 * k0 * k0 + c2 * k1 * k1, fb = c2 * k0 * k0 + c1 * k1 * k1, fc = T(2) * k0 * k1;
    return mkc<T>(fa * a.x + fb * b.x + fc * c.x, fa * a.y + fb * b.y + fc * c.y);
}

}  // namespace pfc
