// Steinhardt bond-order analysis of peak lists on the GPU, restating
// bond_order_analysis (bond-order-analysis/bond-order.cpp:289-349) in FP64:
//   keep atoms with field > ths; neighbours within rlim under the reference's
//   get_diff minimum image (bond-order.cpp:53-64); q_lm = <Y_lm> over neighbours for
//   l = 4, 6, 8; q_l, w_4 (and w_6, which the reference lacks), the neighbour-averaged
//   q-bar_l (self included), the reference's w4b (which averages only the last
//   neighbour, bond-order.cpp:205-219) and the solid-bond count xi (q6 dot > 0.7).
// The neighbour search bins atoms into cells of side >= rlim; each atom's list is
// sorted by index so the sums run in the reference's order.  Y_lm come from the
// normalised associated-Legendre upward recurrences with e^{i m phi} built by complex
// powers of (dx + i dy)/rho; the reference's pole band (prefF, bond-order.cpp:123-133:
// Y_lm = 0 for m > 0 when |1 - cos theta| < 1e-3 and for m < 0 when |1 + cos theta| <
// 1e-3) is kept.  Wigner 3j symbols come from the Racah formula, evaluated on the host.
#include <algorithm>
#include <cmath>
#include <vector>
#include "pfc_ctx.h"

namespace pfc {
namespace {

constexpr int kNQ = 9 + 13 + 17;         // q_lm, l = 4, 6, 8, m = -l..l
constexpr int kW4 = 61, kW6 = 127;       // (l l l; m1 m2 m3) with m1 + m2 + m3 = 0
__constant__ double c_nlm[3][9];         // normalisation of P_l^m, l = 4, 6, 8, m = 0..l
__constant__ double c_w4[kW4];
__constant__ int c_w4m[kW4][2];
__constant__ double c_w6[kW6];
__constant__ int c_w6m[kW6][2];
__constant__ int c_tables_ready;

struct BondScratch {
    double* pos;      // 3 * P
    int* keep_cnt;    // blocks
    int* keep_off;    // blocks + 1
    int* nb;          // P: neighbours of each atom
    int* nb_off;      // P + 1: exclusive scan of nb, the start of each atom's list in the pair buffer
    int* maxj;        // P
    double2* q;       // P * kNQ
    int* row_cnt;     // blocks
    int* row_off;     // blocks + 1
    int* cell_cnt;    // cells
    int* cell_off;    // cells + 1
    int* cell_fill;   // cells
    int* cell_atoms;  // P
    int* flags;       // [1] position outside the box, [2] kept count
};
constexpr int kMaxCellsDim = 64;
constexpr int kBlk = 256;

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

// The per-atom scratch of P atoms (the neighbour lists live in a separate pair buffer,
// sized by the neighbour count the search finds).
size_t scratch_layout(int P, BondScratch* s, char* base) {
    const size_t blocks = (size_t)(P + kBlk - 1) / kBlk + 1;
    const size_t cells = (size_t)kMaxCellsDim * kMaxCellsDim * kMaxCellsDim;
    size_t off = 0;
    auto take = [&](size_t bytes) { char* p = base ? base + off : nullptr; off += align_up(bytes); return p; };
    BondScratch t;
    t.pos = (double*)take(sizeof(double) * 3 * P);
    t.keep_cnt = (int*)take(sizeof(int) * blocks);
    t.keep_off = (int*)take(sizeof(int) * (blocks + 1));
    t.nb = (int*)take(sizeof(int) * P);
    t.nb_off = (int*)take(sizeof(int) * ((size_t)P + 1));
    t.maxj = (int*)take(sizeof(int) * P);
    t.q = (double2*)take(sizeof(double2) * (size_t)P * kNQ);
    t.row_cnt = (int*)take(sizeof(int) * blocks);
    t.row_off = (int*)take(sizeof(int) * (blocks + 1));
    t.cell_cnt = (int*)take(sizeof(int) * cells);
    t.cell_off = (int*)take(sizeof(int) * (cells + 1));
    t.cell_fill = (int*)take(sizeof(int) * cells);
    t.cell_atoms = (int*)take(sizeof(int) * P);
    t.flags = (int*)take(sizeof(int) * 8);
    if (s) *s = t;
    return off;
}

template <typename T> struct MaxRecB;
template <> struct MaxRecB<float> { float i0, i1, i2; float field; };
template <> struct MaxRecB<double> { double i0, i1, i2; float field; };

// ---- compaction helpers -------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_scan_b(const int* __restrict__ counts, int nb, int* __restrict__ offsets) {
    __shared__ int part[1024];
    const int chunk = (nb + 1023) / 1024;
    const int b = threadIdx.x * chunk;
    const int e = min(nb, b + chunk);
    int s = 0;
    for (int i = b; i < e; ++i) s += counts[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int run = part[threadIdx.x] - s;
    for (int i = b; i < e; ++i) { offsets[i] = run; run += counts[i]; }
    if (threadIdx.x == 1023) offsets[nb] = part[1023];
}

__device__ __forceinline__ int block_rank(bool f, int* wsum) {
    const unsigned m = __ballot_sync(0xffffffffu, f);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) wsum[warp] = __popc(m);
    __syncthreads();
    int pos = __popc(m & ((1u << lane) - 1u));
    for (int w = 0; w < warp; ++w) pos += wsum[w];
    return pos;
}

template <typename T>
__global__ void __launch_bounds__(kBlk) k_keep_count(const MaxRecB<T>* __restrict__ in, int n, double ths,
                                                     int* __restrict__ cnt) {
    const int i = blockIdx.x * kBlk + threadIdx.x;
    const bool f = i < n && (double)in[i].field > ths;
    const int c = __syncthreads_count(f);
    if (threadIdx.x == 0) cnt[blockIdx.x] = c;
}

template <typename T>
__global__ void __launch_bounds__(kBlk) k_keep_write(const MaxRecB<T>* __restrict__ in, int n, double ths, double h0,
                                                     double h1, double h2, double box, const int* __restrict__ off,
                                                     double* __restrict__ pos, int* __restrict__ flags) {
    __shared__ int wsum[kBlk / 32];
    const int i = blockIdx.x * kBlk + threadIdx.x;
    const bool f = i < n && (double)in[i].field > ths;
    const int r = block_rank(f, wsum);
    if (!f) return;
    const int p = off[blockIdx.x] + r;
    const double x = (double)in[i].i0 * h0, y = (double)in[i].i1 * h1, z = (double)in[i].i2 * h2;
    pos[3 * p] = x; pos[3 * p + 1] = y; pos[3 * p + 2] = z;
    if (!(x >= 0.0 && x < box && y >= 0.0 && y < box && z >= 0.0 && z < box)) atomicOr(&flags[1], 1);
}

// ---- cells -----------------------------------------------------------------------------
__device__ __forceinline__ int cell_of(double v, double box, int nc) {
    int c = (int)floor(v / box * nc);
    return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__global__ void k_cell_count(const double* __restrict__ pos, const int* __restrict__ np, double box, int nc,
                             int* __restrict__ cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *np) return;
    const int c = (cell_of(pos[3 * i + 2], box, nc) * nc + cell_of(pos[3 * i + 1], box, nc)) * nc +
                  cell_of(pos[3 * i], box, nc);
    atomicAdd(&cnt[c], 1);
}

__global__ void k_cell_fill(const double* __restrict__ pos, const int* __restrict__ np, double box, int nc,
                            const int* __restrict__ off, int* __restrict__ fill, int* __restrict__ atoms) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *np) return;
    const int c = (cell_of(pos[3 * i + 2], box, nc) * nc + cell_of(pos[3 * i + 1], box, nc)) * nc +
                  cell_of(pos[3 * i], box, nc);
    atomicExch(&atoms[off[c] + atomicAdd(&fill[c], 1)], i);
}

// get_diff (bond-order.cpp:53-64) with its tie order
__device__ __forceinline__ double get_diff(double x1, double x2, double w) {
    const double d1 = x1 - x2, d2 = d1 - w, d3 = d1 + w;
    if (fabs(d1) < fabs(d2)) return fabs(d1) < fabs(d3) ? d1 : d3;
    return fabs(d2) < fabs(d3) ? d2 : d3;
}

// kFill false: count the neighbours of atom i; true: also write them to list (whose
// length the counting pass found).
template <bool kFill>
__device__ __forceinline__ void try_pair(const double* __restrict__ pos, int i, int j, double xi, double yi,
                                         double zi, double box, double rlim, int* list, int& cnt, int& maxj) {
    if (j == i) return;
    const double dx = get_diff(pos[3 * j], xi, box);
    const double dy = get_diff(pos[3 * j + 1], yi, box);
    const double dz = get_diff(pos[3 * j + 2], zi, box);
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (r <= rlim) {
        if (kFill) list[cnt] = j;
        ++cnt;
        maxj = max(maxj, j);
    }
}

// One thread per atom; nc == 0 selects all pairs (positions outside the box or a box too
// small for three cells per side).  Counting pass (kFill false): nbc, maxjs.  Filling
// pass: the list of atom i at nbr + nb_off[i], sorted by index (the reference sums over
// neighbours in index order, bond-order.cpp:289-349).
template <bool kFill>
__global__ void k_neighbours(const double* __restrict__ pos, const int* __restrict__ np, double box, double rlim,
                             int nc, const int* __restrict__ cell_off, const int* __restrict__ cell_atoms,
                             const int* __restrict__ nb_off, int* __restrict__ nbr, int* __restrict__ nbc,
                             int* __restrict__ maxjs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int P = *np;
    if (i >= P) return;
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
    int* list = kFill ? nbr + nb_off[i] : nullptr;
    int cnt = 0, maxj = -1;
    if (nc == 0) {
        for (int j = 0; j < P; ++j) try_pair<kFill>(pos, i, j, xi, yi, zi, box, rlim, list, cnt, maxj);
    } else {
        const int cx = cell_of(xi, box, nc), cy = cell_of(yi, box, nc), cz = cell_of(zi, box, nc);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int c = (((cz + dz + nc) % nc) * nc + (cy + dy + nc) % nc) * nc + (cx + dx + nc) % nc;
                    for (int k = cell_off[c]; k < cell_off[c + 1]; ++k)
                        try_pair<kFill>(pos, i, cell_atoms[k], xi, yi, zi, box, rlim, list, cnt, maxj);
                }
    }
    if (!kFill) {
        nbc[i] = cnt;
        maxjs[i] = maxj;
        return;
    }
    for (int a = 1; a < cnt; ++a) {  // insertion sort into index order
        const int v = list[a];
        int b = a - 1;
        while (b >= 0 && list[b] > v) { list[b + 1] = list[b]; --b; }
        list[b + 1] = v;
    }
}

// q_lm for one (atom, l): thread t handles atom t/3, l = 4, 6, 8
template <int L>
__device__ void qlm_atom(const double* __restrict__ pos, int i, const int* __restrict__ list, int cnt, double box,
                         double2* __restrict__ out, int lidx) {
    double2 acc[2 * L + 1];
#pragma unroll
    for (int m = 0; m < 2 * L + 1; ++m) acc[m] = make_double2(0.0, 0.0);
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
    for (int a = 0; a < cnt; ++a) {
        const int j = list[a];
        const double dx = get_diff(pos[3 * j], xi, box);
        const double dy = get_diff(pos[3 * j + 1], yi, box);
        const double dz = get_diff(pos[3 * j + 2], zi, box);
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double x = dz / r;
        const double rho = sqrt(dx * dx + dy * dy);
        double2 eip = rho > 0.0 ? make_double2(dx / rho, dy / rho) : make_double2(1.0, 0.0);
        const double s = sqrt(fmax(0.0, 1.0 - x * x));
        const bool north = fabs(1.0 - x) < 1e-3, south = fabs(1.0 + x) < 1e-3;
        double pmm = 1.0, fct = 1.0;
        double2 em = make_double2(1.0, 0.0);
#pragma unroll
        for (int m = 0; m <= L; ++m) {
            if (m > 0) {
                pmm = -pmm * fct * s;
                fct += 2.0;
                em = make_double2(em.x * eip.x - em.y * eip.y, em.x * eip.y + em.y * eip.x);
            }
            double plm;
            if (m == L) plm = pmm;
            else {
                double p0 = pmm, p1 = x * (2 * m + 1) * pmm;
                for (int ll = m + 2; ll <= L; ++ll) {
                    const double p2 = (x * (2 * ll - 1) * p1 - (ll + m - 1) * p0) / (ll - m);
                    p0 = p1; p1 = p2;
                }
                plm = p1;
            }
            const double v = c_nlm[lidx][m] * plm;
            if (m == 0) {
                acc[L].x += v;
            } else {
                if (!north) { acc[L + m].x += v * em.x; acc[L + m].y += v * em.y; }
                if (!south) {
                    const double sg = (m & 1) ? -1.0 : 1.0;  // Y_l^-m = (-1)^m conj(Y_l^m)
                    acc[L - m].x += sg * v * em.x;
                    acc[L - m].y -= sg * v * em.y;
                }
            }
        }
    }
    const double inv = 1.0 / (double)cnt;
#pragma unroll
    for (int m = 0; m < 2 * L + 1; ++m) out[m] = make_double2(acc[m].x * inv, acc[m].y * inv);
}

__global__ void k_qlm(const double* __restrict__ pos, const int* __restrict__ np, const int* __restrict__ nbr,
                      const int* __restrict__ nb_off, const int* __restrict__ nbc, double box,
                      double2* __restrict__ q) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t / 3, which = t - 3 * (t / 3);
    if (i >= *np) return;
    const int cnt = nbc[i];
    if (cnt == 0) return;
    const int* list = nbr + nb_off[i];
    double2* qi = q + (size_t)i * kNQ;
    if (which == 0) qlm_atom<4>(pos, i, list, cnt, box, qi, 0);
    else if (which == 1) qlm_atom<6>(pos, i, list, cnt, box, qi + 9, 1);
    else qlm_atom<8>(pos, i, list, cnt, box, qi + 22, 2);
}

__device__ __forceinline__ double sumsq(const double2* a, int n) {
    double s = 0.0;
    for (int m = 0; m < n; ++m) s += a[m].x * a[m].x + a[m].y * a[m].y;
    return s;
}
__device__ double wl4(const double2* q) {
    double re = 0.0;
    for (int k = 0; k < kW4; ++k) {
        const int m1 = c_w4m[k][0], m2 = c_w4m[k][1], m3 = -m1 - m2;
        const double2 a = q[m1 + 4], b = q[m2 + 4], c = q[m3 + 4];
        const double2 ab = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
        re += c_w4[k] * (ab.x * c.x - ab.y * c.y);
    }
    const double s = sumsq(q, 9);
    return re / sqrt(s * s * s);
}
__device__ double wl6(const double2* q) {
    double re = 0.0;
    for (int k = 0; k < kW6; ++k) {
        const int m1 = c_w6m[k][0], m2 = c_w6m[k][1], m3 = -m1 - m2;
        const double2 a = q[m1 + 6], b = q[m2 + 6], c = q[m3 + 6];
        const double2 ab = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
        re += c_w6[k] * (ab.x * c.x - ab.y * c.y);
    }
    const double s = sumsq(q, 13);
    return re / sqrt(s * s * s);
}

constexpr double kPi = 3.14159265358979323846;

// per-atom invariants; rows of PFC_BOND_NCOL doubles for atoms with neighbours
__global__ void __launch_bounds__(kBlk) k_bond_rows(const double* __restrict__ pos, const int* __restrict__ np,
                                                    const int* __restrict__ nbr, const int* __restrict__ nb_off,
                                                    const int* __restrict__ nbc,
                                                    const int* __restrict__ maxjs, const double2* __restrict__ q,
                                                    const int* __restrict__ row_off, double* __restrict__ rows,
                                                    int row_capacity, int count_only, int* __restrict__ row_cnt) {
    __shared__ int wsum[kBlk / 32];
    const int i = blockIdx.x * kBlk + threadIdx.x;
    const int P = *np;
    const bool has = i < P && nbc[i] > 0;
    if (count_only) {
        const int c = __syncthreads_count(has);
        if (threadIdx.x == 0) row_cnt[blockIdx.x] = c;
        return;
    }
    const int rank = block_rank(has, wsum);
    if (!has) return;
    const int row = row_off[blockIdx.x] + rank;
    if (row >= row_capacity) return;
    const int cnt = nbc[i];
    const int* list = nbr + nb_off[i];
    const double2* qi = q + (size_t)i * kNQ;
    double out[PFC_BOND_NCOL];
    out[0] = pos[3 * i]; out[1] = pos[3 * i + 1]; out[2] = pos[3 * i + 2];
    out[3] = (double)nbc[i];
    // q_l
    out[5] = sqrt(4.0 * kPi / 9.0 * sumsq(qi, 9));
    out[6] = sqrt(4.0 * kPi / 13.0 * sumsq(qi + 9, 13));
    out[7] = sqrt(4.0 * kPi / 17.0 * sumsq(qi + 22, 17));
    out[8] = wl4(qi);
    out[13] = wl6(qi + 9);
    // q-bar_l, self included (bond-order.cpp:221-250)
    const double invn = 1.0 / (1.0 + (double)nbc[i]);
    const int lofs[3] = {0, 9, 22}, lw[3] = {9, 13, 17};
    for (int li = 0; li < 3; ++li) {
        double ss = 0.0;
        for (int m = 0; m < lw[li]; ++m) {
            double2 s = qi[lofs[li] + m];
            for (int a = 0; a < cnt; ++a) {
                const double2 o = q[(size_t)list[a] * kNQ + lofs[li] + m];
                s.x += o.x; s.y += o.y;
            }
            s.x *= invn; s.y *= invn;
            ss += s.x * s.x + s.y * s.y;
        }
        out[9 + li] = sqrt(4.0 * kPi / (double)lw[li] * ss);
    }
    // w4b as the reference computes it: the last neighbour's q4m divided by Nb
    {
        double2 qb[9];
        const double2* ql = q + (size_t)maxjs[i] * kNQ;
        for (int m = 0; m < 9; ++m) qb[m] = make_double2(ql[m].x / (double)nbc[i], ql[m].y / (double)nbc[i]);
        out[12] = wl4(qb);
    }
    // xi: neighbours with normalised q6 . conj(q6) > 0.7 (bond-order.cpp:267-287)
    {
        const double2* q6 = qi + 9;
        const double ni = sqrt(sumsq(q6, 13));
        int s = 0;
        for (int a = 0; a < cnt; ++a) {
            const double2* o = q + (size_t)list[a] * kNQ + 9;
            double d = 0.0;
            for (int m = 0; m < 13; ++m) d += q6[m].x * o[m].x + q6[m].y * o[m].y;
            if (d / (ni * sqrt(sumsq(o, 13))) > 0.7) ++s;
        }
        out[4] = (double)s;
    }
    for (int c = 0; c < PFC_BOND_NCOL; ++c) rows[(size_t)row * PFC_BOND_NCOL + c] = out[c];
}

double fact(int n) { double r = 1.0; for (int k = 2; k <= n; ++k) r *= k; return r; }

// Wigner 3j (l l l; m1 m2 m3) by the Racah formula, evaluated in long double.
double wigner3j_lll(int l, int m1, int m2, int m3) {
    if (m1 + m2 + m3 != 0) return 0.0;
    const int j1 = l, j2 = l, j3 = l;
    auto lf = [](int n) { long double r = 1.0L; for (int k = 2; k <= n; ++k) r *= k; return r; };
    const long double tri = lf(j1 + j2 - j3) * lf(j1 - j2 + j3) * lf(-j1 + j2 + j3) / lf(j1 + j2 + j3 + 1);
    const long double pref = sqrtl(tri * lf(j1 + m1) * lf(j1 - m1) * lf(j2 + m2) * lf(j2 - m2) * lf(j3 + m3) * lf(j3 - m3));
    const int kmin = std::max(0, std::max(j2 - j3 - m1, j1 - j3 + m2));
    const int kmax = std::min(j1 + j2 - j3, std::min(j1 - m1, j2 + m2));
    long double s = 0.0L;
    for (int k = kmin; k <= kmax; ++k) {
        const long double den = lf(k) * lf(j1 + j2 - j3 - k) * lf(j1 - m1 - k) * lf(j2 + m2 - k) *
                                lf(j3 - j2 + m1 + k) * lf(j3 - j1 - m2 + k);
        s += ((k & 1) ? -1.0L : 1.0L) / den;
    }
    const int sg = ((j1 - j2 - m3) % 2 == 0) ? 1 : -1;
    return (double)(sg * pref * s);
}

cudaError_t upload_tables() {
    int ready = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&ready, c_tables_ready, sizeof(int));
    if (e) return e;
    if (ready) return cudaSuccess;
    double nlm[3][9] = {};
    const int ls[3] = {4, 6, 8};
    for (int li = 0; li < 3; ++li)
        for (int m = 0; m <= ls[li]; ++m)
            nlm[li][m] = std::sqrt((2 * ls[li] + 1) / (4.0 * kPi) * fact(ls[li] - m) / fact(ls[li] + m));
    std::vector<double> w4, w6;
    std::vector<int> m4, m6;
    for (int a = -4; a <= 4; ++a)
        for (int b = -4; b <= 4; ++b)
            if (std::abs(a + b) <= 4) { w4.push_back(wigner3j_lll(4, a, b, -a - b)); m4.push_back(a); m4.push_back(b); }
    for (int a = -6; a <= 6; ++a)
        for (int b = -6; b <= 6; ++b)
            if (std::abs(a + b) <= 6) { w6.push_back(wigner3j_lll(6, a, b, -a - b)); m6.push_back(a); m6.push_back(b); }
    if ((int)w4.size() != kW4 || (int)w6.size() != kW6) return cudaErrorInvalidValue;
    if ((e = cudaMemcpyToSymbol(c_nlm, nlm, sizeof(nlm)))) return e;
    if ((e = cudaMemcpyToSymbol(c_w4, w4.data(), sizeof(double) * kW4))) return e;
    if ((e = cudaMemcpyToSymbol(c_w4m, m4.data(), sizeof(int) * 2 * kW4))) return e;
    if ((e = cudaMemcpyToSymbol(c_w6, w6.data(), sizeof(double) * kW6))) return e;
    if ((e = cudaMemcpyToSymbol(c_w6m, m6.data(), sizeof(int) * 2 * kW6))) return e;
    ready = 1;
    return cudaMemcpyToSymbol(c_tables_ready, &ready, sizeof(int));
}

}  // namespace

size_t bond_scratch_bytes(int max_atoms) { return scratch_layout(max_atoms, nullptr, nullptr); }

// Grows the context's bond-order scratch to hold `atoms` atoms and `pairs` neighbour
// entries (allocation sizes only grow; nothing is kept across calls, so no copy).
cudaError_t bond_reserve(pfc_ctx* c, int atoms, int64_t pairs) {
    cudaError_t e = cudaSuccess;
    if (atoms > c->max_atoms) {
        const int want = std::max(atoms, c->max_atoms + c->max_atoms / 2);
        void* p = nullptr;
        if ((e = cudaMalloc(&p, bond_scratch_bytes(want)))) return e;
        if (c->bond_scratch) cudaFree(c->bond_scratch);
        c->bond_scratch = p;
        c->max_atoms = want;
        c->bond_scratch_bytes = bond_scratch_bytes(want);
    }
    if (pairs > c->max_pairs) {
        const int64_t want = std::max<int64_t>(pairs, c->max_pairs + c->max_pairs / 2);
        void* p = nullptr;
        if ((e = cudaMalloc(&p, sizeof(int) * (size_t)want))) return e;
        if (c->bond_pairs) cudaFree(c->bond_pairs);
        c->bond_pairs = (int*)p;
        c->max_pairs = want;
    }
    return cudaSuccess;
}

cudaError_t launch_bond_order(pfc_ctx* c, const void* maxima, int n, double h0, double h1, double h2, double ths,
                              double boxsize, double rlim, double* out_rows, int row_capacity, int* n_rows_host) {
    cudaError_t e = upload_tables();
    if (e) return e;
    if ((e = bond_reserve(c, n, 0))) return e;
    BondScratch s;
    scratch_layout(c->max_atoms, &s, (char*)c->bond_scratch);
    cudaStream_t st = c->stream;
    const int nblk = (n + kBlk - 1) / kBlk;
    if ((e = cudaMemsetAsync(s.flags, 0, sizeof(int) * 8, st))) return e;
    // 1. keep field > ths (order preserved)
    if (nblk > 0) {
        if (c->dtype == PFC_F64) k_keep_count<double><<<nblk, kBlk, 0, st>>>((const MaxRecB<double>*)maxima, n, ths, s.keep_cnt);
        else k_keep_count<float><<<nblk, kBlk, 0, st>>>((const MaxRecB<float>*)maxima, n, ths, s.keep_cnt);
        k_scan_b<<<1, 1024, 0, st>>>(s.keep_cnt, nblk, s.keep_off);
        if (c->dtype == PFC_F64)
            k_keep_write<double><<<nblk, kBlk, 0, st>>>((const MaxRecB<double>*)maxima, n, ths, h0, h1, h2, boxsize,
                                                         s.keep_off, s.pos, s.flags);
        else
            k_keep_write<float><<<nblk, kBlk, 0, st>>>((const MaxRecB<float>*)maxima, n, ths, h0, h1, h2, boxsize,
                                                        s.keep_off, s.pos, s.flags);
        if ((e = cudaMemcpyAsync(s.flags + 2, s.keep_off + nblk, sizeof(int), cudaMemcpyDeviceToDevice, st))) return e;
    }
    int hflags[3] = {0, 0, 0};
    if ((e = cudaMemcpyAsync(hflags, s.flags, sizeof(int) * 3, cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaStreamSynchronize(st))) return e;
    const int P = hflags[2];
    const int* np = s.flags + 2;
    if (P == 0) { *n_rows_host = 0; return cudaSuccess; }
    // 2. cells of side >= rlim (all pairs when fewer than 3 per side or atoms outside the box)
    int nc = (int)std::floor(boxsize / rlim);
    if (nc > kMaxCellsDim) nc = kMaxCellsDim;
    if (nc < 3 || hflags[1] || !(rlim > 0.0)) nc = 0;
    const int pb = (P + 255) / 256;
    if (nc > 0) {
        const int cells = nc * nc * nc;
        if ((e = cudaMemsetAsync(s.cell_cnt, 0, sizeof(int) * cells, st))) return e;
        if ((e = cudaMemsetAsync(s.cell_fill, 0, sizeof(int) * cells, st))) return e;
        k_cell_count<<<pb, 256, 0, st>>>(s.pos, np, boxsize, nc, s.cell_cnt);
        k_scan_b<<<1, 1024, 0, st>>>(s.cell_cnt, cells, s.cell_off);
        k_cell_fill<<<pb, 256, 0, st>>>(s.pos, np, boxsize, nc, s.cell_off, s.cell_fill, s.cell_atoms);
    }
    // 3. neighbour lists: count, scan into list offsets, grow the pair buffer, fill
    k_neighbours<false><<<pb, 256, 0, st>>>(s.pos, np, boxsize, rlim, nc, s.cell_off, s.cell_atoms, nullptr, nullptr,
                                            s.nb, s.maxj);
    k_scan_b<<<1, 1024, 0, st>>>(s.nb, P, s.nb_off);
    if ((e = cudaGetLastError())) return e;
    int pairs = 0;
    if ((e = cudaMemcpyAsync(&pairs, s.nb_off + P, sizeof(int), cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaStreamSynchronize(st))) return e;
    if ((e = bond_reserve(c, 0, pairs))) return e;
    k_neighbours<true><<<pb, 256, 0, st>>>(s.pos, np, boxsize, rlim, nc, s.cell_off, s.cell_atoms, s.nb_off,
                                           c->bond_pairs, nullptr, nullptr);
    k_qlm<<<(3 * P + 127) / 128, 128, 0, st>>>(s.pos, np, c->bond_pairs, s.nb_off, s.nb, boxsize, s.q);
    const int rb = (P + kBlk - 1) / kBlk;
    k_bond_rows<<<rb, kBlk, 0, st>>>(s.pos, np, c->bond_pairs, s.nb_off, s.nb, s.maxj, s.q, nullptr, nullptr, 0, 1,
                                     s.row_cnt);
    k_scan_b<<<1, 1024, 0, st>>>(s.row_cnt, rb, s.row_off);
    k_bond_rows<<<rb, kBlk, 0, st>>>(s.pos, np, c->bond_pairs, s.nb_off, s.nb, s.maxj, s.q, s.row_off, out_rows,
                                     row_capacity, 0, s.row_cnt);
    if ((e = cudaGetLastError())) return e;
    int rows = 0;
    if ((e = cudaMemcpyAsync(&rows, s.row_off + rb, sizeof(int), cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaStreamSynchronize(st))) return e;
    *n_rows_host = rows;
    return cudaSuccess;
}

}  // namespace pfc
