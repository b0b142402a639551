// jengine.cu -- the McMurchie-Davidson J-engine on sm_100a.
//
// Device layout.  The unique sweep's records (one per primitive pair of each
// shell pair a >= b, i outer; eri/j_coulomb/j.py:395-405) are stored grouped
// by L = l_a + l_b (stable, so each group keeps sweep order and a shell
// pair's records stay contiguous).  Each record owns a Hermite vector of
// NH(L) = (L+1)(L+2)(L+3)/6 doubles at dq_off in two buffers: D_q (its ket
// role) and J_p (its bra role).
//
// Kernels, in stream order, per build:
//   j_dq_kernel      warp per record: the per-axis Hermite tables E^{ij}_t
//                    (mmd/hermite.py:61-79) in shared memory, lanes over q:
//                    D_q = w pre sum_cd D_cd E^{cd}_q, then key = I_pair *
//                    max_q |D_q| (ao/density.py:120-148, launch.py:300-310).
//   segmented radix sort (CUB) of the keys, descending and stable, one
//                    segment per L: the ket order of launch.py:325.
//   j_pq_small_kernel<LP, LQ> (lp + lq <= 6: every Hermite index a template
//   constant, R in registers) / j_pq_kernel<L> (the rest, table-indexed)
//                    one launch per (bra L, ket L) class: a warp per bra
//                    record walks the class's sorted kets 32 at a time, one
//                    lane per ket, and stops after the chunk holding the
//                    first ket with I_bra * key < tau (the sorted break,
//                    j.py:520-536).  A lane forms [0]^(m) = (2/sqrt(pi))
//                    theta (-2 theta^2)^m F_m(theta^2 |PQ|^2) (reference/
//                    pq.py:40-58), raises R_{tuv} in registers by
//                    [r]^(m) = PQ_d [r-1_d]^(m+1) + (r_d - 1) [r-2_d]^(m+1)
//                    along the first nonzero axis (pq.py:103-114), and adds
//                    (-1)^|q| R_{p+q} D_q into its J_p partials; the warp
//                    reduces them by shuffles and one lane adds them to the
//                    record's J_p.
//   j_jab_kernel     warp per unique shell pair: J_ab = sum_records pre
//                    sum_p E^{ab}_p J_p, written to J[a][b] and mirrored to
//                    J[b][a]; on a diagonal pair only the lower triangle
//                    i >= j writes (both positions), so every element of J
//                    has exactly one writer: no atomics and no zeroing
//                    (j.py:303-326's scatter).
// Roofline: j_pq_kernel is FP64-pipe bound (R recursion + NH(LP) x NH(LQ)
// FMAs per bra-ket record pair); the others are small.
#include "jengine.h"

#include <cub/device/device_segmented_radix_sort.cuh>

#include <algorithm>
#include <array>
#include <cmath>
#include <memory>
#include <numeric>
#include <utility>

#include "fock_compiled.cuh"

namespace fjb {

namespace {

constexpr int kJMaxL = 2 * kMaxL;  // L of one record
constexpr int kNHMax = (kJMaxL + 1) * (kJMaxL + 2) * (kJMaxL + 3) / 6;  // 84

__host__ __device__ constexpr int nh(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }

// cartesians(l) components for l <= 3, at offset l(l+1)(l+2)/6.
__constant__ int8_t kCart[20][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {1, 1, 0}, {1, 0, 1},
                                    {0, 2, 0}, {0, 1, 1}, {0, 0, 2}, {3, 0, 0}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0},
                                    {1, 1, 1}, {1, 0, 2}, {0, 3, 0}, {0, 2, 1}, {0, 1, 2}, {0, 0, 3}};

// Hermite indices (t, u, v) of hermite_order(2 * kJMaxL), for R tables.
constexpr int kNRMax = nh(2 * kJMaxL);  // 455
__constant__ int8_t kHermR[kNRMax][3];

struct JRec {
    double P[3], PA[3], PB[3];
    double zeta, pre, G;  // pre = c_a c_b (pi/zeta)^{3/2} exp(-alpha beta/zeta |AB|^2)
    int32_t la, lb, ao_a, ao_b;
    int32_t L, pair, dq_off, pad;
};
static_assert(sizeof(JRec) == 128, "JRec is 128 bytes");

constexpr int kETab = 4 * 4 * (kJMaxL + 1);  // E[i][j][t], i, j <= 3, t <= 6

// One axis's E^{ij}_t for i <= la, j <= lb (E^{00}_0 = 1: the Gaussian
// product factor is in pre), zero beyond t = i + j.
__device__ void e_table(int la, int lb, double h, double pa, double pb, double *E) {
    for (int k = 0; k < kETab; ++k) E[k] = 0.0;
    auto at = [&](int i, int j, int t) -> double & { return E[(i * 4 + j) * (kJMaxL + 1) + t]; };
    at(0, 0, 0) = 1.0;
    for (int i = 0; i < la; ++i)
        for (int t = 0; t <= i + 1; ++t) {
            double v = pa * at(i, 0, t);
            if (t >= 1) v += h * at(i, 0, t - 1);
            if (t + 1 <= i) v += (double)(t + 1) * at(i, 0, t + 1);
            at(i + 1, 0, t) = v;
        }
    for (int i = 0; i <= la; ++i)
        for (int j = 0; j < lb; ++j)
            for (int t = 0; t <= i + j + 1; ++t) {
                double v = pb * at(i, j, t);
                if (t >= 1) v += h * at(i, j, t - 1);
                if (t + 1 <= i + j) v += (double)(t + 1) * at(i, j, t + 1);
                at(i, j + 1, t) = v;
            }
}

__device__ __forceinline__ double etab(const double *E, int i, int j, int t) {
    return E[(i * 4 + j) * (kJMaxL + 1) + t];
}

__global__ void j_dq_kernel(const JRec *__restrict__ recs, int n, const double *__restrict__ D, int n_ao,
                            double *__restrict__ Dq, double *__restrict__ key) {
    __shared__ double Es[4][3][kETab];
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); r < n; r += nw) {
        const JRec R = recs[r];
        if (lane < 3) e_table(R.la, R.lb, 0.5 / R.zeta, R.PA[lane], R.PB[lane], Es[wl][lane]);
        __syncwarp();
        const double *Ex = Es[wl][0], *Ey = Es[wl][1], *Ez = Es[wl][2];
        const int na = (R.la + 1) * (R.la + 2) / 2, nb = (R.lb + 1) * (R.lb + 2) / 2;
        const int ca = R.la * (R.la + 1) * (R.la + 2) / 6, cb = R.lb * (R.lb + 1) * (R.lb + 2) / 6;
        const double w = R.ao_a == R.ao_b ? 1.0 : 2.0;
        double m = 0.0;
        for (int q = lane; q < nh(R.L); q += 32) {
            const int t = kHermR[q][0], u = kHermR[q][1], v = kHermR[q][2];
            double acc = 0.0;
            for (int i = 0; i < na; ++i) {
                const int8_t *c = kCart[ca + i];
                const double *Drow = D + (size_t)(R.ao_a + i) * n_ao + R.ao_b;
                for (int j = 0; j < nb; ++j) {
                    const int8_t *d = kCart[cb + j];
                    const double e = etab(Ex, c[0], d[0], t) * etab(Ey, c[1], d[1], u) * etab(Ez, c[2], d[2], v);
                    acc += Drow[j] * e;
                }
            }
            const double dq = w * (R.pre * acc);
            Dq[R.dq_off + q] = dq;
            m = fmax(m, fabs(dq));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) key[r] = R.G * m;
        __syncwarp();
    }
}

__device__ __forceinline__ int h_index(int t, int u, int v) {
    const int n = t + u + v;
    return (n == 0 ? 0 : nh(n - 1)) + (n - t) * (n - t + 1) / 2 + (n - t - u);
}

// hermite_order index -> (t, u, v), constexpr, for the unrolled kernels.
__host__ __device__ constexpr int hc_total(int idx) {
    int n = 0;
    while (nh(n) <= idx) ++n;
    return n;
}
__host__ __device__ constexpr int hc_t(int idx) {
    const int n = hc_total(idx);
    int r = idx - (n == 0 ? 0 : nh(n - 1)), t = n;
    while (r >= n - t + 1) {
        r -= n - t + 1;
        --t;
    }
    return t;
}
__host__ __device__ constexpr int hc_u(int idx) {
    const int n = hc_total(idx);
    int r = idx - (n == 0 ? 0 : nh(n - 1)), t = n;
    while (r >= n - t + 1) {
        r -= n - t + 1;
        --t;
    }
    return n - t - r;
}
__host__ __device__ constexpr int hc_v(int idx) { return hc_total(idx) - hc_t(idx) - hc_u(idx); }
__host__ __device__ constexpr int hc_idx(int t, int u, int v) {
    const int n = t + u + v;
    return (n == 0 ? 0 : nh(n - 1)) + (n - t) * (n - t + 1) / 2 + (n - t - u);
}

// Compile-time walks of the small classes: every index below is a template
// constant (fold expressions over integer sequences), so R, the signed D_q
// and the J_p partials stay in registers.
// One entry I of the R recursion: [r]^(m) = PQ_d [r-1_d]^(m+1) + (r_d - 1)
// [r-2_d]^(m+1), d the first nonzero axis.
template <int I, typename T>
__device__ __forceinline__ void r_entry(T *R, T X, T Y, T Z) {
    constexpr int t = hc_t(I), u = hc_u(I), v = hc_v(I);
    if constexpr (t > 0) {
        T x = X * R[hc_idx(t - 1, u, v)];
        if constexpr (t >= 2) x += (T)(t - 1) * R[hc_idx(t - 2, u, v)];
        R[I] = x;
    } else if constexpr (u > 0) {
        T x = Y * R[hc_idx(0, u - 1, v)];
        if constexpr (u >= 2) x += (T)(u - 1) * R[hc_idx(0, u - 2, v)];
        R[I] = x;
    } else {
        T x = Z * R[hc_idx(0, 0, v - 1)];
        if constexpr (v >= 2) x += (T)(v - 1) * R[hc_idx(0, 0, v - 2)];
        R[I] = x;
    }
}
template <int I0, typename T, int... K>
__device__ __forceinline__ void r_entries(T *R, T X, T Y, T Z, std::integer_sequence<int, K...>) {
    (r_entry<I0 + K, T>(R, X, Y, Z), ...);
}
// Totals S, S-1, .. 1 of one level (descending: each reads the level above
// at totals S-1 and S-2 before they are rewritten).
template <int S, typename T>
struct RTotals {
    static __device__ __forceinline__ void run(T *R, T X, T Y, T Z) {
        if constexpr (S >= 1) {
            r_entries<nh(S - 1), T>(R, X, Y, Z, std::make_integer_sequence<int, nh(S) - nh(S - 1)>{});
            RTotals<S - 1, T>::run(R, X, Y, Z);
        }
    }
};
// Levels M, M-1, .. 0 of R_{tuv} at total order L.
template <int L, int M, typename T>
struct RLevels {
    static __device__ __forceinline__ void run(T *R, const T *f, T X, T Y, T Z) {
        if constexpr (M >= 0) {
            RTotals<L - M, T>::run(R, X, Y, Z);
            R[0] = f[M];
            RLevels<L, M - 1, T>::run(R, f, X, Y, Z);
        }
    }
};
// d[q] = (-1)^|q| D_q.
template <typename T, int... Q>
__device__ __forceinline__ void signed_dq(T *d, const double *dq, std::integer_sequence<int, Q...>) {
    ((d[Q] = (T)(((hc_total(Q) & 1) ? -1.0 : 1.0) * __ldg(dq + Q))), ...);
}
// jp[p] += R_{p+q} d[q] over I = p * NQ + q.
template <int NQ, int I>
struct PQIndex {
    static constexpr int pi = I / NQ, qi = I % NQ;
    static constexpr int r = hc_idx(hc_t(pi) + hc_t(qi), hc_u(pi) + hc_u(qi), hc_v(pi) + hc_v(qi));
};
template <int NQ, typename T, int... I>
__device__ __forceinline__ void contract(T *jp, const T *R, const T *d, std::integer_sequence<int, I...>) {
    ((jp[PQIndex<NQ, I>::pi] += R[PQIndex<NQ, I>::r] * d[PQIndex<NQ, I>::qi]), ...);
}

// The classes with lp + lq <= kSmallL: the same walk as j_pq_kernel with
// every index a compile-time constant.
constexpr int kSmallL = 6;

// thr32 > 0: a chunk of kets whose first (largest) bound I_bra key is below
// it runs R, D_q and the contraction in FP32 (T, the Boys values and the
// J_p sums stay FP64): the FP32 E/R tier.  The kets are sorted by key, so
// every ket of such a chunk is under the bound too.
template <int LP, int LQ>
__global__ void __launch_bounds__(128) j_pq_small_kernel(const JRec *__restrict__ recs, int bra0, int nbra,
                                                         int ket0, int nket, const double4 *__restrict__ kst, const int *__restrict__ kdq,
                                                         const double *__restrict__ skey,
                                                         const double *__restrict__ Dq, double *__restrict__ Jp,
                                                         double tau, double thr32, const double *__restrict__ boys_tab) {
    constexpr int L = LP + LQ, NP = nh(LP), NQ = nh(LQ), NR = nh(L);
    constexpr double kTwoOverSqrtPi = 1.1283791670955126;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int bi = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); bi < nbra; bi += nw) {
        const JRec B = recs[bra0 + bi];
        double jp[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) jp[p] = 0.0;
        for (int k0 = 0; k0 < nket; k0 += 32) {
            const int k = k0 + lane;
            const bool on = k < nket && !(B.G * skey[ket0 + k] < tau);
            const bool f32 = thr32 > 0.0 && B.G * skey[ket0 + k0] < thr32;  // uniform over the warp
            if (on) {
                const double4 KP = kst[ket0 + k];  // (P, eta) of the k-th ket in key order
                const int kdo = kdq[ket0 + k];
                const double p = B.zeta, q = KP.w;
                const double rho = p * q / (p + q);
                const double X = B.P[0] - KP.x, Y = B.P[1] - KP.y, Z = B.P[2] - KP.z;
                const double T = rho * (X * X + Y * Y + Z * Z);
                double F[L + 1];
                boys_t<L>(T, F, boys_tab);
                const double pref = kTwoOverSqrtPi * sqrt(rho), m2r = -2.0 * rho;
                if (f32) {
                    float f[L + 1];
                    double pw = pref;
#pragma unroll
                    for (int m = 0; m <= L; ++m) {
                        f[m] = (float)(pw * F[m]);
                        pw *= m2r;
                    }
                    float R[NR];
                    R[0] = f[L];
                    RLevels<L, L - 1, float>::run(R, f, (float)X, (float)Y, (float)Z);
                    float d[NQ], j32[NP];
                    signed_dq<float>(d, Dq + kdo, std::make_integer_sequence<int, NQ>{});
#pragma unroll
                    for (int pi = 0; pi < NP; ++pi) j32[pi] = 0.f;
                    contract<NQ, float>(j32, R, d, std::make_integer_sequence<int, NP * NQ>{});
#pragma unroll
                    for (int pi = 0; pi < NP; ++pi) jp[pi] += (double)j32[pi];
                } else {
                    double f[L + 1];
                    double pw = pref;
#pragma unroll
                    for (int m = 0; m <= L; ++m) {
                        f[m] = pw * F[m];
                        pw *= m2r;
                    }
                    double R[NR];
                    R[0] = f[L];
                    RLevels<L, L - 1, double>::run(R, f, X, Y, Z);
                    double d[NQ];
                    signed_dq<double>(d, Dq + kdo, std::make_integer_sequence<int, NQ>{});
                    contract<NQ, double>(jp, R, d, std::make_integer_sequence<int, NP * NQ>{});
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, on);
            if (__popc(bal) < min(32, nket - k0)) break;  // the first ket under tau is in this chunk
        }
#pragma unroll
        for (int pi = 0; pi < NP; ++pi) {
            double v = jp[pi];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) Jp[B.dq_off + pi] += v;
        }
    }
}

// One bra-ket record pair of the table-indexed walk in T (float: the FP32
// E/R tier): R from the FP64 Boys values, then jp[p] += R_{p+q} (-1)^|q| D_q
// summed in T over the ket and added to the FP64 partials.
template <int L, typename T>
__device__ __forceinline__ void pq_lane_general(const JRec &B, double4 KP, const double *dq, int lp, int lq,
                                                const double *boys_tab, double *jp) {
    constexpr int NR = nh(L);
    constexpr double kTwoOverSqrtPi = 1.1283791670955126;
    const int NP = nh(lp), NQ = nh(lq);
    const double p = B.zeta, q = KP.w;
    const double rho = p * q / (p + q);
    const double Xd = B.P[0] - KP.x, Yd = B.P[1] - KP.y, Zd = B.P[2] - KP.z;
    const double Tt = rho * (Xd * Xd + Yd * Yd + Zd * Zd);
    double F[L + 1];
    boys_t<L>(Tt, F, boys_tab);
    const double pref = kTwoOverSqrtPi * sqrt(rho), m2r = -2.0 * rho;
    T f[L + 1];
    double pw = pref;
#pragma unroll
    for (int m = 0; m <= L; ++m) {
        f[m] = (T)(pw * F[m]);
        pw *= m2r;
    }
    const T X = (T)Xd, Y = (T)Yd, Z = (T)Zd;
    T R[NR];
    R[0] = f[L];
    for (int m = L - 1; m >= 0; --m) {
        for (int s = L - m; s >= 1; --s) {
            for (int i = nh(s - 1); i < nh(s); ++i) {
                const int t = kHermR[i][0], u = kHermR[i][1], v = kHermR[i][2];
                T x;
                if (t > 0) {
                    x = X * R[h_index(t - 1, u, v)];
                    if (t >= 2) x += (T)(t - 1) * R[h_index(t - 2, u, v)];
                } else if (u > 0) {
                    x = Y * R[h_index(0, u - 1, v)];
                    if (u >= 2) x += (T)(u - 1) * R[h_index(0, u - 2, v)];
                } else {
                    x = Z * R[h_index(0, 0, v - 1)];
                    if (v >= 2) x += (T)(v - 1) * R[h_index(0, 0, v - 2)];
                }
                R[i] = x;
            }
        }
        R[0] = f[m];
    }
    for (int pi = 0; pi < NP; ++pi) {
        T acc = (T)0;
        for (int qi = 0; qi < NQ; ++qi) {
            const int tq = kHermR[qi][0], uq = kHermR[qi][1], vq = kHermR[qi][2];
            const T d = (T)((((tq + uq + vq) & 1) ? -1.0 : 1.0) * __ldg(dq + qi));
            acc += R[h_index(kHermR[pi][0] + tq, kHermR[pi][1] + uq, kHermR[pi][2] + vq)] * d;
        }
        jp[pi] += (double)acc;
    }
}

// One (bra L, ket L) class at total order L = lp + lq (runtime lp, lq).
template <int L>
__global__ void __launch_bounds__(128) j_pq_kernel(const JRec *__restrict__ recs, int lp, int lq, int bra0, int nbra,
                                                   int ket0, int nket, const double4 *__restrict__ kst, const int *__restrict__ kdq,
                                                   const double *__restrict__ skey, const double *__restrict__ Dq,
                                                   double *__restrict__ Jp, double tau, double thr32,
                                                   const double *__restrict__ boys_tab) {
    constexpr int NR = nh(L), NPMAX = nh(L < kJMaxL ? L : kJMaxL);
    constexpr double kTwoOverSqrtPi = 1.1283791670955126;
    const int NP = nh(lp), NQ = nh(lq);
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int bi = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); bi < nbra; bi += nw) {
        const JRec B = recs[bra0 + bi];
        double jp[NPMAX];
        for (int p = 0; p < NP; ++p) jp[p] = 0.0;
        for (int k0 = 0; k0 < nket; k0 += 32) {
            const int k = k0 + lane;
            const bool on = k < nket && !(B.G * skey[ket0 + k] < tau);
            const bool f32 = thr32 > 0.0 && B.G * skey[ket0 + k0] < thr32;  // uniform over the warp
            if (on && f32) {
                pq_lane_general<L, float>(B, kst[ket0 + k], Dq + kdq[ket0 + k], lp, lq, boys_tab, jp);
            } else if (on) {
                const double4 KP = kst[ket0 + k];  // (P, eta) of the k-th ket in key order
                const int kdo = kdq[ket0 + k];
                const double p = B.zeta, q = KP.w;
                const double rho = p * q / (p + q);
                const double X = B.P[0] - KP.x, Y = B.P[1] - KP.y, Z = B.P[2] - KP.z;
                const double T = rho * (X * X + Y * Y + Z * Z);
                double F[L + 1];
                boys_t<L>(T, F, boys_tab);
                const double pref = kTwoOverSqrtPi * sqrt(rho), m2r = -2.0 * rho;
                double f[L + 1];
                double pw = pref;
#pragma unroll
                for (int m = 0; m <= L; ++m) {
                    f[m] = pw * F[m];
                    pw *= m2r;
                }
                // R_{tuv}: level m = L holds [0]^(L); each lower level
                // rewrites totals L-m .. 1 from the level above (read before
                // they are overwritten: totals descend), then [0]^(m).
                double R[NR];
                R[0] = f[L];
                for (int m = L - 1; m >= 0; --m) {
                    for (int s = L - m; s >= 1; --s) {
                        for (int i = nh(s - 1); i < nh(s); ++i) {
                            const int t = kHermR[i][0], u = kHermR[i][1], v = kHermR[i][2];
                            double x;
                            if (t > 0) {
                                x = X * R[h_index(t - 1, u, v)];
                                if (t >= 2) x += (double)(t - 1) * R[h_index(t - 2, u, v)];
                            } else if (u > 0) {
                                x = Y * R[h_index(0, u - 1, v)];
                                if (u >= 2) x += (double)(u - 1) * R[h_index(0, u - 2, v)];
                            } else {
                                x = Z * R[h_index(0, 0, v - 1)];
                                if (v >= 2) x += (double)(v - 1) * R[h_index(0, 0, v - 2)];
                            }
                            R[i] = x;
                        }
                    }
                    R[0] = f[m];
                }
                const double *dq = Dq + kdo;
                for (int qi = 0; qi < NQ; ++qi) {
                    const int tq = kHermR[qi][0], uq = kHermR[qi][1], vq = kHermR[qi][2];
                    const double d = (((tq + uq + vq) & 1) ? -1.0 : 1.0) * __ldg(dq + qi);
                    for (int pi = 0; pi < NP; ++pi)
                        jp[pi] += R[h_index(kHermR[pi][0] + tq, kHermR[pi][1] + uq, kHermR[pi][2] + vq)] * d;
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, on);
            if (__popc(bal) < min(32, nket - k0)) break;  // the first ket under tau is in this chunk
        }
        for (int pi = 0; pi < NP; ++pi) {
            double v = jp[pi];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) Jp[B.dq_off + pi] += v;
        }
    }
}

// The kets of every L in key order as a contiguous stream: (P, eta) of the
// k-th sorted ket, and its D_q copied into the D_q slot of position k (a
// group's slots have one stride, so position k's slot is record k's), so the
// walk's loads of consecutive kets are consecutive in memory.
__global__ void j_gather_kernel(const JRec *__restrict__ recs, const int *__restrict__ order, int n,
                                const double *__restrict__ Dq, double4 *__restrict__ kst, int *__restrict__ kdq,
                                double *__restrict__ Dqs) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const JRec R = recs[order[k]];
        const int dst = recs[k].dq_off;
        kst[k] = make_double4(R.P[0], R.P[1], R.P[2], R.zeta);
        kdq[k] = dst;
        for (int q = 0; q < nh(R.L); ++q) Dqs[dst + q] = Dq[R.dq_off + q];
    }
}

__global__ void j_jab_kernel(const JRec *__restrict__ recs, const int *__restrict__ pair_rec0,
                             const int *__restrict__ pair_nrec, int n_pairs, const double *__restrict__ Jp,
                             double *__restrict__ J, int n_ao) {
    __shared__ double Es[4][3][kETab];
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int pr = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); pr < n_pairs; pr += nw) {
        const int r0 = pair_rec0[pr], nr = pair_nrec[pr];
        const JRec R0 = recs[r0];
        const int na = (R0.la + 1) * (R0.la + 2) / 2, nb = (R0.lb + 1) * (R0.lb + 2) / 2;
        const int ca = R0.la * (R0.la + 1) * (R0.la + 2) / 6, cb = R0.lb * (R0.lb + 1) * (R0.lb + 2) / 6;
        const int nab = na * nb, np = nh(R0.L);
        double acc[4] = {0.0, 0.0, 0.0, 0.0};  // elements lane, lane + 32, ... (nab <= 100)
        for (int r = r0; r < r0 + nr; ++r) {
            const JRec R = recs[r];
            if (lane < 3) e_table(R.la, R.lb, 0.5 / R.zeta, R.PA[lane], R.PB[lane], Es[wl][lane]);
            __syncwarp();
            const double *Ex = Es[wl][0], *Ey = Es[wl][1], *Ez = Es[wl][2];
            const double *jp = Jp + R.dq_off;
            for (int e = lane, s = 0; e < nab; e += 32, ++s) {
                const int8_t *c = kCart[ca + e / nb];
                const int8_t *d = kCart[cb + e % nb];
                double x = 0.0;
                for (int p = 0; p < np; ++p)
                    x += etab(Ex, c[0], d[0], kHermR[p][0]) * etab(Ey, c[1], d[1], kHermR[p][1]) *
                         etab(Ez, c[2], d[2], kHermR[p][2]) * jp[p];
                acc[s] += R.pre * x;
            }
            __syncwarp();
        }
        for (int e = lane, s = 0; e < nab; e += 32, ++s) {
            const int i = e / nb, j = e % nb;
            if (R0.ao_a == R0.ao_b && i < j) continue;  // diagonal pair: its lower triangle writes both
            const int x = R0.ao_a + i, y = R0.ao_b + j;
            J[(size_t)x * n_ao + y] = acc[s];
            if (x != y) J[(size_t)y * n_ao + x] = acc[s];
        }
    }
}

using PqLaunch = void (*)(int grid, cudaStream_t st, const JRec *, int, int, int, int, int, int, const double4 *,
                          const int *, const double *, const double *, double *, double, double, const double *);

template <int L>
void pq_launch(int grid, cudaStream_t st, const JRec *recs, int lp, int lq, int bra0, int nbra, int ket0, int nket,
               const double4 *kst, const int *kdq, const double *skey, const double *Dq, double *Jp, double tau,
               double thr32, const double *boys) {
    j_pq_kernel<L><<<grid, 128, 0, st>>>(recs, lp, lq, bra0, nbra, ket0, nket, kst, kdq, skey, Dq, Jp, tau, thr32,
                                         boys);
}

template <int... L>
constexpr std::array<PqLaunch, sizeof...(L)> pq_table(std::integer_sequence<int, L...>) {
    return {&pq_launch<L>...};
}
const auto kPqTable = pq_table(std::make_integer_sequence<int, 2 * kJMaxL + 1>{});

using PqSmallLaunch = void (*)(int grid, cudaStream_t st, const JRec *, int, int, int, int, const double4 *,
                               const int *, const double *, const double *, double *, double, double,
                               const double *);

template <int LP, int LQ>
void pq_small_launch(int grid, cudaStream_t st, const JRec *recs, int bra0, int nbra, int ket0, int nket,
                     const double4 *kst, const int *kdq, const double *skey, const double *Dq, double *Jp, double tau,
                     double thr32, const double *boys) {
    if constexpr (LP + LQ <= kSmallL)
        j_pq_small_kernel<LP, LQ><<<grid, 128, 0, st>>>(recs, bra0, nbra, ket0, nket, kst, kdq, skey, Dq, Jp,
                                                        tau, thr32, boys);
}

template <int LP, int... LQ>
constexpr std::array<PqSmallLaunch, sizeof...(LQ)> pq_small_row(std::integer_sequence<int, LQ...>) {
    return {&pq_small_launch<LP, LQ>...};
}
template <int... LP>
constexpr std::array<std::array<PqSmallLaunch, kJMaxL + 1>, sizeof...(LP)> pq_small_table(
    std::integer_sequence<int, LP...>) {
    return {pq_small_row<LP>(std::make_integer_sequence<int, kJMaxL + 1>{})...};
}
const auto kPqSmall = pq_small_table(std::make_integer_sequence<int, kJMaxL + 1>{});

template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    ~DBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t count) {
        if (p) cudaFree(p);
        p = nullptr;
        n = count;
        return count ? cudaMalloc(&p, count * sizeof(T)) : cudaSuccess;
    }
    cudaError_t upload(const std::vector<T> &v) {
        cudaError_t e = alloc(v.size());
        if (e != cudaSuccess || v.empty()) return e;
        return cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    }
};

// The sweep's records of one ordered shell pair (a, b), i outer
// (ao/pairs.py:249-267), with I_pair = fsum_p I_p (ao/pairs.py:299-301).
void pair_records(const HostBasis &B, int a, int b, std::vector<JRec> *out, std::vector<int> *prim) {
    const HostShell &sa = B.shells[a], &sb = B.shells[b];
    const int L = sa.l + sb.l;
    const auto hs = herm_order(L);
    std::vector<double> I(hs.size());
    for (size_t i = 0; i < sa.exps.size(); ++i)
        for (size_t j = 0; j < sb.exps.size(); ++j) {
            const double alpha = sa.exps[i], beta = sb.exps[j], zeta = alpha + beta;
            JRec r{};
            double ex = 1.0;
            for (int d = 0; d < 3; ++d) {
                r.P[d] = (alpha * sa.centre[d] + beta * sb.centre[d]) / zeta;
                r.PA[d] = r.P[d] - sa.centre[d];
                r.PB[d] = r.P[d] - sb.centre[d];
                ex *= std::exp(zeta * r.PA[d] * r.PB[d]);  // e_axis's E^{00}_0 per axis
            }
            r.zeta = zeta;
            r.pre = sa.coefs[i] * sb.coefs[j] * std::pow(M_PI / zeta, 1.5) * ex;
            hermite_bounds(zeta, L, hs, I.data());
            r.G = fsum(I.data(), I.size());
            r.la = sa.l;
            r.lb = sb.l;
            r.ao_a = B.offsets[a];
            r.ao_b = B.offsets[b];
            r.L = L;
            out->push_back(r);
            if (prim) prim->push_back((int)(i * sb.exps.size() + j));
        }
}

}  // namespace

struct JEngine {
    int device = 0, n_ao = 0;
    int n_rec = 0, n_pairs = 0;
    std::vector<int> L_off;       // [kJMaxL + 2] record groups by L
    DBuf<JRec> recs;
    DBuf<int> pair_rec0, pair_nrec, seg_off, iota, order, kdq;
    DBuf<double4> kst;
    DBuf<double> Dq, Dqs, Jp, key, skey;
    DBuf<unsigned char> sort_tmp;
    size_t sort_bytes = 0;
};

JEngine *jengine_create(const HostBasis &basis, int device, std::string *err) {
    auto e = std::make_unique<JEngine>();
    e->device = device;
    e->n_ao = basis.n_ao;
    const int nsh = (int)basis.shells.size();
    for (const auto &s : basis.shells)
        if (s.l > kMaxL) {
            *err = "J-engine: l above the compiled maximum";
            return nullptr;
        }
    // the sweep: pairs a >= b, a outer; records grouped by L, stable
    std::vector<std::vector<JRec>> byL(kJMaxL + 1);
    std::vector<std::vector<int>> pairs_byL(kJMaxL + 1);  // first record (within its L group) per pair
    std::vector<std::vector<int>> pairn_byL(kJMaxL + 1);
    for (int a = 0; a < nsh; ++a)
        for (int b = 0; b <= a; ++b) {
            std::vector<JRec> rs;
            pair_records(basis, a, b, &rs, nullptr);
            const int L = rs[0].L;
            pairs_byL[L].push_back((int)byL[L].size());
            pairn_byL[L].push_back((int)rs.size());
            for (auto &r : rs) byL[L].push_back(r);
        }
    std::vector<JRec> all;
    std::vector<int> p0, pn;
    e->L_off.assign(kJMaxL + 2, 0);
    int dq = 0;
    for (int L = 0; L <= kJMaxL; ++L) {
        e->L_off[L] = (int)all.size();
        for (size_t k = 0; k < pairs_byL[L].size(); ++k) {
            p0.push_back(e->L_off[L] + pairs_byL[L][k]);  // group-relative start, shifted
            pn.push_back(pairn_byL[L][k]);
        }
        for (auto &r : byL[L]) {
            r.dq_off = dq;
            dq += nh(L);
            all.push_back(r);
        }
    }
    e->L_off[kJMaxL + 1] = (int)all.size();
    e->n_rec = (int)all.size();
    e->n_pairs = (int)p0.size();
    if (cudaSetDevice(device) != cudaSuccess) {
        *err = "cudaSetDevice failed";
        return nullptr;
    }
    std::vector<int8_t> herm;
    for (const auto &h : herm_order(2 * kJMaxL))
        for (int d = 0; d < 3; ++d) herm.push_back((int8_t)h[d]);
    std::vector<int> io(e->n_rec);
    std::iota(io.begin(), io.end(), 0);
    cudaError_t ce = cudaMemcpyToSymbol(kHermR, herm.data(), herm.size());
    if (ce == cudaSuccess) ce = e->recs.upload(all);
    if (ce == cudaSuccess) ce = e->pair_rec0.upload(p0);
    if (ce == cudaSuccess) ce = e->pair_nrec.upload(pn);
    if (ce == cudaSuccess) ce = e->seg_off.upload(e->L_off);
    if (ce == cudaSuccess) ce = e->iota.upload(io);
    if (ce == cudaSuccess) ce = e->order.alloc(e->n_rec);
    if (ce == cudaSuccess) ce = e->kdq.alloc(std::max(e->n_rec, 1));
    if (ce == cudaSuccess) ce = e->kst.alloc(std::max(e->n_rec, 1));
    if (ce == cudaSuccess) ce = e->Dq.alloc(std::max(dq, 1));
    if (ce == cudaSuccess) ce = e->Dqs.alloc(std::max(dq, 1));
    if (ce == cudaSuccess) ce = e->Jp.alloc(std::max(dq, 1));
    if (ce == cudaSuccess) ce = e->key.alloc(std::max(e->n_rec, 1));
    if (ce == cudaSuccess) ce = e->skey.alloc(std::max(e->n_rec, 1));
    if (ce == cudaSuccess)
        ce = cub::DeviceSegmentedRadixSort::SortPairsDescending(
            nullptr, e->sort_bytes, e->key.p, e->skey.p, e->iota.p, e->order.p, e->n_rec, kJMaxL + 1,
            e->seg_off.p, e->seg_off.p + 1);
    if (ce == cudaSuccess) ce = e->sort_tmp.alloc(std::max<size_t>(e->sort_bytes, 1));
    if (ce != cudaSuccess) {
        *err = std::string("J-engine setup: ") + cudaGetErrorString(ce);
        return nullptr;
    }
    return e.release();
}

void jengine_destroy(JEngine *e) { delete e; }

int jengine_build(JEngine *e, const double *D_dev, double *J_dev, double tau, double thr32, const double *boys_tab,
                  cudaStream_t st, std::string *err, int *launches) {
    int nl = 0;
    auto check = [&](cudaError_t c, const char *what) {
        if (c == cudaSuccess) return true;
        *err = std::string(what) + ": " + cudaGetErrorString(c);
        return false;
    };
    if (!check(cudaSetDevice(e->device), "cudaSetDevice")) return -2;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
    const int rec_grid = std::max(1, std::min((e->n_rec + 3) / 4, sms * 16));
    j_dq_kernel<<<rec_grid, 128, 0, st>>>(e->recs.p, e->n_rec, D_dev, e->n_ao, e->Dq.p, e->key.p);
    ++nl;
    if (!check(cudaGetLastError(), "j_dq_kernel")) return -2;
    size_t bytes = e->sort_bytes;
    if (!check(cub::DeviceSegmentedRadixSort::SortPairsDescending(e->sort_tmp.p, bytes, e->key.p, e->skey.p,
                                                                  e->iota.p, e->order.p, e->n_rec, kJMaxL + 1,
                                                                  e->seg_off.p, e->seg_off.p + 1, 0,
                                                                  (int)sizeof(double) * 8, st),
               "segmented sort"))
        return -2;
    ++nl;
    j_gather_kernel<<<rec_grid, 128, 0, st>>>(e->recs.p, e->order.p, e->n_rec, e->Dq.p, e->kst.p, e->kdq.p, e->Dqs.p);
    ++nl;
    if (!check(cudaGetLastError(), "j_gather_kernel")) return -2;
    if (!check(cudaMemsetAsync(e->Jp.p, 0, e->Jp.n * sizeof(double), st), "memset")) return -2;
    for (int lp = 0; lp <= kJMaxL; ++lp) {
        const int b0 = e->L_off[lp], nb = e->L_off[lp + 1] - b0;
        if (nb == 0) continue;
        const int grid = std::max(1, std::min((nb + 3) / 4, sms * 8));
        for (int lq = 0; lq <= kJMaxL; ++lq) {
            const int k0 = e->L_off[lq], nk = e->L_off[lq + 1] - k0;
            if (nk == 0) continue;
            if (lp + lq <= kSmallL)
                kPqSmall[lp][lq](grid, st, e->recs.p, b0, nb, k0, nk, e->kst.p, e->kdq.p, e->skey.p, e->Dqs.p, e->Jp.p, tau,
                                 thr32, boys_tab);
            else
                kPqTable[lp + lq](grid, st, e->recs.p, lp, lq, b0, nb, k0, nk, e->kst.p, e->kdq.p, e->skey.p, e->Dqs.p,
                                  e->Jp.p, tau, thr32, boys_tab);
            ++nl;
            if (!check(cudaGetLastError(), "j_pq_kernel")) return -2;
        }
    }
    const int pair_grid = std::max(1, std::min((e->n_pairs + 3) / 4, sms * 16));
    j_jab_kernel<<<pair_grid, 128, 0, st>>>(e->recs.p, e->pair_rec0.p, e->pair_nrec.p, e->n_pairs, e->Jp.p, J_dev,
                                            e->n_ao);
    ++nl;
    if (!check(cudaGetLastError(), "j_jab_kernel")) return -2;
    if (launches) *launches = nl;
    return 0;
}

void jengine_host_lists(const HostBasis &basis, const double *D, JHostLists *out) {
    *out = JHostLists{};
    const int nsh = (int)basis.shells.size();
    const int n = basis.n_ao;
    for (int a = 0; a < nsh; ++a)
        for (int b = 0; b <= a; ++b) {
            const HostShell &sa = basis.shells[a], &sb = basis.shells[b];
            const int L = sa.l + sb.l;
            const auto hs = herm_order(L);
            const auto ca = carts(sa.l), cb = carts(sb.l);
            std::vector<JRec> rs;
            std::vector<int> prim;
            pair_records(basis, a, b, &rs, &prim);
            const double w = a == b ? 1.0 : 2.0;
            for (size_t k = 0; k < rs.size(); ++k) {
                const size_t i = k / sb.exps.size(), j = k % sb.exps.size();
                const double alpha = sa.exps[i], beta = sb.exps[j], zeta = alpha + beta;
                const double scale = sa.coefs[i] * sb.coefs[j] * std::pow(M_PI / zeta, 1.5);
                double P[3];
                for (int d = 0; d < 3; ++d) P[d] = (alpha * sa.centre[d] + beta * sb.centre[d]) / zeta;
                // D_q in make_kets' order (ao/density.py:133-141): rows of
                // the dressed block (c outer), skipping D_cd == 0, then w.
                std::vector<double> dq(hs.size(), 0.0);
                int row = 0;
                for (auto &c : ca)
                    for (auto &d : cb) {
                        const double x = D[(size_t)(basis.offsets[a] + row / (int)cb.size()) * n +
                                           basis.offsets[b] + row % (int)cb.size()];
                        ++row;
                        if (x == 0.0) continue;
                        double ax[3][16];
                        int len[3];
                        for (int dd = 0; dd < 3; ++dd) {
                            e_axis(c[dd], d[dd], zeta, P[dd] - sa.centre[dd], P[dd] - sb.centre[dd], ax[dd]);
                            len[dd] = c[dd] + d[dd] + 1;
                        }
                        for (size_t t = 0; t < hs.size(); ++t) {
                            double v = 1.0;
                            for (int dd = 0; dd < 3; ++dd) v = hs[t][dd] < len[dd] ? v * ax[dd][hs[t][dd]] : 0.0;
                            dq[t] += x * (scale * v);
                        }
                    }
                double dmax = 0.0;
                for (auto &v : dq) dmax = std::max(dmax, std::fabs(w * v));
                out->a.push_back(a);
                out->b.push_back(b);
                out->prim.push_back(prim[k]);
                out->L.push_back(L);
                out->G.push_back(rs[k].G);
                out->key.push_back(rs[k].G * dmax);
            }
        }
    out->L_off.assign(kJMaxL + 2, 0);
    for (int L = 0; L <= kJMaxL; ++L) {
        out->L_off[L] = (int64_t)out->ket_order.size();
        std::vector<int32_t> idx;
        for (size_t r = 0; r < out->L.size(); ++r)
            if (out->L[r] == L) idx.push_back((int32_t)r);
        std::stable_sort(idx.begin(), idx.end(),
                         [&](int32_t x, int32_t y) { return out->key[x] > out->key[y]; });
        out->ket_order.insert(out->ket_order.end(), idx.begin(), idx.end());
    }
    out->L_off[kJMaxL + 1] = (int64_t)out->ket_order.size();
}

}  // namespace fjb
