// rys_fock.cuh -- the class-templated Rys Fock kernel (the large classes).
//
// rys_fock_kernel<LA, LB, LC, LD, R, NT>: one CTA per work unit (a bra shell
// pair and up to 32 of its ket pairs), the unit's computed kets taken G at
// a time.  Per group of kets:
//
//   A  tables: per (ket, primitive quartet, root) one thread evaluates the
//      n-point Rys rule at T (rys_rule.h: a Chebyshev table lookup, n =
//      (LA+LB+LC+LD)/2 + 1) and the three axes' Rys-Dupuis-King 2D integrals
//      I_d(i, k), i <= LA+LB, k <= LC+LD (rys_vrr.h), the root's weight and
//      the quartet's seed U_P U_Q (2/sqrt(pi)) sqrt(rho) folded into the z
//      axis; the tables go to shared memory, a chunk of primitive quartets
//      at a time.
//   B  boundary: per (ket, f) one thread, f a ket Cartesian with
//      LC <= |f| <= LC+LD, holds the bra boundary column [e0|f0] for every
//      e with LA <= |e| <= LA+LB in registers and accumulates over the
//      ket's primitive quartets and roots: per (quartet, root) it reads the
//      3 (LA+LB+1) table entries of its f (shared by the threads of equal
//      f components: broadcast reads), forms the products I_x I_y once per
//      (e_x, e_y) and adds I_x I_y I_z to each e -- no recurrence levels,
//      no barriers inside the chunk.
//   C  bra HRR, from the same registers: X[ab][f] = sum_k C(b,k) AB^(b-k)
//      [a+k, 0|f] (the binomial form of the transfer, hgp_tables.cpp),
//      written to shared memory.
//   D  ket HRR: per (ket, ab) one thread, Y[ab][cd] = sum_k C(d,k)
//      CD^(d-k) X[ab][c+k].
//   E  the six-block digest in FP64 (kernel_f.py:94-131): per output
//      element of the five ket-dependent blocks one thread and one FP64
//      atomic add into J' or K'; the bra block summed over the group's kets
//      in shared memory and added once per unit.
//
// This is the reference's third engine (rys/, eri/fock/kernel_frys.py:194)
// as the VRR of the fused HGP build: the boundary is the same set of values
// the HGP VRR produces, so the HRR and digest are the build's own.  Every
// loop over Cartesians is a compile-time constant of the class.  R = double
// is the plain FP64 path; R = float the routed path's FP32 tier (the rule
// from an FP32 copy of its table, the tables, boundary and HRR in FP32; T,
// the pair scalars, densities and every J/K accumulation FP64).
#pragma once
#include <cuda_runtime.h>

#include "fjb_internal.h"
#include "fock_kernels.cuh"
#include "rys_rule.h"

// The classes the Rys kernel takes: in FP64 every class whose HGP program
// does not fit the register path (the shared-memory interpreter's classes),
// in FP32 every class without an FP32 register body.
#define FJB_RYS64_CLASSES(X)                                                                            \
    X(0, 1, 2, 3) X(0, 1, 3, 3) X(0, 2, 1, 3) X(0, 2, 2, 2) X(0, 2, 2, 3) X(0, 2, 3, 3) X(0, 3, 0, 3)    \
    X(0, 3, 1, 2) X(0, 3, 1, 3) X(0, 3, 2, 2) X(0, 3, 2, 3) X(0, 3, 3, 3) X(1, 1, 1, 3) X(1, 1, 2, 2)    \
    X(1, 1, 2, 3) X(1, 1, 3, 3) X(1, 2, 1, 2) X(1, 2, 1, 3) X(1, 2, 2, 2) X(1, 2, 2, 3) X(1, 2, 3, 3)    \
    X(1, 3, 1, 3) X(1, 3, 2, 2) X(1, 3, 2, 3) X(1, 3, 3, 3) X(2, 2, 2, 2) X(2, 2, 2, 3) X(2, 2, 3, 3)    \
    X(2, 3, 2, 3) X(2, 3, 3, 3) X(3, 3, 3, 3)
// Classes the register kernel also has in FP64, where the Rys kernel can
// take them instead (fjb_set_rys mode 2, and the classes rys_preferred names)
#define FJB_RYS64_EXTRA_CLASSES(X)                                                                      \
    X(0, 0, 0, 1) X(0, 1, 0, 1) X(0, 1, 0, 2) X(0, 1, 0, 3) X(0, 1, 1, 1) X(0, 1, 1, 2) X(0, 1, 1, 3)    \
    X(0, 1, 2, 2) X(0, 2, 0, 3) X(0, 2, 1, 1) X(0, 2, 1, 2) X(0, 3, 1, 1) X(1, 1, 1, 2)
#define FJB_RYS32_CLASSES(X)                                                                            \
    X(0, 2, 2, 3) X(0, 2, 3, 3) X(0, 3, 1, 3) X(0, 3, 2, 2) X(0, 3, 2, 3) X(0, 3, 3, 3) X(1, 1, 2, 3)    \
    X(1, 1, 3, 3) X(1, 2, 1, 3) X(1, 2, 2, 2) X(1, 2, 2, 3) X(1, 2, 3, 3) X(1, 3, 1, 3) X(1, 3, 2, 2)    \
    X(1, 3, 2, 3) X(1, 3, 3, 3) X(2, 2, 2, 2) X(2, 2, 2, 3) X(2, 2, 3, 3) X(2, 3, 2, 3) X(2, 3, 3, 3)    \
    X(3, 3, 3, 3)

namespace fjb {


// host side (rys_fock.cu)
bool rys_available(int la, int lb, int lc, int ld, bool fp32);
// FP64 classes that have a register-path body too: whether the Rys kernel
// is the faster of the two (measured on the 64-atom cluster)
bool rys_extra(int la, int lb, int lc, int ld);
bool rys_preferred(int la, int lb, int lc, int ld);
// The carve-up of a class's kernel for bra and ket degrees up to max_kab,
// max_kcd within `budget` doubles of shared memory: kets per group G from
// the CTA width, then the largest table chunk that fits.  false if none.
bool rys_layout(int la, int lb, int lc, int ld, int max_kab, int max_kcd, bool fp32, int budget, RysDev *out);
int rys_blocks_per_sm(int la, int lb, int lc, int ld, bool fp32, const RysDev &d);
cudaError_t rys_launch(int la, int lb, int lc, int ld, bool fp32, int grid, cudaStream_t st, const KArgs &a);

namespace rys {

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int nrange(int lo, int hi) {
    int n = 0;
    for (int l = lo; l <= hi; ++l) n += ncart(l);
    return n;
}
__host__ __device__ constexpr int binom(int n, int k) {
    int r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

// The Cartesians of levels LO..HI in cartesians(l) order (x descending, then
// y descending), level by level: the boundary's index order.
// idx[i][j][k] is the position of Cartesian (i, j, k) (-1 outside the set).
template <int LO, int HI>
struct CSet {
    static constexpr int N = nrange(LO, HI);
    int x[N], y[N], z[N];
    int idx[HI + 1][HI + 1][HI + 1];
    __host__ __device__ constexpr CSet() : x(), y(), z(), idx() {
        for (int i = 0; i <= HI; ++i)
            for (int j = 0; j <= HI; ++j)
                for (int k = 0; k <= HI; ++k) idx[i][j][k] = -1;
        int n = 0;
        for (int l = LO; l <= HI; ++l)
            for (int i = l; i >= 0; --i)
                for (int j = l - i; j >= 0; --j) {
                    x[n] = i;
                    y[n] = j;
                    z[n] = l - i - j;
                    idx[i][j][l - i - j] = n;
                    ++n;
                }
    }
};

// HRR coefficients of one side (the second shell's l = LY): for b in
// cartesians(LY) and k <= b componentwise, C(b,k) SEP^(b-k); entry
// off[b] + (k_x (b_y+1) + k_y)(b_z+1) + k_z.
template <int LY>
struct HCoefs {
    static constexpr int NB = ncart(LY);
    int off[NB + 1];
    __host__ __device__ constexpr HCoefs() : off() {
        constexpr CSet<LY, LY> c{};
        off[0] = 0;
        for (int b = 0; b < NB; ++b) off[b + 1] = off[b] + (c.x[b] + 1) * (c.y[b] + 1) * (c.z[b] + 1);
    }
    static constexpr int total() {
        constexpr CSet<LY, LY> c{};
        int n = 0;
        for (int b = 0; b < NB; ++b) n += (c.x[b] + 1) * (c.y[b] + 1) * (c.z[b] + 1);
        return n;
    }
};

// The tables as device constants: every access below has a compile-time
// index once the loops are unrolled, so each folds to an immediate.
template <int LO, int HI>
__device__ constexpr CSet<LO, HI> kCart{};
template <int LY>
__device__ constexpr HCoefs<LY> kHCo{};

template <int LA, int LB, int LC, int LD>
struct Shape {
    static constexpr int E = LA + LB, F = LC + LD;
    static constexpr int NR = (E + F) / 2 + 1;  // Rys roots
    static constexpr int TS = (E + 1) * (F + 1);  // one axis' 2D table
    // the tables as stored: per axis F+1 rows (ket index k), each the E+1
    // values of the bra index padded to whole 16-byte vectors (rp); rows
    // rps apart, an odd number of 16-byte vectors, so that the rows of
    // up to eight different k fall in different banks
    template <typename R>
    __host__ __device__ static constexpr int rp() {
        return ((E + 1) * (int)sizeof(R) + 15) / 16 * 16 / (int)sizeof(R);
    }
    template <typename R>
    __host__ __device__ static constexpr int rps() {
        return ((((E + 1) * (int)sizeof(R) + 15) / 16) | 1) * 16 / (int)sizeof(R);
    }
    template <typename R>
    __host__ __device__ static constexpr int tsp() {
        return (F + 1) * rps<R>();
    }
    // one ket's tables for a chunk of P primitive quartets, padded to an odd
    // number of 16-byte vectors so that different kets' rows do not share
    // banks
    template <typename R>
    __host__ __device__ static constexpr int kstride(int P) {
        return P * NR * 3 * tsp<R>() + (((P * NR * 3 * tsp<R>() * (int)sizeof(R) / 16) & 1) ? 0 : 16 / (int)sizeof(R));
    }
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NAB = NA * NB, NCD = NC * ND;
    static constexpr int NBE = nrange(LA, E), NBF = nrange(LC, F);
    static constexpr int NCB = HCoefs<LB>::total(), NCK = HCoefs<LD>::total();
    static constexpr int XS = NBF | 1;  // X row stride, odd: rows start in different banks
    static constexpr int YS = NCD | 1;
    static constexpr int N5 = NCD + NA * NC + NA * ND + NB * NC + NB * ND;
    // CTAs an SM at CTA width t: 512 threads an SM, halved when the bra
    // column the boundary phase keeps in registers is too long for the
    // registers that leaves (df and ff bras in FP64, the ff bra in FP32); a
    // bra column of at most 80 bytes (10 FP64 or 20 FP32 boundary values)
    // fits six CTAs of 128 threads at 80 registers, with no more than a few
    // dozen bytes of spill
    template <typename R>
    __host__ __device__ static constexpr int minb_at(int t) {
        if (t == 128 && NBE * (int)sizeof(R) <= 80) return 6;
        const int m = (512 / t) / (NBE > (sizeof(R) == 8 ? 34 : 52) ? 2 : 1);
        return m > 0 ? m : 1;
    }
    // CTA width: a thread per (ket, f) item, G = NT / NBF kets a group (at
    // most kKetChunk).  128, but 160 for the 52-value kets (3 x 52 of 160
    // threads busy, not 2 x 52 of 128) where that keeps more of them busy
    // on an SM (not when the bra is short enough for six CTAs of 128, or so
    // long that one of 160 fits), and 224 for the 74-value ff kets (3 x 74;
    // 256 left 34 idle).  Measured on the 64-atom cluster: 256-wide CTAs on
    // the 19- to 34-value kets, two an SM, ran 7-21 ms a class slower than
    // four of 128.
    template <typename R>
    __host__ __device__ static constexpr int nt() {
        if (NBF > 64) return 224;
        const bool wide = NBF > 40 && minb_at<R>(160) * (160 / NBF) > minb_at<R>(128) * (128 / NBF);
        return wide ? 160 : 128;
    }
    template <typename R>
    __host__ __device__ static constexpr int minb() {
        return minb_at<R>(nt<R>());
    }
};

// Dynamic shared memory of one CTA (doubles) when `minb` CTAs share an SM:
// its share of the SM's 228 KiB less the 1 KiB the hardware reserves per CTA
// and the kernel's static arrays (below 3 KiB).
__host__ __device__ constexpr int rys_smem_budget(int minb) {
    return minb <= 1 ? kSmemBudgetDoubles : (233472 / minb - 1024 - 3072) / 8;
}

// One root of the n-point rule at T (rys_rule, one root's two series).
template <int N>
__device__ __forceinline__ void rule_root(int r, double T, const double *__restrict__ tab, double *x, double *w) {
    if (T < kRysTSwitch) {
        int i = (int)T;
        if (i > kRysNI - 1) i = kRysNI - 1;
        const double u = 2.0 * (T - (double)i) - 1.0;  // kRysWidth = 1
        const double *blk = tab + ((size_t)(N - 1) * kRysNI + i) * kRysBlock + (size_t)(2 * r) * (kRysDeg + 1);
        double bx1 = 0.0, bx2 = 0.0, bw1 = 0.0, bw2 = 0.0;
        const double u2 = 2.0 * u;
#pragma unroll
        for (int k = kRysDeg; k >= 1; --k) {
            const double bx0 = u2 * bx1 - bx2 + __ldg(blk + k);
            const double bw0 = u2 * bw1 - bw2 + __ldg(blk + kRysDeg + 1 + k);
            bx2 = bx1;
            bx1 = bx0;
            bw2 = bw1;
            bw1 = bw0;
        }
        *x = u * bx1 - bx2 + __ldg(blk);
        *w = u * bw1 - bw2 + __ldg(blk + kRysDeg + 1);
    } else {
        const double *a = tab + kRysAsym + (size_t)(N - 1) * kRysMaxN * 2;
        *x = __ldg(a + 2 * r) / T;
        *w = __ldg(a + 2 * r + 1) * (0.5 / sqrt(T));
    }
}

// The same root in FP32 from the table's FP32 copy (the routed path's FP32
// tier): the interval and its local coordinate from T in FP64, the series
// in FP32 (relative error about 1e-6, inside the tier's own).
template <int N>
__device__ __forceinline__ void rule_root_f(int r, double T, const float *__restrict__ tab, float *x, float *w) {
    if (T < kRysTSwitch) {
        int i = (int)T;
        if (i > kRysNI - 1) i = kRysNI - 1;
        const float u = (float)(2.0 * (T - (double)i) - 1.0);
        const float *blk = tab + ((size_t)(N - 1) * kRysNI + i) * kRysBlock + (size_t)(2 * r) * (kRysDeg + 1);
        float bx1 = 0.f, bx2 = 0.f, bw1 = 0.f, bw2 = 0.f;
        const float u2 = 2.f * u;
#pragma unroll
        for (int k = kRysDeg; k >= 1; --k) {
            const float bx0 = u2 * bx1 - bx2 + __ldg(blk + k);
            const float bw0 = u2 * bw1 - bw2 + __ldg(blk + kRysDeg + 1 + k);
            bx2 = bx1;
            bx1 = bx0;
            bw2 = bw1;
            bw1 = bw0;
        }
        *x = u * bx1 - bx2 + __ldg(blk);
        *w = u * bw1 - bw2 + __ldg(blk + kRysDeg + 1);
    } else {
        const float *a = tab + kRysAsym + (size_t)(N - 1) * kRysMaxN * 2;
        *x = (float)(__ldg(a + 2 * r) / T);
        *w = (float)(__ldg(a + 2 * r + 1) * (0.5 / sqrt(T)));
    }
}

// The HRR coefficient `idx` of side LY for separation sep (= A - B or C - D).
template <int LY, typename R>
__device__ __forceinline__ R hrr_coef(int idx, const double *sep) {
    constexpr const HCoefs<LY> &H = kHCo<LY>;
    constexpr const CSet<LY, LY> &c = kCart<LY, LY>;
    int b = 0;
#pragma unroll
    for (int j = 1; j < HCoefs<LY>::NB; ++j)
        if (idx >= H.off[j]) b = j;
    int bx = 0, by = 0, bz = 0;
#pragma unroll
    for (int j = 0; j < HCoefs<LY>::NB; ++j)
        if (j == b) {
            bx = c.x[j];
            by = c.y[j];
            bz = c.z[j];
        }
    const int rem = idx - H.off[b];
    const int kz = rem % (bz + 1), ky = (rem / (bz + 1)) % (by + 1), kx = rem / ((bz + 1) * (by + 1));
    const double v = (double)(binom(bx, kx) * binom(by, ky) * binom(bz, kz)) * ipow(sep[0], bx - kx) *
                     ipow(sep[1], by - ky) * ipow(sep[2], bz - kz);
    return (R)v;
}


// N values of R from a 16-byte aligned shared-memory row, as 16-byte loads.
template <typename R, int N>
__device__ __forceinline__ void ld_row(const R *p, R *out) {
    static_assert(N * sizeof(R) % 16 == 0, "whole 16-byte vectors");
#pragma unroll
    for (int v = 0; v < N * (int)sizeof(R) / 16; ++v) {
        const float4 t = reinterpret_cast<const float4 *>(p)[v];
        memcpy(out + v * (16 / (int)sizeof(R)), &t, 16);
    }
}

// The position of Cartesian index t of cartesians-range LO..HI as (x, y, z),
// for a run-time index (the thread's own f).
template <int LO, int HI>
__device__ __forceinline__ void cart_of(int t, int *x, int *y, int *z) {
    int l = LO;
#pragma unroll
    for (int m = LO; m < HI; ++m)
        if (t >= ncart(m)) {
            t -= ncart(m);
            l = m + 1;
        } else {
            break;
        }
    int i = l;
    while (t > l - i) {
        t -= l - i + 1;
        --i;
    }
    *x = i;
    *y = l - i - t;
    *z = t;
}

}  // namespace rys

template <int LA, int LB, int LC, int LD, typename R, int NT>
__global__ void __launch_bounds__(NT, (rys::Shape<LA, LB, LC, LD>::template minb<R>()))
    rys_fock_kernel(const KArgs A) {
    using S = rys::Shape<LA, LB, LC, LD>;
    constexpr int E = S::E, F = S::F, NR = S::NR;
    constexpr int RP = S::template rp<R>(), RPS = S::template rps<R>(), TSP = S::template tsp<R>();
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND, NAB = S::NAB, NCD = S::NCD;
    constexpr int NBE = S::NBE, NBF = S::NBF, NCB = S::NCB, NCK = S::NCK, XS = S::XS, YS = S::YS;
    constexpr int N5 = S::N5;
    constexpr const rys::CSet<LA, E> &es = rys::kCart<LA, E>;
    constexpr const rys::CSet<LC, F> &fs = rys::kCart<LC, F>;
    constexpr const rys::CSet<LA, LA> &ca = rys::kCart<LA, LA>;
    constexpr const rys::CSet<LB, LB> &cbs = rys::kCart<LB, LB>;
    constexpr const rys::CSet<LC, LC> &cc = rys::kCart<LC, LC>;
    constexpr const rys::CSet<LD, LD> &cds = rys::kCart<LD, LD>;
    constexpr const rys::CSet<0, LD> &ks = rys::kCart<0, LD>;  // ket transfer shifts k, |k| <= LD
    constexpr const rys::HCoefs<LB> &hb = rys::kHCo<LB>;
    constexpr const rys::HCoefs<LD> &hd = rys::kHCo<LD>;
    constexpr double kTwoOverSqrtPi = 1.1283791670955126;

    extern __shared__ __align__(16) double sm[];
    __shared__ int s_ket[kKetChunk];
    __shared__ PairRec s_pair[kKetChunk];  // the unit's computed kets, in ket order
    __shared__ int s_oc[kKetChunk], s_od[kKetChunk];
    __shared__ double s_deg[kKetChunk];
    __shared__ int s_n;
    const RysDev &L = A.Y;
    double *braP = sm + L.sm_braP;
    R *cb = reinterpret_cast<R *>(sm + L.sm_cb);
    double *Dab = sm + L.sm_Dab;
    double *Jab = sm + L.sm_Jab;
    double *ketP = sm + L.sm_ketP;
    R *ck = reinterpret_cast<R *>(sm + L.sm_ck);
    double *Dk = sm + L.sm_Dk;
    R *tab = reinterpret_cast<R *>(sm + L.sm_tab);
    R *Ym = tab;  // the ket HRR's output reuses the tables' region
    R *X = reinterpret_cast<R *>(sm + L.sm_X);
    const int tid = threadIdx.x;
    const int G = L.group, P = L.chunk;
    const int KSTR = S::template kstride<R>(P);
    const int n_todo = A.unit_list ? *A.unit_count : A.n_units;

    for (int ui = blockIdx.x; ui < n_todo; ui += gridDim.x) {
        const int u = A.unit_list ? A.unit_list[ui] : ui;
        const Unit U = A.units[u];
        const LaunchRec LR = A.launches[U.launch];
        const PairRec bra = A.pairs[LR.bra_pair0 + U.ib];
        const MolCtx M = mol_of(A, U.launch);
        const int n_ao = M.n_ao;
        const int kab = bra.nprim;
        const int oa = bra.ao_a, ob = bra.ao_b;
        {
            const double *src = reinterpret_cast<const double *>(A.prims + bra.prim0);
            for (int i = tid; i < kab * kPrimWords; i += NT) braP[i] = src[i];
        }
        for (int i = tid; i < NCB; i += NT) cb[i] = rys::hrr_coef<LB, R>(i, bra.AB);
        for (int i = tid; i < NAB; i += NT) {
            Dab[i] = M.D[(size_t)(oa + i / NB) * n_ao + ob + i % NB];
            Jab[i] = 0.0;
        }
        if (tid < 32) {
            const int ik = U.k0 + tid;
            bool on = false;
            if (ik < U.k1) {
                const PairRec ket = A.pairs[LR.ket_pair0 + ik];
                on = !skip6(M.Dsh, M.n_sh, bra.a, bra.b, ket.a, ket.b, bra.G, ket.G, A.tau);
            }
            const unsigned m = __ballot_sync(0xffffffffu, on);
            if (on) {
                const int at = __popc(m & ((1u << tid) - 1u));
                s_ket[at] = ik;
                s_pair[at] = A.pairs[LR.ket_pair0 + ik];
            }
            if (tid == 0) s_n = __popc(m);
        }
        __syncthreads();
        const int n_list = s_n;
        const int kcd = A.pairs[LR.ket_pair0 + U.k0].nprim;  // one degree per ket batch
        const int K = kab * kcd;
        const double bra_deg = bra.a == bra.b ? 0.5 : 1.0;

        for (int g0 = 0; g0 < n_list; g0 += G) {
            const int ng = min(G, n_list - g0);
            // -- the group's kets: primitive pairs, HRR coefficients, densities
            for (int i = tid; i < ng * kcd * kPrimWords; i += NT) {
                const int g = i / (kcd * kPrimWords), r = i - g * (kcd * kPrimWords);
                ketP[i] = reinterpret_cast<const double *>(A.prims + s_pair[g0 + g].prim0)[r];
            }
            for (int i = tid; i < ng * NCK; i += NT) {
                const int g = i / NCK;
                ck[i] = rys::hrr_coef<LD, R>(i - g * NCK, s_pair[g0 + g].AB);
            }
            for (int i = tid; i < ng * N5; i += NT) {
                const int g = i / N5, o = i - g * N5;
                const int oc = s_pair[g0 + g].ao_a, od = s_pair[g0 + g].ao_b;
                size_t at;
                if (o < NCD) {
                    at = (size_t)(oc + o / ND) * n_ao + od + o % ND;
                } else if (o < NCD + NA * NC) {
                    const int r = o - NCD;
                    at = (size_t)(oa + r / NC) * n_ao + oc + r % NC;
                } else if (o < NCD + NA * NC + NA * ND) {
                    const int r = o - NCD - NA * NC;
                    at = (size_t)(oa + r / ND) * n_ao + od + r % ND;
                } else if (o < NCD + NA * NC + NA * ND + NB * NC) {
                    const int r = o - NCD - NA * NC - NA * ND;
                    at = (size_t)(ob + r / NC) * n_ao + oc + r % NC;
                } else {
                    const int r = o - NCD - NA * NC - NA * ND - NB * NC;
                    at = (size_t)(ob + r / ND) * n_ao + od + r % ND;
                }
                Dk[i] = M.D[at];
            }
            if (tid < ng) {
                const int ik = s_ket[g0 + tid];
                const PairRec &ket = s_pair[g0 + tid];
                s_oc[tid] = ket.ao_a;
                s_od[tid] = ket.ao_b;
                s_deg[tid] = bra_deg * (ket.a == ket.b ? 0.5 : 1.0) * ((LR.diag && ik == U.ib) ? 0.5 : 1.0);
            }

            // -- A + B: tables chunk by chunk, the boundary column in registers
            const int gme = tid / NBF, fme = tid - gme * NBF;
            const bool item = gme < ng;
            int fx = 0, fy = 0, fz = 0;
            rys::cart_of<LC, F>(fme, &fx, &fy, &fz);
            R acc[NBE];
#pragma unroll
            for (int e = 0; e < NBE; ++e) acc[e] = (R)0;
            for (int c0 = 0; c0 < K; c0 += P) {
                const int np = min(P, K - c0);
                __syncthreads();  // the previous chunk's tables are read; the staging above is written
                for (int it = tid; it < ng * np * NR; it += NT) {
                    const int g = it / (np * NR), rem = it - g * (np * NR), tl = rem / NR, r = rem - tl * NR;
                    const int t = c0 + tl, ikcd = t / kab, ikab = t - ikcd * kab;
                    const double *pb = braP + kPrimWords * ikab;
                    const double *pk = ketP + kPrimWords * (g * kcd + ikcd);
                    const double p = pb[6], q = pk[6];
                    const double inv = 1.0 / (p + q), rho = p * q * inv;
                    const double qi = q * inv, pi = p * inv;  // rho/p, rho/q
                    const double PQ[3] = {pb[0] - pk[0], pb[1] - pk[1], pb[2] - pk[2]};
                    const double T = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
                    // the rule and the 2D recurrences in R: FP64, or FP32 on
                    // the routed FP32 tier (T and the pair scalars FP64)
                    R x, w;
                    if constexpr (sizeof(R) == 4) {
                        rys::rule_root_f<NR>(r, T, A.rys_tab32, &x, &w);
                    } else {
                        rys::rule_root<NR>(r, T, A.rys_tab, &x, &w);
                    }
                    const R seedw = (R)(pb[7] * pk[7] * kTwoOverSqrtPi * sqrt(rho)) * w;
                    const R b00 = (R)(0.5 * inv) * x, b10 = (R)pb[8] * ((R)1 - (R)qi * x),
                            b01 = (R)pk[8] * ((R)1 - (R)pi * x);
                    R *out = tab + (size_t)g * KSTR + (size_t)(tl * NR + r) * (3 * TSP);
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const R c00 = (R)pb[3 + d] - (R)(qi * PQ[d]) * x, c00p = (R)pk[3 + d] + (R)(pi * PQ[d]) * x;
                        R I[E + 1][F + 1];
                        I[0][0] = d == 2 ? seedw : (R)1;
#pragma unroll
                        for (int i = 0; i < E; ++i)
                            I[i + 1][0] = c00 * I[i][0] + (i ? (R)i * b10 * I[i - 1][0] : (R)0);
#pragma unroll
                        for (int k = 0; k < F; ++k)
#pragma unroll
                            for (int i = 0; i <= E; ++i) {
                                R v = c00p * I[i][k];
                                if (k) v += (R)k * b01 * I[i][k - 1];
                                if (i) v += (R)i * b00 * I[i - 1][k];
                                I[i][k + 1] = v;
                            }
#pragma unroll
                        for (int i = 0; i <= E; ++i)
#pragma unroll
                            for (int k = 0; k <= F; ++k) out[d * TSP + k * RPS + i] = I[i][k];
                    }
                }
                __syncthreads();
                if (item) {
                    for (int tl = 0; tl < np; ++tl) {
                        const R *base = tab + (size_t)gme * KSTR + (size_t)tl * NR * (3 * TSP);
#pragma unroll
                        for (int r = 0; r < NR; ++r) {
                            const R *Ix = base + r * (3 * TSP), *Iy = Ix + TSP, *Iz = Iy + TSP;
                            R ix[RP], iy[RP], iz[RP];
                            rys::ld_row<R, RP>(Ix + fx * RPS, ix);
                            rys::ld_row<R, RP>(Iy + fy * RPS, iy);
                            rys::ld_row<R, RP>(Iz + fz * RPS, iz);
                            R pxy[E + 1][E + 1];
#pragma unroll
                            for (int a = 0; a <= E; ++a)
#pragma unroll
                                for (int b = 0; a + b <= E; ++b) pxy[a][b] = ix[a] * iy[b];
#pragma unroll
                            for (int e = 0; e < NBE; ++e) acc[e] += pxy[es.x[e]][es.y[e]] * iz[es.z[e]];
                        }
                    }
                }
            }

            // -- C: the bra HRR from the registers into X[g][ab][f]
            if (item) {
                R *xr = X + (size_t)gme * NAB * XS + fme;
#pragma unroll
                for (int a = 0; a < NA; ++a)
#pragma unroll
                    for (int b = 0; b < NB; ++b) {
                        R v = (R)0;
                        int ci = hb.off[b];
#pragma unroll
                        for (int kx = 0; kx <= cbs.x[b]; ++kx)
#pragma unroll
                            for (int ky = 0; ky <= cbs.y[b]; ++ky)
#pragma unroll
                                for (int kz = 0; kz <= cbs.z[b]; ++kz, ++ci)
                                    v += cb[ci] * acc[es.idx[ca.x[a] + kx][ca.y[a] + ky][ca.z[a] + kz]];
                        xr[(size_t)(a * NB + b) * XS] = v;
                    }
            }
            __syncthreads();

            // -- D: the ket HRR, Y[g][ab][cd], one (ket, ab, c) per thread
            for (int it = tid; it < ng * NAB * NC; it += NT) {
                const int row = it / NC, c = it - row * NC, g = row / NAB;
                const R *xr = X + (size_t)row * XS;
                R *yr = Ym + (size_t)row * YS + c * ND;
                const R *ckg = ck + g * NCK;
                int cx = 0, cy = 0, cz = 0;
#pragma unroll
                for (int j = 0; j < NC; ++j)
                    if (j == c) {
                        cx = cc.x[j];
                        cy = cc.y[j];
                        cz = cc.z[j];
                    }
                R xk[rys::CSet<0, LD>::N];
#pragma unroll
                for (int k = 0; k < rys::CSet<0, LD>::N; ++k) {
                    // f index of c + k: the level offset of |c + k| plus the
                    // position inside cartesians(|c + k|)
                    const int ix = cx + ks.x[k], iy = cy + ks.y[k], l = LC + ks.x[k] + ks.y[k] + ks.z[k];
                    const int f = rys::nrange(LC, l - 1) + (l - ix) * (l - ix + 1) / 2 + (l - ix - iy);
                    xk[k] = xr[f];
                }
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    R v = (R)0;
                    int ci = hd.off[d];
#pragma unroll
                    for (int kx = 0; kx <= cds.x[d]; ++kx)
#pragma unroll
                        for (int ky = 0; ky <= cds.y[d]; ++ky)
#pragma unroll
                            for (int kz = 0; kz <= cds.z[d]; ++kz, ++ci) v += ckg[ci] * xk[ks.idx[kx][ky][kz]];
                    yr[d] = v;
                }
            }
            __syncthreads();

            // -- E: the six-block digest (FP64)
            for (int it = tid; it < NAB + ng * N5; it += NT) {
                if (it < NAB) {  // the bra block, over the group's kets
                    double s = 0.0;
                    for (int g = 0; g < ng; ++g) {
                        const R *yr = Ym + (size_t)(g * NAB + it) * YS;
                        const double *dcd = Dk + g * N5;
                        double t = 0.0;
#pragma unroll
                        for (int cd = 0; cd < NCD; ++cd) t += dcd[cd] * (double)yr[cd];
                        s += 2.0 * s_deg[g] * t;
                    }
                    Jab[it] += s;
                    continue;
                }
                const int g = (it - NAB) / N5, o = it - NAB - g * N5;
                const R *Y = Ym + (size_t)g * NAB * YS;
                const double *dk = Dk + g * N5;
                const double deg = s_deg[g];
                const int oc = s_oc[g], od = s_od[g];
                double acc2 = 0.0;
                if (o < NCD) {
                    const int c = o / ND, d = o - c * ND;
#pragma unroll
                    for (int ab = 0; ab < NAB; ++ab) acc2 += Dab[ab] * (double)Y[ab * YS + o];
                    atomicAdd(M.Jp + (size_t)(oc + c) * n_ao + od + d, 2.0 * deg * acc2);
                } else if (o < NCD + NA * NC) {
                    const int r = o - NCD, a = r / NC, c = r - a * NC;
                    const double *dbd = dk + NCD + NA * NC + NA * ND + NB * NC;
#pragma unroll
                    for (int b = 0; b < NB; ++b)
#pragma unroll
                        for (int d = 0; d < ND; ++d) acc2 += dbd[b * ND + d] * (double)Y[(a * NB + b) * YS + c * ND + d];
                    atomicAdd(M.Kp + (size_t)(oa + a) * n_ao + oc + c, deg * acc2);
                } else if (o < NCD + NA * NC + NA * ND) {
                    const int r = o - NCD - NA * NC, a = r / ND, d = r - a * ND;
                    const double *dbc = dk + NCD + NA * NC + NA * ND;
#pragma unroll
                    for (int b = 0; b < NB; ++b)
#pragma unroll
                        for (int c = 0; c < NC; ++c) acc2 += dbc[b * NC + c] * (double)Y[(a * NB + b) * YS + c * ND + d];
                    atomicAdd(M.Kp + (size_t)(oa + a) * n_ao + od + d, deg * acc2);
                } else if (o < NCD + NA * NC + NA * ND + NB * NC) {
                    const int r = o - NCD - NA * NC - NA * ND, b = r / NC, c = r - b * NC;
                    const double *dad = dk + NCD + NA * NC;
#pragma unroll
                    for (int a = 0; a < NA; ++a)
#pragma unroll
                        for (int d = 0; d < ND; ++d) acc2 += dad[a * ND + d] * (double)Y[(a * NB + b) * YS + c * ND + d];
                    atomicAdd(M.Kp + (size_t)(ob + b) * n_ao + oc + c, deg * acc2);
                } else {
                    const int r = o - NCD - NA * NC - NA * ND - NB * NC, b = r / ND, d = r - b * ND;
                    const double *dac = dk + NCD;
#pragma unroll
                    for (int a = 0; a < NA; ++a)
#pragma unroll
                        for (int c = 0; c < NC; ++c) acc2 += dac[a * NC + c] * (double)Y[(a * NB + b) * YS + c * ND + d];
                    atomicAdd(M.Kp + (size_t)(ob + b) * n_ao + od + d, deg * acc2);
                }
            }
            __syncthreads();
        }
        for (int i = tid; i < NAB; i += NT)
            if (Jab[i] != 0.0) atomicAdd(M.Jp + (size_t)(oa + i / NB) * n_ao + ob + i % NB, Jab[i]);
        if (A.computed && tid == 0 && n_list) atomicAdd(A.computed + U.launch, (unsigned long long)n_list);
        __syncthreads();
    }
}

// One class's kernel: its shared-memory attribute, occupancy and launch
// (instantiated per precision in rys_fock64.cu and rys_fock32.cu).
template <int LA, int LB, int LC, int LD, typename R>
struct RysOne {
    static constexpr int kRysThreads = rys::Shape<LA, LB, LC, LD>::template nt<R>();
    static void attr() {
        static bool done = false;  // per kernel and process: the largest carve-up any layout takes
        if (done) return;
        cudaFuncSetAttribute(rys_fock_kernel<LA, LB, LC, LD, R, kRysThreads>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBudgetDoubles * (int)sizeof(double));
        done = true;
    }
    static int occupancy(const RysDev &d) {
        attr();
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rys_fock_kernel<LA, LB, LC, LD, R, kRysThreads>,
                                                      kRysThreads, (size_t)d.sm_total * sizeof(double));
        return n;
    }
    static cudaError_t launch(int grid, cudaStream_t st, const KArgs &a) {
        attr();
        rys_fock_kernel<LA, LB, LC, LD, R, kRysThreads>
            <<<grid, kRysThreads, (size_t)a.Y.sm_total * sizeof(double), st>>>(a);
        return cudaGetLastError();
    }
};

}  // namespace fjb
