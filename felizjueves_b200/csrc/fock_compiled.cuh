// fock_compiled.cuh -- the class-templated HGP Fock kernel (register path).
//
// hgp_compiled_kernel<LA, LB, LC, LD, R>: one WARP per work unit (a bra pair
// and up to 32 of its ket pairs), one THREAD per contracted quartet.  The bra
// pair is the same for the whole warp, so its records are broadcast loads.
// Per thread: the six-block screen; then for every primitive quartet the
// scalars and the Boys values in FP64, and the class's VRR program
// (HgpCode<...>::vrr, straight-line, generated from the same programs the
// interpreter kernel runs) in the recurrence type R, accumulating the
// boundary in registers; after the primitive loop the two binomial HRR
// transforms in R; then the six-block digest in FP64 with the reference's
// 8-fold weights and degeneracy (kernel_f.py:94-131): the bra block F_ab is
// reduced across the warp by shuffles and added once per unit, the other
// five blocks are added with FP64 atomics.
//
// R = double is the plain FP64 path.  R = float is the routed path's
// recurrence type: the quartet's scalars, Boys values, density blocks and
// every J/K/G accumulation stay FP64.  The router (route_units_kernel) hands
// the FP32 instantiation only units whose every computed quartet is under
// the routing threshold (G_ab G_cd dmax < threshold, the bound the six-block
// screen uses).
#pragma once
#include <cuda_runtime.h>

#include "fjb_internal.h"
#include "fock_kernels.cuh"

namespace fjb {

constexpr int kVrrTab = 8;  // integer multiples held per VRR coefficient

template <typename R>
struct VrrK {
    R pa[3], wp[3], qc[3], wq[3];
    R cp[kVrrTab], rp[kVrrTab], cq[kVrrTab], rq[kVrrTab], e[kVrrTab];
};

template <int LA, int LB, int LC, int LD>
struct HgpCode {
    static constexpr bool kCompiled = false;
};

__host__ __device__ constexpr int cnc(int l) { return (l + 1) * (l + 2) / 2; }

template <int M>
__device__ __forceinline__ void boys_t(double T, double *F, const double *__restrict__ tab) {
    if (T < kBoysTMax) {
        const int i = __double2int_rn(T * (1.0 / kBoysDelta));
        const double d = (double)i * kBoysDelta - T;
        const double *row0 = tab + (size_t)i * kBoysRow;
        const double *row = row0 + M;
        double f = __ldg(row + 6);
        f = __ldg(row + 5) + f * d * (1.0 / 6.0);
        f = __ldg(row + 4) + f * d * (1.0 / 5.0);
        f = __ldg(row + 3) + f * d * (1.0 / 4.0);
        f = __ldg(row + 2) + f * d * (1.0 / 3.0);
        f = __ldg(row + 1) + f * d * (1.0 / 2.0);
        f = __ldg(row + 0) + f * d;
        F[M] = f;
        if (M > 0) {
            const double e = boys_exp(row0, d), t2 = 2.0 * T;
#pragma unroll
            for (int m = M - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) * (1.0 / (double)(2 * m + 1));
        }
    } else {
        const double e = M > 0 ? exp(-T) : 0.0, h = 0.5 / T;
        F[0] = 0.5 * sqrt(3.141592653589793 / T);
#pragma unroll
        for (int m = 0; m < M; ++m) F[m + 1] = ((double)(2 * m + 1) * F[m] - e) * h;
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The primitive loop, the HRR and the digest of one quartet in recurrence
// type R.  jab[] collects this lane's share of the bra block (FP64).
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void quartet_compiled(const KArgs &A, const MolCtx &M, const PairRec &bra,
                                                 const PairRec &ket, double deg, double *jab, double *wq,
                                                 int wstride) {
    using H = HgpCode<LA, LB, LC, LD>;
    constexpr int NA = cnc(LA), NB = cnc(LB), NC = cnc(LC), ND = cnc(LD);
    constexpr int NAB = NA * NB, NCD = NC * ND, L = LA + LB + LC + LD;
    constexpr double kTwoOverSqrtPi = 1.1283791670955126;
    R acc[H::kNB];
#pragma unroll
    for (int t = 0; t < H::kNB; ++t) acc[t] = (R)0;
    for (int kc = 0; kc < ket.nprim; ++kc) {
        const PrimRec Q = A.prims[ket.prim0 + kc];
        for (int kb = 0; kb < bra.nprim; ++kb) {
            const PrimRec P = A.prims[bra.prim0 + kb];
            const double p = P.zeta, q = Q.zeta;
            const double ppq = p + q, inv = 1.0 / ppq, rho = p * q * inv;
            const double PQx = P.P[0] - Q.P[0], PQy = P.P[1] - Q.P[1], PQz = P.P[2] - Q.P[2];
            const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
            double F[L + 1];
            boys_t<L>(T, F, A.boys_tab);
            const double seed = P.U * Q.U * kTwoOverSqrtPi * sqrt(rho);
            R Fs[L + 1];
#pragma unroll
            for (int m = 0; m <= L; ++m) Fs[m] = (R)(seed * F[m]);
            VrrK<R> k;
            const double wp = -q * inv, wq = p * inv;
            // rho/p = q/(p+q) and rho/q = p/(p+q): no division beyond 1/(p+q)
            const double i2p = P.h, i2q = Q.h, rp = i2p * (q * inv), rq = i2q * (p * inv), e2 = 0.5 * inv;
            k.pa[0] = (R)P.X[0];
            k.pa[1] = (R)P.X[1];
            k.pa[2] = (R)P.X[2];
            k.qc[0] = (R)Q.X[0];
            k.qc[1] = (R)Q.X[1];
            k.qc[2] = (R)Q.X[2];
            k.wp[0] = (R)(wp * PQx);
            k.wp[1] = (R)(wp * PQy);
            k.wp[2] = (R)(wp * PQz);
            k.wq[0] = (R)(wq * PQx);
            k.wq[1] = (R)(wq * PQy);
            k.wq[2] = (R)(wq * PQz);
#pragma unroll
            for (int n = 0; n < kVrrTab; ++n) {
                k.cp[n] = (R)(n * i2p);
                k.rp[n] = (R)(n * rp);
                k.cq[n] = (R)(n * i2q);
                k.rq[n] = (R)(n * rq);
                k.e[n] = (R)(n * e2);
            }
            H::template vrr<R>(Fs, k, acc);
        }
    }
    R cb[H::kNCB], ck[H::kNCK], eri[NAB * NCD];
    H::template coef_bra<R>(bra.AB, cb);
    H::template coef_ket<R>(ket.AB, ck);
    H::template hrr<R>(acc, cb, ck, eri);

    // the six-block digest, FP64
    const int n_ao = M.n_ao;
    const int oa = bra.ao_a, ob = bra.ao_b, oc = ket.ao_a, od = ket.ao_b;
    double dab[NAB], dcd[NCD], dac[NA * NC], dad[NA * ND], dbc[NB * NC], dbd[NB * ND];
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
        for (int j = 0; j < NB; ++j) dab[i * NB + j] = __ldg(M.D + (size_t)(oa + i) * n_ao + ob + j);
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < ND; ++j) dcd[i * ND + j] = __ldg(M.D + (size_t)(oc + i) * n_ao + od + j);
#pragma unroll
    for (int i = 0; i < NA; ++i) {
#pragma unroll
        for (int j = 0; j < NC; ++j) dac[i * NC + j] = __ldg(M.D + (size_t)(oa + i) * n_ao + oc + j);
#pragma unroll
        for (int j = 0; j < ND; ++j) dad[i * ND + j] = __ldg(M.D + (size_t)(oa + i) * n_ao + od + j);
    }
#pragma unroll
    for (int i = 0; i < NB; ++i) {
#pragma unroll
        for (int j = 0; j < NC; ++j) dbc[i * NC + j] = __ldg(M.D + (size_t)(ob + i) * n_ao + oc + j);
#pragma unroll
        for (int j = 0; j < ND; ++j) dbd[i * ND + j] = __ldg(M.D + (size_t)(ob + i) * n_ao + od + j);
    }
    double jcd[NCD], kac[NA * NC], kad[NA * ND], kbc[NB * NC], kbd[NB * ND];
#pragma unroll
    for (int t = 0; t < NCD; ++t) jcd[t] = 0.0;
#pragma unroll
    for (int t = 0; t < NA * NC; ++t) kac[t] = 0.0;
#pragma unroll
    for (int t = 0; t < NA * ND; ++t) kad[t] = 0.0;
#pragma unroll
    for (int t = 0; t < NB * NC; ++t) kbc[t] = 0.0;
#pragma unroll
    for (int t = 0; t < NB * ND; ++t) kbd[t] = 0.0;
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            double sab = 0.0;
#pragma unroll
            for (int kk = 0; kk < NC; ++kk)
#pragma unroll
                for (int l = 0; l < ND; ++l) {
                    const double x = (double)eri[(i * NB + j) * NCD + kk * ND + l];
                    sab += dcd[kk * ND + l] * x;
                    jcd[kk * ND + l] += dab[i * NB + j] * x;
                    kac[i * NC + kk] += dbd[j * ND + l] * x;
                    kad[i * ND + l] += dbc[j * NC + kk] * x;
                    kbc[j * NC + kk] += dad[i * ND + l] * x;
                    kbd[j * ND + l] += dac[i * NC + kk] * x;
                }
            jab[i * NB + j] += 2.0 * deg * sab;
        }
    const double w2 = 2.0 * deg;
    if (wq) {
        // the atomics-free build: each contribution into its own slot
        constexpr int KAC = NCD, KAD = KAC + NA * NC, KBC = KAD + NA * ND, KBD = KBC + NB * NC;
#pragma unroll
        for (int t = 0; t < NCD; ++t) wq[(size_t)t * wstride] = w2 * jcd[t];
#pragma unroll
        for (int t = 0; t < NA * NC; ++t) wq[(size_t)(KAC + t) * wstride] = deg * kac[t];
#pragma unroll
        for (int t = 0; t < NA * ND; ++t) wq[(size_t)(KAD + t) * wstride] = deg * kad[t];
#pragma unroll
        for (int t = 0; t < NB * NC; ++t) wq[(size_t)(KBC + t) * wstride] = deg * kbc[t];
#pragma unroll
        for (int t = 0; t < NB * ND; ++t) wq[(size_t)(KBD + t) * wstride] = deg * kbd[t];
        return;
    }
#pragma unroll
    for (int kk = 0; kk < NC; ++kk)
#pragma unroll
        for (int l = 0; l < ND; ++l) atomicAdd(M.Jp + (size_t)(oc + kk) * n_ao + od + l, w2 * jcd[kk * ND + l]);
#pragma unroll
    for (int i = 0; i < NA; ++i) {
#pragma unroll
        for (int kk = 0; kk < NC; ++kk) atomicAdd(M.Kp + (size_t)(oa + i) * n_ao + oc + kk, deg * kac[i * NC + kk]);
#pragma unroll
        for (int l = 0; l < ND; ++l) atomicAdd(M.Kp + (size_t)(oa + i) * n_ao + od + l, deg * kad[i * ND + l]);
    }
#pragma unroll
    for (int j = 0; j < NB; ++j) {
#pragma unroll
        for (int kk = 0; kk < NC; ++kk) atomicAdd(M.Kp + (size_t)(ob + j) * n_ao + oc + kk, deg * kbc[j * NC + kk]);
#pragma unroll
        for (int l = 0; l < ND; ++l) atomicAdd(M.Kp + (size_t)(ob + j) * n_ao + od + l, deg * kbd[j * ND + l]);
    }
}

// The units a kernel takes: all of them, or the device-side queue the
// precision router filled (A.unit_list, *A.unit_count entries).
__device__ __forceinline__ int units_to_do(const KArgs &A) {
    return A.unit_list ? *A.unit_count : A.n_units;
}
__device__ __forceinline__ int unit_at(const KArgs &A, int i) { return A.unit_list ? A.unit_list[i] : i; }

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128) hgp_compiled_kernel(const KArgs A) {
    constexpr int NA = cnc(LA), NB = cnc(LB), NAB = NA * NB;
    const int lane = threadIdx.x & 31;
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    const int n = units_to_do(A);
    for (int ui = warp; ui < n; ui += nwarps) {
        const int u = unit_at(A, ui);
        const Unit U = A.units[u];
        const LaunchRec LR = A.launches[U.launch];
        const PairRec bra = A.pairs[LR.bra_pair0 + U.ib];
        const MolCtx M = mol_of(A, U.launch);
        const int ik = U.k0 + lane;
        bool active = ik < U.k1;
        PairRec ket{};
        if (active) {
            ket = A.pairs[LR.ket_pair0 + ik];
            active = !skip6(M.Dsh, M.n_sh, bra.a, bra.b, ket.a, ket.b, bra.G, ket.G, A.tau);
        }
        const unsigned mask = __ballot_sync(0xffffffffu, active);
        if (!mask) continue;
        if (A.computed && lane == 0) atomicAdd(A.computed + U.launch, (unsigned long long)__popc(mask));
        double jab[NAB];
#pragma unroll
        for (int t = 0; t < NAB; ++t) jab[t] = 0.0;
        if (active) {
            const double deg = (bra.a == bra.b ? 0.5 : 1.0) * (ket.a == ket.b ? 0.5 : 1.0) *
                               ((LR.diag && ik == U.ib) ? 0.5 : 1.0);
            constexpr int NC = cnc(LC), ND = cnc(LD);
            constexpr int S5 = NC * ND + NA * NC + NA * ND + NB * NC + NB * ND;
            double *wq = A.W ? ket_slots(A, U.launch, LR.n_ket, U.ib, ik, NAB, S5) : nullptr;
            quartet_compiled<LA, LB, LC, LD, R>(A, M, bra, ket, deg, jab, wq, LR.n_ket);
        }
#pragma unroll
        for (int t = 0; t < NAB; ++t) {
            const double v = warp_sum(jab[t]);
            if (A.W) {
                if (lane == 0) A.wab[A.wab_off[u] + t] = v;  // the unit's partial, reduced in unit order
            } else if (lane == 0 && v != 0.0) {
                atomicAdd(M.Jp + (size_t)(bra.ao_a + t / NB) * M.n_ao + bra.ao_b + t % NB, v);
            }
        }
    }
}

}  // namespace fjb
