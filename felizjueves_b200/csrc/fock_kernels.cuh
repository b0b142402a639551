// fock_kernels.cuh -- sm_100a device code of the Fock build.
//
//   boys_eval       F_0..F_M(T): tabulated Taylor (7 terms at the nearest
//                   0.05 node) then downward recursion below T = 40; the
//                   erf-free large-T start F_0 = sqrt(pi/T)/2 and upward
//                   recursion above (stable there: (2m+1)/(2T) < 1).
//   skip6           the six-block screen of a quartet, in the reference's
//                   operation order (walk_f.py:344-351; kernel_f.py:152-163).
//   hgp_fock_kernel one CTA per work unit (a bra shell pair and a chunk of
//                   its kets); per computed quartet: staged primitive pairs,
//                   per-primitive-quartet scalars and Boys leaves, the VRR
//                   program level by level over (node x primitive quartet),
//                   the boundary contraction, the two HRR transforms, and
//                   the six-block digest into J and K (thread-private sums,
//                   FP64 atomics for the five ket-dependent blocks, the bra
//                   block F_ab accumulated in shared memory and flushed once
//                   per unit, kernel_f.py:94-131).
#pragma once
#include <cuda_runtime.h>

#include "fjb_internal.h"

namespace fjb {

// One molecule's density, shell-block maxima and accumulators: the batched
// build (fjb_batch_build) runs many molecules' units in one launch per class
// and each unit finds its molecule through its launch.
struct MolCtx {
    const double *D, *Dsh;
    double *Jp, *Kp;
    int n_ao, n_sh;
};

struct KArgs {
    ClassDev C;
    const Unit *units;
    int n_units;
    const LaunchRec *launches;
    const PairRec *pairs;
    const PrimRec *prims;
    const double *D;
    const double *Dsh;
    int n_sh, n_ao;
    double tau;
    double *Jp, *Kp;
    double *tap_out;        // ERI tap mode when non-null
    const int64_t *tap_off; // per unit
    // the split K build (fjb_hjk_k; HGP interpreter only): every visited
    // quartet deposits K[x_p][x_q] += D[x_r][x_s] (x_0 x_1|x_2 x_3) into Kp
    // alone, (p, r, q, s) = the launch's axes (LaunchRec.pad0, two bits
    // each), and is skipped when (G_bra G_ket) max|D_{x_r x_s}| < tau
    int hk;
    const double *boys_tab;
    const uint8_t *route;   // per unit ket flags, routed mode (null: all FP64)
    double route_thresh;
    unsigned long long *computed;  // per launch: quartets computed (null: not counted)
    const int *unit_list;   // device queue of unit indices (null: every unit)
    const int *unit_count;  // its length, on the device
    // the atomics-free build (null W: FP64 atomics into Jp/Kp)
    double *W;               // the launches' slot buffer
    const int64_t *w_base;   // per launch: its first slot in W
    double *wab;             // per unit: the bra block's partial sums
    const int64_t *wab_off;  // per unit of this run: its offset in wab
    // the Rys kernel (rys_fock.cuh): its layout and the tabulated rule
    RysDev Y;
    const double *rys_tab;
    const float *rys_tab32;  // its FP32 copy (the FP32 tier)
    // the batched build: per molecule its context, per launch its molecule
    // (null: one molecule, the fields above)
    const MolCtx *mols;
    const int32_t *launch_mol;
};

__device__ __forceinline__ MolCtx mol_of(const KArgs &A, int launch) {
    if (A.mols) return A.mols[A.launch_mol[launch]];
    return MolCtx{A.D, A.Dsh, A.Jp, A.Kp, A.n_ao, A.n_sh};
}

// A quartet's first ket-block slot (block element 0) in the atomics-free
// build: bra pair ib, ket position ik of launch `launch`; element e of the
// five ket blocks (BLOCKS order cd, ac, ad, bc, bd) is at [e * n_ket].
__device__ __forceinline__ double *ket_slots(const KArgs &A, int launch, int n_ket, int ib, int ik, int n_ab,
                                             int s5) {
    const int64_t row = n_ab + (int64_t)s5 * n_ket;
    return A.W + A.w_base[launch] + (int64_t)ib * row + n_ab + ik;
}

// 1/(2m+1), m = 0 .. kBoysMaxM: the downward recursion multiplies by these
// (each the correctly rounded quotient) instead of dividing.
static __constant__ double kRecipOdd[kBoysMaxM + 1] = {1.0 / 1.0, 1.0 / 3.0, 1.0 / 5.0, 1.0 / 7.0, 1.0 / 9.0, 1.0 / 11.0, 1.0 / 13.0, 1.0 / 15.0, 1.0 / 17.0, 1.0 / 19.0, 1.0 / 21.0, 1.0 / 23.0, 1.0 / 25.0, 1.0 / 27.0, 1.0 / 29.0, 1.0 / 31.0, 1.0 / 33.0, 1.0 / 35.0, 1.0 / 37.0, 1.0 / 39.0, 1.0 / 41.0, 1.0 / 43.0, 1.0 / 45.0, 1.0 / 47.0, 1.0 / 49.0};

// exp(-T) at a table node's offset d = T_i - T (|d| <= kBoysDelta/2):
// exp(-T_i) (the row's last entry) times the degree-8 Taylor polynomial of
// exp(d), by Horner.
__device__ __forceinline__ double boys_exp(const double *__restrict__ row0, double d) {
    double p = 1.0 / 40320.0;
    p = 1.0 / 5040.0 + d * p;
    p = 1.0 / 720.0 + d * p;
    p = 1.0 / 120.0 + d * p;
    p = 1.0 / 24.0 + d * p;
    p = 1.0 / 6.0 + d * p;
    p = 0.5 + d * p;
    p = 1.0 + d * p;
    p = 1.0 + d * p;
    return __ldg(row0 + kBoysMaxM + 1) * p;
}

__device__ __forceinline__ void boys_eval(int M, double T, double *F, const double *__restrict__ tab) {
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
            for (int m = M - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) * kRecipOdd[m];
        }
    } else {
        const double e = exp(-T), h = 0.5 / T;
        F[0] = 0.5 * sqrt(3.141592653589793 / T);
        for (int m = 0; m < M; ++m) F[m + 1] = ((double)(2 * m + 1) * F[m] - e) * h;
    }
}

// The six-block screen: dmax over |w_b| Dsh_b in BLOCKS order (ab, cd, ac,
// ad, bc, bd) with |w| = (2, 2, 1/2, 1/2, 1/2, 1/2), then
// G_ab (G_cd dmax) < tau.  Multiplies and compares only: bit-exact.
__device__ __forceinline__ bool skip6(const double *__restrict__ Dsh, int n_sh, int a, int b, int c,
                                      int d, double Gb, double Gk, double tau) {
    double dmax = 2.0 * __ldg(Dsh + (size_t)a * n_sh + b);
    double t = 2.0 * __ldg(Dsh + (size_t)c * n_sh + d);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)a * n_sh + c);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)a * n_sh + d);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)b * n_sh + c);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)b * n_sh + d);
    if (dmax < t) dmax = t;
    return __dmul_rn(Gb, __dmul_rn(Gk, dmax)) < tau;
}

// G_ab G_cd dmax itself (skip6's left-hand side): the bound on every term
// the quartet deposits, read by the precision router.
__device__ __forceinline__ double six_block_bound(const double *__restrict__ Dsh, int n_sh, int a, int b,
                                                 int c, int d, double Gb, double Gk) {
    double dmax = 2.0 * __ldg(Dsh + (size_t)a * n_sh + b);
    double t = 2.0 * __ldg(Dsh + (size_t)c * n_sh + d);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)a * n_sh + c);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)a * n_sh + d);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)b * n_sh + c);
    if (dmax < t) dmax = t;
    t = 0.5 * __ldg(Dsh + (size_t)b * n_sh + d);
    if (dmax < t) dmax = t;
    return __dmul_rn(Gb, __dmul_rn(Gk, dmax));
}

__device__ __forceinline__ double ipow(double x, int n) {
    double r = 1.0;
    for (int k = 0; k < n; ++k) r *= x;
    return r;
}

}  // namespace fjb
