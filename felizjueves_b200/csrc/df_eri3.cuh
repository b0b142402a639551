// df_eri3.cuh -- the three-centre integrals (mn|P) of density fitting by Rys
// quadrature, written straight into an aux block of the [m][n][P] tensor
// (aux fastest: the reference's layout, eri/density_fit/eri3.py:226).
//
// df_eri3_kernel<LA, LB, LP>: one CTA per work unit -- an AO shell pair
// (a, b) with la >= lb and up to kE3Kets aux shells of angular momentum LP,
// taken G at a time.  An aux shell P is the ket pair (P, unit), the unit an
// s function of exponent 0, so the ket's Gaussian product is P's own
// primitive and the ket side needs no transfer.  Per group of aux shells:
//
//   A  tables: per (aux shell, primitive pair, root) one thread evaluates
//      the Rys rule at T (rys_rule.h) and the three axes' 2D integrals
//      I_d(i, k), i <= LA+LB, k <= LP; the root's weight and the seed
//      U_ab U_P (2/sqrt(pi)) sqrt(rho) folded into the z axis.
//   B  boundary: per (aux shell, P Cartesian f) one thread holds the bra
//      column [e0|f] for LA <= |e| <= LA+LB in registers and accumulates
//      I_x I_y I_z over primitive pairs and roots.
//   C  bra HRR from those registers and the store: (ab|f) for every
//      (a, b), at [m][n][P] and, for a != b, at the mirror [n][m][P]; the
//      threads of one aux shell and its neighbours write consecutive P.
//
// The same recurrences and rule as the Rys Fock kernel (rys_fock.cuh), in
// FP64.  la >= lb puts the larger shell on the transfer's receiving side,
// so (f s|P) needs no HRR at all.
#pragma once
#include <cuda_runtime.h>

#include "fjb_internal.h"
#include "rys_fock.cuh"

// The classes (la >= lb, both <= 3; aux l <= 4)
#define FJB_E3_BRAS(X, LP) \
    X(0, 0, LP) X(1, 0, LP) X(1, 1, LP) X(2, 0, LP) X(2, 1, LP) X(2, 2, LP) X(3, 0, LP) X(3, 1, LP) X(3, 2, LP) X(3, 3, LP)
#define FJB_E3_CLASSES(X) FJB_E3_BRAS(X, 0) FJB_E3_BRAS(X, 1) FJB_E3_BRAS(X, 2) FJB_E3_BRAS(X, 3) FJB_E3_BRAS(X, 4)
#define FJB_E3_MAX_LP 4

namespace fjb {

constexpr int kE3Kets = 128;    // aux shells per work unit
constexpr int kE3Threads = 128;

// A work unit: AO pair `pair`, aux shells [k0, k1) of the l-sorted list.
struct E3Unit {
    int32_t pair, k0, k1, pad;
};

// The shared-memory carve-up of one class (doubles) and its group sizes.
struct E3Dev {
    int group, chunk, kab, kcd;
    int sm_braP, sm_cb, sm_ketP, sm_tab, sm_total;
};

struct E3Args {
    E3Dev Y;
    const E3Unit *units;
    int n_units;
    const PairRec *pairs;  // AO pairs (la >= lb); G = sqrt(max |(ab|ab)|)
    const PrimRec *prims;
    const PairRec *kets;   // aux shells as (P, unit) pairs, sorted by l;
                           // ao_a = P's first function in the aux basis
    const PrimRec *kprims;
    double *out;           // [n_ao][n_ao][nb]
    int n_ao, p0, nb;      // the block: aux functions [p0, p0 + nb)
    double tau;            // (ab|P) is zero by Schwarz when G_ab G_P < tau
    const double *rys_tab;
};

bool eri3_layout(int la, int lb, int lp, int max_kab, int max_kcd, E3Dev *out);
int eri3_blocks_per_sm(int la, int lb, int lp, const E3Dev &d);
cudaError_t eri3_launch(int la, int lb, int lp, int grid, cudaStream_t st, const E3Args &a);

}  // namespace fjb
