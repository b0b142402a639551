// plan.h -- the fused Fock build's pair stream (host side).
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "fjb_internal.h"

namespace fjb {

struct HostShell {
    int l;
    double centre[3];
    std::vector<double> exps, coefs;
};

struct HostBasis {
    std::vector<HostShell> shells;
    std::vector<int> offsets;
    int n_ao = 0;
};

// One kept contracted pair (launch_f.py FPair).
struct PlanPair {
    int a, b, la, lb, n_prim;
    std::vector<int> prims;       // kept primitive-pair indices i*K_b + j
    std::vector<double> prim_G;   // their bounds, in kept order
    double G, dmax, key;
    int mag;
};

struct PlanBatch {
    int la, lb, degree, mag;
    double magnitude;
    std::vector<PlanPair> pairs;
    double g_max() const;
};

struct Plan {
    double tau = 0, eps = 0, g_max = 0;
    int n = 0;
    std::vector<double> mags;
    std::vector<PlanBatch> batches;
    std::vector<std::pair<int, int>> launches, screened, deleted;
    int64_t n_prim_total = 0;
};

// Correctly rounded sum (Shewchuk's partials with a round-half-even fix).
double fsum(const double *x, size_t n);

using Cart3 = std::array<int, 3>;

// hermite_order(L) (mmd/hermite.py): totals 0..L, each tx desc then ty desc.
std::vector<Cart3> herm_order(int L);
// cartesians(l) (ao/shell.py:68): i desc, then j desc.
std::vector<Cart3> carts(int l);
// e_axis (mmd/hermite.py:61-79): E^{ij}_t, t = 0..i+j, with the axis's
// Gaussian-product factor exp(zeta pa pb) in E^{00}_0.
void e_axis(int i, int j, double zeta, double pa, double pb, double *e);
// I_p = sqrt((-1)^|p| [2p]^(0)(PQ = 0, theta = sqrt(zeta/2))) for every p of
// hs (ao/pairs.py:270-287), with F_M(0) the reference's own (boys_zero.h).
void hermite_bounds(double zeta, int L, const std::vector<Cart3> &hs, double *I);

// G_[ab] of every primitive pair of the ordered shell pair (a, b), in
// primitive_pairs order (i outer).
std::vector<double> primitive_schwarz_bounds(const HostShell &sa, const HostShell &sb);

// The bounds of one canonical shell pair: G_[ab] per primitive pair and
// their fsum G.  They depend on the basis alone, not on D or tau.
struct PairBounds {
    int a = 0, b = 0;
    std::vector<double> g;
    double G = 0.0;
};

// The pair stream (launch_f.py:390-466).  Throws std::invalid_argument /
// std::runtime_error with the reference's refusals.  With `bounds` non-null
// the canonical pairs' bounds are taken from it when it is filled, and
// computed into it when it is empty, so plans of one basis for successive
// densities (an SCF loop) compute them once.
Plan f_launches(const HostBasis &basis, const double *D, double tau, int n, int threads,
                std::vector<PairBounds> *bounds = nullptr);

// The split build's ordered pair stream (eri/hjk/launch_hjk.py:280
// hjk_launches): every ORDERED shell pair (a, b) with G = fsum of its
// primitive bounds, nothing pruned; bins (la, lb, degree) in sorted order,
// pairs descending by G, stably (a outer, b inner); every ordered batch pair
// a launch; every ordered quartet of shell pairs a visit with the key
// G_ab G_cd max|D_bd| (screen K) or G_ab G_cd max|D_cd| (screen J), skipped
// when the key is below tau.  Visits are not stored (n_pairs^2 of them):
// hjk_key gives any one, in the plan's order.
struct HjkPair {
    int a, b, la, lb, degree;
    double G;
};
struct HjkBatch {
    int la, lb, degree, p0, n;  // its pairs: pairs[p0, p0 + n)
};
struct HjkPlan {
    double tau = 0.0;
    int mode = 0;    // 0 ordered (each launch its own class), 1 canonical
    int screen = 1;  // 0 J's key, 1 K's key
    int n_sh = 0;
    std::vector<HjkPair> pairs;  // batch by batch, in batch order
    std::vector<HjkBatch> batches;
    std::vector<std::pair<int, int>> launches;  // (bra batch, ket batch), bra outer
    std::vector<double> dmax;                    // n_sh x n_sh: max |D| of each shell block
    // a launch's kernel class and the shell positions that class reads:
    // kernel position j holds the ordered quartet's position shells[j]
    std::array<int, 4> ordered(int launch) const;
    std::array<int, 4> kernel_class(int launch, std::array<int, 4> *shells) const;
    double key(const HjkPair &p, const HjkPair &q) const;
};
constexpr int kHjkModeOrdered = 0, kHjkModeCanonical = 1, kHjkScreenJ = 0, kHjkScreenK = 1;

HjkPlan hjk_launches(const HostBasis &basis, const double *D, double tau, int mode, int screen, int threads);

}  // namespace fjb
