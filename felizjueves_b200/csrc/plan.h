// plan.h -- the fused Fock build's pair stream (host side).
#pragma once
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

// G_[ab] of every primitive pair of the ordered shell pair (a, b), in
// primitive_pairs order (i outer).
std::vector<double> primitive_schwarz_bounds(const HostShell &sa, const HostShell &sb);

// The pair stream (launch_f.py:390-466).  Throws std::invalid_argument /
// std::runtime_error with the reference's refusals.
Plan f_launches(const HostBasis &basis, const double *D, double tau, int n, int threads);

}  // namespace fjb
