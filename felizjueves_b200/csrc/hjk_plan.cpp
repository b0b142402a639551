// hjk_plan.cpp -- the split build's ordered pair stream, restated in C++.
//
// Follows the reference's eri/hjk/launch_hjk.py:280-342 (hjk_launches):
//   * every ORDERED shell pair (a, b), a outer and b inner, with G = the
//     fsum of primitive_schwarz_bounds(sa, sb) over all K_a K_b primitive
//     pairs (nothing pruned; a degree above 128 refused);
//   * dmax of a shell block = max |D| over it;
//   * bins (la, lb, degree) in sorted key order, pairs in a bin descending by
//     G, stably;
//   * every ordered batch pair (bra, ket) a launch, bra outer;
//   * every (bra pair p, ket pair q) of a launch a visit, p outer, with the
//     key (G_p G_q) dmax[b][d] (K, launch_hjk.py:153 k_key) or (G_p G_q)
//     dmax[c][d] (J, j_key), skipped when key < tau (skip, never break).
// The density and tau refusals are the reference's.  A launch's kernel
// class: its ordered class itself (mode ordered, the reference's identity
// orientation), or (mode canonical) the first element of the ERI's 8-fold
// group, in the reference's GROUP order (hgp/orbits.py:73-82), that carries
// the ordered class onto a class with la <= lb, lc <= ld and (la, lb) <=
// (lc, ld) -- the classes this build's kernels are compiled for.  (The
// reference's canonical mode picks the orbit member with the cheapest HGP
// recurrence of its own generated kernels instead; the launches, the visits
// and their keys are the same in both.)
#include <algorithm>
#include <cmath>
#include <map>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>

#include "../../include/fjb.h"
#include "plan.h"

namespace fjb {

namespace {

// hgp/orbits.py GROUP: position j of g . cls holds cls[g[j]]
constexpr int kGroup[8][4] = {{0, 1, 2, 3}, {1, 0, 2, 3}, {0, 1, 3, 2}, {1, 0, 3, 2},
                              {2, 3, 0, 1}, {3, 2, 0, 1}, {2, 3, 1, 0}, {3, 2, 1, 0}};

bool ladder(const std::array<int, 4> &c) {
    return c[0] <= c[1] && c[2] <= c[3] && std::make_pair(c[0], c[1]) <= std::make_pair(c[2], c[3]);
}

}  // namespace

std::array<int, 4> HjkPlan::ordered(int launch) const {
    const HjkBatch &br = batches[launches[launch].first], &kt = batches[launches[launch].second];
    return {br.la, br.lb, kt.la, kt.lb};
}

std::array<int, 4> HjkPlan::kernel_class(int launch, std::array<int, 4> *shells) const {
    const std::array<int, 4> cls = ordered(launch);
    if (mode == kHjkModeOrdered) {
        if (shells) *shells = {0, 1, 2, 3};
        return cls;
    }
    for (const auto &g : kGroup) {
        const std::array<int, 4> c = {cls[g[0]], cls[g[1]], cls[g[2]], cls[g[3]]};
        if (ladder(c)) {
            if (shells) *shells = {g[0], g[1], g[2], g[3]};
            return c;
        }
    }
    throw std::logic_error("no group element orders the class");  // the group always holds one
}

double HjkPlan::key(const HjkPair &p, const HjkPair &q) const {
    const double d = screen == kHjkScreenK ? dmax[(size_t)p.b * n_sh + q.b] : dmax[(size_t)q.a * n_sh + q.b];
    return p.G * q.G * d;
}

HjkPlan hjk_launches(const HostBasis &basis, const double *D, double tau, int mode, int screen, int threads) {
    if (mode != kHjkModeOrdered && mode != kHjkModeCanonical)
        throw std::invalid_argument("mode is not one of ('canonical', 'ordered')");
    if (screen != kHjkScreenJ && screen != kHjkScreenK) throw std::invalid_argument("screen is not one of ('j', 'k')");
    const int nsh = (int)basis.shells.size(), nao = basis.n_ao;
    for (int i = 0; i < nao; ++i)
        for (int j = 0; j < nao; ++j) {
            const double v = D[(size_t)i * nao + j];
            if (!std::isfinite(v)) throw std::invalid_argument("D has a non-finite entry");
            if (j < i && v != D[(size_t)j * nao + i])
                throw std::invalid_argument("D is not symmetric: an asymmetric density is rejected, not symmetrised");
        }
    if (!(std::isfinite(tau) && tau >= 0.0)) throw std::invalid_argument("tau is not a finite float >= 0");
    HjkPlan P;
    P.tau = tau;
    P.mode = mode;
    P.screen = screen;
    P.n_sh = nsh;
    for (int a = 0; a < nsh; ++a)
        for (int b = 0; b < nsh; ++b) {
            const size_t want = basis.shells[a].exps.size() * basis.shells[b].exps.size();
            if (want > (size_t)FJB_MAX_PRIM_PAIRS)
                throw std::length_error("shell pair (" + std::to_string(a) + ", " + std::to_string(b) +
                                        ") has degree " + std::to_string(want) +
                                        " > MAX_PRIM_PAIRS = 128, the kernel's shared staging cap: refused");
        }
    // the ordered pairs' bounds, a outer and b inner
    std::vector<HjkPair> raw((size_t)nsh * nsh);
    const int nt = std::max(1, threads);
    std::vector<std::thread> pool;
    std::vector<std::string> errs(nt);
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&, t]() {
            try {
                for (size_t k = t; k < raw.size(); k += nt) {
                    const int a = (int)(k / nsh), b = (int)(k % nsh);
                    const HostShell &sa = basis.shells[a], &sb = basis.shells[b];
                    const int want = (int)(sa.exps.size() * sb.exps.size());
                    const std::vector<double> g = primitive_schwarz_bounds(sa, sb);
                    for (double x : g)
                        if (!(std::isfinite(x) && x >= 0.0))
                            throw std::invalid_argument("a primitive bound is not a finite float >= 0");
                    raw[k] = HjkPair{a, b, sa.l, sb.l, want, fsum(g.data(), g.size())};
                }
            } catch (const std::exception &e) {
                errs[t] = e.what();
            }
        });
    for (auto &th : pool) th.join();
    for (auto &e : errs)
        if (!e.empty()) throw std::invalid_argument(e);
    // shell-block maxima of |D|
    P.dmax.assign((size_t)nsh * nsh, 0.0);
    for (int a = 0; a < nsh; ++a)
        for (int b = 0; b < nsh; ++b) {
            const int oa = basis.offsets[a], ob = basis.offsets[b];
            const int na = (basis.shells[a].l + 1) * (basis.shells[a].l + 2) / 2;
            const int nb = (basis.shells[b].l + 1) * (basis.shells[b].l + 2) / 2;
            double m = 0.0;
            bool first = true;
            for (int i = oa; i < oa + na; ++i)
                for (int j = ob; j < ob + nb; ++j) {
                    const double v = std::fabs(D[(size_t)i * nao + j]);
                    if (first || v > m) m = v;
                    first = false;
                }
            P.dmax[(size_t)a * nsh + b] = m;
        }
    // bins in key order, each descending by G, stably
    std::map<std::tuple<int, int, int>, std::vector<HjkPair>> bins;
    for (const auto &p : raw) bins[{p.la, p.lb, p.degree}].push_back(p);
    for (auto &kv : bins) {
        std::stable_sort(kv.second.begin(), kv.second.end(), [](const HjkPair &x, const HjkPair &y) { return x.G > y.G; });
        HjkBatch b;
        std::tie(b.la, b.lb, b.degree) = kv.first;
        b.p0 = (int)P.pairs.size();
        b.n = (int)kv.second.size();
        P.pairs.insert(P.pairs.end(), kv.second.begin(), kv.second.end());
        P.batches.push_back(b);
    }
    const int nb = (int)P.batches.size();
    for (int bi = 0; bi < nb; ++bi)
        for (int ki = 0; ki < nb; ++ki) P.launches.emplace_back(bi, ki);
    return P;
}

}  // namespace fjb
