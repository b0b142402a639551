// plan.cpp -- the pair stream of the fused Fock build, restated in C++.
//
// Follows the reference's eri/fock/launch_f.py:390-466 (f_launches) step by
// step, with the bound of ao/pairs.py:528-541 (primitive_schwarz_bound):
//   * one canonical pair per unordered shell pair (la <= lb, lower index
//     first on a tie of l), in i-outer, j >= i order;
//   * G_[ab] per primitive pair = max over Cartesian rows k of
//     fsum_p |E_kp| I_p(zeta), E the dressed Hermite block
//     (mmd/hermite.py:61-117, ao/pairs.py:238-254) and
//     I_p = sqrt((-1)^|p| [2p]^(0)(PQ=0, theta=sqrt(zeta/2)))
//     (ao/pairs.py:270-287; reference/pq.py:50-124);
//   * G = fsum over all primitive pairs; eps = tau/(2 Gmax);
//   * prune: drop the longest tail (descending G, stable) whose fsum < eps;
//     a pair with nothing kept is deleted;
//   * dmax = max |D| over the pair's block, key = G * dmax, eq. 29 magnitude
//     index (the largest i >= 1 with G < tau^(i/n), else 0);
//   * bins (la, lb, degree, mag) in sorted order, pairs in each sorted
//     descending by key, stably;
//   * batch pairs I <= J: screened when mag_I + mag_J >= n (refused unless
//     max G_I * max G_J < tau), launched otherwise.
// Every step is written to give the reference's floating-point results
// operation for operation; F_m(0) is the reference's own quadrature value
// (boys_zero.h), a few ulps from 1/(2m+1).  The lists and bounds are held
// equal to the reference's own on the seeded workloads by tests/test_plan.py.
#include "plan.h"
#include "boys_zero.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <tuple>

namespace fjb {

namespace {
// fsum's partials: at most about 40 non-overlapping doubles ever (their
// exponents are distinct and span the double range), so a fixed buffer on
// the stack holds them; it grows onto the heap only if that bound is passed.
struct Partials {
    double fixed[64];
    std::vector<double> spill;
    double *d = fixed;
    size_t n = 0, cap = 64;
    size_t size() const { return n; }
    double &operator[](size_t i) { return d[i]; }
    void resize(size_t k) { n = k; }
    void push_back(double v) {
        if (n == cap) {
            if (d == fixed) spill.assign(fixed, fixed + n);
            spill.resize(2 * cap);
            d = spill.data();
            cap = spill.size();
        }
        d[n++] = v;
    }
};
}  // namespace

double fsum(const double *x, size_t n) {
    Partials p;
    for (size_t t = 0; t < n; ++t) {
        double v = x[t];
        if (!std::isfinite(v)) throw std::invalid_argument("fsum of a non-finite value");
        size_t i = 0;
        for (size_t j = 0; j < p.size(); ++j) {
            double y = p[j];
            if (std::fabs(v) < std::fabs(y)) std::swap(v, y);
            double hi = v + y;
            double lo = y - (hi - v);
            if (lo != 0.0) p[i++] = lo;
            v = hi;
        }
        p.resize(i);
        p.push_back(v);
    }
    size_t k = p.size();
    if (k == 0) return 0.0;
    double hi = p[--k], lo = 0.0;
    while (k > 0) {
        double xx = hi, y = p[--k];
        hi = xx + y;
        double yr = hi - xx;
        lo = y - yr;
        if (lo != 0.0) break;
    }
    if (k > 0 && ((lo < 0.0 && p[k - 1] < 0.0) || (lo > 0.0 && p[k - 1] > 0.0))) {
        double y = lo * 2.0;
        double xx = hi + y;
        double yr = xx - hi;
        if (y == yr) hi = xx;
    }
    return hi;
}

namespace {
constexpr double kPi = 3.141592653589793;
}  // namespace

std::vector<Cart3> herm_order(int L) {
    std::vector<Cart3> out;
    for (int n = 0; n <= L; ++n)
        for (int tx = n; tx >= 0; --tx)
            for (int ty = n - tx; ty >= 0; --ty) out.push_back({tx, ty, n - tx - ty});
    return out;
}

std::vector<Cart3> carts(int l) {
    std::vector<Cart3> out;
    for (int i = l; i >= 0; --i)
        for (int j = l - i; j >= 0; --j) out.push_back({i, j, l - i - j});
    return out;
}

// e_axis (mmd/hermite.py:61-79): E^{ij}_t, t = 0..i+j.
void e_axis(int i, int j, double zeta, double pa, double pb, double *e) {
    double prev[16], out[16];
    int n = 1;
    prev[0] = std::exp(zeta * pa * pb);
    double h = 0.5 / zeta;
    for (int s = 0; s < i + j; ++s) {
        double x = s < i ? pa : pb;
        for (int t = 0; t <= n; ++t) {
            double v = 0.0;
            if (t >= 1) v += h * prev[t - 1];
            if (t < n) v += x * prev[t];
            if (t + 1 < n) v += (double)(t + 1) * prev[t + 1];
            out[t] = v;
        }
        ++n;
        for (int t = 0; t < n; ++t) prev[t] = out[t];
    }
    for (int t = 0; t < n; ++t) e[t] = prev[t];
}

namespace {
// One recurrence step of e_axis: E of length n -> length n + 1 along an
// axis whose distance is x (the loop body of e_axis, operation for
// operation).
inline void e_step(const double *prev, int n, double x, double h, double *out) {
    for (int t = 0; t <= n; ++t) {
        double v = 0.0;
        if (t >= 1) v += h * prev[t - 1];
        if (t < n) v += x * prev[t];
        if (t + 1 < n) v += (double)(t + 1) * prev[t + 1];
        out[t] = v;
    }
}

// e_axis(i, j, ...) for every i <= la, j <= lb at once: E^{ij} is i steps
// along pa then j along pb from the same exp(zeta pa pb), so E^{i0} is
// carried from i to i + 1 and each E^{ij} extends its E^{i,j-1}.  Every
// value is the one e_axis computes, with the exponential taken once.
void e_axis_all(int la, int lb, double zeta, double pa, double pb, double (*ex)[7][16]) {
    const double h = 0.5 / zeta;
    double ei0[16];
    ei0[0] = std::exp(zeta * pa * pb);
    for (int i = 0; i <= la; ++i) {
        if (i > 0) {
            double nxt[16];
            e_step(ei0, i, pa, h, nxt);
            for (int t = 0; t <= i; ++t) ei0[t] = nxt[t];
        }
        for (int t = 0; t <= i; ++t) ex[i][0][t] = ei0[t];
        for (int j = 1; j <= lb; ++j) e_step(ex[i][j - 1], i + j, pb, h, ex[i][j]);
    }
}

// Per (la, lb): for each Cartesian pair (a, b), in carts(la) x carts(lb)
// order, the Hermite indices t of hermite_order(la + lb) whose every axis
// stays within that pair's E^{a_d b_d} (the others give zero terms), and
// the three axes' E rows.  Built once per process.
struct PairTerms {
    std::vector<int> idx, start;   // start[ab] .. start[ab + 1] into idx
    std::vector<Cart3> ca, cb, hs;
};
const PairTerms &pair_terms(int la, int lb) {
    static std::once_flag once[7][7];
    static PairTerms tab[7][7];
    std::call_once(once[la][lb], [la, lb]() {
        PairTerms &P = tab[la][lb];
        P.hs = herm_order(la + lb);
        P.ca = carts(la);
        P.cb = carts(lb);
        P.start.push_back(0);
        for (auto &a : P.ca)
            for (auto &b : P.cb) {
                for (size_t t = 0; t < P.hs.size(); ++t)
                    if (P.hs[t][0] <= a[0] + b[0] && P.hs[t][1] <= a[1] + b[1] && P.hs[t][2] <= a[2] + b[2])
                        P.idx.push_back((int)t);
                P.start.push_back((int)P.idx.size());
            }
    });
    return tab[la][lb];
}
}  // namespace

// I_p for every p of hermite_order(L) at exponent sum zeta (ao/pairs.py:270).
void hermite_bounds(double zeta, int L, const std::vector<Cart3> &hs, double *I) {
    const double two_over_sqrt_pi = 2.0 / std::sqrt(kPi);
    double theta = std::sqrt(zeta / 2.0);
    double t2 = theta * theta;
    // the order-M factor, once per M (the same left-to-right product)
    if (L > kBoysZeroMax) throw std::invalid_argument("Hermite order above the F_m(0) table");
    double base[kBoysZeroMax + 1];
    for (int M = 0; M <= L; ++M)
        base[M] = two_over_sqrt_pi * theta * std::pow(-2.0 * t2, (double)M) * kBoysZero[M];
    for (size_t k = 0; k < hs.size(); ++k) {
        const Cart3 &p = hs[k];
        int M = p[0] + p[1] + p[2];
        // fundamental(M, 0, theta) with F_M(0) the reference's own value
        double v = base[M];
        // the recursion's integer factors, innermost (z) first
        for (int q = 1; q <= p[2]; ++q) v = (double)(2 * q - 1) * v;
        for (int q = 1; q <= p[1]; ++q) v = (double)(2 * q - 1) * v;
        for (int q = 1; q <= p[0]; ++q) v = (double)(2 * q - 1) * v;
        double s = (M % 2) ? -v : v;
        if (s < 0.0) throw std::runtime_error("negative Hermite self-integral");
        I[k] = std::sqrt(s);
    }
}

std::vector<double> primitive_schwarz_bounds(const HostShell &sa, const HostShell &sb) {
    const double *A = sa.centre, *B = sb.centre;
    const int L = sa.l + sb.l;
    if (sa.l > 6 || sb.l > 6) throw std::invalid_argument("a shell above l = 6 in the pair bounds");
    const PairTerms &PT = pair_terms(sa.l, sb.l);
    const std::vector<Cart3> &hs = PT.hs;
    std::vector<double> out, I(hs.size()), terms(hs.size());
    out.reserve(sa.exps.size() * sb.exps.size());
    for (size_t i = 0; i < sa.exps.size(); ++i)
        for (size_t j = 0; j < sb.exps.size(); ++j) {
            double alpha = sa.exps[i], beta = sb.exps[j];
            double ca_ = sa.coefs[i], cb_ = sb.coefs[j];
            double zeta = alpha + beta;
            double P[3];
            for (int d = 0; d < 3; ++d) P[d] = (alpha * A[d] + beta * B[d]) / zeta;
            double scale = ca_ * cb_ * std::pow(kPi / zeta, 1.5);
            hermite_bounds(zeta, L, hs, I.data());
            // E^{ij}_t of each axis for every i <= la, j <= lb, once per
            // primitive pair (the cartesian pairs below reuse them)
            double ex[3][7][7][16];
            for (int d = 0; d < 3; ++d) e_axis_all(sa.l, sb.l, zeta, P[d] - A[d], P[d] - B[d], ex[d]);
            double best = 0.0;
            bool first = true;
            int ab = 0;
            for (auto &a : PT.ca)
                for (auto &b : PT.cb) {
                    const double *ax[3];
                    for (int d = 0; d < 3; ++d) ax[d] = ex[d][a[d]][b[d]];
                    // only the Hermite indices within every axis's E^{ij}:
                    // the others give zero terms, and fsum is correctly
                    // rounded, so leaving them out changes no bit of g
                    size_t m = 0;
                    for (int k = PT.start[ab]; k < PT.start[ab + 1]; ++k) {
                        const int t = PT.idx[k];
                        double v = 1.0;
                        for (int d = 0; d < 3; ++d) v = v * ax[d][hs[t][d]];
                        double e = scale * v;
                        terms[m++] = std::fabs(e) * I[t];
                    }
                    ++ab;
                    double g = fsum(terms.data(), m);
                    if (first || g > best) best = g;
                    first = false;
                }
            out.push_back(best);
        }
    return out;
}

double PlanBatch::g_max() const {
    double g = pairs.front().G;
    for (auto &p : pairs) g = std::max(g, p.G);
    return g;
}

namespace {

std::vector<int> prune(const std::vector<double> &g, double eps) {
    std::vector<int> order(g.size());
    for (size_t k = 0; k < g.size(); ++k) order[k] = (int)k;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return -g[x] < -g[y]; });
    size_t cut = order.size();
    std::vector<double> tail;
    while (cut > 0) {
        tail.clear();
        for (size_t k = cut - 1; k < order.size(); ++k) tail.push_back(g[order[k]]);
        if (fsum(tail.data(), tail.size()) < eps)
            --cut;
        else
            break;
    }
    order.resize(cut);
    return order;
}

int magnitude_index(double G, const std::vector<double> &mags) {
    for (int i = (int)mags.size() - 1; i > 0; --i)
        if (G < mags[i]) return i;
    return 0;
}

}  // namespace

Plan f_launches(const HostBasis &basis, const double *D, double tau, int n, int threads,
                std::vector<PairBounds> *bounds) {
    if (!(std::isfinite(tau) && tau >= 0.0)) throw std::invalid_argument("tau is not a finite float >= 0");
    if (n < 1) throw std::invalid_argument("n is not an int >= 1 (the number of eq. 29 magnitudes)");
    const int nsh = (int)basis.shells.size(), nao = basis.n_ao;
    for (int i = 0; i < nao; ++i)
        for (int j = 0; j < nao; ++j) {
            double v = D[(size_t)i * nao + j];
            if (!std::isfinite(v)) throw std::invalid_argument("D has a non-finite entry");
            if (j < i && v != D[(size_t)j * nao + i])
                throw std::invalid_argument("D is not symmetric: an asymmetric density is rejected, not symmetrised");
        }
    Plan plan;
    plan.tau = tau;
    plan.n = n;
    for (int i = 0; i < n; ++i) plan.mags.push_back(std::pow(tau, (double)i / (double)n));

    std::vector<PairBounds> local;
    std::vector<PairBounds> &raw = bounds ? *bounds : local;
    if (raw.empty()) {
        std::vector<std::pair<int, int>> canon;
        for (int i = 0; i < nsh; ++i)
            for (int j = i; j < nsh; ++j) {
                bool keep = std::make_pair(basis.shells[i].l, i) <= std::make_pair(basis.shells[j].l, j);
                canon.emplace_back(keep ? i : j, keep ? j : i);
            }
        std::vector<PairBounds> fresh(canon.size());
        int nt = std::max(1, threads);
        std::vector<std::thread> pool;
        std::vector<std::string> errs(nt);
        for (int t = 0; t < nt; ++t)
            pool.emplace_back([&, t]() {
                try {
                    for (size_t k = t; k < canon.size(); k += nt) {
                        auto [a, b] = canon[k];
                        fresh[k].a = a;
                        fresh[k].b = b;
                        fresh[k].g = primitive_schwarz_bounds(basis.shells[a], basis.shells[b]);
                        fresh[k].G = fsum(fresh[k].g.data(), fresh[k].g.size());
                    }
                } catch (const std::exception &e) {
                    errs[t] = e.what();
                }
            });
        for (auto &th : pool) th.join();
        for (auto &e : errs)
            if (!e.empty()) throw std::runtime_error(e);
        raw = std::move(fresh);
    }

    double g_max = 0.0;
    for (auto &r : raw) g_max = std::max(g_max, r.G);
    plan.g_max = g_max;
    plan.eps = (tau > 0.0 && g_max > 0.0) ? tau / (2.0 * g_max) : 0.0;

    std::vector<PlanPair> kept;
    for (auto &r : raw) {
        plan.n_prim_total += (int64_t)r.g.size();
        auto keep = prune(r.g, plan.eps);
        if (keep.empty()) {
            plan.deleted.emplace_back(r.a, r.b);
            continue;
        }
        const HostShell &sa = basis.shells[r.a], &sb = basis.shells[r.b];
        int oa = basis.offsets[r.a], ob = basis.offsets[r.b];
        int na = (sa.l + 1) * (sa.l + 2) / 2, nb = (sb.l + 1) * (sb.l + 2) / 2;
        double dmax = 0.0;
        bool first = true;
        for (int m = oa; m < oa + na; ++m)
            for (int k = ob; k < ob + nb; ++k) {
                double v = std::fabs(D[(size_t)m * nao + k]);
                if (first || v > dmax) dmax = v;
                first = false;
            }
        PlanPair p;
        p.a = r.a;
        p.b = r.b;
        p.la = sa.l;
        p.lb = sb.l;
        p.n_prim = (int)r.g.size();
        p.prims = keep;
        for (int k : keep) p.prim_G.push_back(r.g[k]);
        p.G = r.G;
        p.dmax = dmax;
        p.key = r.G * dmax;
        p.mag = magnitude_index(r.G, plan.mags);
        kept.push_back(std::move(p));
    }
    std::map<std::tuple<int, int, int, int>, std::vector<PlanPair>> bins;
    for (auto &p : kept) {
        const auto key = std::make_tuple(p.la, p.lb, (int)p.prims.size(), p.mag);
        bins[key].push_back(std::move(p));
    }
    for (auto &kv : bins) {
        PlanBatch b;
        std::tie(b.la, b.lb, b.degree, b.mag) = kv.first;
        b.magnitude = plan.mags[b.mag];
        b.pairs = std::move(kv.second);
        std::stable_sort(b.pairs.begin(), b.pairs.end(),
                         [](const PlanPair &x, const PlanPair &y) { return x.key > y.key; });
        plan.batches.push_back(std::move(b));
    }
    const int nb = (int)plan.batches.size();
    for (int bi = 0; bi < nb; ++bi)
        for (int ki = bi; ki < nb; ++ki) {
            const PlanBatch &br = plan.batches[bi], &kt = plan.batches[ki];
            if (br.mag + kt.mag >= n) {
                if (!(br.g_max() * kt.g_max() < tau))
                    throw std::runtime_error("eq. 29's magnitudes rounded past the bound: the pre-launch screen would not be sound");
                plan.screened.emplace_back(bi, ki);
            } else {
                plan.launches.emplace_back(bi, ki);
            }
        }
    return plan;
}

}  // namespace fjb
