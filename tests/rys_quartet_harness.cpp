// One contracted quartet's ERI block with the Rys boundary (rys_vrr.h) in
// place of the HGP VRR, then the HGP class's own HRR tables (hgp_tables.cpp):
// reads four shells (l, centre, primitive count, exponents, coefficients)
// from stdin, prints the block row-major over (ab, cd); built and run by
// tests/test_rys_rule.py.
#include <cmath>
#include <cstdio>
#include <vector>

#include "hgp_tables.h"
#include "rys_vrr.h"

using namespace fjb;

struct Sh {
    int l;
    double c[3];
    std::vector<double> e, k;
};

int main() {
    const std::vector<double> tab = rys_table();
    Sh s[4];
    for (auto &x : s) {
        int np;
        if (std::scanf("%d %lf %lf %lf %d", &x.l, &x.c[0], &x.c[1], &x.c[2], &np) != 5) return 2;
        x.e.resize(np);
        x.k.resize(np);
        for (auto &v : x.e)
            if (std::scanf("%lf", &v) != 1) return 2;
        for (auto &v : x.k)
            if (std::scanf("%lf", &v) != 1) return 2;
    }
    const ClassHost c = build_class(s[0].l, s[1].l, s[2].l, s[3].l);
    std::vector<Cart> eb, fb;
    for (int n = c.la; n <= c.la + c.lb; ++n)
        for (auto &e : cartesians(n)) eb.push_back(e);
    for (int n = c.lc; n <= c.lc + c.ld; ++n)
        for (auto &f : cartesians(n)) fb.push_back(f);
    const int E = c.la + c.lb, F = c.lc + c.ld, nr = (E + F) / 2 + 1;
    std::vector<double> acc((size_t)c.nbe * c.nbf, 0.0);
    const double pi = 3.141592653589793;
    auto d2 = [](const double *u, const double *v) {
        return (u[0] - v[0]) * (u[0] - v[0]) + (u[1] - v[1]) * (u[1] - v[1]) + (u[2] - v[2]) * (u[2] - v[2]);
    };
    for (size_t ia = 0; ia < s[0].e.size(); ++ia)
        for (size_t ib = 0; ib < s[1].e.size(); ++ib)
            for (size_t ic = 0; ic < s[2].e.size(); ++ic)
                for (size_t id = 0; id < s[3].e.size(); ++id) {
                    const double a = s[0].e[ia], b = s[1].e[ib], cc = s[2].e[ic], dd = s[3].e[id];
                    const double p = a + b, q = cc + dd;
                    double P[3], Q[3];
                    for (int x = 0; x < 3; ++x) {
                        P[x] = (a * s[0].c[x] + b * s[1].c[x]) / p;
                        Q[x] = (cc * s[2].c[x] + dd * s[3].c[x]) / q;
                    }
                    const double UP = s[0].k[ia] * s[1].k[ib] * std::pow(pi / p, 1.5) * std::exp(-a * b / p * d2(s[0].c, s[1].c));
                    const double UQ = s[2].k[ic] * s[3].k[id] * std::pow(pi / q, 1.5) * std::exp(-cc * dd / q * d2(s[2].c, s[3].c));
                    const double rho = p * q / (p + q);
                    const double seed = UP * UQ * 2.0 / std::sqrt(pi) * std::sqrt(rho);
                    double w[kRysMaxN];
                    static double I[kRysMaxN][3][kRysMaxE][kRysMaxE];
                    rys_tables(E, F, p, q, P, Q, s[0].c, s[2].c, tab.data(), w, I);
                    for (int i = 0; i < c.nbe; ++i)
                        for (int j = 0; j < c.nbf; ++j) {
                            double v = 0.0;
                            for (int r = 0; r < nr; ++r)
                                v += w[r] * I[r][0][eb[i][0]][fb[j][0]] * I[r][1][eb[i][1]][fb[j][1]] *
                                     I[r][2][eb[i][2]][fb[j][2]];
                            acc[(size_t)i * c.nbf + j] += seed * v;
                        }
                }
    // the class's HRR tables: bra (AB = A - B) then ket (CD = C - D)
    double AB[3], CD[3];
    for (int x = 0; x < 3; ++x) {
        AB[x] = s[0].c[x] - s[1].c[x];
        CD[x] = s[2].c[x] - s[3].c[x];
    }
    auto coef = [](const HCoef &h, const double *v) {
        return (double)h.binom * std::pow(v[0], h.px) * std::pow(v[1], h.py) * std::pow(v[2], h.pz);
    };
    std::vector<double> X((size_t)c.nab * c.nbf, 0.0);
    for (int ab = 0; ab < c.nab; ++ab)
        for (int jf = 0; jf < c.nbf; ++jf) {
            double v = 0.0;
            for (int t = c.bra_off[ab]; t < c.bra_off[ab + 1]; ++t)
                v += coef(c.cb[c.bra_terms[t].cidx], AB) * acc[(size_t)c.bra_terms[t].src * c.nbf + jf];
            X[(size_t)ab * c.nbf + jf] = v;
        }
    for (int ab = 0; ab < c.nab; ++ab)
        for (int cd = 0; cd < c.ncd; ++cd) {
            double v = 0.0;
            for (int t = c.ket_off[cd]; t < c.ket_off[cd + 1]; ++t)
                v += coef(c.ck[c.ket_terms[t].cidx], CD) * X[(size_t)ab * c.nbf + c.ket_terms[t].src];
            std::printf("%.17g\n", v);
        }
    return 0;
}
