// Evaluates the tabulated Rys rule (rys_rule.h, rys_table.cpp) on the host
// for the (n, T) pairs read from stdin, one line each: n, then the nodes and
// weights; built and run by tests/test_rys_rule.py.
#include <cstdio>

#include "rys_rule.h"

int main() {
    const std::vector<double> tab = fjb::rys_table();
    int n;
    double T;
    while (std::scanf("%d %lf", &n, &T) == 2) {
        double x[fjb::kRysMaxN], w[fjb::kRysMaxN];
        fjb::rys_rule(n, T, tab.data(), x, w);
        std::printf("%d", n);
        for (int r = 0; r < n; ++r) std::printf(" %.17g %.17g", x[r], w[r]);
        std::printf("\n");
    }
    return 0;
}
