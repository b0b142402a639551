// boys_table.cpp -- the Taylor table behind the device Boys function.
//
// F_m(T_i) for T_i = i * kBoysDelta (i = 0 .. kBoysNT-1) and m = 0 ..
// kBoysMaxM, from the Kummer series
//   F_m(T) = exp(-T) sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)),
// every term positive, summed in long double (64-bit mantissa) until a term
// falls below 1e-22 of the sum, then rounded once to double.  The device
// evaluates F_M(T) = sum_{k<7} F_{M+k}(T_i) (T_i - T)^k / k! at the nearest
// node (|T_i - T| <= kBoysDelta/2 = 0.025, so the truncation is below
// 0.025^7/7! = 1.2e-15 relative) and recurs downward for m < M.  The last
// entry of each row is exp(-T_i), from which the device takes
// exp(-T) = exp(-T_i) exp(T_i - T) with an 8-term Taylor polynomial of the
// second factor (truncation below 0.025^9/9! = 1e-20 relative): the downward
// recursion's exp costs no call.
#include <cmath>
#include <vector>

#include "fjb_internal.h"

namespace fjb {

std::vector<double> boys_table() {
    std::vector<double> tab((size_t)kBoysNT * kBoysRow);
    for (int i = 0; i < kBoysNT; ++i) {
        long double T = (long double)((double)i * kBoysDelta);  // the node the device uses
        long double ex = expl(-T);
        for (int m = 0; m <= kBoysMaxM; ++m) {
            long double term = 1.0L / (2 * m + 1), sum = term;
            for (int k = 1; k < 100000; ++k) {
                term *= 2.0L * T / (long double)(2 * m + 2 * k + 1);
                sum += term;
                if (term < 1e-22L * sum) break;
            }
            tab[(size_t)i * kBoysRow + m] = (double)(ex * sum);
        }
        tab[(size_t)i * kBoysRow + kBoysMaxM + 1] = (double)ex;
    }
    return tab;
}

}  // namespace fjb
