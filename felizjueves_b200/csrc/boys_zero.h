// boys_zero.h -- F_m(0), m = 0..24, as the reference's Boys function returns
// them (reference/boys.py:218 _boys: 112-node Gauss-Legendre quadrature at
// T = 0, a few ulps from 1/(2m+1)).  Written by tests/golden/make_golden.py
// part boys_zero.  The plans' primitive Schwarz bounds read these, so the
// bounds, and the orders they decide, are the reference's to the bit.
#pragma once

namespace fjb {

constexpr int kBoysZeroMax = 24;
constexpr double kBoysZero[kBoysZeroMax + 1] = {
    0x1.0000000000000p+0,  // m = 0
    0x1.5555555555555p-2,  // m = 1
    0x1.9999999999999p-3,  // m = 2
    0x1.2492492492492p-3,  // m = 3
    0x1.c71c71c71c71dp-4,  // m = 4
    0x1.745d1745d1747p-4,  // m = 5
    0x1.3b13b13b13b15p-4,  // m = 6
    0x1.1111111111113p-4,  // m = 7
    0x1.e1e1e1e1e1e22p-5,  // m = 8
    0x1.af286bca1af2cp-5,  // m = 9
    0x1.861861861861cp-5,  // m = 10
    0x1.642c8590b2168p-5,  // m = 11
    0x1.47ae147ae147ep-5,  // m = 12
    0x1.2f684bda12f6bp-5,  // m = 13
    0x1.1a7b9611a7b99p-5,  // m = 14
    0x1.0842108421087p-5,  // m = 15
    0x1.f07c1f07c1f0dp-6,  // m = 16
    0x1.d41d41d41d422p-6,  // m = 17
    0x1.bacf914c1bad4p-6,  // m = 18
    0x1.a41a41a41a41ep-6,  // m = 19
    0x1.8f9c18f9c18fep-6,  // m = 20
    0x1.7d05f417d05f8p-6,  // m = 21
    0x1.6c16c16c16c1ap-6,  // m = 22
    0x1.5c9882b93105ap-6,  // m = 23
    0x1.4e5e0a72f053cp-6,  // m = 24
};

}  // namespace fjb
