// jengine.h -- the McMurchie-Davidson J-engine (host interface).
//
// J_mn = sum_ls (mn|ls) D_ls without forming (mn|ls), by the reference's
// three-step split (eri/j_coulomb/j.py:1-40, kernel_dq.py, mmd/kernel.py,
// kernel_jab.py):
//   D_q  = w sum_cd E^{cd}_q D_cd      per ket record (primitive pair),
//                                      w = 2 off the diagonal shell pair
//   J_p  = sum_k sum_q [p|q] D_q       per bra record, over every ket class,
//                                      [p|q] = (-1)^|q| R_{p+q}
//   J_ab = sum_p E^{ab}_p J_p          per unique shell pair, mirrored
// over the unique sweep's records (shell pairs a >= b by index, primitive
// pairs i outer), screened as the reference's sorted break: ket records of
// each Hermite order sorted descending by key = I_pair * max_q |D_q|, and a
// bra record stops at its first ket with I_bra * key < tau (launch.py:274-327,
// j.py:500-560).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "plan.h"

namespace fjb {

struct JEngine;

// Records and device buffers of `basis` on `device`; nullptr and *err on
// failure.
JEngine *jengine_create(const HostBasis &basis, int device, std::string *err);
void jengine_destroy(JEngine *e);

// J (n_ao^2, DEVICE, row-major; every element written) from the symmetric
// density D_dev at threshold tau.  thr32 > 0: the record pairs under it run
// their R and contraction in FP32.  boys_tab: the device Boys table.
// *launches receives the kernel launches issued.
int jengine_build(JEngine *e, const double *D_dev, double *J_dev, double tau, double thr32, const double *boys_tab,
                  cudaStream_t st, std::string *err, int *launches);

// The host plan of the same sweep, for the bit-exact comparison with the
// reference's launches(): per record in sweep order its shell pair (a, b),
// primitive index i * K_b + j, L = l_a + l_b, I_pair and ket key; and per L
// the ket records sorted descending by key (stable), concatenated L by L.
struct JHostLists {
    std::vector<int32_t> a, b, prim, L;
    std::vector<double> G, key;
    std::vector<int32_t> ket_order;  // record indices, L = 0.. in turn
    std::vector<int64_t> L_off;      // [2 * kMaxL + 2] into ket_order
};
void jengine_host_lists(const HostBasis &basis, const double *D, JHostLists *out);

}  // namespace fjb
