// onee.h -- the one-electron matrices S, T, V and h = T + V (host interface).
//
// The reference's one-electron path (one_electron/overlap.py,
// one_electron/kinetic.py, one_electron/potential.py, assembled by
// one_electron/one_electron.py:57-110): McMurchie-Davidson Hermite expansion
// of each primitive product; the overlap from E_0, the kinetic energy from
// the ket-shift identity on the overlap tables, the nuclear attraction from
// the Hermite Coulomb integrals R_tuv(p, P - C).  Every unordered shell pair
// once; a diagonal pair writes its upper triangle and the mirror, so each
// matrix is exactly symmetric.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "plan.h"

namespace fjb {

struct OneElectron;

// Shell data and the class-sorted shell-pair list of `basis` on `device`;
// nullptr and *err on failure.
OneElectron *onee_create(const HostBasis &basis, int device, std::string *err);
void onee_destroy(OneElectron *e);

// S, T, V, H = T + V (n_ao^2, DEVICE, row-major; each may be null and is then
// not written, every element of the others is written) for nuclei
// (charges[k], coords[3k..3k+2]) given on the host.  *launches receives the
// kernel launches issued.
int onee_build(OneElectron *e, const double *charges, const double *coords, int n_nuc, double *S,
               double *T, double *V, double *H, const double *boys_tab, cudaStream_t st, std::string *err,
               int *launches);

}  // namespace fjb
