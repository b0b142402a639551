// rys_fock64.cu -- the Rys Fock kernel instantiated for its FP64 classes
// (FJB_RYS64_CLASSES, rys_fock.cuh); compiled apart from the other precision so
// the two build in parallel.
#include "rys_fock.cuh"

namespace fjb {

int rys_blocks_per_sm64(int la, int lb, int lc, int ld, const RysDev &d) {
#define FJB_X(a, b, c, e) \
    if (la == a && lb == b && lc == c && ld == e) return RysOne<a, b, c, e, double>::occupancy(d);
    FJB_RYS64_CLASSES(FJB_X)
    FJB_RYS64_EXTRA_CLASSES(FJB_X)
#undef FJB_X
    return 0;
}

cudaError_t rys_launch64(int la, int lb, int lc, int ld, int grid, cudaStream_t st, const KArgs &a) {
#define FJB_X(a_, b_, c_, e_) \
    if (la == a_ && lb == b_ && lc == c_ && ld == e_) return RysOne<a_, b_, c_, e_, double>::launch(grid, st, a);
    FJB_RYS64_CLASSES(FJB_X)
    FJB_RYS64_EXTRA_CLASSES(FJB_X)
#undef FJB_X
    return cudaErrorInvalidValue;
}

}  // namespace fjb
