// fock_compiled.cu -- instantiations of the class-templated register kernel
// for every class the generator compiled (FJB_COMPILED_CLASSES).
#include "fock_compiled.cuh"
#include "_gen/hgp_classes.cuh"

namespace fjb {

bool compiled_available(int la, int lb, int lc, int ld) {
#define FJB_X(a, b, c, d) \
    if (la == a && lb == b && lc == c && ld == d) return true;
    FJB_COMPILED_CLASSES(FJB_X)
#undef FJB_X
    return false;
}

int compiled_blocks_per_sm(int la, int lb, int lc, int ld) {
    int n = 0;
#define FJB_X(a, b, c, d)                                                                          \
    if (la == a && lb == b && lc == c && ld == d) {                                                \
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, hgp_compiled_kernel<a, b, c, d>, 128, 0); \
        return n;                                                                                  \
    }
    FJB_COMPILED_CLASSES(FJB_X)
#undef FJB_X
    return 0;
}

cudaError_t launch_compiled(int la, int lb, int lc, int ld, int grid, cudaStream_t st, const KArgs &a) {
#define FJB_X(a_, b_, c_, d_)                                                 \
    if (la == a_ && lb == b_ && lc == c_ && ld == d_) {                       \
        hgp_compiled_kernel<a_, b_, c_, d_><<<grid, 128, 0, st>>>(a);         \
        return cudaGetLastError();                                            \
    }
    FJB_COMPILED_CLASSES(FJB_X)
#undef FJB_X
    return cudaErrorInvalidValue;
}

}  // namespace fjb
