// fock_compiled.cu -- instantiations of the class-templated register kernel
// for every class the generator compiled (FJB_COMPILED_CLASSES): the FP32
// body for all of them, the FP64 twin where it fits the register file.
#include "fock_compiled.cuh"
#include "_gen/hgp_classes.cuh"

namespace fjb {

// fp32 = true: the FP32 recurrence body; false: the FP64 one.
bool compiled_available(int la, int lb, int lc, int ld, bool fp32) {
#define FJB_X(a, b, c, d, has64) \
    if (la == a && lb == b && lc == c && ld == d) return fp32 || has64;
    FJB_COMPILED_CLASSES(FJB_X)
#undef FJB_X
    return false;
}

namespace {
template <int A, int B, int C, int D, typename R, bool OK>
struct Inst {
    static int occupancy() {
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, hgp_compiled_kernel<A, B, C, D, R>, 128, 0);
        return n;
    }
    static cudaError_t launch(int grid, cudaStream_t st, const KArgs &a) {
        hgp_compiled_kernel<A, B, C, D, R><<<grid, 128, 0, st>>>(a);
        return cudaGetLastError();
    }
};
template <int A, int B, int C, int D, typename R>
struct Inst<A, B, C, D, R, false> {
    static int occupancy() { return 0; }
    static cudaError_t launch(int, cudaStream_t, const KArgs &) { return cudaErrorInvalidValue; }
};
}  // namespace

int compiled_blocks_per_sm(int la, int lb, int lc, int ld, bool fp32) {
#define FJB_X(a, b, c, d, has64)                                                     \
    if (la == a && lb == b && lc == c && ld == d)                                    \
        return fp32 ? Inst<a, b, c, d, float, true>::occupancy()                     \
                    : Inst<a, b, c, d, double, (bool)has64>::occupancy();
    FJB_COMPILED_CLASSES(FJB_X)
#undef FJB_X
    return 0;
}

cudaError_t launch_compiled(int la, int lb, int lc, int ld, bool fp32, int grid, cudaStream_t st,
                            const KArgs &a) {
#define FJB_X(a_, b_, c_, d_, has64)                                                 \
    if (la == a_ && lb == b_ && lc == c_ && ld == d_)                                \
        return fp32 ? Inst<a_, b_, c_, d_, float, true>::launch(grid, st, a)         \
                    : Inst<a_, b_, c_, d_, double, (bool)has64>::launch(grid, st, a);
    FJB_COMPILED_CLASSES(FJB_X)
#undef FJB_X
    return cudaErrorInvalidValue;
}

}  // namespace fjb
