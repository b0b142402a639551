// rys_fock.cu -- host side of the Rys Fock kernel: which classes it takes,
// its shared-memory carve-up and its launches (the kernel: rys_fock.cuh).
#include <algorithm>

#include "rys_fock.cuh"

namespace fjb {

namespace {

int rd(long n, int rsize) { return (int)((((n * rsize + 7) / 8) + 1) & ~1L); }
int dd(long n) { return (int)((n + 1) & ~1L); }

template <int LA, int LB, int LC, int LD>
bool layout_one(int max_kab, int max_kcd, int rsize, int budget, RysDev *o) {
    using S = rys::Shape<LA, LB, LC, LD>;
    const int minb = rsize == 8 ? S::template minb<double>() : S::template minb<float>();
    budget = std::min(budget, rys::rys_smem_budget(minb));
    const int nt = rsize == 8 ? S::template nt<double>() : S::template nt<float>();
    *o = RysDev{};
    o->threads = nt;
    o->kab = max_kab;
    o->kcd = max_kcd;
    const int K = max_kab * max_kcd;
    for (int G = std::min(kKetChunk, std::max(1, nt / S::NBF)); G >= 1; --G) {
        const int fixed = dd(kPrimWords * max_kab) + rd(S::NCB, rsize) + 2 * dd(S::NAB) +
                          dd((long)G * kPrimWords * max_kcd) + rd((long)G * S::NCK, rsize) + dd((long)G * S::N5) +
                          rd((long)G * S::NAB * S::XS, rsize);
        for (int P = K; P >= 1; --P) {
            const int kst = rsize == 8 ? S::template kstride<double>(P) : S::template kstride<float>(P);
            const int tabs = rd(std::max((long)G * kst, (long)G * S::NAB * S::YS), rsize);
            if (fixed + tabs > budget) continue;
            o->group = G;
            o->chunk = P;
            int off = 0;
            auto take = [&](int n) {
                const int r = off;
                off += n;
                return r;
            };
            o->sm_braP = take(dd(kPrimWords * max_kab));
            o->sm_cb = take(rd(S::NCB, rsize));
            o->sm_Dab = take(dd(S::NAB));
            o->sm_Jab = take(dd(S::NAB));
            o->sm_ketP = take(dd((long)G * kPrimWords * max_kcd));
            o->sm_ck = take(rd((long)G * S::NCK, rsize));
            o->sm_Dk = take(dd((long)G * S::N5));
            o->sm_X = take(rd((long)G * S::NAB * S::XS, rsize));
            o->sm_tab = take(tabs);
            o->sm_total = off;
            return true;
        }
    }
    return false;
}

}  // namespace

bool rys_available(int la, int lb, int lc, int ld, bool fp32) {
#define FJB_X(a, b, c, d) \
    if (la == a && lb == b && lc == c && ld == d) return true;
    if (fp32) {
        FJB_RYS32_CLASSES(FJB_X)
    } else {
        FJB_RYS64_CLASSES(FJB_X)
    }
#undef FJB_X
    return false;
}

bool rys_extra(int la, int lb, int lc, int ld) {
#define FJB_X(a, b, c, d) \
    if (la == a && lb == b && lc == c && ld == d) return true;
    FJB_RYS64_EXTRA_CLASSES(FJB_X)
#undef FJB_X
    return false;
}

bool rys_preferred(int la, int lb, int lc, int ld) {
    (void)la;
    (void)lb;
    (void)lc;
    (void)ld;
    return false;
}

bool rys_layout(int la, int lb, int lc, int ld, int max_kab, int max_kcd, bool fp32, int budget, RysDev *out) {
    const int rsize = fp32 ? 4 : 8;
#define FJB_X(a, b, c, d) \
    if (la == a && lb == b && lc == c && ld == d) return layout_one<a, b, c, d>(max_kab, max_kcd, rsize, budget, out);
    FJB_RYS64_CLASSES(FJB_X)
    FJB_RYS64_EXTRA_CLASSES(FJB_X)
#undef FJB_X
    return false;
}

// rys_fock64.cu / rys_fock32.cu: the instantiations of each precision
int rys_blocks_per_sm64(int la, int lb, int lc, int ld, const RysDev &d);
int rys_blocks_per_sm32(int la, int lb, int lc, int ld, const RysDev &d);
cudaError_t rys_launch64(int la, int lb, int lc, int ld, int grid, cudaStream_t st, const KArgs &a);
cudaError_t rys_launch32(int la, int lb, int lc, int ld, int grid, cudaStream_t st, const KArgs &a);

int rys_blocks_per_sm(int la, int lb, int lc, int ld, bool fp32, const RysDev &d) {
    return fp32 ? rys_blocks_per_sm32(la, lb, lc, ld, d) : rys_blocks_per_sm64(la, lb, lc, ld, d);
}

cudaError_t rys_launch(int la, int lb, int lc, int ld, bool fp32, int grid, cudaStream_t st, const KArgs &a) {
    return fp32 ? rys_launch32(la, lb, lc, ld, grid, st, a) : rys_launch64(la, lb, lc, ld, grid, st, a);
}

}  // namespace fjb
