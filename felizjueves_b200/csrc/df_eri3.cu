// df_eri3.cu -- the three-centre integral kernel (df_eri3.cuh) and its
// host side: carve-up, occupancy and launch per class.
#include <algorithm>

#include "df_eri3.cuh"

namespace fjb {

template <int LA, int LB, int LP>
struct E3Shape {
    using S = rys::Shape<LA, LB, LP, 0>;
    // the bra column in registers: 4 CTAs an SM, 2 for the long ones
    static constexpr int minb() { return S::NBE > 34 ? 2 : 4; }
};

template <int LA, int LB, int LP>
__global__ void __launch_bounds__(kE3Threads, (E3Shape<LA, LB, LP>::minb()))
    df_eri3_kernel(const E3Args A) {
    using S = rys::Shape<LA, LB, LP, 0>;
    constexpr int E = S::E, NR = S::NR;
    constexpr int RP = S::template rp<double>(), RPS = S::template rps<double>(), TSP = S::template tsp<double>();
    constexpr int NA = S::NA, NB = S::NB, NBE = S::NBE, NBF = S::NBF, NCB = S::NCB;
    constexpr const rys::CSet<LA, E> &es = rys::kCart<LA, E>;
    constexpr const rys::CSet<LA, LA> &ca = rys::kCart<LA, LA>;
    constexpr const rys::CSet<LB, LB> &cbs = rys::kCart<LB, LB>;
    constexpr const rys::HCoefs<LB> &hb = rys::kHCo<LB>;
    constexpr double kTwoOverSqrtPi = 1.1283791670955126;
    constexpr int NT = kE3Threads;

    extern __shared__ __align__(16) double sm[];
    __shared__ int s_ket[kE3Kets];
    __shared__ int s_cnt[NT / 32];
    const E3Dev &L = A.Y;
    double *braP = sm + L.sm_braP;
    double *cb = sm + L.sm_cb;
    double *ketP = sm + L.sm_ketP;
    double *tab = sm + L.sm_tab;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int G = L.group, P = L.chunk;
    const int KSTR = S::template kstride<double>(P);
    const size_t n_ao = (size_t)A.n_ao, nb = (size_t)A.nb;

    for (int u = blockIdx.x; u < A.n_units; u += gridDim.x) {
        const E3Unit U = A.units[u];
        const PairRec bra = A.pairs[U.pair];
        const int kab = bra.nprim;
        {
            const double *src = reinterpret_cast<const double *>(A.prims + bra.prim0);
            for (int i = tid; i < kab * kPrimWords; i += NT) braP[i] = src[i];
        }
        for (int i = tid; i < NCB; i += NT) cb[i] = rys::hrr_coef<LB, double>(i, bra.AB);
        // the unit's aux shells that survive the Schwarz screen, in order
        const int ik = U.k0 + tid;
        const bool on = ik < U.k1 && bra.G * A.kets[ik].G >= A.tau;
        const unsigned m = __ballot_sync(0xffffffffu, on);
        if (lane == 0) s_cnt[wid] = __popc(m);
        __syncthreads();
        int before = 0, n_list = 0;
#pragma unroll
        for (int w = 0; w < NT / 32; ++w) {
            if (w < wid) before += s_cnt[w];
            n_list += s_cnt[w];
        }
        if (on) s_ket[before + __popc(m & ((1u << lane) - 1u))] = ik;
        __syncthreads();
        const int kcd = A.kets[U.k0].nprim;  // one degree per unit
        const int K = kab * kcd;

        for (int g0 = 0; g0 < n_list; g0 += G) {
            const int ng = min(G, n_list - g0);
            for (int i = tid; i < ng * kcd * kPrimWords; i += NT) {
                const int g = i / (kcd * kPrimWords), r = i - g * (kcd * kPrimWords);
                ketP[i] = reinterpret_cast<const double *>(A.kprims + A.kets[s_ket[g0 + g]].prim0)[r];
            }
            const int gme = tid / NBF, fme = tid - gme * NBF;
            const bool item = gme < ng;
            int fx = 0, fy = 0, fz = 0;
            rys::cart_of<LP, LP>(fme, &fx, &fy, &fz);
            double acc[NBE];
#pragma unroll
            for (int e = 0; e < NBE; ++e) acc[e] = 0.0;
            for (int c0 = 0; c0 < K; c0 += P) {
                const int np = min(P, K - c0);
                __syncthreads();  // the previous chunk's tables are read; the staging above is written
                for (int it = tid; it < ng * np * NR; it += NT) {
                    const int g = it / (np * NR), rem = it - g * (np * NR), tl = rem / NR, r = rem - tl * NR;
                    const int t = c0 + tl, ikcd = t / kab, ikab = t - ikcd * kab;
                    const double *pb = braP + kPrimWords * ikab;
                    const double *pk = ketP + kPrimWords * (g * kcd + ikcd);
                    const double p = pb[6], q = pk[6];
                    const double inv = 1.0 / (p + q), rho = p * q * inv;
                    const double qi = q * inv, pi = p * inv;
                    const double PQ[3] = {pb[0] - pk[0], pb[1] - pk[1], pb[2] - pk[2]};
                    const double T = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
                    double x, w;
                    rys::rule_root<NR>(r, T, A.rys_tab, &x, &w);
                    const double seedw = pb[7] * pk[7] * kTwoOverSqrtPi * sqrt(rho) * w;
                    const double b00 = 0.5 * inv * x, b10 = pb[8] * (1.0 - qi * x), b01 = pk[8] * (1.0 - pi * x);
                    double *out = tab + (size_t)g * KSTR + (size_t)(tl * NR + r) * (3 * TSP);
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const double c00 = pb[3 + d] - qi * PQ[d] * x, c00p = pk[3 + d] + pi * PQ[d] * x;
                        double I[E + 1][LP + 1];
                        I[0][0] = d == 2 ? seedw : 1.0;
#pragma unroll
                        for (int i = 0; i < E; ++i)
                            I[i + 1][0] = c00 * I[i][0] + (i ? (double)i * b10 * I[i - 1][0] : 0.0);
#pragma unroll
                        for (int k = 0; k < LP; ++k)
#pragma unroll
                            for (int i = 0; i <= E; ++i) {
                                double v = c00p * I[i][k];
                                if (k) v += (double)k * b01 * I[i][k - 1];
                                if (i) v += (double)i * b00 * I[i - 1][k];
                                I[i][k + 1] = v;
                            }
#pragma unroll
                        for (int i = 0; i <= E; ++i)
#pragma unroll
                            for (int k = 0; k <= LP; ++k) out[d * TSP + k * RPS + i] = I[i][k];
                    }
                }
                __syncthreads();
                if (item) {
                    for (int tl = 0; tl < np; ++tl) {
                        const double *base = tab + (size_t)gme * KSTR + (size_t)tl * NR * (3 * TSP);
#pragma unroll
                        for (int r = 0; r < NR; ++r) {
                            const double *Ix = base + r * (3 * TSP), *Iy = Ix + TSP, *Iz = Iy + TSP;
                            double ix[RP], iy[RP], iz[RP];
                            rys::ld_row<double, RP>(Ix + fx * RPS, ix);
                            rys::ld_row<double, RP>(Iy + fy * RPS, iy);
                            rys::ld_row<double, RP>(Iz + fz * RPS, iz);
                            double pxy[E + 1][E + 1];
#pragma unroll
                            for (int a = 0; a <= E; ++a)
#pragma unroll
                                for (int b = 0; a + b <= E; ++b) pxy[a][b] = ix[a] * iy[b];
#pragma unroll
                            for (int e = 0; e < NBE; ++e) acc[e] += pxy[es.x[e]][es.y[e]] * iz[es.z[e]];
                        }
                    }
                }
            }
            // -- C: the bra HRR and the store, (ab|f) at [m][n][P] and its mirror
            if (item) {
                const size_t pcol = (size_t)(A.kets[s_ket[g0 + gme]].ao_a - A.p0 + fme);
                const bool mirror = bra.a != bra.b;
                const size_t rs = n_ao * nb;  // one AO row of the block
                double *o1 = A.out + ((size_t)bra.ao_a * n_ao + bra.ao_b) * nb + pcol;
                double *o2 = A.out + ((size_t)bra.ao_b * n_ao + bra.ao_a) * nb + pcol;
#pragma unroll
                for (int a = 0; a < NA; ++a)
#pragma unroll
                    for (int b = 0; b < NB; ++b) {
                        double v = 0.0;
                        int ci = hb.off[b];
#pragma unroll
                        for (int kx = 0; kx <= cbs.x[b]; ++kx)
#pragma unroll
                            for (int ky = 0; ky <= cbs.y[b]; ++ky)
#pragma unroll
                                for (int kz = 0; kz <= cbs.z[b]; ++kz, ++ci)
                                    v += cb[ci] * acc[es.idx[ca.x[a] + kx][ca.y[a] + ky][ca.z[a] + kz]];
                        o1[(size_t)a * rs + (size_t)b * nb] = v;
                        if (mirror) o2[(size_t)b * rs + (size_t)a * nb] = v;
                    }
            }
            __syncthreads();  // the group's kets are read before the next group's staging
        }
    }
}

namespace {

int dd(long n) { return (int)((n + 1) & ~1L); }

template <int LA, int LB, int LP>
struct E3One {
    static void attr() {
        static bool done = false;
        if (done) return;
        cudaFuncSetAttribute(df_eri3_kernel<LA, LB, LP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSmemBudgetDoubles * (int)sizeof(double));
        done = true;
    }
    static bool layout(int max_kab, int max_kcd, E3Dev *o) {
        using S = rys::Shape<LA, LB, LP, 0>;
        const int budget = std::min(kSmemBudgetDoubles, rys::rys_smem_budget(E3Shape<LA, LB, LP>::minb()));
        *o = E3Dev{};
        o->kab = max_kab;
        o->kcd = max_kcd;
        const int K = max_kab * max_kcd;
        for (int G = std::min(kE3Kets, kE3Threads / S::NBF); G >= 1; --G) {
            const int fixed = dd(kPrimWords * max_kab) + dd(S::NCB) + dd((long)G * kPrimWords * max_kcd);
            for (int P = K; P >= 1; --P) {
                const int tabs = dd((long)G * S::template kstride<double>(P));
                if (fixed + tabs > budget) continue;
                o->group = G;
                o->chunk = P;
                int off = 0;
                o->sm_braP = off;
                off += dd(kPrimWords * max_kab);
                o->sm_cb = off;
                off += dd(S::NCB);
                o->sm_ketP = off;
                off += dd((long)G * kPrimWords * max_kcd);
                o->sm_tab = off;
                off += tabs;
                o->sm_total = off;
                return true;
            }
        }
        return false;
    }
    static int occupancy(const E3Dev &d) {
        attr();
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, df_eri3_kernel<LA, LB, LP>, kE3Threads,
                                                      (size_t)d.sm_total * sizeof(double));
        return n;
    }
    static cudaError_t launch(int grid, cudaStream_t st, const E3Args &a) {
        attr();
        df_eri3_kernel<LA, LB, LP><<<grid, kE3Threads, (size_t)a.Y.sm_total * sizeof(double), st>>>(a);
        return cudaGetLastError();
    }
};

}  // namespace

bool eri3_layout(int la, int lb, int lp, int max_kab, int max_kcd, E3Dev *out) {
#define FJB_X(a, b, p) \
    if (la == a && lb == b && lp == p) return E3One<a, b, p>::layout(max_kab, max_kcd, out);
    FJB_E3_CLASSES(FJB_X)
#undef FJB_X
    return false;
}

int eri3_blocks_per_sm(int la, int lb, int lp, const E3Dev &d) {
#define FJB_X(a, b, p) \
    if (la == a && lb == b && lp == p) return E3One<a, b, p>::occupancy(d);
    FJB_E3_CLASSES(FJB_X)
#undef FJB_X
    return 0;
}

cudaError_t eri3_launch(int la, int lb, int lp, int grid, cudaStream_t st, const E3Args &a) {
#define FJB_X(a_, b_, p_) \
    if (la == a_ && lb == b_ && lp == p_) return E3One<a_, b_, p_>::launch(grid, st, a);
    FJB_E3_CLASSES(FJB_X)
#undef FJB_X
    return cudaErrorInvalidValue;
}

}  // namespace fjb
