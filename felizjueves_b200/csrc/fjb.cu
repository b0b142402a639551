// fjb.cu -- kernels and the C ABI of libfjb.so (include/fjb.h).
//
// Host runtime: a handle owns the basis, the plan (plan.cpp, the reference's
// f_launches), the per-class recurrence programs (hgp_tables.cpp) staged in
// device memory, and the work units.  A build is a short stream-ordered
// sequence: density blocks -> zero J', K' -> one HGP kernel per class present
// -> close (J = J' + J'^T, K = K' + K'^T, G = J - K/2).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/fjb.h"
#include "fjb_internal.h"
#include "fock_kernels.cuh"
#include "hgp_tables.h"
#include "jengine.h"
#include "onee.h"
#include "plan.h"
#include "scatter.h"
#include "router.cuh"
#include "rys_fock.cuh"
#include "df_eri3.cuh"

namespace fjb {
std::vector<double> boys_table();
// fock_compiled.cu: the class-templated register kernels
bool compiled_available(int la, int lb, int lc, int ld, bool fp32);
int compiled_blocks_per_sm(int la, int lb, int lc, int ld, bool fp32);
cudaError_t launch_compiled(int la, int lb, int lc, int ld, bool fp32, int grid, cudaStream_t st,
                            const KArgs &a);
// df_mm.cu: the DF-J/K contractions
size_t df_jk_workspace_bytes(long long nq, long long n);
cudaError_t df_jk_launch(const double *B, long long nq, long long n, const double *D, double *J, double *K,
                         void *work, int *err, cudaStream_t st);
size_t df_syrk_workspace_bytes(long long rows, long long cols);
cudaError_t df_syrk_launch(const double *Z, long long rows, long long cols, double *K, void *work, int *err,
                           cudaStream_t st);
}

using namespace fjb;

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

namespace {

constexpr double kTwoOverSqrtPi = 1.1283791670955126;

// The plan's work units, one CTA a launch, a thread a bra pair
// (write_span_units: the host's own fill of the same list).
__global__ void make_units_kernel(const UnitSpan *__restrict__ spans, Unit *__restrict__ units) {
    const UnitSpan S = spans[blockIdx.x];
    for (int ib = threadIdx.x; ib < S.n_bra; ib += blockDim.x) write_span_units(S, ib, units);
}

__global__ void density_blocks_kernel(const double *__restrict__ D, int n_ao, int n_sh,
                                      const int *__restrict__ off, const int *__restrict__ nc,
                                      double *__restrict__ Dsh) {
    int st = blockIdx.x * blockDim.x + threadIdx.x;
    if (st >= n_sh * n_sh) return;
    int s = st / n_sh, t = st % n_sh;
    double m = 0.0;
    for (int i = 0; i < nc[s]; ++i)
        for (int j = 0; j < nc[t]; ++j) {
            double v = fabs(D[(size_t)(off[s] + i) * n_ao + off[t] + j]);
            if (v > m) m = v;
        }
    Dsh[st] = m;
}

// With the budget check, the sampled FP32 units are in neither queue: their
// contribution is the sample's own FP32 build (Js32, Ks32), or its FP64 one
// (Js64, Ks64) when *flag says the FP32 queue was re-run in FP64.
__global__ void close_kernel(const double *__restrict__ Jp, const double *__restrict__ Kp, int n,
                             double *J, double *K, double *G, const double *__restrict__ Jp2 = nullptr,
                             const double *__restrict__ Kp2 = nullptr, const double *__restrict__ Js32 = nullptr,
                             const double *__restrict__ Ks32 = nullptr, const double *__restrict__ Js64 = nullptr,
                             const double *__restrict__ Ks64 = nullptr, const int *flag = nullptr) {
    size_t ij = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ij >= (size_t)n * n) return;
    size_t i = ij / n, j = ij % n, ji = j * n + i;
    double jv = Jp[ij] + Jp[ji];
    double kv = Kp[ij] + Kp[ji];
    if (Jp2) {  // the routed build's FP32-queue accumulators
        jv += Jp2[ij] + Jp2[ji];
        kv += Kp2[ij] + Kp2[ji];
    }
    if (Js32) {  // the check's sample, in the precision the verdict kept
        const bool over = *flag != 0;
        const double *Js = over ? Js64 : Js32, *Ks = over ? Ks64 : Ks32;
        jv += Js[ij] + Js[ji];
        kv += Ks[ij] + Ks[ji];
    }
    if (J) J[ij] = jv;
    if (K) K[ij] = kv;
    if (G) G[ij] = jv - 0.5 * kv;
}

// The routed build's budget check.  The sampled FP32 units are left out of
// the FP32 queue and built apart twice, in FP64 into (EJ64, EK64) and in
// FP32 into (EJ32, EK32): their G difference, closed as the build closes G,
// is the sample's own FP32 error (close_kernel adds the sample's FP32 build
// when the verdict keeps FP32, its FP64 build when it re-routes).
// Its largest element goes to *max_bits (a non-negative double's bits order
// like the double, so an integer atomicMax takes the maximum).
__global__ void route_check_kernel(const double *__restrict__ EJ64, const double *__restrict__ EK64,
                                   const double *__restrict__ EJ32, const double *__restrict__ EK32, int n,
                                   unsigned long long *max_bits) {
    double m = 0.0;
    for (size_t ij = (size_t)blockIdx.x * blockDim.x + threadIdx.x; ij < (size_t)n * n;
         ij += (size_t)gridDim.x * blockDim.x) {
        const size_t i = ij / n, j = ij % n, ji = j * n + i;
        const double dj = (EJ64[ij] - EJ32[ij]) + (EJ64[ji] - EJ32[ji]);
        const double dk = (EK64[ij] - EK32[ij]) + (EK64[ji] - EK32[ji]);
        m = fmax(m, fabs(dj - 0.5 * dk));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(max_bits, (unsigned long long)__double_as_longlong(m));
}

// The decision: the whole FP32 queue's error is estimated as sqrt(stride)
// x the sample's (every stride-th FP32 unit was sampled; units' FP32
// rounding errors are independent, so a sum over stride times the units
// grows like its square root -- on the 64-atom cluster the whole queue's
// max|dG| was 1.25 x the sample's at stride 16, under the sqrt(16) = 4 the
// estimate allows).  Over budget: *flag = 1 and
// every class's conditional count (counts[4 ri + 3]) becomes its FP32 queue
// length, so the conditional FP64 launches re-run the whole FP32 queue;
// else those counts are 0 and the launches do nothing.
__global__ void route_decide_kernel(const unsigned long long *max_bits, double stride, double budget,
                                    int *counts, int n_runs, int *flag, double *estimate) {
    const double est = sqrt(stride) * __longlong_as_double((long long)*max_bits);
    const int over = est > budget;
    if (threadIdx.x == 0) {
        *flag = over;
        *estimate = est;
    }
    for (int r = threadIdx.x; r < n_runs; r += blockDim.x) counts[4 * r + 3] = over ? counts[4 * r] : 0;
}

__global__ void zero_if_kernel(double *a, double *b, size_t n, const int *flag) {
    if (!*flag) return;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        a[i] = 0.0;
        b[i] = 0.0;
    }
}

// The batched build's per-molecule setup and close: one launch for every
// molecule (blockIdx.y is the molecule).
struct BatchMol {
    const double *D;
    double *Dsh;
    const int *sh_off, *sh_nc;  // this molecule's shell AO offsets and sizes
    int n_sh, n_ao;
    const double *Jp, *Kp;
    double *J, *K, *G;
};

__global__ void batch_density_blocks_kernel(const BatchMol *bm) {
    const BatchMol &m = bm[blockIdx.y];
    const int st = blockIdx.x * blockDim.x + threadIdx.x;
    if (st >= m.n_sh * m.n_sh) return;
    const int s = st / m.n_sh, t = st % m.n_sh;
    double v = 0.0;
    for (int i = 0; i < m.sh_nc[s]; ++i)
        for (int j = 0; j < m.sh_nc[t]; ++j) {
            const double x = fabs(m.D[(size_t)(m.sh_off[s] + i) * m.n_ao + m.sh_off[t] + j]);
            if (x > v) v = x;
        }
    m.Dsh[st] = v;
}

__global__ void batch_close_kernel(const BatchMol *bm) {
    const BatchMol &m = bm[blockIdx.y];
    const size_t nn = (size_t)m.n_ao * m.n_ao;
    for (size_t ij = (size_t)blockIdx.x * blockDim.x + threadIdx.x; ij < nn; ij += (size_t)gridDim.x * blockDim.x) {
        const size_t i = ij / m.n_ao, j = ij % m.n_ao, ji = j * m.n_ao + i;
        const double jv = m.Jp[ij] + m.Jp[ji], kv = m.Kp[ij] + m.Kp[ji];
        if (m.J) m.J[ij] = jv;
        if (m.K) m.K[ij] = kv;
        if (m.G) m.G[ij] = jv - 0.5 * kv;
    }
}

// The atomics-free build (scatter.h).  A bra segment is one bra pair of one
// launch: its units' partial bra blocks are summed in unit order into the
// segment's bra-block slots.
struct BraSeg {
    int64_t slot;     // the launch's first slot + ib * row
    int64_t wab0;     // the first unit's partial in wab
    int32_t n_units;  // consecutive units, each nab partials
    int32_t nab;
};

__global__ void bra_reduce_kernel(const BraSeg *segs, int n_segs, const double *wab, double *W) {
    for (int s = blockIdx.x; s < n_segs; s += gridDim.x) {
        const BraSeg S = segs[s];
        for (int e = threadIdx.x; e < S.nab; e += blockDim.x) {
            double v = 0.0;
            for (int u = 0; u < S.n_units; ++u) v += wab[S.wab0 + (int64_t)u * S.nab + e];
            W[S.slot + e] = v;
        }
    }
}

// One launch's scatter (kernel_f_scatter.py:1-30): a thread per element of
// J' / K' the launch touches sums that element's slots in ascending slot
// order, J' and K' apart (a slot's block, from its position in its row,
// says which: the bra block and cd are J', the other four K'), then one
// plain add per matrix.  Deterministic; no atomics.
__global__ void slot_scatter_kernel(const int32_t *el, const int32_t *ptr, const int32_t *src, int n_el,
                                    const double *W, int row, int n_ab, int n_ket, int n_cd, double *Jp,
                                    double *Kp, int n_ao) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_el) return;
    double sj = 0.0, sk = 0.0;
    for (int t = ptr[e]; t < ptr[e + 1]; ++t) {
        const int s = src[t];
        const int off = s % row;
        if (off < n_ab || (off - n_ab) / n_ket < n_cd)
            sj += W[s];
        else
            sk += W[s];
    }
    const size_t x = (size_t)el[2 * e] * n_ao + el[2 * e + 1];
    Jp[x] += sj;
    Kp[x] += sk;
}

__global__ void boys_kernel(int M, const double *T, int n, double *F, const double *tab) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double f[kBoysMaxM + 1];
    boys_eval(M, T[i], f, tab);
    for (int m = 0; m <= M; ++m) F[(size_t)i * (M + 1) + m] = f[m];
}

__global__ void screen_mask_kernel(const Unit *units, int n_units, const LaunchRec *launches,
                                   const PairRec *pairs, const double *Dsh, int n_sh, double tau,
                                   uint8_t *mask) {
    for (int u = blockIdx.x; u < n_units; u += gridDim.x) {
        const Unit U = units[u];
        const LaunchRec L = launches[U.launch];
        const PairRec bra = pairs[L.bra_pair0 + U.ib];
        const int64_t n = L.n_ket, ib = U.ib;
        const int64_t row = L.diag ? ib * n - ib * (ib - 1) / 2 - ib : ib * n;
        for (int ik = U.k0 + threadIdx.x; ik < U.k1; ik += blockDim.x) {
            const PairRec ket = pairs[L.ket_pair0 + ik];
            mask[L.qbase + row + ik] =
                skip6(Dsh, n_sh, bra.a, bra.b, ket.a, ket.b, bra.G, ket.G, tau) ? 1 : 0;
        }
    }
}

// The precision router: one warp per work unit (a lane per ket).  A unit
// whose every computed quartet has G_ab G_cd dmax under `thresh` goes to the
// FP32 queue, one with any quartet at or above it to the FP64 queue, one with
// no computed quartet to neither.  Skipping stays the six-block screen's.
__global__ void route_units_kernel(const Unit *units, int unit0, int n_units, const LaunchRec *launches,
                                   const PairRec *pairs, const double *Dsh, int n_sh, double tau,
                                   double thresh, int *list32, int *list64, int *counts, int stride,
                                   int *list_s, const MolCtx *mols = nullptr, const int32_t *launch_mol = nullptr) {
    const int lane = threadIdx.x & 31;
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    for (int i = warp; i < n_units; i += nwarps) {
        const Unit U = units[unit0 + i];
        const LaunchRec L = launches[U.launch];
        const PairRec bra = pairs[L.bra_pair0 + U.ib];
        const double *dsh = mols ? mols[launch_mol[U.launch]].Dsh : Dsh;
        const int nsh = mols ? mols[launch_mol[U.launch]].n_sh : n_sh;
        const int ik = U.k0 + lane;
        bool active = false, low = true;
        if (ik < U.k1) {
            const PairRec ket = pairs[L.ket_pair0 + ik];
            const double b = six_block_bound(dsh, nsh, bra.a, bra.b, ket.a, ket.b, bra.G, ket.G);
            active = !(b < tau);
            low = !active || b < thresh;
        }
        const bool any = __any_sync(0xffffffffu, active);
        const bool all_low = __all_sync(0xffffffffu, low);
        if (lane == 0 && any) {
            if (all_low && stride > 0 && i % stride == 0)
                list_s[atomicAdd(counts + 2, 1)] = i;  // the check's sample: built apart, twice
            else if (all_low)
                list32[atomicAdd(counts + 0, 1)] = i;
            else
                list64[atomicAdd(counts + 1, 1)] = i;
        }
    }
}

// The largest gap (decades) below the Schwarz x density bound the router's
// network is asked about by default: the range of gaps it is trained on (4.2
// observed).  fjb_router_reach narrows it to what a trained network predicts.
constexpr double kRouterMaxGap = 5.0;

// The learned router's unit split: as route_units_kernel, but a quartet the
// rigorous bound calls high may still go to FP32 when the network predicts
// its deposit under 10^log_thr -- provided its bound is within the reach
// (reach_factor = 10^decades) of the threshold; a unit with a quartet beyond
// that stays FP64 without running the network.  Screening is untouched (the
// bound decides what is skipped).

__global__ void route_units_mlp_kernel(const Unit *units, int unit0, int n_units, const LaunchRec *launches,
                                       const PairRec *pairs, const PrimRec *prims, const double *Dsh, int n_sh,
                                       double tau, double thresh, const float *params, float log_thr,
                                       double reach_factor, int la,
                                       int lb, int lc, int ld, int *list32, int *list64, int *counts,
                                       int stride, int *list_s, const MolCtx *mols = nullptr,
                                       const int32_t *launch_mol = nullptr) {
    __shared__ float sp[kNParams];
    __shared__ __align__(16) __half wh[kTcSmemHalves];
    __shared__ __align__(16) __half xs[4][32 * kXRow];  // 128 threads
    for (int i = threadIdx.x; i < kNParams; i += blockDim.x) sp[i] = params[i];
    stage_mlp_half(params, wh, wh + kHid * kW1Row);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    for (int i = warp; i < n_units; i += nwarps) {
        const Unit U = units[unit0 + i];
        const LaunchRec L = launches[U.launch];
        const PairRec bra = pairs[L.bra_pair0 + U.ib];
        const double *dsh = mols ? mols[launch_mol[U.launch]].Dsh : Dsh;
        const int nsh = mols ? mols[launch_mol[U.launch]].n_sh : n_sh;
        const int ik = U.k0 + lane;
        bool active = false, need = false, reach = true;
        PairRec ket{};
        double dmax = 0.0;
        if (ik < U.k1) {
            ket = pairs[L.ket_pair0 + ik];
            dmax = six_block_dmax(dsh, nsh, bra.a, bra.b, ket.a, ket.b);
            const double b = __dmul_rn(bra.G, __dmul_rn(ket.G, dmax));
            active = !(b < tau);
            need = active && !(b < thresh);
            // the network learned gaps below the bound of up to kRouterMaxGap
            // decades: a quartet further above the threshold cannot go FP32
            reach = !need || b < thresh * reach_factor;
        }
        const bool any = __any_sync(0xffffffffu, active);
        bool low = !need;
        // a unit goes FP32 only if all its quartets do: if one is out of the
        // network's reach the unit stays FP64 and the network is not run; it
        // runs on the whole warp (the tensor-core products take every lane)
        if (__all_sync(0xffffffffu, reach) && __any_sync(0xffffffffu, need)) {
            float f[kFeat];
            if (need)
                quartet_features(bra, ket, prims, la, lb, lc, ld, dmax, f);
            else
                for (int q = 0; q < kFeat; ++q) f[q] = sp[kOffMu + q];
            const float y = mlp_forward_tc(sp, wh, wh + kHid * kW1Row, xs[threadIdx.x >> 5], f);
            if (need) low = y < log_thr;
        }
        const bool all_low = __all_sync(0xffffffffu, low);
        if (lane == 0 && any) {
            if (all_low && stride > 0 && i % stride == 0)
                list_s[atomicAdd(counts + 2, 1)] = i;  // the check's sample: built apart, twice
            else if (all_low)
                list32[atomicAdd(counts + 0, 1)] = i;
            else
                list64[atomicAdd(counts + 1, 1)] = i;
        }
    }
}

// Features (and the six-block bound) of sampled launched quartets
// (launch, bra index, ket index), for the router's training set.
__global__ void router_features_kernel(const int32_t *samples, int n, const LaunchRec *launches,
                                       const PairRec *pairs, const PrimRec *prims, const double *Dsh, int n_sh,
                                       const int32_t *cls, float *feat, double *bound) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const LaunchRec L = launches[samples[3 * s]];
    const PairRec bra = pairs[L.bra_pair0 + samples[3 * s + 1]];
    const PairRec ket = pairs[L.ket_pair0 + samples[3 * s + 2]];
    const int32_t *c = cls + 4 * samples[3 * s];
    const double dmax = six_block_dmax(Dsh, n_sh, bra.a, bra.b, ket.a, ket.b);
    quartet_features(bra, ket, prims, c[0], c[1], c[2], c[3], dmax, feat + (size_t)kFeat * s);
    bound[s] = __dmul_rn(bra.G, __dmul_rn(ket.G, dmax));
}

// The HGP Fock kernel (file header of fock_kernels.cuh).  R is the
// recurrence type: double for the plain FP64 path; float for the routed
// path's low-magnitude units, where the VRR, the boundary and the HRR run in
// FP32 while the primitive scalars are formed, the Boys leaves evaluated
// and the digest into J and K accumulated in FP64.
//
// One CTA per work unit.  The unit's ket pairs are first screened and
// compacted (warp 0, one lane per ket); the computed kets are then taken in
// groups of G = min(C.group, slots / K) (K = the unit's primitive quartets
// per contracted quartet): the VRR runs over every (ket, primitive quartet)
// of a group at once, slot s of a chunk being flat index c0 + s = g K + t,
// so each level's barrier covers G quartets' work; each ket's boundary is
// kept apart (bound[g]), then the HRR and the digest run ket by ket.  With
// one slot the registers-held single-slot path runs instead.
template <int NT, typename R>
__global__ void __launch_bounds__(NT) hgp_fock_kernel(const KArgs A) {
    extern __shared__ __align__(16) double sm[];
    __shared__ int s_list[kKetChunk];
    __shared__ int s_n;
    const ClassDev &C = A.C;
    R *V = reinterpret_cast<R *>(sm + C.sm_V);
    R *bound_all = reinterpret_cast<R *>(sm + C.sm_bound);
    R *S = reinterpret_cast<R *>(sm + C.sm_S);
    double *braP = sm + C.sm_braP;
    double *ketP = sm + C.sm_ketP;
    R *cb = reinterpret_cast<R *>(sm + C.sm_cb);
    R *ck = reinterpret_cast<R *>(sm + C.sm_ck);
    double *Dab = sm + C.sm_D;
    double *Dcd = Dab + C.nab;
    double *Dac = Dcd + C.ncd;
    double *Dad = Dac + C.na * C.nc;
    double *Dbc = Dad + C.na * C.nd;
    double *Dbd = Dbc + C.nb * C.nc;
    double *Jab = sm + C.sm_Jab;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int slots = C.slots;
    const int na = C.na, nb = C.nb, nc = C.nc, nd = C.nd, nab = C.nab, ncd = C.ncd;
    const int nbe = C.nbe, nbf = C.nbf, L = C.L, n_ao = A.n_ao;
    const int nbnd = nbe * nbf;
    const bool tap = A.tap_out != nullptr;
    const bool hk = A.hk != 0;

    const int n_todo = A.unit_list ? *A.unit_count : A.n_units;
    for (int ui = blockIdx.x; ui < n_todo; ui += gridDim.x) {
        const int u = A.unit_list ? A.unit_list[ui] : ui;
        const Unit U = A.units[u];
        const LaunchRec LR = A.launches[U.launch];
        const PairRec bra = A.pairs[LR.bra_pair0 + U.ib];
        const int kab = bra.nprim;
        {
            const double *src = reinterpret_cast<const double *>(A.prims + bra.prim0);
            for (int i = tid; i < kab * kPrimWords; i += nt) braP[i] = src[i];
        }
        for (int i = tid; i < C.n_cb; i += nt) {
            const HCoef h = C.cb[i];
            cb[i] = (R)((double)h.binom * ipow(bra.AB[0], h.px) * ipow(bra.AB[1], h.py) *
                        ipow(bra.AB[2], h.pz));
        }
        if (!tap && !hk)
            for (int i = tid; i < nab; i += nt) {
                Dab[i] = A.D[(size_t)(bra.ao_a + i / nb) * n_ao + bra.ao_b + i % nb];
                Jab[i] = 0.0;
            }
        // the unit's computed kets, in ket order (units hold <= 32 kets)
        if (tid < 32) {
            const int ik = U.k0 + tid;
            bool on = false;
            if (ik < U.k1) {
                if (tap) {
                    on = true;
                } else if (hk) {  // K's one-block key (launch_hjk.py:153)
                    const PairRec ket = A.pairs[LR.ket_pair0 + ik];
                    const int x[4] = {bra.a, bra.b, ket.a, ket.b};
                    const int r = (LR.pad0 >> 2) & 3, s_ = (LR.pad0 >> 6) & 3;
                    on = !(bra.G * ket.G * A.Dsh[(size_t)x[r] * A.n_sh + x[s_]] < A.tau);
                } else {
                    const PairRec ket = A.pairs[LR.ket_pair0 + ik];
                    on = !skip6(A.Dsh, A.n_sh, bra.a, bra.b, ket.a, ket.b, bra.G, ket.G, A.tau);
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, on);
            if (on) s_list[__popc(m & ((1u << tid) - 1u))] = ik;
            if (tid == 0) s_n = __popc(m);
        }
        __syncthreads();
        const int n_list = s_n;
        const int kcd = A.pairs[LR.ket_pair0 + U.k0].nprim;  // a ket batch has one degree
        const int K = kab * kcd;
        const int G = slots == 1 ? 1 : max(1, min(C.group, slots / K));

        for (int g0 = 0; g0 < n_list; g0 += G) {
            const int ng = min(G, n_list - g0);
            for (int i = tid; i < ng * kcd * kPrimWords; i += nt) {
                const int g = i / (kcd * kPrimWords), r = i - g * (kcd * kPrimWords);
                const PairRec ket = A.pairs[LR.ket_pair0 + s_list[g0 + g]];
                ketP[i] = reinterpret_cast<const double *>(A.prims + ket.prim0)[r];
            }
            for (int i = tid; i < ng * nbnd; i += nt) bound_all[i] = (R)0;
            __syncthreads();

            if (slots == 1) {
                // One primitive quartet at a time (ng == 1): every thread
                // holds its scalars in registers; the Boys leaves of all K
                // primitive quartets are evaluated first, one thread each
                // (layouts give one slot only when those leaves fit).
                double *Fq = sm + C.sm_F;
                for (int t = tid; t < K; t += nt) {
                    const int ikcd = t / kab, ikab = t - ikcd * kab;
                    const double *pb = braP + kPrimWords * ikab, *pk = ketP + kPrimWords * ikcd;
                    const double p = pb[6], q = pk[6];
                    const double rho = p * q * (1.0 / (p + q));
                    const double PQx = pb[0] - pk[0], PQy = pb[1] - pk[1], PQz = pb[2] - pk[2];
                    const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
                    double F[kMaxLQuartet + 1];
                    boys_eval(L, T, F, A.boys_tab);
                    const double seed = pb[7] * pk[7] * kTwoOverSqrtPi * sqrt(rho);
                    for (int m = 0; m <= L; ++m) Fq[t * (L + 1) + m] = seed * F[m];
                }
                __syncthreads();
                for (int t = 0; t < K; ++t) {
                    const int ikcd = t / kab, ikab = t - ikcd * kab;
                    const double *pb = braP + kPrimWords * ikab, *pk = ketP + kPrimWords * ikcd;
                    const double p = pb[6], q = pk[6];
                    const double ppq = p + q, inv = 1.0 / ppq, rho = p * q * inv;
                    const double PQx = pb[0] - pk[0], PQy = pb[1] - pk[1], PQz = pb[2] - pk[2];
                    const double wp = -q * inv, wq = p * inv;
                    const R i2p = (R)pb[8], i2q = (R)pk[8];
                    const R rp = (R)(pb[8] * (q * inv)), rq = (R)(pk[8] * (p * inv)), e2 = (R)(0.5 * inv);
                    const R pa0 = (R)pb[3], pa1 = (R)pb[4], pa2 = (R)pb[5];
                    const R qc0 = (R)pk[3], qc1 = (R)pk[4], qc2 = (R)pk[5];
                    const R wp0 = (R)(wp * PQx), wp1 = (R)(wp * PQy), wp2 = (R)(wp * PQz);
                    const R wq0 = (R)(wq * PQx), wq1 = (R)(wq * PQy), wq2 = (R)(wq * PQz);
                    (void)rho;
                    if (tid == 0) V[0] = (R)0;
                    if (tid <= L) V[__ldg(C.leaf + tid)] = (R)Fq[t * (L + 1) + tid];
                    __syncthreads();
                    for (int lv = 0; lv < C.n_levels; ++lv) {
                        const int o0 = __ldg(C.level_off + lv), o1 = __ldg(C.level_off + lv + 1);
                        // Two ops of the level per thread per pass: a level's
                        // ops read only earlier levels, so both ops' loads
                        // are issued before either store (ILP across ops).
                        auto eval = [&](const VOp &op) -> R {
                            const int d = op.d;
                            R a, b, c, dd;
                            if (op.kind) {
                                a = d == 0 ? qc0 : (d == 1 ? qc1 : qc2);
                                b = d == 0 ? wq0 : (d == 1 ? wq1 : wq2);
                                c = i2q;
                                dd = rq;
                            } else {
                                a = d == 0 ? pa0 : (d == 1 ? pa1 : pa2);
                                b = d == 0 ? wp0 : (d == 1 ? wp1 : wp2);
                                c = i2p;
                                dd = rp;
                            }
                            R v = a * V[op.s0] + b * V[op.s1];
                            v += (R)op.c2 * (c * V[op.s2] - dd * V[op.s3]);
                            v += (R)op.c4 * e2 * V[op.s4];
                            return v;
                        };
                        for (int oi = o0 + tid; oi < o1; oi += 2 * nt) {
                            const int oj = oi + nt < o1 ? oi + nt : oi;
                            const uint4 ra = __ldg(reinterpret_cast<const uint4 *>(C.ops) + oi);
                            const uint4 rb = __ldg(reinterpret_cast<const uint4 *>(C.ops) + oj);
                            VOp opa, opb;
                            memcpy(&opa, &ra, sizeof(opa));
                            memcpy(&opb, &rb, sizeof(opb));
                            const R va = eval(opa), vb = eval(opb);
                            V[opa.dst] = va;
                            if (oj != oi) V[opb.dst] = vb;
                        }
                        __syncthreads();
                    }
                    for (int i = tid; i < nbnd; i += nt) bound_all[i] += V[__ldg(C.tgt + i)];
                    __syncthreads();
                }
            } else {
                const int total = ng * K;
                for (int c0 = 0; c0 < total; c0 += slots) {
                    const int ns = min(slots, total - c0);
                    for (int s = tid; s < ns; s += nt) {
                        const int fl = c0 + s, g = fl / K, t = fl - g * K;
                        const int ikcd = t / kab, ikab = t - ikcd * kab;
                        const double *pb = braP + kPrimWords * ikab, *pk = ketP + kPrimWords * (g * kcd + ikcd);
                        const double p = pb[6], q = pk[6];
                        const double ppq = p + q, inv = 1.0 / ppq, rho = p * q * inv;
                        const double PQx = pb[0] - pk[0], PQy = pb[1] - pk[1], PQz = pb[2] - pk[2];
                        const double wp = -q * inv, wq = p * inv;
                        const double inv2p = pb[8], inv2q = pk[8];
                        R *Ss = S + s;
                        Ss[0 * slots] = pb[3];
                        Ss[1 * slots] = pb[4];
                        Ss[2 * slots] = pb[5];
                        Ss[3 * slots] = wp * PQx;
                        Ss[4 * slots] = wp * PQy;
                        Ss[5 * slots] = wp * PQz;
                        Ss[6 * slots] = inv2p;
                        Ss[7 * slots] = inv2p * (q * inv);
                        Ss[8 * slots] = pk[3];
                        Ss[9 * slots] = pk[4];
                        Ss[10 * slots] = pk[5];
                        Ss[11 * slots] = wq * PQx;
                        Ss[12 * slots] = wq * PQy;
                        Ss[13 * slots] = wq * PQz;
                        Ss[14 * slots] = inv2q;
                        Ss[15 * slots] = inv2q * (p * inv);
                        Ss[16 * slots] = 0.5 * inv;
                        const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
                        double F[kMaxLQuartet + 1];
                        boys_eval(L, T, F, A.boys_tab);
                        const double seed = pb[7] * pk[7] * kTwoOverSqrtPi * sqrt(rho);
                        V[s] = (R)0;
                        for (int m = 0; m <= L; ++m) V[(size_t)__ldg(C.leaf + m) * slots + s] = (R)(seed * F[m]);
                    }
                    __syncthreads();
                    for (int lv = 0; lv < C.n_levels; ++lv) {
                        const int o0 = __ldg(C.level_off + lv), o1 = __ldg(C.level_off + lv + 1);
                        const int items = (o1 - o0) * ns;
                        // two (op, slot) items per thread per pass, as above
                        auto eval = [&](int it, VOp &op) -> R {
                            const int oi = o0 + it / ns, s = it - (it / ns) * ns;
                            const uint4 raw = __ldg(reinterpret_cast<const uint4 *>(C.ops) + oi);
                            memcpy(&op, &raw, sizeof(op));
                            const R *Ss = S + s;
                            const int base = op.kind * 8;
                            const R a = Ss[(base + op.d) * slots];
                            const R b = Ss[(base + 3 + op.d) * slots];
                            const R c = Ss[(base + 6) * slots];
                            const R dd = Ss[(base + 7) * slots];
                            const R e = Ss[16 * slots];
                            R v = a * V[(size_t)op.s0 * slots + s] + b * V[(size_t)op.s1 * slots + s];
                            v += (R)op.c2 * (c * V[(size_t)op.s2 * slots + s] - dd * V[(size_t)op.s3 * slots + s]);
                            v += (R)op.c4 * e * V[(size_t)op.s4 * slots + s];
                            return v;
                        };
                        for (int it = tid; it < items; it += 2 * nt) {
                            const int jt = it + nt < items ? it + nt : it;
                            VOp opa, opb;
                            const R va = eval(it, opa), vb = eval(jt, opb);
                            V[(size_t)opa.dst * slots + (it - (it / ns) * ns)] = va;
                            if (jt != it) V[(size_t)opb.dst * slots + (jt - (jt / ns) * ns)] = vb;
                        }
                        __syncthreads();
                    }
                    // each ket's share of this chunk into its boundary
                    const int glo = c0 / K, ghi = (c0 + ns - 1) / K;
                    for (int it = tid; it < (ghi - glo + 1) * nbnd; it += nt) {
                        const int g = glo + it / nbnd, t = it - (it / nbnd) * nbnd;
                        const int s0 = max(c0, g * K) - c0, s1 = min(c0 + ns, (g + 1) * K) - c0;
                        const size_t node = __ldg(C.tgt + t);
                        R acc = (R)0;
                        for (int s = s0; s < s1; ++s) acc += V[node * slots + s];
                        bound_all[(size_t)g * nbnd + t] += acc;
                    }
                    __syncthreads();
                }
            }

            for (int g = 0; g < ng; ++g) {
                const int ik = s_list[g0 + g];
                const PairRec ket = A.pairs[LR.ket_pair0 + ik];
                const R *bound = bound_all + (size_t)g * nbnd;
                const double deg = (bra.a == bra.b ? 0.5 : 1.0) * (ket.a == ket.b ? 0.5 : 1.0) *
                                   ((LR.diag && ik == U.ib) ? 0.5 : 1.0);
                // HRR, bra side: X[ab][f] = sum_k coefB(b,k) (a+k, 0 | f);
                // alongside, the ket's HRR coefficients and density blocks
                R *X = V, *Y = V + (size_t)nab * nbf;
                for (int i = tid; i < nab * nbf; i += nt) {
                    const int ab = i / nbf, jf = i - ab * nbf;
                    const int t0 = __ldg(C.bra_off + ab), t1 = __ldg(C.bra_off + ab + 1);
                    R acc = (R)0;
                    for (int t = t0; t < t1; ++t) {
                        const HTerm h = C.bra_terms[t];
                        acc += cb[h.cidx] * bound[h.src * nbf + jf];
                    }
                    X[i] = acc;
                }
                for (int i = tid; i < C.n_ck; i += nt) {
                    const HCoef h = C.ck[i];
                    ck[i] = (R)((double)h.binom * ipow(ket.AB[0], h.px) * ipow(ket.AB[1], h.py) *
                                ipow(ket.AB[2], h.pz));
                }
                if (!tap && !hk) {
                    const int oa = bra.ao_a, ob = bra.ao_b, oc = ket.ao_a, od = ket.ao_b;
                    for (int i = tid; i < ncd; i += nt)
                        Dcd[i] = A.D[(size_t)(oc + i / nd) * n_ao + od + i % nd];
                    for (int i = tid; i < na * nc; i += nt)
                        Dac[i] = A.D[(size_t)(oa + i / nc) * n_ao + oc + i % nc];
                    for (int i = tid; i < na * nd; i += nt)
                        Dad[i] = A.D[(size_t)(oa + i / nd) * n_ao + od + i % nd];
                    for (int i = tid; i < nb * nc; i += nt)
                        Dbc[i] = A.D[(size_t)(ob + i / nc) * n_ao + oc + i % nc];
                    for (int i = tid; i < nb * nd; i += nt)
                        Dbd[i] = A.D[(size_t)(ob + i / nd) * n_ao + od + i % nd];
                }
                __syncthreads();
                // HRR, ket side: Y[ab][cd] = sum_k coefK(d,k) X[ab][c+k]
                for (int i = tid; i < nab * ncd; i += nt) {
                    const int ab = i / ncd, cd = i - ab * ncd;
                    const int t0 = __ldg(C.ket_off + cd), t1 = __ldg(C.ket_off + cd + 1);
                    R acc = (R)0;
                    for (int t = t0; t < t1; ++t) {
                        const HTerm h = C.ket_terms[t];
                        acc += ck[h.cidx] * X[ab * nbf + h.src];
                    }
                    Y[i] = acc;
                }
                __syncthreads();
                if (tap) {
                    double *out = A.tap_out + A.tap_off[u] + (size_t)(ik - U.k0) * nab * ncd;
                    for (int i = tid; i < nab * ncd; i += nt) out[i] = Y[i];
                    __syncthreads();
                    continue;
                }
                if (hk) {
                    // K[x_p][x_q] += sum_{k, l} D[x_r][x_s] (x_0 x_1|x_2 x_3), no weight:
                    // every ordered quartet is visited once
                    const int n4[4] = {na, nb, nc, nd};
                    const int o4[4] = {bra.ao_a, bra.ao_b, ket.ao_a, ket.ao_b};
                    const int p = LR.pad0 & 3, r = (LR.pad0 >> 2) & 3, q = (LR.pad0 >> 4) & 3,
                              s_ = (LR.pad0 >> 6) & 3;
                    const int st4[4] = {nb * ncd, ncd, nd, 1};  // strides of Y[e0][e1][e2][e3]
                    for (int o = tid; o < n4[p] * n4[q]; o += nt) {
                        const int i = o / n4[q], j = o - i * n4[q];
                        double acc = 0.0;
                        for (int k = 0; k < n4[r]; ++k) {
                            const double *drow = A.D + (size_t)(o4[r] + k) * n_ao + o4[s_];
                            const R *y = Y + (size_t)i * st4[p] + (size_t)j * st4[q] + (size_t)k * st4[r];
                            for (int l = 0; l < n4[s_]; ++l) acc += drow[l] * (double)y[(size_t)l * st4[s_]];
                        }
                        atomicAdd(A.Kp + (size_t)(o4[p] + i) * n_ao + o4[q] + j, acc);
                    }
                    __syncthreads();
                    continue;
                }
                // the six-block digest (kernel_f.py:94-131): per output
                // element its contraction with one density block, then the
                // bra block into Jab (shared), the five ket blocks by FP64
                // atomics -- or, in the atomics-free build, into the
                // quartet's own slots (this order, n2..n6, is BLOCKS[1:]'s)
                {
                    const int oa = bra.ao_a, ob = bra.ao_b, oc = ket.ao_a, od = ket.ao_b;
                    const int n1 = nab, n2 = n1 + ncd, n3 = n2 + na * nc, n4 = n3 + na * nd,
                              n5 = n4 + nb * nc, n6 = n5 + nb * nd;
                    const double w2 = 2.0 * deg;
                    double *wq = A.W ? ket_slots(A, U.launch, LR.n_ket, U.ib, ik, nab, n6 - n1) : nullptr;
                    for (int o = tid; o < n6; o += nt) {
                        double acc = 0.0, w = deg;
                        size_t x = 0;  // the J' or K' element of an atomic add
                        double *M = A.Kp;
                        if (o < n1) {
                            const R *y = Y + (size_t)o * ncd;
                            for (int kl = 0; kl < ncd; ++kl) acc += Dcd[kl] * y[kl];
                            Jab[o] += w2 * acc;
                            continue;
                        } else if (o < n2) {
                            const int kl = o - n1;
                            for (int ij = 0; ij < nab; ++ij) acc += Dab[ij] * Y[(size_t)ij * ncd + kl];
                            w = w2;
                            M = A.Jp;
                            x = (size_t)(oc + kl / nd) * n_ao + od + kl % nd;
                        } else if (o < n3) {
                            const int r = o - n2, i = r / nc, k = r % nc;
                            for (int j = 0; j < nb; ++j)
                                for (int l = 0; l < nd; ++l)
                                    acc += Dbd[j * nd + l] * Y[(size_t)(i * nb + j) * ncd + k * nd + l];
                            x = (size_t)(oa + i) * n_ao + oc + k;
                        } else if (o < n4) {
                            const int r = o - n3, i = r / nd, l = r % nd;
                            for (int j = 0; j < nb; ++j)
                                for (int k = 0; k < nc; ++k)
                                    acc += Dbc[j * nc + k] * Y[(size_t)(i * nb + j) * ncd + k * nd + l];
                            x = (size_t)(oa + i) * n_ao + od + l;
                        } else if (o < n5) {
                            const int r = o - n4, j = r / nc, k = r % nc;
                            for (int i = 0; i < na; ++i)
                                for (int l = 0; l < nd; ++l)
                                    acc += Dad[i * nd + l] * Y[(size_t)(i * nb + j) * ncd + k * nd + l];
                            x = (size_t)(ob + j) * n_ao + oc + k;
                        } else {
                            const int r = o - n5, j = r / nd, l = r % nd;
                            for (int i = 0; i < na; ++i)
                                for (int k = 0; k < nc; ++k)
                                    acc += Dac[i * nc + k] * Y[(size_t)(i * nb + j) * ncd + k * nd + l];
                            x = (size_t)(ob + j) * n_ao + od + l;
                        }
                        if (wq)
                            wq[(size_t)(o - n1) * LR.n_ket] = w * acc;
                        else
                            atomicAdd(M + x, w * acc);
                    }
                }
                __syncthreads();
            }
        }
        if (!tap && !hk && A.W)
            for (int i = tid; i < nab; i += nt) A.wab[A.wab_off[u] + i] = Jab[i];  // reduced in unit order
        else if (!tap && !hk)
            for (int i = tid; i < nab; i += nt)
                atomicAdd(A.Jp + (size_t)(bra.ao_a + i / nb) * n_ao + bra.ao_b + i % nb, Jab[i]);
        if (A.computed && tid == 0 && n_list)
            atomicAdd(A.computed + U.launch, (unsigned long long)n_list);
        __syncthreads();
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// host runtime
// ---------------------------------------------------------------------------

namespace {


// A class's recurrence programs, built once per process (every handle
// uploads its own copy; the build is the costly part: about 0.2 s for all
// 54 classes, which a batch of molecules would otherwise pay per molecule).
const ClassHost &class_host_cached(int la, int lb, int lc, int ld) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int>, std::unique_ptr<ClassHost>> cache;
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_tuple(la, lb, lc, ld);
    auto it = cache.find(key);
    if (it == cache.end()) it = cache.emplace(key, std::make_unique<ClassHost>(build_class(la, lb, lc, ld))).first;
    return *it->second;
}

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { reset(); }
    void reset() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        if (count == n && p) return;
        reset();
        if (count == 0) return;
        if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) {
            p = nullptr;
            throw std::runtime_error("cudaMalloc failed");
        }
        n = count;
    }
    void upload(const std::vector<T> &v) {
        alloc(v.size());
        if (!v.empty() && cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("cudaMemcpy to device failed");
    }
};

struct ClassEntry {
    ClassHost host;
    DevBuf<int> level_off, bra_off, ket_off;
    DevBuf<VOp> ops;
    DevBuf<uint16_t> leaf, tgt;
    DevBuf<HCoef> cb, ck;
    DevBuf<HTerm> bra_terms, ket_terms;
    void upload() {
        level_off.upload(host.level_off);
        ops.upload(host.ops);
        leaf.upload(host.leaf);
        tgt.upload(host.tgt);
        cb.upload(host.cb);
        bra_off.upload(host.bra_off);
        bra_terms.upload(host.bra_terms);
        ck.upload(host.ck);
        ket_off.upload(host.ket_off);
        ket_terms.upload(host.ket_terms);
    }
    // threads/slots <= 0: the class's default configuration
    // rsize: bytes of the recurrence type (8 FP64, 4 the routed FP32 kernel)
    ClassDev dev(int max_kab, int max_kcd, int threads = 0, int slots = 0, int rsize = 8) const {
        ClassDev d;
        int th = 0, target = 0;
        default_config(host, kSmemBudgetDoubles, &th, &target);
        if (threads > 0) {
            th = threads;
            target = kSmemBudgetDoubles * threads / (16 * 32);
        }
        if (!layout_class(host, max_kab, max_kcd, kSmemBudgetDoubles, th, target, slots, &d, rsize))
            throw std::length_error("class does not fit in shared memory");
        d.level_off = level_off.p;
        d.ops = ops.p;
        d.leaf = leaf.p;
        d.tgt = tgt.p;
        d.cb = cb.p;
        d.bra_off = bra_off.p;
        d.bra_terms = bra_terms.p;
        d.ck = ck.p;
        d.ket_off = ket_off.p;
        d.ket_terms = ket_terms.p;
        return d;
    }
};

struct ClassRun {
    ClassDev dev;  // the interpreter kernel's layout (kept valid for every class)
    // the Rys kernel (rys_fock.cuh) for this class's FP64 / FP32 units, when
    // it takes the class: its carve-up, grid and the tabulated rule it reads
    bool rys64 = false, rys32 = false;
    RysDev ry64{}, ry32{};
    int grid_r64 = 0, grid_r32 = 0;
    const double *rys_tab = nullptr;
    const float *rys_tab32 = nullptr;
    ClassDev dev32;  // the FP32 interpreter's layout (routed builds of classes without has32)
    int unit0 = 0, n_units = 0;
    int grid = 0;
    int max_kab = 1, max_kcd = 1;
    bool compiled = false;  // FP64 units run on the class-templated register kernel
    bool has32 = false;     // the class has an FP32 register body (routed builds)
    int grid32 = 0;         // grid of the routed path's FP32 kernel (register or interpreter)
};

template <int NT, typename R>
int occupancy(const ClassDev &d) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hgp_fock_kernel<NT, R>, NT,
                                                  (size_t)d.sm_total * sizeof(double));
    return per_sm;
}

// Launch the HGP kernel instantiated for the class's CTA width.
template <typename R>
cudaError_t launch_hgp(const ClassDev &d, int grid, cudaStream_t st, const KArgs &a) {
    const size_t smem = (size_t)d.sm_total * sizeof(double);
    switch (d.threads) {
        case 32: hgp_fock_kernel<32, R><<<grid, 32, smem, st>>>(a); break;
        case 64: hgp_fock_kernel<64, R><<<grid, 64, smem, st>>>(a); break;
        case 128: hgp_fock_kernel<128, R><<<grid, 128, smem, st>>>(a); break;
        case 256: hgp_fock_kernel<256, R><<<grid, 256, smem, st>>>(a); break;
        case 512: hgp_fock_kernel<512, R><<<grid, 512, smem, st>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int sm_count() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// Grid of a class run: the register kernel puts one warp on a unit, four
// warps to a CTA; the interpreter one CTA on a unit.
int run_grid(const ClassRun &r);

// The FP64 path of a class run: its register kernel, else the Rys kernel,
// else the interpreter (which alone serves the atomics-free build's slots).
cudaError_t launch_run(const ClassRun &r, cudaStream_t st, const KArgs &a) {
    if (r.rys64 && !a.W) {
        KArgs ar = a;
        ar.Y = r.ry64;
        ar.rys_tab = r.rys_tab;
        ar.rys_tab32 = r.rys_tab32;
        return rys_launch(r.dev.la, r.dev.lb, r.dev.lc, r.dev.ld, false, r.grid_r64, st, ar);
    }
    if (r.compiled) return launch_compiled(r.dev.la, r.dev.lb, r.dev.lc, r.dev.ld, false, r.grid, st, a);
    return launch_hgp<double>(r.dev, r.grid, st, a);
}

// The FP32 kernel of a class run (routed builds): its register kernel, else
// the Rys kernel in FP32, else the interpreter in FP32 with its own layout.
cudaError_t launch_run32(const ClassRun &r, cudaStream_t st, const KArgs &a) {
    if (r.has32) return launch_compiled(r.dev.la, r.dev.lb, r.dev.lc, r.dev.ld, true, r.grid32, st, a);
    if (r.rys32 && !a.W) {
        KArgs ar = a;
        ar.Y = r.ry32;
        ar.rys_tab = r.rys_tab;
        ar.rys_tab32 = r.rys_tab32;
        return rys_launch(r.dev.la, r.dev.lb, r.dev.lc, r.dev.ld, true, r.grid_r32, st, ar);
    }
    KArgs a32 = a;
    a32.C = r.dev32;
    return launch_hgp<float>(r.dev32, r.grid32, st, a32);
}

}  // namespace

struct fjb_handle {
    int device = 0;
    HostBasis basis;
    fjb::JEngine *jeng = nullptr;  // the J-engine, built on first use
    fjb::OneElectron *onee = nullptr;  // the one-electron shell pairs, built on first use
    std::vector<fjb::PairBounds> pair_bounds;  // the plan's D-independent pair bounds, computed once
    int j_launches = 0;            // kernel launches of the last J-engine build
    std::string err;
    std::map<std::tuple<int, int, int, int>, std::unique_ptr<ClassEntry>> classes;
    std::map<std::tuple<int, int, int, int>, std::pair<int, int>> cfg;    // (threads, slots) overrides
    std::map<std::tuple<int, int, int, int>, std::pair<int, int>> cfg32;  // the FP32 interpreter's
    DevBuf<double> boys;
    DevBuf<double> rys;  // the tabulated Rys rule (rys_rule.h)
    DevBuf<float> rys32;  // its FP32 copy (the Rys kernel's FP32 tier)
    DevBuf<unsigned char> df_work;  // fjb_df_jk's workspace
    DevBuf<int> df_err;
    int use_rys = 1;  // which classes the Rys kernel takes (fjb_set_rys)
    DevBuf<int> sh_off, sh_nc;
    // plan
    bool planned = false;
    Plan plan;
    DevBuf<PairRec> pairs;
    DevBuf<PrimRec> prims;
    DevBuf<LaunchRec> launches;
    DevBuf<Unit> units;
    std::vector<ClassRun> runs;
    int64_t quartets_launched = 0;
    int n_units = 0;
    // host copies the atomics-free build's maps are made from (units_host
    // filled from the spans on first use: ensure_units_host)
    std::vector<UnitSpan> spans_host;
    std::vector<Unit> units_host;
    std::vector<LaunchRec> lr_host;
    std::vector<PairRec> pr_host;
    // the atomics-free build (FJB_FP64_SCATTER), staged on its first use
    struct LaunchScatter {
        int64_t el0, ptr0, src0, w0;
        int n_el, row, n_ab, n_ket, n_cd;
    };
    bool scatter_ready = false;
    std::vector<LaunchScatter> lsc;
    DevBuf<double> W, wab;
    DevBuf<int64_t> w_base, wab_off;
    DevBuf<int32_t> sc_el, sc_ptr, sc_src;
    DevBuf<BraSeg> segs;
    // build scratch
    DevBuf<double> Dsh, Jp, Kp;
    DevBuf<double> hD, hJ, hK, hG;  // fjb_fock_build_host staging
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int last_launches = 0;
    // measurement
    DevBuf<unsigned long long> computed;
    DevBuf<int> route_list, route_counts;  // the router's per-class FP32 / FP64 / sampled queues
    // the routed build's budget check (fjb_set_route_check): the FP32 queue's
    // own accumulators, the sample's FP64 and FP32 twins, the verdict
    double check_budget = 1e-8;
    int check_stride = 32;
    DevBuf<double> Jp32, Kp32, EJ64, EK64, EJ32, EK32;
    DevBuf<unsigned long long> check_max;
    DevBuf<int> check_flag;
    DevBuf<double> check_est;
    bool last_checked = false;
    std::vector<fjb_launch_stat> lstat;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> cev;
    bool built = false;
    // the learned router (fjb_router_set) and the per-launch class table it reads
    DevBuf<float> router_p;
    float router_log_thr = 0.f;
    double router_reach = 1e5;  // 10^decades (fjb_router_reach)
    int router_min_l = 0;       // classes below this total l route by the bound alone (fjb_router_classes)
    bool router_on = false;
    bool last_routed = false;
    DevBuf<int32_t> launch_cls;
    // a density-fitting handle: AO shells, then aux shells, then the unit shell
    bool df = false;
    int df_ao_shells = 0, df_aux_shells = 0;
    // the split K build's stream (fjb_hjk_plan) and its staged records
    bool hjk_planned = false, hjk_staged = false;
    HjkPlan hjk;
    DevBuf<PairRec> hk_pairs;
    DevBuf<PrimRec> hk_prims;
    DevBuf<LaunchRec> hk_launches;
    DevBuf<Unit> hk_units;
    DevBuf<unsigned long long> hk_computed;  // per launch: quartets the last fjb_hjk_k computed
    struct HkRun {
        int la, lb, lc, ld, unit0, n_units, max_kab, max_kcd;
    };
    std::vector<HkRun> hk_runs;
    // the three-centre kernel's records (fjb_df_eri3), staged on first use:
    // AO pairs (la >= lb) with their Schwarz factors, the aux shells as
    // (P, unit) pairs sorted by (l, degree, index), the per-class layouts
    bool e3_ready = false;
    DevBuf<PairRec> e3_pairs, e3_kets;
    DevBuf<PrimRec> e3_prims, e3_kprims;
    DevBuf<E3Unit> e3_units;
    std::vector<PairRec> e3_pairs_host, e3_kets_host;
    std::vector<int> e3_ket_pos;  // aux shell -> its position in the sorted list
    std::vector<int> e3_aux_off;  // aux shell -> first function in the aux basis (n_aux at the end)
    double e3_gp_max = 0.0;       // the largest aux Schwarz factor
    std::map<std::tuple<int, int, int>, E3Dev> e3_dev;
    // the captured build (fjb_fock_build_graph)
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t gexec = nullptr;
    const void *g_sig[4] = {nullptr, nullptr, nullptr, nullptr};
    int g_prec = -1;
    double g_thr = 0.0;
    void drop_graph() {
        if (gexec) cudaGraphExecDestroy(gexec);
        gexec = nullptr;
    }

    void free_class_events() {
        for (auto &e : cev) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        cev.clear();
    }
    ~fjb_handle() {
        drop_graph();
        if (cap_stream) cudaStreamDestroy(cap_stream);
        free_class_events();
    }

    ClassEntry &cls(int la, int lb, int lc, int ld) {
        auto key = std::make_tuple(la, lb, lc, ld);
        auto it = classes.find(key);
        if (it != classes.end()) return *it->second;
        auto e = std::make_unique<ClassEntry>();
        e->host = class_host_cached(la, lb, lc, ld);
        e->upload();
        auto &ref = *e;
        classes[key] = std::move(e);
        return ref;
    }
};

namespace {

thread_local std::string g_err;

int fail(fjb_handle *h, int code, const std::string &msg) {
    if (h) h->err = msg;
    g_err = msg;
    return code;
}

#define CUDA_OK(h, x)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            return fail((h), FJB_E_CUDA, std::string(#x ": ") + cudaGetErrorString(e_));     \
    } while (0)

PrimRec prim_record(const HostShell &sa, const HostShell &sb, int k) {
    const int kb = (int)sb.exps.size();
    const int i = k / kb, j = k % kb;
    const double x = sa.exps[i], y = sb.exps[j];
    const double p = x + y;
    double ab2 = 0.0;
    for (int d = 0; d < 3; ++d) ab2 += (sa.centre[d] - sb.centre[d]) * (sa.centre[d] - sb.centre[d]);
    PrimRec r;
    for (int d = 0; d < 3; ++d) {
        r.P[d] = (x * sa.centre[d] + y * sb.centre[d]) / p;
        r.X[d] = r.P[d] - sa.centre[d];
    }
    r.zeta = p;
    r.U = sa.coefs[i] * sb.coefs[j] * std::pow(M_PI / p, 1.5) * std::exp(-x * y / p * ab2);
    r.h = 0.5 / p;
    r.pad = 0.0;
    return r;
}

PairRec pair_record(const HostBasis &B, int a, int b, double G, int prim0, int nprim) {
    PairRec r{};
    r.a = a;
    r.b = b;
    r.ao_a = B.offsets[a];
    r.ao_b = B.offsets[b];
    r.prim0 = prim0;
    r.nprim = nprim;
    r.G = G;
    for (int d = 0; d < 3; ++d) r.AB[d] = B.shells[a].centre[d] - B.shells[b].centre[d];
    return r;
}

template <typename R = double>
int grid_for(const ClassDev &d, int n_units) {
    int per_sm = 0;
    switch (d.threads) {
        case 32: per_sm = occupancy<32, R>(d); break;
        case 64: per_sm = occupancy<64, R>(d); break;
        case 128: per_sm = occupancy<128, R>(d); break;
        case 256: per_sm = occupancy<256, R>(d); break;
        default: per_sm = occupancy<512, R>(d); break;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int g = std::max(1, per_sm) * sms;
    return std::max(1, std::min(n_units, g));
}

int run_grid(const ClassRun &r) {
    if (!r.compiled) return grid_for(r.dev, r.n_units);
    const int per_sm = std::max(1, compiled_blocks_per_sm(r.dev.la, r.dev.lb, r.dev.lc, r.dev.ld, false));
    const int warps_needed = (r.n_units + 3) / 4;
    return std::max(1, std::min(warps_needed, per_sm * sm_count()));
}

int run_grid32(const ClassRun &r) {
    if (!r.has32) return grid_for<float>(r.dev32, r.n_units);
    const int per_sm = std::max(1, compiled_blocks_per_sm(r.dev.la, r.dev.lb, r.dev.lc, r.dev.ld, true));
    const int warps_needed = (r.n_units + 3) / 4;
    return std::max(1, std::min(warps_needed, per_sm * sm_count()));
}

// The atomics-free build's maps and buffers (scatter.h), staged once per
// plan: the per-launch CSR maps, the slot buffer W, the per-unit bra-block
// partials and the bra segments that reduce them.  Refused when the slots
// exceed kScatterMaxSlots (2 GiB of W).
constexpr int64_t kScatterMaxSlots = int64_t(1) << 28;

// The host copy of the plan's work units (the device list's twin).
void ensure_units_host(fjb_handle *h) {
    if ((int64_t)h->units_host.size() == (int64_t)h->n_units) return;
    h->units_host.assign((size_t)h->n_units, Unit{});
    // the spans write disjoint ranges: one stride of them a host thread
    const int nt = (int)std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()),
                                         std::max<size_t>(1, h->spans_host.size() / 64));
    auto fill = [h, nt](int t) {
        for (size_t i = (size_t)t; i < h->spans_host.size(); i += (size_t)nt) {
            const UnitSpan &S = h->spans_host[i];
            for (int ib = 0; ib < S.n_bra; ++ib) write_span_units(S, ib, h->units_host.data());
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(fill, t);
    fill(0);
    for (auto &th : pool) th.join();
}

int ensure_scatter(fjb_handle *h) {
    if (h->scatter_ready) return FJB_OK;
    try {
        ensure_units_host(h);
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, std::string("work units: ") + e.what());
    }
    std::vector<int32_t> el, ptr, src;
    std::vector<int64_t> w_base;
    h->lsc.clear();
    int64_t w = 0;
    try {
        for (size_t li = 0; li < h->lr_host.size(); ++li) {
            const LaunchRec &L = h->lr_host[li];
            const fjb_launch_stat &ls = h->lstat[li];
            const int l[4] = {ls.la, ls.lb, ls.lc, ls.ld};
            std::vector<std::pair<int, int>> bra_ao, ket_ao;
            for (int i = 0; i < L.n_bra; ++i)
                bra_ao.emplace_back(h->pr_host[L.bra_pair0 + i].ao_a, h->pr_host[L.bra_pair0 + i].ao_b);
            for (int k = 0; k < L.n_ket; ++k)
                ket_ao.emplace_back(h->pr_host[L.ket_pair0 + k].ao_a, h->pr_host[L.ket_pair0 + k].ao_b);
            const ScatterMap m = scatter_map(l, bra_ao, ket_ao);
            const SlotShape S = slot_shape(l);
            fjb_handle::LaunchScatter e{};
            e.el0 = (int64_t)el.size() / 2;
            e.ptr0 = (int64_t)ptr.size();
            e.src0 = (int64_t)src.size();
            e.w0 = w;
            e.n_el = (int)m.n_el;
            e.row = S.n_ab + S.s5 * L.n_ket;
            e.n_ab = S.n_ab;
            e.n_ket = L.n_ket;
            e.n_cd = S.n_cd;
            h->lsc.push_back(e);
            w_base.push_back(w);
            w += m.n_slot;
            if (w > kScatterMaxSlots)
                return fail(h, FJB_E_LIMIT, "the atomics-free build needs more than 2^28 slots; use FJB_FP64");
            el.insert(el.end(), m.el.begin(), m.el.end());
            ptr.insert(ptr.end(), m.ptr.begin(), m.ptr.end());
            src.insert(src.end(), m.src.begin(), m.src.end());
        }
        // per unit its bra-block partial; per (launch, bra) its segment
        std::vector<int64_t> wab_off;
        std::vector<BraSeg> segs;
        int64_t at = 0;
        for (size_t u = 0; u < h->units_host.size(); ++u) {
            const Unit &U = h->units_host[u];
            const fjb_launch_stat &ls = h->lstat[U.launch];
            const int nab = (ls.la + 1) * (ls.la + 2) / 2 * ((ls.lb + 1) * (ls.lb + 2) / 2);
            wab_off.push_back(at);
            const bool same = u > 0 && h->units_host[u - 1].launch == U.launch && h->units_host[u - 1].ib == U.ib;
            if (same) {
                ++segs.back().n_units;
            } else {
                const auto &e = h->lsc[U.launch];
                segs.push_back(BraSeg{e.w0 + (int64_t)U.ib * e.row, at, 1, nab});
            }
            at += nab;
        }
        h->W.alloc(std::max<int64_t>(w, 1));
        h->wab.alloc(std::max<int64_t>(at, 1));
        h->w_base.upload(w_base);
        h->wab_off.upload(wab_off);
        h->sc_el.upload(el);
        h->sc_ptr.upload(ptr);
        h->sc_src.upload(src);
        h->segs.upload(segs);
    } catch (const std::length_error &e) {
        return fail(h, FJB_E_LIMIT, e.what());
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, e.what());
    }
    h->scatter_ready = true;
    return FJB_OK;
}

// The budget check's buffers (six n_ao^2 arrays and the verdict), made on
// the first routed build -- before a capture, by fjb_fock_build_graph.
int ensure_check(fjb_handle *h) {
    if (h->Jp32.n) return FJB_OK;
    const size_t nn = (size_t)h->basis.n_ao * h->basis.n_ao;
    try {
        h->Jp32.alloc(nn);
        h->Kp32.alloc(nn);
        h->EJ64.alloc(nn);
        h->EK64.alloc(nn);
        h->EJ32.alloc(nn);
        h->EK32.alloc(nn);
        h->check_max.alloc(1);
        h->check_flag.alloc(1);
        h->check_est.alloc(1);
    } catch (const std::exception &e) {
        h->Jp32.reset();
        return fail(h, FJB_E_CUDA, e.what());
    }
    return FJB_OK;
}

int ensure_smem_attr(fjb_handle *h) {
    static bool done = false;
    if (done) return 0;
    const int bytes = kSmemBudgetDoubles * (int)sizeof(double);
    CUDA_OK(h, cudaFuncSetAttribute(hgp_fock_kernel<32, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CUDA_OK(h, cudaFuncSetAttribute(hgp_fock_kernel<64, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CUDA_OK(h, cudaFuncSetAttribute(hgp_fock_kernel<128, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CUDA_OK(h, cudaFuncSetAttribute(hgp_fock_kernel<256, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CUDA_OK(h, cudaFuncSetAttribute(hgp_fock_kernel<512, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CUDA_OK(h, cudaFuncSetAttribute(hgp_fock_kernel<32, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CUDA_OK(h, cudaFuncSetAttribute(hgp_fock_kernel<64, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CUDA_OK(h, cudaFuncSetAttribute(hgp_fock_kernel<128, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CUDA_OK(h, cudaFuncSetAttribute(hgp_fock_kernel<256, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CUDA_OK(h, cudaFuncSetAttribute(hgp_fock_kernel<512, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    done = true;
    return 0;
}

}  // namespace

extern "C" {

const char *fjb_last_error(const fjb_handle *h) { return h ? h->err.c_str() : g_err.c_str(); }

const char *fjb_version(void) { return "fjb 0.1 sm_100a"; }

}  // extern "C"

namespace {

// Append a basis's shells to the handle's, refusing what the reference
// refuses (ao/shell.py:110-140) and l above `max_l`.
int append_shells(fjb_handle *h, const fjb_basis *b, int max_l) {
    if (!b || b->n_shells <= 0) return fail(nullptr, FJB_E_ARG, "no basis");
    int n = h->basis.n_ao;
    for (int s = 0; s < b->n_shells; ++s) {
        HostShell sh;
        sh.l = b->l[s];
        if (sh.l < 0) return fail(nullptr, FJB_E_ARG, "angular momentum is not an int >= 0");
        if (sh.l > max_l)
            return fail(nullptr, FJB_E_LIMIT, "l = " + std::to_string(sh.l) + " above the compiled maximum " +
                                                   std::to_string(max_l));
        for (int d = 0; d < 3; ++d) {
            sh.centre[d] = b->centre[3 * s + d];
            if (!std::isfinite(sh.centre[d])) return fail(nullptr, FJB_E_ARG, "centre has a non-finite entry");
        }
        if (b->nprim[s] < 1) return fail(nullptr, FJB_E_ARG, "a shell needs at least one primitive");
        for (int k = 0; k < b->nprim[s]; ++k) {
            double e = b->exps[b->prim0[s] + k], c = b->coefs[b->prim0[s] + k];
            if (!(std::isfinite(e) && e > 0)) return fail(nullptr, FJB_E_ARG, "exponents must all be finite and > 0");
            if (!std::isfinite(c)) return fail(nullptr, FJB_E_ARG, "coefficients have a non-finite entry");
            sh.exps.push_back(e);
            sh.coefs.push_back(c);
        }
        h->basis.offsets.push_back(n);
        n += (sh.l + 1) * (sh.l + 2) / 2;
        h->basis.shells.push_back(std::move(sh));
    }
    h->basis.n_ao = n;
    return FJB_OK;
}

// Device staging common to every handle: the Boys table, shell offsets and
// sizes, the build events.
// Which kernels a class run's units take from the Rys kernel: mode 0 none;
// 1 the classes without an FP64 register body, and those with one where the
// Rys kernel is the faster (rys_preferred); 2 every class it has.  FP32:
// the classes without an FP32 register body (modes 1 and 2).
void choose_rys(int mode, ClassRun &r) {
    const int la = r.dev.la, lb = r.dev.lb, lc = r.dev.lc, ld = r.dev.ld;
    const bool take64 = mode >= 1 && ((!r.compiled && rys_available(la, lb, lc, ld, false)) ||
                                      (rys_extra(la, lb, lc, ld) && (mode == 2 || rys_preferred(la, lb, lc, ld))));
    r.rys64 = take64 && rys_layout(la, lb, lc, ld, r.max_kab, r.max_kcd, false, kSmemBudgetDoubles, &r.ry64);
    r.rys32 = mode >= 1 && !r.has32 && rys_available(la, lb, lc, ld, true) &&
              rys_layout(la, lb, lc, ld, r.max_kab, r.max_kcd, true, kSmemBudgetDoubles, &r.ry32);
    const auto rgrid = [&](bool fp32, const RysDev &d) {
        const int per_sm = std::max(1, rys_blocks_per_sm(la, lb, lc, ld, fp32, d));
        return std::max(1, std::min(r.n_units, per_sm * sm_count()));
    };
    if (r.rys64) r.grid_r64 = rgrid(false, r.ry64);
    if (r.rys32) r.grid_r32 = rgrid(true, r.ry32);
}

// The Rys rule's table, built once per process (rys_table.cpp).
const std::vector<double> &rys_table_cached() {
    static std::once_flag once;
    static std::vector<double> t;
    std::call_once(once, [] { t = rys_table(); });
    return t;
}

int finish_create(std::unique_ptr<fjb_handle> &h, fjb_handle **out) {
    const int device = h->device;
    if (device < 0) {  // host-only handle: plans and exports, no builds
        *out = h.release();
        return FJB_OK;
    }
    if (cudaSetDevice(device) != cudaSuccess) return fail(nullptr, FJB_E_CUDA, "cudaSetDevice failed");
    try {
        h->boys.upload(boys_table());
        h->rys.upload(rys_table_cached());
        const std::vector<double> &t = rys_table_cached();
        h->rys32.upload(std::vector<float>(t.begin(), t.end()));
        std::vector<int> off(h->basis.offsets), nc;
        for (auto &s : h->basis.shells) nc.push_back((s.l + 1) * (s.l + 2) / 2);
        h->sh_off.upload(off);
        h->sh_nc.upload(nc);
    } catch (const std::exception &e) {
        return fail(nullptr, FJB_E_CUDA, e.what());
    }
    if (cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess)
        return fail(nullptr, FJB_E_CUDA, "cudaEventCreate failed");
    *out = h.release();
    return FJB_OK;
}

}  // namespace

extern "C" {

int fjb_create(fjb_handle **out, const fjb_basis *b, int device) {
    if (!out || !b || b->n_shells <= 0) return fail(nullptr, FJB_E_ARG, "no basis");
    auto h = std::make_unique<fjb_handle>();
    h->device = device;
    if (int rc = append_shells(h.get(), b, FJB_MAX_L)) return rc;
    return finish_create(h, out);
}

int fjb_create_df(fjb_handle **out, const fjb_basis *ao, const fjb_basis *aux, int device) {
    if (!out || !ao || !aux) return fail(nullptr, FJB_E_ARG, "no basis");
    if (device < 0) return fail(nullptr, FJB_E_ARG, "the integrals need a device");
    auto h = std::make_unique<fjb_handle>();
    h->device = device;
    if (int rc = append_shells(h.get(), ao, FJB_MAX_L)) return rc;
    h->df_ao_shells = (int)h->basis.shells.size();
    if (int rc = append_shells(h.get(), aux, FJB_MAX_L_AUX)) return rc;
    h->df_aux_shells = (int)h->basis.shells.size() - h->df_ao_shells;
    HostShell unit;  // the aux primitives' partner: exponent 0, coefficient 1
    unit.l = 0;
    unit.centre[0] = unit.centre[1] = unit.centre[2] = 0.0;
    unit.exps.push_back(0.0);
    unit.coefs.push_back(1.0);
    h->basis.offsets.push_back(h->basis.n_ao);
    h->basis.n_ao += 1;
    h->basis.shells.push_back(unit);
    h->df = true;
    return finish_create(h, out);
}

void fjb_destroy(fjb_handle *h) {
    if (!h) return;
    if (h->jeng) jengine_destroy(h->jeng);
    if (h->onee) onee_destroy(h->onee);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    delete h;
}

int fjb_n_ao(const fjb_handle *h) { return h ? h->basis.n_ao : -1; }

int fjb_plan(fjb_handle *h, const double *D_host, double tau, int n_mag) {
    if (!h || !D_host) return fail(h, FJB_E_ARG, "null argument");
    if (h->df) return fail(h, FJB_E_STATE, "a density-fitting handle has no pair stream");
    if (h->device >= 0) cudaSetDevice(h->device);
    h->planned = false;
    h->lstat.clear();
    h->drop_graph();
    try {
        unsigned nt = std::max(1u, std::thread::hardware_concurrency());
        h->plan = f_launches(h->basis, D_host, tau, n_mag, (int)nt, &h->pair_bounds);
    } catch (const std::invalid_argument &e) {
        return fail(h, FJB_E_ARG, e.what());
    } catch (const std::exception &e) {
        return fail(h, FJB_E_PLAN, e.what());
    }
    const Plan &P = h->plan;
    // stage pairs and primitive records, batch by batch
    std::vector<PairRec> pr;
    std::vector<PrimRec> pm;
    std::vector<int> batch_pair0;
    int max_deg = 1;
    for (auto &bt : P.batches) {
        batch_pair0.push_back((int)pr.size());
        if (bt.degree > FJB_MAX_PRIM_PAIRS)
            return fail(h, FJB_E_LIMIT, "degree " + std::to_string(bt.degree) +
                                            " exceeds MAX_PRIM_PAIRS = 128, the shared staging cap");
        max_deg = std::max(max_deg, bt.degree);
        for (auto &p : bt.pairs) {
            pr.push_back(pair_record(h->basis, p.a, p.b, p.G, (int)pm.size(), (int)p.prims.size()));
            for (int k : p.prims) pm.push_back(prim_record(h->basis.shells[p.a], h->basis.shells[p.b], k));
        }
    }
    // launches and work units, grouped by class
    std::vector<LaunchRec> lr;
    std::map<std::tuple<int, int, int, int>, std::vector<int>> class_launches;  // launch indices, plan order
    std::map<std::tuple<int, int, int, int>, std::pair<int, int>> class_deg;
    int64_t qbase = 0;
    for (auto &L : P.launches) {
        const PlanBatch &br = P.batches[L.first], &kt = P.batches[L.second];
        LaunchRec r{};
        r.bra_pair0 = batch_pair0[L.first];
        r.n_bra = (int)br.pairs.size();
        r.ket_pair0 = batch_pair0[L.second];
        r.n_ket = (int)kt.pairs.size();
        r.diag = L.first == L.second;
        r.qbase = qbase;
        const int64_t nq = r.diag ? (int64_t)r.n_bra * (r.n_bra + 1) / 2 : (int64_t)r.n_bra * r.n_ket;
        qbase += nq;
        auto key = std::make_tuple(br.la, br.lb, kt.la, kt.lb);
        const int li = (int)lr.size();
        lr.push_back(r);
        h->lstat.push_back(fjb_launch_stat{br.la, br.lb, kt.la, kt.lb, br.degree, kt.degree, nq, 0});
        auto &cd = class_deg[key];
        cd.first = std::max(cd.first, br.degree);
        cd.second = std::max(cd.second, kt.degree);
        class_launches[key].push_back(li);
    }
    // the work units, class by class (the map's order), each class's
    // launches in plan order: one span a launch; the units themselves are
    // written on the device (make_units_kernel), and on the host only where
    // a host copy is needed (host-only handles, the atomics-free build's
    // maps, batches), by the same write_span_units
    std::vector<UnitSpan> spans;
    std::map<std::tuple<int, int, int, int>, std::pair<int, int>> class_units;  // (first unit, count)
    int64_t n_units_total = 0;
    for (auto &kv : class_launches) {
        const int64_t u0 = n_units_total;
        for (int li : kv.second) {
            const LaunchRec &r = lr[li];
            UnitSpan S{n_units_total, 0, li, r.n_bra, r.n_ket, r.diag ? 1 : 0};
            S.count = span_units(S);
            n_units_total += S.count;
            spans.push_back(S);
        }
        if (n_units_total > (int64_t)INT32_MAX)
            return fail(h, FJB_E_LIMIT, "more than 2^31 work units: the unit indices are 32-bit");
        class_units[kv.first] = {(int)u0, (int)(n_units_total - u0)};
    }
    h->runs.clear();
    h->scatter_ready = false;
    h->lr_host = lr;
    h->pr_host = pr;
    h->spans_host = std::move(spans);
    h->units_host.clear();
    h->n_units = (int)n_units_total;
    if (h->device < 0) {  // host-only: the lists are complete, nothing is staged
        try {
            ensure_units_host(h);
        } catch (const std::exception &e) {
            return fail(h, FJB_E_LIMIT, std::string("work units: ") + e.what());
        }
        h->quartets_launched = qbase;
        h->planned = true;
        return FJB_OK;
    }
    try {
        for (auto &kv : class_units) {
            auto [la, lb, lc, ld] = kv.first;
            ClassEntry &ce = h->cls(la, lb, lc, ld);
            ClassRun run;
            auto deg = class_deg[kv.first];
            auto ov = h->cfg.find(kv.first);
            run.max_kab = deg.first;
            run.max_kcd = deg.second;
            const int th = ov == h->cfg.end() ? 0 : ov->second.first;
            run.dev = ov == h->cfg.end() || th == 1 ? ce.dev(deg.first, deg.second)
                                                     : ce.dev(deg.first, deg.second, th, ov->second.second);
            run.dev32 = ov == h->cfg.end() || th == 1
                            ? ce.dev(deg.first, deg.second, 0, 0, 4)
                            : ce.dev(deg.first, deg.second, th, ov->second.second, 4);
            auto ov32 = h->cfg32.find(kv.first);
            if (ov32 != h->cfg32.end())
                run.dev32 = ce.dev(deg.first, deg.second, ov32->second.first, ov32->second.second, 4);
            run.compiled = compiled_available(la, lb, lc, ld, false) && (th == 0 || th == 1);
            run.has32 = compiled_available(la, lb, lc, ld, true);
            run.rys_tab = h->rys.p;
            run.rys_tab32 = h->rys32.p;
            run.unit0 = kv.second.first;
            run.n_units = kv.second.second;
            h->runs.push_back(run);
        }
        h->pairs.upload(pr);
        h->prims.upload(pm);
        h->launches.upload(lr);
        h->units.alloc(std::max<int64_t>(n_units_total, 1));
        if (!h->spans_host.empty()) {
            DevBuf<UnitSpan> dspans;
            dspans.upload(h->spans_host);
            make_units_kernel<<<(unsigned)h->spans_host.size(), 128>>>(dspans.p, h->units.p);
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaStreamSynchronize(0);
            if (e != cudaSuccess) throw std::runtime_error(std::string("make_units_kernel: ") + cudaGetErrorString(e));
        }
        const size_t nn = (size_t)h->basis.n_ao * h->basis.n_ao;
        const size_t ns = h->basis.shells.size();
        h->Dsh.alloc(ns * ns);
        h->Jp.alloc(nn);
        h->Kp.alloc(nn);
    } catch (const std::length_error &e) {
        return fail(h, FJB_E_LIMIT, e.what());
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, e.what());
    }
    if (int rc = ensure_smem_attr(h)) return rc;
    for (auto &r : h->runs) {
        r.grid = run_grid(r);
        r.grid32 = run_grid32(r);
        choose_rys(h->use_rys, r);
    }
    h->free_class_events();
    for (size_t i = 0; i < h->runs.size(); ++i) {
        cudaEvent_t a, b;
        CUDA_OK(h, cudaEventCreate(&a));
        CUDA_OK(h, cudaEventCreate(&b));
        h->cev.emplace_back(a, b);
    }
    try {
        h->computed.alloc(std::max<size_t>(1, lr.size()));
        std::vector<int32_t> lc;
        for (auto &s : h->lstat) {
            lc.push_back(s.la);
            lc.push_back(s.lb);
            lc.push_back(s.lc);
            lc.push_back(s.ld);
        }
        h->launch_cls.upload(lc);
        h->route_list.alloc(std::max<size_t>(1, 3 * (size_t)h->n_units));
        h->route_counts.alloc(std::max<size_t>(1, 4 * h->runs.size()));
        if (h->Jp32.n) {  // the budget check's buffers follow the plan's size
            h->Jp32.reset();
            if (int rc = ensure_check(h)) return rc;
        }
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, e.what());
    }
    h->built = false;
    h->quartets_launched = qbase;
    h->planned = true;
    return FJB_OK;
}

int fjb_plan_units(const fjb_handle *hc, int32_t *units_host, int64_t cap, int64_t *n_units) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h || !n_units || cap < 0) return fail(h, FJB_E_ARG, "null argument");
    if (!h->planned) return fail(h, FJB_E_STATE, "no plan: call fjb_plan first");
    *n_units = h->n_units;
    if (!units_host) return FJB_OK;
    if (cap < h->n_units) return fail(h, FJB_E_ARG, "units_host holds fewer than n_units units");
    if (h->n_units == 0) return FJB_OK;
    if (h->device < 0) {
        std::memcpy(units_host, h->units_host.data(), (size_t)h->n_units * sizeof(Unit));
        return FJB_OK;
    }
    CUDA_OK(h, cudaSetDevice(h->device));
    CUDA_OK(h, cudaMemcpy(units_host, h->units.p, (size_t)h->n_units * sizeof(Unit), cudaMemcpyDeviceToHost));
    return FJB_OK;
}

int fjb_plan_counts(const fjb_handle *hc, fjb_plan_counts_t *o) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h || !o) return fail(h, FJB_E_ARG, "null argument");
    if (!h->planned) return fail(h, FJB_E_STATE, "no plan: call fjb_plan first");
    const Plan &P = h->plan;
    *o = fjb_plan_counts_t{};
    int64_t kept = 0, kprims = 0;
    for (auto &b : P.batches) {
        kept += (int64_t)b.pairs.size();
        for (auto &p : b.pairs) kprims += (int64_t)p.prims.size();
    }
    o->pairs = kept + (int64_t)P.deleted.size();
    o->pairs_deleted = (int64_t)P.deleted.size();
    o->primitive_pairs = P.n_prim_total;
    o->primitive_pairs_pruned = P.n_prim_total - kprims;
    o->batches = (int64_t)P.batches.size();
    o->batch_pairs = o->batches * (o->batches + 1) / 2;
    o->batch_pairs_screened = (int64_t)P.screened.size();
    o->launches = (int64_t)P.launches.size();
    o->kept_pairs = kept;
    o->kept_prims = kprims;
    o->units = h->n_units;
    o->quartets_launched = h->quartets_launched;
    return FJB_OK;
}

int fjb_plan_export(const fjb_handle *hc, fjb_plan_lists *o) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h || !o) return fail(h, FJB_E_ARG, "null argument");
    if (!h->planned) return fail(h, FJB_E_STATE, "no plan: call fjb_plan first");
    const Plan &P = h->plan;
    size_t ip = 0, ik = 0;
    for (size_t bi = 0; bi < P.batches.size(); ++bi) {
        const PlanBatch &b = P.batches[bi];
        if (o->batch_key) {
            o->batch_key[4 * bi + 0] = b.la;
            o->batch_key[4 * bi + 1] = b.lb;
            o->batch_key[4 * bi + 2] = b.degree;
            o->batch_key[4 * bi + 3] = b.mag;
        }
        if (o->batch_npairs) o->batch_npairs[bi] = (int)b.pairs.size();
        for (auto &p : b.pairs) {
            if (o->pair_ab) {
                o->pair_ab[2 * ip] = p.a;
                o->pair_ab[2 * ip + 1] = p.b;
            }
            if (o->pair_G) o->pair_G[ip] = p.G;
            if (o->pair_dmax) o->pair_dmax[ip] = p.dmax;
            if (o->pair_key) o->pair_key[ip] = p.key;
            if (o->pair_mag) o->pair_mag[ip] = p.mag;
            for (size_t k = 0; k < p.prims.size(); ++k, ++ik) {
                if (o->prims) o->prims[ik] = p.prims[k];
                if (o->prim_G) o->prim_G[ik] = p.prim_G[k];
            }
            ++ip;
        }
    }
    for (size_t i = 0; i < P.launches.size(); ++i)
        if (o->launches) {
            o->launches[2 * i] = P.launches[i].first;
            o->launches[2 * i + 1] = P.launches[i].second;
        }
    for (size_t i = 0; i < P.screened.size(); ++i)
        if (o->screened) {
            o->screened[2 * i] = P.screened[i].first;
            o->screened[2 * i + 1] = P.screened[i].second;
        }
    for (size_t i = 0; i < P.deleted.size(); ++i)
        if (o->deleted) {
            o->deleted[2 * i] = P.deleted[i].first;
            o->deleted[2 * i + 1] = P.deleted[i].second;
        }
    if (o->magnitudes)
        for (size_t i = 0; i < P.mags.size(); ++i) o->magnitudes[i] = P.mags[i];
    if (o->eps) *o->eps = P.eps;
    if (o->g_max) *o->g_max = P.g_max;
    return FJB_OK;
}

int fjb_screen_mask(fjb_handle *h, const double *D_dev, uint8_t *mask_dev, void *stream) {
    if (!h || !D_dev || !mask_dev) return fail(h, FJB_E_ARG, "null argument");
    if (!h->planned) return fail(h, FJB_E_STATE, "no plan: call fjb_plan first");
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    cudaSetDevice(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    const int nsh = (int)h->basis.shells.size();
    density_blocks_kernel<<<(nsh * nsh + 255) / 256, 256, 0, st>>>(D_dev, h->basis.n_ao, nsh, h->sh_off.p,
                                                                 h->sh_nc.p, h->Dsh.p);
    if (h->n_units > 0)
        screen_mask_kernel<<<std::min(h->n_units, 148 * 16), 64, 0, st>>>(
            h->units.p, h->n_units, h->launches.p, h->pairs.p, h->Dsh.p, nsh, h->plan.tau, mask_dev);
    CUDA_OK(h, cudaGetLastError());
    return FJB_OK;
}

int fjb_fock_build(fjb_handle *h, const double *D_dev, double *J_dev, double *K_dev, double *G_dev,
                   int precision, double threshold, void *stream) {
    if (!h || !D_dev) return fail(h, FJB_E_ARG, "null argument");
    if (!h->planned) return fail(h, FJB_E_STATE, "no plan: call fjb_plan first");
    if (precision != FJB_FP64 && precision != FJB_ROUTED && precision != FJB_FP64_SCATTER)
        return fail(h, FJB_E_ARG, "unknown precision mode");
    const double route = precision == FJB_ROUTED ? (threshold > 0.0 ? threshold : 1e-9) : 0.0;
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    cudaSetDevice(h->device);
    const bool scatter = precision == FJB_FP64_SCATTER;
    if (scatter)
        if (int rc = ensure_scatter(h)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int nsh = (int)h->basis.shells.size(), nao = h->basis.n_ao;
    const size_t nn = (size_t)nao * nao;
    int launches = 0;
    density_blocks_kernel<<<(nsh * nsh + 255) / 256, 256, 0, st>>>(D_dev, nao, nsh, h->sh_off.p, h->sh_nc.p,
                                                                 h->Dsh.p);
    ++launches;
    CUDA_OK(h, cudaMemsetAsync(h->Jp.p, 0, nn * sizeof(double), st));
    CUDA_OK(h, cudaMemsetAsync(h->Kp.p, 0, nn * sizeof(double), st));
    CUDA_OK(h, cudaMemsetAsync(h->computed.p, 0, h->computed.n * sizeof(unsigned long long), st));
    const bool routed = route > 0.0;
    h->last_routed = routed;
    const bool check = routed && h->check_budget > 0.0;
    h->last_checked = check;
    if (check)
        if (int rc = ensure_check(h)) return rc;
    if (routed) CUDA_OK(h, cudaMemsetAsync(h->route_counts.p, 0, h->route_counts.n * sizeof(int), st));
    if (check) {
        for (double *b : {h->Jp32.p, h->Kp32.p, h->EJ64.p, h->EK64.p, h->EJ32.p, h->EK32.p})
            CUDA_OK(h, cudaMemsetAsync(b, 0, nn * sizeof(double), st));
        CUDA_OK(h, cudaMemsetAsync(h->check_max.p, 0, sizeof(unsigned long long), st));
    }
    if (scatter) {  // unwritten slots (screened quartets, the canonical half) must hold zero
        CUDA_OK(h, cudaMemsetAsync(h->W.p, 0, h->W.n * sizeof(double), st));
        CUDA_OK(h, cudaMemsetAsync(h->wab.p, 0, h->wab.n * sizeof(double), st));
    }
    // Under stream capture the timing events become event-record nodes of
    // the graph (External), so every replay records them and the class and
    // build timings read after a replay are that replay's.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_OK(h, cudaStreamIsCapturing(st, &cap));
    const unsigned ev_flags = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : 0u;
    CUDA_OK(h, cudaEventRecordWithFlags(h->ev0, st, ev_flags));
    for (size_t ri = 0; ri < h->runs.size(); ++ri) {
        const ClassRun &r = h->runs[ri];
        CUDA_OK(h, cudaEventRecordWithFlags(h->cev[ri].first, st, ev_flags));
        KArgs a{};
        a.computed = h->computed.p;
        a.C = r.dev;
        a.units = h->units.p + r.unit0;
        a.n_units = r.n_units;
        a.launches = h->launches.p;
        a.pairs = h->pairs.p;
        a.prims = h->prims.p;
        a.D = D_dev;
        a.Dsh = h->Dsh.p;
        a.n_sh = nsh;
        a.n_ao = nao;
        a.tau = h->plan.tau;
        a.Jp = h->Jp.p;
        a.Kp = h->Kp.p;
        a.boys_tab = h->boys.p;
        a.route_thresh = route;
        if (scatter) {
            a.W = h->W.p;
            a.w_base = h->w_base.p;
            a.wab = h->wab.p;
            a.wab_off = h->wab_off.p + r.unit0;
        }
        if (routed) {
            // the precision router splits the class's units into an FP32 and
            // an FP64 queue; each queue has its own kernel
            int *l32 = h->route_list.p + r.unit0;
            int *l64 = h->route_list.p + h->n_units + r.unit0;
            int *ls = h->route_list.p + 2 * (size_t)h->n_units + r.unit0;
            int *cnt = h->route_counts.p + 4 * ri;
            const int stride = check ? h->check_stride : 0;
            const int rgrid = std::max(1, std::min((r.n_units + 3) / 4, 16 * sm_count()));
            if (h->router_on && r.dev.la + r.dev.lb + r.dev.lc + r.dev.ld >= h->router_min_l)
                route_units_mlp_kernel<<<rgrid, 128, 0, st>>>(
                    h->units.p, r.unit0, r.n_units, h->launches.p, h->pairs.p, h->prims.p, h->Dsh.p, nsh,
                    h->plan.tau, route, h->router_p.p, h->router_log_thr, h->router_reach, r.dev.la, r.dev.lb,
                    r.dev.lc, r.dev.ld,
                    l32, l64, cnt, stride, ls);
            else
                route_units_kernel<<<rgrid, 128, 0, st>>>(h->units.p, r.unit0, r.n_units, h->launches.p,
                                                          h->pairs.p, h->Dsh.p, nsh, h->plan.tau, route, l32,
                                                          l64, cnt, stride, ls);
            KArgs a32 = a, a64 = a;
            a32.unit_list = l32;
            a32.unit_count = cnt;
            a64.unit_list = l64;
            a64.unit_count = cnt + 1;
            if (check) {  // the FP32 queue into its own accumulators
                a32.Jp = h->Jp32.p;
                a32.Kp = h->Kp32.p;
            }
            CUDA_OK(h, launch_run32(r, st, a32));
            CUDA_OK(h, launch_run(r, st, a64));
            launches += 3;
            if (check) {  // the sample of the FP32 queue, in FP32 and in FP64
                KArgs s32 = a32, s64 = a64;
                s32.unit_list = s64.unit_list = ls;
                s32.unit_count = s64.unit_count = cnt + 2;
                s32.Jp = h->EJ32.p;
                s32.Kp = h->EK32.p;
                s64.Jp = h->EJ64.p;
                s64.Kp = h->EK64.p;
                s32.computed = s64.computed = nullptr;
                CUDA_OK(h, launch_run32(r, st, s32));
                CUDA_OK(h, launch_run(r, st, s64));
                launches += 2;
            }
        } else {
            CUDA_OK(h, launch_run(r, st, a));
            ++launches;
        }
        CUDA_OK(h, cudaEventRecordWithFlags(h->cev[ri].second, st, ev_flags));
    }
    if (scatter) {
        // the bra blocks' partials in unit order, then each launch's scatter
        // in launch order: J' and K' are the same sums in the same order on
        // every build
        const int ns = (int)h->segs.n;
        bra_reduce_kernel<<<std::max(1, std::min(ns, 148 * 16)), 128, 0, st>>>(h->segs.p, ns, h->wab.p, h->W.p);
        ++launches;
        for (const auto &e : h->lsc) {
            if (e.n_el == 0) continue;
            slot_scatter_kernel<<<(e.n_el + 127) / 128, 128, 0, st>>>(
                h->sc_el.p + 2 * e.el0, h->sc_ptr.p + e.ptr0, h->sc_src.p + e.src0, e.n_el, h->W.p + e.w0, e.row,
                e.n_ab, e.n_ket, e.n_cd, h->Jp.p, h->Kp.p, nao);
            ++launches;
        }
    }
    if (check) {
        // the verdict, then the FP64 re-run of every FP32 queue if it is
        // over budget (the conditional counts are 0 otherwise)
        const int cgrid = std::max(1, std::min((int)((nn + 255) / 256), 8 * sm_count()));
        route_check_kernel<<<cgrid, 256, 0, st>>>(h->EJ64.p, h->EK64.p, h->EJ32.p, h->EK32.p, nao, h->check_max.p);
        route_decide_kernel<<<1, 256, 0, st>>>(h->check_max.p, (double)h->check_stride, h->check_budget,
                                               h->route_counts.p, (int)h->runs.size(), h->check_flag.p,
                                               h->check_est.p);
        zero_if_kernel<<<cgrid, 256, 0, st>>>(h->Jp32.p, h->Kp32.p, nn, h->check_flag.p);
        launches += 3;
        for (size_t ri = 0; ri < h->runs.size(); ++ri) {
            const ClassRun &r = h->runs[ri];
            KArgs a{};
            a.C = r.dev;
            a.units = h->units.p + r.unit0;
            a.n_units = r.n_units;
            a.launches = h->launches.p;
            a.pairs = h->pairs.p;
            a.prims = h->prims.p;
            a.D = D_dev;
            a.Dsh = h->Dsh.p;
            a.n_sh = nsh;
            a.n_ao = nao;
            a.tau = h->plan.tau;
            a.Jp = h->Jp32.p;
            a.Kp = h->Kp32.p;
            a.boys_tab = h->boys.p;
            a.unit_list = h->route_list.p + r.unit0;
            a.unit_count = h->route_counts.p + 4 * ri + 3;
            CUDA_OK(h, launch_run(r, st, a));
            ++launches;
        }
    }
    h->built = true;
    CUDA_OK(h, cudaEventRecordWithFlags(h->ev1, st, ev_flags));
    close_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(
        h->Jp.p, h->Kp.p, nao, J_dev, K_dev, G_dev, check ? h->Jp32.p : nullptr, check ? h->Kp32.p : nullptr,
        check ? h->EJ32.p : nullptr, check ? h->EK32.p : nullptr, check ? h->EJ64.p : nullptr,
        check ? h->EK64.p : nullptr, check ? h->check_flag.p : nullptr);
    ++launches;
    CUDA_OK(h, cudaGetLastError());
    h->last_launches = launches;
    return FJB_OK;
}

int fjb_fock_build_graph(fjb_handle *h, const double *D_dev, double *J_dev, double *K_dev, double *G_dev,
                         int precision, double threshold, void *stream) {
    if (!h || !D_dev) return fail(h, FJB_E_ARG, "null argument");
    if (!h->planned) return fail(h, FJB_E_STATE, "no plan: call fjb_plan first");
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    CUDA_OK(h, cudaSetDevice(h->device));
    if (precision == FJB_FP64_SCATTER)  // staging allocates: before the capture
        if (int rc = ensure_scatter(h)) return rc;
    if (precision == FJB_ROUTED && h->check_budget > 0.0)
        if (int rc = ensure_check(h)) return rc;
    const void *sig[4] = {D_dev, J_dev, K_dev, G_dev};
    const bool same = h->gexec && std::equal(sig, sig + 4, h->g_sig) && h->g_prec == precision &&
                      h->g_thr == threshold;
    if (!same) {
        h->drop_graph();
        if (!h->cap_stream) CUDA_OK(h, cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking));
        CUDA_OK(h, cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeThreadLocal));
        const int rc = fjb_fock_build(h, D_dev, J_dev, K_dev, G_dev, precision, threshold, h->cap_stream);
        cudaGraph_t graph = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(h->cap_stream, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ec != cudaSuccess) return fail(h, FJB_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
        const cudaError_t ei = cudaGraphInstantiate(&h->gexec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) {
            h->gexec = nullptr;
            return fail(h, FJB_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
        }
        std::copy(sig, sig + 4, h->g_sig);
        h->g_prec = precision;
        h->g_thr = threshold;
    }
    CUDA_OK(h, cudaGraphLaunch(h->gexec, (cudaStream_t)stream));
    return FJB_OK;
}

int fjb_fock_build_host(fjb_handle *h, const double *D_host, double *J_host, double *K_host,
                        double *G_host, int precision, double threshold) {
    if (!h || !D_host) return fail(h, FJB_E_ARG, "null argument");
    if (!h->planned) return fail(h, FJB_E_STATE, "no plan: call fjb_plan first");
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    cudaSetDevice(h->device);
    const size_t nn = (size_t)h->basis.n_ao * h->basis.n_ao;
    try {
        h->hD.alloc(nn);
        h->hJ.alloc(nn);
        h->hK.alloc(nn);
        h->hG.alloc(nn);
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, e.what());
    }
    CUDA_OK(h, cudaMemcpy(h->hD.p, D_host, nn * sizeof(double), cudaMemcpyHostToDevice));
    int rc = fjb_fock_build(h, h->hD.p, J_host ? h->hJ.p : nullptr, K_host ? h->hK.p : nullptr,
                            G_host ? h->hG.p : nullptr, precision, threshold, nullptr);
    if (rc) return rc;
    if (J_host) CUDA_OK(h, cudaMemcpy(J_host, h->hJ.p, nn * sizeof(double), cudaMemcpyDeviceToHost));
    if (K_host) CUDA_OK(h, cudaMemcpy(K_host, h->hK.p, nn * sizeof(double), cudaMemcpyDeviceToHost));
    if (G_host) CUDA_OK(h, cudaMemcpy(G_host, h->hG.p, nn * sizeof(double), cudaMemcpyDeviceToHost));
    CUDA_OK(h, cudaDeviceSynchronize());
    return FJB_OK;
}

namespace {
// The ERI tap: the interpreter kernel in tap mode, FP64 or (fp32) with the
// routed path's FP32 recurrences.
int eri_blocks_impl(fjb_handle *h, const int32_t *quartets, int n, double *out_dev, int64_t *offsets, bool fp32) {
    if (!h || !quartets || n < 0 || !offsets) return fail(h, FJB_E_ARG, "null argument");
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    cudaSetDevice(h->device);
    const int nsh = (int)h->basis.shells.size();
    struct Item {
        int q;
        std::tuple<int, int, int, int> key;
    };
    std::vector<PairRec> pr;
    std::vector<PrimRec> pm;
    std::vector<LaunchRec> lr;
    std::map<std::tuple<int, int, int, int>, std::vector<int>> by_class;
    std::map<std::tuple<int, int, int, int>, std::pair<int, int>> deg;
    offsets[0] = 0;
    auto add_pair = [&](int a, int b) {
        const HostShell &sa = h->basis.shells[a], &sb = h->basis.shells[b];
        int K = (int)(sa.exps.size() * sb.exps.size());
        if (K > FJB_MAX_PRIM_PAIRS) throw std::length_error("degree exceeds MAX_PRIM_PAIRS = 128");
        pr.push_back(pair_record(h->basis, a, b, 0.0, (int)pm.size(), K));
        for (int k = 0; k < K; ++k) pm.push_back(prim_record(sa, sb, k));
        return K;
    };
    try {
        for (int i = 0; i < n; ++i) {
            int q[4];
            for (int k = 0; k < 4; ++k) {
                q[k] = quartets[4 * i + k];
                if (q[k] < 0 || q[k] >= nsh) return fail(h, FJB_E_ARG, "shell index out of range");
            }
            int nabcd = 1;
            for (int k = 0; k < 4; ++k) nabcd *= ncart(h->basis.shells[q[k]].l);
            offsets[i + 1] = offsets[i] + nabcd;
            LaunchRec r{};
            r.bra_pair0 = (int)pr.size();
            r.n_bra = 1;
            int kab = add_pair(q[0], q[1]);
            r.ket_pair0 = (int)pr.size();
            r.n_ket = 1;
            int kcd = add_pair(q[2], q[3]);
            lr.push_back(r);
            auto key = std::make_tuple(h->basis.shells[q[0]].l, h->basis.shells[q[1]].l, h->basis.shells[q[2]].l,
                                       h->basis.shells[q[3]].l);
            by_class[key].push_back(i);
            auto &d = deg[key];
            d.first = std::max(d.first, kab);
            d.second = std::max(d.second, kcd);
        }
        DevBuf<PairRec> dpr;
        DevBuf<PrimRec> dpm;
        DevBuf<LaunchRec> dlr;
        dpr.upload(pr);
        dpm.upload(pm);
        dlr.upload(lr);
        if (int rc = ensure_smem_attr(h)) return rc;
        for (auto &kv : by_class) {
            auto [la, lb, lc, ld] = kv.first;
            ClassEntry &ce = h->cls(la, lb, lc, ld);
            ClassDev dev = fp32 ? ce.dev(deg[kv.first].first, deg[kv.first].second, 0, 0, 4)
                                : ce.dev(deg[kv.first].first, deg[kv.first].second);
            std::vector<Unit> us;
            std::vector<int64_t> toff;
            for (int qi : kv.second) {
                us.push_back(Unit{qi, 0, 0, 1});
                toff.push_back(offsets[qi]);
            }
            DevBuf<Unit> du;
            DevBuf<int64_t> dto;
            du.upload(us);
            dto.upload(toff);
            KArgs a{};
            a.C = dev;
            a.units = du.p;
            a.n_units = (int)us.size();
            a.launches = dlr.p;
            a.pairs = dpr.p;
            a.prims = dpm.p;
            a.n_sh = nsh;
            a.n_ao = h->basis.n_ao;
            a.tau = -1.0;
            a.tap_out = out_dev;
            a.tap_off = dto.p;
            a.boys_tab = h->boys.p;
            if (fp32)
                CUDA_OK(h, launch_hgp<float>(dev, grid_for<float>(dev, a.n_units), nullptr, a));
            else
                CUDA_OK(h, launch_hgp<double>(dev, grid_for(dev, a.n_units), nullptr, a));
            CUDA_OK(h, cudaDeviceSynchronize());
        }
    } catch (const std::length_error &e) {
        return fail(h, FJB_E_LIMIT, e.what());
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, e.what());
    }
    return FJB_OK;
}
}  // namespace

int fjb_eri_blocks(fjb_handle *h, const int32_t *quartets, int n, double *out_dev, int64_t *offsets) {
    return eri_blocks_impl(h, quartets, n, out_dev, offsets, false);
}

int fjb_eri_blocks_fp32(fjb_handle *h, const int32_t *quartets, int n, double *out_dev, int64_t *offsets) {
    return eri_blocks_impl(h, quartets, n, out_dev, offsets, true);
}

int fjb_set_route_check(fjb_handle *h, double budget, int stride) {
    if (!h) return fail(h, FJB_E_ARG, "null handle");
    if (!(budget == budget) || stride < 1) return fail(h, FJB_E_ARG, "fjb_set_route_check: budget must be a number, stride >= 1");
    h->check_budget = budget;
    h->check_stride = stride;
    h->drop_graph();
    return FJB_OK;
}

int fjb_route_check_result(const fjb_handle *hc, double *estimate, int *rerouted) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h || !estimate || !rerouted) return fail(h, FJB_E_ARG, "null argument");
    if (!h->built || !h->last_checked) return fail(h, FJB_E_STATE, "the last build was not a checked routed build");
    CUDA_OK(h, cudaEventSynchronize(h->ev1));
    CUDA_OK(h, cudaDeviceSynchronize());
    CUDA_OK(h, cudaMemcpy(estimate, h->check_est.p, sizeof(double), cudaMemcpyDeviceToHost));
    CUDA_OK(h, cudaMemcpy(rerouted, h->check_flag.p, sizeof(int), cudaMemcpyDeviceToHost));
    return FJB_OK;
}

int fjb_route_stats(const fjb_handle *hc, int64_t *n32, int64_t *n64) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h || !n32 || !n64) return fail(h, FJB_E_ARG, "null argument");
    if (!h->built) return fail(h, FJB_E_STATE, "no build yet");
    CUDA_OK(h, cudaEventSynchronize(h->ev1));
    std::vector<int> c(h->route_counts.n, 0);
    if (!c.empty())
        CUDA_OK(h, cudaMemcpy(c.data(), h->route_counts.p, c.size() * sizeof(int), cudaMemcpyDeviceToHost));
    *n32 = 0;
    *n64 = 0;
    for (size_t ri = 0; ri < h->runs.size(); ++ri) {
        if (h->last_routed) {
            *n32 += c[4 * ri] + (h->last_checked ? c[4 * ri + 2] : 0);  // the check's sample is FP32 too
            *n64 += c[4 * ri + 1];
        } else {
            *n64 += h->runs[ri].n_units;
        }
    }
    return FJB_OK;
}

int fjb_router_reach(fjb_handle *h, double decades) {
    if (!h) return fail(h, FJB_E_ARG, "null handle");
    if (!(decades >= 0.0 && decades <= kRouterMaxGap))
        return fail(h, FJB_E_ARG, "fjb_router_reach: decades must be in [0, 5]");
    h->router_reach = std::pow(10.0, decades);
    h->drop_graph();
    return FJB_OK;
}

int fjb_router_classes(fjb_handle *h, int min_total_l) {
    if (!h) return fail(h, FJB_E_ARG, "null handle");
    if (min_total_l < 0 || min_total_l > 4 * FJB_MAX_L + 1)
        return fail(h, FJB_E_ARG, "fjb_router_classes: min_total_l out of range");
    h->router_min_l = min_total_l;
    h->drop_graph();
    return FJB_OK;
}

int fjb_router_set(fjb_handle *h, const float *params_host, float log10_threshold) {
    if (!h) return fail(h, FJB_E_ARG, "null handle");
    h->drop_graph();
    if (!params_host) {
        h->router_on = false;
        return FJB_OK;
    }
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    CUDA_OK(h, cudaSetDevice(h->device));
    try {
        h->router_p.upload(std::vector<float>(params_host, params_host + kNParams));
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, e.what());
    }
    h->router_log_thr = log10_threshold;
    h->router_on = true;
    return FJB_OK;
}

int fjb_router_features(fjb_handle *h, const double *D_dev, const int32_t *samples, int n, float *feat_dev,
                        double *bound_dev) {
    if (!h || !D_dev || !samples || n < 0 || !feat_dev || !bound_dev) return fail(h, FJB_E_ARG, "null argument");
    if (!h->planned) return fail(h, FJB_E_STATE, "no plan: call fjb_plan first");
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    CUDA_OK(h, cudaSetDevice(h->device));
    const int nl = (int)h->lstat.size();
    for (int i = 0; i < n; ++i) {
        const int li = samples[3 * i], ib = samples[3 * i + 1], ik = samples[3 * i + 2];
        if (li < 0 || li >= nl) return fail(h, FJB_E_ARG, "sample launch out of range");
        const PlanBatch &br = h->plan.batches[h->plan.launches[li].first];
        const PlanBatch &kt = h->plan.batches[h->plan.launches[li].second];
        if (ib < 0 || ib >= (int)br.pairs.size() || ik < 0 || ik >= (int)kt.pairs.size())
            return fail(h, FJB_E_ARG, "sample pair index out of range");
    }
    const int nsh = (int)h->basis.shells.size();
    density_blocks_kernel<<<(nsh * nsh + 255) / 256, 256>>>(D_dev, h->basis.n_ao, nsh, h->sh_off.p, h->sh_nc.p,
                                                          h->Dsh.p);
    if (n == 0) return FJB_OK;
    DevBuf<int32_t> ds;
    try {
        ds.upload(std::vector<int32_t>(samples, samples + 3 * (size_t)n));
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, e.what());
    }
    router_features_kernel<<<(n + 127) / 128, 128>>>(ds.p, n, h->launches.p, h->pairs.p, h->prims.p, h->Dsh.p,
                                                     nsh, h->launch_cls.p, feat_dev, bound_dev);
    CUDA_OK(h, cudaGetLastError());
    CUDA_OK(h, cudaDeviceSynchronize());
    return FJB_OK;
}

int fjb_df_blocks(fjb_handle *h, int kind, const int32_t *items, int n, double *out_dev, int64_t *offsets) {
    if (!h || !items || n < 0 || !offsets) return fail(h, FJB_E_ARG, "null argument");
    if (!h->df) return fail(h, FJB_E_STATE, "not a density-fitting handle (fjb_create_df)");
    const int nao_sh = h->df_ao_shells, nx = h->df_aux_shells, unit = nao_sh + nx;
    std::vector<int32_t> q((size_t)4 * n);
    for (int i = 0; i < n; ++i) {
        if (kind == FJB_DF_METRIC) {
            const int P = items[2 * i], Q = items[2 * i + 1];
            if (P < 0 || P >= nx || Q < 0 || Q >= nx) return fail(h, FJB_E_ARG, "aux shell index out of range");
            q[4 * i + 0] = nao_sh + P;
            q[4 * i + 1] = unit;
            q[4 * i + 2] = nao_sh + Q;
            q[4 * i + 3] = unit;
        } else if (kind == FJB_DF_ERI3) {
            const int a = items[3 * i], b = items[3 * i + 1], P = items[3 * i + 2];
            if (a < 0 || a >= nao_sh || b < 0 || b >= nao_sh || P < 0 || P >= nx)
                return fail(h, FJB_E_ARG, "shell index out of range");
            q[4 * i + 0] = a;
            q[4 * i + 1] = b;
            q[4 * i + 2] = nao_sh + P;
            q[4 * i + 3] = unit;
        } else {
            return fail(h, FJB_E_ARG, "unknown density-fitting kind");
        }
    }
    return fjb_eri_blocks(h, q.data(), n, out_dev, offsets);
}

int fjb_df_jk(fjb_handle *h, const double *B_dev, int64_t n_aux, int64_t n_ao, const double *D_dev, double *J_dev,
              double *K_dev, void *stream) {
    if (!h || !B_dev || !D_dev || !J_dev || !K_dev) return fail(h, FJB_E_ARG, "null argument");
    if (n_aux < 1 || n_ao < 1) return fail(h, FJB_E_ARG, "fjb_df_jk: n_aux and n_ao must be >= 1");
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    CUDA_OK(h, cudaSetDevice(h->device));
    const size_t bytes = df_jk_workspace_bytes(n_aux, n_ao);
    try {
        if (h->df_work.n < bytes) h->df_work.alloc(bytes);
        h->df_err.alloc(1);
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, std::string("fjb_df_jk workspace: ") + e.what());
    }
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_OK(h, cudaMemsetAsync(h->df_err.p, 0, sizeof(int), st));
    CUDA_OK(h, df_jk_launch(B_dev, n_aux, n_ao, D_dev, J_dev, K_dev, h->df_work.p, h->df_err.p, st));
    int err = 0;
    CUDA_OK(h, cudaMemcpyAsync(&err, h->df_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(h, cudaStreamSynchronize(st));
    if (err) return fail(h, FJB_E_TIMEOUT, "fjb_df_jk: a tensor-core wait ran out (the GEMM did not complete)");
    return FJB_OK;
}

int fjb_hjk_plan(fjb_handle *h, const double *D_host, double tau, int mode, int screen) {
    if (!h || !D_host) return fail(h, FJB_E_ARG, "null argument");
    if (h->df) return fail(h, FJB_E_STATE, "a density-fitting handle has no pair stream");
    h->hjk_planned = h->hjk_staged = false;
    try {
        const unsigned nt = std::max(1u, std::thread::hardware_concurrency());
        h->hjk = hjk_launches(h->basis, D_host, tau, mode, screen, (int)nt);
    } catch (const std::length_error &e) {
        return fail(h, FJB_E_LIMIT, e.what());
    } catch (const std::invalid_argument &e) {
        return fail(h, FJB_E_ARG, e.what());
    } catch (const std::exception &e) {
        return fail(h, FJB_E_PLAN, e.what());
    }
    h->hjk_planned = true;
    return FJB_OK;
}

int fjb_hjk_counts(const fjb_handle *hc, int64_t *counts) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h || !counts) return fail(h, FJB_E_ARG, "null argument");
    if (!h->hjk_planned) return fail(h, FJB_E_STATE, "no split stream: call fjb_hjk_plan first");
    const HjkPlan &P = h->hjk;
    std::vector<std::array<int, 4>> cls;
    for (size_t l = 0; l < P.launches.size(); ++l) cls.push_back(P.kernel_class((int)l, nullptr));
    std::sort(cls.begin(), cls.end());
    const int64_t n_cls = (int64_t)(std::unique(cls.begin(), cls.end()) - cls.begin());
    // the skipped visits: every (bra pair, ket pair) of every launch
    const int nt = (int)std::max(1u, std::thread::hardware_concurrency());
    std::vector<int64_t> skipped(nt, 0);
    std::vector<std::thread> pool;
    const size_t np = P.pairs.size();
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&, t]() {
            int64_t n = 0;
            for (size_t i = t; i < np; i += nt)
                for (size_t j = 0; j < np; ++j) n += P.key(P.pairs[i], P.pairs[j]) < P.tau;
            skipped[t] = n;
        });
    for (auto &th : pool) th.join();
    int64_t sk = 0;
    for (int64_t x : skipped) sk += x;
    counts[0] = (int64_t)np;
    counts[1] = (int64_t)P.batches.size();
    counts[2] = (int64_t)P.launches.size();
    counts[3] = n_cls;
    counts[4] = (int64_t)np * (int64_t)np;
    counts[5] = sk;
    return FJB_OK;
}

int fjb_hjk_export(const fjb_handle *hc, int32_t *pairs, double *pair_G, int32_t *batches, int32_t *launches) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h) return fail(h, FJB_E_ARG, "null handle");
    if (!h->hjk_planned) return fail(h, FJB_E_STATE, "no split stream: call fjb_hjk_plan first");
    const HjkPlan &P = h->hjk;
    if (pairs)
        for (size_t i = 0; i < P.pairs.size(); ++i) {
            const HjkPair &p = P.pairs[i];
            const int32_t v[5] = {p.a, p.b, p.la, p.lb, p.degree};
            std::copy(v, v + 5, pairs + 5 * i);
        }
    if (pair_G)
        for (size_t i = 0; i < P.pairs.size(); ++i) pair_G[i] = P.pairs[i].G;
    if (batches)
        for (size_t i = 0; i < P.batches.size(); ++i) {
            const HjkBatch &b = P.batches[i];
            const int32_t v[5] = {b.la, b.lb, b.degree, b.p0, b.n};
            std::copy(v, v + 5, batches + 5 * i);
        }
    if (launches)
        for (size_t l = 0; l < P.launches.size(); ++l) {
            std::array<int, 4> g;
            const std::array<int, 4> o = P.ordered((int)l), k = P.kernel_class((int)l, &g);
            int32_t *w = launches + 14 * l;
            w[0] = P.launches[l].first;
            w[1] = P.launches[l].second;
            for (int j = 0; j < 4; ++j) {
                w[2 + j] = o[j];
                w[6 + j] = k[j];
                w[10 + j] = g[j];
            }
        }
    return FJB_OK;
}

int fjb_hjk_keys(const fjb_handle *hc, int launch, double *keys, uint8_t *skipped) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h) return fail(h, FJB_E_ARG, "null handle");
    if (!h->hjk_planned) return fail(h, FJB_E_STATE, "no split stream: call fjb_hjk_plan first");
    const HjkPlan &P = h->hjk;
    if (launch < 0 || launch >= (int)P.launches.size()) return fail(h, FJB_E_ARG, "launch index out of range");
    const HjkBatch &br = P.batches[P.launches[launch].first], &kt = P.batches[P.launches[launch].second];
    size_t at = 0;
    for (int i = 0; i < br.n; ++i)
        for (int j = 0; j < kt.n; ++j, ++at) {
            const double k = P.key(P.pairs[br.p0 + i], P.pairs[kt.p0 + j]);
            if (keys) keys[at] = k;
            if (skipped) skipped[at] = k < P.tau;
        }
    return FJB_OK;
}

int fjb_hjk_computed(fjb_handle *h, int64_t *per_launch) {
    if (!h || !per_launch) return fail(h, FJB_E_ARG, "null argument");
    if (!h->hjk_staged) return fail(h, FJB_E_STATE, "no split K build yet (fjb_hjk_k)");
    CUDA_OK(h, cudaSetDevice(h->device));
    CUDA_OK(h, cudaDeviceSynchronize());
    std::vector<unsigned long long> c(h->hjk.launches.size());
    if (!c.empty())
        CUDA_OK(h, cudaMemcpy(c.data(), h->hk_computed.p, c.size() * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < c.size(); ++i) per_launch[i] = (int64_t)c[i];
    return FJB_OK;
}

namespace {

// The split K build's records, staged once per stream: each launch's pairs
// in its kernel class's orientation (kernel position j holds the ordered
// quartet's position shells[j]; a pair reversed keeps its ordered G), the
// launch's axes (shells' inverse) packed into LaunchRec.pad0, units of up to
// 32 kets, grouped by kernel class.
int stage_hjk(fjb_handle *h) {
    if (h->hjk_staged) return FJB_OK;
    const HjkPlan &P = h->hjk;
    const HostBasis &B = h->basis;
    std::vector<PairRec> pr;
    std::vector<PrimRec> pm;
    std::vector<LaunchRec> lr;
    std::map<std::tuple<int, int, int, int>, std::vector<Unit>> by_class;
    std::map<std::tuple<int, int, int, int>, std::pair<int, int>> deg;
    auto add_list = [&](const HjkBatch &bt, bool reversed) {
        const int p0 = (int)pr.size();
        for (int i = 0; i < bt.n; ++i) {
            const HjkPair &p = P.pairs[bt.p0 + i];
            const int x = reversed ? p.b : p.a, y = reversed ? p.a : p.b;
            const HostShell &sx = B.shells[x], &sy = B.shells[y];
            const int K = (int)(sx.exps.size() * sy.exps.size());
            pr.push_back(pair_record(B, x, y, p.G, (int)pm.size(), K));
            for (int k = 0; k < K; ++k) pm.push_back(prim_record(sx, sy, k));
        }
        return p0;
    };
    for (size_t l = 0; l < P.launches.size(); ++l) {
        std::array<int, 4> g;
        const std::array<int, 4> kc = P.kernel_class((int)l, &g);
        const HjkBatch &bra = P.batches[P.launches[l].first], &ket = P.batches[P.launches[l].second];
        const bool swap = g[0] >= 2;  // the kernel's bra is the ordered ket
        const HjkBatch &kb = swap ? ket : bra, &kk = swap ? bra : ket;
        LaunchRec r{};
        r.bra_pair0 = add_list(kb, g[0] != (swap ? 2 : 0));
        r.n_bra = kb.n;
        r.ket_pair0 = add_list(kk, g[2] != (swap ? 0 : 2));
        r.n_ket = kk.n;
        int axes[4];
        for (int j = 0; j < 4; ++j) axes[g[j]] = j;
        r.pad0 = axes[0] | axes[1] << 2 | axes[2] << 4 | axes[3] << 6;
        const int li = (int)lr.size();
        lr.push_back(r);
        auto key = std::make_tuple(kc[0], kc[1], kc[2], kc[3]);
        auto &d = deg[key];
        d.first = std::max(d.first, kb.degree);
        d.second = std::max(d.second, kk.degree);
        for (int ib = 0; ib < kb.n; ++ib)
            for (int k0 = 0; k0 < kk.n; k0 += kKetChunk)
                by_class[key].push_back(Unit{li, ib, k0, std::min(kk.n, k0 + kKetChunk)});
    }
    std::vector<Unit> units;
    h->hk_runs.clear();
    for (auto &kv : by_class) {
        auto [la, lb, lc, ld] = kv.first;
        h->hk_runs.push_back({la, lb, lc, ld, (int)units.size(), (int)kv.second.size(), deg[kv.first].first,
                              deg[kv.first].second});
        units.insert(units.end(), kv.second.begin(), kv.second.end());
    }
    try {
        h->hk_pairs.upload(pr);
        h->hk_prims.upload(pm);
        h->hk_launches.upload(lr);
        h->hk_units.upload(units);
        h->hk_computed.alloc(std::max<size_t>(1, lr.size()));
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, e.what());
    }
    h->hjk_staged = true;
    return FJB_OK;
}

}  // namespace

int fjb_hjk_k(fjb_handle *h, const double *D_dev, double *K_dev, void *stream) {
    if (!h || !D_dev || !K_dev) return fail(h, FJB_E_ARG, "null argument");
    if (!h->hjk_planned) return fail(h, FJB_E_STATE, "no split stream: call fjb_hjk_plan first");
    if (h->hjk.screen != kHjkScreenK)
        return fail(h, FJB_E_STATE, "the stream was planned with J's key, which does not bound K's deposits");
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    CUDA_OK(h, cudaSetDevice(h->device));
    if (int rc = stage_hjk(h)) return rc;
    if (int rc = ensure_smem_attr(h)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int nsh = (int)h->basis.shells.size(), nao = h->basis.n_ao;
    try {
        if (h->Dsh.n < (size_t)nsh * nsh) h->Dsh.alloc((size_t)nsh * nsh);
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, e.what());
    }
    density_blocks_kernel<<<(nsh * nsh + 255) / 256, 256, 0, st>>>(D_dev, nao, nsh, h->sh_off.p, h->sh_nc.p,
                                                                 h->Dsh.p);
    CUDA_OK(h, cudaMemsetAsync(K_dev, 0, (size_t)nao * nao * sizeof(double), st));
    CUDA_OK(h, cudaMemsetAsync(h->hk_computed.p, 0, h->hk_computed.n * sizeof(unsigned long long), st));
    for (const auto &r : h->hk_runs) {
        ClassEntry *ce;
        ClassDev dev;
        try {
            ce = &h->cls(r.la, r.lb, r.lc, r.ld);
            dev = ce->dev(r.max_kab, r.max_kcd);
        } catch (const std::length_error &e) {
            return fail(h, FJB_E_LIMIT, e.what());
        } catch (const std::exception &e) {
            return fail(h, FJB_E_CUDA, e.what());
        }
        KArgs a{};
        a.C = dev;
        a.units = h->hk_units.p + r.unit0;
        a.n_units = r.n_units;
        a.launches = h->hk_launches.p;
        a.pairs = h->hk_pairs.p;
        a.prims = h->hk_prims.p;
        a.D = D_dev;
        a.Dsh = h->Dsh.p;
        a.n_sh = nsh;
        a.n_ao = nao;
        a.tau = h->hjk.tau;
        a.Kp = K_dev;
        a.boys_tab = h->boys.p;
        a.hk = 1;
        a.computed = h->hk_computed.p;
        CUDA_OK(h, launch_hgp<double>(dev, grid_for(dev, a.n_units), st, a));
    }
    CUDA_OK(h, cudaGetLastError());
    return FJB_OK;
}

int fjb_df_syrk(fjb_handle *h, const double *Z_dev, int64_t rows, int64_t cols, double *K_dev, void *stream) {
    if (!h || !Z_dev || !K_dev) return fail(h, FJB_E_ARG, "null argument");
    if (rows < 1 || cols < 1) return fail(h, FJB_E_ARG, "fjb_df_syrk: rows and cols must be >= 1");
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    CUDA_OK(h, cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    const size_t bytes = df_syrk_workspace_bytes(rows, cols);
    try {
        if (h->df_work.n < bytes) {
            CUDA_OK(h, cudaStreamSynchronize(st));  // a previous call may still read the old workspace
            h->df_work.alloc(bytes);
        }
        h->df_err.alloc(1);
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, std::string("fjb_df_syrk workspace: ") + e.what());
    }
    CUDA_OK(h, cudaMemsetAsync(h->df_err.p, 0, sizeof(int), st));
    CUDA_OK(h, df_syrk_launch(Z_dev, rows, cols, K_dev, h->df_work.p, h->df_err.p, st));
    int err = 0;
    CUDA_OK(h, cudaMemcpyAsync(&err, h->df_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(h, cudaStreamSynchronize(st));
    if (err) return fail(h, FJB_E_TIMEOUT, "fjb_df_syrk: a tensor-core wait ran out (the GEMM did not complete)");
    return FJB_OK;
}

namespace {

// The three-centre kernel's records, staged once per handle: the Schwarz
// factors sqrt(max |(ab|ab)|) of every AO shell pair and sqrt(max |(P|P)|)
// of every aux shell from the ERI tap, the AO pairs oriented la >= lb, the
// aux shells as (P, unit) pairs sorted by (l, degree, index).
int ensure_eri3(fjb_handle *h) {
    if (h->e3_ready) return FJB_OK;
    const int nao_sh = h->df_ao_shells, nx = h->df_aux_shells, unit = nao_sh + nx;
    const HostBasis &B = h->basis;
    const int ao_end = B.offsets[nao_sh];  // AO functions; the aux basis numbers from here
    // Schwarz factors: one diagonal block per AO pair and per aux shell
    std::vector<int32_t> q;
    std::vector<std::pair<int, int>> ab;
    for (int a = 0; a < nao_sh; ++a)
        for (int b = a; b < nao_sh; ++b) {
            ab.emplace_back(a, b);
            const int x = B.shells[a].l <= B.shells[b].l ? a : b, y = x == a ? b : a;
            q.insert(q.end(), {x, y, x, y});
        }
    for (int P = 0; P < nx; ++P) q.insert(q.end(), {nao_sh + P, unit, nao_sh + P, unit});
    const int nq = (int)(q.size() / 4);
    std::vector<int64_t> off((size_t)nq + 1, 0);
    for (int i = 0; i < nq; ++i) {
        int nabcd = 1;
        for (int k = 0; k < 4; ++k) nabcd *= ncart(B.shells[q[4 * (size_t)i + k]].l);
        off[i + 1] = off[i] + nabcd;
    }
    std::vector<double> diag;
    try {
        DevBuf<double> dv;
        dv.alloc((size_t)off[nq]);
        if (int rc = eri_blocks_impl(h, q.data(), nq, dv.p, off.data(), false)) return rc;
        diag.resize((size_t)off[nq]);
        CUDA_OK(h, cudaMemcpy(diag.data(), dv.p, diag.size() * sizeof(double), cudaMemcpyDeviceToHost));
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, std::string("fjb_df_eri3 Schwarz factors: ") + e.what());
    }
    auto gmax = [&](int i) {
        double m = 0.0;
        for (int64_t k = off[i]; k < off[i + 1]; ++k) m = std::max(m, std::fabs(diag[(size_t)k]));
        return std::sqrt(m);
    };
    std::vector<PairRec> pr;
    std::vector<PrimRec> pm;
    for (size_t i = 0; i < ab.size(); ++i) {
        int a = ab[i].first, b = ab[i].second;
        if (B.shells[a].l < B.shells[b].l) std::swap(a, b);
        const HostShell &sa = B.shells[a], &sb = B.shells[b];
        const int K = (int)(sa.exps.size() * sb.exps.size());
        pr.push_back(pair_record(B, a, b, gmax((int)i), (int)pm.size(), K));
        for (int k = 0; k < K; ++k) pm.push_back(prim_record(sa, sb, k));
    }
    std::vector<int> order(nx);
    for (int P = 0; P < nx; ++P) order[P] = P;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const HostShell &sx = B.shells[nao_sh + x], &sy = B.shells[nao_sh + y];
        if (sx.l != sy.l) return sx.l < sy.l;
        return sx.exps.size() < sy.exps.size();
    });
    std::vector<PairRec> kr;
    std::vector<PrimRec> km;
    h->e3_ket_pos.assign(nx, 0);
    h->e3_gp_max = 0.0;
    for (int i = 0; i < nx; ++i) {
        const int P = order[i];
        const HostShell &sp = B.shells[nao_sh + P];
        const int K = (int)sp.exps.size();
        const double g = gmax((int)ab.size() + P);
        h->e3_gp_max = std::max(h->e3_gp_max, g);
        PairRec r = pair_record(B, nao_sh + P, unit, g, (int)km.size(), K);
        r.ao_a = B.offsets[nao_sh + P] - ao_end;
        kr.push_back(r);
        for (int k = 0; k < K; ++k) km.push_back(prim_record(sp, B.shells[unit], k));
        h->e3_ket_pos[P] = i;
    }
    h->e3_aux_off.assign(nx + 1, 0);
    for (int P = 0; P < nx; ++P) h->e3_aux_off[P] = B.offsets[nao_sh + P] - ao_end;
    h->e3_aux_off[nx] = B.offsets[unit] - ao_end;
    try {
        h->e3_pairs.upload(pr);
        h->e3_prims.upload(pm);
        h->e3_kets.upload(kr);
        h->e3_kprims.upload(km);
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, e.what());
    }
    h->e3_pairs_host = std::move(pr);
    h->e3_kets_host = std::move(kr);
    h->e3_dev.clear();
    h->e3_ready = true;
    return FJB_OK;
}

}  // namespace

int fjb_df_eri3(fjb_handle *h, int aux_shell0, int aux_shell1, double tau, double *out_dev, int32_t *n_launches,
                void *stream) {
    if (!h || !out_dev) return fail(h, FJB_E_ARG, "null argument");
    if (n_launches) *n_launches = 0;
    if (!h->df) return fail(h, FJB_E_STATE, "not a density-fitting handle (fjb_create_df)");
    const int nx = h->df_aux_shells;
    if (aux_shell0 < 0 || aux_shell1 > nx || aux_shell0 >= aux_shell1)
        return fail(h, FJB_E_ARG, "fjb_df_eri3: need 0 <= aux_shell0 < aux_shell1 <= the aux shell count");
    if (!(tau == tau)) return fail(h, FJB_E_ARG, "fjb_df_eri3: tau is not a number");
    CUDA_OK(h, cudaSetDevice(h->device));
    if (int rc = ensure_eri3(h)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const HostBasis &B = h->basis;
    const int n_ao = B.offsets[h->df_ao_shells];
    const int p0 = h->e3_aux_off[aux_shell0], nb = h->e3_aux_off[aux_shell1] - p0;
    // the block's aux shells in sorted order: runs of equal (l, degree),
    // cut into units of at most kE3Kets
    std::vector<int> pos;
    for (int P = aux_shell0; P < aux_shell1; ++P) pos.push_back(h->e3_ket_pos[P]);
    std::sort(pos.begin(), pos.end());
    struct Run {
        int lp, k0, k1;
    };
    std::vector<Run> runs;
    for (size_t i = 0; i < pos.size();) {
        const PairRec &k = h->e3_kets_host[pos[i]];
        const int lp = B.shells[k.a].l, deg = k.nprim;
        size_t j = i + 1;
        while (j < pos.size() && pos[j] == pos[j - 1] + 1 && j - i < (size_t)kE3Kets &&
               B.shells[h->e3_kets_host[pos[j]].a].l == lp && h->e3_kets_host[pos[j]].nprim == deg)
            ++j;
        runs.push_back({lp, pos[i], pos[j - 1] + 1});
        i = j;
    }
    // units class by class: (la, lb) of the pair, lp of the run
    struct Launch {
        int la, lb, lp, max_kab, max_kcd;
        size_t u0, n;
    };
    std::vector<Launch> launches;
    std::vector<E3Unit> units;
    for (const auto &r : runs)
        if (r.lp > FJB_E3_MAX_LP) return fail(h, FJB_E_LIMIT, "fjb_df_eri3: aux l above 4");
    std::map<int, std::vector<int>> by;  // lp -> run indices
    for (size_t r = 0; r < runs.size(); ++r) by[runs[r].lp].push_back((int)r);
    std::map<std::pair<int, int>, std::vector<int>> pairs_of;
    const double gate = tau > 0.0 ? tau / std::max(h->e3_gp_max, 1e-300) : -1.0;
    for (size_t i = 0; i < h->e3_pairs_host.size(); ++i) {
        const PairRec &p = h->e3_pairs_host[i];
        if (gate > 0.0 && p.G < gate) continue;  // below tau against every aux shell
        pairs_of[{B.shells[p.a].l, B.shells[p.b].l}].push_back((int)i);
    }
    for (auto &kv : pairs_of) {
        const int la = kv.first.first, lb = kv.first.second;
        int max_kab = 1;
        for (int i : kv.second) max_kab = std::max(max_kab, h->e3_pairs_host[i].nprim);
        for (int lp = 0; lp <= FJB_E3_MAX_LP; ++lp) {
            auto it = by.find(lp);
            if (it == by.end()) continue;
            int max_kcd = 1;
            for (int r : it->second)
                for (int k = runs[r].k0; k < runs[r].k1; ++k) max_kcd = std::max(max_kcd, h->e3_kets_host[k].nprim);
            Launch L{la, lb, lp, max_kab, max_kcd, units.size(), 0};
            for (int i : kv.second)
                for (int r : it->second) units.push_back(E3Unit{i, runs[r].k0, runs[r].k1, 0});
            L.n = units.size() - L.u0;
            if (L.n) launches.push_back(L);
        }
    }
    try {
        CUDA_OK(h, cudaStreamSynchronize(st));  // an earlier call's kernels may still read the units
        h->e3_units.upload(units);
    } catch (const std::exception &e) {
        return fail(h, FJB_E_CUDA, e.what());
    }
    CUDA_OK(h, cudaMemsetAsync(out_dev, 0, (size_t)n_ao * n_ao * nb * sizeof(double), st));
    const int sms = sm_count();
    for (const Launch &L : launches) {
        auto key = std::make_tuple(L.la, L.lb, L.lp);
        auto it = h->e3_dev.find(key);
        if (it == h->e3_dev.end() || it->second.kab < L.max_kab || it->second.kcd < L.max_kcd) {
            E3Dev d;
            if (!eri3_layout(L.la, L.lb, L.lp, L.max_kab, L.max_kcd, &d))
                return fail(h, FJB_E_LIMIT, "fjb_df_eri3: a class does not fit in shared memory");
            it = h->e3_dev.insert_or_assign(key, d).first;
        }
        E3Args a{};
        a.Y = it->second;
        a.units = h->e3_units.p + L.u0;
        a.n_units = (int)L.n;
        a.pairs = h->e3_pairs.p;
        a.prims = h->e3_prims.p;
        a.kets = h->e3_kets.p;
        a.kprims = h->e3_kprims.p;
        a.out = out_dev;
        a.n_ao = n_ao;
        a.p0 = p0;
        a.nb = nb;
        a.tau = tau;
        a.rys_tab = h->rys.p;
        const int per_sm = std::max(1, eri3_blocks_per_sm(L.la, L.lb, L.lp, a.Y));
        const int grid = (int)std::min<size_t>(L.n, (size_t)per_sm * sms);
        CUDA_OK(h, eri3_launch(L.la, L.lb, L.lp, grid, st, a));
        if (n_launches) ++*n_launches;
    }
    return FJB_OK;
}

int fjb_scatter_map(const fjb_handle *hc, int launch, int32_t *el, int32_t *ptr, int32_t *src, int64_t *n_el,
                    int64_t *n_slot) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h || !n_el || !n_slot) return fail(h, FJB_E_ARG, "null argument");
    if (!h->planned) return fail(h, FJB_E_STATE, "no plan: call fjb_plan first");
    if (launch < 0 || launch >= (int)h->lr_host.size()) return fail(h, FJB_E_ARG, "launch index out of range");
    const LaunchRec &L = h->lr_host[launch];
    const fjb_launch_stat &ls = h->lstat[launch];
    const int l[4] = {ls.la, ls.lb, ls.lc, ls.ld};
    std::vector<std::pair<int, int>> bra_ao, ket_ao;
    for (int i = 0; i < L.n_bra; ++i)
        bra_ao.emplace_back(h->pr_host[L.bra_pair0 + i].ao_a, h->pr_host[L.bra_pair0 + i].ao_b);
    for (int k = 0; k < L.n_ket; ++k)
        ket_ao.emplace_back(h->pr_host[L.ket_pair0 + k].ao_a, h->pr_host[L.ket_pair0 + k].ao_b);
    ScatterMap m;
    try {
        m = scatter_map(l, bra_ao, ket_ao);
    } catch (const std::length_error &e) {
        return fail(h, FJB_E_LIMIT, e.what());
    }
    *n_el = m.n_el;
    *n_slot = m.n_slot;
    if (el) std::copy(m.el.begin(), m.el.end(), el);
    if (ptr) std::copy(m.ptr.begin(), m.ptr.end(), ptr);
    if (src) std::copy(m.src.begin(), m.src.end(), src);
    return FJB_OK;
}

int fjb_coulomb(fjb_handle *h, const double *D_dev, double *J_dev, double tau, void *stream) {
    return fjb_coulomb_mixed(h, D_dev, J_dev, tau, 0.0, stream);
}

int fjb_coulomb_mixed(fjb_handle *h, const double *D_dev, double *J_dev, double tau, double threshold, void *stream) {
    if (!h || !D_dev || !J_dev) return fail(h, FJB_E_ARG, "null argument");
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    if (h->df) return fail(h, FJB_E_STATE, "a density-fitting handle has no J-engine");
    if (!std::isfinite(tau) || tau < 0.0) return fail(h, FJB_E_ARG, "tau must be finite and >= 0");
    if (!std::isfinite(threshold) || threshold < 0.0) return fail(h, FJB_E_ARG, "threshold must be finite and >= 0");
    CUDA_OK(h, cudaSetDevice(h->device));
    std::string err;
    if (!h->jeng) {
        h->jeng = jengine_create(h->basis, h->device, &err);
        if (!h->jeng) return fail(h, FJB_E_CUDA, err);
    }
    int nl = 0;
    if (jengine_build(h->jeng, D_dev, J_dev, tau, threshold, h->boys.p, (cudaStream_t)stream, &err, &nl))
        return fail(h, FJB_E_CUDA, err);
    h->j_launches = nl;
    return FJB_OK;
}

int fjb_one_electron(fjb_handle *h, const double *charges, const double *coords, int n_nuc, double *S_dev,
                     double *T_dev, double *V_dev, double *H_dev, void *stream) {
    if (!h) return fail(h, FJB_E_ARG, "null argument");
    if (n_nuc < 0 || (n_nuc > 0 && (!charges || !coords))) return fail(h, FJB_E_ARG, "nuclei: null or n_nuc < 0");
    for (int q = 0; q < n_nuc; ++q)
        if (!std::isfinite(charges[q]) || !std::isfinite(coords[3 * q]) || !std::isfinite(coords[3 * q + 1]) ||
            !std::isfinite(coords[3 * q + 2]))
            return fail(h, FJB_E_ARG, "nucleus " + std::to_string(q) + " has a non-finite charge or coordinate");
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    if (h->df) return fail(h, FJB_E_STATE, "a density-fitting handle has no one-electron matrices");
    CUDA_OK(h, cudaSetDevice(h->device));
    std::string err;
    if (!h->onee) {
        h->onee = onee_create(h->basis, h->device, &err);
        if (!h->onee) return fail(h, FJB_E_CUDA, err);
    }
    int nl = 0;
    if (onee_build(h->onee, charges, coords, n_nuc, S_dev, T_dev, V_dev, H_dev, h->boys.p, (cudaStream_t)stream,
                   &err, &nl))
        return fail(h, FJB_E_CUDA, err);
    return FJB_OK;
}

int fjb_j_plan_lists(const fjb_handle *hc, const double *D_host, fjb_j_lists *out, int64_t *n_records) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h || !D_host || !n_records) return fail(h, FJB_E_ARG, "null argument");
    if (h->df) return fail(h, FJB_E_STATE, "a density-fitting handle has no J-engine");
    JHostLists L;
    try {
        jengine_host_lists(h->basis, D_host, &L);
    } catch (const std::exception &e) {
        return fail(h, FJB_E_PLAN, e.what());
    }
    *n_records = (int64_t)L.a.size();
    if (!out) return FJB_OK;
    auto put = [](auto *dst, const auto &src) {
        if (dst) std::copy(src.begin(), src.end(), dst);
    };
    put(out->a, L.a);
    put(out->b, L.b);
    put(out->prim, L.prim);
    put(out->L, L.L);
    put(out->G, L.G);
    put(out->key, L.key);
    put(out->ket_order, L.ket_order);
    put(out->L_off, L.L_off);
    return FJB_OK;
}

int fjb_j_last_launches(const fjb_handle *h) { return h ? h->j_launches : -1; }

int fjb_boys(int m, const double *T_dev, int n, double *F_dev) {
    if (m < 0 || m > kBoysMaxM - kBoysTaylor + 1 || n < 0 || !T_dev || !F_dev)
        return fail(nullptr, FJB_E_ARG, "boys: order out of range or null argument");
    static DevBuf<double> *tab = nullptr;
    if (!tab) {
        tab = new DevBuf<double>();
        try {
            tab->upload(boys_table());
        } catch (const std::exception &e) {
            return fail(nullptr, FJB_E_CUDA, e.what());
        }
    }
    if (n == 0) return FJB_OK;
    boys_kernel<<<(n + 127) / 128, 128>>>(m, T_dev, n, F_dev, tab->p);
    CUDA_OK(nullptr, cudaGetLastError());
    CUDA_OK(nullptr, cudaDeviceSynchronize());
    return FJB_OK;
}

int fjb_last_build_stats(const fjb_handle *hc, double *ms, int *n_launches) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h) return fail(nullptr, FJB_E_ARG, "null handle");
    if (ms) {
        float f = 0.f;
        CUDA_OK(h, cudaEventSynchronize(h->ev1));
        CUDA_OK(h, cudaEventElapsedTime(&f, h->ev0, h->ev1));
        *ms = f;
    }
    if (n_launches) *n_launches = h->last_launches;
    return FJB_OK;
}

int fjb_launch_stats(const fjb_handle *hc, fjb_launch_stat *out, int64_t n) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h || !out) return fail(h, FJB_E_ARG, "null argument");
    if (!h->planned) return fail(h, FJB_E_STATE, "no plan: call fjb_plan first");
    if (n < (int64_t)h->lstat.size()) return fail(h, FJB_E_ARG, "output holds fewer entries than launches");
    std::vector<unsigned long long> c(h->lstat.size(), 0);
    if (h->device >= 0 && h->built && !c.empty()) {
        CUDA_OK(h, cudaEventSynchronize(h->ev1));
        CUDA_OK(h, cudaMemcpy(c.data(), h->computed.p, c.size() * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost));
    }
    for (size_t i = 0; i < h->lstat.size(); ++i) {
        out[i] = h->lstat[i];
        out[i].computed = (int64_t)c[i];
    }
    return FJB_OK;
}

int fjb_set_class_config(fjb_handle *h, int la, int lb, int lc, int ld, int threads, int slots) {
    if (!h) return fail(h, FJB_E_ARG, "null handle");
    if (threads != 0 && threads != 1 && threads != 32 && threads != 64 && threads != 128 && threads != 256 &&
        threads != 512)
        return fail(h, FJB_E_ARG, "threads must be 0, 1 (register kernel), 32, 64, 128, 256 or 512");
    if (slots < 0 || slots > kMaxThreads) return fail(h, FJB_E_ARG, "slots out of range");
    auto key = std::make_tuple(la, lb, lc, ld);
    h->drop_graph();  // a captured build holds the old launches
    if (threads == 0 && slots == 0)
        h->cfg.erase(key);
    else
        h->cfg[key] = {threads, slots};
    if (h->device < 0 || !h->planned) return FJB_OK;
    for (auto &r : h->runs) {
        if (std::make_tuple(r.dev.la, r.dev.lb, r.dev.lc, r.dev.ld) != key) continue;
        try {
            if (threads == 1 && !compiled_available(la, lb, lc, ld, false))
                return fail(h, FJB_E_LIMIT, "this class has no compiled register kernel");
            ClassEntry &ce = h->cls(la, lb, lc, ld);
            ClassDev d = threads == 1 ? ce.dev(r.max_kab, r.max_kcd) : ce.dev(r.max_kab, r.max_kcd, threads, slots);
            r.dev32 = threads == 1 ? ce.dev(r.max_kab, r.max_kcd, 0, 0, 4)
                                   : ce.dev(r.max_kab, r.max_kcd, threads, slots, 4);
            auto ov32 = h->cfg32.find(key);
            if (ov32 != h->cfg32.end())
                r.dev32 = ce.dev(r.max_kab, r.max_kcd, ov32->second.first, ov32->second.second, 4);
            r.dev = d;
            r.compiled = compiled_available(la, lb, lc, ld, false) && (threads == 0 || threads == 1);
            r.grid = run_grid(r);
            r.grid32 = run_grid32(r);
        } catch (const std::length_error &e) {
            return fail(h, FJB_E_LIMIT, e.what());
        }
    }
    return FJB_OK;
}

int fjb_set_rys(fjb_handle *h, int mode) {
    if (!h) return fail(h, FJB_E_ARG, "null handle");
    if (mode < 0 || mode > 2) return fail(h, FJB_E_ARG, "fjb_set_rys: mode is 0, 1 or 2");
    h->use_rys = mode;
    if (h->device < 0) return FJB_OK;
    cudaSetDevice(h->device);
    for (auto &r : h->runs) choose_rys(mode, r);
    h->drop_graph();
    return FJB_OK;
}

int fjb_set_class_config32(fjb_handle *h, int la, int lb, int lc, int ld, int threads, int slots) {
    if (!h) return fail(h, FJB_E_ARG, "null handle");
    if (threads != 0 && threads != 32 && threads != 64 && threads != 128 && threads != 256 && threads != 512)
        return fail(h, FJB_E_ARG, "threads must be 0, 32, 64, 128, 256 or 512");
    if (slots < 0 || slots > kMaxThreads) return fail(h, FJB_E_ARG, "slots out of range");
    auto key = std::make_tuple(la, lb, lc, ld);
    h->drop_graph();
    if (threads == 0 && slots == 0)
        h->cfg32.erase(key);
    else
        h->cfg32[key] = {threads, slots};
    if (h->device < 0 || !h->planned) return FJB_OK;
    for (auto &r : h->runs) {
        if (std::make_tuple(r.dev.la, r.dev.lb, r.dev.lc, r.dev.ld) != key) continue;
        try {
            ClassEntry &ce = h->cls(la, lb, lc, ld);
            if (threads == 0 && slots == 0) {  // back to the FP64 configuration's FP32 twin
                auto ov = h->cfg.find(key);
                const int th = ov == h->cfg.end() ? 0 : ov->second.first;
                r.dev32 = ov == h->cfg.end() || th == 1 ? ce.dev(r.max_kab, r.max_kcd, 0, 0, 4)
                                                         : ce.dev(r.max_kab, r.max_kcd, th, ov->second.second, 4);
            } else {
                r.dev32 = ce.dev(r.max_kab, r.max_kcd, threads, slots, 4);
            }
            r.grid32 = run_grid32(r);
        } catch (const std::length_error &e) {
            return fail(h, FJB_E_LIMIT, e.what());
        }
    }
    return FJB_OK;
}

int fjb_class_stats(const fjb_handle *hc, fjb_class_stat *out, int64_t n, int64_t *n_classes) {
    fjb_handle *h = const_cast<fjb_handle *>(hc);
    if (!h) return fail(h, FJB_E_ARG, "null argument");
    if (n_classes) *n_classes = (int64_t)h->runs.size();
    if (!out) return FJB_OK;
    if (!h->built) return fail(h, FJB_E_STATE, "no build yet");
    for (size_t i = 0; i < h->runs.size() && (int64_t)i < n; ++i) {
        const ClassDev &d = h->runs[i].dev;
        float ms = 0.f;
        CUDA_OK(h, cudaEventSynchronize(h->cev[i].second));
        CUDA_OK(h, cudaEventElapsedTime(&ms, h->cev[i].first, h->cev[i].second));
        const ClassRun &r = h->runs[i];
        const int32_t engine = r.rys64 ? 2 : (r.compiled ? 1 : 0);
        out[i] = fjb_class_stat{d.la, d.lb, d.lc, d.ld, (double)ms, (int64_t)r.n_units, engine, 0};
    }
    return FJB_OK;
}

}  // extern "C"

namespace {

template <typename T>
__global__ void fma_probe_kernel(T *out, int iters, T a, T b) {
    T x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = (T)(threadIdx.x + k) * (T)1e-3;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == (T)12345.678) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <typename T>
int run_probe(int reps, double *tflops) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 256, blocks = sms * 8, iters = 4096;
    T *out = nullptr;
    if (cudaMalloc(&out, sizeof(T) * threads * blocks) != cudaSuccess)
        return fail(nullptr, FJB_E_CUDA, "cudaMalloc failed");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e30;
    for (int r = 0; r < reps + 1; ++r) {
        cudaEventRecord(e0);
        fma_probe_kernel<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r > 0) best = std::min(best, (double)ms);  // the first launch warms up
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return fail(nullptr, FJB_E_CUDA, cudaGetErrorString(err));
    *tflops = 2.0 * 8.0 * iters * (double)threads * blocks / (best * 1e-3) / 1e12;
    return FJB_OK;
}

}  // namespace

extern "C" int fjb_fma_probe(int fp32, int reps, double *tflops) {
    if (!tflops || reps < 1) return fail(nullptr, FJB_E_ARG, "bad argument");
    return fp32 ? run_probe<float>(reps, tflops) : run_probe<double>(reps, tflops);
}

// ---------------------------------------------------------------------------
// fjb_fock_build_noalloc: the build with its scratch in a file-scope array
// ---------------------------------------------------------------------------
//
// The scratch -- J' and K' (n_ao^2 each, accumulated by atomics, so they
// must start at zero) and the shell-block maxima Dsh (n_sh^2) -- lives in
// g_noalloc_scratch instead of handle-owned buffers.  In host code the name
// g_noalloc_scratch is only a host-side stand-in for the array, not a device
// address; the address a kernel may use is looked up once per device, with
// that device current, by cudaGetSymbolAddress, and passed to the kernels.

namespace {

static __device__ __align__(256) double g_noalloc_scratch[FJB_NOALLOC_SCRATCH_DOUBLES];

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_ptr[kNoallocMaxDevices] = {};

// The device address of g_noalloc_scratch on `device` (current), looked up
// on the first call for that device.  Returns nullptr on failure.
double *noalloc_scratch(int device, std::string *why) {
    if (device < 0 || device >= kNoallocMaxDevices) {
        *why = "device ordinal out of range for the no-allocation scratch table";
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            *why = std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e);
            return nullptr;
        }
        g_noalloc_ptr[device] = static_cast<double *>(p);
    }
    return g_noalloc_ptr[device];
}

}  // namespace

extern "C" int fjb_fock_build_noalloc(fjb_handle *h, const double *D_dev, double *J_dev, double *K_dev,
                                      double *G_dev, void *stream) {
    if (!h || !D_dev) return fail(h, FJB_E_ARG, "null argument");
    if (!h->planned) return fail(h, FJB_E_STATE, "no plan: call fjb_plan first");
    if (h->device < 0) return fail(h, FJB_E_STATE, "host-only handle (device -1): no device work");
    const int nsh = (int)h->basis.shells.size(), nao = h->basis.n_ao;
    if (nao > FJB_NOALLOC_MAX_AO || nsh > FJB_NOALLOC_MAX_SHELLS)
        return fail(h, FJB_E_LIMIT,
                    "fjb_fock_build_noalloc: n_ao = " + std::to_string(nao) + ", n_shells = " +
                        std::to_string(nsh) + " exceed its fixed scratch (n_ao <= " +
                        std::to_string(FJB_NOALLOC_MAX_AO) + ", n_shells <= " +
                        std::to_string(FJB_NOALLOC_MAX_SHELLS) + "); use fjb_fock_build");
    CUDA_OK(h, cudaSetDevice(h->device));
    std::string why;
    double *scratch = noalloc_scratch(h->device, &why);
    if (!scratch) return fail(h, FJB_E_CUDA, why);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nn = (size_t)nao * nao;
    double *Jp = scratch, *Kp = scratch + nn, *Dsh = scratch + 2 * nn;
    density_blocks_kernel<<<(nsh * nsh + 255) / 256, 256, 0, st>>>(D_dev, nao, nsh, h->sh_off.p, h->sh_nc.p, Dsh);
    CUDA_OK(h, cudaMemsetAsync(Jp, 0, 2 * nn * sizeof(double), st));
    for (const ClassRun &r : h->runs) {
        KArgs a{};
        a.C = r.dev;
        a.units = h->units.p + r.unit0;
        a.n_units = r.n_units;
        a.launches = h->launches.p;
        a.pairs = h->pairs.p;
        a.prims = h->prims.p;
        a.D = D_dev;
        a.Dsh = Dsh;
        a.n_sh = nsh;
        a.n_ao = nao;
        a.tau = h->plan.tau;
        a.Jp = Jp;
        a.Kp = Kp;
        a.boys_tab = h->boys.p;
        CUDA_OK(h, launch_run(r, st, a));
    }
    close_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(Jp, Kp, nao, J_dev, K_dev, G_dev);
    CUDA_OK(h, cudaGetLastError());
    return FJB_OK;
}

// ---------------------------------------------------------------------------
// the batched build: many planned molecules, one launch per class
// ---------------------------------------------------------------------------

struct fjb_batch {
    int device = 0;
    double tau = 0.0;
    std::vector<fjb_handle *> mols;
    DevBuf<PairRec> pairs;
    DevBuf<PrimRec> prims;
    DevBuf<LaunchRec> launches;
    DevBuf<Unit> units;
    DevBuf<int32_t> launch_mol;
    DevBuf<MolCtx> ctx;
    DevBuf<BatchMol> bm;
    DevBuf<int> sh_off, sh_nc;
    DevBuf<double> Dsh, Jp, Kp;
    std::vector<MolCtx> ctx_host;
    std::vector<BatchMol> bm_host;
    std::vector<ClassRun> runs;
    int n_units = 0, max_nsh = 0;
    size_t max_nn = 0;
    DevBuf<int> route_list, route_counts;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> cev;
    bool ready = false;  // densities set
    std::string err;
    ~fjb_batch() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (auto &e : cev) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
    }
};

namespace {
int bfail(fjb_batch *b, int code, const std::string &msg) {
    if (b) b->err = msg;
    g_err = msg;
    return code;
}
#define BCUDA_OK(b, x)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            return bfail((b), FJB_E_CUDA, std::string(#x ": ") + cudaGetErrorString(e_));    \
    } while (0)
}  // namespace

extern "C" {

const char *fjb_batch_last_error(const fjb_batch *b) { return b ? b->err.c_str() : g_err.c_str(); }

int fjb_batch_create(fjb_batch **out, fjb_handle *const *handles, int n) {
    if (!out || !handles || n < 1) return bfail(nullptr, FJB_E_ARG, "fjb_batch_create: no molecules");
    auto b = std::make_unique<fjb_batch>();
    b->device = handles[0] ? handles[0]->device : -1;
    for (int m = 0; m < n; ++m) {
        fjb_handle *h = handles[m];
        if (!h || !h->planned || h->device < 0 || h->df)
            return bfail(nullptr, FJB_E_STATE, "fjb_batch_create: every handle must be a planned device handle");
        if (h->device != b->device) return bfail(nullptr, FJB_E_ARG, "fjb_batch_create: handles on different devices");
        if (m == 0) b->tau = h->plan.tau;
        if (h->plan.tau != b->tau) return bfail(nullptr, FJB_E_ARG, "fjb_batch_create: the plans' tau differ");
        b->mols.push_back(h);
    }
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(nullptr, FJB_E_CUDA, "cudaSetDevice failed");
    std::vector<PairRec> pr;
    std::vector<std::pair<const PrimRec *, size_t>> prim_src;  // each molecule's device primitive pairs
    int64_t n_prims = 0;
    std::vector<LaunchRec> lr;
    std::vector<int32_t> lmol;
    std::map<std::tuple<int, int, int, int>, std::vector<UnitSpan>> by_class;  // the molecules' spans
    std::map<std::tuple<int, int, int, int>, std::pair<const ClassRun *, std::pair<int, int>>> first;
    std::vector<int> sh_off, sh_nc;
    std::vector<int64_t> dsh0, nn0;
    int64_t dsh_total = 0, nn_total = 0;
    try {
        for (int m = 0; m < n; ++m) {
            fjb_handle *h = b->mols[m];
            const int P0 = (int)pr.size(), Q0 = (int)n_prims, L0 = (int)lr.size();
            prim_src.emplace_back(h->prims.p, h->prims.n);
            n_prims += (int64_t)h->prims.n;
            if (n_prims > (int64_t)INT32_MAX)
                return bfail(nullptr, FJB_E_LIMIT, "fjb_batch_create: more than 2^31 primitive pairs");
            for (PairRec p : h->pr_host) {
                p.prim0 += Q0;
                pr.push_back(p);
            }
            for (LaunchRec L : h->lr_host) {
                L.bra_pair0 += P0;
                L.ket_pair0 += P0;
                lr.push_back(L);
                lmol.push_back(m);
            }
            for (UnitSpan S : h->spans_host) {
                const fjb_launch_stat &ls = h->lstat[S.launch];
                S.launch += L0;
                by_class[std::make_tuple(ls.la, ls.lb, ls.lc, ls.ld)].push_back(S);
            }
            for (const ClassRun &r : h->runs) {
                const auto key = std::make_tuple(r.dev.la, r.dev.lb, r.dev.lc, r.dev.ld);
                auto it = first.find(key);
                if (it == first.end())
                    first[key] = {&r, {r.max_kab, r.max_kcd}};
                else
                    it->second.second = {std::max(it->second.second.first, r.max_kab),
                                         std::max(it->second.second.second, r.max_kcd)};
            }
            const int nsh = (int)h->basis.shells.size(), nao = h->basis.n_ao;
            BatchMol bmh{};
            bmh.n_sh = nsh;
            bmh.n_ao = nao;
            b->bm_host.push_back(bmh);
            sh_off.insert(sh_off.end(), h->basis.offsets.begin(), h->basis.offsets.begin() + nsh);
            for (auto &sh : h->basis.shells) sh_nc.push_back((sh.l + 1) * (sh.l + 2) / 2);
            dsh0.push_back(dsh_total);
            nn0.push_back(nn_total);
            dsh_total += (int64_t)nsh * nsh;
            nn_total += (int64_t)nao * nao;
            b->max_nsh = std::max(b->max_nsh, nsh);
            b->max_nn = std::max(b->max_nn, (size_t)nao * nao);
        }
        // the merged units, class by class, each class's molecules in order:
        // the molecules' spans re-based, the units written on the device
        std::vector<UnitSpan> spans;
        int64_t total = 0;
        for (auto &kv : by_class) {
            const ClassRun *src = first[kv.first].first;
            ClassRun r = *src;
            const int64_t u0 = total;
            for (UnitSpan S : kv.second) {
                S.base = total;
                total += S.count;
                spans.push_back(S);
            }
            if (total > (int64_t)INT32_MAX)
                return bfail(nullptr, FJB_E_LIMIT, "fjb_batch_create: more than 2^31 work units");
            r.unit0 = (int)u0;
            r.n_units = (int)(total - u0);
            r.max_kab = first[kv.first].second.first;
            r.max_kcd = first[kv.first].second.second;
            b->runs.push_back(r);
        }
        b->n_units = (int)total;
        b->pairs.upload(pr);
        b->prims.alloc(std::max<int64_t>(n_prims, 1));  // the molecules' records, device to device
        int64_t q = 0;
        for (auto &src : prim_src) {
            if (src.second && cudaMemcpy(b->prims.p + q, src.first, src.second * sizeof(PrimRec),
                                         cudaMemcpyDeviceToDevice) != cudaSuccess)
                throw std::runtime_error("copying a molecule's primitive pairs");
            q += (int64_t)src.second;
        }
        b->launches.upload(lr);
        b->units.alloc(std::max<int64_t>(total, 1));
        if (!spans.empty()) {
            DevBuf<UnitSpan> dspans;
            dspans.upload(spans);
            make_units_kernel<<<(unsigned)spans.size(), 128>>>(dspans.p, b->units.p);
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaStreamSynchronize(0);
            if (e != cudaSuccess) throw std::runtime_error(std::string("make_units_kernel: ") + cudaGetErrorString(e));
        }
        b->launch_mol.upload(lmol);
        b->sh_off.upload(sh_off);
        b->sh_nc.upload(sh_nc);
        b->Dsh.alloc(std::max<int64_t>(1, dsh_total));
        b->Jp.alloc(std::max<int64_t>(1, nn_total));
        b->Kp.alloc(std::max<int64_t>(1, nn_total));
        int sh0 = 0;
        for (int m = 0; m < n; ++m) {
            BatchMol &x = b->bm_host[m];
            x.Dsh = b->Dsh.p + dsh0[m];
            x.sh_off = b->sh_off.p + sh0;
            x.sh_nc = b->sh_nc.p + sh0;
            x.Jp = b->Jp.p + nn0[m];
            x.Kp = b->Kp.p + nn0[m];
            sh0 += x.n_sh;
            b->ctx_host.push_back(MolCtx{nullptr, x.Dsh, b->Jp.p + nn0[m], b->Kp.p + nn0[m], x.n_ao, x.n_sh});
        }
        b->ctx.alloc(n);
        b->bm.alloc(n);
        b->route_list.alloc(std::max<size_t>(1, 2 * (size_t)b->n_units));
        b->route_counts.alloc(std::max<size_t>(1, 4 * b->runs.size()));
    } catch (const std::exception &e) {
        return bfail(nullptr, FJB_E_CUDA, std::string("fjb_batch_create: ") + e.what());
    }
    for (auto &r : b->runs) {
        choose_rys(1, r);
        r.grid = run_grid(r);
        r.grid32 = run_grid32(r);
        if (!r.compiled && !r.rys64)
            return bfail(nullptr, FJB_E_LIMIT, "fjb_batch_create: a class has neither a register nor a Rys kernel");
        cudaEvent_t e0, e1;
        if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
            return bfail(nullptr, FJB_E_CUDA, "cudaEventCreate failed");
        b->cev.emplace_back(e0, e1);
    }
    if (cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess)
        return bfail(nullptr, FJB_E_CUDA, "cudaEventCreate failed");
    *out = b.release();
    return FJB_OK;
}

void fjb_batch_destroy(fjb_batch *b) { delete b; }

int fjb_batch_set_densities(fjb_batch *b, const double *const *D_dev, double *const *J_dev, double *const *K_dev,
                            double *const *G_dev) {
    if (!b || !D_dev) return bfail(b, FJB_E_ARG, "null argument");
    BCUDA_OK(b, cudaSetDevice(b->device));
    const size_t n = b->mols.size();
    for (size_t m = 0; m < n; ++m) {
        if (!D_dev[m]) return bfail(b, FJB_E_ARG, "fjb_batch_set_densities: a null density");
        b->ctx_host[m].D = D_dev[m];
        b->bm_host[m].D = D_dev[m];
        b->bm_host[m].J = J_dev ? J_dev[m] : nullptr;
        b->bm_host[m].K = K_dev ? K_dev[m] : nullptr;
        b->bm_host[m].G = G_dev ? G_dev[m] : nullptr;
    }
    BCUDA_OK(b, cudaMemcpy(b->ctx.p, b->ctx_host.data(), n * sizeof(MolCtx), cudaMemcpyHostToDevice));
    BCUDA_OK(b, cudaMemcpy(b->bm.p, b->bm_host.data(), n * sizeof(BatchMol), cudaMemcpyHostToDevice));
    b->ready = true;
    return FJB_OK;
}

int fjb_batch_build(fjb_batch *b, int precision, double threshold, void *stream) {
    if (!b) return bfail(b, FJB_E_ARG, "null batch");
    if (!b->ready) return bfail(b, FJB_E_STATE, "fjb_batch_build: set the densities first (fjb_batch_set_densities)");
    if (precision != FJB_FP64 && precision != FJB_ROUTED)
        return bfail(b, FJB_E_ARG, "fjb_batch_build: precision FJB_FP64 or FJB_ROUTED");
    const double route = precision == FJB_ROUTED ? (threshold > 0.0 ? threshold : 1e-9) : 0.0;
    BCUDA_OK(b, cudaSetDevice(b->device));
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned nm = (unsigned)b->mols.size();
    batch_density_blocks_kernel<<<dim3((unsigned)((b->max_nsh * b->max_nsh + 255) / 256), nm), 256, 0, st>>>(b->bm.p);
    BCUDA_OK(b, cudaMemsetAsync(b->Jp.p, 0, b->Jp.n * sizeof(double), st));
    BCUDA_OK(b, cudaMemsetAsync(b->Kp.p, 0, b->Kp.n * sizeof(double), st));
    const bool routed = route > 0.0;
    if (routed) BCUDA_OK(b, cudaMemsetAsync(b->route_counts.p, 0, b->route_counts.n * sizeof(int), st));
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    BCUDA_OK(b, cudaStreamIsCapturing(st, &cap));
    const unsigned ev_flags = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : 0u;
    BCUDA_OK(b, cudaEventRecordWithFlags(b->ev0, st, ev_flags));
    const fjb_handle *h0 = b->mols[0];
    for (size_t ri = 0; ri < b->runs.size(); ++ri) {
        const ClassRun &r = b->runs[ri];
        BCUDA_OK(b, cudaEventRecordWithFlags(b->cev[ri].first, st, ev_flags));
        KArgs a{};
        a.C = r.dev;
        a.units = b->units.p + r.unit0;
        a.n_units = r.n_units;
        a.launches = b->launches.p;
        a.pairs = b->pairs.p;
        a.prims = b->prims.p;
        a.tau = b->tau;
        a.boys_tab = h0->boys.p;
        a.mols = b->ctx.p;
        a.launch_mol = b->launch_mol.p;
        if (routed) {
            if (!r.has32 && !r.rys32)
                return bfail(b, FJB_E_LIMIT, "fjb_batch_build: a class has no FP32 kernel for routed units");
            int *l32 = b->route_list.p + r.unit0;
            int *l64 = b->route_list.p + b->n_units + r.unit0;
            int *cnt = b->route_counts.p + 4 * ri;
            const int rgrid = std::max(1, std::min((r.n_units + 3) / 4, 16 * sm_count()));
            // the first molecule's learned router routes the whole batch
            if (h0->router_on && r.dev.la + r.dev.lb + r.dev.lc + r.dev.ld >= h0->router_min_l)
                route_units_mlp_kernel<<<rgrid, 128, 0, st>>>(
                    b->units.p, r.unit0, r.n_units, b->launches.p, b->pairs.p, b->prims.p, nullptr, 0, b->tau,
                    route, h0->router_p.p, h0->router_log_thr, h0->router_reach, r.dev.la, r.dev.lb, r.dev.lc,
                    r.dev.ld, l32, l64,
                    cnt, 0, nullptr, b->ctx.p, b->launch_mol.p);
            else
                route_units_kernel<<<rgrid, 128, 0, st>>>(b->units.p, r.unit0, r.n_units, b->launches.p,
                                                          b->pairs.p, nullptr, 0, b->tau, route, l32, l64, cnt, 0,
                                                          nullptr, b->ctx.p, b->launch_mol.p);
            KArgs a32 = a, a64 = a;
            a32.unit_list = l32;
            a32.unit_count = cnt;
            a64.unit_list = l64;
            a64.unit_count = cnt + 1;
            BCUDA_OK(b, launch_run32(r, st, a32));
            BCUDA_OK(b, launch_run(r, st, a64));
        } else {
            BCUDA_OK(b, launch_run(r, st, a));
        }
        BCUDA_OK(b, cudaEventRecordWithFlags(b->cev[ri].second, st, ev_flags));
    }
    BCUDA_OK(b, cudaEventRecordWithFlags(b->ev1, st, ev_flags));
    const unsigned cx = (unsigned)std::min<size_t>((b->max_nn + 255) / 256, 1024);
    batch_close_kernel<<<dim3(cx, nm), 256, 0, st>>>(b->bm.p);
    BCUDA_OK(b, cudaGetLastError());
    return FJB_OK;
}

int fjb_batch_stats(const fjb_batch *bc, double *ms, int64_t *n_classes, int64_t *n_units) {
    fjb_batch *b = const_cast<fjb_batch *>(bc);
    if (!b) return bfail(b, FJB_E_ARG, "null batch");
    if (n_classes) *n_classes = (int64_t)b->runs.size();
    if (n_units) *n_units = b->n_units;
    if (ms) {
        float f = 0.f;
        BCUDA_OK(b, cudaEventSynchronize(b->ev1));
        BCUDA_OK(b, cudaEventElapsedTime(&f, b->ev0, b->ev1));
        *ms = f;
    }
    return FJB_OK;
}

}  // extern "C"
