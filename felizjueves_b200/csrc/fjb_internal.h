// fjb_internal.h -- structures shared by the host runtime (C++) and the
// sm_100a kernels.  Not part of the public ABI (include/fjb.h is).
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define FJB_HD __host__ __device__
#else
#define FJB_HD
#endif

namespace fjb {

constexpr int kMaxL = 3;          // per shell in the Fock build
constexpr int kMaxLQuartet = 4 * kMaxL;
constexpr int kBoysMaxM = 24;     // orders held by the Taylor table
constexpr int kBoysTaylor = 7;    // Taylor terms (orders m .. m+6)
constexpr double kBoysDelta = 0.05;
constexpr double kBoysTMax = 40.0;  // table covers [0, kBoysTMax]
constexpr int kBoysNT = 801;        // kBoysTMax / kBoysDelta + 1
constexpr int kBoysRow = kBoysMaxM + 2;  // F_0 .. F_kBoysMaxM, then exp(-T_i)
constexpr int kThreads = 128;       // widest CTA of the HGP kernel's default choice
constexpr int kMaxThreads = 512;    // widest CTA the kernel is instantiated for
constexpr int kKetChunk = 32;       // ket pairs per work unit (one per lane of a warp)
constexpr int kSmemBudgetDoubles = 27648;  // the HGP kernel's shared memory: 216 KiB of the 227 KiB a CTA may hold
constexpr int kNumScalars = 17;     // per-primitive-quartet VRR scalars

// One VRR node update, 16 bytes.  value(dst) =
//   A_d V[s0] + B_d V[s1] + c2 (C V[s2] - Dc V[s3]) + c4 E V[s4]
// with (A, B, C, Dc) the bra set (PA, WP, 1/2p, rho/(2p^2)) for kind 0 and
// the ket set (QC, WQ, 1/2q, rho/(2q^2)) for kind 1; E = 1/(2(p+q)).
// Absent terms point at node 0, which always holds 0.
struct VOp {
    uint16_t dst, s0, s1, s2, s3, s4;
    uint8_t d, kind, c2, c4;
};
static_assert(sizeof(VOp) == 16, "VOp is 16 bytes");

// One HRR transform term: out += coef[cidx] * in[src].
struct HTerm {
    uint16_t src, cidx;
};

// A binomial coefficient of the HRR: binom * sep_x^px sep_y^py sep_z^pz.
struct HCoef {
    float binom;
    uint8_t px, py, pz, pad;
};

// A primitive pair as staged for the kernels: P, X = P - A (first centre),
// zeta, U = c_a c_b (pi/zeta)^{3/2} exp(-alpha beta/zeta |AB|^2), and
// h = 1/(2 zeta) (the VRR's e/(2 zeta) factor, so no primitive quartet
// divides by zeta); 80 bytes.
struct PrimRec {
    double P[3], X[3], zeta, U, h, pad;
};
constexpr int kPrimWords = 10;  // doubles per PrimRec
static_assert(sizeof(PrimRec) == kPrimWords * sizeof(double), "PrimRec is kPrimWords doubles");

// A contracted shell pair (canonical: la <= lb, lower index first on a tie).
struct PairRec {
    int32_t a, b, ao_a, ao_b;
    int32_t prim0, nprim, pad0, pad1;
    double G;
    double AB[3];
};

// One launch: a bra batch against a ket batch (bra <= ket).
struct LaunchRec {
    int32_t bra_pair0, n_bra, ket_pair0, n_ket;
    int32_t diag, cls, pad0, pad1;
    int64_t qbase;  // index of this launch's first quartet in screen order
};

// A work unit: bra pair ib of launch `launch`, ket pairs [k0, k1).
struct Unit {
    int32_t launch, ib, k0, k1;
};

// The work units of one launch: for each bra pair ib, its kets from k_begin
// (ib on a diagonal launch, where the bra and ket batches are one; else 0)
// in chunks of kKetChunk.  base is the launch's first unit in the plan's
// unit order (class by class, each class's launches in plan order).
struct UnitSpan {
    int64_t base, count;
    int32_t launch, n_bra, n_ket, diag;
};

// sum over m = 1..x of ceil(m / kKetChunk): the units of a diagonal launch's
// last x bra pairs
FJB_HD inline int64_t diag_chunk_sum(int64_t x) {
    const int64_t q = x / kKetChunk, r = x % kKetChunk;
    return kKetChunk * q * (q + 1) / 2 + r * (q + 1);
}

FJB_HD inline int64_t span_units(const UnitSpan &S) {
    if (S.diag) return diag_chunk_sum(S.n_ket);
    return (int64_t)S.n_bra * ((S.n_ket + kKetChunk - 1) / kKetChunk);
}

// Bra pair ib's units, written at their place in units[]: the host and the
// device fill the plan's unit list with this same code.
FJB_HD inline void write_span_units(const UnitSpan &S, int ib, Unit *units) {
    const int k_begin = S.diag ? ib : 0;
    int64_t at = S.base + (S.diag ? diag_chunk_sum(S.n_ket) - diag_chunk_sum(S.n_ket - ib)
                                  : (int64_t)ib * ((S.n_ket + kKetChunk - 1) / kKetChunk));
    const int64_t end = S.base + S.count;
    for (int k0 = k_begin; k0 < S.n_ket && at < end; k0 += kKetChunk)
        units[at++] = Unit{S.launch, ib, k0, k0 + kKetChunk < S.n_ket ? k0 + kKetChunk : S.n_ket};
}

// Device view of one class's tables (all pointers are device pointers).
struct ClassDev {
    int la, lb, lc, ld;
    int na, nb, nc, nd, nab, ncd;
    int L;
    int n_nodes;      // including node 0 (zero) and node 1 (scratch)
    int n_levels;
    int nbe, nbf;     // boundary extents (e with la<=|e|<=la+lb, f likewise)
    int n_cb, n_ck;   // HRR coefficient counts
    int slots;        // (ket, primitive quartet) slots per VRR chunk
    int group;        // kets whose VRR runs together (at most kKetChunk)
    int threads;      // CTA width: 32, 64, 128, 256 or 512
    const int *level_off;   // [n_levels + 1] into ops
    const VOp *ops;
    const uint16_t *leaf;   // [L + 1] node of [0|0]^(m), 1 (the scratch node) if unread
    const uint16_t *tgt;    // [nbe * nbf] node of boundary (e, f)
    const HCoef *cb;        // [n_cb]
    const int *bra_off;     // [nab + 1]
    const HTerm *bra_terms;
    const HCoef *ck;        // [n_ck]
    const int *ket_off;     // [ncd + 1]
    const HTerm *ket_terms;
    // shared-memory carve-up, in doubles
    int sm_V, sm_bound, sm_S, sm_braP, sm_ketP, sm_cb, sm_ck, sm_D, sm_Jab, sm_F;
    int sm_total;
    int vregion;      // doubles in the V region (also holds X and Y)
};

// The Rys kernel's launch configuration and shared-memory carve-up (offsets
// in doubles), chosen on the host per class and precision (rys_fock.cu).
struct RysDev {
    int threads;   // CTA width
    int group;     // kets per group (G)
    int chunk;     // primitive quartets per table chunk (P)
    int kab, kcd;  // staged primitive-pair capacity of a bra and of a ket
    int sm_braP, sm_cb, sm_Dab, sm_Jab, sm_ketP, sm_ck, sm_Dk, sm_tab, sm_X, sm_total;
};

}  // namespace fjb
