// hgp_tables.cpp -- building the per-class recurrence programs.
//
// VRR (Head-Gordon & Pople, eqs. 25-26; the reference's hgp/vrr.py:1-60 states
// the same reduction rule): a node [e,0|f,0]^(m) with f != 0 is reduced along
// the first nonzero axis d of f,
//   [e|f+1_d]^(m) = QC_d [e|f]^(m) + WQ_d [e|f]^(m+1)
//                 + f_d/(2q) ([e|f-1_d]^(m) - rho/q [e|f-1_d]^(m+1))
//                 + e_d/(2(p+q)) [e-1_d|f]^(m+1),
// else (e != 0) along the first nonzero axis of e by the bra twin; [0|0]^(m)
// is a Boys leaf.  The program is the closure of the boundary set
// {(e, f, 0): la <= |e| <= la+lb, lc <= |f| <= lc+ld} under that rule, so its
// node count equals the reference's pruned DAG (hgp/vrr.py:245 build), which
// tests/test_tables.py checks class by class.  Nodes are grouped into levels
// that read only lower levels: the leaves, then the bra nodes by |e|, then the
// ket nodes by |f|; all updates of one level run in parallel.
//
// HRR: instead of the reference's two-term DAG (hgp/hrr.py:1-60), the
// transfer is applied as the closed binomial sum it telescopes to,
//   (a b| = sum_{k <= b} prod_d C(b_d, k_d) AB_d^(b_d - k_d) (a+k, 0|,
// from (x - B) = (x - A) + AB, first on the bra, then on the ket with CD:
// every output is independent, so one CTA pass does each side.
#include "hgp_tables.h"

#include <algorithm>
#include <map>
#include <stdexcept>
#include <tuple>

namespace fjb {

std::vector<Cart> cartesians(int l) {
    std::vector<Cart> out;
    for (int i = l; i >= 0; --i)
        for (int j = l - i; j >= 0; --j) out.push_back({i, j, l - i - j});
    return out;
}

namespace {

struct Node {
    Cart e, f;
    int m;
    bool operator<(const Node &o) const {
        return std::tie(e, f, m) < std::tie(o.e, o.f, o.m);
    }
};

int asum(const Cart &c) { return c[0] + c[1] + c[2]; }
bool is_zero(const Cart &c) { return c[0] == 0 && c[1] == 0 && c[2] == 0; }
int first_nz(const Cart &c) { return c[0] ? 0 : (c[1] ? 1 : 2); }

struct Reduction {
    bool leaf = true;
    int d = 0, kind = 0, c2 = 0, c4 = 0;
    // children: s0 = lowered (m), s1 = lowered (m+1), s2/s3 = lowered twice
    // (m, m+1), s4 = coupling (e-1_d, f-1_d, m+1)
    bool has[5] = {false, false, false, false, false};
    Node ch[5];
};

Reduction reduce(const Node &n) {
    Reduction r;
    if (!is_zero(n.f)) {
        int d = first_nz(n.f);
        Cart f1 = n.f;
        f1[d] -= 1;
        r.leaf = false;
        r.d = d;
        r.kind = 1;
        r.c2 = f1[d];
        r.c4 = n.e[d];
        r.has[0] = r.has[1] = true;
        r.ch[0] = {n.e, f1, n.m};
        r.ch[1] = {n.e, f1, n.m + 1};
        if (f1[d] >= 1) {
            Cart f2 = f1;
            f2[d] -= 1;
            r.has[2] = r.has[3] = true;
            r.ch[2] = {n.e, f2, n.m};
            r.ch[3] = {n.e, f2, n.m + 1};
        }
        if (n.e[d] >= 1) {
            Cart e1 = n.e;
            e1[d] -= 1;
            r.has[4] = true;
            r.ch[4] = {e1, f1, n.m + 1};
        }
    } else if (!is_zero(n.e)) {
        int d = first_nz(n.e);
        Cart e1 = n.e;
        e1[d] -= 1;
        r.leaf = false;
        r.d = d;
        r.kind = 0;
        r.c2 = e1[d];
        r.c4 = 0;
        r.has[0] = r.has[1] = true;
        r.ch[0] = {e1, n.f, n.m};
        r.ch[1] = {e1, n.f, n.m + 1};
        if (e1[d] >= 1) {
            Cart e2 = e1;
            e2[d] -= 1;
            r.has[2] = r.has[3] = true;
            r.ch[2] = {e2, n.f, n.m};
            r.ch[3] = {e2, n.f, n.m + 1};
        }
    }
    return r;
}

int binom(int n, int k) {
    int r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

// One side's HRR transform: rows (x, y) of cartesians(lx) x cartesians(ly),
// each a list of (boundary index of x + k, coefficient index of (y, k)).
void hrr_side(int lx, int ly, const std::map<Cart, int> &bidx, std::vector<HCoef> &coefs,
              std::vector<int> &off, std::vector<HTerm> &terms) {
    auto cx = cartesians(lx), cy = cartesians(ly);
    std::map<std::pair<int, Cart>, int> cmap;
    off.clear();
    terms.clear();
    coefs.clear();
    for (size_t i = 0; i < cx.size(); ++i)
        for (size_t j = 0; j < cy.size(); ++j) {
            off.push_back((int)terms.size());
            const Cart &b = cy[j];
            for (int kx = 0; kx <= b[0]; ++kx)
                for (int ky = 0; ky <= b[1]; ++ky)
                    for (int kz = 0; kz <= b[2]; ++kz) {
                        Cart k = {kx, ky, kz};
                        Cart e = {cx[i][0] + kx, cx[i][1] + ky, cx[i][2] + kz};
                        auto key = std::make_pair((int)j, k);
                        auto it = cmap.find(key);
                        int ci;
                        if (it == cmap.end()) {
                            ci = (int)coefs.size();
                            cmap[key] = ci;
                            HCoef hc;
                            hc.binom = (float)(binom(b[0], kx) * binom(b[1], ky) * binom(b[2], kz));
                            hc.px = (uint8_t)(b[0] - kx);
                            hc.py = (uint8_t)(b[1] - ky);
                            hc.pz = (uint8_t)(b[2] - kz);
                            hc.pad = 0;
                            coefs.push_back(hc);
                        } else {
                            ci = it->second;
                        }
                        terms.push_back({(uint16_t)bidx.at(e), (uint16_t)ci});
                    }
        }
    off.push_back((int)terms.size());
}

}  // namespace

ClassHost build_class(int la, int lb, int lc, int ld) {
    if (la < 0 || lb < 0 || lc < 0 || ld < 0 || la > 6 || lb > 6 || lc > 6 || ld > 6)
        throw std::invalid_argument("class angular momentum out of range");
    ClassHost c;
    c.la = la;
    c.lb = lb;
    c.lc = lc;
    c.ld = ld;
    c.na = ncart(la);
    c.nb = ncart(lb);
    c.nc = ncart(lc);
    c.nd = ncart(ld);
    c.nab = c.na * c.nb;
    c.ncd = c.nc * c.nd;
    c.L = la + lb + lc + ld;
    const int Lbra = la + lb;

    std::vector<Cart> eb, fb;
    std::map<Cart, int> ebi, fbi;
    for (int n = la; n <= la + lb; ++n)
        for (auto &e : cartesians(n)) {
            ebi[e] = (int)eb.size();
            eb.push_back(e);
        }
    for (int n = lc; n <= lc + ld; ++n)
        for (auto &f : cartesians(n)) {
            fbi[f] = (int)fb.size();
            fb.push_back(f);
        }
    c.nbe = (int)eb.size();
    c.nbf = (int)fb.size();

    // closure of the targets under the reduction rule
    std::map<Node, Reduction> dag;
    std::vector<Node> todo;
    for (auto &e : eb)
        for (auto &f : fb) todo.push_back({e, f, 0});
    while (!todo.empty()) {
        Node n = todo.back();
        todo.pop_back();
        if (dag.count(n)) continue;
        Reduction r = reduce(n);
        dag[n] = r;
        for (int k = 0; k < 5; ++k)
            if (r.has[k] && !dag.count(r.ch[k])) todo.push_back(r.ch[k]);
    }
    auto level_of = [&](const Node &n) {
        if (!is_zero(n.f)) return Lbra + asum(n.f);
        return asum(n.e);
    };
    int n_levels = Lbra + (lc + ld) + 1;
    std::vector<std::vector<Node>> levels(n_levels);
    for (auto &kv : dag) levels[level_of(kv.first)].push_back(kv.first);
    std::map<Node, int> idx;
    int next = 2;
    for (auto &lv : levels)
        for (auto &n : lv) idx[n] = next++;
    c.n_nodes = next;
    if (c.n_nodes > 65535) throw std::length_error("VRR program too large");

    c.leaf.assign(c.L + 1, 1);
    for (auto &n : levels[0]) c.leaf[n.m] = (uint16_t)idx[n];
    c.level_off.push_back(0);
    for (int lv = 1; lv < n_levels; ++lv) {
        if (levels[lv].empty()) continue;
        for (auto &n : levels[lv]) {
            const Reduction &r = dag[n];
            VOp op;
            op.dst = (uint16_t)idx[n];
            uint16_t s[5];
            for (int k = 0; k < 5; ++k) s[k] = r.has[k] ? (uint16_t)idx.at(r.ch[k]) : 0;
            op.s0 = s[0];
            op.s1 = s[1];
            op.s2 = s[2];
            op.s3 = s[3];
            op.s4 = s[4];
            op.d = (uint8_t)r.d;
            op.kind = (uint8_t)r.kind;
            op.c2 = (uint8_t)r.c2;
            op.c4 = (uint8_t)r.c4;
            c.ops.push_back(op);
        }
        c.level_off.push_back((int)c.ops.size());
    }
    c.tgt.resize((size_t)c.nbe * c.nbf);
    for (int i = 0; i < c.nbe; ++i)
        for (int j = 0; j < c.nbf; ++j) c.tgt[(size_t)i * c.nbf + j] = (uint16_t)idx.at({eb[i], fb[j], 0});

    hrr_side(la, lb, ebi, c.cb, c.bra_off, c.bra_terms);
    hrr_side(lc, ld, fbi, c.ck, c.ket_off, c.ket_terms);
    return c;
}

void default_config(const ClassHost &c, int budget, int *threads, int *target) {
    // About 16 warps an SM in every regime: many one-warp CTAs for small
    // programs, four 128-thread CTAs for mid-size ones, one 512-thread CTA
    // for the largest (whose shared memory allows a single CTA an SM).
    if (c.n_nodes <= 1200) {
        *threads = 32;
        *target = budget / 16;
    } else if (c.n_nodes <= 4000) {
        *threads = 128;
        *target = budget / 4;
    } else {
        *threads = 512;
        *target = budget;
    }
}

namespace {

// One carve-up attempt.  stage_leaves: room for the single-slot path's Boys
// leaves of every primitive quartet of a quartet (one slot allowed);
// without it the class keeps at least two slots (the slot path, which
// evaluates its leaves slot by slot).
bool layout_try(const ClassHost &c, int max_kab, int max_kcd, int budget, int threads, int target,
                int force_slots, ClassDev *o, int rsize, bool stage_leaves) {
    *o = ClassDev{};
    o->la = c.la;
    o->lb = c.lb;
    o->lc = c.lc;
    o->ld = c.ld;
    o->na = c.na;
    o->nb = c.nb;
    o->nc = c.nc;
    o->nd = c.nd;
    o->nab = c.nab;
    o->ncd = c.ncd;
    o->L = c.L;
    o->n_nodes = c.n_nodes;
    o->n_levels = c.n_levels();
    o->nbe = c.nbe;
    o->nbf = c.nbf;
    o->n_cb = (int)c.cb.size();
    o->n_ck = (int)c.ck.size();
    // regions of recurrence values (V, bound, S, cb, ck) hold R (rsize
    // bytes); the rest is FP64.  rd(): R elements -> doubles, rounded up
    // to an even count (16-byte alignment).
    auto rd = [&](long n) { return (int)((((n * rsize + 7) / 8) + 1) & ~1L); };
    auto dd = [&](long n) { return (int)((n + 1) & ~1L); };
    const int hr = c.nab * c.nbf + c.nab * c.ncd;
    const int dblk = c.nab + c.ncd + c.na * c.nc + c.na * c.nd + c.nb * c.nc + c.nb * c.nd;
    const int min_slots = stage_leaves ? 1 : 2;
    const int fleaves = stage_leaves ? max_kab * max_kcd * (c.L + 1) : 0;
    const int fixed = dd(kPrimWords * max_kab) + rd(o->n_cb) + rd(o->n_ck) + dd(dblk) + dd(c.nab) + dd(fleaves);
    // Slots span (ket, primitive quartet) pairs: up to one per thread, and
    // no more than a full unit of kets needs.
    int want = std::max(min_slots, std::min(threads, kKetChunk * max_kab * max_kcd));
    int slots = force_slots > 0 ? std::max(min_slots, std::min(force_slots, threads)) : want;
    auto group = [&](int s) { return std::max(1, std::min(kKetChunk, s)); };
    // per ket of a group: its boundary and its staged primitive pairs
    auto total = [&](int s) {
        return rd(std::max((long)s * c.n_nodes, (long)hr)) + rd((long)s * kNumScalars) + fixed +
               rd((long)group(s) * c.nbe * c.nbf) + dd((long)group(s) * kPrimWords * max_kcd);
    };
    // Occupancy first: shrink the chunk until the CTA fits its target,
    // unless one slot already needs more; then stay inside the hard budget.
    if (force_slots <= 0)
        while (slots > min_slots && total(slots) > target) --slots;
    while (slots > min_slots && total(slots) > budget) --slots;
    o->threads = threads;
    if (total(slots) > budget) return false;
    o->slots = slots;
    o->group = group(slots);
    o->vregion = std::max(slots * c.n_nodes, hr);
    int off = 0;
    auto take = [&](int n_doubles) {
        int r = off;
        off += n_doubles;
        return r;
    };
    o->sm_V = take(rd(o->vregion));
    o->sm_bound = take(rd((long)o->group * c.nbe * c.nbf));
    o->sm_S = take(rd((long)slots * kNumScalars));
    o->sm_braP = take(dd(kPrimWords * max_kab));
    o->sm_ketP = take(dd((long)o->group * kPrimWords * max_kcd));
    o->sm_cb = take(rd(o->n_cb));
    o->sm_ck = take(rd(o->n_ck));
    o->sm_D = take(dd(dblk));
    o->sm_Jab = take(dd(c.nab));
    o->sm_F = take(dd(fleaves));
    o->sm_total = off;
    return off <= budget;
}

}  // namespace

bool layout_class(const ClassHost &c, int max_kab, int max_kcd, int budget, int threads, int target,
                  int force_slots, ClassDev *o, int rsize) {
    // The single-slot path's staged leaves first (every layout of the
    // degrees the kernels were tuned on); a class whose leaves do not fit
    // beside its values (high contraction degrees) runs on two or more slots.
    return layout_try(c, max_kab, max_kcd, budget, threads, target, force_slots, o, rsize, true) ||
           layout_try(c, max_kab, max_kcd, budget, threads, target, force_slots, o, rsize, false);
}

}  // namespace fjb
