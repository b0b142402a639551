// hgp_tables.h -- per-class recurrence programs for the HGP kernels, built on
// the host once per class.
#pragma once
#include <array>
#include <vector>

#include "fjb_internal.h"

namespace fjb {

using Cart = std::array<int, 3>;

std::vector<Cart> cartesians(int l);  // i desc, then j desc (ao/shell.py:68)
inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// The host side of one class (la lb | lc ld): the VRR program (Head-Gordon-
// Pople eqs. 25-26 as a level-ordered list of node updates), the boundary
// map, and the HRR as two sparse binomial transforms.
struct ClassHost {
    int la = 0, lb = 0, lc = 0, ld = 0;
    int na = 0, nb = 0, nc = 0, nd = 0, nab = 0, ncd = 0, L = 0;
    int n_nodes = 0;  // including the zero node 0 and the scratch node 1
    int nbe = 0, nbf = 0;
    std::vector<int> level_off;
    std::vector<VOp> ops;
    std::vector<uint16_t> leaf, tgt;
    std::vector<HCoef> cb, ck;
    std::vector<int> bra_off, ket_off;
    std::vector<HTerm> bra_terms, ket_terms;
    int vrr_nodes() const { return n_nodes - 2; }  // the DAG's own node count
    int n_levels() const { return (int)level_off.size() - 1; }
    int hrr_terms() const { return (int)(bra_terms.size() * nbf + ket_terms.size() * nab); }
};

ClassHost build_class(int la, int lb, int lc, int ld);

// Shared-memory carve-up of a class for staging degrees up to kab/kcd, a
// CTA of `threads`, and a chunk of (ket, primitive quartet) slots sized so
// the CTA stays within `target_doubles` when it can (`slots` > 0 forces the
// chunk).  The recurrence regions hold values of `rsize` bytes (8: the FP64
// kernel; 4: the routed path's FP32 kernel).  Returns false if the class
// cannot fit the hard budget.
bool layout_class(const ClassHost &c, int max_kab, int max_kcd, int budget_doubles, int threads,
                  int target_doubles, int slots, ClassDev *out, int rsize = 8);

// The default CTA width and shared-memory target of a class: narrow CTAs
// (a warp) for small programs so many CTAs share an SM, wider ones for the
// large programs whose levels hold thousands of independent updates.
void default_config(const ClassHost &c, int budget_doubles, int *threads, int *target_doubles);

}  // namespace fjb
