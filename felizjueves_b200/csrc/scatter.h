// scatter.h -- the atomics-free write-back's slot layout and map (host).
//
// In the atomics-free build each launch stores every contribution it would
// have added to J' / K' into its own slot of a buffer W, and a scatter then
// sums, per element of J' / K', that element's slots in ascending slot
// order.  The layout and the map are the reference's
// (eri/fock/levers/scatter.py:141-198, eri/fock/kernel_f_scatter.py:203-260):
//   row      = n_ab + S5 * n_ket         one bra pair's slots
//   slot_ab  = bra * row + e             bra block element e = i * n_b + j
//   slot_ket = bra * row + n_ab + (koff[block] + i * n_y + j) * n_ket + k
// with the five ket-dependent blocks in BLOCKS order (cd, ac, ad, bc, bd)
// and S5 their total size; the map lists the distinct elements (row, col)
// ascending, the CSR offsets, and per element its slots ascending.
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

namespace fjb {

struct ScatterMap {
    int64_t n_el = 0, n_slot = 0;
    std::vector<int32_t> el;   // 2 * n_el: (row, col) pairs
    std::vector<int32_t> ptr;  // n_el + 1
    std::vector<int32_t> src;  // n_slot, a permutation of 0 .. n_slot-1
};

// Block sizes of class (l[0] l[1] | l[2] l[3]): n_ab and the five ket blocks.
struct SlotShape {
    int n[4];
    int n_ab, n_cd, s5;
    int koff[5];  // offsets of cd, ac, ad, bc, bd inside S5
};
SlotShape slot_shape(const int l[4]);

// The map of one launch: its class, its bra and ket pairs' AO offsets
// (a, b) in batch order.  Throws std::length_error when the launch has more
// slots than an int32 index holds.
ScatterMap scatter_map(const int l[4], const std::vector<std::pair<int, int>> &bra_ao,
                       const std::vector<std::pair<int, int>> &ket_ao);

}  // namespace fjb
