// scatter.cpp -- the atomics-free write-back's map (scatter.h).
#include "scatter.h"

#include <algorithm>
#include <limits>
#include <stdexcept>

namespace fjb {

SlotShape slot_shape(const int l[4]) {
    SlotShape s{};
    for (int k = 0; k < 4; ++k) s.n[k] = (l[k] + 1) * (l[k] + 2) / 2;
    s.n_ab = s.n[0] * s.n[1];
    s.n_cd = s.n[2] * s.n[3];
    // BLOCKS[1:] = cd, ac, ad, bc, bd
    const int sizes[5] = {s.n[2] * s.n[3], s.n[0] * s.n[2], s.n[0] * s.n[3], s.n[1] * s.n[2], s.n[1] * s.n[3]};
    int at = 0;
    for (int b = 0; b < 5; ++b) {
        s.koff[b] = at;
        at += sizes[b];
    }
    s.s5 = at;
    return s;
}

ScatterMap scatter_map(const int l[4], const std::vector<std::pair<int, int>> &bra_ao,
                       const std::vector<std::pair<int, int>> &ket_ao) {
    const SlotShape S = slot_shape(l);
    const int64_t n_bra = (int64_t)bra_ao.size(), n_ket = (int64_t)ket_ao.size();
    const int64_t row = S.n_ab + (int64_t)S.s5 * n_ket;
    const int64_t total = n_bra * row;
    if (total > std::numeric_limits<int32_t>::max())
        throw std::length_error("a launch's slots exceed an int32 index: split the launch");
    // (element key, slot) for every slot; the key orders (row, col) ascending
    std::vector<std::pair<int64_t, int32_t>> ts((size_t)total);
    auto key = [](int r, int c) { return ((int64_t)r << 32) | (uint32_t)c; };
    // the four shells of a quartet: a, b (bra) and c, d (ket); block (x, y)
    const int bx[5] = {2, 0, 0, 1, 1}, by[5] = {3, 2, 3, 2, 3};
    for (int64_t bra = 0; bra < n_bra; ++bra) {
        const int64_t base = bra * row;
        const int oa = bra_ao[bra].first, ob = bra_ao[bra].second;
        for (int i = 0; i < S.n[0]; ++i)
            for (int j = 0; j < S.n[1]; ++j) {
                const int64_t slot = base + i * S.n[1] + j;
                ts[slot] = {key(oa + i, ob + j), (int32_t)slot};
            }
        for (int64_t k = 0; k < n_ket; ++k) {
            const int o[4] = {oa, ob, ket_ao[k].first, ket_ao[k].second};
            for (int b = 0; b < 5; ++b)
                for (int i = 0; i < S.n[bx[b]]; ++i)
                    for (int j = 0; j < S.n[by[b]]; ++j) {
                        const int64_t slot = base + S.n_ab + (int64_t)(S.koff[b] + i * S.n[by[b]] + j) * n_ket + k;
                        ts[slot] = {key(o[bx[b]] + i, o[by[b]] + j), (int32_t)slot};
                    }
        }
    }
    std::sort(ts.begin(), ts.end());  // by element, then by slot: each element's slots ascending
    ScatterMap m;
    m.n_slot = total;
    m.src.reserve((size_t)total);
    m.ptr.push_back(0);
    for (size_t t = 0; t < ts.size(); ++t) {
        if (t == 0 || ts[t].first != ts[t - 1].first) {
            if (t) m.ptr.push_back((int32_t)t);
            m.el.push_back((int32_t)(ts[t].first >> 32));
            m.el.push_back((int32_t)(ts[t].first & 0xffffffff));
        }
        m.src.push_back(ts[t].second);
    }
    if (!ts.empty()) m.ptr.push_back((int32_t)ts.size());
    m.n_el = (int64_t)m.el.size() / 2;
    return m;
}

}  // namespace fjb
