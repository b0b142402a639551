// Checks the HGP kernel's shared-memory carve-up (hgp_tables.cpp
// layout_class) for every Fock class, recurrence size, CTA width, forced
// slot count and contraction degrees: each region inside the budget, 16-byte
// aligned, disjoint, and as large as the kernel reads.  Prints one line per
// violation and a final count; built and run by tests/test_layouts.py.
#include <cstdio>
#include <vector>

#include "hgp_tables.h"

using namespace fjb;

int main() {
    long n = 0, bad = 0, nofit = 0;
    for (int la = 0; la <= 3; ++la)
        for (int lb = la; lb <= 3; ++lb)
            for (int lc = 0; lc <= 3; ++lc)
                for (int ld = lc; ld <= 3; ++ld) {
                    if (la * 4 + lb > lc * 4 + ld) continue;
                    const ClassHost c = build_class(la, lb, lc, ld);
                    const int hr = c.nab * c.nbf + c.nab * c.ncd;
                    const int dblk = c.nab + c.ncd + c.na * c.nc + c.na * c.nd + c.nb * c.nc + c.nb * c.nd;
                    for (int rs : {8, 4})
                        for (int kab : {1, 3, 9, 16, 81, 121})
                            for (int kcd : {1, 3, 9, 81, 121})
                                for (int th : {0, 32, 64, 128, 256, 512})
                                    for (int force : {0, 1, 2}) {
                                        int threads = 0, target = 0;
                                        default_config(c, kSmemBudgetDoubles, &threads, &target);
                                        if (th > 0) {
                                            threads = th;
                                            target = kSmemBudgetDoubles * th / (16 * 32);
                                        }
                                        ClassDev d;
                                        ++n;
                                        if (!layout_class(c, kab, kcd, kSmemBudgetDoubles, threads, target, force, &d, rs)) {
                                            ++nofit;
                                            continue;
                                        }
                                        auto R = [&](long k) { return (k * rs + 7) / 8; };  // R values -> doubles
                                        struct Reg { const char *name; int off; long need; };
                                        const long vneed = R((long)(d.slots == 1 ? std::max(c.n_nodes, hr)
                                                                                  : std::max((long)d.slots * c.n_nodes, (long)hr)));
                                        std::vector<Reg> regs = {
                                            {"V", d.sm_V, vneed},
                                            {"bound", d.sm_bound, R((long)d.group * c.nbe * c.nbf)},
                                            {"S", d.sm_S, R((long)d.slots * kNumScalars)},
                                            {"braP", d.sm_braP, (long)kPrimWords * kab},
                                            {"ketP", d.sm_ketP, (long)d.group * kPrimWords * kcd},
                                            {"cb", d.sm_cb, R(d.n_cb)},
                                            {"ck", d.sm_ck, R(d.n_ck)},
                                            {"D", d.sm_D, dblk},
                                            {"Jab", d.sm_Jab, c.nab},
                                            {"F", d.sm_F, d.slots == 1 ? (long)kab * kcd * (c.L + 1) : 0}};
                                        const int offs[] = {d.sm_V, d.sm_bound, d.sm_S, d.sm_braP, d.sm_ketP,
                                                            d.sm_cb, d.sm_ck, d.sm_D, d.sm_Jab, d.sm_F, d.sm_total};
                                        bool ok = d.sm_total <= kSmemBudgetDoubles && d.slots >= 1 &&
                                                  d.group >= 1 && d.group <= kKetChunk;
                                        for (size_t k = 0; k < regs.size(); ++k) {
                                            const long room = offs[k + 1] - offs[k];
                                            if (regs[k].off % 2 || room < regs[k].need) {
                                                ok = false;
                                                std::printf("(%d%d|%d%d) rs=%d K=%dx%d th=%d force=%d: %s at %d room %ld need %ld\n",
                                                            la, lb, lc, ld, rs, kab, kcd, threads, force, regs[k].name,
                                                            regs[k].off, room, regs[k].need);
                                            }
                                        }
                                        if (!ok) ++bad;
                                    }
                }
    std::printf("layouts %ld violations %ld unfit %ld\n", n, bad, nofit);
    return bad ? 1 : 0;
}
