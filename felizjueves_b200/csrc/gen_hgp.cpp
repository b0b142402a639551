// gen_hgp.cpp -- build-time generator of the compiled HGP class bodies.
//
// For every class (la lb | lc ld) of the Fock build (la <= lb, lc <= ld,
// (la, lb) <= (lc, ld), each l <= 3) whose programs are small enough to run
// from registers, it writes one specialisation of
//   template <int LA, int LB, int LC, int LD> struct HgpCode
// into the header given on the command line:
//   vrr(F, k, acc)      the VRR program of hgp_tables.cpp (the same nodes,
//                       the same level order), straight-line, each node one
//                       expression over named registers; the boundary
//                       targets are added into acc[].
//   coef_bra/coef_ket   the binomial HRR coefficients from AB / CD powers.
//   hrr(acc, cb, ck, eri)  the two binomial transforms, straight-line.
// The kernel that uses them (fock_compiled.cuh) is hand-written; this file
// only spells the recurrence programs the interpreter kernel also runs, so
// both paths compute the same recurrences.
#include <cstdio>
#include <fstream>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "hgp_tables.h"

using namespace fjb;

namespace {

// Programs above these sizes stay on the interpreter kernel: their straight
// line would outgrow the register file and the instruction cache.
// (Measured with ptxas -v on sm_100a: up to ~500 nodes the FP64 bodies fit
// the 255-register file with at most a few KiB of spill; from ~650 nodes
// ptxas falls back to a 32-register allocation with 20-60 KiB of stack.)
// The FP32 bodies (the routed path's recurrence type) hold twice as many
// values in the same registers, so they are generated up to twice the size;
// their FP64 twins only up to kMaxVrrNodes64.
constexpr int kMaxVrrNodes64 = 500;
constexpr int kMaxVrrNodes = 1100;
constexpr int kMaxHrrTerms = 6000;

std::string n(int i) { return "n" + std::to_string(i); }

void emit_class(std::ostream &o, const ClassHost &c) {
    const int Lb = c.la + c.lb, Lk = c.lc + c.ld;
    o << "template <> struct HgpCode<" << c.la << ", " << c.lb << ", " << c.lc << ", " << c.ld
      << "> {\n";
    o << "    static constexpr bool kCompiled = true;\n";
    o << "    static constexpr int kL = " << c.L << ", kNB = " << c.nbe * c.nbf << ", kNBF = " << c.nbf
      << ", kNAB = " << c.nab << ", kNCD = " << c.ncd << ", kNCB = " << c.cb.size()
      << ", kNCK = " << c.ck.size() << ";\n";
    // VRR
    o << "    template <typename R>\n    static __device__ __forceinline__ void vrr(const R *__restrict__ F, "
         "const VrrK<R> &k, R *__restrict__ acc) {\n";
    // leaves
    std::set<int> defined;
    for (int m = 0; m <= c.L; ++m)
        if (c.leaf[m] >= 2) {
            o << "        const R " << n(c.leaf[m]) << " = F[" << m << "];\n";
            defined.insert(c.leaf[m]);
        }
    const char *A[2] = {"k.pa", "k.qc"}, *B[2] = {"k.wp", "k.wq"}, *Cc[2] = {"k.cp", "k.cq"},
               *Dd[2] = {"k.rp", "k.rq"};
    for (const VOp &op : c.ops) {
        const int kd = op.kind;
        std::ostringstream e;
        e << A[kd] << "[" << (int)op.d << "] * " << n(op.s0) << " + " << B[kd] << "[" << (int)op.d
          << "] * " << n(op.s1);
        if (op.c2) {
            e << " + " << Cc[kd] << "[" << (int)op.c2 << "] * " << n(op.s2) << " - " << Dd[kd] << "["
              << (int)op.c2 << "] * " << n(op.s3);
        }
        if (op.c4) e << " + k.e[" << (int)op.c4 << "] * " << n(op.s4);
        o << "        const R " << n(op.dst) << " = " << e.str() << ";\n";
        defined.insert(op.dst);
    }
    for (int t = 0; t < c.nbe * c.nbf; ++t) o << "        acc[" << t << "] += " << n(c.tgt[t]) << ";\n";
    o << "    }\n";
    // HRR coefficients
    auto coef_fn = [&](const char *name, const std::vector<HCoef> &cs) {
        o << "    template <typename R>\n    static __device__ __forceinline__ void " << name
          << "(const double *s, R *__restrict__ out) {\n";
        o << "        const double x1 = s[0], y1 = s[1], z1 = s[2];\n";
        o << "        const double x2 = x1 * x1, y2 = y1 * y1, z2 = z1 * z1;\n";
        o << "        const double x3 = x2 * x1, y3 = y2 * y1, z3 = z2 * z1;\n";
        const char *px[4] = {"1.0", "x1", "x2", "x3"}, *py[4] = {"1.0", "y1", "y2", "y3"},
                   *pz[4] = {"1.0", "z1", "z2", "z3"};
        for (size_t i = 0; i < cs.size(); ++i) {
            o << "        out[" << i << "] = (R)(" << cs[i].binom << " * " << px[cs[i].px] << " * "
              << py[cs[i].py] << " * " << pz[cs[i].pz] << ");\n";
        }
        o << "    }\n";
    };
    coef_fn("coef_bra", c.cb);
    coef_fn("coef_ket", c.ck);
    // HRR: X[ab][jf] then eri[ab][cd]
    o << "    template <typename R>\n    static __device__ __forceinline__ void hrr(const R *__restrict__ acc, "
         "const R *__restrict__ cb, const R *__restrict__ ck, R *__restrict__ eri) {\n";
    for (int ab = 0; ab < c.nab; ++ab)
        for (int jf = 0; jf < c.nbf; ++jf) {
            o << "        const R x" << ab << "_" << jf << " = ";
            for (int t = c.bra_off[ab]; t < c.bra_off[ab + 1]; ++t) {
                if (t > c.bra_off[ab]) o << " + ";
                o << "cb[" << c.bra_terms[t].cidx << "] * acc[" << c.bra_terms[t].src * c.nbf + jf << "]";
            }
            o << ";\n";
        }
    for (int ab = 0; ab < c.nab; ++ab)
        for (int cd = 0; cd < c.ncd; ++cd) {
            o << "        eri[" << ab * c.ncd + cd << "] = ";
            for (int t = c.ket_off[cd]; t < c.ket_off[cd + 1]; ++t) {
                if (t > c.ket_off[cd]) o << " + ";
                o << "ck[" << c.ket_terms[t].cidx << "] * x" << ab << "_" << c.ket_terms[t].src;
            }
            o << ";\n";
        }
    o << "    }\n};\n\n";
    (void)Lb;
    (void)Lk;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: gen_hgp OUT.cuh [--list]\n");
        return 2;
    }
    std::ofstream o(argv[1]);
    o << "// Generated by gen_hgp.cpp from hgp_tables.cpp's programs; do not edit.\n#pragma once\n\n"
      << "namespace fjb {\n\n";
    std::vector<std::string> names;
    std::vector<int> has64;
    for (int la = 0; la <= kMaxL; ++la)
        for (int lb = la; lb <= kMaxL; ++lb)
            for (int lc = 0; lc <= kMaxL; ++lc)
                for (int ld = lc; ld <= kMaxL; ++ld) {
                    if (std::make_pair(la, lb) > std::make_pair(lc, ld)) continue;
                    ClassHost c = build_class(la, lb, lc, ld);
                    const int hrr = c.hrr_terms();
                    if (c.vrr_nodes() > kMaxVrrNodes || hrr > kMaxHrrTerms) continue;
                    emit_class(o, c);
                    names.push_back(std::to_string(la) + std::to_string(lb) + std::to_string(lc) +
                                    std::to_string(ld));
                    has64.push_back(c.vrr_nodes() <= kMaxVrrNodes64);
                }
    // X(la, lb, lc, ld, fp64): every compiled class has an FP32 body; fp64
    // says whether its FP64 twin is instantiated too.
    o << "}  // namespace fjb\n\n#define FJB_COMPILED_CLASSES(X)";
    for (size_t i = 0; i < names.size(); ++i) {
        const auto &s = names[i];
        o << " X(" << s[0] << ", " << s[1] << ", " << s[2] << ", " << s[3] << ", " << has64[i] << ")";
    }
    o << "\n";
    std::printf("%zu compiled classes\n", names.size());
    return 0;
}
