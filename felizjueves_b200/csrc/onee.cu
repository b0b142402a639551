// onee.cu -- the one-electron matrices on sm_100a.
//
// onee_kernel<LA, LB> (LA <= LB): one thread per unordered shell pair of the
// class, the pair stored with its lower-l shell first.  Per primitive pair
// (a outer, b inner, the reference's primitive_pairs order) the thread
// builds the three axes' Hermite tables E^{ij}_t (mmd/hermite.py e_axis,
// seed exp(-mu X_AB^2) per axis) for i <= LA and j <= LB + 2, then
//   S_ab += c_a c_b (pi/p)^{3/2} E^x_0 E^y_0 E^z_0          (overlap.py:55-66)
//   T_ab += c_a c_b (pi/p)^{3/2} (K_x S_y S_z + S_x K_y S_z + S_x S_y K_z),
//           K_ij = -2 b^2 S_{i,j+2} + b (2j+1) S_ij - j(j-1)/2 S_{i,j-2}
//                                                             (kinetic.py:61-111)
//   V_ab += -Z_C c_a c_b (2 pi / p) sum_tuv E^x_t E^y_u E^z_v R_tuv(p, P - C)
//           per nucleus, R from (-2p)^n F_n(p |PC|^2) by
//           R^n_{t+1,u,v} = X_PC R^{n+1}_{tuv} + t R^{n+1}_{t-1,u,v} (and u, v)
//                                                             (potential.py:1-60)
// Every index is a template constant once the loops unroll, so the tables
// live in registers (the largest classes spill).  The block is written to
// (A, B) and mirrored to (B, A); a diagonal pair writes its upper triangle
// and the mirror only (one_electron.py:90-110), so each matrix is exactly
// symmetric and every element has one writer: no atomics, no zeroing.
// Roofline: FP64 pipe; the work is O(n_shell^2 x K^2 x n_nuclei), small
// beside the O(n^4) G build it feeds.
#include "onee.h"

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "fock_compiled.cuh"

namespace fjb {

namespace {

struct OShell {
    double c[3];
    int32_t l, p0, np, ao;
};
static_assert(sizeof(OShell) == 40, "OShell is 40 bytes");

template <typename T>
struct Buf {
    T *p = nullptr;
    size_t n = 0;
    Buf() = default;
    Buf(const Buf &) = delete;
    Buf &operator=(const Buf &) = delete;
    ~Buf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t k) {
        if (k == n && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        if (k == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, k * sizeof(T));
        if (e == cudaSuccess) n = k;
        return e;
    }
    cudaError_t upload(const std::vector<T> &v) {
        cudaError_t e = alloc(v.size());
        if (e != cudaSuccess || v.empty()) return e;
        return cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    }
};

// Component d of the idx-th entry of cartesians(l) (i descending, then j):
// idx = (l - i)(l - i + 1)/2 + (l - i - j).
__host__ __device__ constexpr int cart_of(int l, int idx, int d) {
    int m = 0;  // m = l - i: entries with a given i form a run of m + 1
    while ((m + 1) * (m + 2) / 2 <= idx) ++m;
    const int i = l - m, j = m - (idx - m * (m + 1) / 2);
    return d == 0 ? i : (d == 1 ? j : l - i - j);
}

constexpr int kClasses = (kMaxL + 1) * (kMaxL + 2) / 2;  // (la <= lb) classes
__host__ __device__ constexpr int cls_index(int la, int lb) { return la * (2 * kMaxL + 3 - la) / 2 + (lb - la); }

template <int LA, int LB>
__global__ void __launch_bounds__(128)
    onee_kernel(const OShell *__restrict__ sh, const double *__restrict__ ex, const double *__restrict__ co,
                const int2 *__restrict__ pairs, int n, const double4 *__restrict__ nuc, int n_nuc, int n_ao,
                double *S, double *T, double *V, double *H, const double *__restrict__ boys) {
    constexpr int NA = cnc(LA), NB = cnc(LB), L = LA + LB;
    constexpr int JB = LB + 3;      // ket columns j = 0 .. LB + 2 (the kinetic shift)
    constexpr int TT = LA + LB + 3; // Hermite t = 0 .. LA + LB + 2
    constexpr double kPi = 3.141592653589793;
    // The component loops unroll for the classes whose blocks fit registers;
    // the larger ones loop at run time over tables in local memory (a full
    // unroll of (ff) takes ptxas minutes and spills all the same).
    constexpr bool kUnrolled = NA * NB < 30;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int2 pr = pairs[k];
    const OShell A = sh[pr.x], B = sh[pr.y];
    double s[NA * NB], t[NA * NB], v[NA * NB];
#pragma unroll
    for (int q = 0; q < NA * NB; ++q) s[q] = t[q] = v[q] = 0.0;
    for (int ia = 0; ia < A.np; ++ia) {
        const double a = ex[A.p0 + ia], ca = co[A.p0 + ia];
        for (int ib = 0; ib < B.np; ++ib) {
            const double b = ex[B.p0 + ib], cb = co[B.p0 + ib];
            const double p = a + b, ip = 1.0 / p, h = 0.5 * ip, mu = a * b * ip;
            double E[3][LA + 1][JB][TT];
            double P[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double ab = A.c[d] - B.c[d];
                P[d] = (a * A.c[d] + b * B.c[d]) * ip;
                const double pa = P[d] - A.c[d], pb = P[d] - B.c[d];
#pragma unroll
                for (int i = 0; i <= LA; ++i)
#pragma unroll
                    for (int j = 0; j < JB; ++j)
#pragma unroll
                        for (int u = 0; u < TT; ++u) E[d][i][j][u] = 0.0;
                E[d][0][0][0] = exp(-mu * ab * ab);
#pragma unroll
                for (int j = 0; j + 1 < JB; ++j)
#pragma unroll
                    for (int u = 0; u <= j + 1; ++u) {
                        double x = pb * E[d][0][j][u];
                        if (u >= 1) x += h * E[d][0][j][u >= 1 ? u - 1 : 0];
                        if (u + 1 <= j) x += (double)(u + 1) * E[d][0][j][u + 1 < TT ? u + 1 : 0];
                        E[d][0][j + 1][u] = x;
                    }
#pragma unroll
                for (int i = 0; i < LA; ++i)
#pragma unroll
                    for (int j = 0; j < JB; ++j)
#pragma unroll
                        for (int u = 0; u <= i + j + 1; ++u) {
                            double x = pa * E[d][i][j][u];
                            if (u >= 1) x += h * E[d][i][j][u >= 1 ? u - 1 : 0];
                            if (u + 1 <= i + j) x += (double)(u + 1) * E[d][i][j][u + 1 < TT ? u + 1 : 0];
                            E[d][i + 1][j][u] = x;
                        }
            }
            // overlap and kinetic energy of component pair (r, c)
            const double dress = ca * cb * ip * sqrt(ip) * (kPi * 1.7724538509055159);  // (pi/p)^{3/2}
            auto st_comp = [&](int r, int c) {
                const int ax = cart_of(LA, r, 0), ay = cart_of(LA, r, 1), az = cart_of(LA, r, 2);
                const int bx = cart_of(LB, c, 0), by = cart_of(LB, c, 1), bz = cart_of(LB, c, 2);
                const double sx = E[0][ax][bx][0], sy = E[1][ay][by][0], sz = E[2][az][bz][0];
                double kx = -2.0 * b * b * E[0][ax][bx + 2][0] + b * (double)(2 * bx + 1) * sx;
                double ky = -2.0 * b * b * E[1][ay][by + 2][0] + b * (double)(2 * by + 1) * sy;
                double kz = -2.0 * b * b * E[2][az][bz + 2][0] + b * (double)(2 * bz + 1) * sz;
                if (bx >= 2) kx -= 0.5 * (double)(bx * (bx - 1)) * E[0][ax][bx >= 2 ? bx - 2 : 0][0];
                if (by >= 2) ky -= 0.5 * (double)(by * (by - 1)) * E[1][ay][by >= 2 ? by - 2 : 0][0];
                if (bz >= 2) kz -= 0.5 * (double)(bz * (bz - 1)) * E[2][az][bz >= 2 ? bz - 2 : 0][0];
                s[r * NB + c] += dress * (sx * sy * sz);
                t[r * NB + c] += dress * (kx * sy * sz + sx * ky * sz + sx * sy * kz);
            };
            if constexpr (kUnrolled) {
#pragma unroll
                for (int r = 0; r < NA; ++r)
#pragma unroll
                    for (int c = 0; c < NB; ++c) st_comp(r, c);
            } else {
#pragma unroll 1
                for (int r = 0; r < NA; ++r)
#pragma unroll 1
                    for (int c = 0; c < NB; ++c) st_comp(r, c);
            }
            // nuclear attraction
            const double pref = ca * cb * 2.0 * kPi * ip;
            for (int q = 0; q < n_nuc; ++q) {
                const double4 C = nuc[q];
                const double pc[3] = {P[0] - C.x, P[1] - C.y, P[2] - C.z};
                const double x = p * (pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2]);
                double F[L + 1];
                boys_t<L>(x, F, boys);
                double Rp[L + 1][L + 1][L + 1], Rc[L + 1][L + 1][L + 1];
                double pws[L + 1];  // (-2p)^m
                pws[0] = 1.0;
#pragma unroll
                for (int m = 1; m <= L; ++m) pws[m] = pws[m - 1] * (-2.0 * p);
#pragma unroll
                for (int m = L; m >= 0; --m) {
#pragma unroll
                    for (int sum = 0; sum <= L - m; ++sum)
#pragma unroll
                        for (int ti = sum; ti >= 0; --ti)
#pragma unroll
                            for (int ui = sum - ti; ui >= 0; --ui) {
                                const int vi = sum - ti - ui;
                                double r;
                                if (sum == 0) {
                                    r = pws[m] * F[m];
                                } else if (ti > 0) {
                                    r = pc[0] * Rp[ti - 1][ui][vi];
                                    if (ti > 1) r += (double)(ti - 1) * Rp[ti > 1 ? ti - 2 : 0][ui][vi];
                                } else if (ui > 0) {
                                    r = pc[1] * Rp[ti][ui - 1][vi];
                                    if (ui > 1) r += (double)(ui - 1) * Rp[ti][ui > 1 ? ui - 2 : 0][vi];
                                } else {
                                    r = pc[2] * Rp[ti][ui][vi - 1];
                                    if (vi > 1) r += (double)(vi - 1) * Rp[ti][ui][vi > 1 ? vi - 2 : 0];
                                }
                                Rc[ti][ui][vi] = r;
                            }
#pragma unroll
                    for (int sum = 0; sum <= L - m; ++sum)
#pragma unroll
                        for (int ti = sum; ti >= 0; --ti)
#pragma unroll
                            for (int ui = sum - ti; ui >= 0; --ui) Rp[ti][ui][sum - ti - ui] = Rc[ti][ui][sum - ti - ui];
                }
                const double w = -C.w * pref;
                auto v_comp = [&](int r, int c) {
                    const int ax = cart_of(LA, r, 0), ay = cart_of(LA, r, 1), az = cart_of(LA, r, 2);
                    const int bx = cart_of(LB, c, 0), by = cart_of(LB, c, 1), bz = cart_of(LB, c, 2);
                    double acc = 0.0;
                    for (int ti = 0; ti <= ax + bx; ++ti)
                        for (int ui = 0; ui <= ay + by; ++ui) {
                            const double exy = E[0][ax][bx][ti] * E[1][ay][by][ui];
                            for (int vi = 0; vi <= az + bz; ++vi) acc += exy * E[2][az][bz][vi] * Rp[ti][ui][vi];
                        }
                    v[r * NB + c] += w * acc;
                };
                if constexpr (kUnrolled) {
#pragma unroll
                    for (int r = 0; r < NA; ++r)
#pragma unroll
                        for (int c = 0; c < NB; ++c) v_comp(r, c);
                } else {
#pragma unroll 1
                    for (int r = 0; r < NA; ++r)
#pragma unroll 1
                        for (int c = 0; c < NB; ++c) v_comp(r, c);
                }
            }
        }
    }
    const bool diag = pr.x == pr.y;
#pragma unroll
    for (int r = 0; r < NA; ++r)
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            if (diag && c < r) continue;
            const size_t e1 = (size_t)(A.ao + r) * n_ao + B.ao + c, e2 = (size_t)(B.ao + c) * n_ao + A.ao + r;
            const int q = r * NB + c;
            if (S) S[e1] = S[e2] = s[q];
            if (T) T[e1] = T[e2] = t[q];
            if (V) V[e1] = V[e2] = v[q];
            if (H) H[e1] = H[e2] = t[q] + v[q];
        }
}

struct ClassFn {
    int la, lb;
    void (*fn)(const OShell *, const double *, const double *, const int2 *, int, const double4 *, int, int,
               double *, double *, double *, double *, const double *);
};

#define FJB_ONEE(a, b) {a, b, onee_kernel<a, b>}
const ClassFn kFns[] = {FJB_ONEE(0, 0), FJB_ONEE(0, 1), FJB_ONEE(0, 2), FJB_ONEE(0, 3), FJB_ONEE(1, 1),
                        FJB_ONEE(1, 2), FJB_ONEE(1, 3), FJB_ONEE(2, 2), FJB_ONEE(2, 3), FJB_ONEE(3, 3)};
#undef FJB_ONEE
static_assert(sizeof(kFns) / sizeof(kFns[0]) == kClasses, "one kernel per (la <= lb) class");

}  // namespace

struct OneElectron {
    int n_ao = 0;
    Buf<OShell> shells;
    Buf<double> ex, co;
    Buf<int2> pairs;
    Buf<double4> nuc;
    std::vector<int> cls_off;  // [kClasses + 1] into pairs
};

OneElectron *onee_create(const HostBasis &basis, int device, std::string *err) {
    auto e = std::make_unique<OneElectron>();
    e->n_ao = basis.n_ao;
    std::vector<OShell> sh;
    std::vector<double> ex, co;
    const int ns = (int)basis.shells.size();
    for (int i = 0; i < ns; ++i) {
        const HostShell &s = basis.shells[i];
        if (s.l < 0 || s.l > kMaxL) {
            *err = "l above the compiled maximum";
            return nullptr;
        }
        sh.push_back(OShell{{s.centre[0], s.centre[1], s.centre[2]}, s.l, (int32_t)ex.size(),
                            (int32_t)s.exps.size(), basis.offsets[i]});
        ex.insert(ex.end(), s.exps.begin(), s.exps.end());
        co.insert(co.end(), s.coefs.begin(), s.coefs.end());
    }
    std::vector<std::vector<int2>> by(kClasses);
    for (int i = 0; i < ns; ++i)
        for (int j = i; j < ns; ++j) {
            const int li = basis.shells[i].l, lj = basis.shells[j].l;
            const int2 pr = li <= lj ? make_int2(i, j) : make_int2(j, i);
            by[cls_index(std::min(li, lj), std::max(li, lj))].push_back(pr);
        }
    std::vector<int2> pairs;
    e->cls_off.assign(kClasses + 1, 0);
    for (int c = 0; c < kClasses; ++c) {
        e->cls_off[c] = (int)pairs.size();
        pairs.insert(pairs.end(), by[c].begin(), by[c].end());
    }
    e->cls_off[kClasses] = (int)pairs.size();
    if (cudaSetDevice(device) != cudaSuccess) {
        *err = "cudaSetDevice failed";
        return nullptr;
    }
    cudaError_t ce = e->shells.upload(sh);
    if (ce == cudaSuccess) ce = e->ex.upload(ex);
    if (ce == cudaSuccess) ce = e->co.upload(co);
    if (ce == cudaSuccess) ce = e->pairs.upload(pairs);
    if (ce != cudaSuccess) {
        *err = std::string("one-electron setup: ") + cudaGetErrorString(ce);
        return nullptr;
    }
    return e.release();
}

void onee_destroy(OneElectron *e) { delete e; }

int onee_build(OneElectron *e, const double *charges, const double *coords, int n_nuc, double *S, double *T,
               double *V, double *H, const double *boys_tab, cudaStream_t st, std::string *err, int *launches) {
    std::vector<double4> nuc(n_nuc);
    for (int q = 0; q < n_nuc; ++q)
        nuc[q] = make_double4(coords[3 * q], coords[3 * q + 1], coords[3 * q + 2], charges[q]);
    // ordered on the build's stream: a later call with other nuclei cannot
    // overwrite them under this call's kernels (pageable source: the call
    // returns once the bytes are staged)
    cudaError_t ce = cudaSuccess;
    if (n_nuc > 0) ce = e->nuc.alloc(nuc.size());
    if (ce == cudaSuccess && n_nuc > 0)
        ce = cudaMemcpyAsync(e->nuc.p, nuc.data(), nuc.size() * sizeof(double4), cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) {
        *err = std::string("one-electron nuclei: ") + cudaGetErrorString(ce);
        return 1;
    }
    int nl = 0;
    for (int c = 0; c < kClasses; ++c) {
        const int n = e->cls_off[c + 1] - e->cls_off[c];
        if (n == 0) continue;
        kFns[c].fn<<<(n + 127) / 128, 128, 0, st>>>(e->shells.p, e->ex.p, e->co.p, e->pairs.p + e->cls_off[c], n,
                                                   e->nuc.p, n_nuc, e->n_ao, S, T, V, H, boys_tab);
        ++nl;
    }
    ce = cudaGetLastError();
    if (ce != cudaSuccess) {
        *err = std::string("one-electron launch: ") + cudaGetErrorString(ce);
        return 1;
    }
    *launches = nl;
    return 0;
}

}  // namespace fjb
