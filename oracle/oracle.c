/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY.  A plain-C, FP64 restatement of the
 * reference's host ERI path and its J/K/G sweeps, used as the checker for the
 * CUDA path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it; nothing in the product links it.
 *
 * What it restates (paths relative to the reference's src/felizjueves/):
 *   or_boys          reference/boys.py:133-218  F_m(T): 112-node Gauss-Legendre
 *                    on [0,1] below T_SWITCH = 125, the large-T asymptote above.
 *   e_axis/e_block   mmd/hermite.py:61-117      pure Hermite E, raised along
 *                    a then b; 3D block over hermite_order(|a|+|b|).
 *   dress            ao/pairs.py:238-247        c_a c_b (pi/zeta)^{3/2} E.
 *   r_table          reference/pq.py:50-124     [r]^(m), each node reduced
 *                    along its first nonzero axis; fundamental with
 *                    theta^2 = zeta eta/(zeta+eta).
 *   or_eri_block     eri/eri.py:86-145          (ab|cd) = sum_prims
 *                    E_bra [p|q] E_ket^T, [p|q] = (-1)^|q| [p+q]^(0); and its
 *                    absolute-value twin `scale`.
 *   or_jk_ordered    eri/fock/fock.py:126-163   every ordered shell quartet,
 *                    weight 1: J[a_i][b_j] += D[c_k][d_l] x,
 *                    K[a_i][c_k] += D[b_j][d_l] x.
 *   or_jk_unique     eri/fock/kernel_f.py:94-131,478-486,621-628  one
 *                    quartet per 8-fold orbit, degeneracy 1/|Stab|, the
 *                    six in-order blocks (Coulomb weight 2, exchange 1 here,
 *                    applied to J and K separately) and the closing
 *                    F <- F + F^T.  Used for systems where the ordered sweep
 *                    is too slow; the two are tested equal.
 *
 * Parity pins: tests/test_oracle.py holds this file to the reference's own
 * outputs recorded in tests/golden/ (Boys grid, sampled ERI blocks, J and K on
 * small nested systems) and to the libcint vj/vk fixtures the reference
 * tracks.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_NODES 112
#define OR_M_MAX 40
#define OR_T_SWITCH 125.0
#define OR_T_MAX 1.0e6
#define OR_LMAX 6           /* per shell */
#define OR_LT (4 * OR_LMAX) /* quartet total */

static double gl_t[OR_NODES], gl_w[OR_NODES];
static int gl_ready = 0;

/* Gauss-Legendre on [0,1]: nodes by Newton on P_n from the usual cosine
 * guesses, weights 2/((1-x^2) P_n'(x)^2), in long double. */
static void gl_init(void) {
    if (gl_ready) return;
    const int n = OR_NODES;
    for (int i = 0; i < n; ++i) {
        long double x = cosl(3.14159265358979323846264338327950288L *
                             ((long double)i + 0.75L) / ((long double)n + 0.5L));
        long double p1 = 0, dp = 0;
        for (int it = 0; it < 100; ++it) {
            long double p0 = 1.0L;
            p1 = x;
            for (int k = 2; k <= n; ++k) {
                long double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            /* p1 = P_n, p0 = P_{n-1} */
            dp = n * (x * p1 - p0) / (x * x - 1.0L);
            long double dx = p1 / dp;
            x -= dx;
            if (fabsl(dx) < 1e-21L) break;
        }
        long double p0 = 1.0L;
        p1 = x;
        for (int k = 2; k <= n; ++k) {
            long double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (x * p1 - p0) / (x * x - 1.0L);
        long double w = 2.0L / ((1.0L - x * x) * dp * dp);
        gl_t[i] = (double)(0.5L * (x + 1.0L));
        gl_w[i] = (double)(0.5L * w);
    }
    gl_ready = 1;
}

static double asymptote(int m, double T) {
    double a = 0.5 * sqrt(M_PI / T);
    for (int k = 1; k <= m; ++k) a *= (2 * k - 1) / (2.0 * T);
    return a;
}

/* F_m(T) for m in 0..mmax into F (reference/boys.py:184-218). Returns 0, or
 * -1 outside the reference's measured domain. */
static int boys_all(int mmax, double T, double *F) {
    if (mmax < 0 || mmax > OR_M_MAX || !(T >= 0.0 && T <= OR_T_MAX)) return -1;
    if (T >= OR_T_SWITCH) {
        for (int m = 0; m <= mmax; ++m) F[m] = asymptote(m, T);
        return 0;
    }
    double acc[OR_M_MAX + 1];
    for (int m = 0; m <= mmax; ++m) acc[m] = 0.0;
    for (int i = 0; i < OR_NODES; ++i) {
        double t = gl_t[i], t2 = t * t;
        double v = gl_w[i] * exp(-t2 * T);
        for (int m = 0; m <= mmax; ++m) {
            acc[m] += v;
            v *= t2;
        }
    }
    for (int m = 0; m <= mmax; ++m) F[m] = acc[m];
    return 0;
}

double or_boys(int m, double T) {
    gl_init();
    double F[OR_M_MAX + 1];
    if (boys_all(m, T, F) != 0) return NAN;
    return F[m];
}

/* ---- basis ---------------------------------------------------------------- */

typedef struct {
    int n_sh;
    const int *l;
    const double *centre; /* n_sh x 3 */
    const int *prim0;
    const int *nprim;
    const double *exps;
    const double *coefs;
    const int *ao_off;
    int n_ao;
} or_basis;

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }
static int nherm(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }

static void cart_list(int l, int out[][3]) {
    int k = 0;
    for (int i = l; i >= 0; --i)
        for (int j = l - i; j >= 0; --j) {
            out[k][0] = i;
            out[k][1] = j;
            out[k][2] = l - i - j;
            ++k;
        }
}

static void herm_list(int L, int out[][3]) {
    int k = 0;
    for (int n = 0; n <= L; ++n)
        for (int tx = n; tx >= 0; --tx)
            for (int ty = n - tx; ty >= 0; --ty) {
                out[k][0] = tx;
                out[k][1] = ty;
                out[k][2] = n - tx - ty;
                ++k;
            }
}

/* e_axis(i, j, zeta, pa, pb) -> e[0..i+j] (mmd/hermite.py:61-79). */
static void e_axis(int i, int j, double zeta, double pa, double pb, double *e) {
    double prev[2 * OR_LMAX + 2], out[2 * OR_LMAX + 2];
    int n = 1;
    prev[0] = exp(zeta * pa * pb);
    double h = 0.5 / zeta;
    for (int s = 0; s < i + j; ++s) {
        double x = s < i ? pa : pb;
        for (int t = 0; t <= n; ++t) {
            double v = 0.0;
            if (t >= 1) v += h * prev[t - 1];
            if (t < n) v += x * prev[t];
            if (t + 1 < n) v += (t + 1) * prev[t + 1];
            out[t] = v;
        }
        ++n;
        memcpy(prev, out, sizeof(double) * n);
    }
    memcpy(e, prev, sizeof(double) * n);
}

/* One ordered primitive pair: P, zeta and the dressed E block
 * [ncart(la)*ncart(lb)][nherm(la+lb)], rows a outer (ao/pairs.py:221-254). */
typedef struct {
    double P[3], zeta;
    double *E; /* owned */
} prim_pair;

typedef struct {
    int a, b, la, lb, n_ab, nh, K;
    prim_pair *pp;
} shell_pair;

static void make_pair(const or_basis *B, int a, int b, shell_pair *sp) {
    int la = B->l[a], lb = B->l[b];
    const double *A = B->centre + 3 * a, *Bc = B->centre + 3 * b;
    int ca[28][3], cb[28][3], h[455][3];
    cart_list(la, ca);
    cart_list(lb, cb);
    int L = la + lb, nh = nherm(L);
    herm_list(L, h);
    sp->a = a;
    sp->b = b;
    sp->la = la;
    sp->lb = lb;
    sp->n_ab = ncart(la) * ncart(lb);
    sp->nh = nh;
    sp->K = B->nprim[a] * B->nprim[b];
    sp->pp = (prim_pair *)calloc((size_t)sp->K, sizeof(prim_pair));
    int k = 0;
    for (int i = 0; i < B->nprim[a]; ++i)
        for (int j = 0; j < B->nprim[b]; ++j, ++k) {
            double al = B->exps[B->prim0[a] + i], be = B->exps[B->prim0[b] + j];
            double cfa = B->coefs[B->prim0[a] + i], cfb = B->coefs[B->prim0[b] + j];
            double zeta = al + be;
            prim_pair *p = &sp->pp[k];
            for (int d = 0; d < 3; ++d) p->P[d] = (al * A[d] + be * Bc[d]) / zeta;
            p->zeta = zeta;
            p->E = (double *)malloc(sizeof(double) * (size_t)sp->n_ab * nh);
            double scale = cfa * cfb * pow(M_PI / zeta, 1.5);
            int row = 0;
            for (int u = 0; u < ncart(la); ++u)
                for (int v = 0; v < ncart(lb); ++v, ++row) {
                    double ax[3][2 * OR_LMAX + 2];
                    int len[3];
                    for (int d = 0; d < 3; ++d) {
                        e_axis(ca[u][d], cb[v][d], zeta, p->P[d] - A[d],
                               p->P[d] - Bc[d], ax[d]);
                        len[d] = ca[u][d] + cb[v][d] + 1;
                    }
                    for (int t = 0; t < nh; ++t) {
                        double val = 1.0;
                        for (int d = 0; d < 3; ++d)
                            val = h[t][d] < len[d] ? val * ax[d][h[t][d]] : 0.0;
                        p->E[(size_t)row * nh + t] = scale * val;
                    }
                }
        }
}

static void free_pair(shell_pair *sp) {
    for (int k = 0; k < sp->K; ++k) free(sp->pp[k].E);
    free(sp->pp);
}

/* [r]^(m) for |r| <= L at one (PQ, theta) (reference/pq.py:50-124). R is
 * indexed [m][rx][ry][rz] with stride (L+1). */
#define RIDX(m, x, y, z, S) ((((m) * (S) + (x)) * (S) + (y)) * (S) + (z))
static void r_table(int L, const double PQ[3], double theta, double *R) {
    const int S = L + 1;
    double t2 = theta * theta;
    double T = t2 * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
    double F[OR_LT + 1];
    boys_all(L, T, F);
    const double two_over_sqrt_pi = 2.0 / sqrt(M_PI);
    for (int m = 0; m <= L; ++m)
        R[RIDX(m, 0, 0, 0, S)] = two_over_sqrt_pi * theta * pow(-2.0 * t2, (double)m) * F[m];
    for (int n = 1; n <= L; ++n)
        for (int x = n; x >= 0; --x)
            for (int y = n - x; y >= 0; --y) {
                int z = n - x - y, r[3] = {x, y, z};
                int d = r[0] ? 0 : (r[1] ? 1 : 2);
                for (int m = 0; m <= L - n; ++m) {
                    int r1[3] = {x, y, z}, r2[3] = {x, y, z};
                    r1[d] -= 1;
                    r2[d] -= 2;
                    double v = PQ[d] * R[RIDX(m + 1, r1[0], r1[1], r1[2], S)];
                    if (r[d] >= 2) v += (r[d] - 1) * R[RIDX(m + 1, r2[0], r2[1], r2[2], S)];
                    R[RIDX(m, x, y, z, S)] = v;
                }
            }
}

/* (ab|cd) for two prepared ordered pairs into blk[n_ab][n_cd] (+ scale). */
static void eri_pairs(const shell_pair *bra, const shell_pair *ket, double *blk,
                      double *scl) {
    int Lb = bra->la + bra->lb, Lk = ket->la + ket->lb, L = Lb + Lk, S = L + 1;
    int hp[455][3], hq[455][3];
    herm_list(Lb, hp);
    herm_list(Lk, hq);
    int np_ = bra->nh, nq = ket->nh, nab = bra->n_ab, ncd = ket->n_ab;
    double *R = (double *)malloc(sizeof(double) * (size_t)S * S * S * S);
    double *M = (double *)malloc(sizeof(double) * (size_t)np_ * nq);
    double *X = (double *)malloc(sizeof(double) * (size_t)np_ * ncd);
    double *AM = scl ? (double *)malloc(sizeof(double) * (size_t)np_ * nq) : NULL;
    double *AX = scl ? (double *)malloc(sizeof(double) * (size_t)np_ * ncd) : NULL;
    memset(blk, 0, sizeof(double) * (size_t)nab * ncd);
    if (scl) memset(scl, 0, sizeof(double) * (size_t)nab * ncd);
    for (int kb = 0; kb < bra->K; ++kb)
        for (int kk = 0; kk < ket->K; ++kk) {
            const prim_pair *P = &bra->pp[kb], *Q = &ket->pp[kk];
            double zeta = P->zeta, eta = Q->zeta;
            double theta = sqrt(zeta * eta / (zeta + eta));
            double PQ[3] = {P->P[0] - Q->P[0], P->P[1] - Q->P[1], P->P[2] - Q->P[2]};
            r_table(L, PQ, theta, R);
            for (int p = 0; p < np_; ++p)
                for (int q = 0; q < nq; ++q) {
                    int s = (hq[q][0] + hq[q][1] + hq[q][2]) & 1;
                    double v = R[RIDX(0, hp[p][0] + hq[q][0], hp[p][1] + hq[q][1],
                                      hp[p][2] + hq[q][2], S)];
                    M[p * nq + q] = s ? -v : v;
                    if (AM) AM[p * nq + q] = fabs(v);
                }
            /* X = M E_ket^T : [np][ncd] */
            for (int p = 0; p < np_; ++p)
                for (int c = 0; c < ncd; ++c) {
                    double acc = 0.0, aacc = 0.0;
                    const double *er = Q->E + (size_t)c * nq;
                    for (int q = 0; q < nq; ++q) {
                        acc += M[p * nq + q] * er[q];
                        if (AM) aacc += AM[p * nq + q] * fabs(er[q]);
                    }
                    X[p * ncd + c] = acc;
                    if (AX) AX[p * ncd + c] = aacc;
                }
            for (int r = 0; r < nab; ++r) {
                const double *eb = P->E + (size_t)r * np_;
                for (int c = 0; c < ncd; ++c) {
                    double acc = 0.0, aacc = 0.0;
                    for (int p = 0; p < np_; ++p) {
                        acc += eb[p] * X[p * ncd + c];
                        if (AX) aacc += fabs(eb[p]) * AX[p * ncd + c];
                    }
                    blk[r * ncd + c] += acc;
                    if (scl) scl[r * ncd + c] += aacc;
                }
            }
        }
    free(R);
    free(M);
    free(X);
    free(AM);
    free(AX);
}

static int check_basis(const or_basis *B) {
    if (!B || B->n_sh <= 0) return -1;
    for (int i = 0; i < B->n_sh; ++i)
        if (B->l[i] < 0 || B->l[i] > OR_LMAX || B->nprim[i] < 1) return -2;
    return 0;
}

int or_eri_block(const or_basis *B, int a, int b, int c, int d, double *out,
                 double *scale) {
    gl_init();
    if (check_basis(B)) return -1;
    shell_pair bra, ket;
    make_pair(B, a, b, &bra);
    make_pair(B, c, d, &ket);
    eri_pairs(&bra, &ket, out, scale);
    free_pair(&bra);
    free_pair(&ket);
    return 0;
}

static shell_pair *all_pairs(const or_basis *B) {
    int n = B->n_sh;
    shell_pair *sp = (shell_pair *)calloc((size_t)n * n, sizeof(shell_pair));
#pragma omp parallel for schedule(dynamic)
    for (int ab = 0; ab < n * n; ++ab) make_pair(B, ab / n, ab % n, &sp[ab]);
    return sp;
}

static void free_all(const or_basis *B, shell_pair *sp) {
    for (int i = 0; i < B->n_sh * B->n_sh; ++i) free_pair(&sp[i]);
    free(sp);
}

/* Every ordered quartet, weight 1 (eri/fock/fock.py:126-163). Rows of J and K
 * written by one outer shell a belong to that shell, so the a loop runs in
 * parallel without sharing. */
int or_jk_ordered(const or_basis *B, const double *D, double *J, double *K,
                  int nthreads) {
    gl_init();
    if (check_basis(B)) return -1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    int n = B->n_sh, nao = B->n_ao;
    memset(J, 0, sizeof(double) * (size_t)nao * nao);
    memset(K, 0, sizeof(double) * (size_t)nao * nao);
    shell_pair *sp = all_pairs(B);
#pragma omp parallel for schedule(dynamic)
    for (int a = 0; a < n; ++a) {
        double *blk = (double *)malloc(sizeof(double) * 28 * 28 * 28 * 28);
        for (int b = 0; b < n; ++b)
            for (int c = 0; c < n; ++c)
                for (int d = 0; d < n; ++d) {
                    const shell_pair *bra = &sp[a * n + b], *ket = &sp[c * n + d];
                    eri_pairs(bra, ket, blk, NULL);
                    int na = ncart(B->l[a]), nb = ncart(B->l[b]), nc = ncart(B->l[c]),
                        nd = ncart(B->l[d]);
                    int oa = B->ao_off[a], ob = B->ao_off[b], oc = B->ao_off[c],
                        od = B->ao_off[d];
                    for (int i = 0; i < na; ++i)
                        for (int j = 0; j < nb; ++j) {
                            const double *row = blk + (size_t)(i * nb + j) * nc * nd;
                            double acc = 0.0;
                            for (int k = 0; k < nc; ++k) {
                                const double *drow = D + (size_t)(oc + k) * nao;
                                for (int l = 0; l < nd; ++l) acc += drow[od + l] * row[k * nd + l];
                            }
                            J[(size_t)(oa + i) * nao + ob + j] += acc;
                            const double *dbj = D + (size_t)(ob + j) * nao;
                            for (int k = 0; k < nc; ++k) {
                                double acc2 = 0.0;
                                for (int l = 0; l < nd; ++l) acc2 += dbj[od + l] * row[k * nd + l];
                                K[(size_t)(oa + i) * nao + oc + k] += acc2;
                            }
                        }
                }
        free(blk);
    }
    free_all(B, sp);
    return 0;
}

/* One quartet per orbit (canonical pairs P = {a<=b} by index, Q >= P),
 * degeneracy (1/2 if a=b)(1/2 if c=d)(1/2 if P=Q), six in-order blocks,
 * closed by M + M^T (eri/fock/kernel_f.py:94-131, 481-486, 621-628). */
int or_jk_unique(const or_basis *B, const double *D, double *J, double *K,
                 int nthreads) {
    gl_init();
    if (check_basis(B)) return -1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    int n = B->n_sh, nao = B->n_ao;
    int npair = n * (n + 1) / 2;
    int *pa = (int *)malloc(sizeof(int) * npair), *pb = (int *)malloc(sizeof(int) * npair);
    for (int a = 0, k = 0; a < n; ++a)
        for (int b = a; b < n; ++b, ++k) {
            pa[k] = a;
            pb[k] = b;
        }
    shell_pair *sp = all_pairs(B);
    size_t nn = (size_t)nao * nao;
    memset(J, 0, sizeof(double) * nn);
    memset(K, 0, sizeof(double) * nn);
#pragma omp parallel
    {
        double *Jp = (double *)calloc(nn, sizeof(double));
        double *Kp = (double *)calloc(nn, sizeof(double));
        double *blk = (double *)malloc(sizeof(double) * 28 * 28 * 28 * 28);
#pragma omp for schedule(dynamic, 4)
        for (int P = 0; P < npair; ++P)
            for (int Q = P; Q < npair; ++Q) {
                int a = pa[P], b = pb[P], c = pa[Q], d = pb[Q];
                double deg = (a == b ? 0.5 : 1.0) * (c == d ? 0.5 : 1.0) * (P == Q ? 0.5 : 1.0);
                eri_pairs(&sp[a * n + b], &sp[c * n + d], blk, NULL);
                int na = ncart(B->l[a]), nb = ncart(B->l[b]), nc = ncart(B->l[c]),
                    nd = ncart(B->l[d]);
                int oa = B->ao_off[a], ob = B->ao_off[b], oc = B->ao_off[c],
                    od = B->ao_off[d];
                for (int i = 0; i < na; ++i)
                    for (int j = 0; j < nb; ++j)
                        for (int k = 0; k < nc; ++k)
                            for (int l = 0; l < nd; ++l) {
                                double x = deg * blk[(size_t)(i * nb + j) * nc * nd + k * nd + l];
#define DD(u, v) D[(size_t)(u) * nao + (v)]
                                Jp[(size_t)(oa + i) * nao + ob + j] += 2.0 * DD(oc + k, od + l) * x;
                                Jp[(size_t)(oc + k) * nao + od + l] += 2.0 * DD(oa + i, ob + j) * x;
                                Kp[(size_t)(oa + i) * nao + oc + k] += DD(ob + j, od + l) * x;
                                Kp[(size_t)(oa + i) * nao + od + l] += DD(ob + j, oc + k) * x;
                                Kp[(size_t)(ob + j) * nao + oc + k] += DD(oa + i, od + l) * x;
                                Kp[(size_t)(ob + j) * nao + od + l] += DD(oa + i, oc + k) * x;
#undef DD
                            }
            }
#pragma omp critical
        {
            for (size_t t = 0; t < nn; ++t) {
                J[t] += Jp[t];
                K[t] += Kp[t];
            }
        }
        free(Jp);
        free(Kp);
        free(blk);
    }
    /* close: M <- M + M^T */
    for (int i = 0; i < nao; ++i)
        for (int j = i; j < nao; ++j) {
            double s = J[(size_t)i * nao + j] + J[(size_t)j * nao + i];
            J[(size_t)i * nao + j] = J[(size_t)j * nao + i] = s;
            s = K[(size_t)i * nao + j] + K[(size_t)j * nao + i];
            K[(size_t)i * nao + j] = K[(size_t)j * nao + i] = s;
        }
    free_all(B, sp);
    free(pa);
    free(pb);
    return 0;
}

/* The reference's per-quartet work of the fused build, timed: for each of n
 * unique quartets (a, b | c, d) given with its degeneracy, the ERI block
 * (eri/eri.py:86-145) and the six-block digest into J and K
 * (eri/fock/kernel_f.py:94-131: Coulomb weight 2 on the ab and cd blocks,
 * exchange 1 on ac, ad, bc, bd).  Pairs are made once per distinct (a, b)
 * of the list, before the timed loop, as a sweep makes them once.  With
 * `kept`, each pair keeps only the plan's primitive pairs (the reference's
 * pruned pair, ao/pairs.py:545): the list of the pair in slot q (the bra of
 * quartet q / 2 when q is even, its ket when odd) is
 * kept[kept_off[q] .. kept_off[q + 1]), indices i * nprim_b + j, in the
 * order they are summed.  The quartets run on nthreads OpenMP threads
 * (dynamic schedule); sec receives each quartet's own wall time on its
 * thread.  J and K come back as the unclosed sums (M, not M + M^T). */
int or_fock_quartets(const or_basis *B, const double *D, int n, const int *quartets,
                     const double *degs, const int *kept_off, const int *kept, double *J,
                     double *K, int nthreads, double *sec) {
    gl_init();
    if (check_basis(B)) return -1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    const int ns = B->n_sh, nao = B->n_ao;
    /* distinct pairs of the list */
    int *slot = (int *)malloc(sizeof(int) * (size_t)ns * ns);
    for (size_t i = 0; i < (size_t)ns * ns; ++i) slot[i] = -1;
    int np = 0;
    for (int q = 0; q < 2 * n; ++q) {
        const int a = quartets[2 * q], b = quartets[2 * q + 1];
        if (slot[a * ns + b] < 0) slot[a * ns + b] = np++;
    }
    shell_pair *sp = (shell_pair *)calloc((size_t)(np ? np : 1), sizeof(shell_pair));
    for (int q = 0; q < 2 * n; ++q) {
        const int a = quartets[2 * q], b = quartets[2 * q + 1];
        shell_pair *p = &sp[slot[a * ns + b]];
        if (p->pp) continue;
        make_pair(B, a, b, p);
        if (kept) {
            /* keep the plan's primitive pairs (index i * nprim_b + j), in order */
            const int k0 = kept_off[q], k1 = kept_off[q + 1];
            prim_pair *sel = (prim_pair *)calloc((size_t)(k1 - k0 ? k1 - k0 : 1), sizeof(prim_pair));
            char *used = (char *)calloc((size_t)p->K, 1);
            for (int k = k0; k < k1; ++k) {
                sel[k - k0] = p->pp[kept[k]];
                used[kept[k]] = 1;
            }
            for (int k = 0; k < p->K; ++k)
                if (!used[k]) free(p->pp[k].E);
            free(used);
            free(p->pp);
            p->pp = sel;
            p->K = k1 - k0;
        }
    }
    size_t nn = (size_t)nao * nao;
    memset(J, 0, sizeof(double) * nn);
    memset(K, 0, sizeof(double) * nn);
#pragma omp parallel
    {
        double *blk = (double *)malloc(sizeof(double) * 28 * 28 * 28 * 28);
#pragma omp for schedule(dynamic, 1)
        for (int q = 0; q < n; ++q) {
            struct timespec t0, t1;
            clock_gettime(CLOCK_MONOTONIC, &t0);
            const int a = quartets[4 * q], b = quartets[4 * q + 1], c = quartets[4 * q + 2],
                      d = quartets[4 * q + 3];
            eri_pairs(&sp[slot[a * ns + b]], &sp[slot[c * ns + d]], blk, NULL);
            const int na = ncart(B->l[a]), nb = ncart(B->l[b]), nc = ncart(B->l[c]),
                      nd = ncart(B->l[d]);
            const int oa = B->ao_off[a], ob = B->ao_off[b], oc = B->ao_off[c], od = B->ao_off[d];
            const double deg = degs[q];
            /* the six blocks of this quartet, then one add per element */
            double jab[28 * 28], jcd[28 * 28], kac[28 * 28], kad[28 * 28], kbc[28 * 28], kbd[28 * 28];
            memset(jab, 0, sizeof(double) * na * nb);
            memset(jcd, 0, sizeof(double) * nc * nd);
            memset(kac, 0, sizeof(double) * na * nc);
            memset(kad, 0, sizeof(double) * na * nd);
            memset(kbc, 0, sizeof(double) * nb * nc);
            memset(kbd, 0, sizeof(double) * nb * nd);
#define DD(u, v) D[(size_t)(u) * nao + (v)]
            for (int i = 0; i < na; ++i)
                for (int j = 0; j < nb; ++j)
                    for (int k = 0; k < nc; ++k)
                        for (int l = 0; l < nd; ++l) {
                            const double x = deg * blk[(size_t)(i * nb + j) * nc * nd + k * nd + l];
                            jab[i * nb + j] += 2.0 * DD(oc + k, od + l) * x;
                            jcd[k * nd + l] += 2.0 * DD(oa + i, ob + j) * x;
                            kac[i * nc + k] += DD(ob + j, od + l) * x;
                            kad[i * nd + l] += DD(ob + j, oc + k) * x;
                            kbc[j * nc + k] += DD(oa + i, od + l) * x;
                            kbd[j * nd + l] += DD(oa + i, oc + k) * x;
                        }
#undef DD
#define ADD(M, r, c_, v) do { double *m_ = &M[(size_t)(r) * nao + (c_)]; const double v_ = (v); \
                              _Pragma("omp atomic") *m_ += v_; } while (0)
            for (int i = 0; i < na; ++i)
                for (int j = 0; j < nb; ++j) ADD(J, oa + i, ob + j, jab[i * nb + j]);
            for (int k = 0; k < nc; ++k)
                for (int l = 0; l < nd; ++l) ADD(J, oc + k, od + l, jcd[k * nd + l]);
            for (int i = 0; i < na; ++i) {
                for (int k = 0; k < nc; ++k) ADD(K, oa + i, oc + k, kac[i * nc + k]);
                for (int l = 0; l < nd; ++l) ADD(K, oa + i, od + l, kad[i * nd + l]);
            }
            for (int j = 0; j < nb; ++j) {
                for (int k = 0; k < nc; ++k) ADD(K, ob + j, oc + k, kbc[j * nc + k]);
                for (int l = 0; l < nd; ++l) ADD(K, ob + j, od + l, kbd[j * nd + l]);
            }
#undef ADD
            clock_gettime(CLOCK_MONOTONIC, &t1);
            if (sec) sec[q] = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
        }
        free(blk);
    }
    for (int i = 0; i < np; ++i) free_pair(&sp[i]);
    free(sp);
    free(slot);
    return 0;
}
