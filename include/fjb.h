/*
 * fjb.h -- the C ABI of libfjb.so, a B200 (sm_100a) Fock-build engine.
 *
 * Plain C: pointers, sizes, status codes.  No torch or CUDA types in the
 * signatures (a stream is passed as `void*`, a cudaStream_t; NULL is the
 * legacy default stream).  Every function returns 0 on success or a negative
 * FJB_E* code; fjb_last_error() then holds a one-line message.
 *
 * Each entry point names the reference interface it replaces (paths within
 * the reference project, whatDiracIsCooking/FelizJueves):
 *
 *   fjb_create        ao/shell.py:110-165   Shell / Basis (l, centre,
 *                                            exponents, coefficients; AO
 *                                            offsets in Basis order)
 *   fjb_plan          eri/fock/launch_f.py:390-466  f_launches(basis, D, *,
 *                                            bound, tau, n) with the bound
 *                                            ao/pairs.py:528-541
 *                                            primitive_schwarz_bounds
 *   fjb_plan_counts,
 *   fjb_plan_export   launch_f.py:312-345   FPlan.counts() and the lists
 *                                            (batches, pairs, prims,
 *                                            launches, screened, deleted)
 *   fjb_screen_mask   eri/fock/walk_f.py:344-380  the six-block in-kernel
 *                                            screen, per launched quartet
 *   fjb_fock_build    eri/fock/walk_f.py:306-415 + kernel_f.py:655 +
 *                                            kernel_f.py:621 close: the fused
 *                                            G = J - K/2 build, and J and K
 *                                            (eri/fock/fock.py:126-176 define
 *                                            them; j.py:436, k.py:482)
 *   fjb_eri_blocks    eri/eri.py:133-145 eri_block and
 *                     eri/hgp_drive.py:206 (the per-quartet ERI tap)
 *   fjb_boys          emit/_c.py:144-210 fj_boys<M> (device Boys)
 *   FJB_FP64_SCATTER,
 *   fjb_scatter_map   eri/fock/levers/scatter.py:141-198 (the slot layout) and
 *                     eri/fock/kernel_f_scatter.py:203-260 scatter_map(cls,
 *                                            n_ket, bra_ao, ket_ao); the build
 *                                            mode is walk_f.py:393-408's
 *                                            scatter lever
 *   fjb_coulomb       eri/j_coulomb/j.py:436-450 coulomb_matrix(basis, D, *,
 *                                            pq, tau) and its screened sweep
 *                                            j.py:538-581 (the MMD J-engine:
 *                                            kernel_dq.py, mmd/kernel.py,
 *                                            kernel_jab.py)
 *   fjb_j_plan_lists  eri/j_coulomb/launch.py:274-327 launches(): the
 *                                            records, bounds, keys and the
 *                                            sorted ket order
 *   fjb_one_electron  one_electron/overlap.py:67 overlap_matrix,
 *                     one_electron/kinetic.py:114 kinetic_matrix,
 *                     one_electron/potential.py:101 potential_matrix (nuclei
 *                                            (Z, centre)), assembled as
 *                                            one_electron/one_electron.py:57
 *                                            matrix; H = T + V the core
 *                                            Hamiltonian
 *   fjb_last_error,
 *   fjb_destroy       the reference raises ValueError with a message
 *
 * Units and conventions are the reference's: Bohr, Cartesian AOs in
 * cartesians(l) order (i desc, then j desc), coefficients multiplying
 * UNNORMALISED primitives; D is n_ao x n_ao row-major, finite and EXACTLY
 * symmetric (refused otherwise, never symmetrised).
 */
#ifndef FJB_H
#define FJB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FJB_OK 0
#define FJB_E_ARG (-1)      /* a refused argument (the reference's ValueError) */
#define FJB_E_CUDA (-2)     /* a CUDA runtime error */
#define FJB_E_STATE (-3)    /* called out of order (e.g. build before plan) */
#define FJB_E_LIMIT (-4)    /* above a compiled limit (L, degree) */
#define FJB_E_TIMEOUT (-5)  /* a bounded device wait ran out */
#define FJB_E_PLAN (-6)     /* the plan's soundness check failed */

#define FJB_MAX_L 3            /* per shell, Fock build */
#define FJB_MAX_PRIM_PAIRS 128 /* kernel_f.py:196-203 MAX_PRIM_PAIRS */

/* precision modes of fjb_fock_build */
#define FJB_FP64 0   /* every quartet in FP64 */
#define FJB_ROUTED 1 /* quartets under the magnitude threshold run E/R/VRR in FP32 */
#define FJB_FP64_SCATTER 2 /* FP64, atomics-free: slot buffer + per-element scatter, bit-reproducible */

typedef struct fjb_handle fjb_handle;

/* A basis: per shell its l, centre (3 doubles), first primitive index and
 * primitive count into exps/coefs. */
typedef struct fjb_basis {
    int32_t n_shells;
    const int32_t *l;
    const double *centre;
    const int32_t *prim0;
    const int32_t *nprim;
    const double *exps;
    const double *coefs;
} fjb_basis;

typedef struct fjb_plan_counts_t {
    int64_t pairs, pairs_deleted, primitive_pairs, primitive_pairs_pruned;
    int64_t batches, batch_pairs, batch_pairs_screened, launches;
    int64_t kept_pairs, kept_prims, units, quartets_launched;
} fjb_plan_counts_t;

/* The plan's lists, written into caller-owned host arrays sized from
 * fjb_plan_counts (any pointer may be NULL to skip that list):
 *   batch_key[4*batches]   (la, lb, degree, mag), batches in plan order
 *   batch_npairs[batches]
 *   pair_ab[2*kept_pairs]  (a, b) of each kept pair, batch by batch, each
 *                          batch's pairs in their sorted order
 *   pair_G, pair_dmax, pair_key [kept_pairs]; pair_mag [kept_pairs]
 *   prims[kept_prims]      kept primitive-pair indices (i*K_b + j), per pair
 *   prim_G[kept_prims]
 *   launches[2*launches], screened[2*batch_pairs_screened],
 *   deleted[2*pairs_deleted]                                               */
typedef struct fjb_plan_lists {
    int32_t *batch_key, *batch_npairs, *pair_ab, *pair_mag, *prims;
    double *pair_G, *pair_dmax, *pair_key, *prim_G;
    int32_t *launches, *screened, *deleted;
    double *magnitudes; /* [n_mag] */
    double *eps, *g_max; /* scalars */
} fjb_plan_lists;

const char *fjb_last_error(const fjb_handle *h);
const char *fjb_version(void);

int fjb_create(fjb_handle **out, const fjb_basis *basis, int device);
void fjb_destroy(fjb_handle *h);

/* Build the pair stream for density D (HOST pointer, n_ao^2) at threshold
 * tau with n_mag eq.29 magnitudes, and stage it on the device.  The plan's
 * sort inside a batch reads D; the builds that follow take any symmetric D
 * (the in-kernel six-block screen reads the density each build is given).
 * The basis's primitive-pair bounds do not depend on D: the first plan of a
 * handle computes them and later plans reuse them. */
int fjb_plan(fjb_handle *h, const double *D_host, double tau, int n_mag);
int fjb_plan_counts(const fjb_handle *h, fjb_plan_counts_t *out);
int fjb_plan_export(const fjb_handle *h, fjb_plan_lists *out);
/* The plan's work units, 4 int32 each (launch, bra pair index, first ket
 * index, end ket index), in the order the build's class kernels take them
 * (class by class, each class's launches in plan order, each bra pair's
 * kets in chunks of 32).  The runtime writes them on the device from one
 * span a launch; this copies them to units_host (HOST, room for cap units;
 * NULL to ask only for n_units).  Synchronises. */
int fjb_plan_units(const fjb_handle *h, int32_t *units_host, int64_t cap, int64_t *n_units);
int fjb_n_ao(const fjb_handle *h);

/* The six-block screen decision of every launched quartet, in (launch, bra
 * pair, ket pair >= bra on the diagonal) order: mask_dev[q] = 1 when the
 * quartet is skipped.  D_dev and mask_dev are DEVICE pointers
 * (quartets_launched bytes). */
int fjb_screen_mask(fjb_handle *h, const double *D_dev, uint8_t *mask_dev,
                    void *stream);

/* The fused build.  D_dev, J_dev, K_dev, G_dev are DEVICE pointers to
 * n_ao^2 doubles (any of J/K/G may be NULL).  precision: FJB_FP64,
 * FJB_ROUTED (then `threshold` is the Schwarz x |D| bound under which a
 * quartet runs its recurrences in FP32; <= 0 means the default 1e-9), or
 * FJB_FP64_SCATTER (FP64 without atomics, bit-reproducible; see
 * fjb_scatter_map; its first call stages the maps and allocates).
 * Stream-ordered; nothing is synchronised. */
int fjb_fock_build(fjb_handle *h, const double *D_dev, double *J_dev, double *K_dev,
                   double *G_dev, int precision, double threshold, void *stream);

/* fjb_fock_build as a CUDA graph: the first call for a given (D_dev, J_dev,
 * K_dev, G_dev, precision, threshold) captures the build's whole kernel
 * sequence on a handle-owned stream and instantiates it; every call then
 * launches that graph on `stream`.  An SCF loop that updates D in place
 * replays one graph per iteration.  A new plan, or other pointers, capture
 * again. */
int fjb_fock_build_graph(fjb_handle *h, const double *D_dev, double *J_dev, double *K_dev,
                         double *G_dev, int precision, double threshold, void *stream);

/* The same build through host buffers: D_host in, J/K/G_host out (any of
 * the outputs may be NULL).  Copies in, builds, copies out, synchronises. */
int fjb_fock_build_host(fjb_handle *h, const double *D_host, double *J_host,
                        double *K_host, double *G_host, int precision, double threshold);

/* ERI blocks (ab|cd) of n ordered shell quartets quartets[4*n], every
 * primitive, by the same HGP recurrences as the build.  out_dev (DEVICE)
 * receives the blocks back to back, each n_a n_b x n_c n_d row-major in the
 * reference's eri_block layout; offsets[n+1] (HOST, filled) gives where.
 * Synchronises. */
int fjb_eri_blocks(fjb_handle *h, const int32_t *quartets, int n, double *out_dev,
                   int64_t *offsets);
/* The same blocks with the routed path's FP32 recurrences (VRR, boundary and
 * HRR in FP32; Boys and scalars FP64): what a quartet routed to FP32
 * contributes, for measuring its FP32 error (eri/fock/levers/mixed.py's
 * fmixed regions). */
int fjb_eri_blocks_fp32(fjb_handle *h, const int32_t *quartets, int n, double *out_dev,
                        int64_t *offsets);

/* The split build's ordered pair stream and its K build
 * (eri/hjk/launch_hjk.py:280 hjk_launches; eri/hjk/kernel_hk.py:324
 * build_hk_kernel).  fjb_hjk_plan: every ORDERED shell pair (a, b) with G
 * the fsum of its primitive Schwarz bounds (none pruned), bins (la, lb,
 * degree) in sorted order, pairs descending by G stably, every ordered batch
 * pair a launch, every ordered quartet of pairs a visit with the key
 * (G_ab G_cd) max|D_bd| (screen FJB_HJK_SCREEN_K, k_key) or (G_ab G_cd)
 * max|D_cd| (FJB_HJK_SCREEN_J, j_key), skipped when below tau.  mode
 * FJB_HJK_ORDERED runs each launch on its own class; FJB_HJK_CANONICAL on
 * the first member of its 8-fold orbit (the reference's GROUP order) with
 * la <= lb, lc <= ld, (la, lb) <= (lc, ld), this library's compiled classes
 * (the reference's canonical mode takes its cheapest generated recurrence
 * instead; launches and visits are the same).  D_host is n_ao^2, exactly
 * symmetric; refusals as the reference's (FJB_E_ARG; FJB_E_LIMIT for a
 * degree above 128).
 * fjb_hjk_counts: counts[6] = pairs, batches, launches, kernel classes,
 * visits (pairs^2), skipped visits (a host sweep over every visit).
 * fjb_hjk_export (HOST arrays, each may be NULL): pairs[5 n_pairs] = (a, b,
 * la, lb, degree) in batch order, pair_G[n_pairs], batches[5 n_batches] =
 * (la, lb, degree, first pair, pairs), launches[14 n_launches] = (bra
 * batch, ket batch, ordered class[4], kernel class[4], shells[4]: kernel
 * position j reads the ordered quartet's position shells[j]).
 * fjb_hjk_keys: one launch's visit keys (bra pair outer) and skip flags.
 * fjb_hjk_k: K (DEVICE, n_ao^2) = sum over every visit not skipped of
 * K[a][c] += D[b][d] (ab|cd), no weights (each ordered quartet once), on
 * the HGP interpreter, the key evaluated on the device in the plan's
 * operation order; needs a stream planned with K's key.  Stream-ordered. */
#define FJB_HJK_ORDERED 0
#define FJB_HJK_CANONICAL 1
#define FJB_HJK_SCREEN_J 0
#define FJB_HJK_SCREEN_K 1
int fjb_hjk_plan(fjb_handle *h, const double *D_host, double tau, int mode, int screen);
int fjb_hjk_counts(const fjb_handle *h, int64_t *counts);
int fjb_hjk_export(const fjb_handle *h, int32_t *pairs, double *pair_G, int32_t *batches, int32_t *launches);
int fjb_hjk_keys(const fjb_handle *h, int launch, double *keys, uint8_t *skipped);
int fjb_hjk_k(fjb_handle *h, const double *D_dev, double *K_dev, void *stream);
/* Per launch (HOST, n_launches): the quartets the last fjb_hjk_k computed
 * (visits not skipped by the device's key).  Synchronises the device. */
int fjb_hjk_computed(fjb_handle *h, int64_t *per_launch);

/* Density fitting (eri/density_fit/metric.py:228 metric_matrix,
 * eri3.py:226 eri3_tensor).  fjb_create_df makes a handle over the AO basis
 * (l <= 3) and an auxiliary basis (l <= FJB_MAX_L_AUX); an auxiliary
 * primitive is the reference's single-Gaussian "pair" (metric.py:1-60),
 * realised here as the primitive paired with a unit s function (exponent 0,
 * coefficient 1), which gives exactly its dressing c (pi/alpha)^{3/2}.
 * fjb_df_blocks computes, on the device, by the build's HGP recurrences:
 *   kind FJB_DF_METRIC: items[2i..2i+1] = aux shells (P, Q) -> (P|Q) block,
 *                       rows cartesians(lP), columns cartesians(lQ);
 *   kind FJB_DF_ERI3:   items[3i..3i+2] = (a, b, P), AO shells a, b and aux
 *                       shell P -> (ab|P) block, rows a outer then b,
 *                       columns cartesians(lP) (the reference's [m][n][P]
 *                       layout, aux fastest).
 * Blocks land back to back in out_dev (DEVICE); offsets[n+1] (HOST) says
 * where.  Synchronises. */
#define FJB_MAX_L_AUX 6
#define FJB_DF_METRIC 0
#define FJB_DF_ERI3 1
int fjb_create_df(fjb_handle **out, const fjb_basis *ao, const fjb_basis *aux, int device);
int fjb_df_blocks(fjb_handle *h, int kind, const int32_t *items, int n, double *out_dev,
                  int64_t *offsets);

/* The learned precision router (no counterpart in the reference; its
 * fmixed lever, eri/fock/levers/mixed.py, is the FP32 path it routes to).
 * A 12 -> 64 -> 64 -> 1 tanh MLP predicts log10 of a quartet's largest
 * deposit from pair features; in FJB_ROUTED builds a unit whose every
 * computed quartet is under the rigorous bound (threshold), or predicted
 * under 10^log10_threshold, runs its recurrences in FP32.  Skipping stays
 * the six-block screen's.  fjb_mlp_n_params() floats, packed
 * mu[12] sd[12] W1[64][12] b1[64] W2[64][64] b2[64] w3[64] b3.
 * params_host NULL turns the learned router off. */
int fjb_mlp_n_params(void);
int fjb_router_set(fjb_handle *h, const float *params_host, float log10_threshold);
/* How far above the threshold (decades, 0..5; default 5) a quartet's bound
 * may be for the network to be asked: a unit with a quartet further above
 * stays FP64 without running it.  Set it to the largest gap below the bound
 * the trained network predicts (plus its margin) so the routing pass runs
 * the network only where it can move a unit to FP32; a smaller reach only
 * keeps more units FP64. */
int fjb_router_reach(fjb_handle *h, double decades);
/* Which classes ask the network: those with la + lb + lc + ld >=
 * min_total_l (default 0, every class).  Asking the network costs a warp
 * of 32 quartets 80 tensor-core products (mma.sync m16n8k16) and 4,096
 * tanh, so below some total angular momentum it can cost more than the
 * FP32 units it adds save; those classes route by the bound alone. */
int fjb_router_classes(fjb_handle *h, int min_total_l);
/* Features (n x 12 floats) and six-block bounds (n doubles) of sampled
 * launched quartets, samples[3i..3i+2] = (launch, bra index, ket index) in
 * the plan's order (HOST); feat_dev, bound_dev DEVICE.  Synchronises. */
int fjb_router_features(fjb_handle *h, const double *D_dev, const int32_t *samples, int n, float *feat_dev,
                        double *bound_dev);
/* Training and inference kernels (DEVICE pointers, FP32): the forward pass;
 * the mean-squared-error gradient of a batch (scratch_dev holds n x 257
 * floats, sq_err_dev n floats); one Adam step (step counts from 1). */
int fjb_mlp_forward(const float *params_dev, const float *X_dev, int n, float *Y_dev, void *stream);
/* The same network's forward in the routing pass's own arithmetic: both
 * hidden layers as FP16 x FP16 -> FP32 tensor-core products (mma.sync
 * m16n8k16), tanh by the hardware approximation.  The router's margin is
 * calibrated through this call.  Same arguments as fjb_mlp_forward. */
int fjb_mlp_forward_tc(const float *params_dev, const float *X_dev, int n, float *Y_dev, void *stream);
int fjb_mlp_gradient(const float *params_dev, const float *X_dev, const float *T_dev, int n, float *grad_dev,
                     float *sq_err_dev, float *scratch_dev, void *stream);
int fjb_mlp_adam(float *params_dev, const float *grad_dev, float *m_dev, float *v_dev, float lr, int step,
                 void *stream);
/* Work units the last routed build sent to the FP32 and FP64 queues (units
 * of classes without an FP32 body, and of FP64 builds, count as FP64).
 * Synchronises on the last build. */
int fjb_route_stats(const fjb_handle *h, int64_t *units_fp32, int64_t *units_fp64);

/* Device Boys F_0..F_m(T[i]) for n arguments into F_dev[i*(m+1) + k]
 * (DEVICE pointers).  Synchronises. */
int fjb_boys(int m, const double *T_dev, int n, double *F_dev);

/* J by the McMurchie-Davidson J-engine: J_dev (n_ao^2, DEVICE) from the
 * symmetric density D_dev at threshold tau (>= 0; 0 screens nothing), the
 * reference's unique sweep with the ket weight 2 off the diagonal and the
 * sorted break on I_bra * (I_ket * max|D_q|) < tau.  Every element of J_dev
 * is written (no accumulation into it).  Stream-ordered; the first call
 * stages the records (allocates), later calls allocate nothing and can be
 * captured in a CUDA graph. */
int fjb_coulomb(fjb_handle *h, const double *D_dev, double *J_dev, double tau, void *stream);
/* The same with the FP32 E/R tier (eri/j_coulomb/levers/mixed.py:101 _f32,
 * as magnitude routing): a chunk of 32 sorted kets whose largest bound
 * I_bra I_ket max|D_q| is below `threshold` runs its R_{tuv} recursion, its
 * signed D_q and the contraction in FP32; T, the Boys values and every J_p
 * sum stay FP64.  threshold 0 is fjb_coulomb. */
int fjb_coulomb_mixed(fjb_handle *h, const double *D_dev, double *J_dev, double tau, double threshold,
                      void *stream);
/* The atomics-free build's map of plan launch `launch` (plan order): n_el
 * distinct elements (row, col) of J'/K' ascending in el[2*n_el], CSR offsets
 * ptr[n_el + 1], and src[n_slot] each element's slots ascending, the slots
 * numbered by the reference's slot layout.  With the arrays NULL only the
 * counts are set.  FJB_FP64_SCATTER builds use these maps: each quartet
 * stores its five ket-dependent blocks into its own slots, bra blocks are
 * reduced in unit order, and every element sums its slots in order -- no
 * atomics, the same bits on every build.  It needs the launches' slots to fit
 * 2^28 (FJB_E_LIMIT otherwise): a small-system mode. */
int fjb_scatter_map(const fjb_handle *h, int launch, int32_t *el, int32_t *ptr, int32_t *src, int64_t *n_el,
                    int64_t *n_slot);

/* Kernel launches of the last fjb_coulomb. */
int fjb_j_last_launches(const fjb_handle *h);

/* The one-electron matrices of the handle's basis: overlap S, kinetic
 * energy T, nuclear attraction V = -sum_C Z_C <a|1/r_C|b> over n_nuc nuclei
 * (charges[k], coords[3k..3k+2], HOST, Bohr; charges finite, n_nuc >= 0) and
 * H = T + V, each n_ao x n_ao row-major on the DEVICE; any of the four may be
 * NULL (not written), every element of the others is written, each exactly
 * symmetric.  Stream-ordered; the first call stages the shell pairs
 * (allocates). */
int fjb_one_electron(fjb_handle *h, const double *charges, const double *coords, int n_nuc, double *S_dev,
                     double *T_dev, double *V_dev, double *H_dev, void *stream);

/* The J-engine's plan on the host for density D_host: per record (sweep
 * order: shell pairs a >= b, a outer; primitive pairs i outer) its shell
 * pair, primitive index i*K_b + j, L, I_pair and ket key I_pair*max|D_q|;
 * the ket order per L (descending key, stable) with L_off[2*FJB_MAX_L + 2]
 * offsets into it.  Caller-allocated arrays of *n_records entries; with
 * out == NULL only *n_records is set.  Host-only handles allowed. */
typedef struct fjb_j_lists {
    int32_t *a, *b, *prim, *L;
    double *G, *key;
    int32_t *ket_order;
    int64_t *L_off;
} fjb_j_lists;
int fjb_j_plan_lists(const fjb_handle *h, const double *D_host, fjb_j_lists *out, int64_t *n_records);

/* Elapsed device milliseconds of the last fjb_fock_build's class kernels
 * (events recorded on the build's stream); and the number of kernel
 * launches that build issued. */
int fjb_last_build_stats(const fjb_handle *h, double *ms_kernels, int *n_launches);

/* Per launch of the plan (launch_f.py FLaunch order): its class, the two
 * sides' contraction degrees, the quartets it meets and the quartets the
 * last build computed (not skipped by the six-block screen).  n = launches
 * of fjb_plan_counts.  Synchronises on the last build. */
typedef struct fjb_launch_stat {
    int32_t la, lb, lc, ld, kab, kcd;
    int64_t launched, computed;
} fjb_launch_stat;
int fjb_launch_stats(const fjb_handle *h, fjb_launch_stat *out, int64_t n);

/* Per class kernel of the last build: its class, device milliseconds
 * (events around the launch on the build's stream), work units and the
 * engine of its FP64 units (0 the HGP interpreter, 1 the register kernel,
 * 2 the Rys kernel). */
typedef struct fjb_class_stat {
    int32_t la, lb, lc, ld;
    double ms;
    int64_t units;
    int32_t engine, pad;
} fjb_class_stat;
int fjb_class_stats(const fjb_handle *h, fjb_class_stat *out, int64_t n, int64_t *n_classes);

/* Per-class launch configuration: the CTA width (32, 64, 128, 256; 0 =
 * the class's default) and the chunk of primitive quartets one CTA pass
 * holds (0 = sized for occupancy).  Applies to the current plan and to later
 * ones.  This is what the autotuner sets after timing candidates, as the
 * reference's performance/dispatch.py:1-45 picks a batch count from measured
 * medians.  FJB_E_LIMIT if the class does not fit that configuration. */
int fjb_set_class_config(fjb_handle *h, int la, int lb, int lc, int ld, int threads, int slots);
/* The same for the routed path's FP32 interpreter kernel of a class (used
 * for its FP32 units when the class has no FP32 register body); threads 0
 * and slots 0 restore the FP64 configuration's FP32 twin. */
int fjb_set_class_config32(fjb_handle *h, int la, int lb, int lc, int ld, int threads, int slots);

/* Which classes run on the Rys kernel -- the Rys quadrature in place of the
 * HGP vertical recurrence, the reference's third engine (rys/roots.py,
 * eri/fock/kernel_frys.py:194), feeding the same HRR and digest.  mode 1
 * (the default): every class without an FP64 register body, and those with
 * one where the Rys kernel measured faster; plus, for the routed build's
 * FP32 units, every class without an FP32 register body.  mode 0: none (the
 * HGP shared-memory interpreter takes them).  mode 2: every class the Rys
 * kernel has.  Applies to the current plan and later ones.  The
 * atomics-free build (FJB_FP64_SCATTER) and the ERI tap keep the HGP
 * kernels. */
int fjb_set_rys(fjb_handle *h, int mode);

/* The batched build: many molecules, each a planned handle (same device,
 * same tau), built together with ONE launch per angular-momentum class --
 * every molecule's work units of that class in one class-sorted queue, each
 * unit finding its molecule's density and accumulators through its launch
 * -- plus one launch for all molecules' density blocks and one for their
 * closing.  The batch reads the handles' plans when it is made (they must
 * outlive it); fjb_batch_set_densities binds each molecule's DEVICE D and
 * its J, K, G outputs (any may be NULL) once, fjb_batch_build then runs and
 * is stream-ordered and capturable (FJB_FP64, or FJB_ROUTED: by the
 * learned router when the first handle has one installed, fjb_router_set,
 * else by the Schwarz x density bound; the budget check is a
 * single-molecule feature).  No counterpart in the reference, whose
 * launches are per molecule (eri/fock/walk_f.py:306). */
typedef struct fjb_batch fjb_batch;
int fjb_batch_create(fjb_batch **out, fjb_handle *const *handles, int n);
int fjb_batch_set_densities(fjb_batch *b, const double *const *D_dev, double *const *J_dev,
                            double *const *K_dev, double *const *G_dev);
int fjb_batch_build(fjb_batch *b, int precision, double threshold, void *stream);
/* Device milliseconds of the last batch build's class launches, the number
 * of class launches and of work units. */
int fjb_batch_stats(const fjb_batch *b, double *ms, int64_t *n_classes, int64_t *n_units);
const char *fjb_batch_last_error(const fjb_batch *b);
void fjb_batch_destroy(fjb_batch *b);

/* Density-fitted J and K of the symmetric density D (DEVICE, n_ao^2) from
 * the factors B (DEVICE, n_aux x n_ao x n_ao, FP64: B_P = sum_Q (L^-1)_PQ
 * (Q|mn), L the Cholesky factor of the metric (P|Q)).  J_mn = sum_P B_P,mn
 * gamma_P, gamma_P = sum_ls B_P,ls D_ls in FP64; K_mn = sum_P (B_P D B_P^T)_mn
 * as two GEMMs on the tensor cores, every operand split into three BF16
 * terms and the six products of total order <= 2 accumulated in FP32.  The
 * handle owns the workspace (about 2 n_aux n_ao^2 doubles).  The reference
 * computes no DF-J/K (eri/density_fit/__init__.py:8-9); its (mn|P) layout
 * ([m][n][P], eri/density_fit/eri3.py:226) is what DFEngine.factors turns
 * into B.  Synchronises `stream`; FJB_E_TIMEOUT if a tensor-core wait ran
 * out. */
int fjb_df_jk(fjb_handle *h, const double *B_dev, int64_t n_aux, int64_t n_ao, const double *D_dev,
              double *J_dev, double *K_dev, void *stream);

/* The three-centre integrals (mn|P) of one aux block, on the device, by
 * Rys quadrature (eri/density_fit/eri3.py:226 eri3_tensor, restricted to
 * the aux functions of aux shells [aux_shell0, aux_shell1)): out_dev
 * (DEVICE, n_ao x n_ao x nb doubles, nb the block's aux functions) receives
 * (mn|P) at [m][n][P - p0], aux fastest, both (m, n) and (n, m) written;
 * p0 is the first function of aux_shell0.  A (shell pair, aux shell) block
 * whose Schwarz product sqrt(max|(ab|ab)|) sqrt(max|(P|P)|) is below tau is
 * zero (tau <= 0: none is).  The first call stages the AO pairs and their
 * Schwarz factors (from the ERI tap; synchronises); every call synchronises
 * `stream` before staging its work units, then runs asynchronously on it.
 * Aux shells to l = 4 (FJB_E_LIMIT above).  A block of nb aux functions
 * holds 8 n_ao^2 nb bytes: this is how a caller streams the DF build of a
 * system whose whole tensor does not fit (DFEngine.jk_streamed).
 * n_launches (HOST, may be NULL) receives the number of class kernels
 * launched. */
int fjb_df_eri3(fjb_handle *h, int aux_shell0, int aux_shell1, double tau, double *out_dev, int32_t *n_launches,
                void *stream);

/* K = Z Z^T (DEVICE, rows x rows, FP64) for Z (DEVICE, rows x cols, FP64,
 * row-major) on the tensor cores: Z split into three BF16 terms, the six
 * products of total order <= 2 accumulated in FP32 over at most 16,384
 * terms of the contraction, those partial sums added in FP64.  The
 * occupied-orbital DF exchange: Z[m][(i, Q)] = sum_P (m i|P) W_PQ, W the
 * metric's inverse factor.  The handle owns the workspace (6 rows cols
 * bytes, rounded up to whole tiles).  Synchronises `stream`; FJB_E_TIMEOUT
 * if a tensor-core wait ran out. */
int fjb_df_syrk(fjb_handle *h, const double *Z_dev, int64_t rows, int64_t cols, double *K_dev, void *stream);

/* The routed build's error-budget check (on by default: budget 1e-8,
 * stride 32).  Every stride-th unit the router would put on the FP32 queue
 * is built apart instead, twice, in FP32 and in FP64, into side
 * accumulators; the largest element of their G difference times
 * sqrt(stride) estimates the FP32 queue's error in G (independent rounding
 * errors of stride times as many units: a statistical estimate, not a
 * bound).  If the estimate is within `budget` the sample's FP32 build joins
 * G; otherwise the same build re-runs every other FP32 unit in FP64 and
 * takes the sample's FP64 build: the build falls back to plain FP64 by
 * itself, on the device, inside a captured graph too.  The
 * first checked build of a handle allocates six n_ao^2 side buffers: make it
 * before any capture of your own (fjb_fock_build_graph does).  budget <= 0
 * turns the check off.  No counterpart in the reference; it is the
 * routed path's "checked against the error budget, re-routed to FP64 on
 * violation". */
int fjb_set_route_check(fjb_handle *h, double budget, int stride);
/* The last routed build's check: the estimate and whether it re-ran the
 * FP32 queue in FP64 (1) or kept it (0).  Synchronises the device. */
int fjb_route_check_result(const fjb_handle *h, double *estimate, int *rerouted);

/* fjb_fock_build without any device allocation (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc while they run the
 * SCF loop: a host framework that owns every byte of device memory through
 * its own pool and refuses raw allocations after start-up, or a loop that
 * must not take the allocator's latency or fail on fragmentation between
 * iterations.  The handle and its plan are made once at set-up (they do
 * allocate); this call then builds J, K and G (FP64) into the caller's
 * DEVICE buffers using, as its scratch (the J', K' accumulators and the
 * shell-block density maxima), one file-scope device array of
 * FJB_NOALLOC_SCRATCH_DOUBLES doubles (4.5 MiB) that every GPU loading the
 * library holds until exit.  Limits: n_ao <= FJB_NOALLOC_MAX_AO and
 * n_shells <= FJB_NOALLOC_MAX_SHELLS, else FJB_E_LIMIT.  The first call on
 * a device looks up the array's device address (cudaGetSymbolAddress), so
 * make that first call before any stream capture.  Every call shares the
 * one array: calls that overlap on the GPU (two streams, two handles, two
 * threads) race and corrupt each other's results; serialise them.  The
 * address is kept per device ordinal for the life of the process and
 * belongs to the device's primary context (the runtime's): do not reset the
 * device (cudaDeviceReset) or drive the call from another context while the
 * library is loaded.  fjb_last_build_stats, fjb_launch_stats and
 * fjb_class_stats describe the last fjb_fock_build only: this call records
 * no statistics and leaves theirs as they were. */
#define FJB_NOALLOC_MAX_AO 512
#define FJB_NOALLOC_MAX_SHELLS 256
#define FJB_NOALLOC_SCRATCH_DOUBLES                                              \
    (2 * FJB_NOALLOC_MAX_AO * FJB_NOALLOC_MAX_AO + FJB_NOALLOC_MAX_SHELLS * FJB_NOALLOC_MAX_SHELLS)
int fjb_fock_build_noalloc(fjb_handle *h, const double *D_dev, double *J_dev, double *K_dev,
                           double *G_dev, void *stream);

/* Achievable CUDA-core FMA throughput (TFLOP/s, 2 flops per FMA) by
 * independent FMA chains on every SM, best of `reps` timed launches
 * (the method of the reference's performance/ceilings.py:17-40).
 * fp32 = 0: FP64, 1: FP32. */
int fjb_fma_probe(int fp32, int reps, double *tflops);

#ifdef __cplusplus
}
#endif
#endif
