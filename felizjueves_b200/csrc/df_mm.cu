// df_mm.cu -- the density-fitting J/K contractions (fjb_df_jk).
//
//   J:  gamma_q = sum_mn B_q,mn D_mn,  J_mn = sum_q B_q,mn gamma_q
//       (two FP64 matrix-vector passes over B, HBM-bound: df_gamma_kernel,
//       df_jmat_kernel)
//   K:  X_q = B_q D,  K = sum_q X_q B_q^T
//       (two GEMMs on the 5th-generation tensor cores, df_mm_kernel)
//
// The reference computes no DF-J/K (eri/density_fit/__init__.py:8-9): this
// is the standard contraction with the factors B = L^{-1} (Q|mn) of the
// metric's Cholesky factor L (DFEngine.factors).
//
// Tensor-core arithmetic ("split BF16"): every FP64 operand is rounded to
// FP32 and written as the sum of three BF16 terms hi + mid + lo
// (df_split_kernel); the six products of total order <= 2 (hi.hi, hi.mid,
// mid.hi, hi.lo, mid.mid, lo.hi) are accumulated in FP32 in tensor memory,
// which keeps the FP32 operands' precision to about 2^-24 relative.
//
// df_mm_kernel: one CTA (four warps) per 128 x 128 output tile.  Per K-tile
// of 64, the threads stage the six BF16 operand tiles (A and B, three parts
// each, 96 KiB) into shared memory in the UMMA canonical K-major layout
// without swizzle (8-row x 16-byte core matrices, 128 bytes each; LBO = 128
// bytes between core matrices along K, SBO = 1024 bytes between 8-row
// groups), one thread issues the 24 tcgen05.mma (six products x four
// K = 16 steps) into the FP32 accumulator in TMEM and commits them to an
// mbarrier that every thread waits on before the tiles are overwritten.
// The epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM
// lanes, i.e. output rows, 32w .. 32w + 31) and writes FP64.  Every wait is
// bounded: on timeout the kernel records an error flag, frees its TMEM and
// returns.  Operands come from this GPU's own memory only; no multicast.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

namespace fjb {

namespace {

constexpr int kMmTile = 128;   // output rows (M) and columns (N) of a CTA
constexpr int kMmK = 64;       // K per staged tile
constexpr int kMmThreads = 128;
constexpr int kPartBytes = kMmTile * kMmK * 2;  // one BF16 operand tile: 16 KiB
constexpr long long kWaitLimit = 1LL << 22;     // mbarrier polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor, K-major, no swizzle (layout type 0),
// descriptor version 1: start address, LBO and SBO in 16-byte units.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of tcgen05.mma kind::f16: D F32, A and B BF16,
// both K-major, N = 128, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kMmTile >> 3) << 17) |
                            ((uint32_t)(kMmTile >> 4) << 24);

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Poll the mbarrier's phase `parity` at most kWaitLimit times; false on
// timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace

// Round v (FP64) to FP32 and split it into three BF16 terms.
__device__ __forceinline__ void split3(double v, __nv_bfloat16 *h, __nv_bfloat16 *m, __nv_bfloat16 *l) {
    const float f = (float)v;
    const __nv_bfloat16 a = __float2bfloat16_rn(f);
    const float r = f - __bfloat162float(a);
    const __nv_bfloat16 b = __float2bfloat16_rn(r);
    const float s = r - __bfloat162float(b);
    *h = a;
    *m = b;
    *l = __float2bfloat16_rn(s);
}

// The split operand of a GEMM, rows x cols (cols = the contraction index),
// written into three BF16 arrays of rows_p rows (a multiple of kMmTile) and
// ldp columns (a multiple of kMmK), zero-padded, in TILE order: the 128 x 64
// tile (row tile rt, K tile kt) is 16 KiB at ((rt * ldp / 64) + kt) * 8192
// elements, laid out exactly as the MMA reads it from shared memory (the
// canonical K-major no-swizzle layout: element (r, k) of the tile at
// (r / 8) * 512 + (k / 8) * 64 + (r % 8) * 8 + k % 8), so that a tile is
// staged by one contiguous bulk copy.  Element (r, c) of the source:
//   mode 0: src[r * ld + c]
//   mode 1: src[(c / n) * n * n + r * n + c % n]  (the aux-batched
//           transpose: row r of every n x n block q, side by side)
__global__ void df_split_kernel(const double *__restrict__ src, int mode, long long rows, long long cols,
                                long long ld, long long n, long long rows_p, long long ldp, __nv_bfloat16 *hi,
                                __nv_bfloat16 *mid, __nv_bfloat16 *lo) {
    const long long total = rows_p * ldp, kts = ldp / kMmK;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long tile = i >> 13, w = i & 8191;
        const long long rt = tile / kts, kt = tile - rt * kts;
        const int rem = (int)(w & 511), r8 = (int)(w >> 9);
        const long long r = rt * kMmTile + r8 * 8 + ((rem & 63) >> 3);
        const long long c = kt * kMmK + (rem >> 6) * 8 + (rem & 7);
        double v = 0.0;
        if (r < rows && c < cols) v = mode == 0 ? src[r * ld + c] : src[(c / n) * n * n + r * n + c % n];
        split3(v, hi + i, mid + i, lo + i);
    }
}

namespace {

// One bulk (non-tensor) TMA copy global -> shared, completing on `bar`.
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

constexpr int kStages = 2;
constexpr int kStageBytes = 6 * kPartBytes;  // A0 A1 A2 B0 B1 B2

}  // namespace

// C[M x N] (FP64, leading dimension ldc) = sum over the six split products
// of A (rows_p x ldp) and B (cols_p x ldp), both in tile order: C = A B^T,
// over this CTA's K tiles [z kt_per_split, (z + 1) kt_per_split).  Thread 0
// drives a two-stage pipeline: the six 16 KiB tiles of a K step arrive by
// bulk copies on the stage's `full` barrier (transaction-counted); the 24
// MMAs that read them are committed to the stage's `empty` barrier, which
// releases the stage for the copies two K steps ahead.
__global__ void __launch_bounds__(kMmThreads, 1)
    df_mm_kernel(const __nv_bfloat16 *__restrict__ A0, const __nv_bfloat16 *__restrict__ A1,
                 const __nv_bfloat16 *__restrict__ A2, const __nv_bfloat16 *__restrict__ B0,
                 const __nv_bfloat16 *__restrict__ B1, const __nv_bfloat16 *__restrict__ B2, long long M,
                 long long N, long long ldp, double *__restrict__ C, long long ldc, int kt_per_split, int *err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], done;
    __shared__ uint32_t tmem_base;
    __shared__ int s_ok;
    const int tid = threadIdx.x, warp = tid >> 5;
    const long long kts = ldp / kMmK;
    const long long mt = blockIdx.x, nt = blockIdx.y;
    const int k_begin = (int)blockIdx.z * kt_per_split;
    const int k_end = (int)min((long long)(k_begin + kt_per_split), kts);
    const bool split = gridDim.z > 1;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(kMmTile));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;");
        s_ok = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    if (tid == 0 && k_begin < k_end) {
        const __nv_bfloat16 *parts[6] = {A0, A1, A2, B0, B1, B2};
        auto issue = [&](int kt, int s) {
            unsigned char *st = smem + s * kStageBytes;
            mbar_expect_tx(&full[s], kStageBytes);
#pragma unroll
            for (int p = 0; p < 6; ++p) {
                const long long tile = (p < 3 ? mt : nt) * kts + kt;
                bulk_copy(st + p * kPartBytes, parts[p] + tile * (kPartBytes / 2), kPartBytes, &full[s]);
            }
        };
        const int nk = k_end - k_begin;
        for (int i = 0; i < kStages && i < nk; ++i) issue(k_begin + i, i);
        bool ok = true;
        for (int i = 0; i < nk && ok; ++i) {
            const int s = i % kStages;
            const uint32_t ph = (uint32_t)((i / kStages) & 1);
            if (!mbar_wait(&full[s], ph)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t base = smem_u32(smem + s * kStageBytes);
            const int pa[6] = {0, 0, 1, 0, 1, 2}, pb[6] = {0, 1, 0, 2, 1, 0};
#pragma unroll
            for (int p = 0; p < 6; ++p)
#pragma unroll
                for (int ks = 0; ks < kMmK / 16; ++ks) {
                    const uint64_t da = umma_desc(base + pa[p] * kPartBytes + ks * 256, 128, 1024);
                    const uint64_t db = umma_desc(base + (3 + pb[p]) * kPartBytes + ks * 256, 128, 1024);
                    const uint32_t acc = (i > 0 || p > 0 || ks > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                        "l"(da), "l"(db), "r"(kIdesc), "r"(acc));
                }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(&empty[s])));
            if (i + kStages < nk) {  // the stage is free once these MMAs have read it
                if (!mbar_wait(&empty[s], ph)) {
                    ok = false;
                    break;
                }
                issue(k_begin + i + kStages, s);
            }
        }
        // every MMA issued so far completes before `done`
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(&done)));
        if (!ok) s_ok = 0;
    }
    __syncthreads();
    bool ok = s_ok != 0;
    if (k_begin < k_end) ok = __syncthreads_and(mbar_wait(&done, 0) && ok) != 0;
    if (k_begin >= k_end) {
        // an empty split: no accumulator to read
    } else if (!ok) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;");
        // epilogue: warp w reads rows 32w + lane, 16 columns at a time
        const long long row = mt * kMmTile + warp * 32 + (tid & 31);
        for (int c0 = 0; c0 < kMmTile; c0 += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                  "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                  "=r"(v[14]), "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;");
            if (row < M)
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const long long col = nt * kMmTile + c0 + j;
                    if (col < N) {
                        // split K: the FP32 partial sums add up in FP64
                        if (split)
                            atomicAdd(C + row * ldc + col, (double)__uint_as_float(v[j]));
                        else
                            C[row * ldc + col] = (double)__uint_as_float(v[j]);
                    }
                }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMmTile));
}

// gamma_q = sum_i B[q][i] D[i], i over the n_ao^2 elements (FP64): one CTA
// per q, a block reduction.
__global__ void df_gamma_kernel(const double *__restrict__ B, const double *__restrict__ D, long long nn,
                                double *gamma) {
    const double *b = B + (long long)blockIdx.x * nn;
    double s = 0.0;
    for (long long i = threadIdx.x; i < nn; i += blockDim.x) s += b[i] * D[i];
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) gamma[blockIdx.x] = s;
    }
}

// J[i] = sum_q B[q][i] gamma_q (FP64): a thread per element, q in order
// (coalesced across i).
__global__ void df_jmat_kernel(const double *__restrict__ B, const double *__restrict__ gamma, long long nq,
                               long long nn, double *J) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nn;
         i += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (long long q = 0; q < nq; ++q) s += B[q * nn + i] * gamma[q];
        J[i] = s;
    }
}

// ---------------------------------------------------------------------------
// host side: the workspace and the launch sequence of one DF-J/K build

namespace {

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

struct DfShape {
    long long nq, n;
    long long rows1, ld1;   // GEMM 1 (X = B D): A is B as (nq n) x n, B is D
    long long rowsn, ld2;   // GEMM 2 (K = sum_q X_q B_q^T): n x (nq n) operands
    long long split1, split2;  // BF16 elements of one split part
};

DfShape df_shape(long long nq, long long n) {
    DfShape s;
    s.nq = nq;
    s.n = n;
    s.rows1 = round_up(nq * n, kMmTile);
    s.ld1 = round_up(n, kMmK);
    s.rowsn = round_up(n, kMmTile);
    s.ld2 = round_up(nq * n, kMmK);
    s.split1 = s.rows1 * s.ld1 + s.rowsn * s.ld1;  // A parts + B parts of GEMM 1, per term
    s.split2 = 2 * s.rowsn * s.ld2;                // A parts + B parts of GEMM 2, per term
    return s;
}

}  // namespace

// Device bytes fjb_df_jk needs as workspace for nq aux functions and n AOs:
// gamma, X (nq n^2 doubles), the error flag and the split operands.
size_t df_jk_workspace_bytes(long long nq, long long n) {
    const DfShape s = df_shape(nq, n);
    const long long split = 3 * (s.split1 > s.split2 ? s.split1 : s.split2);
    return (size_t)round_up((round_up(nq, 32) + nq * n * n) * (long long)sizeof(double), 256) + (size_t)split * 2;
}

// max_per_split > 0 caps the K tiles one CTA accumulates in FP32 (more
// splits, each added into C in FP64): the bound on the FP32 sums' length.
static cudaError_t df_mm(const __nv_bfloat16 *a, long long a_rows, const __nv_bfloat16 *b, long long b_rows,
                         long long ldp, long long M, long long N, double *C, long long ldc, int *err,
                         cudaStream_t st, int max_per_split = 0) {
    static bool attr = false;
    const int smem = kStages * kStageBytes;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(df_mm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const long long pa = a_rows * ldp, pb = b_rows * ldp;
    const long long tiles = (a_rows / kMmTile) * (b_rows / kMmTile);
    const int n_k = (int)(ldp / kMmK);
    // split K until the grid covers the 148 SMs twice, each split keeping
    // at least 8 K-tiles; the splits' FP32 partials are added in FP64
    int splits = 1;
    if (tiles < 2 * 148) splits = (int)std::max(1LL, std::min((long long)(n_k / 8), (2 * 148 + tiles - 1) / tiles));
    if (max_per_split > 0) splits = std::max(splits, (n_k + max_per_split - 1) / max_per_split);
    const int per = (n_k + splits - 1) / splits;
    splits = (n_k + per - 1) / per;
    if (splits > 1) {  // the splits add into C
        cudaError_t e = cudaMemset2DAsync(C, (size_t)ldc * sizeof(double), 0, (size_t)N * sizeof(double),
                                          (size_t)M, st);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((unsigned)(a_rows / kMmTile), (unsigned)(b_rows / kMmTile), (unsigned)splits);
    df_mm_kernel<<<grid, kMmThreads, smem, st>>>(a, a + pa, a + 2 * pa, b, b + pb, b + 2 * pb, M, N, ldp, C, ldc,
                                                 per, err);
    return cudaGetLastError();
}

// J and K of density D from the DF factors B (nq x n x n, FP64, device):
// J in FP64 on the CUDA cores, K by the split-BF16 tensor-core GEMMs.  `work`
// holds df_jk_workspace_bytes(nq, n) device bytes; `err` (device int) is set
// when a bounded wait of the GEMM kernel runs out.
cudaError_t df_jk_launch(const double *B, long long nq, long long n, const double *D, double *J, double *K,
                         void *work, int *err, cudaStream_t st) {
    const DfShape s = df_shape(nq, n);
    double *gamma = static_cast<double *>(work);
    double *X = gamma + round_up(nq, 32);
    // the split operands start on a 256-byte boundary (16-byte vector loads)
    __nv_bfloat16 *sp = reinterpret_cast<__nv_bfloat16 *>(
        static_cast<unsigned char *>(work) + round_up((round_up(nq, 32) + nq * n * n) * (long long)sizeof(double), 256));
    const long long nn = n * n;
    df_gamma_kernel<<<(unsigned)nq, 256, 0, st>>>(B, D, nn, gamma);
    df_jmat_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(B, gamma, nq, nn, J);
    // GEMM 1: X (nq n x n) = B (nq n x n) . D^T (D symmetric)
    __nv_bfloat16 *a1 = sp, *b1 = sp + 3 * s.rows1 * s.ld1;
    const unsigned sgrid = 148 * 16;
    df_split_kernel<<<sgrid, 256, 0, st>>>(B, 0, nq * n, n, n, n, s.rows1, s.ld1, a1, a1 + s.rows1 * s.ld1,
                                           a1 + 2 * s.rows1 * s.ld1);
    df_split_kernel<<<sgrid, 256, 0, st>>>(D, 0, n, n, n, n, s.rowsn, s.ld1, b1, b1 + s.rowsn * s.ld1,
                                           b1 + 2 * s.rowsn * s.ld1);
    cudaError_t e = df_mm(a1, s.rows1, b1, s.rowsn, s.ld1, nq * n, n, X, n, err, st);
    if (e != cudaSuccess) return e;
    // GEMM 2: K (n x n) = [X_q rows side by side] . [B_q rows side by side]^T
    __nv_bfloat16 *a2 = sp, *b2 = sp + 3 * s.rowsn * s.ld2;
    df_split_kernel<<<sgrid, 256, 0, st>>>(X, 1, n, nq * n, 0, n, s.rowsn, s.ld2, a2, a2 + s.rowsn * s.ld2,
                                           a2 + 2 * s.rowsn * s.ld2);
    df_split_kernel<<<sgrid, 256, 0, st>>>(B, 1, n, nq * n, 0, n, s.rowsn, s.ld2, b2, b2 + s.rowsn * s.ld2,
                                           b2 + 2 * s.rowsn * s.ld2);
    e = df_mm(a2, s.rowsn, b2, s.rowsn, s.ld2, n, n, K, n, err, st);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// K = Z Z^T for Z (rows x cols, FP64, row-major, device): the occupied-
// orbital DF exchange, Z[m][(i, Q)] = sum_P Y[m][i][P] W[P][Q] for the
// metric's inverse factor W.  Split-BF16 products on the tensor cores as in
// fjb_df_jk; FP32 sums of at most 256 K tiles (16,384 products), added in
// FP64.  `work` holds df_syrk_workspace_bytes(rows, cols) device bytes.
size_t df_syrk_workspace_bytes(long long rows, long long cols) {
    return (size_t)(3 * round_up(rows, kMmTile) * round_up(cols, kMmK)) * 2;
}

cudaError_t df_syrk_launch(const double *Z, long long rows, long long cols, double *K, void *work, int *err,
                           cudaStream_t st) {
    const long long rp = round_up(rows, kMmTile), ldp = round_up(cols, kMmK);
    __nv_bfloat16 *a = static_cast<__nv_bfloat16 *>(work);
    df_split_kernel<<<148 * 16, 256, 0, st>>>(Z, 0, rows, cols, cols, 0, rp, ldp, a, a + rp * ldp, a + 2 * rp * ldp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = df_mm(a, rp, a, rp, ldp, rows, rows, K, rows, err, st, 256);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace fjb
