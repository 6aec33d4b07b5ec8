// spai.cu -- learned sparse-approximate-inverse (SPAI) preconditioner.
//
// A per-row MLP maps the local stencil of row i of A to the values of row i
// of M, a sparse approximate inverse on A's own pattern, which replaces the
// Jacobi M^-1 = diag(A)^-1 in H = I - M A.  There is no counterpart in the
// reference (its closest relative is the ParaSails preconditioner slot).
//
// Stencil slots.  The operator must be stored by diagonal offsets (K <= 9
// offsets, ascending, the centre among them); slot s is the s-th offset.
// Features of row i (16, BF16): for each non-centre slot s in order,
//   a_s = A[i,i+o_s] / A[i,i]                  (0 where A has no entry)
//   d_s = log(A[j,j] / A[i,i]), j = i + o_s    (0 where A has no entry)
// zero-padded to 16.  Outputs (16, FP32): slot s of row i gives
//   M[i, i+o_s] = (delta(o_s, 0) + out_s) / A[i,i]
// on A's pattern, so a network whose last layer is zero is exactly Jacobi.
//
// Network: 16 -> 64 (ReLU) -> 64 (ReLU) -> 16, BF16 operands with FP32
// accumulation on the tensor cores (tcgen05.mma kind::f16, accumulators in
// tensor memory), FP32 master parameters and Adam moments in HBM.  Flat
// parameter order: W1[64][16], b1[64], W2[64][64], b2[64], W3[16][64], b3[16]
// (weights stored out x in).
//
// Training loss on an operator A and vectors v_1..v_R (residual snapshots
// of MCSA and random vectors):
//   L = (1/R) sum_v |v - M A v|_2^2 / |v|_2^2
// whose gradient with respect to out_{i,s} is
//   G[i,s] = -(2/R) sum_v e_i (A v)_{i+o_s} / (A[i,i] |v|^2),  e = v - M A v.
// The backward kernel propagates G through the network on the tensor cores.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <cstring>
#include <random>
#include <utility>
#include <vector>

#include "internal.h"

namespace mclsgpu {
namespace {

constexpr int kF = 16;      // features
constexpr int kH = 64;      // hidden width
constexpr int kO = 16;      // outputs (stencil slots, padded)
constexpr int kMaxSlots = 9;
constexpr int kTileRows = 128;
constexpr int kThreads = 128;
// Flat parameter offsets.
constexpr int kW1 = 0;
constexpr int kB1 = kW1 + kH * kF;
constexpr int kW2 = kB1 + kH;
constexpr int kB2 = kW2 + kH * kH;
constexpr int kW3 = kB2 + kH;
constexpr int kB3 = kW3 + kO * kH;
constexpr int kParams = kB3 + kO;  // 6288

// ---- shared-memory operand layout ------------------------------------------
// K-major, no swizzle: a tile of R rows (the M or N extent) by C columns (the
// K extent) of BF16 is stored as 8x8 core matrices of 128 contiguous bytes
// (8 rows x 16 bytes); core matrix (r/8, c/8) sits at
// ((c/8) * (R/8) + r/8) * 128.  The same bytes read with the roles of rows
// and columns exchanged form an MN-major operand (rows become K), which the
// weight-gradient products use.
__device__ __forceinline__ uint32_t kmaj_off(int r, int c, int R) {
    return uint32_t((((c >> 3) * (R >> 3)) + (r >> 3)) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

// Shared-memory matrix descriptor (tcgen05), no swizzle.  Fields: start
// address >> 4 in bits 0-13, leading-dimension byte offset >> 4 in 16-29,
// stride-dimension byte offset >> 4 in 32-45, descriptor version 1 in 46-47,
// layout type 0 (no swizzle) in 61-63.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46);
}
// K-major operand: the two 8-column K chunks of one K=16 step are one
// column-chunk stride apart (leading offset); 8-row groups are 128 B apart.
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t tile, int R, int kstep) {
    const uint32_t chunk = uint32_t(R / 8) * 128;
    return smem_desc(tile + uint32_t(2 * kstep) * chunk, chunk, 128);
}
// MN-major view of a tile stored K-major with R rows: MN = the stored
// columns (8-column groups one chunk stride apart: stride offset), K = the
// stored rows (8-row groups 128 B apart: leading offset); K step t covers
// stored rows 16t..16t+15.
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t tile, int R, int kstep) {
    const uint32_t chunk = uint32_t(R / 8) * 128;
    return smem_desc(tile + uint32_t(2 * kstep) * 128, 128, chunk);
}
// Instruction descriptor of kind::f16: FP32 accumulate (bits 4-5 = 1), BF16
// A and B (bits 7-9, 10-12 = 1), majors in bits 15/16 (1 = MN-major),
// N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(a_mn) << 15) | (uint32_t(b_mn) << 16) |
           (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return uint32_t(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t mbar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Polls a bounded mbarrier wait makes before it gives up (host-settable
// through mclsgpu_set_wait_limit; 0 makes every such wait give up at once).
constexpr int kDefaultWaitPolls = 1 << 20;
__device__ int g_wait_polls = kDefaultWaitPolls;

// Bounded wait for the phase `parity` of an mbarrier to complete, at most
// `polls` polls.
__device__ __forceinline__ bool mbar_wait_n(uint32_t mbar, uint32_t parity, int polls) {
    for (int it = 0; it < polls; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(ok)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    return mbar_wait_n(mbar, parity, *reinterpret_cast<volatile int*>(&g_wait_polls));
}
// After a wait gave up, the MMAs of the phase it waited for may still be
// writing tensor memory.  The thread that issued them waits for that phase
// (with the default bound, whatever the host limit) before the columns are
// released.
__device__ __forceinline__ void mbar_drain(uint32_t mbar, uint32_t parity) {
    mbar_wait_n(mbar, parity, kDefaultWaitPolls);
}
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols)
                 : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane (32x32b shape).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ float bf16_round(float x) {
    return __bfloat162float(__float2bfloat16_rn(x));
}
// 8 values -> one 16-byte store of BF16 at a K-major tile position.
__device__ __forceinline__ void store8(unsigned char* tile, int r, int c0, int R, const float* v) {
    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) h[k] = __float2bfloat16_rn(v[k]);
    *reinterpret_cast<uint4*>(tile + kmaj_off(r, c0, R)) = *reinterpret_cast<const uint4*>(h);
}
__device__ __forceinline__ void load8(const unsigned char* tile, int r, int c0, int R, float* v) {
    __align__(16) __nv_bfloat16 h[8];
    *reinterpret_cast<uint4*>(h) = *reinterpret_cast<const uint4*>(tile + kmaj_off(r, c0, R));
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = __bfloat162float(h[k]);
}

struct SlotTable {
    int off[kMaxSlots];
    int K;
    int centre;
    // Two-step offsets o_s + o_t of H = I - M A: distinct values in
    // ascending order, pair[s][t] their index, pcentre the index of 0.
    unsigned char pair[kMaxSlots][kMaxSlots];
    int npair;
    int pcentre;
};

// Features of row i from the diagonal-offset storage of A (FP64 values,
// features formed in FP32: the network reads them in BF16).
__device__ __forceinline__ void row_features(const double* dia, int n, const SlotTable& t, int i,
                                             float* f) {
#pragma unroll
    for (int k = 0; k < kF; ++k) f[k] = 0.f;
    if (i >= n) return;
    const float aii = float(dia[size_t(t.centre) * n + i]);
    int q = 0;
    for (int s = 0; s < t.K; ++s) {
        if (s == t.centre) continue;
        const double a = dia[size_t(s) * n + i];
        const int j = i + t.off[s];
        if (a != 0.0 && j >= 0 && j < n) {
            f[2 * q] = float(a) / aii;
            f[2 * q + 1] = logf(float(dia[size_t(t.centre) * n + j]) / aii);
        }
        ++q;
    }
}

// Stage W (rows x cols, FP32, row-major out x in) as a K-major BF16 tile.
__device__ void stage_weights(unsigned char* tile, const float* W, int rows, int cols) {
    for (int idx = threadIdx.x; idx < rows * (cols / 8); idx += blockDim.x) {
        const int r = idx / (cols / 8), c0 = (idx % (cols / 8)) * 8;
        float v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = W[r * cols + c0 + k];
        store8(tile, r, c0, rows, v);
    }
}

struct SpaiFwdArgs {
    const float* params;
    const double* dia;     // A by diagonal offsets
    const int* rp;         // A's CSR pattern (M shares it)
    const int* ci;
    SlotTable slots;
    int n;
    double* mval;          // M values on A's pattern (may be null)
    float* out;            // raw outputs [n][16] (may be null)
    int* status;
};

// Shared memory of the forward kernel (dynamic, 1024-byte aligned base).
constexpr int kFwdW1 = 0;                          // 64 x 16
constexpr int kFwdW2 = kFwdW1 + kH * kF * 2;       // 64 x 64
constexpr int kFwdW3 = kFwdW2 + kH * kH * 2;       // 16 x 64
constexpr int kFwdX = kFwdW3 + kO * kH * 2;        // 128 x 16
constexpr int kFwdH = kFwdX + kTileRows * kF * 2;  // 128 x 64
constexpr int kFwdBar = kFwdH + kTileRows * kH * 2;
// Requested dynamic shared memory: at most 4 CTAs per SM, so that their
// 4 x 128 tensor-memory columns fit the SM's 512.
constexpr int kFwdSmem = 56 * 1024;
static_assert(kFwdBar + 64 <= kFwdSmem, "forward shared memory");

// Forward pass: one CTA (4 warps, one row per thread) per 128-row tile,
// persistent over tiles.  TMEM: columns 0-63 layer-1 and layer-3
// accumulators, 64-127 layer 2.
__global__ void __launch_bounds__(kThreads, 1) k_spai_forward(SpaiFwdArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kFwdBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kFwdBar + 16);
    const uint32_t mbar = smem_u32(bar);
    stage_weights(smem + kFwdW1, a.params + kW1, kH, kF);
    stage_weights(smem + kFwdW2, a.params + kW2, kH, kH);
    stage_weights(smem + kFwdW3, a.params + kW3, kO, kH);
    if (tid == 0) mbar_init(mbar);
    if (warp == 0) tmem_alloc(smem_u32(tslot), 128);
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t lane_base = tmem + (uint32_t(warp * 32) << 16);
    const uint32_t sX = smem_u32(smem + kFwdX), sH = smem_u32(smem + kFwdH);
    const uint32_t sW1 = smem_u32(smem + kFwdW1), sW2 = smem_u32(smem + kFwdW2),
                   sW3 = smem_u32(smem + kFwdW3);
    const float* b1 = a.params + kB1;
    const float* b2 = a.params + kB2;
    const float* b3 = a.params + kB3;
    uint32_t phase = 0;
    bool ok = true;
    // Thread 0 issues the MMAs, and only while its own waits succeed, so at
    // most one committed phase is outstanding when a wait gives up.
    bool pend = false;
    uint32_t pend_parity = 0;
    auto wait_mma = [&]() {
        const bool got = ok && mbar_wait(mbar, phase);
        if (ok && !got) {
            pend = true;
            pend_parity = phase;
        }
        ok = got;
        phase ^= 1;
        fence_after_sync();
    };
    const int ntiles = (a.n + kTileRows - 1) / kTileRows;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int row = tile * kTileRows + tid;
        {
            float f[kF];
            row_features(a.dia, a.n, a.slots, row, f);
            store8(smem + kFwdX, tid, 0, kTileRows, f);
            store8(smem + kFwdX, tid, 8, kTileRows, f + 8);
        }
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        // Layer 1: Z1 = X W1^T  (M 128, N 64, K 16).
        if (tid == 0 && ok) {
            fence_after_sync();
            mma_bf16(tmem, desc_kmajor(sX, kTileRows, 0), desc_kmajor(sW1, kH, 0),
                     idesc_bf16(128, kH, 0, 0), 0);
            mma_commit(mbar);
        }
        wait_mma();
#pragma unroll 1
        for (int c = 0; c < kH; c += 16) {
            float z[16];
            tmem_ld16(lane_base + c, z);
#pragma unroll
            for (int k = 0; k < 16; ++k) z[k] = fmaxf(z[k] + b1[c + k], 0.f);
            store8(smem + kFwdH, tid, c, kTileRows, z);
            store8(smem + kFwdH, tid, c + 8, kTileRows, z + 8);
        }
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        // Layer 2: Z2 = H1 W2^T  (M 128, N 64, K 64).
        if (tid == 0 && ok) {
            fence_after_sync();
            for (int ks = 0; ks < kH / 16; ++ks)
                mma_bf16(tmem + 64, desc_kmajor(sH, kTileRows, ks), desc_kmajor(sW2, kH, ks),
                         idesc_bf16(128, kH, 0, 0), ks > 0);
            mma_commit(mbar);
        }
        wait_mma();
        // H2 overwrites H1: layer 2's operands are consumed (its MMAs are
        // complete once the barrier phase has flipped).
        float h2[kH];
#pragma unroll
        for (int c = 0; c < kH; c += 16) tmem_ld16(lane_base + 64 + c, h2 + c);
#pragma unroll
        for (int k = 0; k < kH; ++k) h2[k] = fmaxf(h2[k] + b2[k], 0.f);
#pragma unroll
        for (int c = 0; c < kH; c += 8) store8(smem + kFwdH, tid, c, kTileRows, h2 + c);
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        // Layer 3: out = H2 W3^T  (M 128, N 16, K 64).
        if (tid == 0 && ok) {
            fence_after_sync();
            for (int ks = 0; ks < kH / 16; ++ks)
                mma_bf16(tmem, desc_kmajor(sH, kTileRows, ks), desc_kmajor(sW3, kO, ks),
                         idesc_bf16(128, kO, 0, 0), ks > 0);
            mma_commit(mbar);
        }
        wait_mma();
        float o[kO];
        tmem_ld16(lane_base, o);
        fence_before_sync();
        // The next tile's layer 1 reuses these columns; a timed-out wait on
        // any thread ends the loop on all of them.
        ok = __syncthreads_and(ok);
        if (ok && row < a.n) {
#pragma unroll
            for (int k = 0; k < kO; ++k) o[k] += b3[k];
            if (a.out) {
                float4* dst = reinterpret_cast<float4*>(a.out + size_t(row) * kO);
#pragma unroll
                for (int k = 0; k < kO; k += 4) dst[k / 4] = make_float4(o[k], o[k + 1], o[k + 2], o[k + 3]);
            }
            if (a.mval) {
                const double inv = 1.0 / a.dia[size_t(a.slots.centre) * a.n + row];
                for (int p = a.rp[row]; p < a.rp[row + 1]; ++p) {
                    const int d = a.ci[p] - row;
                    double v = 0.0;
                    for (int s = 0; s < a.slots.K; ++s)
                        if (a.slots.off[s] == d) v = ((d == 0 ? 1.0 : 0.0) + double(o[s])) * inv;
                    a.mval[p] = v;
                }
            }
        }
    }
    if (!ok && tid == 0) atomicExch(a.status, MCLSGPU_ERR_TIMEOUT);
    if (tid == 0 && pend) mbar_drain(mbar, pend_parity);
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tmem, 128);
    }
}

struct SpaiBwdArgs {
    const float* params;
    const double* dia;
    SlotTable slots;
    int n;
    const float* G;        // dL/dout [n][16]
    float* grad;           // parameter gradient (accumulated)
    int* status;
};

// Shared memory of the backward kernel.  The H1 and X tiles carry an extra
// 8-column group whose first column is 1 and the rest 0, so that the
// weight-gradient products also produce the bias gradients of layers 2 and 1
// (sum over rows of dZ = dZ^T * ones).
constexpr int kXC = 24;   // X tile columns: 16 features + ones group
constexpr int kH1C = 72;  // H1 tile columns: 64 + ones group
constexpr int kBwW1 = 0;                                // 64 x 16
constexpr int kBwW2 = kBwW1 + kH * kF * 2;              // 64 x 64
constexpr int kBwW3 = kBwW2 + kH * kH * 2;              // 16 x 64
constexpr int kBwX = kBwW3 + kO * kH * 2;               // 128 x 24
constexpr int kBwH1 = kBwX + kTileRows * kXC * 2;       // 128 x 72
constexpr int kBwH2 = kBwH1 + kTileRows * kH1C * 2;     // 128 x 64
constexpr int kBwG = kBwH2 + kTileRows * kH * 2;        // 128 x 16
constexpr int kBwDZ2 = kBwG + kTileRows * kO * 2;       // 128 x 64
constexpr int kBwDZ1 = kBwDZ2 + kTileRows * kH * 2;     // 128 x 64
constexpr int kBwB3 = kBwDZ1 + kTileRows * kH * 2;      // 16 floats
constexpr int kBwBar = kBwB3 + 64;
// Requested dynamic shared memory: one CTA per SM, which allocates all 512
// tensor-memory columns.
constexpr int kBwSmem = 120 * 1024;
static_assert(kBwBar + 64 <= kBwSmem, "backward shared memory");
// TMEM columns of the backward kernel (512 allocated).
constexpr uint32_t kTA = 0;      // Z1, then dH2 (M 128 x 64)
constexpr uint32_t kTB = 64;     // Z2, then dH1 (M 128 x 64)
constexpr uint32_t kTdW3 = 256;  // dW3^T: rows h2, cols o     (M 64 x 16)
constexpr uint32_t kTdW2 = 288;  // dW2: rows h2, cols h1 | db2 (M 64 x 72)
constexpr uint32_t kTdW1 = 384;  // dW1: rows h1, cols in | db1 (M 64 x 24)

// Backward pass: the forward activations of each tile are recomputed, the
// output gradient G is propagated to dZ2 and dZ1, and the weight and bias
// gradients accumulate in TMEM across the CTA's tiles; at the end each CTA
// adds its sums into `grad`.
__global__ void __launch_bounds__(kThreads, 1) k_spai_backward(SpaiBwdArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kBwBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kBwBar + 16);
    float* db3 = reinterpret_cast<float*>(smem + kBwB3);
    const uint32_t mbar = smem_u32(bar);
    stage_weights(smem + kBwW1, a.params + kW1, kH, kF);
    stage_weights(smem + kBwW2, a.params + kW2, kH, kH);
    stage_weights(smem + kBwW3, a.params + kW3, kO, kH);
    if (tid < kO) db3[tid] = 0.f;
    {
        // Ones groups (column 16 of X, column 64 of H1) for every row.
        float one[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        store8(smem + kBwX, tid, 16, kTileRows, one);
        store8(smem + kBwH1, tid, 64, kTileRows, one);
    }
    if (tid == 0) mbar_init(mbar);
    if (warp == 0) tmem_alloc(smem_u32(tslot), 512);
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t lane_base = tmem + (uint32_t(warp * 32) << 16);
    const uint32_t sW1 = smem_u32(smem + kBwW1), sW2 = smem_u32(smem + kBwW2),
                   sW3 = smem_u32(smem + kBwW3), sX = smem_u32(smem + kBwX),
                   sH1 = smem_u32(smem + kBwH1), sH2 = smem_u32(smem + kBwH2),
                   sG = smem_u32(smem + kBwG), sDZ2 = smem_u32(smem + kBwDZ2),
                   sDZ1 = smem_u32(smem + kBwDZ1);
    const float* b1 = a.params + kB1;
    const float* b2 = a.params + kB2;
    uint32_t phase = 0;
    bool ok = true;
    int done = 0;
    // Thread 0 issues the MMAs only while its own waits succeed (at most one
    // committed phase outstanding when a wait gives up).
    bool pend = false;
    uint32_t pend_parity = 0;
    const int ntiles = (a.n + kTileRows - 1) / kTileRows;
    auto stage_sync = [&]() {
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
    };
    auto wait_mma = [&]() {
        const bool got = ok && mbar_wait(mbar, phase);
        if (ok && !got) {
            pend = true;
            pend_parity = phase;
        }
        ok = got;
        phase ^= 1;
        fence_after_sync();
    };
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++done) {
        const int row = tile * kTileRows + tid;
        {
            float f[kF];
            row_features(a.dia, a.n, a.slots, row, f);
            store8(smem + kBwX, tid, 0, kTileRows, f);
            store8(smem + kBwX, tid, 8, kTileRows, f + 8);
        }
        stage_sync();
        if (tid == 0 && ok) {
            fence_after_sync();
            mma_bf16(tmem + kTA, desc_kmajor(sX, kTileRows, 0), desc_kmajor(sW1, kH, 0),
                     idesc_bf16(128, kH, 0, 0), 0);
            mma_commit(mbar);
        }
        wait_mma();
#pragma unroll 1
        for (int c = 0; c < kH; c += 16) {
            float z[16];
            tmem_ld16(lane_base + kTA + c, z);
#pragma unroll
            for (int k = 0; k < 16; ++k) z[k] = fmaxf(z[k] + b1[c + k], 0.f);
            store8(smem + kBwH1, tid, c, kTileRows, z);
            store8(smem + kBwH1, tid, c + 8, kTileRows, z + 8);
        }
        stage_sync();
        if (tid == 0 && ok) {
            fence_after_sync();
            for (int ks = 0; ks < kH / 16; ++ks)
                mma_bf16(tmem + kTB, desc_kmajor(sH1, kTileRows, ks), desc_kmajor(sW2, kH, ks),
                         idesc_bf16(128, kH, 0, 0), ks > 0);
            mma_commit(mbar);
        }
        wait_mma();
#pragma unroll 1
        for (int c = 0; c < kH; c += 16) {
            float z[16];
            tmem_ld16(lane_base + kTB + c, z);
#pragma unroll
            for (int k = 0; k < 16; ++k) z[k] = fmaxf(z[k] + b2[c + k], 0.f);
            store8(smem + kBwH2, tid, c, kTileRows, z);
            store8(smem + kBwH2, tid, c + 8, kTileRows, z + 8);
        }
        {
            float g[kO];
#pragma unroll
            for (int k = 0; k < kO; ++k) g[k] = 0.f;
            if (row < a.n) {
                const float4* src = reinterpret_cast<const float4*>(a.G + size_t(row) * kO);
#pragma unroll
                for (int k = 0; k < kO; k += 4) {
                    const float4 q = src[k / 4];
                    g[k] = q.x;
                    g[k + 1] = q.y;
                    g[k + 2] = q.z;
                    g[k + 3] = q.w;
                }
            }
            store8(smem + kBwG, tid, 0, kTileRows, g);
            store8(smem + kBwG, tid, 8, kTileRows, g + 8);
            // db3: sum over rows of the BF16-rounded G.
#pragma unroll
            for (int k = 0; k < kO; ++k) {
                float s = bf16_round(g[k]);
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
                if (lane == 0) atomicAdd(&db3[k], s);
            }
        }
        stage_sync();
        // dH2 = G W3 (B = W3 read MN-major: N 64 = h2, K 16 = o) and
        // dW3^T += H2^T G (A = H2 MN-major, B = G MN-major; K = 128 rows).
        if (tid == 0 && ok) {
            fence_after_sync();
            mma_bf16(tmem + kTA, desc_kmajor(sG, kTileRows, 0), desc_mnmajor(sW3, kO, 0),
                     idesc_bf16(128, kH, 0, 1), 0);
            for (int ks = 0; ks < kTileRows / 16; ++ks)
                mma_bf16(tmem + kTdW3, desc_mnmajor(sH2, kTileRows, ks),
                         desc_mnmajor(sG, kTileRows, ks), idesc_bf16(64, kO, 1, 1),
                         (done > 0 || ks > 0));
            mma_commit(mbar);
        }
        wait_mma();
#pragma unroll 1
        for (int c = 0; c < kH; c += 16) {
            float d[16], h[16];
            tmem_ld16(lane_base + kTA + c, d);
            load8(smem + kBwH2, tid, c, kTileRows, h);
            load8(smem + kBwH2, tid, c + 8, kTileRows, h + 8);
#pragma unroll
            for (int k = 0; k < 16; ++k) d[k] = h[k] > 0.f ? d[k] : 0.f;
            store8(smem + kBwDZ2, tid, c, kTileRows, d);
            store8(smem + kBwDZ2, tid, c + 8, kTileRows, d + 8);
        }
        stage_sync();
        // dH1 = dZ2 W2 (B = W2 MN-major: N 64 = h1, K 64 = h2) and
        // [dW2 | db2] += dZ2^T [H1 | 1] (K = 128 rows).
        if (tid == 0 && ok) {
            fence_after_sync();
            for (int ks = 0; ks < kH / 16; ++ks)
                mma_bf16(tmem + kTB, desc_kmajor(sDZ2, kTileRows, ks), desc_mnmajor(sW2, kH, ks),
                         idesc_bf16(128, kH, 0, 1), ks > 0);
            for (int ks = 0; ks < kTileRows / 16; ++ks)
                mma_bf16(tmem + kTdW2, desc_mnmajor(sDZ2, kTileRows, ks),
                         desc_mnmajor(sH1, kTileRows, ks), idesc_bf16(64, kH1C, 1, 1),
                         (done > 0 || ks > 0));
            mma_commit(mbar);
        }
        wait_mma();
#pragma unroll 1
        for (int c = 0; c < kH; c += 16) {
            float d[16], h[16];
            tmem_ld16(lane_base + kTB + c, d);
            load8(smem + kBwH1, tid, c, kTileRows, h);
            load8(smem + kBwH1, tid, c + 8, kTileRows, h + 8);
#pragma unroll
            for (int k = 0; k < 16; ++k) d[k] = h[k] > 0.f ? d[k] : 0.f;
            store8(smem + kBwDZ1, tid, c, kTileRows, d);
            store8(smem + kBwDZ1, tid, c + 8, kTileRows, d + 8);
        }
        stage_sync();
        // [dW1 | db1] += dZ1^T [X | 1] (K = 128 rows).
        if (tid == 0 && ok) {
            fence_after_sync();
            for (int ks = 0; ks < kTileRows / 16; ++ks)
                mma_bf16(tmem + kTdW1, desc_mnmajor(sDZ1, kTileRows, ks),
                         desc_mnmajor(sX, kTileRows, ks), idesc_bf16(64, kXC, 1, 1),
                         (done > 0 || ks > 0));
            mma_commit(mbar);
        }
        wait_mma();
        fence_before_sync();
        // TMEM columns A/B and every tile are reused next; a timed-out wait
        // on any thread ends the loop on all of them.
        ok = __syncthreads_and(ok);
    }
    if (!ok && tid == 0) atomicExch(a.status, MCLSGPU_ERR_TIMEOUT);
    if (tid == 0 && pend) mbar_drain(mbar, pend_parity);
    if (ok && done > 0) {
        fence_after_sync();
        // M = 64 accumulators: row 16w + t of the product sits in lane
        // 32w + t (t < 16) of TMEM.
        const int r = 16 * warp + lane;
        float v[16];
        tmem_ld16(lane_base + kTdW3, v);
        if (lane < 16)
            for (int o = 0; o < kO; ++o) atomicAdd(&a.grad[kW3 + o * kH + r], v[o]);
        for (int c = 0; c < 80; c += 16) {
            tmem_ld16(lane_base + kTdW2 + c, v);
            if (lane < 16)
                for (int k = 0; k < 16; ++k) {
                    if (c + k < kH) atomicAdd(&a.grad[kW2 + r * kH + c + k], v[k]);
                    else if (c + k == kH) atomicAdd(&a.grad[kB2 + r], v[k]);
                }
        }
        for (int c = 0; c < 32; c += 16) {
            tmem_ld16(lane_base + kTdW1 + c, v);
            if (lane < 16)
                for (int k = 0; k < 16; ++k) {
                    if (c + k < kF) atomicAdd(&a.grad[kW1 + r * kF + c + k], v[k]);
                    else if (c + k == kF) atomicAdd(&a.grad[kB1 + r], v[k]);
                }
        }
        __syncthreads();
        if (tid < kO) atomicAdd(&a.grad[kB3 + tid], db3[tid]);
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tmem, 512);
    }
}

// e_v = v - M (A v) per row; loss and the output gradient G.  With
// pen_w > 0 the loss adds pen_w/n * sum_i max(0, W_i - pen_c)^2, W_i the
// row sum of |H| for H = I - M A (the factor by which a forward walk's
// weight grows at state i), computed from row i of M and the rows of A at
// its neighbours.
__global__ void k_spai_loss_grad(int n, int nvec, const int* rp, const int* ci, const double* mval,
                                 const double* dia, SlotTable slots, const double* V,
                                 const double* Z, const double* wv, double pen_w, double pen_c,
                                 float* G, double* loss) {
    double part = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double inv = 1.0 / dia[size_t(slots.centre) * n + i];
        double g[kO];
#pragma unroll
        for (int k = 0; k < kO; ++k) g[k] = 0.0;
        if (pen_w > 0.0) {
            double m[kMaxSlots];
            bool has[kMaxSlots];
            for (int s = 0; s < kMaxSlots; ++s) {
                m[s] = 0.0;
                has[s] = false;
            }
            for (int p = rp[i]; p < rp[i + 1]; ++p) {
                const int d = ci[p] - i;
                for (int s = 0; s < slots.K; ++s)
                    if (slots.off[s] == d) {
                        m[s] = mval[p];
                        has[s] = true;
                    }
            }
            double h[kMaxSlots * kMaxSlots];
            for (int q = 0; q < slots.npair; ++q) h[q] = 0.0;
            h[slots.pcentre] = 1.0;
            for (int s = 0; s < slots.K; ++s) {
                const int k = i + slots.off[s];
                if (!has[s] || k < 0 || k >= n) continue;
                for (int t = 0; t < slots.K; ++t)
                    h[slots.pair[s][t]] -= m[s] * dia[size_t(t) * n + k];
            }
            double W = 0.0;
            for (int q = 0; q < slots.npair; ++q) W += fabs(h[q]);
            const double pen = W - pen_c;
            if (pen > 0.0) {
                part += pen_w * pen * pen / double(n);
                const double coef = 2.0 * pen_w * pen / double(n) * inv;
                for (int s = 0; s < slots.K; ++s) {
                    const int k = i + slots.off[s];
                    if (!has[s] || k < 0 || k >= n) continue;
                    double dW = 0.0;
                    for (int t = 0; t < slots.K; ++t) {
                        const double hv = h[slots.pair[s][t]];
                        const double sg = hv > 0.0 ? 1.0 : (hv < 0.0 ? -1.0 : 0.0);
                        dW -= sg * dia[size_t(t) * n + k];
                    }
                    g[s] += coef * dW;
                }
            }
        }
        for (int v = 0; v < nvec; ++v) {
            const double* z = Z + size_t(v) * n;
            double mz = 0.0;
            for (int p = rp[i]; p < rp[i + 1]; ++p) mz += mval[p] * z[ci[p]];
            const double e = V[size_t(v) * n + i] - mz;
            part += e * e * wv[v];
            const double c = -2.0 * e * wv[v] * inv;
            for (int p = rp[i]; p < rp[i + 1]; ++p) {
                const int d = ci[p] - i;
                for (int s = 0; s < slots.K; ++s)
                    if (slots.off[s] == d) g[s] += c * z[ci[p]];
            }
        }
        float4* dst = reinterpret_cast<float4*>(G + size_t(i) * kO);
#pragma unroll
        for (int k = 0; k < kO; k += 4)
            dst[k / 4] = make_float4(float(g[k]), float(g[k + 1]), float(g[k + 2]), float(g[k + 3]));
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) part += __shfl_xor_sync(0xffffffffu, part, d);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, part);
}

// wv[v] = 1 / (nvec * |v|^2) from the per-vector sums of squares.
__global__ void k_spai_weights(const double* sq, int nvec, double* wv) {
    const int v = threadIdx.x;
    if (v < nvec) wv[v] = sq[v] > 0.0 ? 1.0 / (double(nvec) * sq[v]) : 0.0;
}

__global__ void k_adam(float* p, float* m, float* v, const float* g, int count, float lr,
                       float b1, float b2, float eps, float c1, float c2, float clip) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float gi = g[i];
    if (clip > 0.f) gi = fminf(fmaxf(gi, -clip), clip);
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// y = v - M (A v) for the power iteration on H = I - M A.
__global__ void k_sub(int n, const double* v, const double* u, double* y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] = v[i] - u[i];
}
__global__ void k_scale_by_norm(int n, double* v, const double* sq) {
    const double s = *sq > 0.0 ? 1.0 / sqrt(*sq) : 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v[i] *= s;
}

inline int grid_for(long long work, int threads = 256, int cap = 148 * 16) {
    long long g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    return int(g > cap ? cap : g);
}

}  // namespace
}  // namespace mclsgpu

struct mclsgpu_spai {
    mclsgpu_context* ctx = nullptr;
    int slots = 0;
    float* params = nullptr;  // FP32 master parameters
    float* grad = nullptr;
    float* m = nullptr;       // Adam moments
    float* v = nullptr;
    long long step = 0;
    double pen_w = 0.0;       // row-sum penalty weight (0 = off)
    double pen_c = 1.0;       // row-sum threshold
};

namespace mclsgpu {
namespace {

// Slot table of an operator stored by diagonal offsets.
int slot_table(mclsgpu_context* ctx, const mclsgpu_operator* op, int want, SlotTable& t) {
    if (op->dia_k <= 0 || !op->dia_val)
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                         "learned SPAI needs an operator with a fixed stencil (diagonal-offset "
                         "storage)");
    if (op->dia_k > kMaxSlots)
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                         "learned SPAI: %d stencil offsets, at most %d supported", op->dia_k,
                         kMaxSlots);
    if (want > 0 && op->dia_k != want)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                         "learned SPAI network has %d slots, operator has %d stencil offsets",
                         want, op->dia_k);
    t.K = op->dia_k;
    t.centre = -1;
    for (int s = 0; s < t.K; ++s) {
        t.off[s] = op->dia_off[s];
        if (op->dia_off[s] == 0) t.centre = s;
    }
    for (int s = t.K; s < kMaxSlots; ++s) t.off[s] = 0x7fffffff;
    if (t.centre < 0)
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "learned SPAI: operator has no diagonal");
    std::vector<int> sums;
    for (int a = 0; a < t.K; ++a)
        for (int b = 0; b < t.K; ++b) sums.push_back(t.off[a] + t.off[b]);
    std::sort(sums.begin(), sums.end());
    sums.erase(std::unique(sums.begin(), sums.end()), sums.end());
    t.npair = int(sums.size());
    std::memset(t.pair, 0, sizeof(t.pair));
    for (int a = 0; a < t.K; ++a)
        for (int b = 0; b < t.K; ++b)
            t.pair[a][b] = (unsigned char)(std::lower_bound(sums.begin(), sums.end(),
                                                            t.off[a] + t.off[b]) -
                                           sums.begin());
    t.pcentre = int(std::lower_bound(sums.begin(), sums.end(), 0) - sums.begin());
    return MCLSGPU_OK;
}

// The kernels' dynamic shared memory exceeds the 48 KB default: opt in once
// per device (the attribute belongs to the device's context).
std::mutex g_attr_mutex;
bool g_attr_set[64] = {false};

int set_smem_attributes(mclsgpu_context* ctx) {
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    const int d = ctx->device;
    if (d >= 0 && d < 64 && g_attr_set[d]) return MCLSGPU_OK;
    cudaError_t e = cudaFuncSetAttribute(k_spai_forward,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_spai_backward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kBwSmem);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "spai shared-memory opt-in");
    if (d >= 0 && d < 64) g_attr_set[d] = true;
    return MCLSGPU_OK;
}

int launch_forward(mclsgpu_spai* net, mclsgpu_operator* op, const SlotTable& t, double* mval,
                   float* out) {
    mclsgpu_context* ctx = net->ctx;
    int rc = set_smem_attributes(ctx);
    if (rc) return rc;
    SpaiFwdArgs a{};
    a.params = net->params;
    a.dia = op->dia_val;
    a.rp = op->A.rp;
    a.ci = op->A.ci;
    a.slots = t;
    a.n = op->A.n;
    a.mval = mval;
    a.out = out;
    a.status = ctx->d_status;
    const int ntiles = (op->A.n + kTileRows - 1) / kTileRows;
    // Up to 4 CTAs per SM (4 x 128 TMEM columns).
    const int grid = ntiles < ctx->num_sms * 4 ? ntiles : ctx->num_sms * 4;
    k_spai_forward<<<grid, kThreads, kFwdSmem, ctx->stream>>>(a);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(ctx, e, "spai forward launch");
}

// Scratch for the loss/gradient pass.
struct GradScratch {
    double* mval = nullptr;
    double* Z = nullptr;
    double* sq = nullptr;
    double* wv = nullptr;
    double* part = nullptr;
    double* loss = nullptr;
    float* G = nullptr;
    void release() {
        dfree(mval);
        dfree(Z);
        dfree(sq);
        dfree(wv);
        dfree(part);
        dfree(loss);
        dfree(G);
    }
};

// Zero the gradient, then loss + gradient of the parameters on (op, V).
int gradient(mclsgpu_spai* net, mclsgpu_operator* op, const double* V, int nvec, double* loss_out) {
    mclsgpu_context* ctx = net->ctx;
    cudaStream_t s = ctx->stream;
    SlotTable t;
    int rc = slot_table(ctx, op, net->slots, t);
    if (rc) return rc;
    if (nvec < 1 || nvec > 1024)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "spai gradient: 1..1024 vectors");
    const int n = op->A.n;
    GradScratch g;
    cudaError_t e;
    if ((e = dmalloc(&g.mval, size_t(op->A.nnz))) != cudaSuccess ||
        (e = dmalloc(&g.Z, size_t(n) * nvec)) != cudaSuccess ||
        (e = dmalloc(&g.sq, size_t(nvec))) != cudaSuccess ||
        (e = dmalloc(&g.wv, size_t(nvec))) != cudaSuccess ||
        (e = dmalloc(&g.part, size_t(scan_partials_needed(n)))) != cudaSuccess ||
        (e = dmalloc(&g.loss, 1)) != cudaSuccess ||
        (e = dmalloc(&g.G, size_t(n) * kO)) != cudaSuccess) {
        g.release();
        return cuda_fail(ctx, e, "cudaMalloc");
    }
    cudaMemsetAsync(net->grad, 0, sizeof(float) * kParams, s);
    cudaMemsetAsync(g.loss, 0, sizeof(double), s);
    rc = launch_forward(net, op, t, g.mval, nullptr);
    if (!rc) {
        for (int v = 0; v < nvec; ++v) {
            spmv(s, op->A, V + size_t(v) * n, g.Z + size_t(v) * n);
            sum_sq(s, V + size_t(v) * n, n, g.part, g.sq + v);
        }
        k_spai_weights<<<1, 1024, 0, s>>>(g.sq, nvec, g.wv);
        k_spai_loss_grad<<<grid_for(n), 256, 0, s>>>(n, nvec, op->A.rp, op->A.ci, g.mval,
                                                     op->dia_val, t, V, g.Z, g.wv, net->pen_w,
                                                     net->pen_c, g.G, g.loss);
        SpaiBwdArgs b{};
        b.params = net->params;
        b.dia = op->dia_val;
        b.slots = t;
        b.n = n;
        b.G = g.G;
        b.grad = net->grad;
        b.status = ctx->d_status;
        const int ntiles = (n + kTileRows - 1) / kTileRows;
        const int grid = ntiles < ctx->num_sms ? ntiles : ctx->num_sms;
        k_spai_backward<<<grid, kThreads, kBwSmem, s>>>(b);
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "spai backward launch");
    }
    if (!rc) {
        double l = 0.0;
        e = cudaMemcpyAsync(&l, g.loss, sizeof(double), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "spai gradient");
        if (!rc) rc = check_device_status(ctx);
        if (loss_out) *loss_out = l;
    }
    g.release();
    return rc;
}

// Power-iteration estimate of rho(I - M A) (M as CSR on any pattern).
int rho_estimate(mclsgpu_context* ctx, const DevCsr& A, const DevCsr& M, int iters, uint64_t seed,
                 double* rho) {
    const int n = A.n;
    cudaStream_t s = ctx->stream;
    double *v = nullptr, *w = nullptr, *u = nullptr, *part = nullptr, *sq = nullptr;
    cudaError_t e;
    if ((e = dmalloc(&v, n)) != cudaSuccess || (e = dmalloc(&w, n)) != cudaSuccess ||
        (e = dmalloc(&u, n)) != cudaSuccess ||
        (e = dmalloc(&part, size_t(scan_partials_needed(n)))) != cudaSuccess ||
        (e = dmalloc(&sq, size_t(iters + 1))) != cudaSuccess) {
        dfree(v); dfree(w); dfree(u); dfree(part); dfree(sq);
        return cuda_fail(ctx, e, "cudaMalloc");
    }
    std::vector<double> h(n);
    std::mt19937_64 gen(seed);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    for (int i = 0; i < n; ++i) h[i] = U(gen);
    cudaMemcpyAsync(v, h.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s);
    sum_sq(s, v, n, part, sq);
    k_scale_by_norm<<<grid_for(n), 256, 0, s>>>(n, v, sq);
    for (int k = 0; k < iters; ++k) {
        spmv(s, A, v, w);
        spmv(s, M, w, u);
        k_sub<<<grid_for(n), 256, 0, s>>>(n, v, u, w);
        sum_sq(s, w, n, part, sq + 1 + k);
        k_scale_by_norm<<<grid_for(n), 256, 0, s>>>(n, w, sq + 1 + k);
        std::swap(v, w);
    }
    std::vector<double> hs(iters + 1);
    cudaMemcpyAsync(hs.data(), sq, sizeof(double) * (iters + 1), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    dfree(v); dfree(w); dfree(u); dfree(part); dfree(sq);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "power iteration");
    // Geometric mean of the last growth factors.
    const int tail = iters < 10 ? iters : 10;
    double lg = 0.0;
    for (int k = iters - tail; k < iters; ++k) lg += 0.5 * std::log(hs[1 + k]);
    *rho = std::exp(lg / tail);
    return MCLSGPU_OK;
}

}  // namespace

// LEARNED_SPAI preconditioner: M from the network on A's pattern, then the
// spectral-radius gate.  The learned M is kept unless rho(I - M A) reaches
// both `rho_fallback` and the point-Jacobi rho, in which case (or when the
// operator has no fixed stencil) point Jacobi is built instead and
// `fallback` is set.
int spai_build(mclsgpu_context* ctx, mclsgpu_operator* op, const mclsgpu_precond_params* p,
               mclsgpu_precond* pc) {
    mclsgpu_spai* net = static_cast<mclsgpu_spai*>(const_cast<void*>(p->spai_net));
    const double thresh = p->rho_fallback > 0.0 ? p->rho_fallback : 0.95;
    SlotTable t;
    int rc = MCLSGPU_OK;
    const bool usable = net && net->ctx == ctx && slot_table(ctx, op, net->slots, t) == MCLSGPU_OK;
    // Point Jacobi: the fallback and the gate's yardstick.
    DevCsr J;
    double* dinv = nullptr;
    cudaError_t e;
    if ((e = dmalloc(&dinv, op->A.n)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    rc = reciprocal_diagonal(ctx, op->A, dinv);
    if (!rc) rc = point_jacobi_csr(ctx, op->A.n, dinv, J);
    if (rc) {
        dfree(dinv);
        J.release();
        return rc;
    }
    double rho_j = 1.0, rho_l = 1.0;
    bool keep = false;
    if (usable) {
        rc = csr_copy(ctx, op->A, pc->P);
        if (!rc) rc = launch_forward(net, op, t, pc->P.v, nullptr);
        if (!rc) {
            e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) rc = cuda_fail(ctx, e, "spai inference");
        }
        if (!rc) rc = check_device_status(ctx);
        if (!rc) rc = rho_estimate(ctx, op->A, pc->P, 200, 0x5eed5eedull, &rho_l);
        if (!rc) rc = rho_estimate(ctx, op->A, J, 200, 0x5eed5eedull, &rho_j);
        if (rc) {
            dfree(dinv);
            J.release();
            pc->P.release();
            return rc;
        }
        keep = std::isfinite(rho_l) && !(rho_l >= thresh && rho_l >= rho_j);
    }
    if (keep) {
        J.release();
        dfree(dinv);
        // M on A's diagonals too, for the fused MCSA iteration.
        rc = csr_to_dia(ctx, pc->P, op->dia_k, op->dia_off, &pc->mdia);
        if (rc) {
            pc->P.release();
            return rc;
        }
        pc->kind = MCLSGPU_PREC_LEARNED_SPAI;
        pc->rho = rho_l;
        pc->fallback = 0;
    } else {
        pc->P.release();
        pc->P = J;
        pc->diag = dinv;
        pc->kind = MCLSGPU_PREC_POINT_JACOBI;
        pc->rho = usable ? rho_l : -1.0;
        pc->fallback = 1;
    }
    return MCLSGPU_OK;
}

}  // namespace mclsgpu

using namespace mclsgpu;

extern "C" {

int mclsgpu_set_wait_limit(mclsgpu_context* ctx, int32_t polls) {
    if (!ctx) return MCLSGPU_ERR_INVALID_ARG;
    const int v = polls < 0 ? kDefaultWaitPolls : polls;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess)
        e = cudaMemcpyToSymbolAsync(g_wait_polls, &v, sizeof(int), 0, cudaMemcpyHostToDevice,
                                    ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(ctx, e, "set wait limit");
}

int mclsgpu_spai_num_params(void) { return kParams; }

int mclsgpu_spai_create(mclsgpu_context* ctx, int slots, uint64_t seed, mclsgpu_spai** out) {
    if (!ctx || !out) return MCLSGPU_ERR_INVALID_ARG;
    *out = nullptr;
    if (slots < 3 || slots > kMaxSlots)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "spai: 3..%d stencil slots", kMaxSlots);
    mclsgpu_spai* net = new mclsgpu_spai;
    net->ctx = ctx;
    net->slots = slots;
    cudaError_t e;
    if ((e = dmalloc(&net->params, kParams)) != cudaSuccess ||
        (e = dmalloc(&net->grad, kParams)) != cudaSuccess ||
        (e = dmalloc(&net->m, kParams)) != cudaSuccess ||
        (e = dmalloc(&net->v, kParams)) != cudaSuccess) {
        dfree(net->params); dfree(net->grad); dfree(net->m); dfree(net->v);
        delete net;
        return cuda_fail(ctx, e, "cudaMalloc");
    }
    // He-uniform hidden layers, zero biases, zero output layer (= Jacobi).
    std::vector<float> h(kParams, 0.f);
    std::mt19937_64 gen(seed);
    std::uniform_real_distribution<float> U(-1.f, 1.f);
    const float a1 = std::sqrt(6.f / kF), a2 = std::sqrt(6.f / kH);
    for (int i = 0; i < kH * kF; ++i) h[kW1 + i] = a1 * U(gen);
    for (int i = 0; i < kH * kH; ++i) h[kW2 + i] = a2 * U(gen);
    cudaMemcpyAsync(net->params, h.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice,
                    ctx->stream);
    cudaMemsetAsync(net->m, 0, sizeof(float) * kParams, ctx->stream);
    cudaMemsetAsync(net->v, 0, sizeof(float) * kParams, ctx->stream);
    cudaMemsetAsync(net->grad, 0, sizeof(float) * kParams, ctx->stream);
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        dfree(net->params); dfree(net->grad); dfree(net->m); dfree(net->v);
        delete net;
        return cuda_fail(ctx, e, "spai create");
    }
    *out = net;
    return MCLSGPU_OK;
}

int mclsgpu_spai_destroy(mclsgpu_spai* net) {
    if (!net) return MCLSGPU_OK;
    dfree(net->params);
    dfree(net->grad);
    dfree(net->m);
    dfree(net->v);
    delete net;
    return MCLSGPU_OK;
}

int mclsgpu_spai_set_penalty(mclsgpu_spai* net, double weight, double threshold) {
    if (!net || !(weight >= 0.0) || !(threshold > 0.0)) return MCLSGPU_ERR_INVALID_ARG;
    net->pen_w = weight;
    net->pen_c = threshold;
    return MCLSGPU_OK;
}

int mclsgpu_spai_get_params(mclsgpu_spai* net, float* host) {
    if (!net || !host) return MCLSGPU_ERR_INVALID_ARG;
    cudaError_t e = cudaMemcpyAsync(host, net->params, sizeof(float) * kParams,
                                    cudaMemcpyDeviceToHost, net->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(net->ctx->stream);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(net->ctx, e, "spai get params");
}

int mclsgpu_spai_set_params(mclsgpu_spai* net, const float* host) {
    if (!net || !host) return MCLSGPU_ERR_INVALID_ARG;
    cudaError_t e = cudaMemcpyAsync(net->params, host, sizeof(float) * kParams,
                                    cudaMemcpyHostToDevice, net->ctx->stream);
    cudaMemsetAsync(net->m, 0, sizeof(float) * kParams, net->ctx->stream);
    cudaMemsetAsync(net->v, 0, sizeof(float) * kParams, net->ctx->stream);
    net->step = 0;
    if (e == cudaSuccess) e = cudaStreamSynchronize(net->ctx->stream);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(net->ctx, e, "spai set params");
}

int mclsgpu_spai_infer(mclsgpu_spai* net, mclsgpu_operator* op, float* out, double* mvals) {
    if (!net || !op || (!out && !mvals)) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = net->ctx;
    SlotTable t;
    int rc = slot_table(ctx, op, net->slots, t);
    if (rc) return rc;
    const int n = op->A.n;
    float* dout = nullptr;
    double* dm = nullptr;
    cudaError_t e;
    if ((e = dmalloc(&dout, size_t(n) * kO)) != cudaSuccess ||
        (e = dmalloc(&dm, size_t(op->A.nnz))) != cudaSuccess) {
        dfree(dout);
        return cuda_fail(ctx, e, "cudaMalloc");
    }
    rc = launch_forward(net, op, t, dm, dout);
    if (!rc) {
        if (out)
            cudaMemcpyAsync(out, dout, sizeof(float) * n * kO, cudaMemcpyDeviceToHost, ctx->stream);
        if (mvals)
            cudaMemcpyAsync(mvals, dm, sizeof(double) * op->A.nnz, cudaMemcpyDeviceToHost,
                            ctx->stream);
        e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "spai infer");
        if (!rc) rc = check_device_status(ctx);
    }
    dfree(dout);
    dfree(dm);
    return rc;
}

int mclsgpu_spai_infer_dev(mclsgpu_spai* net, mclsgpu_operator* op, float* out_dev,
                           double* mvals_dev, float* ms) {
    if (!net || !op || (!out_dev && !mvals_dev)) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = net->ctx;
    SlotTable t;
    int rc = slot_table(ctx, op, net->slots, t);
    if (rc) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ms) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, ctx->stream);
    }
    rc = launch_forward(net, op, t, mvals_dev, out_dev);
    if (ms) cudaEventRecord(e1, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (!rc && e != cudaSuccess) rc = cuda_fail(ctx, e, "spai infer");
    if (ms) {
        *ms = 0.f;
        if (!rc) cudaEventElapsedTime(ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (!rc) rc = check_device_status(ctx);
    return rc;
}

int mclsgpu_spai_gradient(mclsgpu_spai* net, mclsgpu_operator* op, const double* v_dev, int nvec,
                          double* loss, float* grad) {
    if (!net || !op || !v_dev) return MCLSGPU_ERR_INVALID_ARG;
    int rc = gradient(net, op, v_dev, nvec, loss);
    if (rc || !grad) return rc;
    cudaError_t e = cudaMemcpyAsync(grad, net->grad, sizeof(float) * kParams,
                                    cudaMemcpyDeviceToHost, net->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(net->ctx->stream);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(net->ctx, e, "spai gradient copy");
}

int mclsgpu_spai_train_step(mclsgpu_spai* net, mclsgpu_operator* op, const double* v_dev, int nvec,
                            const mclsgpu_spai_adam* opt, double* loss) {
    if (!net || !op || !v_dev || !opt) return MCLSGPU_ERR_INVALID_ARG;
    if (opt->size < sizeof(mclsgpu_spai_adam))
        return set_error(net->ctx, MCLSGPU_ERR_INVALID_ARG, "adam params: size mismatch");
    int rc = gradient(net, op, v_dev, nvec, loss);
    if (rc) return rc;
    ++net->step;
    const float c1 = 1.f - std::pow(float(opt->beta1), float(net->step));
    const float c2 = 1.f - std::pow(float(opt->beta2), float(net->step));
    k_adam<<<(kParams + 255) / 256, 256, 0, net->ctx->stream>>>(
        net->params, net->m, net->v, net->grad, kParams, float(opt->lr), float(opt->beta1),
        float(opt->beta2), float(opt->eps), c1, c2, float(opt->grad_clip));
    cudaError_t e = cudaStreamSynchronize(net->ctx->stream);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(net->ctx, e, "spai adam");
}

int mclsgpu_spai_smooth_vectors(mclsgpu_spai* net, mclsgpu_operator* op, double* v_dev, int nvec,
                                int iters) {
    if (!net || !op || !v_dev || nvec < 1 || iters < 0) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = net->ctx;
    cudaStream_t s = ctx->stream;
    SlotTable t;
    int rc = slot_table(ctx, op, net->slots, t);
    if (rc) return rc;
    const int n = op->A.n;
    DevCsr M;
    double *w = nullptr, *u = nullptr, *part = nullptr, *sq = nullptr;
    cudaError_t e;
    if ((e = dmalloc(&w, n)) != cudaSuccess || (e = dmalloc(&u, n)) != cudaSuccess ||
        (e = dmalloc(&part, size_t(scan_partials_needed(n)))) != cudaSuccess ||
        (e = dmalloc(&sq, 1)) != cudaSuccess) {
        dfree(w); dfree(u); dfree(part); dfree(sq);
        return cuda_fail(ctx, e, "cudaMalloc");
    }
    rc = csr_copy(ctx, op->A, M);
    if (!rc) rc = launch_forward(net, op, t, M.v, nullptr);
    if (!rc) {
        for (int k = 0; k < nvec; ++k) {
            double* v = v_dev + size_t(k) * n;
            for (int it = 0; it < iters; ++it) {
                spmv(s, op->A, v, w);
                spmv(s, M, w, u);
                k_sub<<<grid_for(n), 256, 0, s>>>(n, v, u, v);
                sum_sq(s, v, n, part, sq);
                k_scale_by_norm<<<grid_for(n), 256, 0, s>>>(n, v, sq);
            }
        }
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "spai smooth vectors");
    }
    M.release();
    dfree(w); dfree(u); dfree(part); dfree(sq);
    return rc;
}

int mclsgpu_spai_rho(mclsgpu_spai* net, mclsgpu_operator* op, int iters, double* rho_learned,
                     double* rho_jacobi) {
    if (!net || !op) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = net->ctx;
    SlotTable t;
    int rc = slot_table(ctx, op, net->slots, t);
    if (rc) return rc;
    DevCsr M, J;
    double* dinv = nullptr;
    cudaError_t e = dmalloc(&dinv, op->A.n);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    rc = csr_copy(ctx, op->A, M);
    if (!rc) rc = launch_forward(net, op, t, M.v, nullptr);
    if (!rc && rho_learned) rc = rho_estimate(ctx, op->A, M, iters, 0x5eed5eedull, rho_learned);
    if (!rc && rho_jacobi) {
        rc = reciprocal_diagonal(ctx, op->A, dinv);
        if (!rc) rc = point_jacobi_csr(ctx, op->A.n, dinv, J);
        if (!rc) rc = rho_estimate(ctx, op->A, J, iters, 0x5eed5eedull, rho_jacobi);
    }
    M.release();
    J.release();
    dfree(dinv);
    return rc;
}

}  // extern "C"
