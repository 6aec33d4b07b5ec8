// domain.cu -- device build of the Monte Carlo domain.
//
// Restates AlmostOptimalDomain::addMatrixToDomain
// (src/MCLS_AlmostOptimalDomain_impl.hpp:257-366) as two passes over the
// composite operator's rows: count the retained entries, then write the signed
// iteration-matrix values h, the normalised CDF of |h| and the row weight
// W = sum |h|.  FP64 arithmetic uses explicitly rounded operations so that
// no multiply-add contraction changes the reference's rounding.  A third pass
// packs the FP32 walk records: one fixed-stride record per row,
//   slot 0:      { W (float bits), row length }
//   slot 1..K:   { cdf_j (float bits), col_j | (h_j <= 0) << 31 }
//   padding:     { 2.0f, 0 }  (never selected: every uniform is < 1)
// so that one walk step reads exactly one contiguous record.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <vector>

#include "internal.h"

namespace mclsgpu {
int exclusive_scan_counts_dev(mclsgpu_context* ctx, const int* d_cnt, int n, int* d_rp,
                              long long* total);

namespace {

inline int grid_for(long long work, int threads = 256) {
    long long g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    return int(g > 148 * 16 ? 148 * 16 : g);
}

__device__ __forceinline__ double iteration_value(int row, int col, double m, double relax) {
    // (col == row) ? 1 - w*m : -w*m, each operation rounded separately.
    const double prod = __dmul_rn(relax, m);
    return col == row ? __dsub_rn(1.0, prod) : -prod;
}

__global__ void k_domain_count(const int* rp, const int* ci, const double* v, int n, int row0,
                               double relax, int* cnt, int* status, int* max_len) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int c = 0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            double h = iteration_value(row0 + i, ci[k], v[k], relax);
            if (!(fabs(h) < DBL_EPSILON)) ++c;  // :312-317
        }
        cnt[i] = c;
        if (c == 0) atomicOr(status, DEV_ERR_DEGENERATE);  // MCLS_CHECK(num_entries > 0)
        atomicMax(max_len, c);
    }
}

__global__ void k_domain_fill(const int* rp, const int* ci, const double* v, int n, int row0,
                              double relax, const int* drp, int* dcol, double* dh,
                              double* dcdf, double* dw, int* status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int o = drp[i];
        double c = 0.0;
        const int o0 = o;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            double h = iteration_value(row0 + i, ci[k], v[k], relax);
            if (fabs(h) < DBL_EPSILON) continue;
            dcol[o] = ci[k];
            dh[o] = h;
            c = (o == o0) ? fabs(h) : __dadd_rn(fabs(h), c);  // :342-348
            dcdf[o] = c;
            ++o;
        }
        const double W = c;  // :353
        dw[i] = W;
        if (!(W > 0.0) || !isfinite(W)) {
            atomicOr(status, DEV_ERR_DEGENERATE);
            continue;
        }
        for (int k = o0; k < o; ++k) dcdf[k] = __ddiv_rn(dcdf[k], W);  // :357-362
    }
}

__global__ void k_pack_records(const int* drp, const int* dcol, const double* dh,
                               const double* dcdf, const double* dw, int n, int slots,
                               uint2* rec) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint2* r = rec + size_t(i) * slots;
        const int a = drp[i], len = drp[i + 1] - drp[i];
        r[0] = make_uint2(__float_as_uint(__double2float_rn(dw[i])), unsigned(len));
        for (int t = 0; t < slots - 1; ++t) {
            if (t < len) {
                unsigned cs = unsigned(dcol[a + t]) | (dh[a + t] > 0.0 ? 0u : 0x80000000u);
                r[1 + t] = make_uint2(__float_as_uint(__double2float_rn(dcdf[a + t])), cs);
            } else {
                r[1 + t] = make_uint2(__float_as_uint(2.0f), 0u);
            }
        }
    }
}

// Distinct column offsets (col - row) into a max_k-slot table; an offset
// takes the first free slot it meets scanning from slot 0, so each offset
// owns one slot.  More than max_k distinct offsets sets *overflow.
__global__ void k_collect_offsets(const int* rp, const int* ci, int n, int row0, int max_k,
                                  int* tab, int* overflow) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        // Once the table has overflowed the answer is known: stop early
        // instead of contending on the full table.
        if (*reinterpret_cast<volatile int*>(overflow)) return;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int d = ci[k] - (row0 + i);
            bool placed = false;
            for (int t = 0; t < max_k && !placed; ++t) {
                int cur = tab[t];
                if (cur == INT_MIN) cur = atomicCAS(&tab[t], INT_MIN, d);
                if (cur == INT_MIN || cur == d) placed = true;
            }
            if (!placed) *overflow = 1;
        }
    }
}

// Stencil record of row i: word 0 = W, word 1 = tally source (forward),
// word 2 + j = CDF value at offset off[j] with the sign of h in its sign bit,
// or NaN when the row has no entry at that offset (never selected).
__global__ void k_pack_stencil(const int* drp, const int* dcol, const double* dh,
                               const double* dcdf, const double* dw, int n, int row0, int K,
                               const int* off, int words, uint32_t* rec) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t* r = rec + size_t(i) * words;
        r[0] = __float_as_uint(__double2float_rn(dw[i]));
        r[1] = 0u;
        for (int j = 2; j < words; ++j) r[j] = 0x7fc00000u;
        for (int k = drp[i]; k < drp[i + 1]; ++k) {
            const int d = dcol[k] - (row0 + i);
            int j = 0;
            while (j < K && off[j] != d) ++j;
            if (j == K) continue;  // cannot happen: every offset is in the table
            const float c = __double2float_rn(dcdf[k]);
            r[2 + j] = __float_as_uint(dh[k] > 0.0 ? c : -c);
        }
    }
}

// Stencil record with 16-bit thresholds (stencil16): word 0 = W, word 1 =
// tally source, word 2 = sign bits of h (bit j), slot j's threshold t_j =
// round(65536 cdf_j) (65535 for the row's last entry; 0, never selected, for
// offsets the row lacks) in the 16-bit half j of words 3...
__global__ void k_pack_stencil16(const int* drp, const int* dcol, const double* dh,
                                 const double* dcdf, const double* dw, int n, int row0, int K,
                                 const int* off, int words, uint32_t* rec) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t* r = rec + size_t(i) * words;
        r[0] = __float_as_uint(__double2float_rn(dw[i]));
        r[1] = 0u;
        for (int j = 2; j < words; ++j) r[j] = 0u;
        const int last = drp[i + 1] - 1;
        for (int k = drp[i]; k <= last; ++k) {
            const int d = dcol[k] - (row0 + i);
            int j = 0;
            while (j < K && off[j] != d) ++j;
            if (j == K) continue;  // cannot happen: every offset is in the table
            double t = rint(dcdf[k] * 65536.0);
            if (k == last || t > 65535.0) t = 65535.0;
            r[3 + j / 2] |= uint32_t(t) << (16 * (j & 1));
            if (!(dh[k] > 0.0)) r[2] |= 1u << j;
        }
    }
}

__global__ void k_to_float(const double* a, float* b, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        b[i] = __double2float_rn(a[i]);
}

}  // namespace

// Sorted distinct column offsets of D (at most max_k <= 32; *K = 0 when
// there are more).
int collect_offsets(mclsgpu_context* ctx, const DevCsr& D, int max_k, int* offsets, int* K,
                    int row0) {
    cudaStream_t s = ctx->stream;
    if (max_k < 1 || max_k > 32) return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "offset table size");
    int* tab = nullptr;
    cudaError_t e = dmalloc(&tab, size_t(max_k) + 1);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    std::vector<int> init(max_k + 1, INT_MIN);
    init[max_k] = 0;
    cudaMemcpyAsync(tab, init.data(), (max_k + 1) * sizeof(int), cudaMemcpyHostToDevice, s);
    k_collect_offsets<<<grid_for(D.n), 256, 0, s>>>(D.rp, D.ci, D.n, row0, max_k, tab,
                                                    tab + max_k);
    std::vector<int> h(max_k + 1);
    cudaMemcpyAsync(h.data(), tab, (max_k + 1) * sizeof(int), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    dfree(tab);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "collect offsets");
    *K = 0;
    for (int t = 0; t < max_k; ++t) offsets[t] = 0;
    if (h[max_k]) return MCLSGPU_OK;
    std::vector<int> v;
    for (int t = 0; t < max_k; ++t)
        if (h[t] != INT_MIN) v.push_back(h[t]);
    std::sort(v.begin(), v.end());
    for (size_t t = 0; t < v.size(); ++t) offsets[t] = v[t];
    *K = int(v.size());
    return MCLSGPU_OK;
}

// Build the FP64 domain arrays and FP32 records from the composite M.
int build_domain_arrays(mclsgpu_context* ctx, const DevCsr& M, double relax,
                        mclsgpu_domain* dom, int row0) {
    cudaStream_t s = ctx->stream;
    const int n = M.n;
    int* cnt = nullptr;
    int* maxlen = nullptr;
    cudaError_t e;
    if ((e = dmalloc(&cnt, n + 1)) != cudaSuccess || (e = dmalloc(&maxlen, 1)) != cudaSuccess) {
        dfree(cnt);
        return cuda_fail(ctx, e, "cudaMalloc");
    }
    cudaMemsetAsync(maxlen, 0, sizeof(int), s);
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s);
    k_domain_count<<<grid_for(n), 256, 0, s>>>(M.rp, M.ci, M.v, n, row0, relax, cnt,
                                               ctx->d_status, maxlen);
    DevCsr& D = dom->D;
    D.release();
    D.n = n;
    int rc = MCLSGPU_OK;
    if ((e = dmalloc(&D.rp, n + 1)) != cudaSuccess) rc = cuda_fail(ctx, e, "cudaMalloc");
    long long tot = 0;
    if (!rc) rc = exclusive_scan_counts_dev(ctx, cnt, n, D.rp, &tot);
    int hmax = 0;
    if (!rc) {
        cudaMemcpyAsync(&hmax, maxlen, sizeof(int), cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "domain count");
    }
    dfree(cnt);
    dfree(maxlen);
    if (rc) return rc;
    if ((rc = check_device_status(ctx))) return rc;
    D.nnz = int(tot);
    dom->max_row = hmax;
    if ((e = dmalloc(&D.ci, tot + 1)) != cudaSuccess || (e = dmalloc(&D.v, tot + 1)) != cudaSuccess ||
        (e = dmalloc(&dom->cdf, tot + 1)) != cudaSuccess || (e = dmalloc(&dom->w, n + 1)) != cudaSuccess)
        return cuda_fail(ctx, e, "cudaMalloc");
    k_domain_fill<<<grid_for(n), 256, 0, s>>>(M.rp, M.ci, M.v, n, row0, relax, D.rp, D.ci, D.v,
                                              dom->cdf, dom->w, ctx->d_status);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "domain fill");
    if ((rc = check_device_status(ctx))) return rc;

    // FP32 records, packed format: slot count = 1 + longest row, rounded up to
    // a supported stride.
    static const int kStrides[] = {4, 8, 12, 16, 24, 32};
    int slots = 0;
    for (int st : kStrides)
        if (hmax + 1 <= st) {
            slots = st;
            break;
        }
    // Stencil format: every row's columns are row + d for d in a global set
    // of K offsets.  A record is {W, tally source, K signed CDF slots} with NaN
    // for offsets the row lacks: 2 + K words instead of 2 + 2 * row length.
    dom->stencil_k = 0;
    const int fmt = dom->p.record_format;
    if (dom->p.precision == MCLSGPU_FP32 && fmt != MCLSGPU_RECORD_PACKED) {
        int K = 0;
        if ((rc = collect_offsets(ctx, D, 30, dom->stencil_off, &K, row0))) return rc;
        // 32-, 64- or 128-byte records; stencil16: 3 words + K halves in 32 or
        // 64 bytes.
        const bool q16 = fmt == MCLSGPU_RECORD_STENCIL16;
        const int words = K <= 0 ? 0
                          : q16  ? (K <= 10 ? 8 : (K <= 26 ? 16 : 0))
                                 : (K <= 6 ? 8 : (K <= 14 ? 16 : (K <= 30 ? 32 : 0)));
        const int packed_words = slots ? 2 * slots : 1 << 30;
        if (words && (fmt == MCLSGPU_RECORD_STENCIL || q16 || words < packed_words)) {
            dom->stencil_k = K;
            dom->rec_q16 = q16 ? 1 : 0;
            slots = words / 2;
        } else if (fmt == MCLSGPU_RECORD_STENCIL || q16) {
            return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                             "stencil records need at most %d distinct column offsets (found %d)",
                             q16 ? 26 : 30, K);
        }
    }
    dom->slots = slots;  // 0: rows too long for packed records (FP64 walk only)
    if (slots) {
        if ((e = dmalloc(&dom->rec, size_t(n) * slots)) != cudaSuccess)
            return cuda_fail(ctx, e, "cudaMalloc records");
        if (dom->stencil_k) {
            int* doff = nullptr;
            if ((e = dmalloc(&doff, 32)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
            cudaMemcpyAsync(doff, dom->stencil_off, 32 * sizeof(int), cudaMemcpyHostToDevice, s);
            if (dom->rec_q16)
                k_pack_stencil16<<<grid_for(n), 256, 0, s>>>(
                    D.rp, D.ci, D.v, dom->cdf, dom->w, n, row0, dom->stencil_k, doff, 2 * slots,
                    reinterpret_cast<uint32_t*>(dom->rec));
            else
                k_pack_stencil<<<grid_for(n), 256, 0, s>>>(
                    D.rp, D.ci, D.v, dom->cdf, dom->w, n, row0, dom->stencil_k, doff, 2 * slots,
                    reinterpret_cast<uint32_t*>(dom->rec));
            e = cudaStreamSynchronize(s);
            dfree(doff);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "stencil records");
        } else {
            k_pack_records<<<grid_for(n), 256, 0, s>>>(D.rp, D.ci, D.v, dom->cdf, dom->w, n,
                                                       slots, dom->rec);
        }
    }
    // SELL-32 copy for the forward tally source (c = H b per solve).
    if (dom->p.direction == MCLSGPU_FORWARD && !dom->stencil_k) {
        if ((rc = csr_to_sell(ctx, D, dom->DS))) return rc;
    }
    // Transposed domain for the adjoint expected-value estimator.
    if (dom->p.direction == MCLSGPU_ADJOINT && dom->p.estimator == MCLSGPU_EXPECTED_VALUE) {
        if ((rc = csr_transpose(ctx, D, dom->DT))) return rc;
        if ((e = dmalloc(&dom->dt_h32, dom->DT.nnz + 1)) != cudaSuccess)
            return cuda_fail(ctx, e, "cudaMalloc");
        k_to_float<<<grid_for(dom->DT.nnz), 256, 0, s>>>(dom->DT.v, dom->dt_h32, dom->DT.nnz);
    }
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "domain records");
    return MCLSGPU_OK;
}

}  // namespace mclsgpu
