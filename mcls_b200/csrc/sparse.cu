// sparse.cu -- device CSR plumbing for the composite operator and the
// preconditioners: upload/validation, transpose, SpGEMM with the reference's
// relative filter, FP64 SpMV, point- and block-Jacobi builds.  All of it is
// set-up work (once per operator) except spmv.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "internal.h"

namespace mclsgpu {

void DevCsr::release() {
    dfree(rp);
    dfree(ci);
    dfree(v);
    n = nnz = 0;
}

void DevSell::release() {
    dfree(off);
    dfree(col);
    dfree(val);
    n = nslices = 0;
}

namespace {

inline int grid_for(long long work, int threads = 256, int cap = 148 * 16) {
    long long g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    return int(g > cap ? cap : g);
}

__global__ void k_count_cols(const int* ci, int nnz, int* cnt) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x)
        atomicAdd(&cnt[ci[k]], 1);
}

__global__ void k_scatter_transpose(const int* rp, const int* ci, const double* v, int n,
                                    int* cursor, int* tci, double* tv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            int p = atomicAdd(&cursor[ci[k]], 1);
            tci[p] = i;
            tv[p] = v[k];
        }
}

// Sort each row by column (rows are short: insertion sort).
__global__ void k_sort_rows(const int* rp, int* ci, double* v, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int a = rp[i], b = rp[i + 1];
        for (int k = a + 1; k < b; ++k) {
            int c = ci[k];
            double x = v[k];
            int m = k - 1;
            while (m >= a && ci[m] > c) {
                ci[m + 1] = ci[m];
                v[m + 1] = v[m];
                --m;
            }
            ci[m + 1] = c;
            v[m + 1] = x;
        }
    }
}

// Upper bound of the product row length: sum of |B_k| over A's row.
__global__ void k_spgemm_bound(const int* arp, const int* aci, const int* brp, int n,
                               long long* ub) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        long long s = 0;
        for (int k = arp[i]; k < arp[i + 1]; ++k) s += brp[aci[k] + 1] - brp[aci[k]];
        ub[i] = s;
    }
}

// Build each product row in its scratch segment: products arrive in A's row
// order then B's row order and accumulate into a sorted list; then the
// reference filter (tpetra/src/MCLS_TpetraHelpers.hpp:196-259) is applied.
__global__ void k_spgemm_rows(const int* arp, const int* aci, const double* av,
                              const int* brp, const int* bci, const double* bv, int n,
                              const long long* off, int* sc, double* sv, int* len,
                              double threshold) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int* c = sc + off[i];
        double* v = sv + off[i];
        int m = 0;
        for (int ka = arp[i]; ka < arp[i + 1]; ++ka) {
            const int k = aci[ka];
            const double a = av[ka];
            for (int kb = brp[k]; kb < brp[k + 1]; ++kb) {
                const int j = bci[kb];
                const double prod = a * bv[kb];
                // binary search in the sorted prefix c[0..m)
                int lo = 0, hi = m;
                while (lo < hi) {
                    int mid = (lo + hi) >> 1;
                    if (c[mid] < j) lo = mid + 1; else hi = mid;
                }
                if (lo < m && c[lo] == j) {
                    v[lo] = v[lo] + prod;
                } else {
                    for (int t = m; t > lo; --t) {
                        c[t] = c[t - 1];
                        v[t] = v[t - 1];
                    }
                    c[lo] = j;
                    v[lo] = prod;
                    ++m;
                }
            }
        }
        if (m == 0) {
            len[i] = 0;
            continue;
        }
        double mx = v[0];
        for (int t = 1; t < m; ++t) mx = v[t] > mx ? v[t] : mx;
        const double row_thr = mx * threshold;
        for (int t = 0; t < m; ++t)
            if (fabs(v[t]) <= row_thr) {
                v[t] = 0.0;
                c[t] = -1;
            }
        int nv = 0, nc = 0;
        for (int t = 0; t < m; ++t)
            if (v[t] != 0.0) v[nv++] = v[t];
        for (int t = 0; t < m; ++t)
            if (c[t] != -1) c[nc++] = c[t];
        for (int t = nc; t < nv; ++t) c[t] = -1;
        len[i] = nv;
    }
}

__global__ void k_gather_rows(const long long* off, const int* sc, const double* sv,
                              const int* rp, int n, int* ci, double* v, int* bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int a = rp[i], len = rp[i + 1] - rp[i];
        for (int t = 0; t < len; ++t) {
            int c = sc[off[i] + t];
            if (c < 0) atomicOr(bad, DEV_ERR_BOUNDS);
            ci[a + t] = c;
            v[a + t] = sv[off[i] + t];
        }
    }
}

__global__ void k_scale_cols(int* ci, double* v, int nnz, const double* s) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x)
        v[k] = v[k] * s[ci[k]];
}

__global__ void __launch_bounds__(256) k_spmv(const int* rp, const int* ci, const double* v,
                                              int n, const double* x, double* y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) s = fma(v[k], x[ci[k]], s);
        y[i] = s;
    }
}

__global__ void k_recip_diag(const int* rp, const int* ci, const double* v, int n,
                             double* dinv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) d = v[k];
        dinv[i] = 1.0 / d;  // Vector::reciprocal of the diagonal copy
    }
}

__global__ void k_diag_csr(int n, const double* d, int* rp, int* ci, double* v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        rp[i] = i;
        if (i < n) {
            ci[i] = i;
            v[i] = d[i];
        }
    }
}

constexpr int kMaxBlock = 32;

// LU with partial pivoting and inverse from the factors (the GETRF/GETRI
// algorithm) of one contiguous block per thread.  The block is assembled as
// the reference does (transposed, column-major) and row i of the result is
// row i of inv(B) (tpetra/src/MCLS_TpetraBlockJacobiPreconditioner_impl.hpp:
// 155-191).
__global__ void k_block_jacobi(const int* rp, const int* ci, const double* v, int n, int bs,
                               double* work, int* prp, int* pci, double* pv, int* bad) {
    const int nblk = n / bs;
    for (int blk = blockIdx.x * blockDim.x + threadIdx.x; blk < nblk;
         blk += gridDim.x * blockDim.x) {
        double* a = work + size_t(blk) * bs * bs;
        const int b0 = blk * bs;
        for (int t = 0; t < bs * bs; ++t) a[t] = 0.0;
        for (int i = 0; i < bs; ++i)
            for (int k = rp[b0 + i]; k < rp[b0 + i + 1]; ++k) {
                int c = ci[k] - b0;
                if (c >= 0 && c < bs) a[c + i * bs] = v[k];
            }
        int piv[kMaxBlock];
        bool ok = true;
        for (int j = 0; j < bs && ok; ++j) {
            int p = j;
            double mx = fabs(a[j + j * bs]);
            for (int i = j + 1; i < bs; ++i)
                if (fabs(a[i + j * bs]) > mx) {
                    mx = fabs(a[i + j * bs]);
                    p = i;
                }
            piv[j] = p;
            if (a[p + j * bs] == 0.0) {
                ok = false;
                break;
            }
            if (p != j)
                for (int c = 0; c < bs; ++c) {
                    double t = a[j + c * bs];
                    a[j + c * bs] = a[p + c * bs];
                    a[p + c * bs] = t;
                }
            double r = 1.0 / a[j + j * bs];
            for (int i = j + 1; i < bs; ++i) a[i + j * bs] *= r;
            for (int c = j + 1; c < bs; ++c)
                for (int i = j + 1; i < bs; ++i) a[i + c * bs] -= a[i + j * bs] * a[j + c * bs];
        }
        if (!ok) {
            atomicOr(bad, DEV_ERR_DEGENERATE);
            continue;
        }
        for (int j = 0; j < bs; ++j) {
            a[j + j * bs] = 1.0 / a[j + j * bs];
            double ajj = -a[j + j * bs];
            for (int i = 0; i < j; ++i) {
                double s = 0.0;
                for (int k = i; k < j; ++k) s += a[i + k * bs] * a[k + j * bs];
                a[i + j * bs] = s;
            }
            for (int i = 0; i < j; ++i) a[i + j * bs] *= ajj;
        }
        double wk[kMaxBlock];
        for (int j = bs - 2; j >= 0; --j) {
            for (int i = j + 1; i < bs; ++i) {
                wk[i] = a[i + j * bs];
                a[i + j * bs] = 0.0;
            }
            for (int i = 0; i < bs; ++i) {
                double s = 0.0;
                for (int k = j + 1; k < bs; ++k) s += a[i + k * bs] * wk[k];
                a[i + j * bs] -= s;
            }
        }
        for (int j = bs - 2; j >= 0; --j)
            if (piv[j] != j)
                for (int i = 0; i < bs; ++i) {
                    double t = a[i + j * bs];
                    a[i + j * bs] = a[i + piv[j] * bs];
                    a[i + piv[j] * bs] = t;
                }
        for (int i = 0; i < bs; ++i) {
            const int row = b0 + i;
            prp[row + 1] = (row + 1) * bs;
            for (int j = 0; j < bs; ++j) {
                pci[row * bs + j] = b0 + j;
                pv[row * bs + j] = a[j + i * bs];
            }
        }
        if (blk == 0) prp[0] = 0;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
int upload_csr(mclsgpu_context* ctx, int64_t n, const int64_t* rp, const int64_t* ci,
               const double* v, DevCsr& out, int64_t ncols) {
    if (ncols < 0) ncols = n;
    if (n <= 0 || n >= (int64_t(1) << 31) || ncols <= 0 || ncols >= (int64_t(1) << 31) || !rp ||
        !ci || !v)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "operator: bad size or null array");
    if (rp[0] != 0) return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "operator: rowptr[0] != 0");
    const int64_t nnz = rp[n];
    if (nnz < 0 || nnz >= (int64_t(1) << 31))
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "operator: bad nnz");
    std::vector<int> hrp(n + 1), hci(nnz);
    std::vector<double> hv(nnz);
    // Rows are sorted by column and duplicate entries summed, as Tpetra's
    // fillComplete leaves them.
    std::vector<std::pair<int, double>> row;
    int64_t out_k = 0;
    hrp[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (rp[i + 1] < rp[i])
            return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "operator: rowptr not monotone at %lld",
                             (long long)i);
        row.clear();
        bool sorted = true;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
            if (ci[k] < 0 || ci[k] >= ncols)
                return set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                                 "operator: column %lld out of range in row %lld",
                                 (long long)ci[k], (long long)i);
            if (!std::isfinite(v[k]))
                return set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                                 "operator: non-finite value in row %lld", (long long)i);
            if (!row.empty() && ci[k] <= row.back().first) sorted = false;
            row.emplace_back(int(ci[k]), v[k]);
        }
        if (!sorted) {
            std::stable_sort(row.begin(), row.end(),
                             [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
                                 return a.first < b.first;
                             });
        }
        for (size_t t = 0; t < row.size(); ++t) {
            if (t > 0 && row[t].first == hci[out_k - 1]) {
                hv[out_k - 1] += row[t].second;
            } else {
                hci[out_k] = row[t].first;
                hv[out_k] = row[t].second;
                ++out_k;
            }
        }
        hrp[i + 1] = int(out_k);
    }
    out.release();
    out.n = int(n);
    out.nnz = int(out_k);
    cudaError_t e;
    if ((e = dmalloc(&out.rp, n + 1)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    if ((e = dmalloc(&out.ci, out_k + 1)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    if ((e = dmalloc(&out.v, out_k + 1)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    cudaMemcpyAsync(out.rp, hrp.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(out.ci, hci.data(), out_k * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
    e = cudaMemcpyAsync(out.v, hv.data(), out_k * sizeof(double), cudaMemcpyHostToDevice,
                        ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "upload");
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "upload sync");
    return MCLSGPU_OK;
}

// Exclusive scan of n counts into rp[0..n] on the host-visible path: the
// counts are small set-up arrays, so a device scan is not worth a kernel
// family here; copy, scan, copy back.
int exclusive_scan_counts_dev(mclsgpu_context* ctx, const int* d_cnt, int n, int* d_rp,
                                 long long* total) {
    std::vector<int> h(n);
    cudaError_t e = cudaMemcpyAsync(h.data(), d_cnt, n * sizeof(int), cudaMemcpyDeviceToHost,
                                    ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "scan counts");
    std::vector<int> r(n + 1);
    long long s = 0;
    for (int i = 0; i < n; ++i) {
        r[i] = int(s);
        s += h[i];
    }
    if (s >= (1LL << 31)) return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "more than 2^31 entries");
    r[n] = int(s);
    e = cudaMemcpyAsync(d_rp, r.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice,
                        ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "scan counts");
    *total = s;
    return MCLSGPU_OK;
}

int csr_transpose(mclsgpu_context* ctx, const DevCsr& A, DevCsr& T) {
    cudaStream_t s = ctx->stream;
    T.release();
    T.n = A.n;
    int* cnt = nullptr;
    cudaError_t e = dmalloc(&cnt, A.n + 1);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    cudaMemsetAsync(cnt, 0, (A.n + 1) * sizeof(int), s);
    k_count_cols<<<grid_for(A.nnz), 256, 0, s>>>(A.ci, A.nnz, cnt);
    if ((e = dmalloc(&T.rp, A.n + 1)) != cudaSuccess) { dfree(cnt); return cuda_fail(ctx, e, "cudaMalloc"); }
    long long tot = 0;
    int rc = exclusive_scan_counts_dev(ctx, cnt, A.n, T.rp, &tot);
    if (rc) { dfree(cnt); return rc; }
    T.nnz = int(tot);
    if ((e = dmalloc(&T.ci, T.nnz + 1)) != cudaSuccess) { dfree(cnt); return cuda_fail(ctx, e, "cudaMalloc"); }
    if ((e = dmalloc(&T.v, T.nnz + 1)) != cudaSuccess) { dfree(cnt); return cuda_fail(ctx, e, "cudaMalloc"); }
    cudaMemcpyAsync(cnt, T.rp, A.n * sizeof(int), cudaMemcpyDeviceToDevice, s);
    k_scatter_transpose<<<grid_for(A.n), 256, 0, s>>>(A.rp, A.ci, A.v, A.n, cnt, T.ci, T.v);
    k_sort_rows<<<grid_for(T.n), 256, 0, s>>>(T.rp, T.ci, T.v, T.n);
    e = cudaStreamSynchronize(s);
    dfree(cnt);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "transpose");
    return MCLSGPU_OK;
}

int csr_multiply(mclsgpu_context* ctx, const DevCsr& A, const DevCsr& B, double threshold,
                 DevCsr& C) {
    cudaStream_t s = ctx->stream;
    const int n = A.n;
    long long* ub = nullptr;
    cudaError_t e = dmalloc(&ub, n + 1);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    k_spgemm_bound<<<grid_for(n), 256, 0, s>>>(A.rp, A.ci, B.rp, n, ub);
    std::vector<long long> hub(n), hoff(n + 1);
    cudaMemcpyAsync(hub.data(), ub, n * sizeof(long long), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { dfree(ub); return cuda_fail(ctx, e, "spgemm bound"); }
    hoff[0] = 0;
    for (int i = 0; i < n; ++i) hoff[i + 1] = hoff[i] + hub[i];
    const long long U = hoff[n];
    int* sc = nullptr;
    double* sv = nullptr;
    int* len = nullptr;
    int* bad = nullptr;
    if ((e = dmalloc(&sc, U + 1)) != cudaSuccess || (e = dmalloc(&sv, U + 1)) != cudaSuccess ||
        (e = dmalloc(&len, n + 1)) != cudaSuccess || (e = dmalloc(&bad, 1)) != cudaSuccess) {
        dfree(ub); dfree(sc); dfree(sv); dfree(len); dfree(bad);
        return cuda_fail(ctx, e, "cudaMalloc spgemm");
    }
    cudaMemcpyAsync(ub, hoff.data(), n * sizeof(long long), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(bad, 0, sizeof(int), s);
    k_spgemm_rows<<<grid_for(n, 128), 128, 0, s>>>(A.rp, A.ci, A.v, B.rp, B.ci, B.v, n, ub, sc,
                                                  sv, len, threshold);
    C.release();
    C.n = n;
    int rc = MCLSGPU_OK;
    if ((e = dmalloc(&C.rp, n + 1)) != cudaSuccess) rc = cuda_fail(ctx, e, "cudaMalloc");
    long long tot = 0;
    if (!rc) rc = exclusive_scan_counts_dev(ctx, len, n, C.rp, &tot);
    if (!rc) {
        C.nnz = int(tot);
        if ((e = dmalloc(&C.ci, tot + 1)) != cudaSuccess || (e = dmalloc(&C.v, tot + 1)) != cudaSuccess)
            rc = cuda_fail(ctx, e, "cudaMalloc");
    }
    if (!rc) {
        k_gather_rows<<<grid_for(n), 256, 0, s>>>(ub, sc, sv, C.rp, n, C.ci, C.v, bad);
        int hbad = 0;
        cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "spgemm");
        else if (hbad) rc = set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                                      "composite filter left mismatched entries");
    }
    dfree(ub); dfree(sc); dfree(sv); dfree(len); dfree(bad);
    return rc;
}

int csr_copy(mclsgpu_context* ctx, const DevCsr& A, DevCsr& B) {
    B.release();
    B.n = A.n;
    B.nnz = A.nnz;
    cudaError_t e;
    if ((e = dmalloc(&B.rp, A.n + 1)) != cudaSuccess || (e = dmalloc(&B.ci, A.nnz + 1)) != cudaSuccess ||
        (e = dmalloc(&B.v, A.nnz + 1)) != cudaSuccess)
        return cuda_fail(ctx, e, "cudaMalloc");
    cudaMemcpyAsync(B.rp, A.rp, (A.n + 1) * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream);
    cudaMemcpyAsync(B.ci, A.ci, A.nnz * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream);
    cudaMemcpyAsync(B.v, A.v, A.nnz * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
    return MCLSGPU_OK;
}

void csr_scale_cols(mclsgpu_context* ctx, DevCsr& T, const double* sc) {
    k_scale_cols<<<grid_for(T.nnz), 256, 0, ctx->stream>>>(T.ci, T.v, T.nnz, sc);
}

int csr_filter(mclsgpu_context* ctx, const DevCsr& A, double threshold, DevCsr& out,
               int ncols) {
    // Filtering is a product with the identity: reuse the SpGEMM row builder
    // with B = I (ncols x ncols: A's columns index its rows) so that the
    // reference filter code path is shared.
    if (ncols < 0) ncols = A.n;
    DevCsr I;
    I.n = ncols;
    I.nnz = ncols;
    cudaError_t e;
    double* ones = nullptr;
    if ((e = dmalloc(&ones, ncols)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    std::vector<double> h(ncols, 1.0);
    cudaMemcpyAsync(ones, h.data(), size_t(ncols) * sizeof(double), cudaMemcpyHostToDevice,
                    ctx->stream);
    int rc = point_jacobi_csr(ctx, ncols, ones, I);
    if (!rc) rc = csr_multiply(ctx, A, I, threshold, out);
    I.release();
    dfree(ones);
    return rc;
}

void spmv(cudaStream_t s, const DevCsr& A, const double* x, double* y) {
    k_spmv<<<grid_for(A.n, 256, 148 * 8), 256, 0, s>>>(A.rp, A.ci, A.v, A.n, x, y);
}

int reciprocal_diagonal(mclsgpu_context* ctx, const DevCsr& A, double* dinv) {
    k_recip_diag<<<grid_for(A.n), 256, 0, ctx->stream>>>(A.rp, A.ci, A.v, A.n, dinv);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(ctx, e, "reciprocal diagonal");
}

int point_jacobi_csr(mclsgpu_context* ctx, int n, const double* dinv, DevCsr& P) {
    P.release();
    P.n = n;
    P.nnz = n;
    cudaError_t e;
    if ((e = dmalloc(&P.rp, n + 1)) != cudaSuccess || (e = dmalloc(&P.ci, n + 1)) != cudaSuccess ||
        (e = dmalloc(&P.v, n + 1)) != cudaSuccess)
        return cuda_fail(ctx, e, "cudaMalloc");
    k_diag_csr<<<grid_for(n + 1), 256, 0, ctx->stream>>>(n, dinv, P.rp, P.ci, P.v);
    return MCLSGPU_OK;
}

int block_jacobi(mclsgpu_context* ctx, const DevCsr& A, int bs, DevCsr& P) {
    if (bs < 1 || bs > kMaxBlock || A.n % bs)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                         "Jacobi Block Size %d must divide the row count and be <= %d", bs,
                         kMaxBlock);
    cudaStream_t s = ctx->stream;
    P.release();
    P.n = A.n;
    P.nnz = A.n * bs;
    double* work = nullptr;
    int* bad = nullptr;
    cudaError_t e;
    if ((e = dmalloc(&P.rp, A.n + 1)) != cudaSuccess || (e = dmalloc(&P.ci, P.nnz + 1)) != cudaSuccess ||
        (e = dmalloc(&P.v, P.nnz + 1)) != cudaSuccess ||
        (e = dmalloc(&work, size_t(A.n) * bs)) != cudaSuccess || (e = dmalloc(&bad, 1)) != cudaSuccess) {
        dfree(work); dfree(bad);
        return cuda_fail(ctx, e, "cudaMalloc");
    }
    cudaMemsetAsync(bad, 0, sizeof(int), s);
    k_block_jacobi<<<grid_for(A.n / bs, 64), 64, 0, s>>>(A.rp, A.ci, A.v, A.n, bs, work, P.rp,
                                                         P.ci, P.v, bad);
    int hbad = 0;
    cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    dfree(work);
    dfree(bad);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "block jacobi");
    if (hbad) return set_error(ctx, MCLSGPU_ERR_DEGENERATE, "singular Jacobi block");
    return MCLSGPU_OK;
}

namespace {

__global__ void k_slice_width(const int* rp, int n, int nslices, int* width) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nslices; s += gridDim.x * blockDim.x) {
        int w = 0;
        for (int r = 32 * s; r < 32 * s + 32 && r < n; ++r) w = max(w, rp[r + 1] - rp[r]);
        width[s] = 32 * w;
    }
}

__global__ void k_sell_fill(const int* rp, const int* ci, const double* v, int n, int nslices,
                            const int* off, int* scol, double* sval) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < 32 * nslices;
         r += gridDim.x * blockDim.x) {
        const int s = r >> 5, lane = r & 31;
        const int o = off[s], w = (off[s + 1] - o) >> 5;
        const int a = r < n ? rp[r] : 0, len = r < n ? rp[r + 1] - rp[r] : 0;
        for (int k = 0; k < w; ++k) {
            const bool real = k < len;
            scol[o + 32 * k + lane] = real ? ci[a + k] : (r < n ? r : 0);
            sval[o + 32 * k + lane] = real ? v[a + k] : 0.0;
        }
    }
}

__global__ void __launch_bounds__(256) k_sell_spmv(const int* off, const int* col,
                                                   const double* val, int n, const double* x,
                                                   double* y) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int o = off[r >> 5] + (r & 31), w = (off[(r >> 5) + 1] - off[r >> 5]) >> 5;
        double s = 0.0;
        for (int k = 0; k < w; ++k) s = fma(val[o + 32 * k], x[col[o + 32 * k]], s);
        y[r] = s;
    }
}

}  // namespace

int csr_to_sell(mclsgpu_context* ctx, const DevCsr& A, DevSell& S) {
    cudaStream_t s = ctx->stream;
    S.release();
    S.n = A.n;
    S.nslices = (A.n + 31) / 32;
    int* width = nullptr;
    cudaError_t e = dmalloc(&width, S.nslices + 1);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    if ((e = dmalloc(&S.off, S.nslices + 1)) != cudaSuccess) {
        dfree(width);
        return cuda_fail(ctx, e, "cudaMalloc");
    }
    k_slice_width<<<grid_for(S.nslices), 256, 0, s>>>(A.rp, A.n, S.nslices, width);
    long long tot = 0;
    int rc = exclusive_scan_counts_dev(ctx, width, S.nslices, S.off, &tot);
    dfree(width);
    if (rc) return rc;
    if ((e = dmalloc(&S.col, tot + 1)) != cudaSuccess || (e = dmalloc(&S.val, tot + 1)) != cudaSuccess)
        return cuda_fail(ctx, e, "cudaMalloc SELL");
    k_sell_fill<<<grid_for(32LL * S.nslices), 256, 0, s>>>(A.rp, A.ci, A.v, A.n, S.nslices, S.off,
                                                          S.col, S.val);
    e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(ctx, e, "SELL build");
}

namespace {

struct DiaOffsets {
    int off[16];
};

__global__ void k_fill_dia(const int* rp, const int* ci, const double* v, int n, int K,
                           DiaOffsets o, double* val) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        for (int j = 0; j < K; ++j) val[size_t(j) * n + r] = 0.0;
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            const int d = ci[k] - r;
            for (int j = 0; j < K; ++j)
                if (o.off[j] == d) val[size_t(j) * n + r] = v[k];
        }
    }
}

// Symmetry of a diagonal pair: val[jneg][r] == val[jpos][r - o] bit for bit
// (A(r, r - o) == A(r - o, r)); rows without the column hold 0.
__global__ void k_dia_symmetric(const double* val, int n, int jneg, int jpos, int o, int* bad) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const double a = val[size_t(jneg) * n + r];
        const double b = r >= o ? val[size_t(jpos) * n + r - o] : 0.0;
        if (__double_as_longlong(a) != __double_as_longlong(b)) atomicOr(bad, 1);
    }
}

}  // namespace

int dia_symmetric(mclsgpu_context* ctx, int n, int K, const int* offsets, const double* val,
                  double** sym, int* kh, int* sym_off) {
    *sym = nullptr;
    *kh = 0;
    // Offsets -o_h < ... < -o_1 < 0 < o_1 < ... < o_h (ascending).
    if (K < 3 || (K & 1) == 0 || offsets[K / 2] != 0) return MCLSGPU_OK;
    const int H = K / 2;
    for (int h = 0; h < H; ++h)
        if (offsets[K / 2 + 1 + h] <= 0 || offsets[K / 2 - 1 - h] != -offsets[K / 2 + 1 + h])
            return MCLSGPU_OK;
    cudaStream_t s = ctx->stream;
    int* bad = nullptr;
    cudaError_t e = dmalloc(&bad, 1);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    cudaMemsetAsync(bad, 0, sizeof(int), s);
    for (int h = 0; h < H; ++h) {
        const int jpos = K / 2 + 1 + h, jneg = K / 2 - 1 - h;
        k_dia_symmetric<<<grid_for(n), 256, 0, s>>>(val, n, jneg, jpos, offsets[jpos], bad);
    }
    int hb = 1;
    cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    dfree(bad);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "DIA symmetry");
    if (hb) return MCLSGPU_OK;
    // Diagonal first, then the positive offsets in ascending order.
    if ((e = dmalloc(sym, size_t(1 + H) * n)) != cudaSuccess)
        return cuda_fail(ctx, e, "cudaMalloc symmetric DIA");
    cudaMemcpyAsync(*sym, val + size_t(K / 2) * n, size_t(n) * sizeof(double),
                    cudaMemcpyDeviceToDevice, s);
    for (int h = 0; h < H; ++h) {
        cudaMemcpyAsync(*sym + size_t(1 + h) * n, val + size_t(K / 2 + 1 + h) * n,
                        size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
        sym_off[h] = offsets[K / 2 + 1 + h];
    }
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        dfree(*sym);
        return cuda_fail(ctx, e, "symmetric DIA");
    }
    *kh = H;
    return MCLSGPU_OK;
}

int csr_to_dia(mclsgpu_context* ctx, const DevCsr& A, int K, const int* offsets, double** val) {
    *val = nullptr;
    cudaError_t e = dmalloc(val, size_t(K) * A.n);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc DIA");
    DiaOffsets o{};
    for (int j = 0; j < K && j < 16; ++j) o.off[j] = offsets[j];
    k_fill_dia<<<grid_for(A.n), 256, 0, ctx->stream>>>(A.rp, A.ci, A.v, A.n, K, o, *val);
    e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(ctx, e, "DIA build");
}

void sell_spmv(cudaStream_t s, const DevSell& A, const double* x, double* y) {
    k_sell_spmv<<<grid_for(A.n, 256, 148 * 8), 256, 0, s>>>(A.off, A.col, A.val, A.n, x, y);
}

}  // namespace mclsgpu
