// walk.cu -- Neumann-Ulam random-walk kernels.
//
// One history restates DomainTransporter::transport
// (src/MCLS_DomainTransporter_impl.hpp:70-119): tally at the pre-transition
// state, then AlmostOptimalDomain::processTransition
// (src/MCLS_AlmostOptimalDomain.hpp:254-284): u ~ U[0,1),
// j = lower_bound(cdf_row, u), state <- col_j, w *= W_row * sign(h_j), and
// termination once the history has taken "History Length" steps
// (:135-136) or, with the legacy "Weight Cutoff", once |w| < cutoff * |w0|.
//
// walk32: the production kernel.  Persistent warps pull histories from a
// work-queue counter and refill lanes as histories terminate.  A step reads
// one packed FP32 record (slots * 8 bytes, 16-byte vector loads), selects the
// first entry whose CDF value is >= u with predicated compares (the records'
// padding entries hold 2.0 and are never selected) and carries the weight in
// FP32.  Tallies reduce into FP64: the adjoint collision tally with a
// fire-and-forget FP64 reduction per step, the forward history sum
// Kahan-compensated in FP32 and reduced into FP64 once per history.  The
// adjoint step-0 tally is made by the source build (counts * w0), so walks
// tally from step 1.
//
// walk64: the parity kernel.  FP64 CSR domain, binary search with
// std::lower_bound semantics, FP64 weights and tallies, optional trajectory
// trace.  With the reference stream it reproduces the reference's
// trajectories bit for bit.
#include <climits>

#include "internal.h"
#include "rng.cuh"

namespace mclsgpu {

struct WalkArgs {
    int n;
    int L;
    int per;                    // forward: histories per state
    int rng_mode;
    const int* d_nh;
    int* d_counter;
    const int* start;           // adjoint: state | sign<<31
    const double* sc;           // [0] weight
    float cutoff;               // relative weight cutoff (0 = off)
    double cutoff64;
    uint64_t seed;
    const unsigned long long* d_epoch;
    const uint64_t* jump;
    const unsigned long long* d_pos;
    // FP32 records
    const uint2* rec;
    // FP64 domain
    const int* rp;
    const int* col;
    const double* h;
    const double* cdf;
    const double* W;
    // tallies
    double* y64;
    const float* c32;
    const double* c64;
    unsigned long long* d_steps;
    unsigned long long* d_tim;  // [0] first warp start, [1] last warp end (ns)
    int* status;
    int row0;                   // global index of the first record / tally row
    int l1;                     // record loads allocate in L1
    int stoff[32];              // stencil records: column offset of each slot
    // variable-length histories on the reference stream (FP64 only): history
    // e's first draw is *d_pos + hoff[e]; hlen[e] receives its length
    const int* hoff;
    int* hlen;
    // trace (FP64 only)
    long long max_trace;
    long long* tr_states;
    double* tr_w;
    int* tr_ev;
    long long* tr_start;
};

namespace {

constexpr unsigned kFull = 0xffffffffu;

// 256-bit read-only load of half a record, not allocated in L1 (records are
// read once per step and reused across steps only through L2).
__device__ __forceinline__ void ld_record256(const void* p, uint32_t* r) {
    asm volatile(
        "ld.global.nc.L1::no_allocate.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7])
        : "l"(p));
}
// The same load allocated in L1: histories of one block start at neighbouring
// states and step to neighbours, so their records are often fetched again by
// the block's other warps.
__device__ __forceinline__ void ld_record256_l1(const void* p, uint32_t* r) {
    asm volatile(
        "ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7])
        : "l"(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint64_t history_state(const WalkArgs& a, uint64_t ekey, long long e) {
    if (a.rng_mode == MCLSGPU_RNG_COUNTER) return counter_state(ekey, 2, uint64_t(e));
    const uint64_t off = a.hoff ? uint64_t(a.hoff[e]) : uint64_t(e) * uint64_t(a.L);
    return xs_jump(a.jump, a.seed, *a.d_pos + off);
}

// Small records (up to 8 slots) run at full occupancy: 8 blocks of 256 threads
// per SM, i.e. at most 32 registers per thread.  The per-launch constants
// that are only needed when a lane takes a new history (history count,
// stream key, starting weight) live in shared memory, not registers.
template <int S>
struct WalkOccupancy {
    static constexpr int kMinBlocks = S <= 8 ? 8 : (S <= 24 ? 4 : 2);
};

// Record kinds of the FP32 walk (template parameter ST).
//   0 packed:      slot 0 = {W, len or tally source}, slots 1.. = {cdf (f32),
//                  column | sign << 31}, padding CDF 2.0
//   1 stencil:     word 0 = W, word 1 = tally source, word 2 + j = the CDF at
//                  column offset off[j] with the sign of h_j in its sign bit,
//                  NaN where the row has no entry at that offset
//   2 stencil16:   word 0 = W, word 1 = tally source, word 2 = the signs of
//                  h_j (bit j), then 16-bit thresholds t_j two to a word
//                  (slot j in word 3 + j/2, bits 16 (j % 2)..): t_j =
//                  round(65536 cdf_j), 65535 for the row's last entry, 0 where
//                  the row has no entry at off[j]
constexpr int kPacked = 0, kStencil = 1, kStencil16 = 2;

// Selection in one FP32 record (the S-slot words q of state s) for the draw
// x: the first entry whose CDF value is >= u (sampleDiscreteCDF's
// lower_bound) with u the draw's 24-bit uniform, or for stencil16 the first
// slot with u16 < t_j, u16 = min(top 16 bits, 65534).  s becomes the selected
// column; neg is the sign bit of the selected h.
template <int S, int ST>
__device__ __forceinline__ void select32(const WalkArgs& a, const uint32_t* q, uint64_t x, int& s,
                                         unsigned& neg) {
    if constexpr (ST == kPacked) {
        const float u = canonical32(x);
        unsigned sel = q[3];  // slot 1 (first entry)
        bool found = __uint_as_float(q[2]) >= u;
#pragma unroll
        for (int t = 2; t < S; ++t) {
            const bool c = !found && __uint_as_float(q[2 * t]) >= u;
            sel = c ? q[2 * t + 1] : sel;
            found = found || c;
        }
        neg = sel & 0x80000000u;
        s = int(sel & 0x7fffffffu);
    } else if constexpr (ST == kStencil) {
        // Stencil slots: first |cdf_j| >= u (NaN slots never match); the next
        // state is s + offset_j, the sign of h_j is the sign bit of the slot.
        const float u = canonical32(x);
        int dsel = 0;
        unsigned ng = 0u;
        bool found = false;
#pragma unroll
        for (int j = 0; j < 2 * S - 2; ++j) {
            const bool c = !found && fabsf(__uint_as_float(q[2 + j])) >= u;
            dsel = c ? a.stoff[j] : dsel;
            ng = c ? (q[2 + j] & 0x80000000u) : ng;
            found = found || c;
        }
        neg = ng;
        s += dsel;
    } else {
        const unsigned u16 = min(unsigned(x >> 48), 65534u);
        int dsel = 0, jsel = 0;
        bool found = false;
#pragma unroll
        for (int j = 0; j < 2 * (2 * S - 3); ++j) {
            const unsigned t = (q[3 + j / 2] >> (16 * (j & 1))) & 0xffffu;
            const bool c = !found && u16 < t;
            dsel = c ? a.stoff[j] : dsel;
            jsel = c ? j : jsel;
            found = found || c;
        }
        neg = ((q[2] >> jsel) & 1u) << 31;
        s += dsel;
    }
}

// Selection in the FP64 domain row of state s for the uniform u
// (std::lower_bound over the row's CDF, as the reference samples it).
// Returns the entry index within the row; the caller checks it is < len.
__device__ __forceinline__ int select64(const WalkArgs& a, int s, double u, int& r0, int& len) {
    r0 = a.rp[s];
    len = a.rp[s + 1] - r0;
    int lo = 0, hi = len;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a.cdf[r0 + mid] < u) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// One transition of a history at state s (DomainTransporter::transport's
// loop body): tally at the pre-transition state, read the state's record,
// draw u, select the first entry whose CDF value is >= u, update the state
// and the weight.
template <int S, int DIR, int ST>
__device__ __forceinline__ void walk_step(const WalkArgs& a, const char* rec, int& s, float& w,
                                          uint64_t& x, float& acc, float& comp, int k) {
    // One record: S/4 256-bit loads, bypassing L1 (each step touches exactly
    // the record's own sectors) or allocated in it (the launch shape says).
    const char* r = rec + size_t(s - a.row0) * (S * 8);
    uint32_t q[2 * S];
    if (a.l1) {
#pragma unroll
        for (int t = 0; t < S / 4; ++t) ld_record256_l1(r + 32 * t, q + 8 * t);
    } else {
#pragma unroll
        for (int t = 0; t < S / 4; ++t) ld_record256(r + 32 * t, q + 8 * t);
    }
    if (DIR == MCLSGPU_ADJOINT) {
        // FP32 weight, FP64 reduction (fire-and-forget RED.ADD.F64).
        if (k > 0) atomicAdd(&a.y64[s - a.row0], double(w));
    } else {
        // Kahan-compensated FP32 history sum; the tally source of the state
        // rides in the record header (slot 0, second word).
        const float term = w * __uint_as_float(q[1]) - comp;
        const float t = acc + term;
        comp = (t - acc) - term;
        acc = t;
    }
    x = xs_step(x);
    const float Wt = __uint_as_float(q[0]);
    unsigned neg;
    select32<S, ST>(a, q, x, s, neg);
    w = neg ? -(w * Wt) : w * Wt;
}

// Starting state, weight and stream of history e.
template <int DIR>
__device__ __forceinline__ void walk_start(const WalkArgs& a, int e, uint64_t ekey, float wnorm,
                                           int& s, float& w, uint64_t& x) {
    if (DIR == MCLSGPU_ADJOINT) {
        const int sv = a.start[e];
        s = sv & 0x7fffffff;
        w = sv < 0 ? -wnorm : wnorm;
    } else {
        s = e / a.per;
        w = 1.f;
    }
    x = history_state(a, ekey, e);
}

// FIXED: every history takes exactly History Length steps (no weight
// cutoff), so the lanes of a warp start and finish their histories together:
// the warp takes 32 histories at a time and runs them without per-step
// termination checks.  Otherwise lanes refill one by one from the queue as
// their histories terminate.
template <int S, int DIR, int ST, bool FIXED, int ILP = 1>
__global__ void __launch_bounds__(256, ILP == 1   ? WalkOccupancy<S>::kMinBlocks
                                      : ILP == 2 ? 5
                                      : ILP == 4 ? 4
                                                 : 3)
    walk32(WalkArgs a) {
    static_assert(S % 4 == 0, "records are whole 32-byte halves");
    __shared__ uint64_t s_ekey;
    __shared__ int s_nh;
    __shared__ float s_wnorm;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        s_ekey = epoch_key(a.seed, *a.d_epoch);
        s_nh = *a.d_nh;
        s_wnorm = float(a.sc[0]);
    }
    __syncthreads();
    const char* rec = reinterpret_cast<const char*>(a.rec);
    if (lane == 0) atomicMin(&a.d_tim[0], global_ns());
    unsigned steps = 0;
    if constexpr (FIXED) {
        // ILP histories per lane, interleaved step by step so that each lane
        // has ILP independent record loads in flight.
        const int L = a.L;
        while (true) {
            int base = 0;
            if (lane == 0) base = atomicAdd(a.d_counter, 32 * ILP);
            base = __shfl_sync(kFull, base, 0);
            const int nh = s_nh;
            if (base >= nh) break;
            int s[ILP], s0[ILP];
            float w[ILP], acc[ILP], comp[ILP];
            uint64_t x[ILP];
            bool alive[ILP];
#pragma unroll
            for (int m = 0; m < ILP; ++m) {
                const int e = base + lane + 32 * m;
                alive[m] = e < nh;
                s[m] = 0;
                w[m] = acc[m] = comp[m] = 0.f;
                x[m] = 0;
                if (alive[m]) walk_start<DIR>(a, e, s_ekey, s_wnorm, s[m], w[m], x[m]);
                s0[m] = s[m];
            }
            for (int k = 0; k < L; ++k) {
#pragma unroll
                for (int m = 0; m < ILP; ++m)
                    if (alive[m]) walk_step<S, DIR, ST>(a, rec, s[m], w[m], x[m], acc[m], comp[m], k);
            }
#pragma unroll
            for (int m = 0; m < ILP; ++m) {
                if (alive[m]) {
                    steps += L;
                    if (DIR == MCLSGPU_FORWARD)
                        atomicAdd(&a.y64[s0[m]], double(acc[m]) - double(comp[m]));
                }
            }
        }
    } else {
        int s = 0, s0 = 0, k = 0;
        float w = 0.f, wcut = 0.f, acc = 0.f, comp = 0.f;
        uint64_t x = 0;
        bool alive = false, drained = false;
        while (true) {
            const unsigned need = __ballot_sync(kFull, !alive);
            if (need && !drained) {
                const int leader = __ffs(need) - 1;
                const int cnt = __popc(need);
                const int nh = s_nh;
                int base = 0;
                if (lane == leader) base = atomicAdd(a.d_counter, cnt);
                base = __shfl_sync(kFull, base, leader);
                if (base + cnt >= nh) drained = true;
                if (!alive) {
                    const int e = base + __popc(need & ((1u << lane) - 1));
                    if (e < nh) {
                        walk_start<DIR>(a, e, s_ekey, s_wnorm, s, w, x);
                        acc = 0.f;
                        comp = 0.f;
                        s0 = s;
                        wcut = a.cutoff * fabsf(w);
                        k = 0;
                        alive = true;
                    }
                }
            }
            if (!__any_sync(kFull, alive)) break;
            if (alive) {
                walk_step<S, DIR, ST>(a, rec, s, w, x, acc, comp, k);
                ++k;
                ++steps;
                if (k >= a.L || fabsf(w) < wcut) {
                    alive = false;
                    if (DIR == MCLSGPU_FORWARD)
                        atomicAdd(&a.y64[s0], double(acc) - double(comp));
                }
            }
        }
    }
    // Step count: one reduction per warp.
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) steps += __shfl_down_sync(kFull, steps, d);
    if (lane == 0) {
        if (steps) atomicAdd(a.d_steps, (unsigned long long)steps);
        atomicMax(&a.d_tim[1], global_ns());
    }
}

// Device-side duration of the last walk launch (first warp start to last warp
// end), accumulated into d_tim[2] with the launch count in d_tim[3].
__global__ void k_walk_time_acc(unsigned long long* t) {
    if (t[1] > t[0]) t[2] += t[1] - t[0];
    t[3] += 1;
    t[0] = ~0ULL;
    t[1] = 0;
}

template <int DIR>
__global__ void __launch_bounds__(128) walk64(WalkArgs a) {
    const int nh = *a.d_nh;
    const double weight = a.sc[0];
    const int L = a.L;
    const uint64_t ekey = epoch_key(a.seed, *a.d_epoch);
    unsigned long long steps = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nh;
         e += (long long)gridDim.x * blockDim.x) {
        int s;
        double w;
        if (DIR == MCLSGPU_ADJOINT) {
            const int sv = a.start[e];
            s = sv & 0x7fffffff;
            w = sv < 0 ? -weight : weight;
        } else {
            s = int(e / a.per);
            w = 1.0;
        }
        const int s0 = s;
        const double wcut = a.cutoff64 * fabs(w);
        uint64_t x = history_state(a, ekey, e);
        double acc = 0.0;
        const bool tr = a.tr_states && e < a.max_trace;
        if (tr) {
            for (int t = 0; t <= L; ++t) a.tr_states[e * (L + 1) + t] = -1;
            a.tr_states[e * (L + 1)] = s;
        }
        int k = 0;
        while (true) {
            if (DIR == MCLSGPU_ADJOINT) {
                if (k > 0) atomicAdd(&a.y64[s], w);
            } else {
                acc = __dadd_rn(acc, __dmul_rn(w, a.c64[s]));
            }
            x = xs_step(x);
            const double u = canonical64(x);
            int r0, len;
            int lo = select64(a, s, u, r0, len);
            if (lo >= len) {
                atomicOr(a.status, DEV_ERR_BOUNDS);
                lo = len - 1;
            }
            const double Ws = a.h[r0 + lo] > 0.0 ? a.W[s] : -a.W[s];
            w = __dmul_rn(w, Ws);
            s = a.col[r0 + lo];
            ++k;
            ++steps;
            if (tr) a.tr_states[e * (L + 1) + k] = s;
            if (k >= L || fabs(w) < wcut) break;
        }
        if (!isfinite(w)) atomicOr(a.status, DEV_ERR_NONFINITE);
        if (a.hlen) a.hlen[e] = k;
        if (DIR == MCLSGPU_FORWARD) atomicAdd(&a.y64[s0], acc);
        if (e < a.max_trace) {
            if (a.tr_w) a.tr_w[e] = w;
            if (a.tr_ev) a.tr_ev[e] = 2;  // Event::CUTOFF
            if (a.tr_start) a.tr_start[e] = s0;
        }
    }
    // Step count: one atomic per warp (one per thread serialises on the
    // counter when most threads have no history).
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) steps += __shfl_down_sync(kFull, steps, d);
    if ((threadIdx.x & 31) == 0 && steps) atomicAdd(a.d_steps, steps);
}

template <int S, int DIR, int ST, bool FX, int ILP>
int blocks_per_sm(int block) {
    static int cached[5] = {0, 0, 0, 0, 0};  // block sizes 128..1024 by log2
    const int slot = block <= 128 ? 0 : block <= 256 ? 1 : block <= 512 ? 2 : 3;
    if (!cached[slot]) {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, walk32<S, DIR, ST, FX, ILP>, block, 0);
        cached[slot] = b > 0 ? b : 1;
    }
    return cached[slot];
}

// Dispatch on the record stride; `launch` false only caches the occupancy.
// Persistent grid: as many blocks as fit on every SM at once.
template <int DIR, int ST, bool FX, int ILP>
void launch32_slots(int slots, const WalkArgs& a, int sms, int block, cudaStream_t st,
                    bool launch) {
#define MCLSGPU_WALK_CASE(SL)                                                             \
    case SL:                                                                              \
        if (launch)                                                                       \
            walk32<SL, DIR, ST, FX, ILP>                                                  \
                <<<sms * blocks_per_sm<SL, DIR, ST, FX, ILP>(block), block, 0, st>>>(a);  \
        else                                                                              \
            blocks_per_sm<SL, DIR, ST, FX, ILP>(block);                                   \
        break;
    if constexpr (ILP >= 4) {
        // four or eight histories per lane: 32-byte records only
        switch (slots) {
            default:
                MCLSGPU_WALK_CASE(4)
        }
    } else if constexpr (ILP > 1 || ST == kStencil16) {
        switch (slots) {
            MCLSGPU_WALK_CASE(4)
            default:
                MCLSGPU_WALK_CASE(8)
        }
    } else if constexpr (ST == kStencil) {
        switch (slots) {
            MCLSGPU_WALK_CASE(4)
            MCLSGPU_WALK_CASE(8)
            default:
                MCLSGPU_WALK_CASE(16)
        }
    } else {
        switch (slots) {
            MCLSGPU_WALK_CASE(4)
            MCLSGPU_WALK_CASE(8)
            MCLSGPU_WALK_CASE(12)
            MCLSGPU_WALK_CASE(16)
            MCLSGPU_WALK_CASE(24)
            default:
                MCLSGPU_WALK_CASE(32)
        }
    }
#undef MCLSGPU_WALK_CASE
}

void dispatch_walk32(const mclsgpu_domain* dom, const WalkArgs& a, bool launch) {
    const int sms = dom->ctx->num_sms;
    cudaStream_t st = dom->ctx->stream;
    const bool adj = dom->p.direction == MCLSGPU_ADJOINT;
    const bool fixed = !(dom->p.weight_cutoff > 0.0);
    // Several histories per lane only for fixed-length histories: two on
    // records of at most 8 slots (the register budget of 5 blocks per SM),
    // four or eight on 32-byte records (4 or 3 blocks per SM).
    const bool ilp8 = fixed && dom->walk_ilp == 8 && dom->slots == 4;
    const bool ilp4 = fixed && dom->walk_ilp >= 4 && dom->slots == 4 && !ilp8;
    const bool ilp2 = fixed && dom->walk_ilp >= 2 && dom->slots <= 8 && !ilp4 && !ilp8;
    const int block = dom->walk_block;
#define MCLSGPU_WALK_DIR(DIRV, STV)                                                           \
    (ilp8   ? launch32_slots<DIRV, STV, true, 8>(dom->slots, a, sms, block, st, launch)       \
     : ilp4 ? launch32_slots<DIRV, STV, true, 4>(dom->slots, a, sms, block, st, launch)       \
     : ilp2 ? launch32_slots<DIRV, STV, true, 2>(dom->slots, a, sms, block, st, launch)       \
     : fixed ? launch32_slots<DIRV, STV, true, 1>(dom->slots, a, sms, block, st, launch)      \
             : launch32_slots<DIRV, STV, false, 1>(dom->slots, a, sms, block, st, launch))
    if (dom->stencil_k && dom->rec_q16) {
        if (adj) MCLSGPU_WALK_DIR(MCLSGPU_ADJOINT, kStencil16);
        else MCLSGPU_WALK_DIR(MCLSGPU_FORWARD, kStencil16);
    } else if (dom->stencil_k) {
        if (adj) MCLSGPU_WALK_DIR(MCLSGPU_ADJOINT, kStencil);
        else MCLSGPU_WALK_DIR(MCLSGPU_FORWARD, kStencil);
    } else {
        if (adj) MCLSGPU_WALK_DIR(MCLSGPU_ADJOINT, kPacked);
        else MCLSGPU_WALK_DIR(MCLSGPU_FORWARD, kPacked);
    }
#undef MCLSGPU_WALK_DIR
}

}  // namespace

// Cache the occupancy of the walk kernel this domain will launch (set-up time,
// outside any stream capture).
void prepare_walk(mclsgpu_domain* dom) {
    if (dom->p.precision != MCLSGPU_FP32) return;
    WalkArgs a{};
    dispatch_walk32(dom, a, false);
}

namespace {

// Forward walks shared by the right-hand sides of a batch (batched MCSA): the
// walk does not depend on the source, so each history carries one
// Kahan-compensated FP32 sum of w * c_r(state) per column r of its start
// row's width class (cR holds the tally source of every column at every
// state, in the batch's element layout) and adds them into Y at the start
// row's elements in FP64.  Fixed-length histories only; a history never
// leaves its system, so every state it visits has its start row's width.
struct BatchWalk {
    const float* cR;
    double* Y;
    BatchList list;
    BatchClasses cls;
    int grab;
    int per;
};

// The list entry k with hcum[k] <= h < hcum[k+1] (count entries).
__device__ __forceinline__ int list_entry(const int* hcum, int count, int h) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (hcum[mid] <= h) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// The tally-source row of state s in class c (W = 2^c columns).
template <int W>
__device__ __forceinline__ void load_source_row(const float* p, float (&c)[W]) {
    if constexpr (W >= 4) {
#pragma unroll
        for (int r = 0; r < W; r += 4) {
            const float4 q = __ldg(reinterpret_cast<const float4*>(p + r));
            c[r] = q.x;
            c[r + 1] = q.y;
            c[r + 2] = q.z;
            c[r + 3] = q.w;
        }
    } else if constexpr (W == 2) {
        const float2 q = __ldg(reinterpret_cast<const float2*>(p));
        c[0] = q.x;
        c[1] = q.y;
    } else {
        c[0] = __ldg(p);
    }
}

// One history of a row of class C (2^C columns), returns its steps.
template <int S, bool ST, int C>
__device__ __forceinline__ unsigned batch_history(const WalkArgs& a, const char* rec,
                                                  const BatchWalk& m, int s, float w,
                                                  uint64_t x) {
    constexpr int W = 1 << C;
    const int r0 = m.cls.crow[C];
    const float* cbase = m.cR + m.cls.cel[C];
    const int s0 = s;
    float acc[W], comp[W];
#pragma unroll
    for (int r = 0; r < W; ++r) acc[r] = comp[r] = 0.f;
    const int L = a.L;
    for (int k = 0; k < L; ++k) {
        float c[W];
        load_source_row<W>(cbase + size_t(s - r0) * W, c);
#pragma unroll
        for (int r = 0; r < W; ++r) {
            const float term = w * c[r] - comp[r];
            const float t = acc[r] + term;
            comp[r] = (t - acc[r]) - term;
            acc[r] = t;
        }
        float da = 0.f, dc = 0.f;  // the record header's own tally is unused here
        walk_step<S, MCLSGPU_FORWARD, ST ? kStencil : kPacked>(a, rec, s, w, x, da, dc, k);
    }
    double* y = m.Y + m.cls.cel[C] + size_t(s0 - r0) * W;
#pragma unroll
    for (int r = 0; r < W; ++r)
        if (acc[r] != 0.f || comp[r] != 0.f) atomicAdd(&y[r], double(acc[r]) - double(comp[r]));
    return unsigned(L);
}

template <int S, bool ST>
__global__ void __launch_bounds__(256, 3) walk32_batch(WalkArgs a, BatchWalk m) {
    static_assert(S % 4 == 0, "records are whole 32-byte halves");
    __shared__ uint64_t s_ekey;
    __shared__ int s_nh, s_count;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        s_ekey = epoch_key(a.seed, *a.d_epoch);
        s_count = *m.list.lcount;
        s_nh = s_count > 0 ? m.list.hcum[s_count] : 0;
    }
    __syncthreads();
    const char* rec = reinterpret_cast<const char*>(a.rec);
    if (lane == 0) atomicMin(&a.d_tim[0], global_ns());
    unsigned steps = 0;
    const int chunk = 32 * m.grab;
    const int count = s_count;
    while (true) {
        int base = 0;
        if (lane == 0) base = atomicAdd(a.d_counter, chunk);
        base = __shfl_sync(kFull, base, 0);
        const int nh = s_nh;
        if (base >= nh) break;
        // The list entry of the grab's first history (one search per warp);
        // the lanes step forward from it.
        int k0 = 0;
        if (lane == 0) k0 = list_entry(m.list.hcum, count, base);
        k0 = __shfl_sync(kFull, k0, 0);
        for (int g = 0; g < m.grab; ++g) {
            const int h = base + 32 * g + lane;
            if (h >= nh) break;
            int k = k0;
            while (k + 1 < count && h >= m.list.hcum[k + 1]) ++k;
            const int sys = m.list.lsys[k];
            const int e = m.list.srow0[sys] * m.per + (h - m.list.hcum[k]);
            int s;
            float w;
            uint64_t x;
            walk_start<MCLSGPU_FORWARD>(a, e, s_ekey, 1.f, s, w, x);
            int c = 0;
            while (c < 4 && s >= m.cls.crow[c + 1]) ++c;
            switch (c) {
                case 0: steps += batch_history<S, ST, 0>(a, rec, m, s, w, x); break;
                case 1: steps += batch_history<S, ST, 1>(a, rec, m, s, w, x); break;
                case 2: steps += batch_history<S, ST, 2>(a, rec, m, s, w, x); break;
                case 3: steps += batch_history<S, ST, 3>(a, rec, m, s, w, x); break;
                default: steps += batch_history<S, ST, 4>(a, rec, m, s, w, x); break;
            }
        }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) steps += __shfl_down_sync(kFull, steps, d);
    if (lane == 0) {
        if (steps) atomicAdd(a.d_steps, (unsigned long long)steps);
        atomicMax(&a.d_tim[1], global_ns());
    }
}

template <int S, bool ST>
void launch_batch_s(const WalkArgs& a, const BatchWalk& m, int sms, int block, cudaStream_t st) {
    static int cached[2] = {0, 0};
    const int slot = block == 128 ? 0 : 1;
    if (!cached[slot]) {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, walk32_batch<S, ST>, block, 0);
        cached[slot] = b > 0 ? b : 1;
    }
    walk32_batch<S, ST><<<sms * cached[slot], block, 0, st>>>(a, m);
}

}  // namespace

// Fill the walk arguments of a domain (shared by the single- and the
// multi-right-hand-side walks).
static void fill_walk_args(mclsgpu_domain* dom, WalkArgs& a) {
    mclsgpu_context* ctx = dom->ctx;
    const mclsgpu_mc_params& p = dom->p;
    a.n = dom->n;
    a.L = p.history_length;
    a.per = p.sample_ratio > 0.0 ? int(ceil(p.sample_ratio)) : 1;
    a.rng_mode = p.rng_mode;
    a.d_nh = dom->d_nh;
    a.d_counter = dom->d_counter;
    a.start = dom->start;
    a.sc = dom->d_scalars;
    a.seed = dom->seed;
    a.d_epoch = dom->d_epoch;
    a.jump = dom->d_jump;
    a.d_pos = dom->d_pos;
    a.rec = dom->rec;
    a.d_steps = dom->d_steps;
    a.d_tim = dom->d_tim;
    a.status = ctx->d_status;
    a.l1 = dom->walk_l1;
    for (int j = 0; j < 32; ++j) a.stoff[j] = dom->stencil_off[j];
}

// Batched forward walks over the domain's FP32 records (records of at most
// 16 slots; see launch_walk_batch in internal.h).
int launch_walk_batch(mclsgpu_domain* dom, const BatchClasses& cls, const BatchList& list,
                      const float* cR, double* Y, int grab) {
    mclsgpu_context* ctx = dom->ctx;
    if (dom->p.precision != MCLSGPU_FP32 || dom->p.direction != MCLSGPU_FORWARD || !dom->slots ||
        dom->rec_q16)
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                         "batched walks need FP32 forward packed or stencil records");
    if (grab < 1 || grab > 8)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "batched walks: grab %d not in 1..8", grab);
    WalkArgs a{};
    fill_walk_args(dom, a);
    const int sms = ctx->num_sms;
    const int block = dom->walk_block;
    cudaStream_t st = ctx->stream;
    const BatchWalk m{cR, Y, list, cls, grab, a.per};
    bool ok = true;
    if (dom->stencil_k) {
        switch (dom->slots) {
            case 4: launch_batch_s<4, true>(a, m, sms, block, st); break;
            case 8: launch_batch_s<8, true>(a, m, sms, block, st); break;
            default: ok = false;
        }
    } else {
        switch (dom->slots) {
            case 4: launch_batch_s<4, false>(a, m, sms, block, st); break;
            case 8: launch_batch_s<8, false>(a, m, sms, block, st); break;
            case 12: launch_batch_s<12, false>(a, m, sms, block, st); break;
            case 16: launch_batch_s<16, false>(a, m, sms, block, st); break;
            default: ok = false;
        }
    }
    if (!ok)
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "batched walks: %d-slot records not supported",
                         dom->slots);
    return MCLSGPU_OK;
}

__global__ void k_fill_offsets(int* hoff, const int* d_nh, int L) {
    const int nh = *d_nh;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nh; e += gridDim.x * blockDim.x)
        hoff[e] = e * L;
}

// hoff2 (exclusive prefix of the lengths) against hoff: *changed = 1 when
// any offset moved; hoff takes the new offsets.
__global__ void k_update_offsets(int* hoff, const int* hoff2, const int* d_nh, int* changed) {
    const int nh = *d_nh;
    int c = 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nh; e += gridDim.x * blockDim.x) {
        if (hoff[e] != hoff2[e]) {
            c = 1;
            hoff[e] = hoff2[e];
        }
    }
    if (__syncthreads_or(c) && threadIdx.x == 0) atomicOr(changed, 1);
}

__global__ void k_advance_pos_by(unsigned long long* d_pos, long long draws) { *d_pos += draws; }

// Variable-length histories on the reference stream (a Weight Cutoff with
// "Reproducible MC Mode"): the reference draws history e's uniforms right
// after history e-1's, so e's first draw depends on every earlier length.
// Round 1 walks with offsets e * L; each later round walks again with the
// offsets the previous round's lengths give, until no offset moves.  The
// histories before the first moved offset are final after each round, so the
// rounds end (at most one more than the histories); in practice lengths
// repeat and a few rounds suffice.  Tallies and the step count are restored
// before each repeated round.  Host-synchronous.
static void walk_reference_rounds(mclsgpu_domain* dom, WalkArgs a, int grid) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t st = ctx->stream;
    const int n = dom->n;
    const int L = dom->p.history_length;
    int nh = 0;
    unsigned long long steps0 = 0;
    cudaMemcpyAsync(&nh, dom->d_nh, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&steps0, dom->d_steps, sizeof(steps0), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(dom->y_save, dom->y64, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice,
                    st);
    k_fill_offsets<<<grid, 128, 0, st>>>(dom->hoff, dom->d_nh, L);
    a.hoff = dom->hoff;
    a.hlen = dom->hlen;
    int* changed = reinterpret_cast<int*>(dom->hoff2 + dom->nh_cap + 1);
    long long total = 0;
    int rounds = 0;
    for (;;) {
        ++rounds;
        if (dom->p.direction == MCLSGPU_ADJOINT)
            walk64<MCLSGPU_ADJOINT><<<grid, 128, 0, st>>>(a);
        else
            walk64<MCLSGPU_FORWARD><<<grid, 128, 0, st>>>(a);
        if (nh == 0 || exclusive_scan_counts_dev(ctx, dom->hlen, nh, dom->hoff2, &total)) break;
        cudaMemsetAsync(changed, 0, sizeof(int), st);
        k_update_offsets<<<grid, 128, 0, st>>>(dom->hoff, dom->hoff2, dom->d_nh, changed);
        int h_changed = 0;
        cudaMemcpyAsync(&h_changed, changed, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess || !h_changed || rounds > nh) break;
        cudaMemcpyAsync(dom->y64, dom->y_save, size_t(n) * sizeof(double),
                        cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(dom->d_steps, &steps0, sizeof(steps0), cudaMemcpyHostToDevice, st);
    }
    dom->walk_rounds = rounds;
    k_advance_pos_by<<<1, 1, 0, st>>>(dom->d_pos, total);
}

// Launch the walks of the current source.  Trace arrays only with FP64.
// `fused`: the work-queue counter reset and the timing accumulation are done
// by the fused residual kernel that follows the walk (MCSA loop).
void launch_walk(mclsgpu_domain* dom, long long max_trace, long long* tr_states, double* tr_w,
                 int* tr_ev, long long* tr_start, bool fused) {
    mclsgpu_context* ctx = dom->ctx;
    const mclsgpu_mc_params& p = dom->p;
    WalkArgs a{};
    fill_walk_args(dom, a);
    a.cutoff = float(p.weight_cutoff > 0.0 ? p.weight_cutoff : 0.0);
    a.cutoff64 = p.weight_cutoff > 0.0 ? p.weight_cutoff : 0.0;
    a.rp = dom->D.rp;
    a.col = dom->D.ci;
    a.h = dom->D.v;
    a.cdf = dom->cdf;
    a.W = dom->w;
    a.y64 = dom->y64;
    a.c32 = dom->c32;
    a.c64 = dom->c64;
    a.max_trace = max_trace;
    a.tr_states = tr_states;
    a.tr_w = tr_w;
    a.tr_ev = tr_ev;
    a.tr_start = tr_start;
    cudaStream_t st = ctx->stream;
    if (p.precision == MCLSGPU_FP32) {
        if (!fused) cudaMemsetAsync(dom->d_counter, 0, sizeof(int), st);
        dispatch_walk32(dom, a, true);
        if (!fused) k_walk_time_acc<<<1, 1, 0, st>>>(dom->d_tim);
    } else {
        // One thread per history up to 8 blocks per SM (the kernel strides
        // beyond that); no more blocks than the history capacity needs.
        long long g = (dom->nh_cap + 127) / 128;
        if (g < 1) g = 1;
        const int grid = int(g < ctx->num_sms * 8 ? g : ctx->num_sms * 8);
        if (walk_needs_rounds(dom))
            walk_reference_rounds(dom, a, grid);
        else if (p.direction == MCLSGPU_ADJOINT)
            walk64<MCLSGPU_ADJOINT><<<grid, 128, 0, st>>>(a);
        else
            walk64<MCLSGPU_FORWARD><<<grid, 128, 0, st>>>(a);
    }
}

// ---- row-partitioned domains (domain-decomposed transport) -----------------
//
// One part holds the records and tallies of rows [row0, row0 + n).  A
// history walks while its state stays in the part; when a transition takes
// it to another part's row and the history goes on (steps left, weight above
// the cutoff), it is written to that part's outbox (HistoryWire: Xorshift
// state, state, step, weight and, forward, its running sum) and continues
// there in a later round, on the same random stream.  An adjoint history
// tallies where it stands, so its tallies land in the parts it visits.  A
// forward history's sum belongs to its start row: when it ends outside the
// part that owns that row, the sum travels there as a tally return (state
// -1).  Every transition and tally is therefore the one the whole-domain walk
// would make.
namespace {

__device__ __forceinline__ int part_owner(const int* sb, int nparts, int s) {
    int lo = 0, up = nparts;  // sb[lo] <= s < sb[lo + 1]
    while (up - lo > 1) {
        const int mid = (lo + up) >> 1;
        if (sb[mid] <= s) lo = mid; else up = mid;
    }
    return lo;
}

__device__ __forceinline__ void part_send(const PartWalk& p, int q, const HistoryWire& h) {
    const unsigned long long slot = atomicAdd(&p.out_cnt[q], 1ULL);
    if (slot < (unsigned long long)p.cap)
        p.out[size_t(q) * size_t(p.cap) + slot] = h;
    else
        atomicOr(p.status, DEV_ERR_CAPACITY);
}

template <int S, int DIR, int ST>
__global__ void __launch_bounds__(256) walk32_part(PartWalk p) {
    __shared__ int sb[kMaxParts + 1];
    for (int t = threadIdx.x; t <= p.nparts; t += blockDim.x) sb[t] = p.bounds[t];
    __syncthreads();
    WalkArgs a{};
    a.y64 = p.y;
    a.row0 = p.row0;
    if constexpr (ST != kPacked) {
#pragma unroll
        for (int j = 0; j < 32; ++j) a.stoff[j] = p.stoff[j];
    }
    const uint64_t ekey = epoch_key(p.seed, *p.d_epoch);
    const float wnorm = DIR == MCLSGPU_ADJOINT ? float(p.sc[0]) : 1.f;
    const float wcut = p.cutoff * wnorm;
    const long long nwork = p.in ? p.n_in : p.e_end - p.e_begin;
    const char* rec = reinterpret_cast<const char*>(p.rec);
    const int hi = p.row0 + p.n;
    unsigned steps = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nwork;
         t += (long long)gridDim.x * blockDim.x) {
        int s, k, id;
        float w, acc = 0.f, comp = 0.f;
        uint64_t x;
        if (p.in) {
            const HistoryWire h = p.in[t];
            if (DIR == MCLSGPU_FORWARD && h.state < 0) {  // a tally return
                const int s0 = h.id / p.per;
                if (s0 < p.row0 || s0 >= hi)
                    atomicOr(p.status, DEV_ERR_BOUNDS);
                else
                    atomicAdd(&p.y[s0 - p.row0], double(h.acc) - double(h.comp));
                continue;
            }
            s = h.state;
            k = h.step;
            w = h.weight;
            x = h.rng;
            id = h.id;
            acc = h.acc;
            comp = h.comp;
        } else {
            const long long e = p.e_begin + t;
            if (DIR == MCLSGPU_ADJOINT) {
                const int sv = p.start[e];
                s = sv & 0x7fffffff;
                w = sv < 0 ? -wnorm : wnorm;
            } else {
                s = int(e / p.per);
                w = 1.f;
            }
            x = counter_state(ekey, 2, uint64_t(e));
            k = 0;
            id = int(e);
        }
        if (s < p.row0 || s >= hi) {  // not this part's history
            atomicOr(p.status, DEV_ERR_BOUNDS);
            continue;
        }
        while (true) {
            walk_step<S, DIR, ST>(a, rec, s, w, x, acc, comp, k);
            ++k;
            ++steps;
            if (k >= p.L || fabsf(w) < wcut) {
                if (DIR == MCLSGPU_FORWARD) {
                    const int s0 = id / p.per;
                    if (s0 >= p.row0 && s0 < hi) {
                        atomicAdd(&p.y[s0 - p.row0], double(acc) - double(comp));
                    } else {
                        HistoryWire h;
                        h.rng = 0;
                        h.state = -1;
                        h.step = k;
                        h.weight = w;
                        h.id = id;
                        h.acc = acc;
                        h.comp = comp;
                        part_send(p, part_owner(sb, p.nparts, s0), h);
                    }
                }
                break;
            }
            if (s < p.row0 || s >= hi) {
                HistoryWire h;
                h.rng = x;
                h.state = s;
                h.step = k;
                h.weight = w;
                h.id = id;
                h.acc = acc;
                h.comp = comp;
                part_send(p, part_owner(sb, p.nparts, s), h);
                break;
            }
        }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) steps += __shfl_down_sync(kFull, steps, d);
    if ((threadIdx.x & 31) == 0 && steps) atomicAdd(p.d_steps, (unsigned long long)steps);
}

// FP32-versus-FP64 transition agreement.  History e starts at state e mod n
// on its counter stream and walks `L` transitions along the FP64 domain
// (walk64's selection with u = canonical64(x)); at every transition the FP32
// record of the same state is searched with u = canonical32(x) of the same
// draw (walk32's selection).  A transition disagrees when the two select a
// different column or sign; out[0] += histories with at least one
// disagreement, out[1] += disagreeing transitions.
template <int S, int ST>
__global__ void __launch_bounds__(256) k_walk_agreement(WalkArgs a, long long nh, uint64_t ekey,
                                                        unsigned long long* out) {
    const char* rec = reinterpret_cast<const char*>(a.rec);
    unsigned long long hd = 0, td = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nh;
         e += (long long)gridDim.x * blockDim.x) {
        int s = int(e % a.n);
        uint64_t x = counter_state(ekey, 2, uint64_t(e));
        bool differ = false;
        for (int k = 0; k < a.L; ++k) {
            uint32_t q[2 * S];
            const char* r = rec + size_t(s) * (S * 8);
#pragma unroll
            for (int t = 0; t < S / 4; ++t) ld_record256(r + 32 * t, q + 8 * t);
            x = xs_step(x);
            int s32 = s;
            unsigned neg32;
            select32<S, ST>(a, q, x, s32, neg32);
            int r0, len;
            int j = select64(a, s, canonical64(x), r0, len);
            if (j >= len) {
                atomicOr(a.status, DEV_ERR_BOUNDS);
                j = len - 1;
            }
            const int s64 = a.col[r0 + j];
            const bool neg64 = !(a.h[r0 + j] > 0.0);
            if (s32 != s64 || (neg32 != 0u) != neg64) {
                ++td;
                differ = true;
            }
            s = s64;
        }
        hd += differ ? 1 : 0;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        hd += __shfl_down_sync(kFull, hd, d);
        td += __shfl_down_sync(kFull, td, d);
    }
    if ((threadIdx.x & 31) == 0) {
        if (hd) atomicAdd(&out[0], hd);
        if (td) atomicAdd(&out[1], td);
    }
}

}  // namespace

int walk_agreement(mclsgpu_domain* dom, long long histories, uint64_t seed, long long* hist_diff,
                   long long* trans_diff) {
    mclsgpu_context* ctx = dom->ctx;
    if (dom->p.precision != MCLSGPU_FP32 || !dom->rec)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "walk agreement needs FP32 records");
    if (histories < 1) return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "histories < 1");
    WalkArgs a{};
    fill_walk_args(dom, a);
    a.rp = dom->D.rp;
    a.col = dom->D.ci;
    a.h = dom->D.v;
    a.cdf = dom->cdf;
    a.W = dom->w;
    unsigned long long* d_out = nullptr;
    cudaError_t e = dmalloc(&d_out, 2);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    cudaStream_t st = ctx->stream;
    cudaMemsetAsync(d_out, 0, 2 * sizeof(unsigned long long), st);
    const long long g = (histories + 255) / 256;
    const int grid = int(g < ctx->num_sms * 8 ? g : ctx->num_sms * 8);
    const uint64_t ekey = epoch_key(seed, 0);
    bool ok = true;
#define MCLSGPU_AGREE(SL, STV) k_walk_agreement<SL, STV><<<grid, 256, 0, st>>>(a, histories, ekey, d_out)
    if (dom->stencil_k && dom->rec_q16) {
        switch (dom->slots) {
            case 4: MCLSGPU_AGREE(4, kStencil16); break;
            case 8: MCLSGPU_AGREE(8, kStencil16); break;
            default: ok = false;
        }
    } else if (dom->stencil_k) {
        switch (dom->slots) {
            case 4: MCLSGPU_AGREE(4, kStencil); break;
            case 8: MCLSGPU_AGREE(8, kStencil); break;
            case 16: MCLSGPU_AGREE(16, kStencil); break;
            default: ok = false;
        }
    } else {
        switch (dom->slots) {
            case 4: MCLSGPU_AGREE(4, kPacked); break;
            case 8: MCLSGPU_AGREE(8, kPacked); break;
            case 12: MCLSGPU_AGREE(12, kPacked); break;
            case 16: MCLSGPU_AGREE(16, kPacked); break;
            case 24: MCLSGPU_AGREE(24, kPacked); break;
            case 32: MCLSGPU_AGREE(32, kPacked); break;
            default: ok = false;
        }
    }
#undef MCLSGPU_AGREE
    unsigned long long h[2] = {0, 0};
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_out, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    dfree(d_out);
    if (!ok) return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "walk agreement: %d-slot records",
                              dom->slots);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "walk agreement");
    int rc = check_device_status(ctx);
    if (rc) return rc;
    *hist_diff = (long long)h[0];
    *trans_diff = (long long)h[1];
    return MCLSGPU_OK;
}

void launch_walk_part(const PartWalk& p, mclsgpu_context* ctx) {
    const long long nwork = p.in ? p.n_in : p.e_end - p.e_begin;
    if (nwork <= 0) return;
    long long g = (nwork + 255) / 256;
    const int grid = int(g < ctx->num_sms * 8 ? g : ctx->num_sms * 8);
    cudaStream_t st = ctx->stream;
#define MCLSGPU_PART_SLOTS(D)                                                 \
    if (p.kind == kStencil16) {                                               \
        if (p.slots == 4) walk32_part<4, D, kStencil16><<<grid, 256, 0, st>>>(p);  \
        else walk32_part<8, D, kStencil16><<<grid, 256, 0, st>>>(p);            \
    } else if (p.kind == kStencil) {                                          \
        switch (p.slots) {                                                    \
            case 4: walk32_part<4, D, kStencil><<<grid, 256, 0, st>>>(p); break;   \
            case 8: walk32_part<8, D, kStencil><<<grid, 256, 0, st>>>(p); break;   \
            default: walk32_part<16, D, kStencil><<<grid, 256, 0, st>>>(p); break; \
        }                                                                     \
    } else {                                                                  \
        switch (p.slots) {                                                    \
            case 4: walk32_part<4, D, kPacked><<<grid, 256, 0, st>>>(p); break;   \
            case 8: walk32_part<8, D, kPacked><<<grid, 256, 0, st>>>(p); break;   \
            case 12: walk32_part<12, D, kPacked><<<grid, 256, 0, st>>>(p); break; \
            case 16: walk32_part<16, D, kPacked><<<grid, 256, 0, st>>>(p); break; \
            case 24: walk32_part<24, D, kPacked><<<grid, 256, 0, st>>>(p); break; \
            default: walk32_part<32, D, kPacked><<<grid, 256, 0, st>>>(p); break; \
        }                                                                     \
    }
    if (p.dir == MCLSGPU_FORWARD) {
        MCLSGPU_PART_SLOTS(MCLSGPU_FORWARD)
    } else {
        MCLSGPU_PART_SLOTS(MCLSGPU_ADJOINT)
    }
#undef MCLSGPU_PART_SLOTS
}

}  // namespace mclsgpu
