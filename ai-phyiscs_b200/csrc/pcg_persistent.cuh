// Persistent block-Jacobi PCG over one or many cloth instances.
//
// One cooperative launch runs the whole solve: the CTAs stay resident and
// meet at a software grid barrier twice per iteration (after A p, after the
// x/r/z update), replacing the reference's 8 launches per iteration
// (src/solver/pcg_solver.cu:542-592) and the two-kernel graph loop.  The same
// kernel solves a packed batch: every instance owns a contiguous range of
// 32-row slices, keeps its own rho/alpha/beta/iteration count, and stops
// (its rows are skipped) when ||r_b|| <= tol ||b_b|| or max_iter is reached;
// the kernel ends when every instance is done.
//
// Reductions are deterministic: per-slice FP64 warp sums -> per-(CTA,
// instance) segment sums in fixed slice order -> per-instance totals summed
// over the segment slots in CTA order by every CTA that needs them.
//
// The barrier waits are bounded (globaltimer); on a timeout a CTA raises
// the barrier's error flag, every CTA leaves the loop at its next barrier,
// and the solve status becomes kSolveKernelError so the caller's buffers
// are left untouched.
#pragma once

#include "cloth_kernels.cuh"
#include "coarse_types.h"

namespace chysx_b200 {

constexpr int kSolveKernelError = 3;
constexpr int kSlotW = 8;      // doubles per reduction slot and per slice partial
constexpr int kStartW = 8;     // start partials (the first phase)
constexpr int kCoarseOff = 2;  // slot entry where the coarse values start (after up to 2 scalars):
                               // up to 12 floats (48 bytes) there
constexpr int kCoarsePartW = 12;  // per-slice coarse partials (floats), beside the slice partials
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s

struct alignas(128) GridBarrier {
    unsigned count;
    unsigned pad0[31];
    unsigned gen;
    unsigned pad1[31];
    int error;
    unsigned ndone;  // instances finished
    unsigned pad2[30];
};

struct InstState {
    double rho, rr, bb, tol2, rr0;
    int iter, status, done, fallback;
};

struct BatchPlan {
    int n_inst;
    int max_slices_per_cta;
    int max_inst_per_cta;
    const int* __restrict__ slice_inst;   // [n_slices] instance of each slice
    const int* __restrict__ inst_slice;   // [n_inst + 1] slice range of each instance
    const int* __restrict__ cta_slice;    // [grid + 1] slice range of each CTA
    const int* __restrict__ cta_inst_lo;  // [grid] first instance a CTA touches
    const int* __restrict__ cta_inst_hi;  // [grid] last instance (inclusive), lo-1 if none
    const int* __restrict__ inst_cta_lo;  // [n_inst] first CTA touching an instance
    const int* __restrict__ inst_slot;    // [n_inst + 1] segment-slot ranges
    double* slots;                        // [inst_slot[n_inst] * kSlotW]
    InstState* inst;                      // [n_inst]
    GridBarrier* bar;
    int n_slots = 0;                      // inst_slot[n_inst]
    unsigned long long* fslots = nullptr; // [3][n_slots][kSlotW] rotating polled slots (SYNC = 1)
    // coarse level of the two-level preconditioner, in device memory (null:
    // none); a pointer keeps this kernel parameter small (carrying the whole
    // struct here slowed the streamed kernel by ~17 us per iteration)
    const CoarseArgs* cg = nullptr;
};

// (z, p) of one row for the register-resident kernel's neighbour exchange
struct ZP {
    float4 z;
    float4 p;
};

// CTA-local copy of one instance's solver state plus, set once per solve,
// where its slices and reduction slots are (kept in shared memory so the
// per-phase work reads no global metadata).
struct LocalInst {
    double rho, rr, bb, tol2, sigma;
    float alpha, beta;
    float scale, scale_b;  // warm guess factor c and 1 - c
    int iter, done, status, fallback;
    int b;                 // instance id
    int seg_lo, seg_hi;    // this CTA's slices of it, relative to the CTA's first slice
    int own_slot;          // this CTA's segment slot
    int slot_lo, slot_hi;  // the instance's segment slots
    int first;             // this CTA publishes the instance's state
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Count-based grid barrier, run by one thread (lane 0 of warp 0): a
// fire-and-forget release reduction on a monotonic counter, then acquire
// loads until it reaches this barrier's target.  The wait is bounded in
// time; returns false once any CTA flagged an error.
__device__ __forceinline__ bool barrier_arrive_wait(GridBarrier* gb, unsigned& target) {
    target += gridDim.x;
    red_release_add(&gb->count, 1u);
    const unsigned long long t0 = global_ns();
    unsigned spins = 0;
    while ((int)(ld_acquire_gpu(&gb->count) - target) < 0) {
        if ((++spins & 255u) == 0) {
            if (*(volatile int*)&gb->error) return false;
            if (global_ns() - t0 > kBarrierTimeoutNs) {
                atomicExch(&gb->error, 1);
                return false;
            }
        }
    }
    return *(volatile int*)&gb->error == 0;
}

// The wait of barrier_arrive_wait without the arrival, for a second warp of
// a CTA whose first warp arrives: returns once the counter reaches `target`
// (bounded in time like the barrier; false on an error).
__device__ __forceinline__ bool barrier_wait_only(GridBarrier* gb, unsigned target) {
    const unsigned long long t0 = global_ns();
    unsigned spins = 0;
    while ((int)(ld_acquire_gpu(&gb->count) - target) < 0) {
        if ((++spins & 255u) == 0) {
            if (*(volatile int*)&gb->error) return false;
            if (global_ns() - t0 > kBarrierTimeoutNs) {
                atomicExch(&gb->error, 1);
                return false;
            }
        }
    }
    return *(volatile int*)&gb->error == 0;
}

__device__ __forceinline__ float4 ldcg4(const float4* p) { return __ldcg(p); }

// ---------------------------------------------------------------------------
// Slot-polling synchronisation (kernels instantiated with SYNC = 1).
//
// Instead of a grid-wide counter followed by a read of the partial sums,
// every reduction phase ph publishes each CTA's per-instance partial sums in
// slot set ph % 3 (each value stored after a release fence), and the CTAs
// of an instance poll that instance's slots until every segment is there:
// the poll is both the barrier and the data read.  A slot holds kSlotEmpty
// until written; its owner resets the set-(ph-1) copy during phase ph, after
// seeing every segment of phase ph: each reader published its phase-ph
// segment after reading phase ph-1, so no reader still needs the old value,
// and a reader of phase ph+2 (same set) has acquired the owner's phase-ph+1
// value, which orders the reset before it.  An instance waits only for its
// own CTAs, and a CTA whose instances are all done leaves the kernel.  Waits
// are bounded like the counter barrier's and raise the same error flag.
// ---------------------------------------------------------------------------
// a NaN payload no arithmetic produces; published NaNs are canonicalised
constexpr unsigned long long kSlotEmpty = 0x7FF4C10E5107E000ull;
constexpr int kPollMax = 5;  // slots per lane in flight: one pass covers 160 CTAs
// CTA-local Chebyshev preconditioner: power iterations for the block's
// lambda_max and the margin put on the estimate (24 iterations from a +-1
// vector land within 4% below lambda_max on cloth blocks)
constexpr int kPcPowerIts = 24;
constexpr double kPcMargin = 1.1;
// fixed pseudo-random sign of vector entry q (multiplicative hash)
__device__ __forceinline__ float pc_sign(unsigned q) { return ((q * 2654435761u) >> 31) ? -1.0f : 1.0f; }

__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long slot_bits(double x) {
    return isnan(x) ? 0x7FF8000000000000ull : (unsigned long long)__double_as_longlong(x);
}

// Waits for every segment of instance L in slot set `set` and sums them in
// the same order as the counter-barrier read (ascending slot per lane, then
// an xor tree), so both modes give identical iterates; lane 0 then resets
// this CTA's slot of the previous set.  Returns false on every lane once the
// wait timed out or another CTA raised the error flag.
template <int NV, int KP>
__device__ __forceinline__ bool poll_total(const BatchPlan& bp, const LocalInst& L, int set, double (&out)[NV]) {
    const int lane = threadIdx.x & 31;
    const int lo = L.slot_lo, hi = L.slot_hi;
    const unsigned long long* base = bp.fslots + (size_t)set * bp.n_slots * kSlotW;
#pragma unroll
    for (int q = 0; q < NV; ++q) out[q] = 0.0;
    bool ok = true;
    for (int c0 = lo; c0 < hi && ok; c0 += 32 * KP) {
        unsigned long long val[KP][NV];
#pragma unroll
        for (int j = 0; j < KP; ++j) {
            const int k = c0 + j * 32 + lane;
#pragma unroll
            for (int q = 0; q < NV; ++q) val[j][q] = k < hi ? ld_relaxed_u64(base + (size_t)k * kSlotW + q) : 0ull;
        }
        const unsigned long long t0 = global_ns();
        unsigned spins = 0;
        while (true) {
            bool pending = false;
#pragma unroll
            for (int j = 0; j < KP; ++j) {
                const int k = c0 + j * 32 + lane;
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    if (val[j][q] == kSlotEmpty) {
                        pending = true;
                        val[j][q] = ld_relaxed_u64(base + (size_t)k * kSlotW + q);
                    }
                }
            }
            if (!pending) break;
            if ((++spins & 63u) == 0) {
                if (*(volatile int*)&bp.bar->error) { ok = false; break; }
                if (global_ns() - t0 > kBarrierTimeoutNs) {
                    atomicExch(&bp.bar->error, 1);
                    ok = false;
                    break;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < KP; ++j) {
            if (c0 + j * 32 + lane < hi) {
#pragma unroll
                for (int q = 0; q < NV; ++q) out[q] += __longlong_as_double((long long)val[j][q]);
            }
        }
    }
    fence_acq_rel_gpu();  // acquire: the publishers' data is visible from here on
#pragma unroll
    for (int q = 0; q < NV; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) out[q] += __shfl_xor_sync(0xffffffffu, out[q], o);
    }
    ok = __all_sync(0xffffffffu, ok);
    if (ok && lane == 0) {
        unsigned long long* d = bp.fslots + ((size_t)((set + 2) % 3) * bp.n_slots + L.own_slot) * kSlotW;
#pragma unroll
        for (int q = 0; q < kSlotW; ++q) st_relaxed_u64(d + q, kSlotEmpty);
    }
    return ok;
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

__device__ __forceinline__ double dot3d(float3 a, float3 b) {
    return (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z;
}

// ---------------------------------------------------------------------------
// Per-instance bookkeeping
// ---------------------------------------------------------------------------
// Where this CTA's instances live (all threads of the CTA, once per solve;
// a __syncthreads must follow).
__device__ __forceinline__ void init_local(const BatchPlan& bp, LocalInst* li, int s0, int s1, int il0, int il1) {
    for (int t = threadIdx.x; t <= il1 - il0; t += blockDim.x) {
        const int b = il0 + t;
        LocalInst& L = li[t];
        L.b = b;
        L.seg_lo = max(s0, bp.inst_slice[b]) - s0;
        L.seg_hi = min(s1, bp.inst_slice[b + 1]) - s0;
        L.slot_lo = bp.inst_slot[b];
        L.slot_hi = bp.inst_slot[b + 1];
        L.own_slot = L.slot_lo + ((int)blockIdx.x - bp.inst_cta_lo[b]);
        L.first = (int)blockIdx.x == bp.inst_cta_lo[b];
        L.done = 0;
        L.iter = 0;
        L.status = kSolveConverged;
        L.fallback = 0;
    }
}

// Publication of one reduction phase, run by warp 0 after a __syncthreads:
// sums the slice partials spart[slice * kSlotW + q] (q < NV) of every
// unfinished instance of the CTA and stores the CTA's segment (plain store
// in counter mode; release fence + relaxed stores in polled mode).
template <int NV, int SYNC>
__device__ __forceinline__ void warp0_publish(const BatchPlan& bp, const double* spart, const LocalInst* li, int nloc,
                                              int set) {
    const int lane = threadIdx.x & 31;
    for (int t = 0; t < nloc; ++t) {
        const LocalInst& L = li[t];
        if (L.done) continue;
        double acc[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] = 0.0;
        for (int sl = L.seg_lo + lane; sl < L.seg_hi; sl += 32) {
#pragma unroll
            for (int q = 0; q < NV; ++q) acc[q] += spart[sl * kSlotW + q];
        }
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] = warp_sum(acc[q]);
        if (lane == 0) {
            if (SYNC) {
                unsigned long long* d = bp.fslots + ((size_t)set * bp.n_slots + L.own_slot) * kSlotW;
                fence_acq_rel_gpu();  // release: the CTA's writes before the __syncthreads
#pragma unroll
                for (int q = 0; q < NV; ++q) st_relaxed_u64(d + q, slot_bits(acc[q]));
            } else {
#pragma unroll
                for (int q = 0; q < NV; ++q) bp.slots[((size_t)set * bp.n_slots + L.own_slot) * kSlotW + q] = acc[q];
            }
        }
    }
}

// The counter-mode read of a phase (after the barrier): every instance's
// totals of the first NR values, all of a lane's slots in flight at once
// (fixed unroll), summed in ascending slot order; lane 0 applies `step`.
template <int NR, int KP, class Step>
__device__ __forceinline__ void warp0_read_totals(const BatchPlan& bp, LocalInst* li, int nloc, int set, Step&& step) {
    const int lane = threadIdx.x & 31;
    for (int t = 0; t < nloc; ++t) {
        LocalInst& L = li[t];
        if (L.done) continue;
        double tot[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) tot[q] = 0.0;
        for (int c0 = L.slot_lo; c0 < L.slot_hi; c0 += 32 * KP) {
            double val[KP][NR];
#pragma unroll
            for (int j = 0; j < KP; ++j) {
                const int k = c0 + j * 32 + lane;
#pragma unroll
                for (int q = 0; q < NR; ++q)
                    val[j][q] = k < L.slot_hi ? __ldcg(bp.slots + ((size_t)set * bp.n_slots + k) * kSlotW + q) : 0.0;
            }
#pragma unroll
            for (int j = 0; j < KP; ++j) {
                if (c0 + j * 32 + lane < L.slot_hi) {
#pragma unroll
                    for (int q = 0; q < NR; ++q) tot[q] += val[j][q];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NR; ++q) tot[q] = warp_sum(tot[q]);
        if (lane == 0) step(L, tot);
        __syncwarp();
    }
}

// One reduction phase, run by warp 0 between two __syncthreads: publishes
// the CTA's segments, waits for the other CTAs (counter barrier or polled
// slots), reads each instance's total in a fixed order and lets lane 0
// apply `step(L, total)`.  For instances spanning at most 32 * KP CTAs (one
// pass of loads).  Returns false (on all lanes) after a failed wait.
template <int NV, int SYNC, int KP, class Step>
__device__ __forceinline__ bool warp0_phase(const BatchPlan& bp, const double* spart, LocalInst* li, int nloc,
                                            int set, unsigned& target, Step&& step) {
    const int lane = threadIdx.x & 31;
    warp0_publish<NV, SYNC>(bp, spart, li, nloc, set);
    if constexpr (!SYNC) {
        bool ok = true;
        if (lane == 0) ok = barrier_arrive_wait(bp.bar, target);
        if (!__shfl_sync(0xffffffffu, ok, 0)) return false;
        warp0_read_totals<NV, KP>(bp, li, nloc, set, step);
        return true;
    } else {
        for (int t = 0; t < nloc; ++t) {
            LocalInst& L = li[t];
            if (L.done) continue;
            double tot[NV];
            if (!poll_total<NV, KP>(bp, L, set, tot)) return false;
            if (lane == 0) step(L, tot);
            __syncwarp();
        }
        return true;
    }
}

// ---- coarse level of a single-instance two-level plan (counter barrier) --
// Its parameters, read once per solve (into registers, or shared memory
// where registers are short): every grid barrier ends in an acquire, which
// invalidates L1, so a field read through bp.cg after a barrier would put an
// L2 round trip on the phase's critical path.
struct CoarseRegs {
    const float* ainv;  // [blocks][U][m] rows of A_c^-1 (batched level: per-instance inverses)
    const float4* w;    // per-row field weights (nq = 4)
    int nq, U, G, m;    // fields, values per block, CTAs per block, unknowns
    // the batched level's block layout (CoarseArgs)
    const int *blk_slot, *inst_blk, *inst_aoff, *slot_cb;
};
__device__ __forceinline__ CoarseRegs coarse_regs(const BatchPlan& bp, bool on) {
    CoarseRegs c{nullptr, nullptr, 1, 3, 1, 0, nullptr, nullptr, nullptr, nullptr};
    if (on) {
        c.ainv = bp.cg->ainv;
        c.w = bp.cg->w;
        c.nq = bp.cg->nq;
        c.U = 3 * bp.cg->nq;
        c.G = bp.cg->g;
        c.m = bp.cg->m;
        c.blk_slot = bp.cg->blk_slot;
        c.inst_blk = bp.cg->inst_blk;
        c.inst_aoff = bp.cg->inst_aoff;
        c.slot_cb = bp.cg->slot_cb;
    }
    return c;
}
// Coarse values of a phase sit in slot entries kCoarseOff.. of every CTA;
// coarse block C's value is the sum over its CTAs C G .. C G + G - 1.

// Per-warp restriction of one row's v: the U = 3 nq sums over the warp's
// lanes of w_iq v (w_i0 = 1), written to dst[0..U) (fixed summation order).
// nq = 4: recursive halving of 16 values (12 used), 16 shuffles; value k's
// total lands in lanes 2k and 2k + 1.
__device__ __forceinline__ void warp_restrict(int nq, float3 v, float4 w, float* dst) {
    const int lane = threadIdx.x & 31;
    if (nq == 1) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
            v.z += __shfl_xor_sync(0xffffffffu, v.z, o);
        }
        if (lane == 0) {
            dst[0] = v.x;
            dst[1] = v.y;
            dst[2] = v.z;
        }
        return;
    }
    float a[16] = {v.x, v.y, v.z, w.x * v.x, w.x * v.y, w.x * v.z, w.y * v.x, w.y * v.y,
                   w.y * v.z, w.z * v.x, w.z * v.y, w.z * v.z, 0.f, 0.f, 0.f, 0.f};
    float b8[8], b4[4], b2[2];
    const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4, h2 = lane & 2;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        b8[k] = (h16 ? a[k + 8] : a[k]) + __shfl_xor_sync(0xffffffffu, h16 ? a[k] : a[k + 8], 16);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        b4[k] = (h8 ? b8[k + 4] : b8[k]) + __shfl_xor_sync(0xffffffffu, h8 ? b8[k] : b8[k + 4], 8);
#pragma unroll
    for (int k = 0; k < 2; ++k)
        b2[k] = (h4 ? b4[k + 2] : b4[k]) + __shfl_xor_sync(0xffffffffu, h4 ? b4[k] : b4[k + 2], 4);
    float b1 = (h2 ? b2[1] : b2[0]) + __shfl_xor_sync(0xffffffffu, h2 ? b2[0] : b2[1], 2);
    b1 += __shfl_xor_sync(0xffffffffu, b1, 1);
    const int k = lane >> 1;
    if ((lane & 1) == 0 && k < 12) dst[k] = b1;
}

// Float view of the coarse values of slot k of `set`.
__device__ __forceinline__ float* coarse_slot(const BatchPlan& bp, int set, int k) {
    return reinterpret_cast<float*>(bp.slots + ((size_t)set * bp.n_slots + k) * kSlotW + kCoarseOff);
}

// The CTA's coarse values (lane q < U: the sum over the CTA's nsl slices'
// partials, in slice order) into its slot of `set` (warp 1).
__device__ __forceinline__ void warp1_coarse_publish(const BatchPlan& bp, int U, const float* cpart, int nsl,
                                                     int own_slot, int set) {
    const int lane = threadIdx.x & 31;
    if (lane < U) {
        float acc = 0.0f;
        for (int w = 0; w < nsl; ++w) acc += cpart[w * kCoarsePartW + lane];
        coarse_slot(bp, set, own_slot)[lane] = acc;
    }
}

// The whole slot set `set` (n_slots x kSlotW doubles: the scalars, then the
// coarse floats at kCoarseOff) into shared memory, one 16-byte load per
// thread and pass; called by every thread of the CTA.
__device__ __forceinline__ void coarse_stage_slots(const BatchPlan& bp, int set, double* dst) {
    constexpr int kPer = kSlotW / 2;  // 16-byte pieces per slot
    const float4* src = reinterpret_cast<const float4*>(bp.slots + (size_t)set * bp.n_slots * kSlotW);
    float4* d = reinterpret_cast<float4*>(dst);
    for (int x = threadIdx.x; x < bp.n_slots * kPer; x += blockDim.x) d[x] = __ldcg(src + x);
}

// Scalar totals of the single instance from the staged slots (warp 0):
// lane l adds the slots l, l + 32, ... in ascending order, then the xor
// tree, so the totals equal those of warp0_read_totals; lane 0 applies
// `step`.
template <int NR, class Step>
__device__ __forceinline__ void warp0_staged_totals(LocalInst* li, const double* slots, Step&& step) {
    const int lane = threadIdx.x & 31;
    LocalInst& L = li[0];
    if (L.done) return;
    double tot[NR];
#pragma unroll
    for (int q = 0; q < NR; ++q) tot[q] = 0.0;
    for (int k = L.slot_lo + lane; k < L.slot_hi; k += 32) {
#pragma unroll
        for (int q = 0; q < NR; ++q) tot[q] += slots[(size_t)k * kSlotW + q];
    }
#pragma unroll
    for (int q = 0; q < NR; ++q) tot[q] = warp_sum(tot[q]);
    if (lane == 0) step(L, tot);
    __syncwarp();
}

// Every coarse block's values v[B * U + u] (floats) from the staged slots:
// the sum of its G CTAs' coarse floats, added in slot order (threads tid
// of nthreads).
__device__ __forceinline__ void coarse_block_values(const double* slots, int n_slots, int U, int G, int m, int tid,
                                                    int nthreads, float* v) {
    const float* f = reinterpret_cast<const float*>(slots) + 2 * kCoarseOff;
    for (int j = tid; j < m; j += nthreads) {
        const int B = j / U, u = j - B * U;
        const int c1 = min((B + 1) * G, n_slots);
        float acc = 0.0f;
        for (int c = B * G; c < c1; ++c) acc += f[(size_t)c * 2 * kSlotW + u];
        v[j] = acc;
    }
}

// Row r of this CTA's block of A_c^-1 v (v the m staged block values, row r
// of A_c^-1 at ainv + r m); lane 0 writes it to out[r].  Lanes take
// consecutive entries (conflict-free shared-memory reads).
__device__ __forceinline__ void warp_coarse_row(int m, const float* v, const float* ainv, int r, float* out) {
    const int lane = threadIdx.x & 31;
    const float* arow = ainv + (size_t)r * m;
    float acc = 0.f;
#pragma unroll 4
    for (int j = lane; j < m; j += 32) acc = fmaf(arow[j], v[j], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[r] = acc;
}

__device__ __forceinline__ void named_barrier_w01() { asm volatile("bar.sync 1, 64;" ::: "memory"); }
// warps 1.. alone: the staged values are complete
__device__ __forceinline__ void named_barrier_stage(int nthreads) {
    asm volatile("bar.sync 3, %0;" ::"r"(nthreads) : "memory");
}

// This row's share of a coarse vector c ([U]): c_0 + sum_q w_q c_q per component.
__device__ __forceinline__ float3 coarse_prolong(int nq, const float* c, float4 w) {
    float3 o = make_float3(c[0], c[1], c[2]);
    if (nq == 4) {
        o.x = fmaf(w.x, c[3], fmaf(w.y, c[6], fmaf(w.z, c[9], o.x)));
        o.y = fmaf(w.x, c[4], fmaf(w.y, c[7], fmaf(w.z, c[10], o.y)));
        o.z = fmaf(w.x, c[5], fmaf(w.y, c[8], fmaf(w.z, c[11], o.z)));
    }
    return o;
}

// The same phase with the whole CTA reading the slots, for instances that
// span many CTAs (the streamed kernel runs up to ~1200): thread j reads (or
// polls) slots slot_lo + j + BLOCK * i, i < KB, all in flight at once, sums
// them in ascending order into red[j], and warp 0 adds red[] in a fixed
// order (lane-strided, then an xor tree).  Called by every thread after the
// __syncthreads that follows the partials; ends with a __syncthreads and
// leaves s_flag = 1 after a failed wait.  Both modes sum in the same order.
template <int NV, int SYNC, int BLOCK, int KB, class Step>
__device__ __forceinline__ void block_phase(const BatchPlan& bp, const double* spart, LocalInst* li, int nloc,
                                            int set, unsigned& target, double* red, int* s_flag, Step&& step) {
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid < 32) {
        warp0_publish<NV, SYNC>(bp, spart, li, nloc, set);
        if (!SYNC && lane == 0 && !barrier_arrive_wait(bp.bar, target)) *s_flag = 1;
    }
    __syncthreads();
    if (*s_flag) return;
    for (int t = 0; t < nloc; ++t) {
        LocalInst& L = li[t];
        if (L.done) continue;  // uniform: li is only written between barriers
        double acc[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] = 0.0;
        bool ok = true;
        const unsigned long long* fbase = bp.fslots + (size_t)set * bp.n_slots * kSlotW;
        for (int c0 = L.slot_lo; c0 < L.slot_hi && ok; c0 += BLOCK * KB) {
            unsigned long long val[KB][NV];
#pragma unroll
            for (int j = 0; j < KB; ++j) {
                const int k = c0 + j * BLOCK + tid;
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    if (k >= L.slot_hi) val[j][q] = 0ull;
                    else if (SYNC) val[j][q] = ld_relaxed_u64(fbase + (size_t)k * kSlotW + q);
                    else
                        val[j][q] = (unsigned long long)__double_as_longlong(
                            __ldcg(bp.slots + ((size_t)set * bp.n_slots + k) * kSlotW + q));
                }
            }
            if (SYNC) {
                const unsigned long long t0 = global_ns();
                unsigned spins = 0;
                while (true) {
                    bool pending = false;
#pragma unroll
                    for (int j = 0; j < KB; ++j) {
                        const int k = c0 + j * BLOCK + tid;
#pragma unroll
                        for (int q = 0; q < NV; ++q) {
                            if (val[j][q] == kSlotEmpty) {
                                pending = true;
                                val[j][q] = ld_relaxed_u64(fbase + (size_t)k * kSlotW + q);
                            }
                        }
                    }
                    if (!pending) break;
                    if ((++spins & 63u) == 0) {
                        if (*(volatile int*)&bp.bar->error) { ok = false; break; }
                        if (global_ns() - t0 > kBarrierTimeoutNs) {
                            atomicExch(&bp.bar->error, 1);
                            ok = false;
                            break;
                        }
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < KB; ++j) {
                if (c0 + j * BLOCK + tid < L.slot_hi) {
#pragma unroll
                    for (int q = 0; q < NV; ++q) acc[q] += __longlong_as_double((long long)val[j][q]);
                }
            }
        }
        if (SYNC) fence_acq_rel_gpu();  // acquire: the publishers' data is visible from here on
        if (!ok) *s_flag = 1;
#pragma unroll
        for (int q = 0; q < NV; ++q) red[tid * NV + q] = acc[q];
        __syncthreads();
        if (*s_flag) return;
        if (tid < 32) {
            double tot[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) tot[q] = 0.0;
            for (int j = lane; j < BLOCK; j += 32) {
#pragma unroll
                for (int q = 0; q < NV; ++q) tot[q] += red[j * NV + q];
            }
#pragma unroll
            for (int q = 0; q < NV; ++q) tot[q] = warp_sum(tot[q]);
            if (lane == 0) {
                if (SYNC) {
                    // this CTA's slot of the previous phase can be reused
                    unsigned long long* d =
                        bp.fslots + ((size_t)((set + 2) % 3) * bp.n_slots + L.own_slot) * kSlotW;
#pragma unroll
                    for (int q = 0; q < kSlotW; ++q) st_relaxed_u64(d + q, kSlotEmpty);
                }
                step(L, tot);
            }
        }
        __syncthreads();
    }
}

// Start partials of one row, kStartW wide: r.z, r.r, b.b, b.M^-1 b, x0.b,
// x0.r, b.z, b.r (with r = b - A x0, z = M^-1 r; the zero guess has x0 = 0,
// r = b, z = M^-1 b).  The warp sums land in sp[q].
__device__ __forceinline__ void start_partials(double* sp, bool write, float3 b, float3 zb, float3 x0, float3 r,
                                               float3 z) {
    double q[kStartW] = {dot3d(r, z), dot3d(r, r), dot3d(b, b), dot3d(b, zb),
                         dot3d(x0, b), dot3d(x0, r), dot3d(b, z), dot3d(b, r)};
#pragma unroll
    for (int k = 0; k < kStartW; ++k) q[k] = warp_sum(q[k]);
    if (write) {
#pragma unroll
        for (int k = 0; k < kStartW; ++k) sp[k] = q[k];
    }
}

// The instance's start applied to one row: the warm guess scaled by the
// energy-minimising factor c (x = c x0, r = (1 - c) b + c r0), or the zero
// guess when the instance fell back.
// The same start for a general linear preconditioner P: z = P(r) is formed
// from zb = P(b) and z0 = P(r0) of the unscaled start.
__device__ __forceinline__ void start_row_linear(const LocalInst& L, float3 b, float3 zb, float3& x, float3& r,
                                                 float3& z) {
    if (L.fallback) {
        x = f3(0.f, 0.f, 0.f);
        r = b;
        z = zb;
    } else {
        const float c = L.scale, cb = L.scale_b;
        x = f3(c * x.x, c * x.y, c * x.z);
        r = f3(fmaf(c, r.x, cb * b.x), fmaf(c, r.y, cb * b.y), fmaf(c, r.z, cb * b.z));
        z = f3(fmaf(c, z.x, cb * zb.x), fmaf(c, z.y, cb * zb.y), fmaf(c, z.z, cb * zb.z));
    }
}
__device__ __forceinline__ void start_row(const LocalInst& L, float3 b, const S6& Mi, float3& x, float3& r,
                                          float3& z) {
    if (L.fallback) {
        x = f3(0.f, 0.f, 0.f);
        r = b;
    } else {
        const float c = L.scale, cb = L.scale_b;
        x = f3(c * x.x, c * x.y, c * x.z);
        r = f3(fmaf(c, r.x, cb * b.x), fmaf(c, r.y, cb * b.y), fmaf(c, r.z, cb * b.z));
    }
    z = mul(Mi, r);
}

// Scalar steps (lane 0 of warp 0, on the CTA-local copy; the instance's
// first CTA also publishes the state and counts the instance when done).
// Start: the warm guess x0 is scaled by c = x0.b / x0.A x0 (x0.A x0 =
// x0.(b - r0)), the factor minimising 1/2 x.A x - b.x along x0, so the start
// is never worse than the zero guess in the A-norm (warm == 2); warm == 1
// keeps the guess as given (the reference's previous-dx start).  c <= 0 or
// a non-finite partial falls back to the zero guess.
__device__ __forceinline__ void step_start(const BatchPlan& bp, LocalInst& L, const double* tot, const SolverCfg& cfg,
                                           int warm) {
    const double bb = tot[2];
    double c = 0.0;
    if (warm == 1) {
        c = isfinite(tot[0]) && isfinite(tot[1]) ? 1.0 : 0.0;
    } else if (warm == 2) {
        const double xax = tot[4] - tot[5];
        c = xax > 0.0 ? tot[4] / xax : 0.0;
        if (!(c > 0.0) || !isfinite(c) || !isfinite(tot[0]) || !isfinite(tot[1])) c = 0.0;
    }
    L.fallback = warm && c == 0.0 ? 1 : 0;
    L.scale = (float)c;
    L.scale_b = (float)(1.0 - c);
    if (c == 1.0) {
        L.rho = tot[0];
        L.rr = tot[1];
    } else if (c > 0.0) {
        // r = (1 - c) b + c r0: its r.z and r.r from the start partials
        const double cb = 1.0 - c;
        L.rho = fmax(cb * cb * tot[3] + 2.0 * c * cb * tot[6] + c * c * tot[0], 0.0);
        L.rr = fmax(cb * cb * bb + 2.0 * c * cb * tot[7] + c * c * tot[1], 0.0);
    } else {
        L.rho = tot[3];
        L.rr = bb;
    }
    L.bb = bb;
    L.tol2 = cfg.rel_tol * cfg.rel_tol * bb;
    L.iter = 0;
    L.alpha = 0.0f;
    L.beta = 0.0f;
    const bool bad = !isfinite(L.rho) || !isfinite(L.rr) || !isfinite(bb);
    const bool conv = cfg.use_tol && L.rr <= L.tol2;
    L.status = bad ? kSolveNonfinite : kSolveConverged;
    L.done = (bad || conv || cfg.max_iter <= 0) ? 1 : 0;
    if (L.first) {
        InstState& G = bp.inst[L.b];
        G.rr0 = L.rr;
        G.bb = bb;
        G.fallback = L.fallback;
        if (L.done) {
            G.rho = L.rho; G.rr = L.rr; G.iter = 0; G.status = L.status; G.done = 1;
            atomicAdd(&bp.bar->ndone, 1u);
        }
    }
}

// alpha = rho / sigma (pcg_solver.cu:421-423)
__device__ __forceinline__ void step_alpha(LocalInst& L, const double* tot) {
    const double sigma = tot[0];
    const double alpha = (sigma > 1.0e-37 || sigma < -1.0e-37) ? L.rho / sigma : 0.0;
    L.sigma = sigma;
    L.alpha = (float)alpha;
    if (!isfinite(sigma) || !isfinite(alpha)) L.status = kSolveNonfinite;
}

// beta, iteration count, convergence (pcg_solver.cu:436-454)
__device__ __forceinline__ void step_beta(const BatchPlan& bp, LocalInst& L, const double* tot, const SolverCfg& cfg) {
    const double rho_new = tot[0], rr = tot[1];
    const double beta = (L.rho > 1.0e-37 || L.rho < -1.0e-37) ? rho_new / L.rho : 0.0;
    L.beta = (float)beta;
    L.rho = rho_new;
    L.rr = rr;
    L.iter += 1;
    const bool bad = L.status == kSolveNonfinite || !isfinite(rho_new) || !isfinite(rr);
    const bool conv = cfg.use_tol && rr <= L.tol2;
    int done = 0;
    if (bad) { L.status = kSolveNonfinite; done = 1; }
    else if (conv) { L.status = kSolveConverged; done = 1; }
    else if (L.iter >= cfg.max_iter) { L.status = cfg.use_tol ? kSolveMaxIter : kSolveConverged; done = 1; }
    if (done) {
        L.done = 1;
        if (L.first) {
            InstState& G = bp.inst[L.b];
            G.rho = L.rho; G.rr = L.rr; G.iter = L.iter; G.status = L.status; G.done = 1;
            atomicAdd(&bp.bar->ndone, 1u);
        }
    }
}

// A barrier failure leaves every unfinished instance flagged.
__device__ __forceinline__ void instances_fail(const BatchPlan& bp, const LocalInst* li, int nloc) {
    if (threadIdx.x != 0) return;
    for (int t = 0; t < nloc; ++t) {
        if (li[t].first) {
            InstState& G = bp.inst[li[t].b];
            G.status = kSolveKernelError;
            G.iter = li[t].iter;
            G.done = 1;
        }
    }
}

// Slot set of reduction phase ph: the polled mode rotates three sets; the
// counter mode alternates two by parity, so a CTA that has passed a barrier
// and publishes the next phase never overwrites values another CTA may
// still be reading from the phase before (it can only publish phase ph + 2
// into that set after the barrier of phase ph + 1, which every reader of
// phase ph must have reached).
#define slot_set(ph) (SYNC ? (ph) % 3 : (ph) & 1)

// The phase protocol shared by both kernels.  After the CTA's slice
// partials are in spart and a __syncthreads, this runs the warp-0 phase and
// leaves, after a closing __syncthreads, s_flag = 1 on a failed wait and
// (counter mode, with `exit_test`) s_exit = 1 when every instance of the
// batch is done.
#define CHYSX_REDUCE_PHASE(NV, KP, exit_test, STEP)                                                  \
    do {                                                                                             \
        if (warp == 0) {                                                                             \
            const bool w0ok = warp0_phase<NV, SYNC, KP>(bp, spart, li, nloc, slot_set(ph), target, STEP); \
            if (lane == 0) {                                                                         \
                if (!w0ok) s_flag = 1;                                                               \
                if (!SYNC && (exit_test) && w0ok)                                                    \
                    s_exit = *(volatile unsigned*)&bp.bar->ndone >= (unsigned)bp.n_inst;            \
            }                                                                                        \
        }                                                                                            \
        ++ph;                                                                                        \
        __syncthreads();                                                                             \
    } while (0)

// The same protocol for single-instance two-level plans: warp 0 publishes
// the NR scalars (spart entries 0..NR-1), warp 1 the coarse values (floats
// from the per-slice coarse partials), both before warp 0 arrives (named
// barrier of warps 0 and 1: warp 0's release then covers warp 1's stores);
// warp 0 waits on the grid barrier, and after a CTA barrier (its acquire
// orders their reads) every thread copies one 16-byte piece of the phase's
// slot set into shared memory: one L2 round trip, and the fewest requests
// on the lines every CTA reads at that moment.  Then warp 0 adds the
// scalar totals while warps 1.. add every coarse block's values (the sums
// of its CTAs' slots) and form one row each of this CTA's block of
// A_c^-1 v into OUT[0..U).
#define CHYSX_COARSE_PHASE(NR, OUT, exit_test, STEP)                                                 \
    do {                                                                                             \
        if (warp == 0) {                                                                             \
            warp0_publish<NR, 0>(bp, spart, li, nloc, slot_set(ph));                                 \
            named_barrier_w01();                                                                     \
            bool w0ok = true;                                                                        \
            if (lane == 0) w0ok = barrier_arrive_wait(bp.bar, target);                               \
            if (lane == 0 && !w0ok) s_flag = 1;                                                      \
        } else if (warp == 1) {                                                                      \
            warp1_coarse_publish(bp, c_U, s_cpart, s1 - s0, li[0].own_slot, slot_set(ph));           \
            named_barrier_w01();                                                                     \
        }                                                                                            \
        __syncthreads();                                                                             \
        if (!s_flag) coarse_stage_slots(bp, slot_set(ph), c_slots);                                  \
        __syncthreads();                                                                             \
        if (!s_flag) {                                                                               \
            if (warp == 0) {                                                                         \
                warp0_staged_totals<NR>(li, c_slots, STEP);                                          \
                /* one instance, whose done flag every CTA sets alike */                             \
                if (lane == 0 && (exit_test)) s_exit = li[0].done;                                   \
            } else {                                                                                 \
                coarse_block_values(c_slots, bp.n_slots, c_U, c_g, c_m, threadIdx.x - 32, 32 * (W - 1), \
                                    c_stage);                                                        \
                named_barrier_stage(32 * (W - 1));                                                   \
                for (int r = warp - 1; r < c_U; r += W - 1) warp_coarse_row(c_m, c_stage, c_ainv, r, OUT); \
            }                                                                                        \
        }                                                                                            \
        ++ph;                                                                                        \
        __syncthreads();                                                                             \
    } while (0)

// The same protocol with block_phase (the whole CTA reads the totals).
#define CHYSX_BLOCK_PHASE(NV, KB, exit_test, STEP)                                                   \
    do {                                                                                             \
        block_phase<NV, SYNC, BLOCK, KB>(bp, spart, li, nloc, slot_set(ph), target, s_red, &s_flag, STEP); \
        if (!SYNC && (exit_test) && threadIdx.x == 0 && !s_flag)                                     \
            s_exit = *(volatile unsigned*)&bp.bar->ndone >= (unsigned)bp.n_inst;                    \
        ++ph;                                                                                        \
        __syncthreads();                                                                             \
    } while (0)

// ---------------------------------------------------------------------------
// Coarse level of the streamed kernel (dense mode).  Each CTA belongs to
// coarse block blockIdx.x / G and needs its U entries of y = A_c^-1 v, v the
// restriction of a vector: every CTA publishes its rows' restriction in its
// reduction slot (floats at kCoarseOff) before the phase's barrier; after it
// every CTA sums the slots of each coarse block into vbuf[m] (shared memory)
// and forms its block's U rows of A_c^-1 vbuf, one row per warp.
// ---------------------------------------------------------------------------
// Restriction partials of one slice into its spart entry (floats at
// kCoarseOff): sum over the warp's rows of w_iq v_i (w_i0 = 1).
__device__ __forceinline__ float* slice_cpart(double* spart, int sl) {
    return reinterpret_cast<float*>(spart + (size_t)sl * kSlotW + kCoarseOff);
}
// The restriction of each of the CTA's segments (an instance's slices in
// this CTA, or all of them for the single-instance level) into the
// segment's slot of `set`, by the whole CTA: P threads per value each add
// every P-th slice's partial, then one thread adds the P sums in order (a
// fixed order: bitwise repeatable).  seg(q, lo, hi, slot) gives segment q's
// slices [lo, hi) relative to the CTA's first slice and its slot; tmp holds
// BLOCK floats.  Called by every thread; ends with a __syncthreads.
template <int BLOCK, typename Seg>
__device__ __forceinline__ void coarse_publish(const BatchPlan& bp, int U, double* spart, int nseg, Seg&& seg,
                                               int set, float* tmp) {
    const int nv = nseg * 12;
    const int P = nv == 0 || 2 * nv > BLOCK ? 1 : min(8, BLOCK / nv);
    for (int x = threadIdx.x; x < nv * P; x += BLOCK) {
        const int h = x % P, qu = x / P, q = qu / 12, u = qu - 12 * q;
        int lo, hi, slot;
        seg(q, lo, hi, slot);
        float acc = 0.0f;
        if (u < U)
            for (int sl = lo + h; sl < hi; sl += P) acc += slice_cpart(spart, sl)[u];
        if (P > 1) tmp[x] = acc;
        else if (u < U) coarse_slot(bp, set, slot)[u] = acc;
    }
    if (P > 1) {
        __syncthreads();
        for (int x = threadIdx.x; x < nv; x += BLOCK) {
            const int q = x / 12, u = x - 12 * q;
            if (u >= U) continue;
            int lo, hi, slot;
            seg(q, lo, hi, slot);
            float acc = 0.0f;
            for (int h = 0; h < P; ++h) acc += tmp[x * P + h];
            coarse_slot(bp, set, slot)[u] = acc;
        }
    }
    __syncthreads();
}
template <int BLOCK>
__device__ __forceinline__ void coarse_apply_dense(const BatchPlan& bp, const CoarseRegs& cr, int set, float* vbuf,
                                                   float* out) {
    constexpr int kChunk = 4;  // slot loads in flight per value
    const int U = cr.U, m = cr.m, G = cr.G, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (U % 4 == 0) {
        // one 16-byte piece (4 values) of one block per thread: its G slots
        // added in slot order, all loads of a chunk in flight at once
        const int per = U / 4;
        for (int x = tid; x < m / 4; x += BLOCK) {
            const int B = x / per, q = x - B * per;
            const int c1 = min((B + 1) * G, bp.n_slots);
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
            for (int c0 = B * G; c0 < c1; c0 += kChunk) {
                float4 val[kChunk];
#pragma unroll
                for (int k = 0; k < kChunk; ++k)
                    val[k] = c0 + k < c1 ? __ldcg(reinterpret_cast<const float4*>(coarse_slot(bp, set, c0 + k)) + q)
                                         : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int k = 0; k < kChunk; ++k) {
                    acc.x += val[k].x;
                    acc.y += val[k].y;
                    acc.z += val[k].z;
                    acc.w += val[k].w;
                }
            }
            reinterpret_cast<float4*>(vbuf)[x] = acc;
        }
    } else {
        for (int j = tid; j < m; j += BLOCK) {
            const int B = j / U, u = j % U;
            const int c1 = min((B + 1) * G, bp.n_slots);
            float acc = 0.0f;
            for (int c0 = B * G; c0 < c1; c0 += kChunk) {
                float val[kChunk];
#pragma unroll
                for (int k = 0; k < kChunk; ++k) val[k] = c0 + k < c1 ? __ldcg(coarse_slot(bp, set, c0 + k) + u) : 0.0f;
#pragma unroll
                for (int k = 0; k < kChunk; ++k) acc += val[k];
            }
            vbuf[j] = acc;
        }
    }
    __syncthreads();
    const float* rows = cr.ainv + (size_t)((int)blockIdx.x / G) * U * m;
    if (U == 12 && m % 4 == 0) {
        // every thread takes the 16-byte pieces j = tid, tid + BLOCK, ... of
        // all 12 rows at once (12 loads in flight per piece), then the
        // CTA's per-row sums (warp trees, then the warps in order)
        __shared__ float s_rsum[BLOCK / 32][12];
        const int m4 = m / 4;
        const float4* v4 = reinterpret_cast<const float4*>(vbuf);
        const float4* a4 = reinterpret_cast<const float4*>(rows);
        float acc[12];
#pragma unroll
        for (int r = 0; r < 12; ++r) acc[r] = 0.0f;
        for (int j = tid; j < m4; j += BLOCK) {
            const float4 vv = v4[j];
#pragma unroll
            for (int r = 0; r < 12; ++r) {
                const float4 av = __ldg(a4 + (size_t)r * m4 + j);
                acc[r] = fmaf(av.x, vv.x, fmaf(av.y, vv.y, fmaf(av.z, vv.z, fmaf(av.w, vv.w, acc[r]))));
            }
        }
#pragma unroll
        for (int r = 0; r < 12; ++r) {
            float x = acc[r];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) s_rsum[warp][r] = x;
        }
        __syncthreads();
        if (tid < 12) {
            float x = 0.0f;
            for (int w = 0; w < BLOCK / 32; ++w) x += s_rsum[w][tid];
            out[tid] = x;
        }
    } else if (m % 4 == 0) {
        // one half-warp per row, 16-byte loads of the row, 8 in flight per
        // lane (rows are 16-byte aligned: m % 4 == 0)
        const int hw = tid >> 4, hl = lane & 15, m4 = m / 4;
        const float4* v4 = reinterpret_cast<const float4*>(vbuf);
        for (int r = hw; r < U; r += BLOCK / 16) {
            const float4* a = reinterpret_cast<const float4*>(rows + (size_t)r * m);
            float acc = 0.0f;
#pragma unroll 4
            for (int j = hl; j < m4; j += 16) {
                const float4 av = __ldg(a + j), vv = v4[j];
                acc = fmaf(av.x, vv.x, fmaf(av.y, vv.y, fmaf(av.z, vv.z, fmaf(av.w, vv.w, acc))));
            }
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (hl == 0) out[r] = acc;
        }
    } else {
        for (int r = warp; r < U; r += BLOCK / 32) {
            const float* a = rows + (size_t)r * m;
            float acc = 0.0f;
#pragma unroll 8
            for (int j = lane; j < m; j += 32) acc = fmaf(__ldg(a + j), vbuf[j], acc);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) out[r] = acc;
        }
    }
    __syncthreads();
}

// ---- batched coarse level of the streamed kernel: coarse blocks inside
// instances (an instance's rows in one CTA, or a run of such segments), so
// A_c is block-diagonal by instance and a block's coarse values ride on its
// segments' own reduction slots.  Per local instance the CTA keeps
// kInstCoarseW floats for its own block: A_b^-1 R_b^T r (kCU) and of the
// new r (kCN).
constexpr int kInstCoarseW = 24, kCU = 0, kCN = 12;
static_assert(kBatchMaxBlocks * 12 <= 160, "coarse_apply_inst: five coarse values per lane");
// Sums over a warp's lanes of 16 values per lane by recursive halving (16
// shuffles): value k's total lands in lanes 2k and 2k + 1.
__device__ __forceinline__ float warp_sum16(const float (&a)[16]) {
    const int lane = threadIdx.x & 31;
    float b8[8], b4[4], b2[2];
    const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4, h2 = lane & 2;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        b8[k] = (h16 ? a[k + 8] : a[k]) + __shfl_xor_sync(0xffffffffu, h16 ? a[k] : a[k + 8], 16);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        b4[k] = (h8 ? b8[k + 4] : b8[k]) + __shfl_xor_sync(0xffffffffu, h8 ? b8[k] : b8[k + 4], 8);
#pragma unroll
    for (int k = 0; k < 2; ++k)
        b2[k] = (h4 ? b4[k + 2] : b4[k]) + __shfl_xor_sync(0xffffffffu, h4 ? b4[k] : b4[k + 2], 4);
    float b1 = (h2 ? b2[1] : b2[0]) + __shfl_xor_sync(0xffffffffu, h2 ? b2[0] : b2[1], 2);
    b1 += __shfl_xor_sync(0xffffffffu, b1, 1);
    return b1;
}

// Each unfinished local instance's 12 values of y = (A_b^-1 R_b^T v) on the
// CTA's own coarse block (the batched level always carries the translation
// and three linear fields), one warp per instance: lane l takes the
// instance's coarse values j = l, l + 32, ... (< m_b = 12 x its blocks),
// each the sum of its block's segment slots in slot order, multiplies them
// with the own block's 12 rows of the instance's A_b^-1 (coalesced rows
// from L2) and the warp adds the 12 products by recursive halving.  Writes
// y into out[q * kInstCoarseW + off + u], or, with alpha (the phase after
// A p), A_b^-1 R_b^T r_new = out[kCU] - alpha_b y into kCN.
__device__ __forceinline__ void coarse_apply_inst(const BatchPlan& bp, const CoarseRegs& cr, const LocalInst* li,
                                                  int nloc, int set, float* out, int off, int nwarps,
                                                  bool with_alpha) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = warp; q < nloc; q += nwarps) {
        const LocalInst& L = li[q];
        if (L.done) continue;
        const int B0 = cr.inst_blk[L.b], m = 12 * (cr.inst_blk[L.b + 1] - B0);
        const int ob = cr.slot_cb[L.own_slot] - B0;
        const float* A = cr.ainv + cr.inst_aoff[L.b] + (size_t)(12 * ob) * m;
        float c[5];
#pragma unroll
        for (int t = 0; t < 5; ++t) {
            const int j = lane + 32 * t;
            float sum = 0.0f;
            if (j < m) {
                const int jb = j / 12, u = j - 12 * jb;
                const int k1 = cr.blk_slot[B0 + jb + 1];
                for (int k = cr.blk_slot[B0 + jb]; k < k1; ++k) sum += __ldcg(coarse_slot(bp, set, k) + u);
            }
            c[t] = sum;
        }
        float prod[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) prod[r] = 0.0f;
#pragma unroll
        for (int t = 0; t < 5; ++t) {
            const int j = lane + 32 * t;
            if (j < m) {
#pragma unroll
                for (int r = 0; r < 12; ++r) prod[r] = fmaf(__ldg(A + (size_t)r * m + j), c[t], prod[r]);
            }
        }
        const float y = warp_sum16(prod);
        const int u = lane >> 1;
        float* o = out + q * kInstCoarseW;
        if ((lane & 1) == 0 && u < 12) {
            if (with_alpha) o[kCN + u] = fmaf(-L.alpha, y, o[kCU + u]);
            else o[off + u] = y;
        }
    }
}

// ---------------------------------------------------------------------------
// Streamed persistent kernel: rows are re-read from HBM every iteration.
// Preconditioner: block-Jacobi, or (CO = 1: single instance, counter
// barrier, dense coarse level planned) block-Jacobi plus the coarse correction
//     z = D^-1 r + R A_c^-1 R^T r,
// a fixed symmetric positive-definite operator, so the outer iteration stays
// plain PCG.  The coarse part of z rides on the existing phases: phase 1
// publishes R^T (A p) beside sigma, phase 2 forms A_c^-1 R^T r_new as
// A_c^-1 R^T r - alpha A_c^-1 R^T A p and publishes R^T r_new beside the
// dots, from which the next iteration's A_c^-1 R^T r restarts (no drift).
// ---------------------------------------------------------------------------
template <int BLOCK, int SYNC = 0, int CO = 0>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK)  // 1024 threads per SM: at most 64 registers
pcg_persistent_kernel(DevTopo t, Vecs v, BatchPlan bp, SolverCfg cfg, int warm, ZP*, ZP*) {
    extern __shared__ double s_mem[];
    __shared__ int s_flag;
    __shared__ int s_exit;
    __shared__ double s_red[BLOCK * kStartW];  // per-thread slot sums of block_phase (NV <= kStartW)
    // coarse level: A_c^-1 R^T of b, of r0, of A p, of r; the new r's
    __shared__ float s_cb[12], s_c0[12], s_cw[12], s_cu[12], s_cn[12];
    constexpr int W = BLOCK / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s0 = bp.cta_slice[blockIdx.x], s1 = bp.cta_slice[blockIdx.x + 1];
    const int il0 = bp.cta_inst_lo[blockIdx.x], il1 = bp.cta_inst_hi[blockIdx.x];
    const int nloc = il1 - il0 + 1;
    double* spart = s_mem;
    LocalInst* li = reinterpret_cast<LocalInst*>(s_mem + (size_t)bp.max_slices_per_cta * kSlotW);
    // dense coarse level (CO = 1 builds; uniform over the grid): off when
    // the step's inversion failed.  The CO = 0 builds keep the block-Jacobi
    // code alone, so both synchronisation modes compile to the same
    // arithmetic (bit-identical iterates)
    const bool coarse = CO == 1 && !SYNC && bp.cg != nullptr && bp.cg->on && bp.cg->dense &&
                        *(volatile int*)bp.cg->fail == 0;
    // batched coarse level (CO = 2 builds; zero-guess solves of several
    // instances): one coarse block per instance
    const bool coarse_b = CO == 2 && !SYNC && !warm && bp.cg != nullptr && bp.cg->on && bp.cg->batched &&
                          *(volatile int*)bp.cg->fail == 0;
    __shared__ CoarseRegs creg;
    if (threadIdx.x == 0) creg = coarse_regs(bp, coarse || coarse_b);  // ordered by the __syncthreads after init_local
    const int& c_U = creg.U;
    const int& c_nq = creg.nq;
    // the coarse block values behind the records, 16-byte aligned (float4 stores)
    float* c_vbuf = reinterpret_cast<float*>(
        (reinterpret_cast<uintptr_t>(li + bp.max_inst_per_cta) + 15) & ~static_cast<uintptr_t>(15));
    float* c_inst = c_vbuf;  // the batched level's per-instance values ([nloc][kInstCoarseW]) in the same place
    unsigned target = 0;  // barrier target; the counter starts at 0 every solve
    int ph = 0;           // reduction phase (SYNC = 1 slot set ph % 3)
    if (threadIdx.x == 0) {
        s_flag = 0;
        s_exit = 0;
    }
    init_local(bp, li, s0, s1, il0, il1);
    __syncthreads();
    bool ok = true;
    auto no_step = [](LocalInst&, const double*) {};
    auto cw = [&](int i) { return c_nq == 4 ? __ldg(creg.w + i) : make_float4(0.f, 0.f, 0.f, 0.f); };
    // coarse publication: the segments of the single-instance and batched
    // levels, and scratch for the partial sums (s_red is idle between phases)
    auto seg_cta = [&](int, int& lo, int& hi, int& slot) {
        lo = 0;
        hi = s1 - s0;
        slot = li[0].own_slot;
    };
    auto seg_inst = [&](int q, int& lo, int& hi, int& slot) {
        lo = li[q].seg_lo;
        hi = li[q].seg_hi;
        slot = li[q].own_slot;
    };
    float* c_tmp = reinterpret_cast<float*>(s_red);
    // one exchange phase carrying only the CTA's restriction of a vector;
    // leaves A_c^-1 R^T v (this block's U entries) in out
    auto coarse_exchange = [&](float* out) {
        coarse_publish<BLOCK>(bp, c_U, spart, 1, seg_cta, slot_set(ph), c_tmp);
        const int set = slot_set(ph);
        CHYSX_BLOCK_PHASE(1, 5, false, no_step);
        if (!s_flag) coarse_apply_dense<BLOCK>(bp, creg, set, c_vbuf, out);
    };

    // ---- phase 0: initial residual and per-instance start ----------------
    // zero guess: r = b, z = M^-1 b were written by the assembly kernel.
    // warm guess: r = b - A x0, z = M^-1 r (pcg_solver.cu:29-51).
    if (coarse) {
        // A_c^-1 R^T b and, for a warm start, A_c^-1 R^T r0
        for (int s = s0 + warp; s < s1; s += W) {
            const int i = s * 32 + lane;
            const float3 b = i < t.n ? xyz(v.b[i]) : f3(0.f, 0.f, 0.f);
            if (lane == 0) spart[(s - s0) * kSlotW] = 0.0;
            warp_restrict(c_nq, b, i < t.n ? cw(i) : make_float4(0.f, 0.f, 0.f, 0.f), slice_cpart(spart, s - s0));
        }
        __syncthreads();
        coarse_exchange(s_cb);
        ok = s_flag == 0;
    }
    if (coarse_b) {
        // every instance's A_b^-1 R_b^T b (the zero guess's r) into kCU
        for (int s = s0 + warp; s < s1; s += W) {
            const int i = s * 32 + lane;
            const float3 b = i < t.n ? xyz(v.b[i]) : f3(0.f, 0.f, 0.f);
            if (lane == 0) spart[(s - s0) * kSlotW] = 0.0;
            warp_restrict(c_nq, b, i < t.n ? cw(i) : make_float4(0.f, 0.f, 0.f, 0.f), slice_cpart(spart, s - s0));
        }
        __syncthreads();
        coarse_publish<BLOCK>(bp, c_U, spart, nloc, seg_inst, slot_set(ph), c_tmp);
        const int set = slot_set(ph);
        CHYSX_BLOCK_PHASE(1, 5, false, no_step);
        if (!s_flag) coarse_apply_inst(bp, creg, li, nloc, set, c_inst, kCU, W, false);
        __syncthreads();
        ok = s_flag == 0;
    }
    for (int s = s0 + warp; s < s1 && ok; s += W) {
        const int i = s * 32 + lane;
        float3 b = f3(0.f, 0.f, 0.f), zb = b, x0 = b, r = b, z = b;
        if (i < t.n) {
            b = xyz(v.b[i]);
            const S6 Mi = ld6(t.minv + (size_t)s * 192 + lane);
            zb = mul(Mi, b);
            if (coarse) zb = zb + coarse_prolong(c_nq, s_cb, cw(i));
            if (coarse_b)
                zb = zb + coarse_prolong(c_nq, c_inst + (bp.slice_inst[s] - il0) * kInstCoarseW + kCU, cw(i));
            r = b;
            z = zb;
            if (warm) {
                const int so = t.slice_off[s];
                const int w = (t.slice_off[s + 1] - so) >> 5;
                const S6 D = ld6(t.dnl + (size_t)s * 192 + lane);
                x0 = xyz(v.x[i]);
                float3 ax = mul(D, x0);
                const int ow = off_width(t);
                const float* vb = t.val + (size_t)so * ow + lane;
                for (int k = 0; k < w; ++k) {
                    const int j = t.col[so + k * 32 + lane];
                    ax = ax + mul_off(vb + k * ow * 32, t.nsym, xyz(v.x[j]) - x0);
                }
                if (t.co.active && t.co.residual)
                    ax = ax + contact_spmv_row(t.co, i, [&](int j) { return xyz(v.x[j]); });
                r = b - ax;
                z = mul(Mi, r);
                v.r[i] = f4(r);
            } else if (coarse || coarse_b) {
                v.z[i] = f4(zb);
            }
        }
        if (!coarse || !warm) start_partials(spart + (s - s0) * kSlotW, lane == 0, b, zb, x0, r, z);
    }
    if (coarse && warm && ok) {
        // A_c^-1 R^T r0, then the start partials with z = M^-1 r0 + its prolongation
        __syncthreads();
        for (int s = s0 + warp; s < s1; s += W) {
            const int i = s * 32 + lane;
            const float3 r = i < t.n ? xyz(v.r[i]) : f3(0.f, 0.f, 0.f);
            if (lane == 0) spart[(s - s0) * kSlotW] = 0.0;
            warp_restrict(c_nq, r, i < t.n ? cw(i) : make_float4(0.f, 0.f, 0.f, 0.f), slice_cpart(spart, s - s0));
        }
        __syncthreads();
        coarse_exchange(s_c0);
        ok = s_flag == 0;
        for (int s = s0 + warp; s < s1 && ok; s += W) {
            const int i = s * 32 + lane;
            float3 b = f3(0.f, 0.f, 0.f), zb = b, x0 = b, r = b, z = b;
            if (i < t.n) {
                const S6 Mi = ld6(t.minv + (size_t)s * 192 + lane);
                const float4 w4 = cw(i);
                b = xyz(v.b[i]);
                zb = mul(Mi, b) + coarse_prolong(c_nq, s_cb, w4);
                x0 = xyz(v.x[i]);
                r = xyz(v.r[i]);
                z = mul(Mi, r) + coarse_prolong(c_nq, s_c0, w4);
            }
            start_partials(spart + (s - s0) * kSlotW, lane == 0, b, zb, x0, r, z);
        }
    }
    __syncthreads();
    if (ok) {
        CHYSX_BLOCK_PHASE(kStartW, 1, false,
                          ([&](LocalInst& L, const double* tot) { step_start(bp, L, tot, cfg, warm); }));
        ok = s_flag == 0;
    }
    if (ok && warm) {
        // the scaled guess, or the zero guess where the instance fell back
        for (int s = s0 + warp; s < s1; s += W) {
            const int i = s * 32 + lane;
            if (i >= t.n) continue;
            const S6 Mi = ld6(t.minv + (size_t)s * 192 + lane);
            float3 x = xyz(v.x[i]), r = xyz(v.r[i]), z;
            const LocalInst& L = li[bp.slice_inst[s] - il0];
            if (coarse) {
                const float4 w4 = cw(i);
                const float3 b = xyz(v.b[i]);
                const float3 zb = mul(Mi, b) + coarse_prolong(c_nq, s_cb, w4);
                z = mul(Mi, r) + coarse_prolong(c_nq, s_c0, w4);
                start_row_linear(L, b, zb, x, r, z);
            } else {
                start_row(L, xyz(v.b[i]), Mi, x, r, z);
            }
            v.x[i] = f4(x);
            v.r[i] = f4(r);
            v.z[i] = f4(z);
        }
        // a data-free phase orders the new rows before any gather
        for (int q = threadIdx.x; q < s1 - s0; q += BLOCK) spart[q * kSlotW] = 0.0;
        __syncthreads();
        CHYSX_BLOCK_PHASE(1, 5, false, no_step);
        ok = s_flag == 0;
    }
    if (coarse && ok) {
        // A_c^-1 R^T r of the start: of r0, of the scaled mix of r0 and b, or of b
        const LocalInst& L0 = li[0];
        const bool from_r0 = warm && !L0.fallback;
        if ((int)threadIdx.x < c_U)
            s_cu[threadIdx.x] = from_r0 ? fmaf(L0.scale, s_c0[threadIdx.x], L0.scale_b * s_cb[threadIdx.x])
                                        : s_cb[threadIdx.x];
        __syncthreads();
    }

    // ---- iterations ---------------------------------------------------------
    const int iter_cap = cfg.max_iter + 2;  // belt: every instance is done by max_iter
    for (int guard = 0; ok && guard < iter_cap; ++guard) {
        if (SYNC) {
            // leave once every instance of this CTA is done
            if (threadIdx.x == 0) {
                int all = 1;
                for (int q = 0; q < nloc; ++q) all &= li[q].done;
                s_exit = all;
            }
            __syncthreads();
            if (s_exit) break;
        }
        // phase 1: p = z + beta p (own row and recomputed for neighbours),
        // Ap = A p, sigma = p.Ap (and the restriction of Ap)
        for (int s = s0 + warp; s < s1; s += W) {
            const LocalInst& L = li[bp.slice_inst[s] - il0];
            const int i = s * 32 + lane;
            double sig = 0.0;
            float3 acc = f3(0.f, 0.f, 0.f);
            // the coarse weights first: their load overlaps the row's
            const float4 w4 = (coarse || (coarse_b && !L.done)) && i < t.n ? cw(i) : make_float4(0.f, 0.f, 0.f, 0.f);
            if (!L.done && i < t.n) {
                const bool first = L.iter == 0;
                const float beta = L.beta;
                const float4* pold = (L.iter & 1) ? v.p1 : v.p0;
                float4* pnew = (L.iter & 1) ? v.p0 : v.p1;
                const int so = t.slice_off[s];
                const int w = (t.slice_off[s + 1] - so) >> 5;
                const float4 zi = ldcg4(v.z + i);
                float3 pi = xyz(zi);
                if (!first) {
                    const float4 po = ldcg4(pold + i);
                    pi = f3(fmaf(beta, po.x, zi.x), fmaf(beta, po.y, zi.y), fmaf(beta, po.z, zi.z));
                }
                pnew[i] = f4(pi);
                acc = mul(ld6(t.dnl + (size_t)s * 192 + lane), pi);
                const int ow = off_width(t);
                const float* vb = t.val + (size_t)so * ow + lane;
                const int* cb = t.col + so + lane;
                for (int k = 0; k < w; ++k) {
                    const int j = cb[k * 32];
                    const float4 zj = ldcg4(v.z + j);
                    float3 pj = xyz(zj);
                    if (!first) {
                        const float4 po = ldcg4(pold + j);
                        pj = f3(fmaf(beta, po.x, zj.x), fmaf(beta, po.y, zj.y), fmaf(beta, po.z, zj.z));
                    }
                    acc = acc + mul_off(vb + k * ow * 32, t.nsym, pj - pi);
                }
                if (t.co.active)
                    acc = acc + contact_spmv_row(t.co, i, [&](int j) {
                              const float4 zj = ldcg4(v.z + j);
                              if (first) return xyz(zj);
                              const float4 po = ldcg4(pold + j);
                              return f3(fmaf(beta, po.x, zj.x), fmaf(beta, po.y, zj.y), fmaf(beta, po.z, zj.z));
                          });
                v.ap[i] = f4(acc);
                sig = (double)pi.x * acc.x + (double)pi.y * acc.y + (double)pi.z * acc.z;
            }
            sig = warp_sum(sig);
            if (lane == 0) spart[(s - s0) * kSlotW] = sig;
            // (a finished instance's restriction is never read: left out of batches)
            if (coarse || (coarse_b && !L.done)) warp_restrict(c_nq, acc, w4, slice_cpart(spart, s - s0));
        }
        __syncthreads();
        if (coarse) coarse_publish<BLOCK>(bp, c_U, spart, 1, seg_cta, slot_set(ph), c_tmp);
        if (coarse_b) coarse_publish<BLOCK>(bp, c_U, spart, nloc, seg_inst, slot_set(ph), c_tmp);
        const int set1 = slot_set(ph);
        // ndone only changes in the start and beta steps, i.e. never between
        // this barrier and the next, so every CTA takes the same exit decision
        CHYSX_BLOCK_PHASE(1, 5, true, ([&](LocalInst& L, const double* tot) { step_alpha(L, tot); }));
        if (s_flag) {
            ok = false;
            break;
        }
        if (!SYNC && s_exit) break;
        if (coarse) {
            coarse_apply_dense<BLOCK>(bp, creg, set1, c_vbuf, s_cw);
            // A_c^-1 R^T r_new = A_c^-1 R^T r - alpha A_c^-1 R^T A p
            if ((int)threadIdx.x < c_U) s_cn[threadIdx.x] = fmaf(-li[0].alpha, s_cw[threadIdx.x], s_cu[threadIdx.x]);
            __syncthreads();
        }
        if (coarse_b) {
            // per instance: A_b^-1 R_b^T r_new = A_b^-1 R_b^T r - alpha_b A_b^-1 R_b^T A p
            coarse_apply_inst(bp, creg, li, nloc, set1, c_inst, 0, W, true);
            __syncthreads();
        }

        // phase 2: x += alpha p; r -= alpha Ap; z = M^-1 r (+ its coarse part)
        for (int s = s0 + warp; s < s1; s += W) {
            const int q = bp.slice_inst[s] - il0;
            const LocalInst& L = li[q];
            const int i = s * 32 + lane;
            double rz = 0.0, rr = 0.0;
            float3 rn = f3(0.f, 0.f, 0.f);
            const float4 w4 = (coarse || (coarse_b && !L.done)) && i < t.n ? cw(i) : make_float4(0.f, 0.f, 0.f, 0.f);
            if (!L.done && i < t.n) {
                const float alpha = L.alpha;
                const float4 pi = ((L.iter & 1) ? v.p0 : v.p1)[i];
                const float4 api = v.ap[i], xi = v.x[i], ri = v.r[i];
                const float3 xn = f3(fmaf(alpha, pi.x, xi.x), fmaf(alpha, pi.y, xi.y), fmaf(alpha, pi.z, xi.z));
                rn = f3(fmaf(-alpha, api.x, ri.x), fmaf(-alpha, api.y, ri.y), fmaf(-alpha, api.z, ri.z));
                float3 zn = mul(ld6(t.minv + (size_t)s * 192 + lane), rn);
                if (coarse) zn = zn + coarse_prolong(c_nq, s_cn, w4);
                if (coarse_b) zn = zn + coarse_prolong(c_nq, c_inst + q * kInstCoarseW + kCN, w4);
                v.x[i] = f4(xn);
                v.r[i] = f4(rn);
                v.z[i] = f4(zn);
                rz = (double)rn.x * zn.x + (double)rn.y * zn.y + (double)rn.z * zn.z;
                rr = (double)rn.x * rn.x + (double)rn.y * rn.y + (double)rn.z * rn.z;
            }
            rz = warp_sum(rz);
            rr = warp_sum(rr);
            if (lane == 0) {
                spart[(s - s0) * kSlotW] = rz;
                spart[(s - s0) * kSlotW + 1] = rr;
            }
            if (coarse || (coarse_b && !L.done)) warp_restrict(c_nq, rn, w4, slice_cpart(spart, s - s0));
        }
        __syncthreads();
        if (coarse) coarse_publish<BLOCK>(bp, c_U, spart, 1, seg_cta, slot_set(ph), c_tmp);
        if (coarse_b) coarse_publish<BLOCK>(bp, c_U, spart, nloc, seg_inst, slot_set(ph), c_tmp);
        const int set2 = slot_set(ph);
        // phase 3: beta, iteration count, convergence
        CHYSX_BLOCK_PHASE(2, 5, false,
                          ([&](LocalInst& L, const double* tot) { step_beta(bp, L, tot, cfg); }));
        if (s_flag) {
            ok = false;
            break;
        }
        // the coarse part restarts from R^T r_new (no recurrence drift)
        if (coarse) coarse_apply_dense<BLOCK>(bp, creg, set2, c_vbuf, s_cu);
        if (coarse_b) {
            coarse_apply_inst(bp, creg, li, nloc, set2, c_inst, kCU, W, false);
            __syncthreads();
        }
    }
    if (!ok) instances_fail(bp, li, nloc);
}


}  // namespace chysx_b200

#include "coarse.cuh"

namespace chysx_b200 {

// ---------------------------------------------------------------------------
// Register-resident variant for systems with at most one 32-row slice per
// warp: every thread owns one row for the whole solve and keeps its diagonal
// block, Jacobi inverse, off-diagonal blocks + columns (up to MAXW) and
// x, r, z, p in registers.  Per iteration it publishes only p (phase 1) and
// z (phase 2) for its neighbours, packed as one 32-byte entry per row in a
// double-buffered array, so a neighbour's (z, p_old) pair is one sector.
// The CTA's own rows' z and p are also kept in shared memory: neighbours in
// the same CTA are read from there, the others from L2, a batch of gathers
// in flight at once.  Same phases, reductions, barrier and per-instance
// logic as pcg_persistent_kernel.
// ---------------------------------------------------------------------------
template <int W, int MAXW, int SYNC = 0, int PC = 0>
__global__ void __launch_bounds__(W * 32, 512 / (W * 32))  // 512 threads of rows per SM
pcg_resident_kernel(DevTopo t, Vecs v, BatchPlan bp, SolverCfg cfg, int warm, ZP* zp0, ZP* zp1) {
    extern __shared__ double s_mem[];
    __shared__ int s_flag;
    __shared__ int s_exit;
    __shared__ float4 s_z[W * 32], s_p[2][W * 32];
    // CTA-local preconditioner: exchange buffers, block sums, Chebyshev
    // constants (theta, 1/theta, sigma, 2/delta) of this CTA's block
    __shared__ float4 s_d[PC ? 2 : 1][PC ? W * 32 : 1];
    __shared__ double s_bsum[PC ? W : 1];
    __shared__ float s_cheb[4];
    __shared__ float2 s_ccoef[PC ? 64 : 1];  // per term m of the polynomial: (rn rho, rn 2/delta)
    // coarse level: this block of A_c^-1 R^T (A p) and of A_c^-1 R^T r
    __shared__ float s_cw[12], s_cu[12];  // this block of A_c^-1 R^T (Ap) / A_c^-1 R^T r
    __shared__ float s_cpart[PC == 2 ? W * kCoarsePartW : 1];  // per-slice coarse partials
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s0 = bp.cta_slice[blockIdx.x], s1 = bp.cta_slice[blockIdx.x + 1];
    const int il0 = bp.cta_inst_lo[blockIdx.x], il1 = bp.cta_inst_hi[blockIdx.x];
    const int nloc = il1 - il0 + 1;
    const int row0 = s0 * 32, nrows = (s1 - s0) * 32;  // the CTA's rows
    double* spart = s_mem;  // [W * kSlotW]
    LocalInst* li = reinterpret_cast<LocalInst*>(s_mem + (size_t)W * kSlotW);
    unsigned target = 0;
    int ph = 0;  // reduction phase (SYNC = 1 slot set ph % 3)
    if (threadIdx.x == 0) {
        s_flag = 0;
        s_exit = 0;
    }
    init_local(bp, li, s0, s1, il0, il1);
    bool ok = true;
    auto no_step = [](LocalInst&, const double*) {};

    const int s = s0 + warp;
    const bool has = s < s1;
    const int i = s * 32 + lane;
    const bool row = has && i < t.n;
    const int li_idx = has ? bp.slice_inst[s] - il0 : 0;

    // ---- load the row --------------------------------------------------
    // D: the row's non-elastic diagonal D'; the operator is applied in the
    // difference form D'_i p_i + sum_k B_k (p_j - p_i)
    S6 D{0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, Mi{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    S6 B[MAXW];
    // column indices: registers, or shared memory in the slot-polling build
    // (its waits need the registers)
    int cols_r[SYNC ? 1 : MAXW];
    __shared__ int s_cols[SYNC ? MAXW * W * 32 : 1];
    auto col_at = [&](int k) -> int & { return SYNC ? s_cols[k * W * 32 + threadIdx.x] : cols_r[SYNC ? 0 : k]; };
    int w = 0;
    float3 b = f3(0.f, 0.f, 0.f), x = b, r = b, z = b, p = b;
#pragma unroll
    for (int k = 0; k < MAXW; ++k) {
        B[k] = S6{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        col_at(k) = row ? i : 0;
    }
    if (row) {
        D = ld6(t.dnl + (size_t)s * 192 + lane);
        Mi = ld6(t.minv + (size_t)s * 192 + lane);
        b = xyz(v.b[i]);
        const int so = t.slice_off[s];
        w = (t.slice_off[s + 1] - so) >> 5;
#pragma unroll
        for (int k = 0; k < MAXW; ++k) {
            if (k < w) {
                col_at(k) = t.col[so + k * 32 + lane];
                B[k] = ld6(t.val + (size_t)so * 6 + (size_t)k * 192 + lane);  // symmetric blocks only
            }
        }
    }
    __syncthreads();  // init_local

    // ---- CTA-local Chebyshev preconditioner (PC) ---------------------------
    // z = P(r): a fixed-degree Chebyshev iteration for A_cc z = r from z = 0,
    // A_cc the CTA's diagonal block of rows (couplings to other CTAs
    // dropped), block-Jacobi inner preconditioner; a fixed polynomial, so P is
    // linear and symmetric and the outer PCG stays plain PCG.  Called by every
    // thread of the CTA (it synchronises); inactive rows pass r = 0.  A_cc in
    // the difference form: columns outside the CTA count as zero, their
    // blocks still enter the row's implied diagonal.
    auto local_spmv = [&](const float4* buf, float3 in) {
        float3 acc = mul(D, in);
#pragma unroll
        for (int k = 0; k < MAXW; ++k) {
            if (k >= w) continue;
            const int lr = col_at(k) - row0;
            const float3 nb = (unsigned)lr < (unsigned)nrows ? xyz(buf[lr]) : f3(0.f, 0.f, 0.f);
            acc = acc + mul(B[k], nb - in);
        }
        return acc;
    };
    // the full diagonal block times a vector: D' v - sum_k B_k v
    auto full_diag = [&](float3 in) {
        float3 acc = mul(D, in);
#pragma unroll
        for (int k = 0; k < MAXW; ++k)
            if (k < w) acc = acc - mul(B[k], in);
        return acc;
    };
    auto block_sum = [&](double q) {
        q = warp_sum(q);
        if (lane == 0) s_bsum[warp] = q;
        __syncthreads();
        double tot = 0.0;
#pragma unroll
        for (int k = 0; k < W; ++k) tot += s_bsum[k];
        __syncthreads();
        return tot;
    };
    auto precond = [&](float3 rin) {
        const float th_inv = s_cheb[1];
        float3 res = rin;
        float3 d = mul(Mi, res) * th_inv;
        float3 zc = d;
        for (int m = 1; m < cfg.pc_degree; ++m) {
            float4* buf = s_d[PC ? (m & 1) : 0];
            buf[threadIdx.x] = f4(d);
            __syncthreads();
            res = res - local_spmv(buf, d);
            const float3 mr = mul(Mi, res);
            const float2 c = s_ccoef[PC ? m : 0];  // (rn rho, rn 2/delta) of term m
            d = f3(fmaf(c.x, d.x, c.y * mr.x), fmaf(c.x, d.y, c.y * mr.y), fmaf(c.x, d.z, c.y * mr.z));
            zc = zc + d;
        }
        return zc;
    };
    if (PC) {
        // lambda_max of D^-1 A_cc by power iteration from a fixed +-1 vector,
        // Rayleigh quotient v.A v / v.D v, times a margin; interval
        // [lambda / ratio, lambda]
        float3 pv = f3(0.f, 0.f, 0.f);
        if (row) pv = f3(pc_sign(3 * i), pc_sign(3 * i + 1), pc_sign(3 * i + 2));
        for (int it = 0; it < kPcPowerIts; ++it) {
            float4* buf = s_d[PC ? (it & 1) : 0];
            buf[threadIdx.x] = f4(pv);
            __syncthreads();
            const float3 wv = mul(Mi, local_spmv(buf, pv));
            const double nn = block_sum(dot3d(wv, wv));
            const float sc = nn > 0.0 ? (float)(1.0 / sqrt(nn)) : 0.0f;
            pv = wv * sc;
        }
        float4* buf = s_d[PC ? (kPcPowerIts & 1) : 0];
        buf[threadIdx.x] = f4(pv);
        __syncthreads();
        const double num = block_sum(dot3d(pv, local_spmv(buf, pv)));
        const double den = block_sum(dot3d(pv, full_diag(pv)));
        if (threadIdx.x == 0) {
            double hi = den > 0.0 ? kPcMargin * num / den : 1.0;
            if (!(hi > 0.0) || !isfinite(hi)) hi = 1.0;
            const double lo = hi / (double)cfg.pc_ratio;
            const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
            s_cheb[0] = (float)theta;
            s_cheb[1] = (float)(1.0 / theta);
            s_cheb[2] = (float)(theta / delta);
            s_cheb[3] = (float)(2.0 / delta);
            // the three-term recurrence's coefficients of every term, in the
            // FP32 arithmetic the terms used to form them in
            const float sg = s_cheb[2], two_de = s_cheb[3];
            float rho = 1.0f / sg;
            for (int m = 1; m < cfg.pc_degree && m < 64; ++m) {
                const float rn = 1.0f / (2.0f * sg - rho);
                s_ccoef[PC ? m : 0] = make_float2(rn * rho, rn * two_de);
                rho = rn;
            }
        }
        __syncthreads();
    }

    // ---- coarse level (PC = 2 with bp.cg->on): this CTA's coarse block
    // Bc = blockIdx.x / G; its U rows of A_c^-1 in dynamic shared memory
    // behind the LocalInst records; every row's field weights in a register
    // quad.  Warps 1..3 form this block of A_c^-1 R^T v during the phases.
    constexpr bool kCoarse = PC == 2;
    const bool coarse = kCoarse && bp.cg != nullptr && bp.cg->on && *(volatile int*)bp.cg->fail == 0;
    const CoarseRegs creg = coarse_regs(bp, coarse);
    const int c_U = creg.U, c_nq = creg.nq, c_g = creg.G, c_m = creg.m;
    float* c_ainv = reinterpret_cast<float*>(li + bp.max_inst_per_cta);
    // a phase's coarse block values ([m]) behind c_ainv, then its staged
    // slot set ([n_slots][kSlotW] doubles), each 16-byte aligned
    float* c_stage = reinterpret_cast<float*>(
        (reinterpret_cast<uintptr_t>(c_ainv + (coarse ? c_U * c_m : 0)) + 15) & ~static_cast<uintptr_t>(15));
    double* c_slots = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(c_stage + (coarse ? c_m : 0)) + 15) & ~static_cast<uintptr_t>(15));
    float4 c_w = make_float4(0.f, 0.f, 0.f, 0.f);
    if (coarse) {
        const int m = c_m;
        const float* src = creg.ainv + (size_t)(blockIdx.x / c_g) * c_U * m;
        for (int q = threadIdx.x; q < c_U * m; q += blockDim.x) c_ainv[q] = src[q];
        if (c_nq == 4 && row) c_w = creg.w[i];
        __syncthreads();
    }

    // ---- phase 0 -------------------------------------------------------
    float3 pc_zb = f3(0.f, 0.f, 0.f);  // P(b), for the start of a scaled guess
    if (PC) {
        float3 zb = f3(0.f, 0.f, 0.f);
        if (row) {
            r = b;
            if (warm) {
                x = xyz(v.x[i]);
                float3 ax = mul(D, x);
#pragma unroll
                for (int k = 0; k < MAXW; ++k)
                    if (k < w) ax = ax + mul(B[k], xyz(v.x[col_at(k)]) - x);
                r = b - ax;
            }
        }
        float3 cb = f3(0.f, 0.f, 0.f), cr = cb;
        if (coarse) {
            // A_c^-1 R^T b (s_cw) and, for a warm start, A_c^-1 R^T r0 (s_cu):
            // one exchange phase each
            for (int pass = 0; pass < (warm ? 2 : 1); ++pass) {
                const float3 sv = row ? (pass ? r : b) : f3(0.f, 0.f, 0.f);
                if (lane == 0) spart[warp * kSlotW] = 0.0;
                warp_restrict(c_nq, sv, c_w, s_cpart + (PC == 2 ? warp * kCoarsePartW : 0));
                __syncthreads();
                CHYSX_COARSE_PHASE(1, pass ? s_cu : s_cw, false, no_step);
                if (s_flag) break;
            }
            ok = s_flag == 0;
            if (ok) {
                cb = coarse_prolong(c_nq, s_cw, c_w);
                if (warm) cr = coarse_prolong(c_nq, s_cu, c_w);
            }
        }
        zb = precond(b) + cb;
        z = warm ? precond(r) + cr : zb;
        pc_zb = zb;
        if (row) {
            zp0[i].z = f4(z);
            s_z[threadIdx.x] = f4(z);
        }
        start_partials(spart + warp * kSlotW, lane == 0 && has, b, zb, x, r, z);
    } else {
        float3 zb = f3(0.f, 0.f, 0.f);
        if (row) {
            zb = mul(Mi, b);
            r = b;
            z = zb;
            if (warm) {
                x = xyz(v.x[i]);
                float3 ax = mul(D, x);
#pragma unroll
                for (int k = 0; k < MAXW; ++k)
                    if (k < w) ax = ax + mul(B[k], xyz(v.x[col_at(k)]) - x);
                r = b - ax;
                z = mul(Mi, r);
            }
            zp0[i].z = f4(z);
            s_z[threadIdx.x] = f4(z);
        }
        start_partials(spart + warp * kSlotW, lane == 0 && has, b, zb, x, r, z);
    }
    __syncthreads();
    CHYSX_REDUCE_PHASE(kStartW, 1, false,
                       ([&](LocalInst& L, const double* tot) { step_start(bp, L, tot, cfg, warm); }));
    ok = s_flag == 0;
    if (ok && warm) {
        // the scaled guess, or the zero guess where the instance fell back
        if (row) {
            if (PC) start_row_linear(li[li_idx], b, pc_zb, x, r, z);
            else start_row(li[li_idx], b, Mi, x, r, z);
            zp0[i].z = f4(z);
            s_z[threadIdx.x] = f4(z);
        }
        // a data-free phase orders the new z before any gather
        if (threadIdx.x < W) spart[threadIdx.x * kSlotW] = 0.0;
        __syncthreads();
        CHYSX_REDUCE_PHASE(1, kPollMax, false, no_step);
        ok = s_flag == 0;
    }
    if (coarse && ok) {
        // A_c^-1 R^T r of the start: of r0, of the scaled mix of r0 and b,
        // or of b
        const LocalInst& L0 = li[0];
        const bool from_r0 = warm && !L0.fallback;
        __syncthreads();  // every thread has read s_cw, s_cu
        if ((int)threadIdx.x < c_U) {
            const float ub = s_cw[threadIdx.x], u0 = s_cu[threadIdx.x];
            s_cu[threadIdx.x] = from_r0 ? fmaf(L0.scale, u0, L0.scale_b * ub) : ub;
        }
        __syncthreads();
    }
    float3 c_blk = f3(0.f, 0.f, 0.f);  // this block's coarse correction of the iteration

    // ---- iterations ----------------------------------------------------
    const int iter_cap = cfg.max_iter + 2;
    float3 ap = f3(0.f, 0.f, 0.f);
    for (int guard = 0; ok && guard < iter_cap; ++guard) {
        if (SYNC) {
            // leave once every instance of this CTA is done
            if (threadIdx.x == 0) {
                int all = 1;
                for (int q = 0; q < nloc; ++q) all &= li[q].done;
                s_exit = all;
            }
            __syncthreads();
            if (s_exit) break;
        }
        double sig = 0.0;
        if (row && !li[li_idx].done) {
            const LocalInst& L = li[li_idx];
            const bool first = L.iter == 0;
            const float beta = L.beta;
            const ZP* E = (L.iter & 1) ? zp1 : zp0;
            ZP* En = (L.iter & 1) ? zp0 : zp1;
            p = first ? z : f3(fmaf(beta, p.x, z.x), fmaf(beta, p.y, z.y), fmaf(beta, p.z, z.z));
            En[i].p = f4(p);
            s_p[(L.iter + 1) & 1][threadIdx.x] = f4(p);
            const float4* sp_old = s_p[L.iter & 1];
            float3 acc = mul(D, p);
            // gathers in batches of up to 6 entries (the valence of a
            // triangulated grid): every load of a batch is in flight at once,
            // padding entries read the row itself and are masked
            constexpr int kBatch = MAXW < 6 ? MAXW : 6;
#pragma unroll
            for (int k0 = 0; k0 < MAXW; k0 += kBatch) {
                if (k0 > 0 && k0 >= w) break;
                float4 zj[kBatch], pj[kBatch];
#pragma unroll
                for (int k = 0; k < kBatch; ++k) {
                    const int cj = k0 + k < MAXW ? col_at(k0 + k) : i;
                    const int lr = cj - row0;
                    if ((unsigned)lr < (unsigned)nrows) {
                        zj[k] = s_z[lr];
                        pj[k] = sp_old[lr];
                    } else {
                        zj[k] = __ldcg(&E[cj].z);
                        pj[k] = __ldcg(&E[cj].p);
                    }
                }
#pragma unroll
                for (int k = 0; k < kBatch; ++k) {
                    if (k0 + k >= w || k0 + k >= MAXW) continue;
                    const float3 q = first ? xyz(zj[k])
                                           : f3(fmaf(beta, pj[k].x, zj[k].x), fmaf(beta, pj[k].y, zj[k].y),
                                                fmaf(beta, pj[k].z, zj[k].z));
                    acc = acc + mul(B[k0 + k], q - p);
                }
            }
            ap = acc;
            sig = (double)p.x * acc.x + (double)p.y * acc.y + (double)p.z * acc.z;
        }
        sig = warp_sum(sig);
        if (coarse) {
            // the warp's restriction of Ap, for the coarse correction's
            // update (it only feeds the preconditioner: float sums)
            const bool act = row && !li[li_idx].done;
            warp_restrict(c_nq, act ? ap : f3(0.f, 0.f, 0.f), c_w, s_cpart + (PC == 2 ? warp * kCoarsePartW : 0));
        }
        if (lane == 0 && has) spart[warp * kSlotW] = sig;
        __syncthreads();
        if (coarse)
            CHYSX_COARSE_PHASE(1, s_cw, true, ([&](LocalInst& L, const double* tot) { step_alpha(L, tot); }));
        else
            CHYSX_REDUCE_PHASE(1, kPollMax, true, ([&](LocalInst& L, const double* tot) { step_alpha(L, tot); }));
        if (s_flag) {
            ok = false;
            break;
        }
        if (!SYNC && s_exit) break;
        if (coarse) {
            // A_c^-1 R^T r_new = A_c^-1 R^T r - alpha A_c^-1 R^T A p, this row's share
            const float al = li[0].alpha;
            float cn[12];
#pragma unroll
            for (int u = 0; u < 12; ++u) cn[u] = u < c_U ? fmaf(-al, s_cw[u], s_cu[u]) : 0.f;
            c_blk = coarse_prolong(c_nq, cn, c_w);
        }

        double rz = 0.0, rr = 0.0;
        const bool act = row && !li[li_idx].done;
        if (act) {
            const float alpha = li[li_idx].alpha;
            x = f3(fmaf(alpha, p.x, x.x), fmaf(alpha, p.y, x.y), fmaf(alpha, p.z, x.z));
            r = f3(fmaf(-alpha, ap.x, r.x), fmaf(-alpha, ap.y, r.y), fmaf(-alpha, ap.z, r.z));
        }
        if (PC) {
            const float3 zn = precond(act ? r : f3(0.f, 0.f, 0.f));
            if (act) z = zn + c_blk;
        }
        if (act) {
            const LocalInst& L = li[li_idx];
            ZP* En = (L.iter & 1) ? zp0 : zp1;
            if (!PC) z = mul(Mi, r);
            En[i].z = f4(z);
            s_z[threadIdx.x] = f4(z);
            rz = (double)r.x * z.x + (double)r.y * z.y + (double)r.z * z.z;
            rr = (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z;
        }
        rz = warp_sum(rz);
        rr = warp_sum(rr);
        if (lane == 0 && has) {
            spart[warp * kSlotW] = rz;
            spart[warp * kSlotW + 1] = rr;
        }
        if (coarse) {
            // the warp's restriction of the new r: the coarse correction
            // restarts from R^T r every iteration (no drift)
            warp_restrict(c_nq, act ? r : f3(0.f, 0.f, 0.f), c_w, s_cpart + (PC == 2 ? warp * kCoarsePartW : 0));
        }
        __syncthreads();
        if (coarse)
            CHYSX_COARSE_PHASE(2, s_cu, false, ([&](LocalInst& L, const double* tot) { step_beta(bp, L, tot, cfg); }));
        else
            CHYSX_REDUCE_PHASE(2, kPollMax, false, ([&](LocalInst& L, const double* tot) { step_beta(bp, L, tot, cfg); }));
        if (s_flag) {
            ok = false;
            break;
        }
    }
    if (row) {
        v.x[i] = f4(x);
        v.r[i] = f4(r);
        v.z[i] = f4(z);
    }
    if (!ok) instances_fail(bp, li, nloc);
}

// x_{n+1} = x_n + dx, v = dx/dt * exp(-c dt) (cloth_simulator.cu:222-244) for
// the rows of every instance whose solve finished without NaN/Inf or a
// kernel error; other instances keep the caller's state.
__global__ void finalize_batch_kernel(StepArgs a, Vecs v, BatchPlan bp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int e = a.row_to_ext ? a.row_to_ext[i] : i;
    if (e < 0) return;
    const int st = bp.inst[bp.slice_inst[i >> 5]].status;
    if (st == kSolveNonfinite || st == kSolveKernelError) {
        keep_state(a, e);
        return;
    }
    const float4 d = v.x[i];
    const float3 xn = ld3(a.pos, e);
    st3(a.pos_out, e, f3(xn.x + d.x, xn.y + d.y, xn.z + d.z));
    const float inv_dt = 1.0f / a.dt;
    float3 vn = f3(d.x * inv_dt, d.y * inv_dt, d.z * inv_dt);
    if (a.damping > 0.0f) vn = vn * expf(-a.damping * a.dt);
    st3(a.vel_out, e, vn);
}

// Resets the barrier and per-instance states before a solve.
__global__ void pcg_persistent_reset_kernel(BatchPlan bp) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b == 0) {
        bp.bar->count = 0u;
        bp.bar->error = 0;
        bp.bar->ndone = 0u;
    }
    if (b < bp.n_inst) {
        InstState& G = bp.inst[b];
        G.rho = 0.0; G.rr = 0.0; G.bb = 0.0; G.tol2 = 0.0; G.rr0 = 0.0;
        G.iter = 0; G.status = kSolveConverged; G.done = 0; G.fallback = 0;
    }
    if (bp.fslots) {
        const size_t total = (size_t)3 * bp.n_slots * kSlotW;
        for (size_t k = b; k < total; k += (size_t)gridDim.x * blockDim.x) bp.fslots[k] = kSlotEmpty;
    }
}

}  // namespace chysx_b200
