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

namespace chysx_b200 {

constexpr int kSolveKernelError = 3;
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
    double* slots;                        // [inst_slot[n_inst] * 4]
    InstState* inst;                      // [n_inst]
    GridBarrier* bar;
};

// (z, p) of one row for the register-resident kernel's neighbour exchange
struct ZP {
    float4 z;
    float4 p;
};

struct LocalInst {
    double rho, rr, bb, tol2, sigma;
    float alpha, beta;
    int iter, done, status, fallback;
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

// Count-based grid barrier: every CTA adds 1 to a monotonic counter (a
// fire-and-forget release reduction) and thread 0 polls it with acquire
// loads until it reaches this barrier's target.  The wait is bounded in time;
// returns false (uniformly across the CTA) once any CTA flagged an error.
__device__ __forceinline__ bool grid_sync(GridBarrier* gb, unsigned& target, int* s_flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        target += gridDim.x;
        red_release_add(&gb->count, 1u);
        const unsigned long long t0 = global_ns();
        unsigned spins = 0;
        while ((int)(ld_acquire_gpu(&gb->count) - target) < 0) {
            if ((++spins & 255u) == 0) {
                if (*(volatile int*)&gb->error) break;
                if (global_ns() - t0 > kBarrierTimeoutNs) {
                    atomicExch(&gb->error, 1);
                    break;
                }
            }
        }
        *s_flag = *(volatile int*)&gb->error;
    }
    __syncthreads();
    return *s_flag == 0;
}

__device__ __forceinline__ float4 ldcg4(const float4* p) { return __ldcg(p); }

// ---------------------------------------------------------------------------
// Segmented reductions
// ---------------------------------------------------------------------------
// spart[(s - s0) * 4 + q] holds slice partials; write, for every instance
// this CTA touches, the sum over its slices into the instance's slot.
template <int BLOCK, int NV>
__device__ __forceinline__ void write_segment_slots(const BatchPlan& bp, const double* spart, int s0, int s1,
                                                    int il0, int il1) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int W = BLOCK / 32;
    for (int b = il0 + warp; b <= il1; b += W) {
        const int lo = max(s0, bp.inst_slice[b]), hi = min(s1, bp.inst_slice[b + 1]);
        double acc[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] = 0.0;
        for (int s = lo + lane; s < hi; s += 32) {
#pragma unroll
            for (int q = 0; q < NV; ++q) acc[q] += spart[(s - s0) * 4 + q];
        }
#pragma unroll
        for (int q = 0; q < NV; ++q) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        }
        if (lane == 0) {
            const int slot = bp.inst_slot[b] + ((int)blockIdx.x - bp.inst_cta_lo[b]);
#pragma unroll
            for (int q = 0; q < NV; ++q) bp.slots[(size_t)slot * 4 + q] = acc[q];
        }
    }
}

// Warp `warp` sums instance b's slots (after a barrier); every lane gets it.
template <int NV>
__device__ __forceinline__ void read_instance_total(const BatchPlan& bp, int b, double (&out)[NV]) {
    const int lane = threadIdx.x & 31;
    const int lo = bp.inst_slot[b], hi = bp.inst_slot[b + 1];
#pragma unroll
    for (int q = 0; q < NV; ++q) out[q] = 0.0;
    for (int k = lo + lane; k < hi; k += 32) {
#pragma unroll
        for (int q = 0; q < NV; ++q) out[q] += __ldcg(bp.slots + (size_t)k * 4 + q);
    }
#pragma unroll
    for (int q = 0; q < NV; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) out[q] += __shfl_xor_sync(0xffffffffu, out[q], o);
    }
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// ---------------------------------------------------------------------------
// Per-instance scalar steps shared by the persistent kernels.  Each runs on
// one warp per instance (the whole warp reads the instance's slots) and
// lane 0 updates the CTA-local copy; the first CTA touching an instance
// also publishes its state and counts it when it finishes.
// ---------------------------------------------------------------------------
template <int W>
__device__ __forceinline__ void instances_start(const BatchPlan& bp, LocalInst* li, int il0, int il1,
                                                const SolverCfg& cfg, int warm) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int b = il0 + warp; b <= il1; b += W) {
        double tot[4];
        read_instance_total<4>(bp, b, tot);
        if (lane != 0) continue;
        LocalInst& L = li[b - il0];
        const double bb = tot[2];
        const bool warm_ok = !warm || (isfinite(tot[0]) && isfinite(tot[1]) && tot[1] <= bb);
        L.fallback = warm_ok ? 0 : 1;
        L.rho = warm_ok ? tot[0] : tot[3];
        L.rr = warm_ok ? tot[1] : bb;
        L.bb = bb;
        L.tol2 = cfg.rel_tol * cfg.rel_tol * bb;
        L.iter = 0;
        L.alpha = 0.0f;
        L.beta = 0.0f;
        const bool bad = !isfinite(L.rho) || !isfinite(L.rr) || !isfinite(bb);
        const bool conv = cfg.use_tol && L.rr <= L.tol2;
        L.status = bad ? kSolveNonfinite : kSolveConverged;
        L.done = (bad || conv || cfg.max_iter <= 0) ? 1 : 0;
        if ((int)blockIdx.x == bp.inst_cta_lo[b]) {
            InstState& G = bp.inst[b];
            G.rr0 = L.rr;
            G.bb = bb;
            G.fallback = L.fallback;
            if (L.done) {
                G.rho = L.rho; G.rr = L.rr; G.iter = 0; G.status = L.status; G.done = 1;
                atomicAdd(&bp.bar->ndone, 1u);
            }
        }
    }
}

template <int W>
__device__ __forceinline__ void instances_alpha(const BatchPlan& bp, LocalInst* li, int il0, int il1) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int b = il0 + warp; b <= il1; b += W) {
        LocalInst& L = li[b - il0];
        if (L.done) continue;
        double tot[1];
        read_instance_total<1>(bp, b, tot);
        if (lane == 0) {
            const double sigma = tot[0];
            const double alpha = (sigma > 1.0e-37 || sigma < -1.0e-37) ? L.rho / sigma : 0.0;
            L.sigma = sigma;
            L.alpha = (float)alpha;
            if (!isfinite(sigma) || !isfinite(alpha)) L.status = kSolveNonfinite;
        }
    }
}

template <int W>
__device__ __forceinline__ void instances_beta(const BatchPlan& bp, LocalInst* li, int il0, int il1,
                                               const SolverCfg& cfg) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int b = il0 + warp; b <= il1; b += W) {
        LocalInst& L = li[b - il0];
        if (L.done) continue;
        double tot[2];
        read_instance_total<2>(bp, b, tot);
        if (lane != 0) continue;
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
            if ((int)blockIdx.x == bp.inst_cta_lo[b]) {
                InstState& G = bp.inst[b];
                G.rho = L.rho; G.rr = L.rr; G.iter = L.iter; G.status = L.status; G.done = 1;
                atomicAdd(&bp.bar->ndone, 1u);
            }
        }
    }
}

// A barrier failure leaves every unfinished instance flagged.
__device__ __forceinline__ void instances_fail(const BatchPlan& bp, const LocalInst* li, int il0, int il1) {
    if (threadIdx.x != 0) return;
    for (int b = il0; b <= il1; ++b) {
        if ((int)blockIdx.x == bp.inst_cta_lo[b]) {
            InstState& G = bp.inst[b];
            G.status = kSolveKernelError;
            G.iter = li[b - il0].iter;
            G.done = 1;
        }
    }
}

// ---------------------------------------------------------------------------
// The kernel
// ---------------------------------------------------------------------------
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
pcg_persistent_kernel(DevTopo t, Vecs v, BatchPlan bp, SolverCfg cfg, int warm, ZP*, ZP*) {
    extern __shared__ double s_mem[];
    __shared__ int s_flag;
    __shared__ int s_exit;
    constexpr int W = BLOCK / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s0 = bp.cta_slice[blockIdx.x], s1 = bp.cta_slice[blockIdx.x + 1];
    const int il0 = bp.cta_inst_lo[blockIdx.x], il1 = bp.cta_inst_hi[blockIdx.x];
    double* spart = s_mem;
    LocalInst* li = reinterpret_cast<LocalInst*>(s_mem + (size_t)bp.max_slices_per_cta * 4);
    GridBarrier* gb = bp.bar;
    unsigned gen = 0;  // barrier target; the counter starts at 0 every solve
    if (threadIdx.x == 0) s_flag = 0;
    bool ok = true;

    // ---- phase 0: initial residual and per-instance start ----------------
    // zero guess: r = b, z = M^-1 b were written by the assembly kernel.
    // warm guess: r = b - A x0, z = M^-1 r (pcg_solver.cu:29-51).
    for (int s = s0 + warp; s < s1; s += W) {
        const int i = s * 32 + lane;
        double rz = 0.0, rr = 0.0, bb = 0.0, bmb = 0.0;
        if (i < t.n) {
            const float3 b = xyz(v.b[i]);
            const S6 Mi = ld6(t.minv + (size_t)s * 192 + lane);
            const float3 zb = mul(Mi, b);
            bb = (double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z;
            bmb = (double)b.x * zb.x + (double)b.y * zb.y + (double)b.z * zb.z;
            if (warm) {
                const int so = t.slice_off[s];
                const int w = (t.slice_off[s + 1] - so) >> 5;
                const S6 D = ld6(t.diag + (size_t)s * 192 + lane);
                float3 ax = mul(D, xyz(v.x[i]));
                const float* vb = t.val + (size_t)so * 6 + lane;
                for (int k = 0; k < w; ++k) {
                    const int j = t.col[so + k * 32 + lane];
                    ax = ax + mul(ld6(vb + k * 192), xyz(v.x[j]));
                }
                const float3 r = b - ax;
                const float3 z = mul(Mi, r);
                v.r[i] = f4(r);
                v.z[i] = f4(z);
                rz = (double)r.x * z.x + (double)r.y * z.y + (double)r.z * z.z;
                rr = (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z;
            } else {
                rz = bmb;
                rr = bb;
            }
        }
        rz = warp_sum(rz); rr = warp_sum(rr); bb = warp_sum(bb); bmb = warp_sum(bmb);
        if (lane == 0) {
            double* sp = spart + (s - s0) * 4;
            sp[0] = rz; sp[1] = rr; sp[2] = bb; sp[3] = bmb;
        }
    }
    __syncthreads();
    write_segment_slots<BLOCK, 4>(bp, spart, s0, s1, il0, il1);
    ok = grid_sync(gb, gen, &s_flag);
    if (ok) {
        instances_start<W>(bp, li, il0, il1, cfg, warm);
        __syncthreads();
        if (warm) {
            // zero-guess fallback for instances whose guess was worse than zero
            bool any = false;
            for (int b = il0; b <= il1; ++b) any |= li[b - il0].fallback != 0;
            if (any) {
                for (int s = s0 + warp; s < s1; s += W) {
                    const int i = s * 32 + lane;
                    if (i >= t.n || !li[bp.slice_inst[s] - il0].fallback) continue;
                    const S6 Mi = ld6(t.minv + (size_t)s * 192 + lane);
                    const float4 b = v.b[i];
                    v.x[i] = make_float4(0.f, 0.f, 0.f, 0.f);
                    v.r[i] = b;
                    v.z[i] = f4(mul(Mi, xyz(b)));
                }
            }
            ok = grid_sync(gb, gen, &s_flag);
        }
    }

    // ---- iterations ---------------------------------------------------------
    const int iter_cap = cfg.max_iter + 2;  // belt: every instance is done by max_iter
    for (int guard = 0; ok && guard < iter_cap; ++guard) {
        // phase 1: p = z + beta p (own row and recomputed for neighbours),
        // Ap = A p, sigma = p.Ap
        for (int s = s0 + warp; s < s1; s += W) {
            const LocalInst& L = li[bp.slice_inst[s] - il0];
            const int i = s * 32 + lane;
            double sig = 0.0;
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
                float3 acc = mul(ld6(t.diag + (size_t)s * 192 + lane), pi);
                const float* vb = t.val + (size_t)so * 6 + lane;
                const int* cb = t.col + so + lane;
                for (int k = 0; k < w; ++k) {
                    const int j = cb[k * 32];
                    const S6 B = ld6(vb + k * 192);
                    const float4 zj = ldcg4(v.z + j);
                    float3 pj = xyz(zj);
                    if (!first) {
                        const float4 po = ldcg4(pold + j);
                        pj = f3(fmaf(beta, po.x, zj.x), fmaf(beta, po.y, zj.y), fmaf(beta, po.z, zj.z));
                    }
                    acc = acc + mul(B, pj);
                }
                v.ap[i] = f4(acc);
                sig = (double)pi.x * acc.x + (double)pi.y * acc.y + (double)pi.z * acc.z;
            }
            sig = warp_sum(sig);
            if (lane == 0) spart[(s - s0) * 4] = sig;
        }
        __syncthreads();
        write_segment_slots<BLOCK, 1>(bp, spart, s0, s1, il0, il1);
        ok = grid_sync(gb, gen, &s_flag);
        if (!ok) break;
        // ndone only changes in phase 3 and phase 0, i.e. never between this
        // barrier and the next, so every CTA takes the same decision here
        if (threadIdx.x == 0) s_exit = *(volatile unsigned*)&gb->ndone >= (unsigned)bp.n_inst;
        __syncthreads();
        if (s_exit) break;

        // phase 2: alpha = rho / sigma; x += alpha p; r -= alpha Ap; z = M^-1 r
        instances_alpha<W>(bp, li, il0, il1);
        __syncthreads();
        for (int s = s0 + warp; s < s1; s += W) {
            const LocalInst& L = li[bp.slice_inst[s] - il0];
            const int i = s * 32 + lane;
            double rz = 0.0, rr = 0.0;
            if (!L.done && i < t.n) {
                const float alpha = L.alpha;
                const float4 pi = ((L.iter & 1) ? v.p0 : v.p1)[i];
                const float4 api = v.ap[i], xi = v.x[i], ri = v.r[i];
                const float3 xn = f3(fmaf(alpha, pi.x, xi.x), fmaf(alpha, pi.y, xi.y), fmaf(alpha, pi.z, xi.z));
                const float3 rn = f3(fmaf(-alpha, api.x, ri.x), fmaf(-alpha, api.y, ri.y), fmaf(-alpha, api.z, ri.z));
                const float3 zn = mul(ld6(t.minv + (size_t)s * 192 + lane), rn);
                v.x[i] = f4(xn);
                v.r[i] = f4(rn);
                v.z[i] = f4(zn);
                rz = (double)rn.x * zn.x + (double)rn.y * zn.y + (double)rn.z * zn.z;
                rr = (double)rn.x * rn.x + (double)rn.y * rn.y + (double)rn.z * rn.z;
            }
            rz = warp_sum(rz);
            rr = warp_sum(rr);
            if (lane == 0) {
                spart[(s - s0) * 4] = rz;
                spart[(s - s0) * 4 + 1] = rr;
            }
        }
        __syncthreads();
        write_segment_slots<BLOCK, 2>(bp, spart, s0, s1, il0, il1);
        ok = grid_sync(gb, gen, &s_flag);
        if (!ok) break;

        // phase 3: beta, iteration count, convergence (pcg_solver.cu:436-454)
        instances_beta<W>(bp, li, il0, il1, cfg);
        __syncthreads();
    }
    if (!ok) instances_fail(bp, li, il0, il1);
}


// ---------------------------------------------------------------------------
// Register-resident variant for systems with at most one 32-row slice per
// warp: every thread owns one row for the whole solve and keeps its diagonal
// block, Jacobi inverse, off-diagonal blocks + columns (up to MAXW) and
// x, r, z, p in registers.  Per iteration it publishes only p (phase 1) and
// z (phase 2) for its neighbours, packed as one 32-byte entry per row in a
// double-buffered array, so a neighbour's (z, p_old) pair is one sector.
// Same phases, reductions, barrier and per-instance logic as
// pcg_persistent_kernel.
// ---------------------------------------------------------------------------

template <int W, int MAXW>
__global__ void __launch_bounds__(W * 32)
pcg_resident_kernel(DevTopo t, Vecs v, BatchPlan bp, SolverCfg cfg, int warm, ZP* zp0, ZP* zp1) {
    extern __shared__ double s_mem[];
    __shared__ int s_flag;
    __shared__ int s_exit;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s0 = bp.cta_slice[blockIdx.x], s1 = bp.cta_slice[blockIdx.x + 1];
    const int il0 = bp.cta_inst_lo[blockIdx.x], il1 = bp.cta_inst_hi[blockIdx.x];
    double* spart = s_mem;  // [W * 4]
    LocalInst* li = reinterpret_cast<LocalInst*>(s_mem + (size_t)W * 4);
    GridBarrier* gb = bp.bar;
    unsigned target = 0;
    if (threadIdx.x == 0) s_flag = 0;
    bool ok = true;

    const int s = s0 + warp;
    const bool has = s < s1;
    const int i = s * 32 + lane;
    const bool row = has && i < t.n;
    const int li_idx = has ? bp.slice_inst[s] - il0 : 0;

    // ---- load the row --------------------------------------------------
    S6 D{0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, Mi{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    S6 B[MAXW];
    int cols[MAXW];
    int w = 0;
    float3 b = f3(0.f, 0.f, 0.f), x = b, r = b, z = b, p = b;
#pragma unroll
    for (int k = 0; k < MAXW; ++k) {
        B[k] = S6{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        cols[k] = row ? i : 0;
    }
    if (row) {
        D = ld6(t.diag + (size_t)s * 192 + lane);
        Mi = ld6(t.minv + (size_t)s * 192 + lane);
        b = xyz(v.b[i]);
        const int so = t.slice_off[s];
        w = (t.slice_off[s + 1] - so) >> 5;
#pragma unroll
        for (int k = 0; k < MAXW; ++k) {
            if (k < w) {
                cols[k] = t.col[so + k * 32 + lane];
                B[k] = ld6(t.val + (size_t)so * 6 + (size_t)k * 192 + lane);
            }
        }
    }

    // ---- phase 0 -------------------------------------------------------
    {
        double rz = 0.0, rr = 0.0, bb = 0.0, bmb = 0.0;
        if (row) {
            const float3 zb = mul(Mi, b);
            bb = (double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z;
            bmb = (double)b.x * zb.x + (double)b.y * zb.y + (double)b.z * zb.z;
            if (warm) {
                x = xyz(v.x[i]);
                float3 ax = mul(D, x);
#pragma unroll
                for (int k = 0; k < MAXW; ++k)
                    if (k < w) ax = ax + mul(B[k], xyz(v.x[cols[k]]));
                r = b - ax;
                z = mul(Mi, r);
                rz = (double)r.x * z.x + (double)r.y * z.y + (double)r.z * z.z;
                rr = (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z;
            } else {
                r = b;
                z = zb;
                rz = bmb;
                rr = bb;
            }
            zp0[i].z = f4(z);
        }
        rz = warp_sum(rz); rr = warp_sum(rr); bb = warp_sum(bb); bmb = warp_sum(bmb);
        if (lane == 0 && has) {
            double* sp = spart + warp * 4;
            sp[0] = rz; sp[1] = rr; sp[2] = bb; sp[3] = bmb;
        }
    }
    __syncthreads();
    write_segment_slots<W * 32, 4>(bp, spart, s0, s1, il0, il1);
    ok = grid_sync(gb, target, &s_flag);
    if (ok) {
        instances_start<W>(bp, li, il0, il1, cfg, warm);
        __syncthreads();
        if (warm) {
            if (row && li[li_idx].fallback) {
                x = f3(0.f, 0.f, 0.f);
                r = b;
                z = mul(Mi, b);
                zp0[i].z = f4(z);
            }
            ok = grid_sync(gb, target, &s_flag);
        }
    }

    // ---- iterations ----------------------------------------------------
    const int iter_cap = cfg.max_iter + 2;
    float3 ap = f3(0.f, 0.f, 0.f);
    for (int guard = 0; ok && guard < iter_cap; ++guard) {
        double sig = 0.0;
        if (row && !li[li_idx].done) {
            const LocalInst& L = li[li_idx];
            const bool first = L.iter == 0;
            const float beta = L.beta;
            const ZP* E = (L.iter & 1) ? zp1 : zp0;
            ZP* En = (L.iter & 1) ? zp0 : zp1;
            p = first ? z : f3(fmaf(beta, p.x, z.x), fmaf(beta, p.y, z.y), fmaf(beta, p.z, z.z));
            En[i].p = f4(p);
            float3 acc = mul(D, p);
#pragma unroll
            for (int k = 0; k < MAXW; ++k) {
                if (k >= w) continue;
                const float4 zj = __ldcg(&E[cols[k]].z);
                float3 pj = xyz(zj);
                if (!first) {
                    const float4 po = __ldcg(&E[cols[k]].p);
                    pj = f3(fmaf(beta, po.x, zj.x), fmaf(beta, po.y, zj.y), fmaf(beta, po.z, zj.z));
                }
                acc = acc + mul(B[k], pj);
            }
            ap = acc;
            sig = (double)p.x * acc.x + (double)p.y * acc.y + (double)p.z * acc.z;
        }
        sig = warp_sum(sig);
        if (lane == 0 && has) spart[warp * 4] = sig;
        __syncthreads();
        write_segment_slots<W * 32, 1>(bp, spart, s0, s1, il0, il1);
        ok = grid_sync(gb, target, &s_flag);
        if (!ok) break;
        if (threadIdx.x == 0) s_exit = *(volatile unsigned*)&gb->ndone >= (unsigned)bp.n_inst;
        __syncthreads();
        if (s_exit) break;

        instances_alpha<W>(bp, li, il0, il1);
        __syncthreads();
        double rz = 0.0, rr = 0.0;
        if (row && !li[li_idx].done) {
            const LocalInst& L = li[li_idx];
            const float alpha = L.alpha;
            ZP* En = (L.iter & 1) ? zp0 : zp1;
            x = f3(fmaf(alpha, p.x, x.x), fmaf(alpha, p.y, x.y), fmaf(alpha, p.z, x.z));
            r = f3(fmaf(-alpha, ap.x, r.x), fmaf(-alpha, ap.y, r.y), fmaf(-alpha, ap.z, r.z));
            z = mul(Mi, r);
            En[i].z = f4(z);
            rz = (double)r.x * z.x + (double)r.y * z.y + (double)r.z * z.z;
            rr = (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z;
        }
        rz = warp_sum(rz);
        rr = warp_sum(rr);
        if (lane == 0 && has) {
            spart[warp * 4] = rz;
            spart[warp * 4 + 1] = rr;
        }
        __syncthreads();
        write_segment_slots<W * 32, 2>(bp, spart, s0, s1, il0, il1);
        ok = grid_sync(gb, target, &s_flag);
        if (!ok) break;
        instances_beta<W>(bp, li, il0, il1, cfg);
        __syncthreads();
    }
    if (row) {
        v.x[i] = f4(x);
        v.r[i] = f4(r);
        v.z[i] = f4(z);
    }
    if (!ok) instances_fail(bp, li, il0, il1);
}


// ---------------------------------------------------------------------------
// Single-reduction variant of the register-resident solve (Chronopoulos-Gear
// PCG): one grid barrier per iteration instead of two.  With u = M^-1 r,
// w = A u, m = M^-1 w, q = M^-1 s, s = A p:
//   q_k = m_k + b_k q_k-1,  s_k = w_k + b_k s_k-1,  p_k = u_k + b_k p_k-1
//   x += a_k p_k,  r -= a_k s_k,  u_k+1 = u_k - a_k q_k
//   w_k+1 = A u_k+1,  m_k+1 = M^-1 w_k+1
//   g = (r,u), d = (w,u), rr = (r,r) in one reduction
//   b_k+1 = g_k+1 / g_k,  a_k+1 = g_k+1 / (d_k+1 - b_k+1 g_k+1 / a_k)
// Every row publishes (u_k, m_k, q_k-1); a neighbour's u_k+1 is rebuilt from
// them with the owner's exact FMA sequence, so A u_k+1 sees one consistent
// vector and needs no second barrier.  Mathematically the same iterates as
// PCG (pcg_solver.cu:467-593); round-off differs.  Off-diagonal blocks of
// the CTA's rows live in shared memory.
// ---------------------------------------------------------------------------
struct UMQ {
    float4 u;
    float4 m;
    float4 q;
    float4 pad;
};

__device__ __forceinline__ float3 fma3(float a, float3 x, float3 y) {
    return f3(fmaf(a, x.x, y.x), fmaf(a, x.y, y.y), fmaf(a, x.z, y.z));
}

template <int W, int MAXW>
__global__ void __launch_bounds__(W * 32, 1)
pcg_resident_cg1_kernel(DevTopo t, Vecs v, BatchPlan bp, SolverCfg cfg, int warm, UMQ* e0, UMQ* e1) {
    extern __shared__ double s_mem[];
    __shared__ int s_flag;
    __shared__ int s_exit;
    constexpr int R = W * 32;  // rows per CTA
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s0 = bp.cta_slice[blockIdx.x], s1 = bp.cta_slice[blockIdx.x + 1];
    const int il0 = bp.cta_inst_lo[blockIdx.x], il1 = bp.cta_inst_hi[blockIdx.x];
    double* spart = s_mem;  // [W * 4]
    LocalInst* li = reinterpret_cast<LocalInst*>(s_mem + (size_t)W * 4);
    float* sblk = reinterpret_cast<float*>(li + bp.max_inst_per_cta);  // [MAXW * 6][R]
    int* scol = reinterpret_cast<int*>(sblk + (size_t)MAXW * 6 * R);   // [MAXW][R]
    GridBarrier* gb = bp.bar;
    unsigned target = 0;
    if (threadIdx.x == 0) s_flag = 0;
    bool ok = true;

    const int s = s0 + warp;
    const bool has = s < s1;
    const int i = s * 32 + lane;
    const bool row = has && i < t.n;
    const int li_idx = has ? bp.slice_inst[s] - il0 : 0;
    const int tid = threadIdx.x;

    S6 D{0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, Mi{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int w = 0;
    float3 b = f3(0.f, 0.f, 0.f);
    if (row) {
        D = ld6(t.diag + (size_t)s * 192 + lane);
        Mi = ld6(t.minv + (size_t)s * 192 + lane);
        b = xyz(v.b[i]);
        const int so = t.slice_off[s];
        w = (t.slice_off[s + 1] - so) >> 5;
        for (int k = 0; k < MAXW; ++k) {
            if (k < w) {
                scol[k * R + tid] = t.col[so + k * 32 + lane];
                const float* src = t.val + (size_t)so * 6 + (size_t)k * 192 + lane;
#pragma unroll
                for (int c = 0; c < 6; ++c) sblk[(k * 6 + c) * R + tid] = src[c * 32];
            }
        }
    }
    auto offdiag = [&](int k) {
        return S6{sblk[(k * 6 + 0) * R + tid], sblk[(k * 6 + 1) * R + tid], sblk[(k * 6 + 2) * R + tid],
                  sblk[(k * 6 + 3) * R + tid], sblk[(k * 6 + 4) * R + tid], sblk[(k * 6 + 5) * R + tid]};
    };

    // ---- initial residual: r0 = b - A x0, u0 = M^-1 r0 (phase 0a) -----------
    float3 x = f3(0.f, 0.f, 0.f), r = b, u = f3(0.f, 0.f, 0.f);
    double rz = 0.0, rr = 0.0, bb = 0.0, bmb = 0.0;
    if (row) {
        const float3 zb = mul(Mi, b);
        bb = (double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z;
        bmb = (double)b.x * zb.x + (double)b.y * zb.y + (double)b.z * zb.z;
        if (warm) {
            x = xyz(v.x[i]);
            float3 ax = mul(D, x);
            for (int k = 0; k < w; ++k) ax = ax + mul(offdiag(k), xyz(v.x[scol[k * R + tid]]));
            r = b - ax;
            u = mul(Mi, r);
            rz = (double)r.x * u.x + (double)r.y * u.y + (double)r.z * u.z;
            rr = (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z;
        } else {
            u = zb;
            rz = bmb;
            rr = bb;
        }
    }
    {
        double a0 = warp_sum(rz), a1 = warp_sum(rr), a2 = warp_sum(bb), a3 = warp_sum(bmb);
        if (lane == 0 && has) {
            double* sp = spart + warp * 4;
            sp[0] = a0; sp[1] = a1; sp[2] = a2; sp[3] = a3;
        }
    }
    __syncthreads();
    write_segment_slots<R, 4>(bp, spart, s0, s1, il0, il1);
    ok = grid_sync(gb, target, &s_flag);
    if (ok) {
        instances_start<W>(bp, li, il0, il1, cfg, warm);
        __syncthreads();
        if (row && li[li_idx].fallback) {
            x = f3(0.f, 0.f, 0.f);
            r = b;
            u = mul(Mi, b);
        }
        if (row) e0[i].u = f4(u);
    }
    // ---- w0 = A u0, m0 = M^-1 w0, first (g, d) -----------------------------------
    if (ok) ok = grid_sync(gb, target, &s_flag);
    float3 wv = f3(0.f, 0.f, 0.f), m = wv, q = wv, sv = wv, p = wv;
    if (ok) {
        double d = 0.0;
        if (row) {
            wv = mul(D, u);
            for (int k = 0; k < w; ++k) wv = wv + mul(offdiag(k), xyz(__ldcg(&e0[scol[k * R + tid]].u)));
            m = mul(Mi, wv);
            d = (double)wv.x * u.x + (double)wv.y * u.y + (double)wv.z * u.z;
            e0[i].m = f4(m);
            e0[i].q = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        d = warp_sum(d);
        if (lane == 0 && has) spart[warp * 4] = d;
        __syncthreads();
        write_segment_slots<R, 1>(bp, spart, s0, s1, il0, il1);
        ok = grid_sync(gb, target, &s_flag);
    }
    if (ok) {
        // a0 = g0 / d0, b0 = 0 (L.rho holds g; L.sigma holds alpha in FP64)
        for (int bq = il0 + warp; bq <= il1; bq += W) {
            LocalInst& L = li[bq - il0];
            double tot[1];
            read_instance_total<1>(bp, bq, tot);
            if (lane == 0 && !L.done) {
                const double a = (tot[0] > 1.0e-37 || tot[0] < -1.0e-37) ? L.rho / tot[0] : 0.0;
                L.sigma = a;
                L.alpha = (float)a;
                L.beta = 0.0f;
                if (!isfinite(a)) L.status = kSolveNonfinite;
            }
        }
        __syncthreads();
    }

    // ---- iterations: one reduction each ------------------------------------
    const int iter_cap = cfg.max_iter + 2;
    // single instance only (the host guarantees it): every CTA holds the same
    // instance state, so the exit decision below is uniform across the grid
    for (int guard = 0; ok && guard < iter_cap; ++guard) {
        if (threadIdx.x == 0) s_exit = li[0].done;
        __syncthreads();
        if (s_exit) break;
        double g = 0.0, d = 0.0, r2 = 0.0;
        if (row && !li[li_idx].done) {
            const LocalInst& L = li[li_idx];
            const float alpha = L.alpha, beta = L.beta;
            const UMQ* E = (L.iter & 1) ? e1 : e0;
            UMQ* En = (L.iter & 1) ? e0 : e1;
            q = fma3(beta, q, m);
            sv = fma3(beta, sv, wv);
            p = fma3(beta, p, u);
            x = fma3(alpha, p, x);
            r = fma3(-alpha, sv, r);
            u = fma3(-alpha, q, u);  // == what neighbours rebuild below
            float3 acc = mul(D, u);
            for (int k = 0; k < w; ++k) {
                const UMQ* ej = E + scol[k * R + tid];
                const float3 uj = xyz(__ldcg(&ej->u)), mj = xyz(__ldcg(&ej->m)), qj = xyz(__ldcg(&ej->q));
                const float3 qn = fma3(beta, qj, mj);
                acc = acc + mul(offdiag(k), fma3(-alpha, qn, uj));
            }
            wv = acc;
            m = mul(Mi, wv);
            En[i].u = f4(u);
            En[i].m = f4(m);
            En[i].q = f4(q);
            g = (double)r.x * u.x + (double)r.y * u.y + (double)r.z * u.z;
            d = (double)wv.x * u.x + (double)wv.y * u.y + (double)wv.z * u.z;
            r2 = (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z;
        }
        g = warp_sum(g);
        d = warp_sum(d);
        r2 = warp_sum(r2);
        if (lane == 0 && has) {
            spart[warp * 4] = g;
            spart[warp * 4 + 1] = d;
            spart[warp * 4 + 2] = r2;
        }
        __syncthreads();
        write_segment_slots<R, 3>(bp, spart, s0, s1, il0, il1);
        ok = grid_sync(gb, target, &s_flag);
        if (!ok) break;
        for (int bq = il0 + warp; bq <= il1; bq += W) {
            LocalInst& L = li[bq - il0];
            if (L.done) continue;
            double tot[3];
            read_instance_total<3>(bp, bq, tot);
            if (lane != 0) continue;
            const double g1 = tot[0], d1 = tot[1], rr1 = tot[2];
            const double g0 = L.rho, a0 = L.sigma;
            const double be = (g0 > 1.0e-37 || g0 < -1.0e-37) ? g1 / g0 : 0.0;
            const double den = d1 - (a0 != 0.0 ? be * g1 / a0 : 0.0);
            const double al = (den > 1.0e-37 || den < -1.0e-37) ? g1 / den : 0.0;
            L.rho = g1;
            L.rr = rr1;
            L.beta = (float)be;
            L.alpha = (float)al;
            L.sigma = al;
            L.iter += 1;
            const bool bad = L.status == kSolveNonfinite || !isfinite(g1) || !isfinite(rr1) || !isfinite(al);
            const bool conv = cfg.use_tol && rr1 <= L.tol2;
            int done = 0;
            if (bad) { L.status = kSolveNonfinite; done = 1; }
            else if (conv) { L.status = kSolveConverged; done = 1; }
            else if (L.iter >= cfg.max_iter) { L.status = cfg.use_tol ? kSolveMaxIter : kSolveConverged; done = 1; }
            if (done) {
                L.done = 1;
                if ((int)blockIdx.x == bp.inst_cta_lo[bq]) {
                    InstState& G = bp.inst[bq];
                    G.rho = L.rho; G.rr = L.rr; G.iter = L.iter; G.status = L.status; G.done = 1;
                    atomicAdd(&gb->ndone, 1u);
                }
            }
        }
        __syncthreads();
    }
    if (row) {
        v.x[i] = f4(x);
        v.r[i] = f4(r);
        v.z[i] = f4(u);
    }
    if (!ok) instances_fail(bp, li, il0, il1);
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
    if (st == kSolveNonfinite || st == kSolveKernelError) return;
    const float4 d = v.x[i];
    const float3 xn = ld3(a.pos, e);
    st3(a.pos, e, f3(xn.x + d.x, xn.y + d.y, xn.z + d.z));
    const float inv_dt = 1.0f / a.dt;
    float3 vn = f3(d.x * inv_dt, d.y * inv_dt, d.z * inv_dt);
    if (a.damping > 0.0f) vn = vn * expf(-a.damping * a.dt);
    st3(a.vel, e, vn);
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
}

}  // namespace chysx_b200
