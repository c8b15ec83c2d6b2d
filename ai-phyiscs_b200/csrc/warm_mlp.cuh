// Learned warm start: a per-vertex MLP that predicts the velocity change of
// the step from 1-ring features, giving the PCG an initial guess
// dx0 = dt (v + dv).  The solve still runs to the same relative residual (and
// falls back to the zero guess per instance when the guess is worse), so the
// network only changes the iteration count.  No counterpart in the
// reference.
//
// Network: 20 features -> 64 -> 64 -> 64 -> 3, GELU (erf form), BF16 weights
// and activations, FP32 accumulation on the tensor cores
// (mma.sync.m16n8k16 bf16).  A warp evaluates 16 rows at a time; the
// accumulator fragment of one layer (rows g, g+8; columns 2t, 2t+1 of each
// 8-wide tile) is exactly the A-operand fragment of the next layer, so
// activations never leave registers between layers.
//
// Features of row i (raw; standardised with the network's stored mean/std):
//   0-2   v_i
//   3-5   dt * (g + f_i / m_i)                 external velocity change
//   6-8   mean_j (x_j - x_i) / mean_j |x_j - x_i|   shape of the 1-ring
//   9-11  mean_j (v_j - v_i)
//   12-14 dt * a_i,  a_i = -grad E_i / m_i     explicit elastic velocity change
//   15-17 dt * mean_j a_j
//   18    1 if the vertex is pinned
//   19    mean log10 spring stiffness of its edges (0 without springs)
// Output: dv standardised by the stored output mean/std.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "cloth_kernels.cuh"

namespace chysx_b200 {

constexpr int kMlpIn = 20;
constexpr int kMlpInPad = 32;
constexpr int kMlpHid = 64;
constexpr int kMlpOut = 3;
constexpr int kMlpOutPad = 8;

// Flat FP32 parameter vector (host and master copy), in this order.
struct MlpOffsets {
    static constexpr int mu_in = 0;
    static constexpr int sd_in = mu_in + kMlpIn;
    static constexpr int mu_out = sd_in + kMlpIn;
    static constexpr int sd_out = mu_out + kMlpOut;
    static constexpr int w1 = sd_out + kMlpOut;             // [in][hid]
    static constexpr int b1 = w1 + kMlpIn * kMlpHid;
    static constexpr int w2 = b1 + kMlpHid;                 // [hid][hid]
    static constexpr int b2 = w2 + kMlpHid * kMlpHid;
    static constexpr int w3 = b2 + kMlpHid;
    static constexpr int b3 = w3 + kMlpHid * kMlpHid;
    static constexpr int w4 = b3 + kMlpHid;                 // [hid][out]
    static constexpr int b4 = w4 + kMlpHid * kMlpOut;
    static constexpr int total = b4 + kMlpOut;
};

// Packed BF16 weights for the tensor-core kernels.  Forward B operands are
// the transposed weights Wt[out][in] (k-pairs contiguous), rows padded by 8
// elements so the 8 fragment rows of a warp fall in distinct banks.
constexpr int kT1 = kMlpInPad + 8;   // 40
constexpr int kTH = kMlpHid + 8;     // 72
struct MlpFwd {
    __nv_bfloat16 wt1[kMlpHid * kT1];
    __nv_bfloat16 wt2[kMlpHid * kTH];
    __nv_bfloat16 wt3[kMlpHid * kTH];
    __nv_bfloat16 wt4[kMlpOutPad * kTH];
    float b1[kMlpHid], b2[kMlpHid], b3[kMlpHid], b4[kMlpOutPad];
    float mu_in[kMlpInPad], inv_sd_in[kMlpInPad];
    float mu_out[4], sd_out[4];
};
// backward B operands: W[in][out], rows padded (k-pairs along out)
struct MlpBwd {
    __nv_bfloat16 w2[kMlpHid * kTH];
    __nv_bfloat16 w3[kMlpHid * kTH];
    __nv_bfloat16 w4[kMlpHid * 24];  // out padded to 16 (+8)
};
struct MlpPacked {
    MlpFwd f;
    MlpBwd b;
};

__device__ __forceinline__ double warp_sum_d(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// ---------------------------------------------------------------------------
// tensor-core helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ uint32_t ld_u32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// One dense layer for a 16-row tile: acc[nt][4] = A(16 x 16*KT) * Wt^T,
// Wt given as [n][k] with row stride `ld` (in elements).
template <int KT, int NT>
__device__ __forceinline__ void layer_mma(float (&acc)[NT][4], const uint32_t (&a)[KT][4],
                                          const __nv_bfloat16* wt, int ld, int lane) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int n = 0; n < NT; ++n) {
        acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
#pragma unroll
        for (int k = 0; k < KT; ++k) {
            const __nv_bfloat16* base = wt + (size_t)(n * 8 + g) * ld + k * 16 + 2 * t;
            mma16816(acc[n], a[k], ld_u32(base), ld_u32(base + 8));
        }
    }
}

// Accumulator layout of 8 n-tiles (16 x 64) -> A fragments of 4 k-tiles.
__device__ __forceinline__ void acc_to_a(const float (&h)[8][4], uint32_t (&a)[4][4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        a[k][0] = pack_bf16(h[2 * k][0], h[2 * k][1]);
        a[k][1] = pack_bf16(h[2 * k][2], h[2 * k][3]);
        a[k][2] = pack_bf16(h[2 * k + 1][0], h[2 * k + 1][1]);
        a[k][3] = pack_bf16(h[2 * k + 1][2], h[2 * k + 1][3]);
    }
}

// bias + GELU in place; column of element (n, e) is 8n + 2t + (e & 1)
__device__ __forceinline__ void bias_gelu(float (&h)[8][4], const float* bias, int lane, float (*pre)[4] = nullptr) {
    const int t = lane & 3;
#pragma unroll
    for (int n = 0; n < 8; ++n)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float z = h[n][e] + bias[8 * n + 2 * t + (e & 1)];
            if (pre) pre[n][e] = z;
            h[n][e] = gelu(z);
        }
}

// Loads the A fragments of a 16 x 32 feature tile stored [row][kT1] in smem.
__device__ __forceinline__ void load_a_features(uint32_t (&a)[2][4], const __nv_bfloat16* f, int lane) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        a[k][0] = ld_u32(f + g * kT1 + k * 16 + 2 * t);
        a[k][1] = ld_u32(f + (g + 8) * kT1 + k * 16 + 2 * t);
        a[k][2] = ld_u32(f + g * kT1 + k * 16 + 2 * t + 8);
        a[k][3] = ld_u32(f + (g + 8) * kT1 + k * 16 + 2 * t + 8);
    }
}

// Full forward of one 16-row tile whose standardised BF16 features sit in
// smem; returns the 16 x 8 output accumulator (rows g, g+8; cols 2t, 2t+1).
__device__ __forceinline__ void mlp_tile_forward(const MlpFwd& W, const __nv_bfloat16* feat, int lane,
                                                 float (&out)[1][4]) {
    uint32_t a0[2][4];
    load_a_features(a0, feat, lane);
    float h[8][4];
    uint32_t a[4][4];
    layer_mma<2, 8>(h, a0, W.wt1, kT1, lane);
    bias_gelu(h, W.b1, lane);
    acc_to_a(h, a);
    layer_mma<4, 8>(h, a, W.wt2, kTH, lane);
    bias_gelu(h, W.b2, lane);
    acc_to_a(h, a);
    layer_mma<4, 8>(h, a, W.wt3, kTH, lane);
    bias_gelu(h, W.b3, lane);
    acc_to_a(h, a);
    layer_mma<4, 1>(out, a, W.wt4, kTH, lane);
    const int t = lane & 3;
#pragma unroll
    for (int e = 0; e < 4; ++e) out[0][e] += W.b4[2 * t + (e & 1)];
}

// ---------------------------------------------------------------------------
// Per-row feature gathering
// ---------------------------------------------------------------------------
// Assembly leaves, when features are requested: ap[i] = (a_i, pinned),
// b[i].w = mean log10 k of the row's springs.
__device__ __forceinline__ void row_features(const StepArgs& a, const DevTopo& t, const Vecs& v, int i,
                                             float (&f)[kMlpIn]) {
    const int e = a.row_to_ext ? a.row_to_ext[i] : i;
    const int s = i >> 5, lane = i & 31;
    const float3 xi = ld3(a.pos, e), vi = ld3(a.vel, e);
    float m = 1.0f;
    if (a.inv_mass) {
        const float wi = a.inv_mass[e];
        m = (wi > 1.0e-12f) ? (1.0f / wi) : 1.0e8f;
    }
    float3 ext = f3(a.gx, a.gy, a.gz);
    if (a.apply_force && a.force) ext = ext + ld3(a.force, e) * (1.0f / m);
    const float4 ai = v.ap[i];
    float3 dx = f3(0.f, 0.f, 0.f), dv = dx, aj = dx;
    float len = 0.f;
    const int so = t.slice_off[s];
    const int w = (t.slice_off[s + 1] - so) >> 5;
    int cnt = 0;
    for (int k = 0; k < w; ++k) {
        const int j = t.col[so + k * 32 + lane];
        if (j == i) continue;  // padding entry
        const int ej = a.row_to_ext ? a.row_to_ext[j] : j;
        const float3 d = ld3(a.pos, ej) - xi;
        dx = dx + d;
        len += len3(d);
        dv = dv + (ld3(a.vel, ej) - vi);
        aj = aj + xyz(v.ap[j]);
        ++cnt;
    }
    const float ic = cnt ? 1.0f / (float)cnt : 0.0f;
    const float il = len > 0.f ? (float)cnt / len : 0.f;
    const float dt = a.dt;
    f[0] = vi.x; f[1] = vi.y; f[2] = vi.z;
    f[3] = dt * ext.x; f[4] = dt * ext.y; f[5] = dt * ext.z;
    f[6] = dx.x * ic * il; f[7] = dx.y * ic * il; f[8] = dx.z * ic * il;
    f[9] = dv.x * ic; f[10] = dv.y * ic; f[11] = dv.z * ic;
    f[12] = dt * ai.x; f[13] = dt * ai.y; f[14] = dt * ai.z;
    f[15] = dt * aj.x * ic; f[16] = dt * aj.y * ic; f[17] = dt * aj.z * ic;
    f[18] = ai.w;
    f[19] = v.b[i].w;
}

// ---------------------------------------------------------------------------
// Fifth-generation tensor cores (tcgen05, sm_100a) for the network's
// inference: one elected thread issues the MMAs, operands sit in shared
// memory in the canonical K-major layout without swizzle (8-row x 16-byte
// core matrices), the FP32 accumulator lives in tensor memory (TMEM) and
// comes back to registers with tcgen05.ld.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// Byte offset of element (r, k) of a K-major bf16 operand with `sbo` bytes
// between 8-row groups and 128 bytes between K-adjacent core matrices.
__device__ __forceinline__ uint32_t umma_off(int r, int k, uint32_t sbo) {
    return (uint32_t)(r >> 3) * sbo + (uint32_t)(k >> 3) * 128u + (uint32_t)(r & 7) * 16u + (uint32_t)(k & 7) * 2u;
}
// Shared-memory matrix descriptor of that layout (start address, leading
// byte offset 128 = the two K-halves of one K = 16 step, stride byte offset
// `sbo`, descriptor version 1, no swizzle).
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
           (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, int accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// Bounded wait for phase `parity` of an mbarrier (1 s of globaltimer).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    unsigned long long t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        unsigned long long t1;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
        if (t1 - t0 > 1000000000ull) return false;
    }
}
// 16 consecutive FP32 columns of this warp's 32 TMEM lanes (one per thread).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&r)[16]) {
    uint32_t u[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n\ttcgen05.wait::ld.sync.aligned;"
        : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]), "=r"(u[8]),
          "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) r[q] = __uint_as_float(u[q]);
}

// ---------------------------------------------------------------------------
// Step kernel: features (optionally exported in caller order) and, when a
// network is loaded, the initial guess x = dt (v + dv).  One CTA of 128
// threads per 128-row tile, one row per thread: the thread gathers its
// row's features and writes them, standardised, as row `tid` of the A
// operand; thread 0 issues the layer's tcgen05 MMAs (M = 128, N = 64,
// K = 32 or 64; the last layer N = 16) into the TMEM accumulator, commits
// them to an mbarrier, and each warp reads its 32 rows back, adds the bias,
// applies GELU and writes the next layer's A rows.  Every wait is bounded;
// a failed wait leaves the guess of that tile as it was (the solve is
// correct from any start) and the CTA stops predicting.
// ---------------------------------------------------------------------------
constexpr int kGuessThreads = 128;  // = the tile's rows = the MMA's M
constexpr int kGuessTmemCols = 64;

__global__ void __launch_bounds__(kGuessThreads)
learned_guess_kernel(StepArgs a, DevTopo t, Vecs v, const MlpPacked* __restrict__ net, float* feat_out,
                     float* pred_out, int predict) {
    constexpr uint32_t kSbo32 = 4 * 128, kSbo64 = 8 * 128;  // 8-row group strides for K = 32, 64
    __shared__ __align__(1024) uint8_t s_a[kGuessThreads * kMlpHid * 2];
    __shared__ __align__(1024) uint8_t s_w1[kMlpHid * kMlpInPad * 2];
    __shared__ __align__(1024) uint8_t s_w2[kMlpHid * kMlpHid * 2];
    __shared__ __align__(1024) uint8_t s_w3[kMlpHid * kMlpHid * 2];
    __shared__ __align__(1024) uint8_t s_w4[16 * kMlpHid * 2];
    __shared__ float s_b[3][kMlpHid], s_b4[4], s_mu[kMlpInPad], s_isd[kMlpInPad], s_muo[4], s_sdo[4];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5;
    if (predict) {
        // the weights as B operands ([N][K], K-major), biases and scalings
        const MlpFwd& F = net->f;
        for (int q = tid; q < kMlpHid * kMlpInPad; q += kGuessThreads) {
            const int nn = q / kMlpInPad, k = q % kMlpInPad;
            *reinterpret_cast<__nv_bfloat16*>(s_w1 + umma_off(nn, k, kSbo32)) = F.wt1[nn * kT1 + k];
        }
        for (int q = tid; q < kMlpHid * kMlpHid; q += kGuessThreads) {
            const int nn = q / kMlpHid, k = q % kMlpHid;
            *reinterpret_cast<__nv_bfloat16*>(s_w2 + umma_off(nn, k, kSbo64)) = F.wt2[nn * kTH + k];
            *reinterpret_cast<__nv_bfloat16*>(s_w3 + umma_off(nn, k, kSbo64)) = F.wt3[nn * kTH + k];
        }
        for (int q = tid; q < 16 * kMlpHid; q += kGuessThreads) {
            const int nn = q / kMlpHid, k = q % kMlpHid;
            *reinterpret_cast<__nv_bfloat16*>(s_w4 + umma_off(nn, k, kSbo64)) =
                nn < kMlpOutPad ? F.wt4[nn * kTH + k] : __float2bfloat16_rn(0.f);
        }
        for (int q = tid; q < kMlpHid; q += kGuessThreads) {
            s_b[0][q] = F.b1[q];
            s_b[1][q] = F.b2[q];
            s_b[2][q] = F.b3[q];
        }
        if (tid < kMlpInPad) {
            s_mu[tid] = F.mu_in[tid];
            s_isd[tid] = F.inv_sd_in[tid];
        }
        if (tid < 4) {
            s_b4[tid] = F.b4[tid];
            s_muo[tid] = F.mu_out[tid];
            s_sdo[tid] = F.sd_out[tid];
        }
        if (warp == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                         "r"(kGuessTmemCols)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        if (tid == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&s_bar)), "r"(1) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        fence_async_smem();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t tmem_warp = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 lanes
    uint32_t phase = 0;
    bool live = predict != 0;  // uniform over the CTA
    const uint32_t a0 = smem_addr(s_a), w1 = smem_addr(s_w1), w2 = smem_addr(s_w2), w3 = smem_addr(s_w3),
                   w4 = smem_addr(s_w4);
    // one layer: MMAs over K in steps of 16, commit, bounded wait; every
    // thread then reads its row of the accumulator; false after a failed wait
    auto layer = [&](uint32_t wb, int kdim, int n) -> bool {
        const uint32_t sbo = kdim == kMlpInPad ? kSbo32 : kSbo64;
        fence_async_smem();  // the A rows written by every thread, for the tensor core
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            for (int s = 0; s < kdim / 16; ++s)
                umma_bf16(tmem, umma_desc(a0 + 256u * s, sbo), umma_desc(wb + 256u * s, sbo), umma_idesc_bf16(n), s > 0);
            umma_commit(&s_bar);
        }
        const bool ok = mbar_wait(&s_bar, phase);
        phase ^= 1u;
        tc_fence_after();
        return __syncthreads_and(ok) != 0;
    };
    // bias, GELU and BF16 of this thread's 64 accumulator columns into its A row (K = 64 layout)
    auto hidden = [&](const float* bias) {
#pragma unroll
        for (int c = 0; c < kMlpHid; c += 16) {
            float h[16];
            tmem_ld16(tmem_warp + c, h);
#pragma unroll
            for (int q = 0; q < 16; q += 8) {
                uint4 pk;
                pk.x = pack_bf16(gelu(h[q] + bias[c + q]), gelu(h[q + 1] + bias[c + q + 1]));
                pk.y = pack_bf16(gelu(h[q + 2] + bias[c + q + 2]), gelu(h[q + 3] + bias[c + q + 3]));
                pk.z = pack_bf16(gelu(h[q + 4] + bias[c + q + 4]), gelu(h[q + 5] + bias[c + q + 5]));
                pk.w = pack_bf16(gelu(h[q + 6] + bias[c + q + 6]), gelu(h[q + 7] + bias[c + q + 7]));
                *reinterpret_cast<uint4*>(s_a + umma_off(tid, c + q, kSbo64)) = pk;
            }
        }
    };
    const int n_tiles = (t.n + kGuessThreads - 1) / kGuessThreads;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int i = tile * kGuessThreads + tid;
        const int e = (i < t.n) ? (a.row_to_ext ? a.row_to_ext[i] : i) : -1;
        float f[kMlpIn];
#pragma unroll
        for (int q = 0; q < kMlpIn; ++q) f[q] = 0.f;
        if (e >= 0) {
            row_features(a, t, v, i, f);
            if (feat_out) {
#pragma unroll
                for (int q = 0; q < kMlpIn; ++q) feat_out[(size_t)e * kMlpIn + q] = f[q];
            }
        }
        if (!live) continue;
        // standardised BF16 features: row tid of A (K = 32 layout)
#pragma unroll
        for (int q = 0; q < kMlpInPad; q += 8) {
            float z[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
                z[u] = (e >= 0 && q + u < kMlpIn) ? (f[q + u] - s_mu[q + u]) * s_isd[q + u] : 0.f;
            uint4 pk;
            pk.x = pack_bf16(z[0], z[1]);
            pk.y = pack_bf16(z[2], z[3]);
            pk.z = pack_bf16(z[4], z[5]);
            pk.w = pack_bf16(z[6], z[7]);
            *reinterpret_cast<uint4*>(s_a + umma_off(tid, q, kSbo32)) = pk;
        }
        if (!layer(w1, kMlpInPad, kMlpHid)) { live = false; continue; }
        hidden(s_b[0]);
        if (!layer(w2, kMlpHid, kMlpHid)) { live = false; continue; }
        hidden(s_b[1]);
        if (!layer(w3, kMlpHid, kMlpHid)) { live = false; continue; }
        hidden(s_b[2]);
        if (!layer(w4, kMlpHid, 16)) { live = false; continue; }
        float o[16];
        tmem_ld16(tmem_warp, o);
        if (e >= 0) {
            const float dt = a.dt;
            const float3 dv = f3((o[0] + s_b4[0]) * s_sdo[0] + s_muo[0], (o[1] + s_b4[1]) * s_sdo[1] + s_muo[1],
                                 (o[2] + s_b4[2]) * s_sdo[2] + s_muo[2]);
            v.x[i] = make_float4(dt * (f[0] + dv.x), dt * (f[1] + dv.y), dt * (f[2] + dv.z), 0.f);
            if (pred_out) {
                pred_out[(size_t)e * 3] = dv.x;
                pred_out[(size_t)e * 3 + 1] = dv.y;
                pred_out[(size_t)e * 3 + 2] = dv.z;
            }
        }
    }
    // every MMA has completed (or its wait gave up: one more bounded wait
    // for it) before the columns are released
    if (predict) {
        if (!live) (void)mbar_wait(&s_bar, phase ^ 1u);  // the phase whose wait gave up
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (warp == 0)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kGuessTmemCols)
                         : "memory");
    }
}

// ---------------------------------------------------------------------------
// Training (standalone kernels over feature / target rows)
// ---------------------------------------------------------------------------

// Packs the FP32 master parameters into the BF16 tensor-core layout.
__global__ void mlp_pack_kernel(const float* __restrict__ p, MlpPacked* __restrict__ W) {
    using O = MlpOffsets;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nth = gridDim.x * blockDim.x;
    const __nv_bfloat16 z = __float2bfloat16_rn(0.f);
    for (int q = tid; q < kMlpHid * kT1; q += nth) {
        const int o = q / kT1, k = q % kT1;
        W->f.wt1[q] = k < kMlpIn ? __float2bfloat16_rn(p[O::w1 + k * kMlpHid + o]) : z;
    }
    for (int q = tid; q < kMlpHid * kTH; q += nth) {
        const int r = q / kTH, k = q % kTH;
        const bool in = k < kMlpHid;
        W->f.wt2[q] = in ? __float2bfloat16_rn(p[O::w2 + k * kMlpHid + r]) : z;   // Wt[out=r][in=k]
        W->f.wt3[q] = in ? __float2bfloat16_rn(p[O::w3 + k * kMlpHid + r]) : z;
        W->b.w2[q] = in ? __float2bfloat16_rn(p[O::w2 + r * kMlpHid + k]) : z;    // W[in=r][out=k]
        W->b.w3[q] = in ? __float2bfloat16_rn(p[O::w3 + r * kMlpHid + k]) : z;
    }
    for (int q = tid; q < kMlpOutPad * kTH; q += nth) {
        const int o = q / kTH, k = q % kTH;
        W->f.wt4[q] = (o < kMlpOut && k < kMlpHid) ? __float2bfloat16_rn(p[O::w4 + k * kMlpOut + o]) : z;
    }
    for (int q = tid; q < kMlpHid * 24; q += nth) {
        const int r = q / 24, k = q % 24;
        W->b.w4[q] = k < kMlpOut ? __float2bfloat16_rn(p[O::w4 + r * kMlpOut + k]) : z;
    }
    for (int q = tid; q < kMlpHid; q += nth) {
        W->f.b1[q] = p[O::b1 + q];
        W->f.b2[q] = p[O::b2 + q];
        W->f.b3[q] = p[O::b3 + q];
    }
    for (int q = tid; q < kMlpOutPad; q += nth) W->f.b4[q] = q < kMlpOut ? p[O::b4 + q] : 0.f;
    for (int q = tid; q < kMlpInPad; q += nth) {
        W->f.mu_in[q] = q < kMlpIn ? p[O::mu_in + q] : 0.f;
        const float sd = q < kMlpIn ? p[O::sd_in + q] : 1.f;
        W->f.inv_sd_in[q] = sd > 0.f ? 1.0f / sd : 0.f;
    }
    for (int q = tid; q < 4; q += nth) {
        W->f.mu_out[q] = q < kMlpOut ? p[O::mu_out + q] : 0.f;
        W->f.sd_out[q] = q < kMlpOut ? p[O::sd_out + q] : 1.f;
    }
}

// Forward + backward of one minibatch, one warp per 16 rows.  Writes the
// BF16 layer inputs A0..A3 ([rows][64], A0 padded to 32 in a 64-wide row)
// and BF16 pre-activation gradients dZ1..dZ4 ([rows][64], dZ4 uses 8
// columns) for the weight-gradient GEMM, the FP32 output (optional) and the
// per-warp sum of squared errors of the standardised output.
struct MlpTrainBufs {
    __nv_bfloat16* act[4];   // A0..A3, [rows][64]
    __nv_bfloat16* dz[4];    // dZ1..dZ4, [rows][64]
    float* out;              // [rows][3] predicted dv (de-standardised), may be null
    double* sse;             // [blocks * warps]
};

constexpr int kTrainWarps = 4;
constexpr size_t kTrainSmem = sizeof(MlpPacked) + sizeof(__nv_bfloat16) * kTrainWarps * 16 * kT1 +
                              sizeof(float) * kTrainWarps * 2 * 16 * 64;

__global__ void __launch_bounds__(kTrainWarps * 32)
mlp_train_tile_kernel(const MlpPacked* __restrict__ net, const float* __restrict__ feat,
                      const float* __restrict__ target, int rows, float grad_scale, MlpTrainBufs bufs) {
    // dynamic shared memory: packed weights, feature tiles, pre-activations
    extern __shared__ __align__(16) unsigned char s_raw[];
    MlpPacked& Wp = *reinterpret_cast<MlpPacked*>(s_raw);
    auto s_feat = reinterpret_cast<__nv_bfloat16(*)[16 * kT1]>(s_raw + sizeof(MlpPacked));
    auto s_z = reinterpret_cast<float(*)[2][16 * 64]>(s_raw + sizeof(MlpPacked) +
                                                     sizeof(__nv_bfloat16) * kTrainWarps * 16 * kT1);
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(net);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&Wp);
        for (int q = threadIdx.x; q < (int)(sizeof(MlpPacked) / 4); q += blockDim.x) dst[q] = src[q];
    }
    __syncthreads();
    const MlpFwd& W = Wp.f;
    const MlpBwd& WB = Wp.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int tiles = (rows + 15) / 16;
    double sse = 0.0;
    for (int tile = blockIdx.x * kTrainWarps + warp; tile < tiles; tile += gridDim.x * kTrainWarps) {
        const int r0 = tile * 16;
        // standardised features -> smem (lanes 0..15: one row each)
        if (lane < 16) {
            const int r = r0 + lane;
            __nv_bfloat16* fr = s_feat[warp] + lane * kT1;
            for (int q = 0; q < kMlpInPad; ++q) {
                float z = 0.f;
                if (r < rows && q < kMlpIn) z = (feat[(size_t)r * kMlpIn + q] - W.mu_in[q]) * W.inv_sd_in[q];
                fr[q] = __float2bfloat16_rn(z);
                if (r < rows) bufs.act[0][(size_t)r * 64 + q] = fr[q];
            }
        }
        __syncwarp();
        auto store_rows = [&](__nv_bfloat16* dst, const float (&h)[8][4]) {
#pragma unroll
            for (int n = 0; n < 8; ++n) {
                const int c = 8 * n + 2 * t;
                if (r0 + g < rows)
                    *reinterpret_cast<uint32_t*>(dst + (size_t)(r0 + g) * 64 + c) = pack_bf16(h[n][0], h[n][1]);
                if (r0 + g + 8 < rows)
                    *reinterpret_cast<uint32_t*>(dst + (size_t)(r0 + g + 8) * 64 + c) = pack_bf16(h[n][2], h[n][3]);
            }
        };
        // ---- forward
        uint32_t a0[2][4];
        load_a_features(a0, s_feat[warp], lane);
        float h[8][4], z3[8][4];
        float pre[8][4];
        uint32_t a[4][4];
        layer_mma<2, 8>(h, a0, W.wt1, kT1, lane);
        bias_gelu(h, W.b1, lane, pre);
#pragma unroll
        for (int n = 0; n < 8; ++n)
#pragma unroll
            for (int e = 0; e < 4; ++e) s_z[warp][0][(g + 8 * (e >> 1)) * 64 + 8 * n + 2 * t + (e & 1)] = pre[n][e];
        store_rows(bufs.act[1], h);
        acc_to_a(h, a);
        layer_mma<4, 8>(h, a, W.wt2, kTH, lane);
        bias_gelu(h, W.b2, lane, pre);
#pragma unroll
        for (int n = 0; n < 8; ++n)
#pragma unroll
            for (int e = 0; e < 4; ++e) s_z[warp][1][(g + 8 * (e >> 1)) * 64 + 8 * n + 2 * t + (e & 1)] = pre[n][e];
        store_rows(bufs.act[2], h);
        acc_to_a(h, a);
        layer_mma<4, 8>(h, a, W.wt3, kTH, lane);
        bias_gelu(h, W.b3, lane, z3);
        store_rows(bufs.act[3], h);
        acc_to_a(h, a);
        float o[1][4];
        layer_mma<4, 1>(o, a, W.wt4, kTH, lane);
        // ---- loss: standardised MSE over the 3 outputs
        float d4[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int r = r0 + g + 8 * (e >> 1), c = 2 * t + (e & 1);
            const float y = o[0][e] + W.b4[c];
            float d = 0.f;
            if (r < rows && c < kMlpOut) {
                if (target) {
                    const float tgt = (target[(size_t)r * kMlpOut + c] - W.mu_out[c]) / W.sd_out[c];
                    d = y - tgt;
                    sse += (double)d * d;
                }
                if (bufs.out) bufs.out[(size_t)r * kMlpOut + c] = y * W.sd_out[c] + W.mu_out[c];
            }
            d4[e] = d * grad_scale;  // dL/dy for L = grad_scale/2 * sum d^2
        }
        // dZ4 (16 x 8) -> global, and as A fragment of one k-tile (cols 8..15 zero)
        if (r0 + g < rows)
            *reinterpret_cast<uint32_t*>(bufs.dz[3] + (size_t)(r0 + g) * 64 + 2 * t) = pack_bf16(d4[0], d4[1]);
        if (r0 + g + 8 < rows)
            *reinterpret_cast<uint32_t*>(bufs.dz[3] + (size_t)(r0 + g + 8) * 64 + 2 * t) = pack_bf16(d4[2], d4[3]);
        uint32_t ad[1][4];
        ad[0][0] = pack_bf16(d4[0], d4[1]);
        ad[0][1] = pack_bf16(d4[2], d4[3]);
        ad[0][2] = 0u;
        ad[0][3] = 0u;
        // ---- backward: dA3 = dZ4 W4^T  (B(k=out, n=in) = W4[in][out])
        float dA[8][4];
        layer_mma<1, 8>(dA, ad, WB.w4, 24, lane);
        float dz[8][4];
#pragma unroll
        for (int n = 0; n < 8; ++n)
#pragma unroll
            for (int e = 0; e < 4; ++e) dz[n][e] = dA[n][e] * gelu_grad(z3[n][e]);
        store_rows(bufs.dz[2], dz);
        acc_to_a(dz, a);
        layer_mma<4, 8>(dA, a, WB.w3, kTH, lane);  // dA2 = dZ3 W3^T
#pragma unroll
        for (int n = 0; n < 8; ++n)
#pragma unroll
            for (int e = 0; e < 4; ++e)
                dz[n][e] = dA[n][e] * gelu_grad(s_z[warp][1][(g + 8 * (e >> 1)) * 64 + 8 * n + 2 * t + (e & 1)]);
        store_rows(bufs.dz[1], dz);
        acc_to_a(dz, a);
        layer_mma<4, 8>(dA, a, WB.w2, kTH, lane);  // dA1 = dZ2 W2^T
#pragma unroll
        for (int n = 0; n < 8; ++n)
#pragma unroll
            for (int e = 0; e < 4; ++e)
                dz[n][e] = dA[n][e] * gelu_grad(s_z[warp][0][(g + 8 * (e >> 1)) * 64 + 8 * n + 2 * t + (e & 1)]);
        store_rows(bufs.dz[0], dz);
        __syncwarp();
    }
    sse = warp_sum_d(sse);
    if (lane == 0) bufs.sse[(size_t)blockIdx.x * kTrainWarps + warp] = sse;
}

// Weight gradients on the fifth-generation tensor cores, split over the
// rows (the GEMM's K): CTA c forms the partial dW = act^T dz of rows
// [c kDwRows, (c + 1) kDwRows) as one M = 128 (in features, padded with
// zero rows) x N = 64 (out features, zero-padded) MMA chain from shared
// memory -- both operands MN-major (features contiguous, as act and dz are
// stored [row][64]) in the no-swizzle layout -- into TMEM, and its partial
// bias gradient; mlp_dw_reduce_kernel adds the partials in chunk order.
constexpr int kDwRows = 64;
constexpr int kDwThreads = 128;
constexpr int kDwPadSmem = 12 * 1024;
__host__ __device__ constexpr uint32_t umma_idesc_bf16_mn(int n) {
    return umma_idesc_bf16(n) | (1u << 15) | (1u << 16);  // A and B MN-major
}
__global__ void __launch_bounds__(kDwThreads)
mlp_dw_kernel(const __nv_bfloat16* __restrict__ act, const __nv_bfloat16* __restrict__ dz, int rows, int in_dim,
              int out_dim, float* __restrict__ part_w, float* __restrict__ part_b) {
    constexpr uint32_t kSbo = (kDwRows / 8) * 128;  // bytes between 8-feature groups
    __shared__ __align__(1024) uint8_t s_a[128 * kDwRows * 2];
    __shared__ __align__(1024) uint8_t s_b[64 * kDwRows * 2];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, c = blockIdx.x;
    const int r0 = c * kDwRows, nr = min(kDwRows, rows - r0);
    // element (f, k) of a feature-major operand: feature group f / 8 at
    // kSbo, row group k / 8 at 128 bytes, row k % 8 at 16, feature f % 8 at 2
    auto keep8 = [](uint4 v, int f0, int dim) {  // features f0 .. f0 + 7, those >= dim zeroed
        uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t lo = f0 + 2 * q < dim ? 0x0000FFFFu : 0u, hi = f0 + 2 * q + 1 < dim ? 0xFFFF0000u : 0u;
            w[q] &= lo | hi;
        }
        return make_uint4(w[0], w[1], w[2], w[3]);
    };
    for (int x = tid; x < kDwRows * 8; x += kDwThreads) {
        const int k = x >> 3, g = x & 7;
        uint4 va = make_uint4(0u, 0u, 0u, 0u), vb = va;
        if (k < nr) {
            va = keep8(*reinterpret_cast<const uint4*>(act + (size_t)(r0 + k) * 64 + g * 8), g * 8, in_dim);
            vb = keep8(*reinterpret_cast<const uint4*>(dz + (size_t)(r0 + k) * 64 + g * 8), g * 8, out_dim);
        }
        const uint32_t off = (uint32_t)g * kSbo + (uint32_t)(k >> 3) * 128u + (uint32_t)(k & 7) * 16u;
        *reinterpret_cast<uint4*>(s_a + off) = va;
        *reinterpret_cast<uint4*>(s_b + off) = vb;
    }
    for (int x = tid; x < 8 * (int)kSbo / 16; x += kDwThreads)  // feature groups 8..15 of A: zero
        reinterpret_cast<uint4*>(s_a + 8 * kSbo)[x] = make_uint4(0u, 0u, 0u, 0u);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                     "r"(64)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&s_bar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    if (tid == 0) {
        const uint32_t a0 = smem_addr(s_a), b0 = smem_addr(s_b);
        for (int s = 0; s < kDwRows / 16; ++s)
            umma_bf16(tmem, umma_desc(a0 + 256u * s, kSbo), umma_desc(b0 + 256u * s, kSbo), umma_idesc_bf16_mn(64),
                      s > 0);
        umma_commit(&s_bar);
    }
    const bool ok = __syncthreads_and(mbar_wait(&s_bar, 0)) != 0;
    tc_fence_after();
    float* pw = part_w + (size_t)c * 64 * 64;
    if (warp < 2) {  // TMEM lanes 0..63: the in features
        const int m = tid;
#pragma unroll
        for (int c16 = 0; c16 < 64; c16 += 16) {
            float h[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c16, h);
#pragma unroll
            for (int q = 0; q < 16; ++q) pw[m * 64 + c16 + q] = ok ? h[q] : __int_as_float(0x7fc00000);
        }
    }
    if (tid < 64) {  // partial bias gradient of output tid
        float bacc = 0.f;
        if (tid < out_dim)
            for (int k = 0; k < nr; ++k) bacc += __bfloat162float(dz[(size_t)(r0 + k) * 64 + tid]);
        part_b[(size_t)c * 64 + tid] = bacc;
    }
    if (!ok) (void)mbar_wait(&s_bar, 0);  // the MMAs must be done before the columns go
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64) : "memory");
}

// gw[in][out] and gb[out]: the chunks' partials added in chunk order.
__global__ void mlp_dw_reduce_kernel(const float* __restrict__ part_w, const float* __restrict__ part_b, int chunks,
                                     int in_dim, int out_dim, float* __restrict__ gw, float* __restrict__ gb) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < in_dim * out_dim) {
        const int m = q / out_dim, n = q % out_dim;
        float acc = 0.f;
        for (int c = 0; c < chunks; ++c) acc += part_w[(size_t)c * 64 * 64 + m * 64 + n];
        gw[q] = acc;
    } else if (q < in_dim * out_dim + out_dim) {
        const int n = q - in_dim * out_dim;
        float acc = 0.f;
        for (int c = 0; c < chunks; ++c) acc += part_b[(size_t)c * 64 + n];
        gb[n] = acc;
    }
}

// Adam on the FP32 master weights (only the trainable slice, from w1).
__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ grad, float* __restrict__ m1,
                                float* __restrict__ m2, int begin, int end, float lr, float b1, float b2,
                                float eps, float c1, float c2) {
    for (int q = begin + blockIdx.x * blockDim.x + threadIdx.x; q < end; q += gridDim.x * blockDim.x) {
        const float gq = grad[q];
        const float a = b1 * m1[q] + (1.f - b1) * gq;
        const float b = b2 * m2[q] + (1.f - b2) * gq * gq;
        m1[q] = a;
        m2[q] = b;
        p[q] -= lr * (a * c1) / (sqrtf(b * c2) + eps);
    }
}

}  // namespace chysx_b200
