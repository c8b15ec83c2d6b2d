// Coarse level of the two-level preconditioner of the register-resident PCG
// kernel (no counterpart in the reference, whose PCG is block-Jacobi).
//
// Coarse block B is the rows of G consecutive CTAs of the plan; its fields
// are the block's translation and, optionally, its three linear fields along
// the principal axes of its positions (coarse_types.h).  With R the matrix
// that maps a block's field amplitudes to its rows, the coarse system is
// A_c = R^T A R, block-sparse (a block's rows touch a handful of other
// blocks).  The preconditioner
//     M^-1 = P_local + R A_c^-1 R^T,
// P_local the CTA-local Chebyshev polynomial, is a fixed symmetric
// positive-definite operator, so the outer iteration stays plain PCG.  Per
// step: coarse_fields_kernel (the weights), coarse_assemble_kernel (CTAs per
// block, field pair and slice split, deterministic per-lane partial sums
// added in lane order, the splits added in order by the inversion) and
// coarse_invert_kernel (A_c^-1 densely, FP64 blocked
// Gauss-Jordan across the grid); per iteration the resident kernel forms its
// block of A_c^-1 R^T r from the blocks' restricted residuals, which ride on
// the existing reduction slots.
#pragma once

#include "coarse_types.h"

namespace chysx_b200 {

// row-major 3x3 component c -> plane of a symmetric 6-plane block
__device__ __forceinline__ int sym_plane(int c) {
    const int r = c / 3, k = c % 3;
    const int lo = r < k ? r : k, hi = r < k ? k : r;
    return lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
}

// Weight of field q of internal row i (q = 0: the translation).
__device__ __forceinline__ float coarse_weight(const CoarseArgs& ca, int i, int q) {
    if (q == 0) return 1.0f;
    const float4 w = ca.w[i];
    return q == 1 ? w.x : (q == 2 ? w.y : w.z);
}

// Sums of K doubles over a CTA of NT threads; every thread gets the totals.
template <int K, int NT>
__device__ __forceinline__ void cta_sums(double* v, double (*red)[K]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const double s = warp_sum(v[q]);
        if (lane == 0) red[warp][q] = s;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q) {
        double tot = 0.0;
        for (int w = 0; w < NT / 32; ++w) tot += red[w][q];
        v[q] = tot;
    }
    __syncthreads();
}

// The linear-field weights of coarse block B (nq = 4): centroid and
// covariance of the block's positions x_n (double), the principal axes by
// cyclic Jacobi rotations (thread 0), then s_a = (x_i - c).u_a / sd_a for
// every row, sd_a^2 = the variance along u_a per row; axes with variance
// below 1e-6 of the largest get weight 0.  Padding rows get weight 0.
__global__ void __launch_bounds__(256) coarse_fields_kernel(StepArgs a, CoarseArgs ca) {
    __shared__ double red[8][6];
    __shared__ float s_ax[3][3], s_isd[3], s_c[3];
    const int B = blockIdx.x;
    const int r0 = ca.cb_row0[B], r1 = min(ca.cb_row0[B + 1], a.n);
    auto ext_of = [&](int i) { return a.row_to_ext ? a.row_to_ext[i] : i; };
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = r0 + (int)threadIdx.x; i < r1; i += blockDim.x) {
        const int e = ext_of(i);
        if (e < 0) continue;
        v[0] += a.pos[3 * (size_t)e];
        v[1] += a.pos[3 * (size_t)e + 1];
        v[2] += a.pos[3 * (size_t)e + 2];
        v[3] += 1.0;
    }
    cta_sums<6, 256>(v, red);
    const double cnt = v[3] > 0.0 ? v[3] : 1.0;
    const double c0 = v[0] / cnt, c1 = v[1] / cnt, c2 = v[2] / cnt;
    double q[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = r0 + (int)threadIdx.x; i < r1; i += blockDim.x) {
        const int e = ext_of(i);
        if (e < 0) continue;
        const double d0 = a.pos[3 * (size_t)e] - c0, d1 = a.pos[3 * (size_t)e + 1] - c1, d2 = a.pos[3 * (size_t)e + 2] - c2;
        q[0] += d0 * d0; q[1] += d0 * d1; q[2] += d0 * d2;
        q[3] += d1 * d1; q[4] += d1 * d2; q[5] += d2 * d2;
    }
    cta_sums<6, 256>(q, red);
    if (threadIdx.x == 0) {
        double A[9] = {q[0], q[1], q[2], q[1], q[3], q[4], q[2], q[4], q[5]};
        double V[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        for (int sweep = 0; sweep < 30; ++sweep) {
            const double off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
            const double dia = A[0] * A[0] + A[4] * A[4] + A[8] * A[8];
            if (!(off > 1e-30 * dia)) break;  // diagonal to double precision
            for (int p = 0; p < 2; ++p)
                for (int r = p + 1; r < 3; ++r) {
                    const double apr = A[3 * p + r];
                    if (fabs(apr) < 1e-300) continue;
                    const double th = 0.5 * (A[3 * r + r] - A[3 * p + p]) / apr;
                    const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                    const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                    for (int k = 0; k < 3; ++k) {
                        const double akp = A[3 * k + p], akr = A[3 * k + r];
                        A[3 * k + p] = cs * akp - sn * akr;
                        A[3 * k + r] = sn * akp + cs * akr;
                    }
                    for (int k = 0; k < 3; ++k) {
                        const double apk = A[3 * p + k], ark = A[3 * r + k];
                        A[3 * p + k] = cs * apk - sn * ark;
                        A[3 * r + k] = sn * apk + cs * ark;
                    }
                    for (int k = 0; k < 3; ++k) {
                        const double vkp = V[3 * k + p], vkr = V[3 * k + r];
                        V[3 * k + p] = cs * vkp - sn * vkr;
                        V[3 * k + r] = sn * vkp + cs * vkr;
                    }
                }
        }
        int ord[3] = {0, 1, 2};  // by decreasing variance (stable)
        for (int x = 0; x < 3; ++x)
            for (int y = 0; y < 2; ++y)
                if (A[4 * ord[y + 1]] > A[4 * ord[y]]) { const int tmp = ord[y]; ord[y] = ord[y + 1]; ord[y + 1] = tmp; }
        const double lmax = fmax(A[0], fmax(A[4], A[8]));
        for (int k = 0; k < 3; ++k) {
            const int ax = ord[k];
            const double lam = A[4 * ax];
            const bool keep = lam > 1e-6 * lmax && lam > 0.0;
            for (int c = 0; c < 3; ++c) s_ax[k][c] = (float)V[3 * c + ax];
            s_isd[k] = keep ? (float)(1.0 / sqrt(lam / cnt)) : 0.0f;
        }
        s_c[0] = (float)c0; s_c[1] = (float)c1; s_c[2] = (float)c2;
    }
    __syncthreads();
    for (int i = r0 + (int)threadIdx.x; i < ca.cb_row0[B + 1]; i += blockDim.x) {
        const int e = i < a.n ? ext_of(i) : -1;
        float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
        if (e >= 0) {
            const float d0 = a.pos[3 * (size_t)e] - s_c[0], d1 = a.pos[3 * (size_t)e + 1] - s_c[1],
                        d2 = a.pos[3 * (size_t)e + 2] - s_c[2];
            w.x = (d0 * s_ax[0][0] + d1 * s_ax[0][1] + d2 * s_ax[0][2]) * s_isd[0];
            w.y = (d0 * s_ax[1][0] + d1 * s_ax[1][1] + d2 * s_ax[1][2]) * s_isd[1];
            w.z = (d0 * s_ax[2][0] + d1 * s_ax[2][1] + d2 * s_ax[2][2]) * s_isd[2];
        }
        ca.w[i] = w;
    }
}

// A_c block row of coarse block B for the row field qa = blockIdx.y and
// every column field, over split blockIdx.z of the block's slices (every
// ca.splits-th slice): 9 warps (one per component of the 3x3 block), lane l
// takes the rows l of the split's slices; per-lane sums of
// w_iqa w_jqb A_ij (the operator in its difference form, so the inertia of
// a block's translation is not lost against its elastic diagonal) by
// column block and qb in dynamic shared memory
// ([nq][9][max_nbr][32] floats), then each (qb, column block, component) sum
// over lanes in lane order (double) into the split's partial block row.  A
// row's entries are gathered once for all qb.
__global__ void __launch_bounds__(288) coarse_assemble_kernel(DevTopo t, CoarseArgs ca) {
    extern __shared__ float acc_s[];
    const int B = blockIdx.x, qa = blockIdx.y, nq = ca.nq, mn = ca.max_nbr;
    const int U = 3 * nq;
    const int c = threadIdx.x >> 5, l = threadIdx.x & 31;
    auto acc = [&](int qb, int k) -> float& { return acc_s[(((size_t)qb * 9 + c) * mn + k) * 32 + l]; };
    for (int qb = 0; qb < nq; ++qb)
        for (int k = 0; k < mn; ++k) acc(qb, k) = 0.0f;
    const int pl = sym_plane(c);
    const int self = ca.self_idx[B];
    const int s0 = ca.cb_row0[B] >> 5, s1 = ca.cb_row0[B + 1] >> 5;
    auto weights = [&](int i) {  // (w_i0, w_i1, w_i2, w_i3) = (1, s_1, s_2, s_3)
        if (nq == 1) return make_float4(1.f, 0.f, 0.f, 0.f);
        const float4 w = ca.w[i];
        return make_float4(1.f, w.x, w.y, w.z);
    };
    auto pick = [](float4 w, int q) { return q == 0 ? w.x : (q == 1 ? w.y : (q == 2 ? w.z : w.w)); };
    for (int s = s0 + (int)blockIdx.z; s < s1; s += ca.splits) {
        const int i = s * 32 + l;
        if (i >= t.n) break;
        const float4 wi4 = weights(i);
        const float wi = pick(wi4, qa);
        const float dv = wi * t.dnl[(size_t)s * 192 + pl * 32 + l];
        for (int qb = 0; qb < nq; ++qb) acc(qb, self) += dv * pick(wi4, qb);
        const int so = t.slice_off[s];
        const int w = (t.slice_off[s + 1] - so) >> 5;
        // the row's entries 8 at a time: every load of a batch in flight
        for (int k0 = 0; k0 < w; k0 += 8) {
            int nb8[8];
            float vv[8];
            float4 wv[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const bool in = k0 + k < w;
                const int e = so + (k0 + k) * 32 + l;
                const int cj = in ? t.col[e] : i;
                nb8[k] = in ? ca.ell_nbr[e] : 0;
                vv[k] = in ? wi * t.val[(size_t)so * 6 + (size_t)(k0 + k) * 192 + pl * 32 + l] : 0.0f;
                wv[k] = weights(cj);
            }
            // difference form: entry (i, j) adds w_i A_ij w_j^C to (B, C)
            // and -w_i A_ij w_i to (B, B) (the row's implied elastic
            // diagonal); inside the block both land on (B, B) as one term
            // w_i A_ij (w_j - w_i), a difference of smooth fields
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (k0 + k < w) {
                    if (nb8[k] == self) {
                        for (int qb = 0; qb < nq; ++qb) acc(qb, self) += vv[k] * (pick(wv[k], qb) - pick(wi4, qb));
                    } else {
                        for (int qb = 0; qb < nq; ++qb) {
                            acc(qb, nb8[k]) += vv[k] * pick(wv[k], qb);
                            acc(qb, self) -= vv[k] * pick(wi4, qb);
                        }
                    }
                }
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < nq * mn * 9; x += blockDim.x) {
        const int qb = x / (mn * 9), rem = x % (mn * 9), k = rem / 9, cc = rem % 9;
        double sum = 0.0;
        for (int y = 0; y < 32; ++y) sum += acc_s[(((size_t)qb * 9 + cc) * mn + k) * 32 + y];
        const int r = cc / 3, col = cc % 3;
        ca.acp[(size_t)blockIdx.z * ca.nb * mn * U * U + (((size_t)B * mn + k) * U + qa * 3 + r) * U + qb * 3 + col] =
            sum;
    }
}

// Inverse of the block-diagonal A_c of the batched coarse level: one CTA
// per instance b builds the dense m_b x m_b matrix of its coarse blocks
// (m_b = U x blocks <= U kBatchMaxBlocks) from their block rows, adding the
// assembly's splits in order and rounding once to FP32 (the stored A_c),
// scales by S = diag^-1/2, shifts by ca.shift I and inverts by Gauss-Jordan
// without pivoting in FP64 shared memory (per pivot the pivot row and column
// are copied aside, then every entry updated: two CTA barriers per pivot);
// an unknown whose field has zero weight on its whole block gets an identity
// row.  Output S W S (FP32) into ca.ainv + ca.inst_aoff[b]; a non-positive
// pivot sets ca.fail (the level is then off in the step's solve).  Dynamic
// shared memory: batched_invert_smem(max m_b) bytes.
constexpr int kBatchInvThreads = 256;
__host__ __device__ constexpr size_t batched_invert_smem(int m) {
    return ((size_t)m * (m + 1) + 3 * (size_t)m) * sizeof(double);
}
__global__ void __launch_bounds__(kBatchInvThreads) coarse_invert_batched_kernel(CoarseArgs ca) {
    extern __shared__ double inv_s[];
    const int b = blockIdx.x, U = 3 * ca.nq, mn = ca.max_nbr, tid = threadIdx.x;
    const int B0 = ca.inst_blk[b], nbk = ca.inst_blk[b + 1] - B0, m = U * nbk, ld = m + 1;
    double* a = inv_s;
    double* prow = a + (size_t)m * ld;
    double* pcol = prow + m;
    double* s_sc = pcol + m;
    const size_t total = (size_t)ca.nb * mn * U * U;
    for (int x = tid; x < m * ld; x += kBatchInvThreads) a[x] = 0.0;
    __syncthreads();
    for (int e = tid; e < nbk * mn * U * U; e += kBatchInvThreads) {
        const int Bl = e / (mn * U * U), rem = e % (mn * U * U), k = rem / (U * U), rc = rem % (U * U);
        const int B = B0 + Bl;
        if (k >= ca.nbr_cnt[B]) continue;
        const int C = ca.nbr[(size_t)B * mn + k] - B0;  // blocks couple inside their instance only
        const size_t src = ((size_t)B * mn + k) * U * U + rc;
        double v = 0.0;
        for (int z = 0; z < ca.splits; ++z) v += __ldcg(ca.acp + (size_t)z * total + src);
        const float vf = (float)v;
        ca.ac[src] = vf;
        a[(size_t)(Bl * U + rc / U) * ld + C * U + rc % U] = (double)vf;
    }
    __syncthreads();
    for (int i = tid; i < m; i += kBatchInvThreads) {
        const double d = a[(size_t)i * ld + i];
        s_sc[i] = d > 0.0 ? 1.0 / sqrt(d) : 0.0;
    }
    __syncthreads();
    for (int x = tid; x < m * m; x += kBatchInvThreads) {
        const int i = x / m, j = x % m;
        const double si = s_sc[i], sj = s_sc[j];
        double& v = a[(size_t)i * ld + j];
        v = si == 0.0 || sj == 0.0 ? (i == j ? 1.0 : 0.0) : v * si * sj + (i == j ? ca.shift : 0.0);
    }
    __syncthreads();
    bool bad = false;
    for (int k = 0; k < m; ++k) {
        const double p = a[(size_t)k * ld + k];
        const bool good = p > 1.0e-12;
        bad = bad || !good;
        const double ip = good ? 1.0 / p : 0.0;
        for (int x = tid; x < m; x += kBatchInvThreads) {
            prow[x] = a[(size_t)k * ld + x];
            pcol[x] = a[(size_t)x * ld + k];
        }
        __syncthreads();
        // row k: (j == k ? 1 : a_kj) / p; the others subtract a_ik times it
        // (warp w takes rows w, w + 8, ..., lane l columns l, l + 32, ...)
        for (int j = tid & 31; j < m; j += 32) {
            const double rk = (j == k ? 1.0 : prow[j]) * ip;
            for (int i = tid >> 5; i < m; i += kBatchInvThreads / 32) {
                double& v = a[(size_t)i * ld + j];
                v = i == k ? rk : fma(-pcol[i], rk, j == k ? 0.0 : v);
            }
        }
        __syncthreads();
    }
    if (bad && tid == 0) atomicExch(ca.fail, 1);
    float* out = ca.ainv + ca.inst_aoff[b];
    for (int x = tid; x < m * m; x += kBatchInvThreads) {
        const int i = x / m, j = x % m;
        const double vv = a[(size_t)i * ld + j] * s_sc[i] * s_sc[j];
        out[x] = (bad || !isfinite(vv)) ? 0.0f : (float)vv;
    }
}

// Dense inverse of A_c for both two-level preconditioners (m <=
// kCoarseDenseMax): FP64 blocked Gauss-Jordan elimination in place on the
// symmetrically scaled and shifted matrix S A_c S + ca.shift I
// (S = diag(A_c)^-1/2), padded to a multiple of 32 with identity rows, no
// pivoting (the shifted matrix is symmetric positive definite; an unknown
// whose field has zero weight on its whole block has an empty row and column
// and is given an identity row).  Per 32-column panel K, with T the inverse
// of the diagonal tile:
//     P1  W_KK <- T = W_KK^-1                      (one CTA, in shared memory)
//     P2  W_KJ <- T W_KJ             (J != K)
//     P3  W_IJ <- W_IJ - W_IK W_KJ   (I, J != K)
//     P4  W_IK <- -W_IK T            (I != K; done beside the next panel's P1)
// with a grid barrier between the phases (three per panel).  Cooperative
// launch (all CTAs co-resident), the barrier's counter zeroed before the
// launch, every wait bounded; a failed wait or a non-positive pivot sets
// ca.fail and the PCG kernel then runs without the coarse level.  Cross-CTA
// data goes through L2 (__ldcg / __stcg).  Output: ca.ainv = S W S (FP32).
constexpr int kInvTile = 32;
static_assert(kInvTile * kInvTile % kCoarseInvertThreads == 0, "P3 gives every thread whole tile entries");

// c = a * b for 32 x 32 tiles in shared memory (row stride 33); thread t
// of the kCoarseInvertThreads computes the outputs (t / 32 + j * R, t % 32),
// j < kTileOut, R = kCoarseInvertThreads / 32: one b entry serves its
// kTileOut independent sums; sign -1 stores -a * b.
constexpr int kTileOut = kInvTile * kInvTile / kCoarseInvertThreads;
__device__ __forceinline__ void tile_mul(const double (*a)[kInvTile + 1], const double (*b)[kInvTile + 1],
                                         double (*c)[kInvTile + 1], double sign) {
    constexpr int R = kCoarseInvertThreads / kInvTile;
    const int r0 = threadIdx.x / kInvTile, q = threadIdx.x % kInvTile;
    double acc[kTileOut];
#pragma unroll
    for (int j = 0; j < kTileOut; ++j) acc[j] = 0.0;
#pragma unroll 8
    for (int k = 0; k < kInvTile; ++k) {
        const double bk = b[k][q];
#pragma unroll
        for (int j = 0; j < kTileOut; ++j) acc[j] = fma(a[r0 + j * R][k], bk, acc[j]);
    }
#pragma unroll
    for (int j = 0; j < kTileOut; ++j) c[r0 + j * R][q] = sign * acc[j];
}

__global__ void __launch_bounds__(kCoarseInvertThreads) coarse_invert_kernel(CoarseArgs ca, GridBarrier* gb) {
    __shared__ int s_ok;
    __shared__ double sa[kInvTile][kInvTile + 1], sb[kInvTile][kInvTile + 1], sc_[kInvTile][kInvTile + 1];
    const int m = ca.m, U = 3 * ca.nq, mn = ca.max_nbr, nb = ca.nb;
    const int nt = (m + kInvTile - 1) / kInvTile, mp = nt * kInvTile;
    double* W = ca.work;                   // [mp][mp]
    double* sc = W + (size_t)mp * mp;      // [mp] scaling
    double* Tg = sc + mp;                  // [2][32][32] diagonal-tile inverses by panel parity
    const int tid = threadIdx.x;
    const int gt = blockIdx.x * blockDim.x + tid, gn = gridDim.x * blockDim.x;
    unsigned target = 0;
    if (tid == 0) s_ok = 1;
    __syncthreads();
    auto gsync = [&]() -> bool {
        __syncthreads();
        if (tid == 0 && s_ok) s_ok = barrier_arrive_wait(gb, target) ? 1 : 0;
        __syncthreads();
        return s_ok != 0;
    };
    auto ld_tile = [&](double (*t)[kInvTile + 1], const double* src) {  // tile at src, row stride mp
        for (int o = tid; o < kInvTile * kInvTile; o += blockDim.x)
            t[o / kInvTile][o % kInvTile] = __ldcg(src + (size_t)(o / kInvTile) * mp + o % kInvTile);
    };
    auto st_tile = [&](double* dst, const double (*t)[kInvTile + 1]) {
        for (int o = tid; o < kInvTile * kInvTile; o += blockDim.x)
            __stcg(dst + (size_t)(o / kInvTile) * mp + o % kInvTile, t[o / kInvTile][o % kInvTile]);
    };
    auto tile_at = [&](int I, int J) { return W + (size_t)I * kInvTile * mp + (size_t)J * kInvTile; };
    // dense A_c from its block rows
    for (size_t q = gt; q < (size_t)mp * mp; q += gn) __stcg(W + q, 0.0);
    if (!gsync()) goto fail;
    for (int e = gt; e < nb * mn * U * U; e += gn) {
        const int B = e / (mn * U * U), rem = e % (mn * U * U), k = rem / (U * U), rc = rem % (U * U);
        // the assembly's splits added in order, rounded once to FP32 (the
        // stored A_c that the inverse is of)
        double v = 0.0;
        for (int z = 0; z < ca.splits; ++z) v += __ldcg(ca.acp + (size_t)z * nb * mn * U * U + e);
        const float vf = (float)v;
        ca.ac[e] = vf;
        if (k >= ca.nbr_cnt[B]) continue;
        const int C = ca.nbr[B * mn + k];
        __stcg(W + (size_t)(B * U + rc / U) * mp + C * U + rc % U, (double)vf);
    }
    if (!gsync()) goto fail;
    for (int i = gt; i < mp; i += gn) {
        const double d = i < m ? __ldcg(W + (size_t)i * mp + i) : 0.0;
        __stcg(sc + i, d > 0.0 ? 1.0 / sqrt(d) : 0.0);
    }
    if (!gsync()) goto fail;
    for (size_t q = gt; q < (size_t)mp * mp; q += gn) {
        const int i = (int)(q / mp), j = (int)(q % mp);
        const double si = __ldcg(sc + i), sj = __ldcg(sc + j);
        __stcg(W + q, si == 0.0 || sj == 0.0 ? (i == j ? 1.0 : 0.0)
                                             : __ldcg(W + q) * si * sj + (i == j ? ca.shift : 0.0));
    }
    if (!gsync()) goto fail;
    for (int K = 0; K <= nt; ++K) {
        // P4 of the previous panel: W_I,K-1 <- -W_I,K-1 T_{K-1}
        if (K > 0) {
            const double* Tp = Tg + (size_t)((K - 1) & 1) * kInvTile * kInvTile;
            for (int I = blockIdx.x; I < nt; I += gridDim.x) {
                if (I == K - 1) continue;
                for (int o = tid; o < kInvTile * kInvTile; o += blockDim.x)
                    sb[o / kInvTile][o % kInvTile] = __ldcg(Tp + o);
                ld_tile(sa, tile_at(I, K - 1));
                __syncthreads();
                tile_mul(sa, sb, sc_, -1.0);
                __syncthreads();
                st_tile(tile_at(I, K - 1), sc_);
                __syncthreads();
            }
        }
        if (K == nt) {
            if (!gsync()) goto fail;
            break;
        }
        // P1: T = W_KK^-1 by Gauss-Jordan in shared memory (the last CTA,
        // the others being busy with P4 above): every pivot step reads the
        // tile of the previous step and writes the other of two buffers, so
        // one CTA barrier per pivot; every thread forms 1 / pivot itself
        if (blockIdx.x == gridDim.x - 1) {
            ld_tile(sa, tile_at(K, K));
            __syncthreads();
            double(*cur)[kInvTile + 1] = sa;
            double(*nxt)[kInvTile + 1] = sc_;
            bool bad = false;
            for (int k = 0; k < kInvTile; ++k) {
                const double p = cur[k][k];
                const bool good = p > 1.0e-12;
                bad = bad || !good;
                const double ip = good ? 1.0 / p : 0.0;
                // the thread's outputs (tid / 32 + j * R, tid % 32), as in tile_mul;
                // row k: (q == k ? 1 : a_kq) / p; the others subtract a_rk times it
                constexpr int R = kCoarseInvertThreads / kInvTile;
                const int r0 = tid / kInvTile, q = tid % kInvTile;
                const double rk = (q == k ? 1.0 : cur[k][q]) * ip;
#pragma unroll
                for (int j = 0; j < kTileOut; ++j) {
                    const int r = r0 + j * R;
                    nxt[r][q] = r == k ? rk : fma(-cur[r][k], rk, q == k ? 0.0 : cur[r][q]);
                }
                __syncthreads();
                double(*t)[kInvTile + 1] = cur;
                cur = nxt;
                nxt = t;
            }
            if (bad && tid == 0) atomicExch(ca.fail, 1);
            double* Tk = Tg + (size_t)(K & 1) * kInvTile * kInvTile;
            for (int o = tid; o < kInvTile * kInvTile; o += blockDim.x) __stcg(Tk + o, cur[o / kInvTile][o % kInvTile]);
            st_tile(tile_at(K, K), cur);
        }
        if (!gsync()) goto fail;
        // P2: W_KJ <- T W_KJ
        {
            const double* Tk = Tg + (size_t)(K & 1) * kInvTile * kInvTile;
            for (int J = blockIdx.x; J < nt; J += gridDim.x) {
                if (J == K) continue;
                for (int o = tid; o < kInvTile * kInvTile; o += blockDim.x)
                    sa[o / kInvTile][o % kInvTile] = __ldcg(Tk + o);
                ld_tile(sb, tile_at(K, J));
                __syncthreads();
                tile_mul(sa, sb, sc_, 1.0);
                __syncthreads();
                st_tile(tile_at(K, J), sc_);
                __syncthreads();
            }
        }
        if (!gsync()) goto fail;
        // P3: W_IJ <- W_IJ - W_IK W_KJ
        for (int x = blockIdx.x; x < nt * nt; x += gridDim.x) {
            const int I = x / nt, J = x % nt;
            if (I == K || J == K) continue;
            // the tile to update is read with the two factors (one round trip)
            double* dst = tile_at(I, J);
            double cur[kInvTile * kInvTile / kCoarseInvertThreads];
#pragma unroll
            for (int j = 0; j < kInvTile * kInvTile / kCoarseInvertThreads; ++j) {
                const int o = tid + j * kCoarseInvertThreads;
                cur[j] = __ldcg(dst + (size_t)(o / kInvTile) * mp + o % kInvTile);
            }
            ld_tile(sa, tile_at(I, K));
            ld_tile(sb, tile_at(K, J));
            __syncthreads();
            tile_mul(sa, sb, sc_, 1.0);
            __syncthreads();
#pragma unroll
            for (int j = 0; j < kInvTile * kInvTile / kCoarseInvertThreads; ++j) {
                const int o = tid + j * kCoarseInvertThreads;
                __stcg(dst + (size_t)(o / kInvTile) * mp + o % kInvTile, cur[j] - sc_[o / kInvTile][o % kInvTile]);
            }
            __syncthreads();
        }
        if (!gsync()) goto fail;
    }
    {
        const bool bad = *(volatile int*)ca.fail != 0;
        for (size_t q = gt; q < (size_t)m * m; q += gn) {
            const int i = (int)(q / m), j = (int)(q % m);
            const double v = __ldcg(W + (size_t)i * mp + j) * __ldcg(sc + i) * __ldcg(sc + j);
            ca.ainv[q] = (bad || !isfinite(v)) ? 0.0f : (float)v;
        }
    }
    return;
fail:
    if (tid == 0) atomicExch(ca.fail, 1);
}

}  // namespace chysx_b200
