// Coarse level of the two-level preconditioner of the register-resident PCG
// kernel (no counterpart in the reference, whose PCG is block-Jacobi).
//
// Each CTA block B of rows contributes three coarse unknowns: the block's
// rigid translation.  With R the matrix that copies a block's translation to
// every row of the block, the coarse system is A_c = R^T A R: the 3x3 block
// (B, C) sums A_ij over rows i of B and columns j of C.  It is block-sparse
// (a CTA's rows touch a handful of other CTAs' rows).  The preconditioner
//     M^-1 = P_local + R A_c^-1 R^T,
// P_local the CTA-local Chebyshev polynomial, is a fixed symmetric
// positive-definite operator, so the outer iteration stays plain PCG.  Per
// step: coarse_assemble_kernel (one CTA per block, deterministic per-lane
// partial sums added in lane order) and coarse_inverse_kernel (CTA B solves
// A_c X = [e_3B e_3B+1 e_3B+2] by block-Jacobi CG, giving rows 3B..3B+2 of
// A_c^-1); per iteration the resident kernel forms its block of
// A_c^-1 R^T r as one block sum, the blocks' restricted residuals riding on
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

// A_c block row of CTA block B: 9 warps (one per component), lane l takes
// the rows l of every slice of the block; per-lane sums in shared memory,
// then each (neighbour, component) sum over lanes in lane order (double).
__global__ void __launch_bounds__(288) coarse_assemble_kernel(DevTopo t, const int* __restrict__ cta_slice,
                                                              CoarseArgs ca) {
    __shared__ float acc[9][kCoarseMaxNbr][32];
    const int B = blockIdx.x;
    const int c = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (int q = 0; q < ca.max_nbr; ++q) acc[c][q][l] = 0.0f;
    const int pl = sym_plane(c);
    const int self = ca.self_idx[B];
    for (int s = cta_slice[B]; s < cta_slice[B + 1]; ++s) {
        const int i = s * 32 + l;
        if (i >= t.n) break;
        acc[c][self][l] += t.diag[(size_t)s * 192 + pl * 32 + l];
        const int so = t.slice_off[s];
        const int w = (t.slice_off[s + 1] - so) >> 5;
        for (int k = 0; k < w; ++k) {
            const int e = so + k * 32 + l;
            const int nb = ca.ell_nbr[e];
            acc[c][nb][l] += t.val[(size_t)so * 6 + (size_t)k * 192 + pl * 32 + l];
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < ca.max_nbr * 9; q += blockDim.x) {
        const int nb = q / 9, cc = q % 9;
        double sum = 0.0;
        for (int k = 0; k < 32; ++k) sum += acc[cc][nb][k];
        ca.ac[((size_t)B * ca.max_nbr + nb) * 9 + cc] = (float)sum;
    }
}

// Rows 3B..3B+2 of A_c^-1 (A_c symmetric: the columns), B = blockIdx.x:
// three block-Jacobi preconditioned CG solves in lockstep, one thread per
// coarse unknown, A_c in shared memory.  Stops when every relative residual
// is below kCoarseTol or after kCoarseMaxIts iterations; a non-finite solve
// leaves zero rows (the coarse level then adds nothing).  Dynamic shared
// memory: nb * max_nbr * 9 + 6 * 3 nb floats.
__global__ void __launch_bounds__(kCoarseThreads) coarse_inverse_kernel(CoarseArgs ca) {
    extern __shared__ float cs_mem[];
    __shared__ int s_nbr[kCoarseMaxBlocks * kCoarseMaxNbr];
    __shared__ int s_cnt[kCoarseMaxBlocks];
    __shared__ double s_red[2][kCoarseThreads / 32][6];
    const int nb = ca.nb, mn = ca.max_nbr, m3 = 3 * nb;
    const int B = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    constexpr int kWarps = kCoarseThreads / 32;
    float* a_s = cs_mem;                        // [nb][mn][9]
    float* p_s = a_s + (size_t)nb * mn * 9;     // [3][m3] search directions
    float* r_s = p_s + 3 * m3;                  // [3][m3] residuals
    for (int q = t; q < nb * mn * 9; q += blockDim.x) a_s[q] = ca.ac[q];
    for (int q = t; q < nb * mn; q += blockDim.x) s_nbr[q] = ca.nbr[q];
    for (int q = t; q < nb; q += blockDim.x) s_cnt[q] = ca.nbr_cnt[q];
    __syncthreads();
    const bool own = t < m3;
    const int blk = own ? t / 3 : 0, comp = own ? t % 3 : 0;
    // row `comp` of the inverse of A_c's diagonal block of `blk` (double)
    float di[3] = {0.f, 0.f, 0.f};
    if (own) {
        const float* a = a_s + ((size_t)blk * mn + ca.self_idx[blk]) * 9;
        const double a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3], a4 = a[4], a5 = a[5], a6 = a[6], a7 = a[7], a8 = a[8];
        const double det = a0 * (a4 * a8 - a5 * a7) - a1 * (a3 * a8 - a5 * a6) + a2 * (a3 * a7 - a4 * a6);
        const double s = det != 0.0 ? 1.0 / det : 0.0;
        const double adj[9] = {a4 * a8 - a5 * a7, a2 * a7 - a1 * a8, a1 * a5 - a2 * a4,
                               a5 * a6 - a3 * a8, a0 * a8 - a2 * a6, a2 * a3 - a0 * a5,
                               a3 * a7 - a4 * a6, a1 * a6 - a0 * a7, a0 * a4 - a1 * a3};
        for (int c = 0; c < 3; ++c) di[c] = (float)(adj[3 * comp + c] * s);
    }
    // sums of up to 6 values over the CTA, every thread gets the totals
    auto block_sums = [&](double* v, int k, int set) {
        for (int q = 0; q < k; ++q) {
            const double w = warp_sum(v[q]);
            if (lane == 0) s_red[set][warp][q] = w;
        }
        __syncthreads();
        for (int q = 0; q < k; ++q) {
            double tot = 0.0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) tot += s_red[set][w][q];
            v[q] = tot;
        }
    };
    auto precond = [&](int j) {  // (D_c^-1 r_j)_t from r_s
        const float* r = r_s + j * m3 + 3 * blk;
        return own ? di[0] * r[0] + di[1] * r[1] + di[2] * r[2] : 0.f;
    };
    float x[3], r[3], z[3], p[3];
    double rz[3];
    for (int j = 0; j < 3; ++j) {
        x[j] = 0.f;
        r[j] = own && t == 3 * B + j ? 1.f : 0.f;
        if (own) r_s[j * m3 + t] = r[j];
    }
    __syncthreads();
    {
        double v[3];
        for (int j = 0; j < 3; ++j) {
            z[j] = precond(j);
            p[j] = z[j];
            v[j] = (double)r[j] * z[j];
        }
        block_sums(v, 3, 1);
        for (int j = 0; j < 3; ++j) rz[j] = v[j];
    }
    bool bad = false;
    for (int it = 0; it < kCoarseMaxIts; ++it) {
        if (own)
            for (int j = 0; j < 3; ++j) p_s[j * m3 + t] = p[j];
        __syncthreads();
        float ap[3] = {0.f, 0.f, 0.f};
        if (own) {
            for (int k = 0; k < s_cnt[blk]; ++k) {
                const float* a = a_s + ((size_t)blk * mn + k) * 9 + 3 * comp;
                const int cb = 3 * s_nbr[blk * mn + k];
                const float a0 = a[0], a1 = a[1], a2 = a[2];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const float* pj = p_s + j * m3 + cb;
                    ap[j] = fmaf(a0, pj[0], fmaf(a1, pj[1], fmaf(a2, pj[2], ap[j])));
                }
            }
        }
        double v[6];
        for (int j = 0; j < 3; ++j) v[j] = (double)p[j] * ap[j];
        block_sums(v, 3, 0);
        for (int j = 0; j < 3; ++j) {
            const double al = (v[j] > 1e-300 || v[j] < -1e-300) ? rz[j] / v[j] : 0.0;
            if (!isfinite(al)) bad = true;
            x[j] = fmaf((float)al, p[j], x[j]);
            r[j] = fmaf(-(float)al, ap[j], r[j]);
            if (own) r_s[j * m3 + t] = r[j];
        }
        __syncthreads();
        for (int j = 0; j < 3; ++j) {
            z[j] = precond(j);
            v[j] = (double)r[j] * z[j];
            v[3 + j] = (double)r[j] * r[j];
        }
        block_sums(v, 6, 1);
        bool conv = true;
        for (int j = 0; j < 3; ++j) {
            const double be = (rz[j] > 1e-300 || rz[j] < -1e-300) ? v[j] / rz[j] : 0.0;
            rz[j] = v[j];
            p[j] = fmaf((float)be, p[j], z[j]);
            conv = conv && v[3 + j] <= kCoarseTol * kCoarseTol;
            if (!isfinite(v[3 + j])) bad = true;
        }
        if (bad || conv) break;  // uniform: every thread holds the same totals
    }
    if (own)
        for (int j = 0; j < 3; ++j) ca.ainv[(size_t)(3 * B + j) * m3 + t] = bad ? 0.f : x[j];
}

}  // namespace chysx_b200
