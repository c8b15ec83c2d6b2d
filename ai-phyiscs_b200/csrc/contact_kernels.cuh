// Contact terms of the implicit cloth step.
//
// Two kinds, both folded into the row-owner kernels rather than scattered
// with atomics into the assembled system:
//
//  * Static shapes (planes, oriented boxes): a particle's deepest
//    penetration gives a penalty gradient, a lagged IPC friction force, the
//    diagonal block k n n^T + alpha (I - n n^T) and a Coulomb-cone
//    projection of its residual (collision/static_contact.h:6-62,
//    static_contact.cu:111-381).  Everything is row-local, so the assembly
//    kernel's row owner evaluates it in registers.
//
//  * The contact operator (collision/contact_spmv.h:1-96): a caller-filled
//    list of four-particle contacts (pairs, weights w0..w3 + normal + depth,
//    a device-side count) that adds the penalty Hessian
//        C[i][j] = sum_c w_ci w_cj (k n n^T + alpha (I - n n^T))
//    to the system.  Its diagonal blocks are baked into the row's diagonal
//    and its gradient into the row's right-hand side by the assembly kernel;
//    its off-diagonal blocks ride inside every solver SpMV.  Contacts churn
//    every frame, so instead of atomics the step rebuilds, on the device, a
//    per-row list of the contact slots touching each row (count, scan,
//    fill; the assembly kernel then sorts each row's list, which makes every
//    sum run in a fixed order).
#pragma once

#include "contact_types.h"

namespace chysx_b200 {

// IPC smoothed 1/|u| (collision/friction.cuh:29-37).
__device__ __forceinline__ float f1_over_x(float u, float eps) {
    return u > eps ? 1.0f / u : (-u / eps + 2.0f) / eps;
}

// Deepest static-shape penetration of x: depth > 0 and the outward normal,
// or depth 0 (static_contact.cu:41-146: planes first, then boxes, a strictly
// deeper primitive wins).
__device__ __forceinline__ float static_deepest(const StaticContacts& sc, float3 x, float3& bn) {
    float best = 0.0f;
    bn = f3(0.f, 0.f, 0.f);
    const float* s = sc.shapes;
    for (int q = 0; q < sc.n_planes; ++q, s += 4) {
        const float3 nv = f3(s[0], s[1], s[2]);
        const float depth = sc.thickness - (dot3(nv, x) + s[3]);
        if (depth > best) { best = depth; bn = nv; }
    }
    for (int q = 0; q < sc.n_boxes; ++q, s += 15) {
        const float3 rel = x - f3(s[0], s[1], s[2]);
        const float3 ex = f3(s[6], s[7], s[8]), ey = f3(s[9], s[10], s[11]), ez = f3(s[12], s[13], s[14]);
        const float qx = dot3(rel, ex), qy = dot3(rel, ey), qz = dot3(rel, ez);
        const float dx = fabsf(qx) - s[3], dy = fabsf(qy) - s[4], dz = fabsf(qz) - s[5];
        float d;
        float3 nv;
        if (dx <= 0.0f && dy <= 0.0f && dz <= 0.0f) {
            // inside: the nearest face
            if (dx >= dy && dx >= dz) { nv = qx >= 0.0f ? ex : ex * -1.0f; d = dx; }
            else if (dy >= dz) { nv = qy >= 0.0f ? ey : ey * -1.0f; d = dy; }
            else { nv = qz >= 0.0f ? ez : ez * -1.0f; d = dz; }
        } else {
            const float cx = dx > 0.0f ? dx : 0.0f, cy = dy > 0.0f ? dy : 0.0f, cz = dz > 0.0f ? dz : 0.0f;
            d = sqrtf(cx * cx + cy * cy + cz * cz);
            const float inv = 1.0f / fmaxf(d, 1.0e-30f);
            const float sx = qx > 0.0f ? cx : -cx, sy = qy > 0.0f ? cy : -cy, sz = qz > 0.0f ? cz : -cz;
            nv = ex * (sx * inv) + ey * (sy * inv) + ez * (sz * inv);
        }
        const float depth = sc.thickness - d;
        if (depth > best) { best = depth; bn = nv; }
    }
    return best;
}

// Static contact of one row at x_n with velocity vel: adds the penalty and
// lagged-friction gradient to g and the block k n n^T + alpha (I - n n^T) to
// D (static_contact.cu:186-285).  Returns the depth (0: no contact).
__device__ __forceinline__ float static_contact_row(const StaticContacts& sc, float3 x, float3 vel, float dt,
                                                    float3& g, S6& D, float3& bn) {
    const float depth = static_deepest(sc, x, bn);
    if (!(depth > 0.0f)) return 0.0f;
    const float kd = -sc.k * depth;
    g = f3(g.x + kd * bn.x, g.y + kd * bn.y, g.z + kd * bn.z);
    float al = 0.0f;
    if (sc.mu > 0.0f) {
        const float3 dxv = vel * dt;
        const float vn = dot3(bn, dxv);
        const float3 ut = dxv - bn * vn;
        const float un = sqrtf(ut.x * ut.x + ut.y * ut.y + ut.z * ut.z);
        al = sc.mu * (sc.k * depth) * f1_over_x(un, sc.eps);
        g = f3(g.x - al * ut.x, g.y - al * ut.y, g.z - al * ut.z);
    }
    const float k = sc.k;
    D.xx += k * bn.x * bn.x + al * (1.0f - bn.x * bn.x);
    D.xy += k * bn.x * bn.y + al * (-bn.x * bn.y);
    D.xz += k * bn.x * bn.z + al * (-bn.x * bn.z);
    D.yy += k * bn.y * bn.y + al * (1.0f - bn.y * bn.y);
    D.yz += k * bn.y * bn.z + al * (-bn.y * bn.z);
    D.zz += k * bn.z * bn.z + al * (1.0f - bn.z * bn.z);
    return depth;
}

// Coulomb-cone projection of the assembled residual b of a row in static
// contact (static_contact.cu:306-381): F0 = b - k depth n; only F0's push
// into the surface loads the cone.
__device__ __forceinline__ float3 coulomb_project(const StaticContacts& sc, float3 b, float3 bn, float depth) {
    const float push = sc.k * depth;
    const float3 F0 = f3(b.x - push * bn.x, b.y - push * bn.y, b.z - push * bn.z);
    const float f0n = F0.x * bn.x + F0.y * bn.y + F0.z * bn.z;
    const float fn = fmaxf(0.0f, -f0n);
    if (fn <= 0.0f) return b;
    const float3 F0t = f3(F0.x - f0n * bn.x, F0.y - f0n * bn.y, F0.z - f0n * bn.z);
    const float ft2 = F0t.x * F0t.x + F0t.y * F0t.y + F0t.z * F0t.z;
    if (ft2 <= 0.0f) return b;
    const float ft = sqrtf(ft2);
    const float cone = sc.mu * fn;
    if (ft <= cone) return f3(b.x - F0t.x, b.y - F0t.y, b.z - F0t.z);
    const float shrink = cone / ft;
    return f3(b.x - shrink * F0t.x, b.y - shrink * F0t.y, b.z - shrink * F0t.z);
}

__device__ __forceinline__ float sel4(float4 v, int s) {
    return s == 0 ? v.x : (s == 1 ? v.y : (s == 2 ? v.z : v.w));
}

// Gradient and diagonal of the contact operator for row i (contact_spmv.cu:
// 84-165, self_collision_constraint.cu:45-95).  Sorts the row's list first,
// so this and every later pass over it sum in (contact, slot) order.
__device__ __forceinline__ void contact_assemble_row(const ContactOp& co, int i, float3& g, S6& D) {
    const int lo = co.off[i], hi = co.off[i + 1];
    for (int a = lo + 1; a < hi; ++a) {
        const int key = co.ent[a];
        int b = a - 1;
        while (b >= lo && co.ent[b] > key) {
            co.ent[b + 1] = co.ent[b];
            --b;
        }
        co.ent[b + 1] = key;
    }
    for (int e = lo; e < hi; ++e) {
        const int code = co.ent[e];
        const PrepContact& r = co.rec[code >> 2];
        const float ws = sel4(r.w, code & 3);
        const float4 nk = r.nk, ga = r.ga;
        g = f3(g.x + ws * ga.x, g.y + ws * ga.y, g.z + ws * ga.z);
        const float ww = ws * ws;
        const float d = nk.w, al = ga.w;
        D.xx += ww * (d * nk.x * nk.x + al);
        D.xy += ww * (d * nk.x * nk.y);
        D.xz += ww * (d * nk.x * nk.z);
        D.yy += ww * (d * nk.y * nk.y + al);
        D.yz += ww * (d * nk.y * nk.z);
        D.zz += ww * (d * nk.z * nk.z + al);
    }
}

// Off-diagonal part of the contact operator applied to a vector, row i:
// sum over the row's slots s of w_s ((k - alpha) (n.t) n + alpha t) with
// t = sum_{j != s} w_j p_j (contact_spmv.cu:171-236).  pf(j) yields p_j.
template <class PF>
__device__ __forceinline__ float3 contact_spmv_row(const ContactOp& co, int i, PF&& pf) {
    float3 acc = f3(0.f, 0.f, 0.f);
    const int lo = co.off[i], hi = co.off[i + 1];
    for (int e = lo; e < hi; ++e) {
        const int code = co.ent[e];
        const int s = code & 3;
        const PrepContact& r = co.rec[code >> 2];
        const int4 rows = r.rows;
        const float4 w = r.w, nk = r.nk;
        const float al = r.ga.w;
        const int rr[4] = {rows.x, rows.y, rows.z, rows.w};
        const float wv[4] = {w.x, w.y, w.z, w.w};
        float3 t = f3(0.f, 0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (j == s || rr[j] < 0) continue;
            const float3 pj = pf(rr[j]);
            t = f3(fmaf(wv[j], pj.x, t.x), fmaf(wv[j], pj.y, t.y), fmaf(wv[j], pj.z, t.z));
        }
        const float wi = sel4(w, s);
        const float dn = nk.x * t.x + nk.y * t.y + nk.z * t.z;
        const float nc = wi * nk.w * dn;
        const float wa = wi * al;
        acc = f3(acc.x + nc * nk.x + wa * t.x, acc.y + nc * nk.y + wa * t.y, acc.z + nc * nk.z + wa * t.z);
    }
    return acc;
}

// ---------------------------------------------------------------------------
// Per-step list build
// ---------------------------------------------------------------------------

// Prepares every live contact (index < min(*count, max_contacts)) and
// counts its slots per row.  A contact whose stiffness is not finite and
// positive is skipped (contact_spmv.cu:102-106); one with a weighted slot
// outside [0, n_particles) is dropped and counted in stats[1].
// stats[0] = live contacts.  cnt and stats were zeroed by the step.
__global__ void contact_prep_kernel(ContactInput in, int n_particles, int* __restrict__ cnt,
                                    PrepContact* __restrict__ rec, int* __restrict__ stats) {
    const int raw = *in.count;
    const int nc = raw < in.max_contacts ? (raw > 0 ? raw : 0) : in.max_contacts;
    if (blockIdx.x == 0 && threadIdx.x == 0) stats[0] = nc;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        PrepContact r;
        r.rows = make_int4(-1, -1, -1, -1);
        const float k = in.stiffnesses ? in.stiffnesses[c] : in.stiffness;
        const int4 ids = in.pairs[c];
        const float4 w = in.weights[2 * c], nd = in.weights[2 * c + 1];
        r.w = w;
        int rows[4] = {ids.x, ids.y, ids.z, ids.w};
        const float wv[4] = {w.x, w.y, w.z, w.w};
        bool live = k > 0.0f && isfinite(k);
        bool bad = false;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (wv[s] == 0.0f) rows[s] = -1;
            else if (rows[s] < 0 || rows[s] >= n_particles) bad = true;
            else if (in.ext_to_row) rows[s] = in.ext_to_row[rows[s]];
        }
        if (bad && live) atomicAdd(&stats[1], 1);
        live = live && !bad;
        float al = 0.0f;
        float3 gc = f3(0.f, 0.f, 0.f);
        if (live) {
            const float kd = -k * nd.w;
            gc = f3(kd * nd.x, kd * nd.y, kd * nd.z);
            if (in.mu > 0.0f && in.slips) {
                const float4 u = in.slips[c];
                al = in.mu * (k * nd.w) * f1_over_x(u.w, in.eps);
                gc = f3(gc.x - al * u.x, gc.y - al * u.y, gc.z - al * u.z);
            }
            r.rows = make_int4(rows[0], rows[1], rows[2], rows[3]);
#pragma unroll
            for (int s = 0; s < 4; ++s)
                if (rows[s] >= 0) atomicAdd(&cnt[rows[s]], 1);
        }
        r.nk = make_float4(nd.x, nd.y, nd.z, k - al);
        r.ga = make_float4(gc.x, gc.y, gc.z, al);
        rec[c] = r;
    }
}

// Exclusive scan of the per-row counts, kScanChunk rows per block of 1024
// threads: local prefixes into off, block totals into bsum.
__global__ void __launch_bounds__(1024) contact_scan_local_kernel(const int* __restrict__ cnt, int n,
                                                                  int* __restrict__ off, int* __restrict__ bsum) {
    __shared__ int s_w[32];
    const int base = blockIdx.x * kScanChunk + threadIdx.x * 4;
    int v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = (base + q < n) ? cnt[base + q] : 0;
    const int own = v[0] + v[1] + v[2] + v[3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = own;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int x = s_w[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        s_w[lane] = x;  // inclusive warp totals
    }
    __syncthreads();
    int run = inc - own + (warp > 0 ? s_w[warp - 1] : 0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (base + q < n) off[base + q] = run;
        run += v[q];
    }
    if (threadIdx.x == 1023) bsum[blockIdx.x] = run;
}

// Exclusive scan of the block totals in place (one block); bsum[nb] = total.
__global__ void __launch_bounds__(1024) contact_scan_top_kernel(int* __restrict__ bsum, int nb) {
    __shared__ int s_w[32];
    __shared__ int s_carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += 1024) {
        const int i = base + threadIdx.x;
        const int own = i < nb ? bsum[i] : 0;
        int inc = own;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            int x = s_w[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            s_w[lane] = x;
        }
        __syncthreads();
        const int carry = s_carry;
        const int ex = carry + inc - own + (warp > 0 ? s_w[warp - 1] : 0);
        if (i < nb) bsum[i] = ex;
        __syncthreads();
        if (threadIdx.x == 1023) s_carry = ex + own;
        __syncthreads();
    }
    if (threadIdx.x == 0) bsum[nb] = s_carry;
}

// off[i] += block prefix; off[n] = total; stats[2] = total slots.
__global__ void contact_scan_add_kernel(int* __restrict__ off, int n, const int* __restrict__ bsum, int nb,
                                        int* __restrict__ stats) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) off[i] += bsum[i / kScanChunk];
    if (i == 0) {
        off[n] = bsum[nb];
        stats[2] = bsum[nb];
    }
}

// Writes every live slot into its row's list; counting cnt back down
// leaves it zero for the next step.
__global__ void contact_fill_kernel(const PrepContact* __restrict__ rec, const int* __restrict__ stats,
                                    const int* __restrict__ off, int* __restrict__ cnt, int* __restrict__ ent) {
    const int nc = stats[0];
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const int4 rows = rec[c].rows;
        const int rr[4] = {rows.x, rows.y, rows.z, rows.w};
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int row = rr[s];
            if (row < 0) continue;
            const int k = atomicSub(&cnt[row], 1) - 1;
            ent[off[row] + k] = (c << 2) | s;
        }
    }
}

}  // namespace chysx_b200
