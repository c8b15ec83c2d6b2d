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
__device__ __forceinline__ double f1_over_x(double u, double eps) {
    return u > eps ? 1.0 / u : (-u / eps + 2.0) / eps;
}

// Static contacts are evaluated in FP64 like the elastic elements: the depth
// is a small difference of positions of order one, and its FP32 round-off
// times the contact stiffness is a spurious force.
//
// Deepest static-shape penetration of x: depth > 0 and the outward normal,
// or depth 0 (static_contact.cu:41-146: planes first, then boxes, a strictly
// deeper primitive wins).
__device__ __forceinline__ double static_deepest(const StaticContacts& sc, double3 x, double3& bn) {
    double best = 0.0;
    bn = make_double3(0.0, 0.0, 0.0);
    const float* s = sc.shapes;
    auto v3 = [](const float* p) { return make_double3(p[0], p[1], p[2]); };
    for (int q = 0; q < sc.n_planes; ++q, s += 4) {
        const double3 nv = v3(s);
        const double depth = (double)sc.thickness - (dot3(nv, x) + (double)s[3]);
        if (depth > best) { best = depth; bn = nv; }
    }
    for (int q = 0; q < sc.n_boxes; ++q, s += 15) {
        const double3 rel = x - v3(s);
        const double3 ex = v3(s + 6), ey = v3(s + 9), ez = v3(s + 12);
        const double qx = dot3(rel, ex), qy = dot3(rel, ey), qz = dot3(rel, ez);
        const double dx = fabs(qx) - s[3], dy = fabs(qy) - s[4], dz = fabs(qz) - s[5];
        double d;
        double3 nv;
        if (dx <= 0.0 && dy <= 0.0 && dz <= 0.0) {
            // inside: the nearest face
            if (dx >= dy && dx >= dz) { nv = qx >= 0.0 ? ex : ex * -1.0; d = dx; }
            else if (dy >= dz) { nv = qy >= 0.0 ? ey : ey * -1.0; d = dy; }
            else { nv = qz >= 0.0 ? ez : ez * -1.0; d = dz; }
        } else {
            const double cx = dx > 0.0 ? dx : 0.0, cy = dy > 0.0 ? dy : 0.0, cz = dz > 0.0 ? dz : 0.0;
            d = sqrt(cx * cx + cy * cy + cz * cz);
            const double inv = 1.0 / fmax(d, 1.0e-300);
            const double sx = qx > 0.0 ? cx : -cx, sy = qy > 0.0 ? cy : -cy, sz = qz > 0.0 ? cz : -cz;
            nv = ex * (sx * inv) + ey * (sy * inv) + ez * (sz * inv);
        }
        const double depth = (double)sc.thickness - d;
        if (depth > best) { best = depth; bn = nv; }
    }
    return best;
}

// Static contact of one row at x_n with velocity vel: adds the penalty and
// lagged-friction gradient to g and the block k n n^T + alpha (I - n n^T) to
// D (static_contact.cu:186-285).  Returns the depth (0: no contact).
__device__ __forceinline__ double static_contact_row(const StaticContacts& sc, double3 x, double3 vel, double dt,
                                                     double3& g, S6d& D, double3& bn) {
    const double depth = static_deepest(sc, x, bn);
    if (!(depth > 0.0)) return 0.0;
    const double k = sc.k;
    g = g + bn * (-k * depth);
    double al = 0.0;
    if (sc.mu > 0.0f) {
        const double3 dxv = vel * dt;
        const double vn = dot3(bn, dxv);
        const double3 ut = dxv - bn * vn;
        const double un = len3(ut);
        al = (double)sc.mu * (k * depth) * f1_over_x(un, (double)sc.eps);
        g = g - ut * al;
    }
    D.xx += k * bn.x * bn.x + al * (1.0 - bn.x * bn.x);
    D.xy += k * bn.x * bn.y + al * (-bn.x * bn.y);
    D.xz += k * bn.x * bn.z + al * (-bn.x * bn.z);
    D.yy += k * bn.y * bn.y + al * (1.0 - bn.y * bn.y);
    D.yz += k * bn.y * bn.z + al * (-bn.y * bn.z);
    D.zz += k * bn.z * bn.z + al * (1.0 - bn.z * bn.z);
    return depth;
}

// Coulomb-cone projection of the assembled residual b of a row in static
// contact (static_contact.cu:306-381): F0 = b - k depth n; only F0's push
// into the surface loads the cone.
__device__ __forceinline__ double3 coulomb_project(const StaticContacts& sc, double3 b, double3 bn, double depth) {
    const double push = (double)sc.k * depth;
    const double3 F0 = b - bn * push;
    const double f0n = dot3(F0, bn);
    const double fn = fmax(0.0, -f0n);
    if (fn <= 0.0) return b;
    const double3 F0t = F0 - bn * f0n;
    const double ft2 = dot3(F0t, F0t);
    if (ft2 <= 0.0) return b;
    const double ft = sqrt(ft2);
    const double cone = (double)sc.mu * fn;
    if (ft <= cone) return b - F0t;
    return b - F0t * (cone / ft);
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
