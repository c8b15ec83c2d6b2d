// Device kernels of the B200-native implicit cloth step.
//
// Data layout in HBM (all owned by the simulator unless noted):
//   caller's pos / vel / inv_mass / force : float3 AoS (12 B), borrowed
//   b, r, z, x(=dx), Ap, p0, p1           : float4 per row (16-B vector loads,
//                                           .w unused), rows padded to 32
//   diag, dnl, minv                       : symmetric 3x3 blocks as 6 planes
//                                           per 32-row slice (xx,xy,xz,yy,yz,zz):
//                                           full diagonal, its non-elastic part
//                                           (inertia, pins, contacts) and the
//                                           Jacobi inverse
//   col, val                              : sliced ELL (see topology.h); val
//                                           holds 6 planes per entry column
//                                           (9 with bending)
// Pin kI, spring H_blk, the Baraff-Witkin blocks c_a c_b M_u + d_a d_b M_v,
// inertia and contact blocks are symmetric, so a block is stored as 6
// floats (24 B) instead of the reference's 9 (36 B); the bending blocks
// k a_i a_j^T are not, and a system with bending keeps its off-diagonal
// blocks as 9 row-major planes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "contact_types.h"

namespace chysx_b200 {

constexpr int kWarp = 32;

// ---------------------------------------------------------------------------
// Views passed by value to kernels
// ---------------------------------------------------------------------------
struct DevTopo {
    int n;
    int n_slices;
    const int* __restrict__ slice_off;
    const int* __restrict__ col;
    float* val;
    float* diag;  // full diagonal blocks (Jacobi inverse, debug dump)
    float* dnl;   // non-elastic diagonal D': the operator is D'_i p_i + sum_j A_ij (p_j - p_i)
    float* minv;
    const int* __restrict__ tinc_off;
    const int* __restrict__ tinc;
    const unsigned* __restrict__ tinc_meta;
    const int* __restrict__ sinc_off;
    const int* __restrict__ sinc;
    const unsigned* __restrict__ sinc_meta;
    const int* __restrict__ pin_off;
    const int* __restrict__ pin_row;
    const float* __restrict__ pin_tgt;  // 3 floats per sorted pin
    const int* __restrict__ dinc_off;   // dihedral incidence (bending)
    const int* __restrict__ dinc;
    const unsigned* __restrict__ dinc_meta;
    // off-diagonal blocks: 6 planes (symmetric blocks), or 9 (row-major,
    // general blocks) once bending makes the off-diagonal blocks unsymmetric
    int nsym;
    ContactOp co;  // the contact operator's per-row lists (co.active = 0: none)
};

// Rest shape of a triangle, Dm^-1 row-major (Mat2f layout), kept in FP64:
// the grid's triangles are all nearly the same shape, so FP32 rounding of
// their rest data is correlated across the cloth and acts as a uniform
// pre-strain whose smooth response (2.7e-4 m after one step of the 256 x 256
// grid) would dominate the difference to the FP64 oracle.
struct RestShape {
    double m00, m01, m10, m11;
};

struct ElemData {
    const int* __restrict__ tris;         // 3 per triangle
    const RestShape* __restrict__ dminv;  // stretch
    const float* __restrict__ area;
    const float* __restrict__ ktri;
    const RestShape* __restrict__ dminv_s;  // shear: the same with the material axes turned by pi/4
    const float* __restrict__ area_s;
    const float* __restrict__ ktri_s;
    const int* __restrict__ edges;     // 2 per edge
    const double* __restrict__ rest;   // rest lengths (FP64, like the rest shapes)
    const float* __restrict__ kedge;
    const int4* __restrict__ dih;         // bending dihedrals (v0, v1, v2, v3)
    const double* __restrict__ rest_angle;
    float k_bend;
    int use_bending;
    float pin_k;
    int use_tris;     // triangles in the Hessian pattern (stretch or shear)
    int use_stretch;
    int use_shear;
    int use_springs;
    StaticContacts sc;
};

struct StepArgs {
    float* pos;      // x_n, v_n (read)
    float* vel;
    float* pos_out;  // x_{n+1}, v_{n+1} (written; == pos / vel for an in-place step)
    float* vel_out;
    const float* inv_mass;
    const float* force;
    const int* row_to_ext;  // internal row -> particle (-1 padding), null = identity
    int n;                  // internal rows
    int want_features;      // leave per-row feature inputs in ap / b.w
    float dt;
    float gx, gy, gz;
    float damping;
    int apply_force;
};

struct Vecs {
    float4* b;
    float4* r;
    float4* z;
    float4* x;
    float4* ap;
    float4* p0;
    float4* p1;
};

struct SolverCfg {
    int max_iter;
    int use_tol;
    double rel_tol;
    int pc_degree;   // CTA-local Chebyshev preconditioner: polynomial degree (odd); 0 = block-Jacobi
    float pc_ratio;  // its interval [lambda_max / ratio, lambda_max]
};

// Device-resident solver scalars.  Written only by the single "last block"
// of each grid reduction, read by every block of the next kernel.
struct SolveState {
    double rho, sigma, rr, bb, tol2, rr0;
    double alpha, beta;
    float alpha_f, beta_f;
    float scale, scale_b;  // warm guess factor c and 1 - c
    int iter, max_iter, done, status, use_tol, fallback;
    unsigned counter[4];
};

enum : int { kSolveConverged = 0, kSolveMaxIter = 1, kSolveNonfinite = 2 };

// ---------------------------------------------------------------------------
// Small math
// ---------------------------------------------------------------------------
struct S6 {
    float xx, xy, xz, yy, yz, zz;
};

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float3 ld3(const float* p, int i) {
    const float* q = p + 3 * (size_t)i;
    return f3(q[0], q[1], q[2]);
}
__device__ __forceinline__ void st3(float* p, int i, float3 v) {
    float* q = p + 3 * (size_t)i;
    q[0] = v.x; q[1] = v.y; q[2] = v.z;
}
__device__ __forceinline__ float3 xyz(float4 v) { return f3(v.x, v.y, v.z); }
__device__ __forceinline__ float4 f4(float3 v) { return make_float4(v.x, v.y, v.z, 0.f); }

__device__ __forceinline__ float3 mul(const S6& a, float3 v) {
    return f3(a.xx * v.x + a.xy * v.y + a.xz * v.z,
              a.xy * v.x + a.yy * v.y + a.yz * v.z,
              a.xz * v.x + a.yz * v.y + a.zz * v.z);
}
__device__ __forceinline__ void axpy6(S6& d, float s, const S6& a) {
    d.xx += s * a.xx; d.xy += s * a.xy; d.xz += s * a.xz;
    d.yy += s * a.yy; d.yz += s * a.yz; d.zz += s * a.zz;
}
// Adjugate inverse (no determinant guard), the symmetric specialisation of
// math::inverse(Mat3f) (src/math/matrix.cuh:219-235).
__device__ __forceinline__ S6 inverse6(const S6& m) {
    const float a00 = m.yy * m.zz - m.yz * m.yz;
    const float a01 = -m.xy * m.zz + m.xz * m.yz;
    const float a02 = m.xy * m.yz - m.xz * m.yy;
    const float a11 = m.xx * m.zz - m.xz * m.xz;
    const float a12 = -m.xx * m.yz + m.xz * m.xy;
    const float a22 = m.xx * m.yy - m.xy * m.xy;
    const float det = m.xx * a00 + m.xy * a01 + m.xz * a02;
    const float inv = 1.0f / det;
    return S6{a00 * inv, a01 * inv, a02 * inv, a11 * inv, a12 * inv, a22 * inv};
}
// 6 planes strided by 32 floats (one slice).
__device__ __forceinline__ S6 ld6(const float* p) {
    return S6{p[0], p[32], p[64], p[96], p[128], p[160]};
}
__device__ __forceinline__ void st6(float* p, const S6& a) {
    p[0] = a.xx; p[32] = a.xy; p[64] = a.xz; p[96] = a.yy; p[128] = a.yz; p[160] = a.zz;
}
// Floats per off-diagonal block of the topology.
__device__ __forceinline__ int off_width(const DevTopo& t) { return t.nsym ? 9 : 6; }
// y = B x for the off-diagonal block at p (planes strided by 32 floats):
// symmetric 6-plane blocks, or row-major 9-plane blocks when nsym.
__device__ __forceinline__ float3 mul_off(const float* p, int nsym, float3 v) {
    if (!nsym) return mul(ld6(p), v);
    return f3(p[0] * v.x + p[32] * v.y + p[64] * v.z,
              p[96] * v.x + p[128] * v.y + p[160] * v.z,
              p[192] * v.x + p[224] * v.y + p[256] * v.z);
}


// ---------------------------------------------------------------------------
// Single-pass deterministic grid reduction of NV doubles.  Each block writes
// its partial, the last block to arrive (atomic ticket, no waiting) sums the
// partials in block order and returns true with the totals in `out`.
// ---------------------------------------------------------------------------
template <int BLOCK, int NV>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], double* __restrict__ part,
                                            unsigned* counter, double (&out)[NV]) {
    constexpr int W = BLOCK / 32;
    __shared__ double sred[NV][W];
    __shared__ int s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sred[q][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < W; ++w) s += sred[q][w];
            part[(size_t)blockIdx.x * NV + q] = s;
        }
        __threadfence();
        // wraps to 0 after the last ticket, so the counter is ready for the
        // next launch without a reset (and self-heals if it was ever dirty)
        const unsigned prev = atomicInc(counter, gridDim.x - 1);
        s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += BLOCK) {
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] += __ldcg(part + (size_t)b * NV + q);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double x = acc[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sred[q][warp] = x;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) s += sred[q][w];
        out[q] = s;
    }
    return true;
}

__device__ __forceinline__ bool finite_d(double x) { return isfinite(x); }

// ---------------------------------------------------------------------------
// Element physics, evaluated in FP64 (same formulas as the reference kernels)
//
// The assembled system is stiff against its inertia: on the 256 x 256 grid a
// vertex's elastic diagonal is ~2.6e4 N/m and its m/dt^2 ~5.5e-3 N/m, a
// ratio of 2e-7, i.e. about three FP32 ulps.  FP32 element arithmetic (a few
// ulps per block) therefore loses the inertia of the smooth modes.  Every
// element quantity is formed in FP64 from the FP32 state and rounded once
// when the row is written; together with the difference form of the
// operator (assemble_kernel) and FP64 rest data (RestShape) this keeps the
// FP32 system within rounding of the FP64 one.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double3 d3(double x, double y, double z) { return make_double3(x, y, z); }
__device__ __forceinline__ double3 d3(float3 v) { return make_double3(v.x, v.y, v.z); }
__device__ __forceinline__ double3 operator+(double3 a, double3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ double3 operator-(double3 a, double3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 operator*(double3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double dot3(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double len3(double3 a) { return sqrt(dot3(a, a)); }
__device__ __forceinline__ double3 cross3(double3 a, double3 b) {
    return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double3 ld3d(const float* p, int i) { return d3(ld3(p, i)); }

struct S6d {
    double xx, xy, xz, yy, yz, zz;
};
__device__ __forceinline__ void axpy6(S6d& d, double s, const S6d& a) {
    d.xx += s * a.xx; d.xy += s * a.xy; d.xz += s * a.xz;
    d.yy += s * a.yy; d.yz += s * a.yz; d.zz += s * a.zz;
}
__device__ __forceinline__ void add6(S6d& d, const S6& a) {
    d.xx += a.xx; d.xy += a.xy; d.xz += a.xz; d.yy += a.yy; d.yz += a.yz; d.zz += a.zz;
}
__device__ __forceinline__ S6 round6(const S6d& a) {
    return S6{(float)a.xx, (float)a.xy, (float)a.xz, (float)a.yy, (float)a.yz, (float)a.zz};
}
// Adjugate inverse (no determinant guard), the symmetric specialisation of
// math::inverse(Mat3f) (src/math/matrix.cuh:219-235), in FP64.
__device__ __forceinline__ S6d inverse6(const S6d& m) {
    const double a00 = m.yy * m.zz - m.yz * m.yz;
    const double a01 = -m.xy * m.zz + m.xz * m.yz;
    const double a02 = m.xy * m.yz - m.xz * m.yy;
    const double a11 = m.xx * m.zz - m.xz * m.xz;
    const double a12 = -m.xx * m.yz + m.xz * m.xy;
    const double a22 = m.xx * m.yy - m.xy * m.xy;
    const double det = m.xx * a00 + m.xy * a01 + m.xz * a02;
    const double inv = 1.0 / det;
    return S6d{a00 * inv, a01 * inv, a02 * inv, a11 * inv, a12 * inv, a22 * inv};
}
__device__ __forceinline__ double sel3(const double (&a)[3], int i) {
    return i == 0 ? a[0] : (i == 1 ? a[1] : a[2]);
}
__device__ __forceinline__ double3 sel4(const double3 (&a)[4], int i) {
    return i == 0 ? a[0] : (i == 1 ? a[1] : (i == 2 ? a[2] : a[3]));
}

// Spring contribution to row `end` (0: row is edges[e].x, 1: row is .y).
// Gradient: spring_constraint.cu:76-103; block: spring_constraint.cu:110-151.
__device__ __forceinline__ void spring_row(const ElemData& el, const float* pos, int e, int end,
                                           double3& g, S6d& blk) {
    const int ia = el.edges[2 * e], ib = el.edges[2 * e + 1];
    const double3 d = ld3d(pos, ia) - ld3d(pos, ib);
    double l = len3(d);
    if (l < 1.0e-6) l = 1.0e-6;
    const double inv_l = 1.0 / l;
    const double3 dh = d * inv_l;
    const double k = el.kedge[e];
    const double L = el.rest[e];
    const double3 gv = dh * (k * (l - L));
    g = end == 0 ? g + gv : g - gv;
    const double a = k * L * inv_l;
    const double diag_term = (l < L) ? 0.0 : (k - a);
    blk = S6d{diag_term + a * dh.x * dh.x, a * dh.x * dh.y, a * dh.x * dh.z,
              diag_term + a * dh.y * dh.y, a * dh.y * dh.z, diag_term + a * dh.z * dh.z};
}

// Baraff-Witkin stretch of triangle t seen from its local vertex `la`:
// gradient triangle_stretch_constraint.cu:153-217, Hessian :231-311 written
// as H_ab = dwu_a dwu_b Mu + dwv_a dwv_b Mv with
//   Mu = k_eff (u u^T + [cu > 0] cu/lu (I - u u^T)), Mv likewise.
// Shear is the same element with the material axes turned by pi/4 in the
// rest shape (cloth_simulator.cu:423-449, triangle_stretch_constraint.cu:
// 87-109), i.e. a second (Dm^-1, area, k) set over the same triangles.
struct TriRow {
    double3 g;  // gradient at the row's vertex
    S6d Mu, Mv;
    double du[3], dv[3];
};

__device__ __forceinline__ void tri_row(const ElemData& el, const RestShape* __restrict__ dminv,
                                        const float* __restrict__ area, const float* __restrict__ ktri,
                                        const float* pos, int t, int la, TriRow& o) {
    const int v0 = el.tris[3 * t], v1 = el.tris[3 * t + 1], v2 = el.tris[3 * t + 2];
    const double3 x0 = ld3d(pos, v0), x1 = ld3d(pos, v1), x2 = ld3d(pos, v2);
    const double2 d01 = __ldg(reinterpret_cast<const double2*>(dminv + t));
    const double2 d23 = __ldg(reinterpret_cast<const double2*>(dminv + t) + 1);
    const double4 Dm = make_double4(d01.x, d01.y, d23.x, d23.y);  // (0,0) (0,1) (1,0) (1,1)
    const double3 a = x1 - x0, b = x2 - x0;
    const double3 wu = a * Dm.x + b * Dm.z;
    const double3 wv = a * Dm.y + b * Dm.w;
    double lu = len3(wu), lv = len3(wv);
    if (lu < 1.0e-6) lu = 1.0e-6;
    if (lv < 1.0e-6) lv = 1.0e-6;
    const double inv_lu = 1.0 / lu, inv_lv = 1.0 / lv;
    const double cu = lu - 1.0, cv = lv - 1.0;
    const double3 uh = wu * inv_lu, vh = wv * inv_lv;
    o.du[0] = -Dm.x - Dm.z; o.du[1] = Dm.x; o.du[2] = Dm.z;
    o.dv[0] = -Dm.y - Dm.w; o.dv[1] = Dm.y; o.dv[2] = Dm.w;
    const double k_eff = (double)area[t] * (double)ktri[t];
    const double dua = sel3(o.du, la), dva = sel3(o.dv, la);
    o.g = (uh * (cu * dua) + vh * (cv * dva)) * k_eff;
    const double su = cu > 0.0 ? k_eff * cu * inv_lu : 0.0;
    const double sv = cv > 0.0 ? k_eff * cv * inv_lv : 0.0;
    // k_eff u u^T + su (I - u u^T) = (k_eff - su) u u^T + su I
    const double cuu = k_eff - su, cvv = k_eff - sv;
    o.Mu = S6d{cuu * uh.x * uh.x + su, cuu * uh.x * uh.y, cuu * uh.x * uh.z,
               cuu * uh.y * uh.y + su, cuu * uh.y * uh.z, cuu * uh.z * uh.z + su};
    o.Mv = S6d{cvv * vh.x * vh.x + sv, cvv * vh.x * vh.y, cvv * vh.x * vh.z,
               cvv * vh.y * vh.y + sv, cvv * vh.y * vh.z, cvv * vh.z * vh.z + sv};
}

// c * a added to an FP64 off-diagonal accumulator of `ow` planes (6:
// symmetric storage; 9: row-major, the symmetric block mirrored).
__device__ __forceinline__ void smem_acc6(double* s, int stride, int slot, double c, const S6d& a, int ow = 6) {
    double* q = s + (size_t)slot * ow * stride;
    if (ow == 6) {
        q[0] += c * a.xx; q[stride] += c * a.xy; q[2 * stride] += c * a.xz;
        q[3 * stride] += c * a.yy; q[4 * stride] += c * a.yz; q[5 * stride] += c * a.zz;
    } else {
        q[0] += c * a.xx; q[stride] += c * a.xy; q[2 * stride] += c * a.xz;
        q[3 * stride] += c * a.xy; q[4 * stride] += c * a.yy; q[5 * stride] += c * a.yz;
        q[6 * stride] += c * a.xz; q[7 * stride] += c * a.yz; q[8 * stride] += c * a.zz;
    }
}
// c * u v^T added to a row-major 9-plane FP64 accumulator.
__device__ __forceinline__ void smem_acc_outer(double* s, int stride, int slot, double c, double3 u, double3 v) {
    double* q = s + (size_t)slot * 9 * stride;
    const double ux = c * u.x, uy = c * u.y, uz = c * u.z;
    q[0] += ux * v.x; q[stride] += ux * v.y; q[2 * stride] += ux * v.z;
    q[3 * stride] += uy * v.x; q[4 * stride] += uy * v.y; q[5 * stride] += uy * v.z;
    q[6 * stride] += uz * v.x; q[7 * stride] += uz * v.y; q[8 * stride] += uz * v.z;
}

// Discrete bending of a dihedral (v0, v1 = hinge; v2, v3 = the two wing
// vertices), Bridson's formulation as the reference uses it
// (constraint/cloth/bending_constraint.cu:46-123): signed angle
// theta = atan2((n1 x n2).e, n1.n2) between the wing normals and its shape
// gradients a_i = d theta / d x_i.  Energy k/2 (theta - theta0)^2,
// gradient k (theta - theta0) a_i, Gauss-Newton Hessian k a_i a_j^T.
// `valid` is false for a collapsed hinge or a wing without height.
struct Dihedral {
    double theta;
    double3 a[4];
    bool valid;
};

__device__ __forceinline__ Dihedral dihedral(double3 x0, double3 x1, double3 x2, double3 x3) {
    constexpr double kFloor = 1.0e-12;
    Dihedral d;
    d.valid = false;
    d.theta = 0.0;
    const double3 e = x1 - x0, e2 = x2 - x0, e3 = x3 - x0;
    const double le = len3(e);
    if (le < kFloor) return d;
    const double inv_le = 1.0 / le;
    const double3 m1 = cross3(e2, e), m2 = cross3(e, e3);
    const double l1 = len3(m1), l2 = len3(m2);
    if (l1 < kFloor || l2 < kFloor) return d;
    const double3 n1 = m1 * (1.0 / l1), n2 = m2 * (1.0 / l2);
    const double st = fmin(1.0, fmax(-1.0, dot3(cross3(n1, n2), e * inv_le)));
    d.theta = atan2(st, dot3(n1, n2));
    // foot points of the wing vertices on the hinge and their heights
    const double inv_le2 = inv_le * inv_le;
    const double w1 = dot3(e, e2) * inv_le2, w2 = dot3(e, e3) * inv_le2;
    const double h1 = len3(e2 - e * w1), h2 = len3(e3 - e * w2);
    if (h1 < kFloor || h2 < kFloor) return d;
    const double g1 = 1.0 / h1, g2 = 1.0 / h2;
    d.a[0] = n1 * ((w1 - 1.0) * g1) + n2 * ((w2 - 1.0) * g2);
    d.a[1] = n1 * (-w1 * g1) + n2 * (-w2 * g2);
    d.a[2] = n1 * g1;
    d.a[3] = n2 * g2;
    d.valid = true;
    return d;
}

}  // namespace chysx_b200

#include "contact_kernels.cuh"

namespace chysx_b200 {

// ---------------------------------------------------------------------------
// Fused per-row assembly: predictor (cloth_simulator.cu:83-106), mass
// (:66-77), gradient at x_n (pins/springs/stretch), RHS (:127-142), Hessian
// rows (pins, springs, stretch, inertia :199-210), block-Jacobi inverse
// (pcg_solver.cu:41-42) and, for the zero guess, the PCG start
// r = b, z = M^-1 b (pcg_solver.cu:386-404) with FP64 r.z and b.b.
// One thread owns one row and writes every block of it exactly once; all
// sums are FP64 (off-diagonal accumulators in shared memory) and each block
// is rounded to FP32 once.
//
// Difference form.  Springs, stretch, shear, bending and the contact
// operator's pairs depend on positions only through differences, so each
// element's Hessian blocks sum to zero along a block row and a row's
// elastic diagonal block is minus the sum of its off-diagonal blocks.  The
// row therefore also stores its non-elastic diagonal D' (inertia m/dt^2 I,
// pins, static contacts, the contact operator's slots) in t.dnl, and the
// solvers apply the operator as
//     (A p)_i = D'_i p_i + sum_j A_ij (p_j - p_i)     (+ contact pairs),
// which in FP32 keeps the inertia that the full diagonal (stored in t.diag
// for the Jacobi inverse and the debug dump) cannot resolve.
// ---------------------------------------------------------------------------
// COND = 1: the graph-loop build, which sets the WHILE node's condition for
// an already-converged zero-guess start; the persistent path launches the
// COND = 0 build, free of the device graph API.
template <int BLOCK, int COND>
__global__ void __launch_bounds__(BLOCK)
assemble_kernel(StepArgs a, ElemData el, DevTopo t, Vecs v, SolveState* st, double* part,
                SolverCfg cfg, int zero_guess, cudaGraphConditionalHandle cond) {
    extern __shared__ double s_off[];  // [width * ow][BLOCK]
    const int ow = off_width(t);
    const int tid = threadIdx.x;
    const int i = blockIdx.x * BLOCK + tid;
    double red[2] = {0.0, 0.0};
    const int e = (i < a.n) ? (a.row_to_ext ? a.row_to_ext[i] : i) : -1;
    if (i < a.n && e < 0) {
        // padding row of a batched layout: identity block, zero right-hand side
        const int s = i >> 5, lane = i & 31;
        const int so = t.slice_off[s];
        const int w = (t.slice_off[s + 1] - so) >> 5;
        const S6 I{1.f, 0.f, 0.f, 1.f, 0.f, 1.f};
        st6(t.diag + (size_t)s * 6 * 32 + lane, I);
        st6(t.dnl + (size_t)s * 6 * 32 + lane, I);
        st6(t.minv + (size_t)s * 6 * 32 + lane, I);
        float* vb = t.val + (size_t)so * ow + lane;
        for (int q = 0; q < ow * w; ++q) vb[q * 32] = 0.0f;
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        v.b[i] = z4;
        v.r[i] = z4;
        v.z[i] = z4;
        v.x[i] = z4;
    } else if (i < a.n) {
        const int s = i >> 5, lane = i & 31;
        const int so = t.slice_off[s];
        const int w = (t.slice_off[s + 1] - so) >> 5;
        for (int q = 0; q < ow * w; ++q) s_off[q * BLOCK + tid] = 0.0;

        const float3 xf = ld3(a.pos, e);
        const double3 x = d3(xf);
        const float3 velf = ld3(a.vel, e);
        const double3 vel = d3(velf);
        double m = 1.0;
        if (a.inv_mass) {
            const float wi = a.inv_mass[e];
            m = (wi > 1.0e-12f) ? (1.0 / (double)wi) : 1.0e8;
        }
        double3 acc = d3(a.gx, a.gy, a.gz);
        if (a.apply_force && a.force) {
            const double im = (m > 0.0) ? (1.0 / m) : 0.0;
            const double3 f = ld3d(a.force, e);
            acc = acc + f * im;
        }
        const double dt = a.dt;

        double3 g = d3(0.0, 0.0, 0.0);
        S6d Del{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // elastic diagonal (element blocks on the row)
        S6d Dnl{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // non-elastic diagonal D'
        float pinned = 0.f, logk = 0.f;
        int n_springs = 0;
        // pins (pin_constraint.cu:61-92)
        for (int p = t.pin_off[s]; p < t.pin_off[s + 1]; ++p) {
            if (t.pin_row[p] == i) {
                const double3 tg = ld3d(t.pin_tgt, p);
                g = g + (x - tg) * (double)el.pin_k;
                Dnl.xx += el.pin_k; Dnl.yy += el.pin_k; Dnl.zz += el.pin_k;
                pinned = 1.f;
            }
        }
        // springs
        if (el.use_springs) {
            const int o = t.sinc_off[s];
            const int ws = (t.sinc_off[s + 1] - o) >> 5;
            for (int k = 0; k < ws; ++k) {
                const int ed = t.sinc[o + k * 32 + lane];
                if (ed < 0) continue;
                const unsigned meta = t.sinc_meta[o + k * 32 + lane];
                S6d H;
                spring_row(el, a.pos, ed, (int)(meta & 1u), g, H);
                if (a.want_features) {
                    logk += log10f(fmaxf(el.kedge[ed], 1.0e-30f));
                    ++n_springs;
                }
                const unsigned slot = (meta >> 8) & 0xFFu;
                // a self-edge adds H - H to the diagonal
                if (slot != 0xFFu) {
                    axpy6(Del, 1.0, H);
                    smem_acc6(s_off + tid, BLOCK, (int)slot, -1.0, H, ow);
                }
            }
        }
        // Baraff-Witkin stretch, then shear, per incident triangle
        if (el.use_tris) {
            const int o = t.tinc_off[s];
            const int wt = (t.tinc_off[s + 1] - o) >> 5;
            for (int k = 0; k < wt; ++k) {
              const int tri = t.tinc[o + k * 32 + lane];
              if (tri < 0) continue;
              const unsigned meta = t.tinc_meta[o + k * 32 + lane];
              const int la = (int)(meta & 3u);
              for (int set = 0; set < 2; ++set) {
                if (set == 0 ? !el.use_stretch : !el.use_shear) continue;
                TriRow tr;
                if (set == 0) tri_row(el, el.dminv, el.area, el.ktri, a.pos, tri, la, tr);
                else tri_row(el, el.dminv_s, el.area_s, el.ktri_s, a.pos, tri, la, tr);
                g = g + tr.g;
                const double dua = sel3(tr.du, la), dva = sel3(tr.dv, la);
                axpy6(Del, dua * dua, tr.Mu);
                axpy6(Del, dva * dva, tr.Mv);
#pragma unroll
                for (int q = 1; q <= 2; ++q) {
                    const int lb = (la + q) % 3;
                    const unsigned slot = (meta >> (8 * q)) & 0xFFu;
                    const double cu_ = dua * sel3(tr.du, lb), cv_ = dva * sel3(tr.dv, lb);
                    if (slot == 0xFFu) {
                        axpy6(Del, cu_, tr.Mu);
                        axpy6(Del, cv_, tr.Mv);
                    } else {
                        smem_acc6(s_off + tid, BLOCK, (int)slot, cu_, tr.Mu, ow);
                        smem_acc6(s_off + tid, BLOCK, (int)slot, cv_, tr.Mv, ow);
                    }
                }
              }
            }
        }
        // bending dihedrals (bending_constraint.cu:163-244): gradient
        // k (theta - theta0) a_l, Hessian blocks k a_l a_m^T (general blocks)
        if (el.use_bending) {
            const int o = t.dinc_off[s];
            const int wd = (t.dinc_off[s + 1] - o) >> 5;
            for (int k = 0; k < wd; ++k) {
                const int d = t.dinc[o + k * 32 + lane];
                if (d < 0) continue;
                const unsigned meta = t.dinc_meta[o + k * 32 + lane];
                const int la = (int)(meta & 3u);
                const int4 q4 = el.dih[d];
                const Dihedral f = dihedral(ld3d(a.pos, q4.x), ld3d(a.pos, q4.y), ld3d(a.pos, q4.z),
                                            ld3d(a.pos, q4.w));
                if (!f.valid) continue;
                const double3 al = sel4(f.a, la);
                const double kb = el.k_bend;
                g = g + al * (kb * (f.theta - el.rest_angle[d]));
                Del.xx += kb * al.x * al.x; Del.xy += kb * al.x * al.y; Del.xz += kb * al.x * al.z;
                Del.yy += kb * al.y * al.y; Del.yz += kb * al.y * al.z; Del.zz += kb * al.z * al.z;
#pragma unroll
                for (int q = 1; q <= 3; ++q) {
                    const double3 am = sel4(f.a, (la + q) & 3);
                    const unsigned slot = (meta >> (8 * q)) & 0xFFu;
                    if (slot == 0xFFu) {
                        // a repeated vertex (degenerate dihedral): the block
                        // lands on the diagonal, kept symmetric
                        const double h = 0.5 * kb;
                        Del.xx += 2.0 * h * al.x * am.x; Del.yy += 2.0 * h * al.y * am.y;
                        Del.zz += 2.0 * h * al.z * am.z;
                        Del.xy += h * (al.x * am.y + al.y * am.x); Del.xz += h * (al.x * am.z + al.z * am.x);
                        Del.yz += h * (al.y * am.z + al.z * am.y);
                    } else {
                        smem_acc_outer(s_off + tid, BLOCK, (int)slot, kb, al, am);
                    }
                }
            }
        }
        // contact operator: gradient and diagonal blocks of the row's slots;
        // static shapes at x_n (cloth_simulator.cu:997-1008, 1189-1193)
        if (t.co.active) {
            float3 gc = f3(0.f, 0.f, 0.f);
            S6 Dc{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            contact_assemble_row(t.co, i, gc, Dc);
            g = g + d3(gc);
            add6(Dnl, Dc);
        }
        double3 sn = d3(0.0, 0.0, 0.0);
        double sdepth = 0.0;
        if (el.sc.active) sdepth = static_contact_row(el.sc, x, vel, dt, g, Dnl, sn);
        // RHS and inertia: m/dt^2 (x~ - x_n) = m (v / dt + acc)
        const double mi = m / (dt * dt);
        double3 b_d = (vel * (1.0 / dt) + acc) * m - g;
        // Coulomb cone on the assembled residual (cloth_simulator.cu:1073-1078)
        if (sdepth > 0.0 && el.sc.mu > 0.0f) b_d = coulomb_project(el.sc, b_d, sn, sdepth);
        const float3 b = f3((float)b_d.x, (float)b_d.y, (float)b_d.z);
        Dnl.xx += mi; Dnl.yy += mi; Dnl.zz += mi;
        S6d D = Dnl;
        axpy6(D, 1.0, Del);

        // write the row: diagonal, non-elastic diagonal, off-diagonal blocks, M^-1
        st6(t.diag + (size_t)s * 6 * 32 + lane, round6(D));
        st6(t.dnl + (size_t)s * 6 * 32 + lane, round6(Dnl));
        float* vb = t.val + (size_t)so * ow + lane;
        for (int q = 0; q < ow * w; ++q) vb[q * 32] = (float)s_off[q * BLOCK + tid];
        const S6 Mi = round6(inverse6(D));
        st6(t.minv + (size_t)s * 6 * 32 + lane, Mi);
        v.b[i] = make_float4(b.x, b.y, b.z, n_springs ? logk / (float)n_springs : 0.f);
        if (a.want_features) {
            const double im = 1.0 / m;
            v.ap[i] = make_float4((float)(-g.x * im), (float)(-g.y * im), (float)(-g.z * im), pinned);
        }
        red[1] = (double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z;
        if (zero_guess) {
            const float3 z = mul(Mi, b);
            v.r[i] = f4(b);
            v.z[i] = f4(z);
            v.x[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            red[0] = (double)b.x * z.x + (double)b.y * z.y + (double)b.z * z.z;
        }
    }
    double out[2];
    if (grid_reduce<BLOCK, 2>(red, part, &st->counter[0], out) && threadIdx.x == 0) {
        const double bb = out[1];
        st->bb = bb;
        st->use_tol = cfg.use_tol;
        st->max_iter = cfg.max_iter;
        st->tol2 = cfg.rel_tol * cfg.rel_tol * bb;
        st->iter = 0;
        st->beta = 0.0;
        st->beta_f = 0.0f;
        st->fallback = 0;
        if (zero_guess) {
            st->rho = out[0];
            st->rr = bb;
            st->rr0 = bb;
            const bool bad = !finite_d(out[0]) || !finite_d(bb);
            const bool conv = cfg.use_tol && bb <= st->tol2;
            st->status = bad ? kSolveNonfinite : kSolveConverged;
            st->done = (bad || conv || cfg.max_iter <= 0) ? 1 : 0;
            if (COND && cond) cudaGraphSetConditional(cond, st->done ? 0u : 1u);
        } else {
            st->status = finite_d(bb) ? kSolveConverged : kSolveNonfinite;
            st->done = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Warm-start initialisation (pcg_solver.cu:29-51 residual + :386-404):
// r = b - A x0 and the start partials.  With `scaled` the last block scales
// the guess by the energy-minimising factor c = x0.b / x0.A x0 (never worse
// than the zero guess in the A-norm), else keeps it (c = 1); when c <= 0 or
// a partial is not finite it flags the zero-guess fallback.
// `warm_fixup_kernel` applies either to every row.
// ---------------------------------------------------------------------------
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
warm_init_kernel(DevTopo t, Vecs v, SolveState* st, double* part, cudaGraphConditionalHandle cond, int scaled) {
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    // r.z, r.r, b.M^-1 b, x0.b, x0.r, b.z, b.r
    double red[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < t.n) {
        const int s = i >> 5, lane = i & 31;
        const int so = t.slice_off[s];
        const int w = (t.slice_off[s + 1] - so) >> 5;
        const S6 D = ld6(t.dnl + (size_t)s * 6 * 32 + lane);
        const float3 xi = xyz(v.x[i]);
        float3 ax = mul(D, xi);
        const int ow = off_width(t);
        const float* vb = t.val + (size_t)so * ow + lane;
        for (int k = 0; k < w; ++k) {
            const int j = t.col[so + k * 32 + lane];
            ax = ax + mul_off(vb + k * ow * 32, t.nsym, xyz(v.x[j]) - xi);
        }
        if (t.co.active && t.co.residual) ax = ax + contact_spmv_row(t.co, i, [&](int j) { return xyz(v.x[j]); });
        const float3 b = xyz(v.b[i]);
        const float3 r = b - ax;
        const S6 Mi = ld6(t.minv + (size_t)s * 6 * 32 + lane);
        const float3 z = mul(Mi, r);
        const float3 zb = mul(Mi, b);
        v.r[i] = f4(r);
        auto dot = [](float3 a, float3 c) { return (double)a.x * c.x + (double)a.y * c.y + (double)a.z * c.z; };
        red[0] = dot(r, z);
        red[1] = dot(r, r);
        red[2] = dot(b, zb);
        red[3] = dot(xi, b);
        red[4] = dot(xi, r);
        red[5] = dot(b, z);
        red[6] = dot(b, r);
    }
    double out[7];
    if (grid_reduce<BLOCK, 7>(red, part, &st->counter[1], out) && threadIdx.x == 0) {
        const double bb = st->bb;
        // energy-minimising scale of the guess (as the persistent kernels):
        // c = x0.b / x0.A x0, zero guess when c <= 0 or not finite
        // (scaled = 0 keeps the guess as given unless a partial is not finite)
        double c = finite_d(out[0]) && finite_d(out[1]) ? 1.0 : 0.0;
        if (scaled) {
            const double xax = out[3] - out[4];
            c = xax > 0.0 ? out[3] / xax : 0.0;
            if (!(c > 0.0) || !finite_d(c) || !finite_d(out[0]) || !finite_d(out[1])) c = 0.0;
        }
        st->fallback = c > 0.0 ? 0 : 1;
        st->scale = (float)c;
        st->scale_b = (float)(1.0 - c);
        if (c == 1.0) {
            st->rho = out[0];
            st->rr = out[1];
        } else if (c > 0.0) {
            const double cb = 1.0 - c;
            st->rho = fmax(cb * cb * out[2] + 2.0 * c * cb * out[5] + c * c * out[0], 0.0);
            st->rr = fmax(cb * cb * bb + 2.0 * c * cb * out[6] + c * c * out[1], 0.0);
        } else {
            st->rho = out[2];
            st->rr = bb;
        }
        st->rr0 = st->rr;
        const bool bad = !finite_d(st->rho) || !finite_d(st->rr);
        const bool conv = st->use_tol && st->rr <= st->tol2;
        if (bad) st->status = kSolveNonfinite;
        st->done = (bad || conv || st->max_iter <= 0 || st->status == kSolveNonfinite) ? 1 : 0;
        if (cond) cudaGraphSetConditional(cond, st->done ? 0u : 1u);
    }
}

__global__ void warm_fixup_kernel(DevTopo t, Vecs v, const SolveState* st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n) return;
    const int s = i >> 5, lane = i & 31;
    const S6 Mi = ld6(t.minv + (size_t)s * 6 * 32 + lane);
    const float3 b = xyz(v.b[i]);
    float3 x = f3(0.f, 0.f, 0.f), r = b;
    if (!st->fallback) {
        // x = c x0, r = (1 - c) b + c r0
        const float c = st->scale, cb = st->scale_b;
        const float3 x0 = xyz(v.x[i]), r0 = xyz(v.r[i]);
        x = f3(c * x0.x, c * x0.y, c * x0.z);
        r = f3(fmaf(c, r0.x, cb * b.x), fmaf(c, r0.y, cb * b.y), fmaf(c, r0.z, cb * b.z));
    }
    v.x[i] = f4(x);
    v.r[i] = f4(r);
    v.z[i] = f4(mul(Mi, r));
}

// ---------------------------------------------------------------------------
// PCG iteration, kernel 1: p = z + beta p (own row and, recomputed
// identically, every gathered neighbour: double-buffered p), Ap = A p
// (block_csr.cu:54-83), sigma = p.Ap in FP64; the last block forms
// alpha = rho / sigma (pcg_solver.cu:421-423, 456-464).
// ---------------------------------------------------------------------------
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
pcg_spmv_kernel(DevTopo t, Vecs v, SolveState* st, double* part, cudaGraphConditionalHandle cond) {
    if (st->done) return;
    const int it = st->iter;
    const float beta = st->beta_f;
    const bool first = (it == 0);
    const float4* __restrict__ pold = (it & 1) ? v.p1 : v.p0;
    float4* __restrict__ pnew = (it & 1) ? v.p0 : v.p1;
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    double red[1] = {0.0};
    if (i < t.n) {
        const int s = i >> 5, lane = i & 31;
        const int so = t.slice_off[s];
        const int w = (t.slice_off[s + 1] - so) >> 5;
        const float4 zi = v.z[i];
        float3 pi = xyz(zi);
        if (!first) {
            const float4 po = pold[i];
            pi = f3(fmaf(beta, po.x, zi.x), fmaf(beta, po.y, zi.y), fmaf(beta, po.z, zi.z));
        }
        pnew[i] = f4(pi);
        const S6 D = ld6(t.dnl + (size_t)s * 6 * 32 + lane);
        float3 acc = mul(D, pi);
        const int ow = off_width(t);
        const float* vb = t.val + (size_t)so * ow + lane;
        const int* cb = t.col + so + lane;
        for (int k = 0; k < w; ++k) {
            const int j = cb[k * 32];
            const float4 zj = v.z[j];
            float3 pj = xyz(zj);
            if (!first) {
                const float4 po = pold[j];
                pj = f3(fmaf(beta, po.x, zj.x), fmaf(beta, po.y, zj.y), fmaf(beta, po.z, zj.z));
            }
            acc = acc + mul_off(vb + k * ow * 32, t.nsym, pj - pi);
        }
        if (t.co.active)
            acc = acc + contact_spmv_row(t.co, i, [&](int j) {
                      const float4 zj = v.z[j];
                      if (first) return xyz(zj);
                      const float4 po = pold[j];
                      return f3(fmaf(beta, po.x, zj.x), fmaf(beta, po.y, zj.y), fmaf(beta, po.z, zj.z));
                  });
        v.ap[i] = f4(acc);
        red[0] = (double)pi.x * acc.x + (double)pi.y * acc.y + (double)pi.z * acc.z;
    }
    double out[1];
    if (grid_reduce<BLOCK, 1>(red, part, &st->counter[2], out) && threadIdx.x == 0) {
        const double sigma = out[0];
        st->sigma = sigma;
        const double alpha = (sigma > 1.0e-37 || sigma < -1.0e-37) ? st->rho / sigma : 0.0;
        st->alpha = alpha;
        st->alpha_f = (float)alpha;
        if (!finite_d(sigma) || !finite_d(alpha)) {
            st->status = kSolveNonfinite;
            st->done = 1;
            if (cond) cudaGraphSetConditional(cond, 0u);
        }
    }
}

// ---------------------------------------------------------------------------
// PCG iteration, kernel 2: x += alpha p, r -= alpha Ap, z = M^-1 r, FP64
// r.z and r.r (pcg_solver.cu:406-434); the last block forms beta
// (:436-454), counts the iteration, tests ||r||^2 <= tol^2 ||b||^2 and sets
// the graph's loop condition.
// ---------------------------------------------------------------------------
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
pcg_update_kernel(DevTopo t, Vecs v, SolveState* st, double* part, cudaGraphConditionalHandle cond) {
    if (st->done) {
        if (cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0u);
        return;
    }
    const int it = st->iter;
    const float alpha = st->alpha_f;
    const float4* __restrict__ p = (it & 1) ? v.p0 : v.p1;
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    double red[2] = {0.0, 0.0};
    if (i < t.n) {
        const int s = i >> 5, lane = i & 31;
        const float4 pi = p[i], api = v.ap[i], xi = v.x[i], ri = v.r[i];
        const float3 xn = f3(fmaf(alpha, pi.x, xi.x), fmaf(alpha, pi.y, xi.y), fmaf(alpha, pi.z, xi.z));
        const float3 rn = f3(fmaf(-alpha, api.x, ri.x), fmaf(-alpha, api.y, ri.y), fmaf(-alpha, api.z, ri.z));
        const S6 Mi = ld6(t.minv + (size_t)s * 6 * 32 + lane);
        const float3 zn = mul(Mi, rn);
        v.x[i] = f4(xn);
        v.r[i] = f4(rn);
        v.z[i] = f4(zn);
        red[0] = (double)rn.x * zn.x + (double)rn.y * zn.y + (double)rn.z * zn.z;
        red[1] = (double)rn.x * rn.x + (double)rn.y * rn.y + (double)rn.z * rn.z;
    }
    double out[2];
    if (grid_reduce<BLOCK, 2>(red, part, &st->counter[3], out) && threadIdx.x == 0) {
        const double rho_new = out[0], rr = out[1];
        const double rho = st->rho;
        const double beta = (rho > 1.0e-37 || rho < -1.0e-37) ? rho_new / rho : 0.0;
        st->beta = beta;
        st->beta_f = (float)beta;
        st->rho = rho_new;
        st->rr = rr;
        const int iter = it + 1;
        st->iter = iter;
        const bool bad = !finite_d(rho_new) || !finite_d(rr);
        const bool conv = st->use_tol && rr <= st->tol2;
        int done = 0;
        if (bad) {
            st->status = kSolveNonfinite;
            done = 1;
        } else if (conv) {
            st->status = kSolveConverged;
            done = 1;
        } else if (iter >= st->max_iter) {
            st->status = st->use_tol ? kSolveMaxIter : kSolveConverged;
            done = 1;
        }
        st->done = done;
        if (cond) cudaGraphSetConditional(cond, done ? 0u : 1u);
    }
}

// A step whose solve failed leaves the caller's state as it was: in place
// nothing is written, into separate output buffers x_n and v_n are copied.
__device__ __forceinline__ void keep_state(const StepArgs& a, int e) {
    if (a.pos_out == a.pos && a.vel_out == a.vel) return;
    st3(a.pos_out, e, ld3(a.pos, e));
    st3(a.vel_out, e, ld3(a.vel, e));
}

// ---------------------------------------------------------------------------
// x_{n+1} = x_n + dx, v_{n+1} = dx/dt * exp(-c dt)  (cloth_simulator.cu:222-244)
// The caller's buffers are left untouched when the solve met NaN/Inf.
// ---------------------------------------------------------------------------
__global__ void finalize_kernel(StepArgs a, Vecs v, const SolveState* st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int e = a.row_to_ext ? a.row_to_ext[i] : i;
    if (e < 0) return;
    if (st->status == kSolveNonfinite) {
        keep_state(a, e);
        return;
    }
    const float4 d = v.x[i];
    const float3 xn = ld3(a.pos, e);
    st3(a.pos_out, e, f3(xn.x + d.x, xn.y + d.y, xn.z + d.z));
    const float inv_dt = 1.0f / a.dt;
    float3 vn = f3(d.x * inv_dt, d.y * inv_dt, d.z * inv_dt);
    if (a.damping > 0.0f) {
        const float decay = expf(-a.damping * a.dt);
        vn = vn * decay;
    }
    st3(a.vel_out, e, vn);
}

// ---------------------------------------------------------------------------
// True residual of the returned iterate (the reference's optional
// compute_true_residual pass, src/solver/pcg_solver.cu:595-641): r = b -
// (A + C) x recomputed from the stored FP32 system (difference form) and the
// final x, with the
// products accumulated in FP64, so that the recurrence residual the solver
// stopped on can be checked against what the iterate actually satisfies.
// One warp per 32-row slice; out[slice] = (sum r.r, sum b.b) of its rows,
// summed by a fixed shuffle tree (deterministic).
// ---------------------------------------------------------------------------
__global__ void true_residual_kernel(DevTopo t, Vecs v, double2* __restrict__ out) {
    const int s = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= t.n_slices) return;
    const int i = s * 32 + lane;
    double rr = 0.0, bb = 0.0;
    if (i < t.n) {
        const int so = t.slice_off[s];
        const int w = (t.slice_off[s + 1] - so) >> 5;
        const float* d = t.dnl + (size_t)s * 6 * 32 + lane;
        const float3 xi = xyz(v.x[i]);
        // D' x_i in FP64: symmetric planes xx, xy, xz, yy, yz, zz
        const double dxx = d[0], dxy = d[32], dxz = d[64], dyy = d[96], dyz = d[128], dzz = d[160];
        double ax = dxx * xi.x + dxy * xi.y + dxz * xi.z;
        double ay = dxy * xi.x + dyy * xi.y + dyz * xi.z;
        double az = dxz * xi.x + dyz * xi.y + dzz * xi.z;
        const int ow = off_width(t);
        const float* vb = t.val + (size_t)so * ow + lane;
        for (int k = 0; k < w; ++k) {
            const int j = t.col[so + k * 32 + lane];
            const float3 xjf = xyz(v.x[j]);
            const double3 xj = make_double3((double)xjf.x - xi.x, (double)xjf.y - xi.y, (double)xjf.z - xi.z);
            const float* q = vb + (size_t)k * ow * 32;
            if (t.nsym) {
                ax += (double)q[0] * xj.x + (double)q[32] * xj.y + (double)q[64] * xj.z;
                ay += (double)q[96] * xj.x + (double)q[128] * xj.y + (double)q[160] * xj.z;
                az += (double)q[192] * xj.x + (double)q[224] * xj.y + (double)q[256] * xj.z;
            } else {
                const double qxx = q[0], qxy = q[32], qxz = q[64], qyy = q[96], qyz = q[128], qzz = q[160];
                ax += qxx * xj.x + qxy * xj.y + qxz * xj.z;
                ay += qxy * xj.x + qyy * xj.y + qyz * xj.z;
                az += qxz * xj.x + qyz * xj.y + qzz * xj.z;
            }
        }
        if (t.co.active) {
            const float3 c = contact_spmv_row(t.co, i, [&](int j) { return xyz(v.x[j]); });
            ax += c.x;
            ay += c.y;
            az += c.z;
        }
        const float3 b = xyz(v.b[i]);
        const double rx = b.x - ax, ry = b.y - ay, rz = b.z - az;
        rr = rx * rx + ry * ry + rz * rz;
        bb = (double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z;
    }
    for (int o = 16; o > 0; o >>= 1) {
        rr += __shfl_down_sync(0xffffffffu, rr, o);
        bb += __shfl_down_sync(0xffffffffu, bb, o);
    }
    if (lane == 0) out[s] = make_double2(rr, bb);
}

// ---------------------------------------------------------------------------
// Setup kernels
// ---------------------------------------------------------------------------

// triangle_stretch_constraint.cu:50-110
__global__ void rest_shape_kernel(const int* __restrict__ tris, const float* __restrict__ pos,
                                  RestShape* __restrict__ dminv, float* __restrict__ area, int T,
                                  float det_eps, float cos_t, float sin_t) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const double3 a = ld3d(pos, tris[3 * t]), b = ld3d(pos, tris[3 * t + 1]), c = ld3d(pos, tris[3 * t + 2]);
    const double3 ab = b - a, ac = c - a;
    const double lab = len3(ab), lac = len3(ac);
    const double3 abh = (lab > 1.0e-6) ? ab * (1.0 / lab) : d3(1.0, 0.0, 0.0);
    const double u_c = dot3(abh, ac);
    const double v_c2 = lac * lac - u_c * u_c;
    const double v_c = (v_c2 > 0.0) ? sqrt(v_c2) : 0.0;
    area[t] = (float)(0.5 * lab * v_c);
    const double det = lab * v_c;
    double i00 = 1.0, i01 = 0.0, i10 = 0.0, i11 = 1.0;
    if (det > (double)det_eps) {
        const double inv_det = 1.0 / det;
        i00 = v_c * inv_det;
        i01 = -u_c * inv_det;
        i11 = lab * inv_det;
    }
    const double ct = cos_t, st = sin_t;
    dminv[t] = RestShape{i00 * ct - i01 * st, i00 * st + i01 * ct, i10 * ct - i11 * st, i10 * st + i11 * ct};
}

// Rest angle of every bending dihedral (bending_constraint.cu:126-142);
// degenerate dihedrals rest at 0.
__global__ void bending_rest_kernel(const int4* __restrict__ dih, const float* __restrict__ pos,
                                    double* __restrict__ rest, int D) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= D) return;
    const int4 q = dih[d];
    const Dihedral f = dihedral(ld3d(pos, q.x), ld3d(pos, q.y), ld3d(pos, q.z), ld3d(pos, q.w));
    rest[d] = f.valid ? f.theta : 0.0;
}

// spring_constraint.cu:41-52
__global__ void rest_length_kernel(const int* __restrict__ edges, const float* __restrict__ pos,
                                   double* __restrict__ rest, int E) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    rest[e] = len3(ld3d(pos, edges[2 * e]) - ld3d(pos, edges[2 * e + 1]));
}

// Lumped area-weighted mass, cloth_simulator.cu:151-190, gathered per vertex
// over its incident triangles (in triangle order) instead of atomics.
__global__ void lumped_inv_mass_kernel(const int* __restrict__ vt_off, const int* __restrict__ vt_list,
                                       const int* __restrict__ tris, const float* __restrict__ pos,
                                       float density_over_3, float* __restrict__ inv_mass, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float m = 0.0f;
    for (int q = vt_off[i]; q < vt_off[i + 1]; ++q) {
        const int t = vt_list[q];
        const float3 x0 = ld3(pos, tris[3 * t]), x1 = ld3(pos, tris[3 * t + 1]), x2 = ld3(pos, tris[3 * t + 2]);
        const float3 e1 = x1 - x0, e2 = x2 - x0;
        const float3 cr = f3(e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x);
        m += density_over_3 * (0.5f * len3(cr));
    }
    inv_mass[i] = (m > 1.0e-12f) ? (1.0f / m) : 0.0f;
}

}  // namespace chysx_b200
