// Vertex Block Descent for triangle cloth (Chen, Macklin, Yu et al., "Vertex
// Block Descent", SIGGRAPH 2024): an implicit-Euler step solved by colour
// sweeps of per-vertex 3x3 Newton updates, vertices of one colour in
// parallel.  Energies (the reference's choice, solver/cloth_vbd_kernels.cuh,
// solver/vbd_solver.cu:64-92,284-293,304-407):
//   * membrane: the 2D Stable Neo-Hookean energy of Smith, de Goes and Kim
//     (2018) on F = [x1 - x0, x2 - x0] Dm^-1 (3x2), with mu, lambda' = lambda
//     + mu, alpha = 1 + mu / lambda', the projected Hessian
//     I (mu |dF/dx|^2 + r (...)) + (lambda' - r) dJ dJ^T - r w w^T,
//     r = max(0, lambda' (J - alpha)) / J, and Rayleigh-style damping of the
//     Green strain's deviatoric (mu) and volumetric (lambda) parts;
//   * bending: the discrete-shell hinge energy of Grinspun et al. (2003),
//     k/2 (theta - theta0)^2 with k = stiffness x rest length, theta the
//     signed dihedral angle of the two face normals, Gauss-Newton Hessian
//     k dtheta dtheta^T with the closed-form angle gradient of Bridson et
//     al. (2003), damping on dtheta/dt.
#pragma once

#include <cuda_runtime.h>

namespace chysx_b200 {
namespace vbd {

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float norm(V3 a) { return sqrtf(dot(a, a)); }

// Row-major 3x3.
struct M3 {
    float m[9];
};
__device__ __forceinline__ M3 zero3() {
    M3 r;
#pragma unroll
    for (int k = 0; k < 9; ++k) r.m[k] = 0.0f;
    return r;
}
__device__ __forceinline__ void add_scaled_identity(M3& h, float s) {
    h.m[0] += s;
    h.m[4] += s;
    h.m[8] += s;
}
__device__ __forceinline__ void add_outer(M3& h, V3 a, V3 b, float s) {
    const float av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) h.m[3 * r + c] += s * av[r] * bv[c];
}
__device__ __forceinline__ V3 mul(const M3& a, V3 v) {
    return v3(a.m[0] * v.x + a.m[1] * v.y + a.m[2] * v.z, a.m[3] * v.x + a.m[4] * v.y + a.m[5] * v.z,
              a.m[6] * v.x + a.m[7] * v.y + a.m[8] * v.z);
}
__device__ __forceinline__ float det3(const M3& a) {
    return a.m[0] * (a.m[4] * a.m[8] - a.m[5] * a.m[7]) - a.m[1] * (a.m[3] * a.m[8] - a.m[5] * a.m[6]) +
           a.m[2] * (a.m[3] * a.m[7] - a.m[4] * a.m[6]);
}
// inverse by the adjugate over the determinant
__device__ __forceinline__ M3 inv3(const M3& a, float d) {
    const float s = 1.0f / d;
    M3 r;
    r.m[0] = (a.m[4] * a.m[8] - a.m[5] * a.m[7]) * s;
    r.m[1] = (a.m[2] * a.m[7] - a.m[1] * a.m[8]) * s;
    r.m[2] = (a.m[1] * a.m[5] - a.m[2] * a.m[4]) * s;
    r.m[3] = (a.m[5] * a.m[6] - a.m[3] * a.m[8]) * s;
    r.m[4] = (a.m[0] * a.m[8] - a.m[2] * a.m[6]) * s;
    r.m[5] = (a.m[2] * a.m[3] - a.m[0] * a.m[5]) * s;
    r.m[6] = (a.m[3] * a.m[7] - a.m[4] * a.m[6]) * s;
    r.m[7] = (a.m[1] * a.m[6] - a.m[0] * a.m[7]) * s;
    r.m[8] = (a.m[0] * a.m[4] - a.m[1] * a.m[3]) * s;
    return r;
}

__device__ __forceinline__ V3 ld(const float* p, int i) { return v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ void st(float* p, int i, V3 v) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}

// Adds s * (first-order damping of a strain measure c): with c's gradient
// gc at the vertex and its rate cdot, the force -kd cdot gc and the
// Hessian kd / dt gc gc^T, both times the element area (the reference's
// Rayleigh-style damping of the membrane's two strain measures and of the
// hinge angle).
__device__ __forceinline__ void add_damping(float kd, V3 gc, float cdot, float inv_dt, float area, V3& force,
                                            M3& hm) {
    force = force - gc * (kd * cdot * area);
    add_outer(hm, gc, gc, kd * inv_dt * area);
}

// Membrane force and Hessian block of vertex `which` (0, 1, 2) of one
// triangle, added to f and h.  Dm^-1 row-major {d00, d01, d10, d11}.
//
// Energy density: 2D Stable Neo-Hookean (Smith, de Goes & Kim 2018) of the
// 3x2 deformation gradient F = [f0 f1] = [x1 - x0, x2 - x0] Dm^-1,
//     psi = mu/2 (|f0|^2 + |f1|^2 - 2) + lam/2 (J - alpha)^2,
// with lam = lambda + mu, alpha = 1 + mu / lam and J = |f0 x f1| the area
// ratio.  Seen from one vertex, whose displacement dx moves the columns by
// df_k = q_k dx, the area normal nrm = f0 x f1 moves by dx x w with
// w = q0 f1 - q1 f0, which does not depend on dx.  Hence
//     dJ/dx = w x nhat,   d2J/dx2 = (|w|^2 I - w w^T - dJ dJ^T) / J,
// the latter positive semi-definite, and the vertex Hessian
//     mu |q|^2 I + lam dJ dJ^T + max(0, lam (J - alpha)) d2J/dx2
// keeps only the non-negative part of the volumetric coefficient (the
// reference's projection), so it is PSD by construction.
// Damping acts on the Green strain G = (F^T F - I) / 2 through its norm |G|
// (weight mu * damping) and its trace (weight lambda * damping), with rates
// from the step's displacement (x - p) / dt.
__device__ void membrane(int which, V3 x0, V3 x1, V3 x2, V3 p0, V3 p1, V3 p2, const float* dmi, float area,
                         float mu, float lambda, float damping, float dt, V3& f, M3& h) {
    const float d00 = dmi[0], d01 = dmi[1], d10 = dmi[2], d11 = dmi[3];
    const V3 e1 = x1 - x0, e2 = x2 - x0;
    const V3 f0 = e1 * d00 + e2 * d10, f1 = e1 * d01 + e2 * d11;
    // column weights of this vertex: f_k = sum_v x_v q_k(v)
    float q0, q1;
    if (which == 0) {
        q0 = -(d00 + d10);
        q1 = -(d01 + d11);
    } else if (which == 1) {
        q0 = d00;
        q1 = d01;
    } else {
        q0 = d10;
        q1 = d11;
    }
    const V3 nrm = cross(f0, f1);
    const float J = fmaxf(norm(nrm), 1.0e-10f);
    const V3 nhat = nrm * (1.0f / J);
    const V3 w = f1 * q0 - f0 * q1;
    const V3 dJ = cross(w, nhat);
    const float lam = lambda + mu;
    const float alpha = lam != 0.0f ? 1.0f + mu / lam : 1.0f;
    const float vol = lam * (J - alpha);  // d psi / dJ
    // gradient of psi at the vertex: mu (q0 f0 + q1 f1) + vol dJ
    V3 force = ((f0 * q0 + f1 * q1) * mu + dJ * vol) * (-area);
    const float r = fmaxf(vol, 0.0f) / J;
    const float ww = dot(w, w);
    M3 hm = zero3();
    add_scaled_identity(hm, (mu * (q0 * q0 + q1 * q1) + r * ww) * area);
    add_outer(hm, dJ, dJ, (lam - r) * area);
    add_outer(hm, w, w, -r * area);
    if (damping > 0.0f) {
        const float c00 = dot(f0, f0), c11 = dot(f1, f1), c01 = dot(f0, f1);
        const float g00 = 0.5f * (c00 - 1.0f), g11 = 0.5f * (c11 - 1.0f), g01 = 0.5f * c01;
        const float gnorm2 = g00 * g00 + g11 * g11 + 2.0f * g01 * g01;
        if (gnorm2 >= 1.0e-20f) {
            const float inv_dt = 1.0f / dt;
            // column rates from the element's displacement over the step
            const V3 u1 = (e1 - (p1 - p0)) * inv_dt, u2 = (e2 - (p2 - p0)) * inv_dt;
            const V3 f0d = u1 * d00 + u2 * d10, f1d = u1 * d01 + u2 * d11;
            // Gdot = (F^T Fdot + Fdot^T F) / 2
            const float gd00 = dot(f0, f0d), gd11 = dot(f1, f1d), gd01 = 0.5f * (dot(f0, f1d) + dot(f1, f0d));
            // |G|: gradient sum_kl (G_kl / |G|) f_k q_l, rate (G : Gdot) / |G|
            const float ig = 1.0f / sqrtf(gnorm2);
            const V3 gdev = (f0 * g00 + f1 * g01) * (q0 * ig) + (f0 * g01 + f1 * g11) * (q1 * ig);
            const float rdev = (g00 * gd00 + g11 * gd11 + 2.0f * g01 * gd01) * ig;
            add_damping(mu * damping, gdev, rdev, inv_dt, area, force, hm);
            // tr G: gradient q0 f0 + q1 f1, rate tr Gdot
            add_damping(lambda * damping, f0 * q0 + f1 * q1, gd00 + gd11, inv_dt, area, force, hm);
        }
    }
    f = f + force;
#pragma unroll
    for (int k = 0; k < 9; ++k) h.m[k] += hm.m[k];
}

// Hinge bending force and Hessian block of vertex `which` (0..3) of one
// edge: x0, x1 the wing vertices opposite the hinge x2 -> x3.
//
// Energy k/2 (theta - theta0)^2, k = stiffness * rest length (discrete
// shells, Grinspun et al. 2003), theta the signed angle between the face
// normals n1 = (x2 - x0) x (x3 - x0) and n2 = (x3 - x1) x (x2 - x1) about
// the hinge direction.  Its gradient in closed form (Bridson, Marino &
// Fedkiw 2003; Tamstorf & Grinspun 2013): with a = n1 / |n1|^2,
// b = n2 / |n2|^2, e = x3 - x2 and t = e / |e|,
//     dtheta/dx0 = -|e| a,                dtheta/dx1 = -|e| b,
//     dtheta/dx2 = -((x0 - x3).t) a - ((x1 - x3).t) b,
//     dtheta/dx3 =  ((x0 - x2).t) a + ((x1 - x2).t) b
// (they sum to zero).  Gauss-Newton Hessian k g g^T; damping on the angle's
// rate sum_i g_i . (x_i - p_i) / dt with weight damping * k.  A hinge with
// a collapsed face or edge contributes nothing.
__device__ void bending(int which, const V3 (&x)[4], const V3 (&p)[4], float rest_angle, float rest_length,
                        float stiffness, float damping, float dt, V3& f, M3& h) {
    constexpr float kMin = 1.0e-6f;
    const V3 e = x[3] - x[2];
    const V3 n1 = cross(x[2] - x[0], x[3] - x[0]);
    const V3 n2 = cross(x[3] - x[1], x[2] - x[1]);
    const float l1sq = dot(n1, n1), l2sq = dot(n2, n2), le = norm(e);
    if (sqrtf(l1sq) < kMin || sqrtf(l2sq) < kMin || le < kMin) return;
    const V3 t = e * (1.0f / le);
    const V3 a = n1 * (1.0f / l1sq), b = n2 * (1.0f / l2sq);
    // signed angle: sin from the normals' cross product along the hinge
    const float l12 = sqrtf(l1sq * l2sq);
    const float theta = atan2f(dot(cross(n1, n2), t) / l12, dot(n1, n2) / l12);
    V3 g[4];
    g[0] = a * (-le);
    g[1] = b * (-le);
    g[2] = a * (-dot(x[0] - x[3], t)) - b * dot(x[1] - x[3], t);
    g[3] = a * dot(x[0] - x[2], t) + b * dot(x[1] - x[2], t);
    const V3 gv = which == 0 ? g[0] : (which == 1 ? g[1] : (which == 2 ? g[2] : g[3]));
    const float k = stiffness * rest_length;
    V3 force = gv * (-k * (theta - rest_angle));
    M3 hb = zero3();
    add_outer(hb, gv, gv, k);
    if (damping > 0.0f) {
        const float inv_dt = 1.0f / dt;
        float rate = 0.0f;
#pragma unroll
        for (int i = 0; i < 4; ++i) rate += dot(g[i], x[i] - p[i]);
        add_damping(damping * k, gv, rate * inv_dt, inv_dt, 1.0f, force, hb);
    }
    f = f + force;
#pragma unroll
    for (int q = 0; q < 9; ++q) h.m[q] += hb.m[q];
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

struct ClothArgs {
    float* pos;
    float* vel;
    const float* inv_mass;
    float* q_prev;   // x at the start of the step
    float* inertia;  // x + dt (v + dt g)
    float* disp;     // x - q_prev accumulated by the sweeps
    float* mass;
    const int* tris;       // 3 per triangle
    const float* poses;    // Dm^-1, 4 per triangle
    const float* areas;
    const float* mats;     // mu, lambda, damping per triangle
    const int* tri_off;    // per vertex: (triangle, local vertex) pairs
    const int* tri_adj;
    const int* edges;      // 4 per edge: o0, o1, v2, v3
    const float* rest_angle;
    const float* rest_length;
    const float* bend;     // stiffness, damping per edge
    const int* edge_off;
    const int* edge_adj;
    int n;
    float gx, gy, gz;
    float dt;
};

// predictor: q_prev = x, m = 1/w, inertia = x + dt v', x = x + dt v' with
// v' = v + dt g; a particle with w == 0 stays (vbd_solver.cu:64-92)
__global__ void vbd_forward_kernel(ClothArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const V3 x = ld(a.pos, i);
    st(a.q_prev, i, x);
    const float w = a.inv_mass[i];
    a.mass[i] = (w > 1.0e-12f) ? (1.0f / w) : 0.0f;
    if (w == 0.0f) {
        st(a.inertia, i, x);
        st(a.disp, i, v3(0.f, 0.f, 0.f));
        return;
    }
    const V3 vn = ld(a.vel, i) + v3(a.gx, a.gy, a.gz) * a.dt;
    const V3 y = x + vn * a.dt;
    st(a.inertia, i, y);
    st(a.disp, i, vn * a.dt);
    st(a.pos, i, y);
}

// One colour's vertices (vbd_solver.cu:304-407), LANES lanes per vertex:
// the vertex's incident triangles and hinges are dealt round-robin over the
// lanes, each lane sums its share of forces and Hessian blocks, a shuffle
// tree adds the lanes' sums and the group's first lane takes the 3x3 Newton
// step.  The reference walks the elements one thread per vertex; the work
// per vertex (a few hundred flops per triangle, over a thousand per hinge)
// then sets the sweep's latency.  Small colours take 8 lanes a vertex, a
// colour that fills the GPU one (the host picks).
template <int LANES>
__global__ void __launch_bounds__(256) vbd_color_kernel(ClothArgs a, const int* __restrict__ ids, int count) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = gt / LANES, lane = gt % LANES;
    const bool live = t < count;
    const int i = live ? ids[t] : 0;
    const float m = live ? a.mass[i] : 0.0f;
    const float dt = a.dt;
    V3 f = v3(0.f, 0.f, 0.f);
    M3 h = zero3();
    if (live && m != 0.0f) {
        const int t0 = a.tris ? a.tri_off[i] : 0, t1 = a.tris ? a.tri_off[i + 1] : 0;
        const int e0 = a.edges ? a.edge_off[i] : 0, e1 = a.edges ? a.edge_off[i + 1] : 0;
        const int nt = (t1 - t0) >> 1, ne = (e1 - e0) >> 1;
        for (int k = lane; k < nt + ne; k += LANES) {
            if (k < nt) {
                const int q = t0 + 2 * k;
                const int tri = a.tri_adj[q], which = a.tri_adj[q + 1];
                const float mu = a.mats[3 * tri], lambda = a.mats[3 * tri + 1], damp = a.mats[3 * tri + 2];
                if (mu <= 0.0f && lambda <= 0.0f) continue;
                const int v0 = a.tris[3 * tri], v1 = a.tris[3 * tri + 1], v2 = a.tris[3 * tri + 2];
                membrane(which, ld(a.pos, v0), ld(a.pos, v1), ld(a.pos, v2), ld(a.q_prev, v0), ld(a.q_prev, v1),
                         ld(a.q_prev, v2), a.poses + 4 * tri, a.areas[tri], mu, lambda, damp, dt, f, h);
            } else {
                const int q = e0 + 2 * (k - nt);
                const int e = a.edge_adj[q], which = a.edge_adj[q + 1];
                const float ks = a.bend[2 * e], damp = a.bend[2 * e + 1];
                if (ks <= 0.0f) continue;
                const int* ev = a.edges + 4 * e;
                if (ev[0] < 0 || ev[1] < 0) continue;  // boundary edge
                const V3 x[4] = {ld(a.pos, ev[0]), ld(a.pos, ev[1]), ld(a.pos, ev[2]), ld(a.pos, ev[3])};
                const V3 p[4] = {ld(a.q_prev, ev[0]), ld(a.q_prev, ev[1]), ld(a.q_prev, ev[2]),
                                 ld(a.q_prev, ev[3])};
                bending(which, x, p, a.rest_angle[e], a.rest_length[e], ks, damp, dt, f, h);
            }
        }
    }
    // lane sums, fixed order
    float acc[12] = {f.x, f.y, f.z};
#pragma unroll
    for (int q = 0; q < 9; ++q) acc[3 + q] = h.m[q];
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < 12; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o, LANES);
    if (!live || lane != 0) return;
    if (m == 0.0f) {
        st(a.disp, i, v3(0.f, 0.f, 0.f));
        return;
    }
    const float md = m * (1.0f / (dt * dt));
    // inertia term, then the elements' sums
    f = (ld(a.inertia, i) - ld(a.pos, i)) * md + v3(acc[0], acc[1], acc[2]);
#pragma unroll
    for (int q = 0; q < 9; ++q) h.m[q] = acc[3 + q];
    add_scaled_identity(h, md);
    const float d = det3(h);
    V3 disp = ld(a.disp, i);
    if (fabsf(d) > 1.0e-8f) {
        disp = disp + mul(inv3(h, d), f);
        st(a.disp, i, disp);
    }
    st(a.pos, i, ld(a.q_prev, i) + disp);
}

// v = (x - q_prev) / dt (vbd_solver.cu:284-293)
__global__ void vbd_velocity_kernel(ClothArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    st(a.vel, i, (ld(a.pos, i) - ld(a.q_prev, i)) * (1.0f / a.dt));
}

}  // namespace vbd
}  // namespace chysx_b200
