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
//     signed dihedral angle atan2((n1 x n2).e, n1.n2) of the two unit face
//     normals, Gauss-Newton Hessian k dtheta dtheta^T, damping on dtheta/dt.
// Every function below is written from those formulas.
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
__device__ __forceinline__ V3 mul_t(const M3& a, V3 v) {  // a^T v
    return v3(a.m[0] * v.x + a.m[3] * v.y + a.m[6] * v.z, a.m[1] * v.x + a.m[4] * v.y + a.m[7] * v.z,
              a.m[2] * v.x + a.m[5] * v.y + a.m[8] * v.z);
}
// [a]_x: the matrix of u -> a x u
__device__ __forceinline__ M3 skew(V3 a) {
    M3 r;
    r.m[0] = 0.f; r.m[1] = -a.z; r.m[2] = a.y;
    r.m[3] = a.z; r.m[4] = 0.f; r.m[5] = -a.x;
    r.m[6] = -a.y; r.m[7] = a.x; r.m[8] = 0.f;
    return r;
}
__device__ __forceinline__ M3 mul(const M3& a, const M3& b) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            r.m[3 * i + j] = a.m[3 * i] * b.m[j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
    return r;
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

// Membrane force and Hessian block of vertex `which` (0, 1, 2) of one
// triangle, added to f and h.  Dm^-1 row-major {d00, d01, d10, d11}.
__device__ void membrane(int which, V3 x0, V3 x1, V3 x2, V3 p0, V3 p1, V3 p2, const float* dmi, float area,
                         float mu, float lambda, float damping, float dt, V3& f, M3& h) {
    const float d00 = dmi[0], d01 = dmi[1], d10 = dmi[2], d11 = dmi[3];
    const V3 e1 = x1 - x0, e2 = x2 - x0;
    // columns of F
    const V3 c0 = e1 * d00 + e2 * d10;
    const V3 c1 = e1 * d01 + e2 * d11;
    const float a00 = dot(c0, c0), a11 = dot(c1, c1), a01 = dot(c0, c1);
    // J = area ratio = sqrt(det F^T F)
    const float jj = fmaxf(a00 * a11 - a01 * a01, 1.0e-20f);
    const float J = sqrtf(jj);
    const float inv_j = 1.0f / J;
    const float lam = lambda + mu;
    const float lam_guard = copysignf(fmaxf(fabsf(lam), 1.0e-6f), lam);
    const float alpha = 1.0f + mu / lam_guard;
    // dJ/dF columns
    const V3 g0 = (c0 * a11 - c1 * a01) * inv_j;
    const V3 g1 = (c1 * a00 - c0 * a01) * inv_j;
    const float s = lam * (J - alpha);
    const V3 P0 = c0 * mu + g0 * s;
    const V3 P1 = c1 * mu + g1 * s;
    // d(F columns)/dx_which = scalar weights of the vertex
    const float w1 = which == 1 ? 1.0f : 0.0f, w2 = which == 2 ? 1.0f : 0.0f, w0 = which == 0 ? 1.0f : 0.0f;
    const float q0 = d00 * (w1 - w0) + d10 * (w2 - w0);
    const float q1 = d01 * (w1 - w0) + d11 * (w2 - w0);
    V3 force = (P0 * q0 + P1 * q1) * (-area);
    const float r = fmaxf(0.0f, s) * inv_j;
    const V3 dj = g0 * q0 + g1 * q1;
    const V3 w = c1 * q0 - c0 * q1;
    M3 hm = zero3();
    add_scaled_identity(hm, mu * (q0 * q0 + q1 * q1) + r * (q0 * q0 * a11 + q1 * q1 * a00 - 2.0f * q0 * q1 * a01));
    add_outer(hm, dj, dj, lam - r);
    add_outer(hm, w, w, -r);
    if (damping > 0.0f) {
        // Green strain G = (F^T F - I) / 2
        const float G00 = 0.5f * (a00 - 1.0f), G11 = 0.5f * (a11 - 1.0f), G01 = 0.5f * a01;
        const float gn2 = G00 * G00 + G11 * G11 + 2.0f * G01 * G01;
        if (gn2 >= 1.0e-20f) {
            const float inv_dt = 1.0f / dt;
            const V3 v1 = (e1 - (p1 - p0)) * inv_dt, v2 = (e2 - (p2 - p0)) * inv_dt;
            const V3 dc0 = v1 * d00 + v2 * d10, dc1 = v1 * d01 + v2 * d11;
            const float gn = sqrtf(gn2);
            const float n00 = G00 / gn, n01 = G01 / gn, n11 = G11 / gn;
            const float r00 = dot(c0, dc0), r11 = dot(c1, dc1), r01 = 0.5f * (dot(c0, dc1) + dot(c1, dc0));
            // deviatoric part: C_mu = |G|
            const float cmu_t = n00 * r00 + n11 * r11 + 2.0f * n01 * r01;
            const V3 cmu_x = (c0 * n00 + c1 * n01) * q0 + (c0 * n01 + c1 * n11) * q1;
            const float kmu = mu * damping;
            force = force - cmu_x * (kmu * cmu_t * area);
            add_outer(hm, cmu_x, cmu_x, kmu * inv_dt);
            // volumetric part: C_lambda = tr G
            const float clam_t = r00 + r11;
            const V3 clam_x = c0 * q0 + c1 * q1;
            const float klam = lambda * damping;
            force = force - clam_x * (klam * clam_t * area);
            add_outer(hm, clam_x, clam_x, klam * inv_dt);
        }
    }
    f = f + force;
#pragma unroll
    for (int k = 0; k < 9; ++k) h.m[k] += hm.m[k] * area;
}

// Hinge bending force and Hessian block of vertex `which` (0..3) of one
// edge (x0, x1 the opposite vertices, x2 -> x3 the hinge).
__device__ void bending(int which, const V3 (&x)[4], const V3 (&p)[4], float rest_angle, float rest_length,
                        float stiffness, float damping, float dt, V3& f, M3& h) {
    const float eps = 1.0e-6f;
    const V3 x02 = x[2] - x[0], x03 = x[3] - x[0], x13 = x[3] - x[1], x12 = x[2] - x[1];
    const V3 e = x[3] - x[2];
    const V3 n1 = cross(x02, x03), n2 = cross(x13, x12);
    const float l1 = norm(n1), l2 = norm(n2), le = norm(e);
    if (l1 < eps || l2 < eps || le < eps) return;
    const V3 u1 = n1 * (1.0f / l1), u2 = n2 * (1.0f / l2), ue = e * (1.0f / le);
    const float sn = dot(cross(u1, u2), ue), cs = dot(u1, u2);
    const float theta = atan2f(sn, cs);
    const float k = stiffness * rest_length;
    const float dedt = k * (theta - rest_angle);
    // d(unit normal)/dx = (I - u u^T) / |n| dn/dx
    auto unit_d = [](float len, V3 u, const M3& raw) {
        M3 pr = zero3();
        add_scaled_identity(pr, 1.0f);
        add_outer(pr, u, u, -1.0f);
        M3 r = mul(pr, raw);
#pragma unroll
        for (int q = 0; q < 9; ++q) r.m[q] *= 1.0f / len;
        return r;
    };
    const M3 su1 = skew(u1), su2 = skew(u2);
    // dtheta/dx_i = cos d(sin) - sin d(cos)
    auto dtheta = [&](const M3& du1, const M3& du2) {
        const M3 a = mul(su1, du2), b = mul(su2, du1);
        M3 ds;
#pragma unroll
        for (int q = 0; q < 9; ++q) ds.m[q] = a.m[q] - b.m[q];
        const V3 dsin = mul_t(ds, ue);
        const V3 dcos = mul_t(du1, u2) + mul_t(du2, u1);
        return dsin * cs - dcos * sn;
    };
    const M3 z = zero3();
    const M3 se = skew(e);
    M3 se_n;
#pragma unroll
    for (int q = 0; q < 9; ++q) se_n.m[q] = -se.m[q];
    // dn1/dx: x0 -> [e]_x, x2 -> -[x03]_x, x3 -> [x02]_x; dn2/dx: x1 -> -[e]_x,
    // x2 -> [x13]_x, x3 -> -[x12]_x
    V3 dth[4];
    {
        dth[0] = dtheta(unit_d(l1, u1, se), z);
        dth[1] = dtheta(z, unit_d(l2, u2, se_n));
        M3 a = skew(x03), b = skew(x12);
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            a.m[q] = -a.m[q];
            b.m[q] = -b.m[q];
        }
        dth[2] = dtheta(unit_d(l1, u1, a), unit_d(l2, u2, skew(x13)));
        dth[3] = dtheta(unit_d(l1, u1, skew(x02)), unit_d(l2, u2, b));
    }
    const V3 dv = which == 0 ? dth[0] : (which == 1 ? dth[1] : (which == 2 ? dth[2] : dth[3]));
    V3 force = dv * (-dedt);
    M3 hb = zero3();
    add_outer(hb, dv, dv, k);
    if (damping > 0.0f) {
        const float inv_dt = 1.0f / dt;
        float rate = 0.0f;
#pragma unroll
        for (int i = 0; i < 4; ++i) rate += dot(dth[i], x[i] - p[i]);
        rate *= inv_dt;
        const float dk = damping * k;
        force = force - dv * (dk * rate);
        add_outer(hb, dv, dv, dk * inv_dt);
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
