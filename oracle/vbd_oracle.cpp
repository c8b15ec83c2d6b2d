// ============================================================================
// TEST INFRASTRUCTURE ONLY — CPU oracle of the cloth Vertex Block Descent step.
//
// The checker, never the product: only tests/ may load it.  It restates the
// reference's ClothVBDSolver::step_cloth (caixiao-0725/Ai-Phyiscs,
// src/solver/vbd_solver.cu:64-92 predictor, 304-407 colour sweep, 284-293
// velocity, 897-979 driver; element formulas src/solver/cloth_vbd_kernels.cuh)
// in plain C++ templated on the scalar (double: oracle, float: FP32 port),
// from the published methods: Vertex Block Descent (Chen et al. 2024), the 2D
// Stable Neo-Hookean membrane (Smith, de Goes, Kim 2018) and discrete-shell
// hinge bending (Grinspun et al. 2003).  Parity is pinned against fixtures
// of the compiled reference run on a B200 (tests/golden/), the element
// forces against finite differences of the energies (tests/).
// ============================================================================
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <vector>

namespace {

template <class R>
struct V {
    R x, y, z;
};
template <class R> V<R> operator+(V<R> a, V<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> V<R> operator-(V<R> a, V<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> V<R> operator*(V<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> R dot(V<R> a, V<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> V<R> cross(V<R> a, V<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> R len(V<R> a) { return std::sqrt(dot(a, a)); }
template <class R> V<R> get(const R* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
template <class R> void put(R* p, int i, V<R> v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }

template <class R>
struct M {
    R m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
};
template <class R> void outer_add(M<R>& h, V<R> a, V<R> b, R s) {
    const R av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) h.m[3 * r + c] += s * av[r] * bv[c];
}
template <class R> V<R> mv(const M<R>& a, V<R> v) {
    return {a.m[0] * v.x + a.m[1] * v.y + a.m[2] * v.z, a.m[3] * v.x + a.m[4] * v.y + a.m[5] * v.z,
            a.m[6] * v.x + a.m[7] * v.y + a.m[8] * v.z};
}
template <class R> V<R> mtv(const M<R>& a, V<R> v) {
    return {a.m[0] * v.x + a.m[3] * v.y + a.m[6] * v.z, a.m[1] * v.x + a.m[4] * v.y + a.m[7] * v.z,
            a.m[2] * v.x + a.m[5] * v.y + a.m[8] * v.z};
}
template <class R> M<R> mm(const M<R>& a, const M<R>& b) {
    M<R> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[3 * i + j] = a.m[3 * i] * b.m[j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
    return r;
}
template <class R> M<R> skew(V<R> a) {
    M<R> r;
    r.m[1] = -a.z; r.m[2] = a.y; r.m[3] = a.z; r.m[5] = -a.x; r.m[6] = -a.y; r.m[7] = a.x;
    return r;
}
template <class R> M<R> scaled(M<R> a, R s) {
    for (R& v : a.m) v *= s;
    return a;
}

// 2D Stable Neo-Hookean membrane: force on vertex `which` and its Hessian
// block (cloth_vbd_kernels.cuh:21-128).
template <class R>
void membrane(int which, const V<R> (&x)[3], const V<R> (&p)[3], const R* dmi, R area, R mu, R lambda, R damping,
              R dt, V<R>& f, M<R>& h) {
    const R d00 = dmi[0], d01 = dmi[1], d10 = dmi[2], d11 = dmi[3];
    const V<R> e1 = x[1] - x[0], e2 = x[2] - x[0];
    const V<R> c0 = e1 * d00 + e2 * d10, c1 = e1 * d01 + e2 * d11;
    const R a00 = dot(c0, c0), a11 = dot(c1, c1), a01 = dot(c0, c1);
    const R J = std::sqrt(std::max(a00 * a11 - a01 * a01, R(1e-20)));
    const R ij = R(1) / J;
    const R lam = lambda + mu;
    const R guard = std::copysign(std::max(std::fabs(lam), R(1e-6)), lam);
    const R alpha = R(1) + mu / guard;
    const V<R> g0 = (c0 * a11 - c1 * a01) * ij, g1 = (c1 * a00 - c0 * a01) * ij;
    const R s = lam * (J - alpha);
    const V<R> P0 = c0 * mu + g0 * s, P1 = c1 * mu + g1 * s;
    const R w0 = which == 0, w1 = which == 1, w2 = which == 2;
    const R q0 = d00 * (w1 - w0) + d10 * (w2 - w0), q1 = d01 * (w1 - w0) + d11 * (w2 - w0);
    V<R> force = (P0 * q0 + P1 * q1) * (-area);
    const R r = std::max(R(0), s) * ij;
    const V<R> dj = g0 * q0 + g1 * q1, w = c1 * q0 - c0 * q1;
    M<R> hm;
    const R di = mu * (q0 * q0 + q1 * q1) + r * (q0 * q0 * a11 + q1 * q1 * a00 - R(2) * q0 * q1 * a01);
    hm.m[0] += di; hm.m[4] += di; hm.m[8] += di;
    outer_add(hm, dj, dj, lam - r);
    outer_add(hm, w, w, -r);
    if (damping > R(0)) {
        const R G00 = R(0.5) * (a00 - R(1)), G11 = R(0.5) * (a11 - R(1)), G01 = R(0.5) * a01;
        const R gn2 = G00 * G00 + G11 * G11 + R(2) * G01 * G01;
        if (gn2 >= R(1e-20)) {
            const R idt = R(1) / dt;
            const V<R> v1 = (e1 - (p[1] - p[0])) * idt, v2 = (e2 - (p[2] - p[0])) * idt;
            const V<R> dc0 = v1 * d00 + v2 * d10, dc1 = v1 * d01 + v2 * d11;
            const R gn = std::sqrt(gn2);
            const R n00 = G00 / gn, n01 = G01 / gn, n11 = G11 / gn;
            const R r00 = dot(c0, dc0), r11 = dot(c1, dc1), r01 = R(0.5) * (dot(c0, dc1) + dot(c1, dc0));
            const R cmu_t = n00 * r00 + n11 * r11 + R(2) * n01 * r01;
            const V<R> cmu_x = (c0 * n00 + c1 * n01) * q0 + (c0 * n01 + c1 * n11) * q1;
            force = force - cmu_x * (mu * damping * cmu_t * area);
            outer_add(hm, cmu_x, cmu_x, mu * damping * idt);
            const V<R> cl_x = c0 * q0 + c1 * q1;
            force = force - cl_x * (lambda * damping * (r00 + r11) * area);
            outer_add(hm, cl_x, cl_x, lambda * damping * idt);
        }
    }
    f = f + force;
    for (int k = 0; k < 9; ++k) h.m[k] += hm.m[k] * area;
}

// Membrane energy area (mu/2 (|F|^2 - 2) + lambda'/2 (J - alpha)^2), the
// potential of the force above.
template <class R>
R membrane_energy(const V<R> (&x)[3], const R* dmi, R area, R mu, R lambda) {
    const V<R> e1 = x[1] - x[0], e2 = x[2] - x[0];
    const V<R> c0 = e1 * dmi[0] + e2 * dmi[2], c1 = e1 * dmi[1] + e2 * dmi[3];
    const R a00 = dot(c0, c0), a11 = dot(c1, c1), a01 = dot(c0, c1);
    const R J = std::sqrt(std::max(a00 * a11 - a01 * a01, R(1e-20)));
    const R lam = lambda + mu;
    const R alpha = R(1) + mu / std::copysign(std::max(std::fabs(lam), R(1e-6)), lam);
    return area * (R(0.5) * mu * (a00 + a11 - R(2)) + R(0.5) * lam * (J - alpha) * (J - alpha));
}

// Signed hinge angle of (x0, x1 opposite; x2 -> x3 hinge) and the unit normals.
template <class R>
bool hinge(const V<R> (&x)[4], R& theta, V<R>& u1, V<R>& u2, V<R>& ue, R& l1, R& l2) {
    const V<R> n1 = cross(x[2] - x[0], x[3] - x[0]), n2 = cross(x[3] - x[1], x[2] - x[1]);
    const V<R> e = x[3] - x[2];
    l1 = len(n1);
    l2 = len(n2);
    const R le = len(e);
    const R eps = R(1e-6);
    if (l1 < eps || l2 < eps || le < eps) return false;
    u1 = n1 * (R(1) / l1);
    u2 = n2 * (R(1) / l2);
    ue = e * (R(1) / le);
    theta = std::atan2(dot(cross(u1, u2), ue), dot(u1, u2));
    return true;
}

// Hinge bending force on vertex `which` and its Gauss-Newton block
// (cloth_vbd_kernels.cuh:133-231).
template <class R>
void bending(int which, const V<R> (&x)[4], const V<R> (&p)[4], R rest_angle, R rest_length, R stiffness,
             R damping, R dt, V<R>& f, M<R>& h) {
    R theta, l1, l2;
    V<R> u1, u2, ue;
    if (!hinge(x, theta, u1, u2, ue, l1, l2)) return;
    const R sn = dot(cross(u1, u2), ue), cs = dot(u1, u2);
    const R k = stiffness * rest_length;
    const R dedt = k * (theta - rest_angle);
    auto unit_d = [](R l, V<R> u, const M<R>& raw) {
        M<R> pr;
        pr.m[0] = pr.m[4] = pr.m[8] = R(1);
        outer_add(pr, u, u, R(-1));
        return scaled(mm(pr, raw), R(1) / l);
    };
    const M<R> su1 = skew(u1), su2 = skew(u2);
    auto dtheta = [&](const M<R>& d1, const M<R>& d2) {
        const M<R> a = mm(su1, d2), b = mm(su2, d1);
        M<R> ds;
        for (int q = 0; q < 9; ++q) ds.m[q] = a.m[q] - b.m[q];
        const V<R> dsn = mtv(ds, ue), dcs = mtv(d1, u2) + mtv(d2, u1);
        return dsn * cs - dcs * sn;
    };
    const V<R> e = x[3] - x[2];
    const M<R> z;
    V<R> d[4];
    d[0] = dtheta(unit_d(l1, u1, skew(e)), z);
    d[1] = dtheta(z, unit_d(l2, u2, scaled(skew(e), R(-1))));
    d[2] = dtheta(unit_d(l1, u1, scaled(skew(x[3] - x[0]), R(-1))), unit_d(l2, u2, skew(x[3] - x[1])));
    d[3] = dtheta(unit_d(l1, u1, skew(x[2] - x[0])), unit_d(l2, u2, scaled(skew(x[2] - x[1]), R(-1))));
    const V<R> dv = d[which];
    V<R> force = dv * (-dedt);
    M<R> hb;
    outer_add(hb, dv, dv, k);
    if (damping > R(0)) {
        const R idt = R(1) / dt;
        R rate = 0;
        for (int i = 0; i < 4; ++i) rate += dot(d[i], x[i] - p[i]);
        rate *= idt;
        force = force - dv * (damping * k * rate);
        outer_add(hb, dv, dv, damping * k * idt);
    }
    f = f + force;
    for (int q = 0; q < 9; ++q) h.m[q] += hb.m[q];
}

template <class R>
R det(const M<R>& a) {
    return a.m[0] * (a.m[4] * a.m[8] - a.m[5] * a.m[7]) - a.m[1] * (a.m[3] * a.m[8] - a.m[5] * a.m[6]) +
           a.m[2] * (a.m[3] * a.m[7] - a.m[4] * a.m[6]);
}
template <class R>
V<R> solve(const M<R>& a, R d, V<R> f) {  // adjugate / det
    const R s = R(1) / d;
    M<R> r;
    r.m[0] = (a.m[4] * a.m[8] - a.m[5] * a.m[7]) * s;
    r.m[1] = (a.m[2] * a.m[7] - a.m[1] * a.m[8]) * s;
    r.m[2] = (a.m[1] * a.m[5] - a.m[2] * a.m[4]) * s;
    r.m[3] = (a.m[5] * a.m[6] - a.m[3] * a.m[8]) * s;
    r.m[4] = (a.m[0] * a.m[8] - a.m[2] * a.m[6]) * s;
    r.m[5] = (a.m[2] * a.m[3] - a.m[0] * a.m[5]) * s;
    r.m[6] = (a.m[3] * a.m[7] - a.m[4] * a.m[6]) * s;
    r.m[7] = (a.m[1] * a.m[6] - a.m[0] * a.m[7]) * s;
    r.m[8] = (a.m[0] * a.m[4] - a.m[1] * a.m[3]) * s;
    return mv(r, f);
}

// One VBD step over host arrays (vbd_solver.cu:897-979), colours given.
template <class R>
void vbd_step(int n, R* pos, R* vel, const R* inv_mass, const int* tris, const R* poses, const R* areas,
              const R* mats, int T, const int* edges, const R* rest_angle, const R* rest_length, const R* bend, int E,
              const int* colors, const R* g, R dt, int iterations) {
    // adjacency in element order (vbd_solver.cu:813-895)
    std::vector<std::vector<std::pair<int, int>>> tadj(n), eadj(n);
    for (int t = 0; t < T; ++t)
        for (int k = 0; k < 3; ++k) tadj[tris[3 * t + k]].push_back({t, k});
    for (int e = 0; e < E; ++e)
        for (int k = 0; k < 4; ++k)
            if (edges[4 * e + k] >= 0) eadj[edges[4 * e + k]].push_back({e, k});
    int nc = 0;
    for (int i = 0; i < n; ++i) nc = std::max(nc, colors[i] + 1);
    std::vector<std::vector<int>> groups(nc);
    for (int i = 0; i < n; ++i) groups[colors[i]].push_back(i);
    std::vector<R> q(3 * (size_t)n), y(3 * (size_t)n), disp(3 * (size_t)n), m(n);
    // predictor (vbd_solver.cu:64-92)
    for (int i = 0; i < n; ++i) {
        const V<R> x = get(pos, i);
        put(q.data(), i, x);
        const R w = inv_mass[i];
        m[i] = w > R(1e-12) ? R(1) / w : R(0);
        if (w == R(0)) {
            put(y.data(), i, x);
            put(disp.data(), i, V<R>{0, 0, 0});
            continue;
        }
        const V<R> vn = get(vel, i) + V<R>{g[0], g[1], g[2]} * dt;
        put(y.data(), i, x + vn * dt);
        put(disp.data(), i, vn * dt);
        put(pos, i, x + vn * dt);
    }
    const R idt2 = R(1) / (dt * dt);
    for (int it = 0; it < iterations; ++it)
        for (int c = 0; c < nc; ++c)
            for (int i : groups[c]) {  // independent within a colour
                if (m[i] == R(0)) {
                    put(disp.data(), i, V<R>{0, 0, 0});
                    continue;
                }
                const R md = m[i] * idt2;
                V<R> f = (get(y.data(), i) - get(pos, i)) * md;
                M<R> h;
                h.m[0] = h.m[4] = h.m[8] = md;
                for (auto [t, k] : tadj[i]) {
                    const R mu = mats[3 * t], lambda = mats[3 * t + 1], damp = mats[3 * t + 2];
                    if (mu <= R(0) && lambda <= R(0)) continue;
                    const int* v = tris + 3 * t;
                    const V<R> x[3] = {get(pos, v[0]), get(pos, v[1]), get(pos, v[2])};
                    const V<R> p[3] = {get(q.data(), v[0]), get(q.data(), v[1]), get(q.data(), v[2])};
                    membrane(k, x, p, poses + 4 * t, areas[t], mu, lambda, damp, dt, f, h);
                }
                for (auto [e, k] : eadj[i]) {
                    const R ks = bend[2 * e], damp = bend[2 * e + 1];
                    if (ks <= R(0)) continue;
                    const int* v = edges + 4 * e;
                    if (v[0] < 0 || v[1] < 0) continue;
                    const V<R> x[4] = {get(pos, v[0]), get(pos, v[1]), get(pos, v[2]), get(pos, v[3])};
                    const V<R> p[4] = {get(q.data(), v[0]), get(q.data(), v[1]), get(q.data(), v[2]),
                                       get(q.data(), v[3])};
                    bending(k, x, p, rest_angle[e], rest_length[e], ks, damp, dt, f, h);
                }
                const R dh = det(h);
                V<R> d = get(disp.data(), i);
                if (std::fabs(dh) > R(1e-8)) {
                    d = d + solve(h, dh, f);
                    put(disp.data(), i, d);
                }
                put(pos, i, get(q.data(), i) + d);
            }
    // velocity (vbd_solver.cu:284-293)
    for (int i = 0; i < n; ++i) put(vel, i, (get(pos, i) - get(q.data(), i)) * (R(1) / dt));
}

template <class R>
std::vector<R> conv(const double* a, size_t k) {
    return a ? std::vector<R>(a, a + k) : std::vector<R>();
}

}  // namespace

extern "C" {

// One step on double host arrays; fp64 = 0 runs the FP32 port (inputs and
// outputs rounded through float).
int orc_vbd_step(int n, double* pos, double* vel, const double* inv_mass, const int* tris, const double* poses,
                 const double* areas, const double* mats, int T, const int* edges, const double* rest_angle,
                 const double* rest_length, const double* bend, int E, const int* colors, const double* g, double dt,
                 int iterations, int fp64) {
    if (n <= 0) return 0;
    if (fp64) {
        vbd_step<double>(n, pos, vel, inv_mass, tris, poses, areas, mats, T, edges, rest_angle, rest_length, bend, E,
                         colors, g, dt, iterations);
        return 0;
    }
    auto P = conv<float>(pos, 3 * (size_t)n), Vv = conv<float>(vel, 3 * (size_t)n), W = conv<float>(inv_mass, n);
    auto Po = conv<float>(poses, 4 * (size_t)T), A = conv<float>(areas, T), Ma = conv<float>(mats, 3 * (size_t)T);
    auto Ra = conv<float>(rest_angle, E), Rl = conv<float>(rest_length, E), B = conv<float>(bend, 2 * (size_t)E);
    const float gf[3] = {(float)g[0], (float)g[1], (float)g[2]};
    vbd_step<float>(n, P.data(), Vv.data(), W.data(), tris, Po.data(), A.data(), Ma.data(), T, edges, Ra.data(),
                    Rl.data(), B.data(), E, colors, gf, (float)dt, iterations);
    for (size_t k = 0; k < P.size(); ++k) { pos[k] = P[k]; vel[k] = Vv[k]; }
    return 0;
}

// Element evaluations (FP64) for finite-difference tests: force on vertex
// `which` and its Hessian block; energies.
void orc_vbd_membrane(int which, const double* x9, const double* p9, const double* dmi, double area, double mu,
                      double lambda, double damping, double dt, double* f3, double* h9) {
    const V<double> x[3] = {get(x9, 0), get(x9, 1), get(x9, 2)}, p[3] = {get(p9, 0), get(p9, 1), get(p9, 2)};
    V<double> f{0, 0, 0};
    M<double> h;
    membrane(which, x, p, dmi, area, mu, lambda, damping, dt, f, h);
    f3[0] = f.x; f3[1] = f.y; f3[2] = f.z;
    std::copy(h.m, h.m + 9, h9);
}
double orc_vbd_membrane_energy(const double* x9, const double* dmi, double area, double mu, double lambda) {
    const V<double> x[3] = {get(x9, 0), get(x9, 1), get(x9, 2)};
    return membrane_energy(x, dmi, area, mu, lambda);
}
void orc_vbd_bending(int which, const double* x12, const double* p12, double rest_angle, double rest_length,
                     double stiffness, double damping, double dt, double* f3, double* h9) {
    const V<double> x[4] = {get(x12, 0), get(x12, 1), get(x12, 2), get(x12, 3)};
    const V<double> p[4] = {get(p12, 0), get(p12, 1), get(p12, 2), get(p12, 3)};
    V<double> f{0, 0, 0};
    M<double> h;
    bending(which, x, p, rest_angle, rest_length, stiffness, damping, dt, f, h);
    f3[0] = f.x; f3[1] = f.y; f3[2] = f.z;
    std::copy(h.m, h.m + 9, h9);
}
// Signed hinge angle (0 when degenerate).
double orc_vbd_hinge_angle(const double* x12) {
    const V<double> x[4] = {get(x12, 0), get(x12, 1), get(x12, 2), get(x12, 3)};
    double th = 0, l1, l2;
    V<double> u1, u2, ue;
    return hinge(x, th, u1, u2, ue, l1, l2) ? th : 0.0;
}

}  // extern "C"
