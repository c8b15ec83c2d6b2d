// pybind11 facade `_chysx_native` over the C ABI (include/chysx_cloth.h).
//
// Mirrors the cloth part of the reference's module (src/bindings.cpp:25-600):
// ClothMaterial with the same fields, ClothSimulator with the same method
// names, argument names, defaults and exception types (ValueError for
// std::invalid_argument, IndexError for std::out_of_range, RuntimeError
// otherwise).  Every call goes through the extern "C" entry points; this
// file holds no simulation logic.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/chysx_cloth.h"
#include "../../include/chysx_vbd.h"

namespace py = pybind11;

namespace {

void check(int rc) {
    if (rc == CHYSX_OK) return;
    const std::string msg = chysx_last_error();
    if (rc == CHYSX_ERR_INVALID_ARGUMENT) throw py::value_error(msg);
    if (rc == CHYSX_ERR_OUT_OF_RANGE) throw py::index_error(msg);
    throw std::runtime_error(msg);
}

class PyClothSimulator {
public:
    PyClothSimulator() { check(chysx_cloth_create(&h_)); }
    ~PyClothSimulator() { chysx_cloth_destroy(h_); }
    PyClothSimulator(const PyClothSimulator&) = delete;
    PyClothSimulator& operator=(const PyClothSimulator&) = delete;
    chysx_cloth* h() const { return h_; }

private:
    chysx_cloth* h_ = nullptr;
};

class PyVbd {
public:
    PyVbd() { check(chysx_vbd_create(&h_)); }
    ~PyVbd() { chysx_vbd_destroy(h_); }
    PyVbd(const PyVbd&) = delete;
    PyVbd& operator=(const PyVbd&) = delete;
    chysx_vbd* h() const { return h_; }

private:
    chysx_vbd* h_ = nullptr;
};

using F32 = py::array_t<float, py::array::c_style | py::array::forcecast>;
using I32 = py::array_t<int32_t, py::array::c_style | py::array::forcecast>;

}  // namespace

PYBIND11_MODULE(_chysx_native, m) {
    m.doc() = "ChysX cloth step, B200-native (sm_100a) implementation";

    py::class_<chysx_cloth_material>(m, "ClothMaterial",
                                     "Plain-old-data material parameters for the cloth simulator.")
        .def(py::init([] { return chysx_cloth_material{0.0f, 0.0f, 0.0f, 0.05f, 0.0f, 0.0f, 0.0f, -9.81f}; }))
        .def_readwrite("lame_mu", &chysx_cloth_material::lame_mu)
        .def_readwrite("lame_lambda", &chysx_cloth_material::lame_lambda)
        .def_readwrite("bending", &chysx_cloth_material::bending)
        .def_readwrite("density", &chysx_cloth_material::density)
        .def_readwrite("damping", &chysx_cloth_material::damping)
        .def_readwrite("gx", &chysx_cloth_material::gx)
        .def_readwrite("gy", &chysx_cloth_material::gy)
        .def_readwrite("gz", &chysx_cloth_material::gz);

    py::class_<PyClothSimulator>(m, "ClothSimulator", "Implicit-Euler cloth simulator (device-pointer API).")
        .def(py::init<>())
        .def("set_material",
             [](PyClothSimulator& s, const chysx_cloth_material& mat) { check(chysx_cloth_set_material(s.h(), &mat)); },
             py::arg("material"))
        .def("material",
             [](const PyClothSimulator& s) {
                 chysx_cloth_material out;
                 check(chysx_cloth_get_material(s.h(), &out));
                 return out;
             })
        .def("set_external_buffers",
             [](PyClothSimulator& s, std::uintptr_t pos, std::uintptr_t vel, int n, std::uintptr_t inv_mass,
                std::uintptr_t force) { check(chysx_cloth_set_external_buffers(s.h(), pos, vel, n, inv_mass, force)); },
             py::arg("pos_ptr"), py::arg("vel_ptr"), py::arg("particle_count"), py::arg("inv_mass_ptr") = 0,
             py::arg("force_ptr") = 0)
        .def("step",
             [](PyClothSimulator& s, float dt, std::uintptr_t stream) { check(chysx_cloth_step(s.h(), dt, stream)); },
             py::arg("dt"), py::arg("cuda_stream") = 0)
        .def("set_pins",
             [](PyClothSimulator& s, I32 indices, F32 targets, float stiffness) {
                 if (indices.ndim() != 1) throw py::value_error("ClothSimulator.set_pins: indices must be 1-D");
                 if (targets.ndim() != 2 || targets.shape(1) != 3)
                     throw py::value_error("ClothSimulator.set_pins: targets must have shape (N, 3)");
                 if (indices.shape(0) != targets.shape(0))
                     throw py::value_error("ClothSimulator.set_pins: indices and targets must have the same length");
                 check(chysx_cloth_set_pins(s.h(), indices.data(), targets.data(), (int)indices.shape(0), stiffness));
             },
             py::arg("indices"), py::arg("targets"), py::arg("stiffness") = 1.0e6f)
        .def("clear_pins", [](PyClothSimulator& s) { check(chysx_cloth_clear_pins(s.h())); })
        .def("num_pins",
             [](const PyClothSimulator& s) {
                 int n = 0;
                 check(chysx_cloth_num_pins(s.h(), &n));
                 return n;
             })
        .def("update_pin_targets",
             [](PyClothSimulator& s, F32 targets, std::uintptr_t stream) {
                 if (targets.ndim() != 2 || targets.shape(1) != 3)
                     throw py::value_error(
                         "ClothSimulator.update_pin_targets: targets must have shape (N, 3) and dtype float32");
                 check(chysx_cloth_update_pin_targets(s.h(), targets.data(), (int)targets.shape(0), stream));
             },
             py::arg("targets"), py::arg("cuda_stream") = 0)
        .def("set_mesh",
             [](PyClothSimulator& s, I32 tris) {
                 if (tris.ndim() != 2 || tris.shape(1) != 3)
                     throw py::value_error("ClothSimulator.set_mesh: triangles must have shape (M, 3) and dtype int32");
                 check(chysx_cloth_set_mesh(s.h(), tris.data(), (int)tris.shape(0)));
             },
             py::arg("triangles"))
        .def("edges",
             [](const PyClothSimulator& s) {
                 int e = 0;
                 check(chysx_cloth_num_edges(s.h(), &e));
                 py::array_t<int32_t> out({e, 2});
                 check(chysx_cloth_get_edges(s.h(), out.mutable_data()));
                 return out;
             })
        .def("build_springs_from_current_positions",
             [](PyClothSimulator& s, py::object stiffness, std::uintptr_t stream) {
                 if (py::isinstance<py::array>(stiffness)) {
                     F32 k = stiffness.cast<F32>();
                     int e = 0;
                     check(chysx_cloth_num_edges(s.h(), &e));
                     if (k.ndim() != 1 || k.shape(0) != e)
                         throw py::value_error("per-edge stiffness must have shape (num_edges,)");
                     check(chysx_cloth_build_springs(s.h(), 0.0f, k.data(), stream));
                 } else {
                     check(chysx_cloth_build_springs(s.h(), stiffness.cast<float>(), nullptr, stream));
                 }
             },
             py::arg("stiffness"), py::arg("cuda_stream") = 0)
        .def("num_springs",
             [](const PyClothSimulator& s) {
                 int n = 0;
                 check(chysx_cloth_num_springs(s.h(), &n));
                 return n;
             })
        .def("redistribute_mass_area_weighted",
             [](PyClothSimulator& s, float rho, std::uintptr_t inv_mass, int n, std::uintptr_t stream) {
                 check(chysx_cloth_redistribute_mass(s.h(), rho, inv_mass, n, stream));
             },
             py::arg("surface_density"), py::arg("inv_mass_ptr"), py::arg("particle_count"),
             py::arg("cuda_stream") = 0)
        .def("build_fem_stretch_from_current_positions",
             [](PyClothSimulator& s, py::object stiffness, std::uintptr_t stream) {
                 if (py::isinstance<py::array>(stiffness)) {
                     F32 k = stiffness.cast<F32>();
                     if (k.ndim() != 1) throw py::value_error("per-triangle stiffness must be 1-D");
                     check(chysx_cloth_build_fem_stretch(s.h(), 0.0f, k.data(), stream));
                 } else {
                     check(chysx_cloth_build_fem_stretch(s.h(), stiffness.cast<float>(), nullptr, stream));
                 }
             },
             py::arg("stiffness"), py::arg("cuda_stream") = 0)
        .def("build_fem_shear_from_current_positions",
             [](PyClothSimulator& s, py::object stiffness, std::uintptr_t stream) {
                 if (py::isinstance<py::array>(stiffness)) {
                     F32 k = stiffness.cast<F32>();
                     if (k.ndim() != 1) throw py::value_error("per-triangle stiffness must be 1-D");
                     check(chysx_cloth_build_fem_shear(s.h(), 0.0f, k.data(), stream));
                 } else {
                     check(chysx_cloth_build_fem_shear(s.h(), stiffness.cast<float>(), nullptr, stream));
                 }
             },
             py::arg("stiffness"), py::arg("cuda_stream") = 0)
        .def("build_bending_from_current_positions",
             [](PyClothSimulator& s, float stiffness, std::uintptr_t stream) {
                 check(chysx_cloth_build_bending(s.h(), stiffness, stream));
             },
             py::arg("stiffness"), py::arg("cuda_stream") = 0)
        // ---- static-shape contact (src/bindings.cpp:596-698) ----------
        .def("add_static_plane",
             [](PyClothSimulator& s, F32 n, float d) {
                 if (n.ndim() != 1 || n.shape(0) != 3)
                     throw py::value_error("ClothSimulator.add_static_plane: n must be a (3,) float32 vector");
                 check(chysx_cloth_add_static_plane(s.h(), n.data(), d));
             },
             py::arg("n"), py::arg("d"))
        .def("add_static_box",
             [](PyClothSimulator& s, F32 center, F32 half_ext, F32 ex, F32 ey, F32 ez) {
                 const std::pair<F32*, const char*> args[] = {
                     {&center, "center"}, {&half_ext, "half_ext"}, {&ex, "ex"}, {&ey, "ey"}, {&ez, "ez"}};
                 for (const auto& a : args)
                     if (a.first->ndim() != 1 || a.first->shape(0) != 3)
                         throw py::value_error(std::string("ClothSimulator.add_static_box: ") + a.second +
                                               " must be a (3,) float32 vector");
                 check(chysx_cloth_add_static_box(s.h(), center.data(), half_ext.data(), ex.data(), ey.data(),
                                                  ez.data()));
             },
             py::arg("center"), py::arg("half_ext"), py::arg("ex"), py::arg("ey"), py::arg("ez"))
        .def("clear_static_shapes", [](PyClothSimulator& s) { check(chysx_cloth_clear_static_shapes(s.h())); })
        .def("set_static_contact_thickness",
             [](PyClothSimulator& s, float t) { check(chysx_cloth_set_static_contact_thickness(s.h(), t)); },
             py::arg("thickness"))
        .def("set_static_contact_stiffness",
             [](PyClothSimulator& s, float k) { check(chysx_cloth_set_static_contact_stiffness(s.h(), k)); },
             py::arg("stiffness"))
        .def("set_static_contact_friction",
             [](PyClothSimulator& s, float mu) { check(chysx_cloth_set_static_contact_friction(s.h(), mu)); },
             py::arg("mu"))
        .def("set_static_contact_friction_epsilon",
             [](PyClothSimulator& s, float e) { check(chysx_cloth_set_static_contact_friction_epsilon(s.h(), e)); },
             py::arg("eps_u"))
        .def("static_contact_thickness",
             [](const PyClothSimulator& s) {
                 float v = 0.f;
                 check(chysx_cloth_get_static_contact(s.h(), &v, nullptr, nullptr, nullptr));
                 return v;
             })
        .def("static_contact_stiffness",
             [](const PyClothSimulator& s) {
                 float v = 0.f;
                 check(chysx_cloth_get_static_contact(s.h(), nullptr, &v, nullptr, nullptr));
                 return v;
             })
        .def("static_contact_friction",
             [](const PyClothSimulator& s) {
                 float v = 0.f;
                 check(chysx_cloth_get_static_contact(s.h(), nullptr, nullptr, &v, nullptr));
                 return v;
             })
        .def("static_contact_friction_epsilon",
             [](const PyClothSimulator& s) {
                 float v = 0.f;
                 check(chysx_cloth_get_static_contact(s.h(), nullptr, nullptr, nullptr, &v));
                 return v;
             })
        .def("static_plane_count",
             [](const PyClothSimulator& s) {
                 int p = 0;
                 check(chysx_cloth_static_shape_counts(s.h(), &p, nullptr));
                 return p;
             })
        .def("static_box_count",
             [](const PyClothSimulator& s) {
                 int b = 0;
                 check(chysx_cloth_static_shape_counts(s.h(), nullptr, &b));
                 return b;
             })
        // ---- contact operator (collision::ContactSpMVOp) --------------
        .def("set_contact_operator",
             [](PyClothSimulator& s, std::uintptr_t pairs, std::uintptr_t weights, std::uintptr_t count,
                int max_contacts, float stiffness, std::uintptr_t stiffnesses, std::uintptr_t slips, float mu,
                float eps, int residual_mode) {
                 chysx_contact_op op{};
                 op.pairs = pairs;
                 op.weights = weights;
                 op.count = count;
                 op.max_contacts = max_contacts;
                 op.stiffness = stiffness;
                 op.stiffnesses = stiffnesses;
                 op.slips = slips;
                 op.friction_mu = mu;
                 op.friction_epsilon = eps;
                 op.residual_mode = residual_mode;
                 check(chysx_cloth_set_contact_op(s.h(), &op));
             },
             py::arg("pairs"), py::arg("weights"), py::arg("count"), py::arg("max_contacts"), py::arg("stiffness"),
             py::arg("stiffnesses") = 0, py::arg("slips") = 0, py::arg("friction_mu") = 0.0f,
             py::arg("friction_epsilon") = 1.0e-4f, py::arg("residual_mode") = 0,
             "Fold a device-resident contact list (int32 pairs (M,4), float32 weights (M,8) = w0..w3, normal, "
             "depth, int32 count) into every step's system.")
        .def("clear_contact_operator", [](PyClothSimulator& s) { check(chysx_cloth_clear_contact_op(s.h())); })
        .def("contact_stats",
             [](PyClothSimulator& s) {
                 int live = 0, dropped = 0, slots = 0;
                 check(chysx_cloth_contact_stats(s.h(), &live, &dropped, &slots));
                 py::dict d;
                 d["live"] = live;
                 d["dropped"] = dropped;
                 d["slots"] = slots;
                 return d;
             })
        .def("step_into",
             [](PyClothSimulator& s, float dt, std::uintptr_t pos_in, std::uintptr_t vel_in, std::uintptr_t pos_out,
                std::uintptr_t vel_out, std::uintptr_t stream) {
                 check(chysx_cloth_step_into(s.h(), dt, pos_in, vel_in, pos_out, vel_out, stream));
             },
             py::arg("dt"), py::arg("pos_in"), py::arg("vel_in"), py::arg("pos_out"), py::arg("vel_out"),
             py::arg("cuda_stream") = 0,
             "One step from (pos_in, vel_in) into (pos_out, vel_out) without a copy pass.")
        .def("set_row_order", [](PyClothSimulator& s, int mode) { check(chysx_cloth_set_row_order(s.h(), mode)); },
             py::arg("mode"), "0: the caller's particle order; 1: spatially compact row blocks")
        .def("set_preconditioner",
             [](PyClothSimulator& s, const std::string& kind, int degree, float ratio) {
                 int k = -1;
                 if (kind == "block_jacobi") k = 0;
                 if (kind == "chebyshev") k = 1;
                 if (kind == "chebyshev_coarse") k = 2;
                 if (k < 0)
                     throw py::value_error(
                         "preconditioner kind must be 'block_jacobi', 'chebyshev' or 'chebyshev_coarse'");
                 check(chysx_cloth_set_preconditioner(s.h(), k, degree, ratio));
             },
             py::arg("kind"), py::arg("degree") = 7, py::arg("ratio") = 30.0f)
        .def("set_pcg_iterations",
             [](PyClothSimulator& s, int m) { check(chysx_cloth_set_pcg_iterations(s.h(), m)); }, py::arg("max_iter"))
        .def("pcg_iterations",
             [](const PyClothSimulator& s) {
                 int m = 0;
                 check(chysx_cloth_pcg_iterations(s.h(), &m));
                 return m;
             })
        .def("set_solver",
             [](PyClothSimulator& s, int max_iter, double rel_tol, const std::string& warm) {
                 int w = -1;
                 if (warm == "zero") w = CHYSX_WARM_ZERO;
                 if (warm == "previous") w = CHYSX_WARM_PREVIOUS;
                 if (warm == "learned") w = CHYSX_WARM_LEARNED;
                 if (warm == "previous_scaled") w = CHYSX_WARM_PREVIOUS_SCALED;
                 if (w < 0)
                     throw py::value_error("warm_start must be 'zero', 'previous', 'learned' or 'previous_scaled'");
                 check(chysx_cloth_set_solver(s.h(), max_iter, rel_tol, w));
             },
             py::arg("max_iter") = 50, py::arg("rel_tol") = 0.0, py::arg("warm_start") = "previous")
        .def("set_options",
             [](PyClothSimulator& s, bool springs_in_step, bool apply_external_force, float fem_det_eps) {
                 check(chysx_cloth_set_options(s.h(), springs_in_step, apply_external_force, fem_det_eps));
             },
             py::arg("springs_in_step") = true, py::arg("apply_external_force") = false,
             py::arg("fem_det_eps") = 1.0e-6f)
        .def("last_stats",
             [](PyClothSimulator& s) {
                 int it = 0, st = 0;
                 double rr = 0.0;
                 check(chysx_cloth_last_stats(s.h(), &it, &rr, &st));
                 return py::make_tuple(it, rr, st);
             },
             "(iterations, relative residual ||r||/||b||, status) of the last step; synchronises.")
        .def("set_true_residual",
             [](PyClothSimulator& s, bool on) { check(chysx_cloth_set_true_residual(s.h(), on ? 1 : 0)); },
             py::arg("on") = true,
             "Also recompute ||b - A dx|| / ||b|| of the returned dx after every solve "
             "(PCGParams::compute_true_residual).")
        .def("last_true_residual",
             [](PyClothSimulator& s) {
                 int n = 0;
                 check(chysx_cloth_num_instances(s.h(), &n));
                 py::array_t<double> rel(n);
                 double worst = 0.0;
                 check(chysx_cloth_true_residual(s.h(), n, rel.mutable_data(), &worst));
                 return py::make_tuple(rel, worst);
             },
             "(per-instance true relative residuals, the largest) of the last step; synchronises "
             "(PCGSolver::host_last_true_relative_residual).")
        .def("num_particles",
             [](const PyClothSimulator& s) {
                 int n = 0;
                 check(chysx_cloth_num_particles(s.h(), &n));
                 return n;
             })
        .def("num_off_diag_blocks",
             [](const PyClothSimulator& s) {
                 int n = 0;
                 check(chysx_cloth_num_off_diag_blocks(s.h(), &n));
                 return n;
             })
        .def("set_instances",
             [](PyClothSimulator& s, py::object offsets) {
                 if (offsets.is_none()) {
                     check(chysx_cloth_set_instances(s.h(), nullptr, 0));
                     return;
                 }
                 I32 o = offsets.cast<I32>();
                 if (o.ndim() != 1 || o.shape(0) < 2)
                     throw py::value_error("set_instances: offsets must be 1-D with at least 2 entries");
                 check(chysx_cloth_set_instances(s.h(), o.data(), (int)o.shape(0) - 1));
             },
             py::arg("offsets"),
             "Declare independent cloth instances: particles [offsets[b], offsets[b+1]); None = one system.")
        .def("instance_stats",
             [](PyClothSimulator& s) {
                 int n = 0;
                 check(chysx_cloth_num_instances(s.h(), &n));
                 py::array_t<int32_t> it(n), st(n);
                 py::array_t<double> rr(n);
                 check(chysx_cloth_instance_stats(s.h(), n, it.mutable_data(), rr.mutable_data(), st.mutable_data()));
                 return py::make_tuple(it, rr, st);
             })
        .def("set_network",
             [](PyClothSimulator& s, F32 params) {
                 if (params.ndim() != 1) throw py::value_error("set_network: params must be 1-D float32");
                 check(chysx_cloth_set_network(s.h(), params.data(), (int)params.shape(0)));
             },
             py::arg("params"))
        .def("set_feature_output",
             [](PyClothSimulator& s, std::uintptr_t features, std::uintptr_t predictions) {
                 check(chysx_cloth_set_feature_output(s.h(), features, predictions));
             },
             py::arg("features_ptr"), py::arg("predictions_ptr") = 0)
        .def("guess_kept",
             [](PyClothSimulator& s) {
                 int k = 0;
                 check(chysx_cloth_guess_kept(s.h(), &k));
                 return k;
             })
        .def("set_tuning",
             [](PyClothSimulator& s, int path, int block, int grid) { check(chysx_cloth_set_tuning(s.h(), path, block, grid)); },
             py::arg("solver_path") = 0, py::arg("block") = 0, py::arg("grid") = 0)
        .def("solver_info",
             [](const PyClothSimulator& s) {
                 int p = 0, g = 0, b = 0;
                 check(chysx_cloth_solver_info(s.h(), &p, &g, &b));
                 static const char* names[] = {"resident", "loop", "streamed"};
                 return py::make_tuple(names[p], g, b);
             })
        .def("set_sync_mode", [](PyClothSimulator& s, int mode) { check(chysx_cloth_set_sync_mode(s.h(), mode)); },
             py::arg("mode"))
        .def("autotune",
             [](PyClothSimulator& s, float dt, int repetitions, std::uintptr_t stream) {
                 check(chysx_cloth_autotune(s.h(), dt, repetitions, stream));
                 int count = 0;
                 check(chysx_cloth_autotune_results(s.h(), 0, &count, nullptr, nullptr));
                 std::vector<int32_t> cfg(8 * (size_t)std::max(count, 1));
                 std::vector<float> ms(std::max(count, 1));
                 check(chysx_cloth_autotune_results(s.h(), count, &count, cfg.data(), ms.data()));
                 static const char* names[] = {"resident", "loop", "streamed"};
                 py::list out;
                 for (int k = 0; k < count; ++k) {
                     const int32_t* c = &cfg[8 * (size_t)k];
                     py::dict d;
                     d["path"] = c[0]; d["block"] = c[1]; d["sync"] = c[2]; d["kernel"] = names[c[3]];
                     d["grid"] = c[4]; d["threads"] = c[5]; d["iters"] = c[6]; d["status"] = c[7];
                     d["solve_ms"] = ms[k];
                     out.append(d);
                 }
                 return out;
             },
             py::arg("dt"), py::arg("repetitions") = 2, py::arg("cuda_stream") = 0)
        .def("debug_dump_last_solve", [](PyClothSimulator& s) {
            int n = 0, nnz = 0;
            check(chysx_cloth_num_particles(s.h(), &n));
            check(chysx_cloth_num_off_diag_blocks(s.h(), &nnz));
            py::array_t<float> diag({n, 3, 3});
            py::array_t<int32_t> row_offsets({n + 1});
            py::array_t<int32_t> col_indices({nnz});
            py::array_t<float> values({nnz, 3, 3});
            py::array_t<float> rhs({n, 3});
            py::array_t<float> dx({n, 3});
            if (n > 0)
                check(chysx_cloth_debug_dump(s.h(), diag.mutable_data(), row_offsets.mutable_data(),
                                             nnz > 0 ? col_indices.mutable_data() : nullptr,
                                             nnz > 0 ? values.mutable_data() : nullptr, rhs.mutable_data(),
                                             dx.mutable_data()));
            return py::make_tuple(diag, row_offsets, col_indices, values, rhs, dx);
        });

    // ---- ClothVBDSolver (src/bindings.cpp:1868-1957) --------------------
    py::class_<PyVbd>(m, "ClothVBDSolver",
                      "Vertex Block Descent solver for cloth (triangle membrane + dihedral bending).")
        .def(py::init<>())
        .def("build_cloth_coloring",
             [](PyVbd& s, I32 tris, I32 edges, int n) {
                 if (tris.ndim() != 2 || tris.shape(1) != 3) throw py::value_error("tri_indices must be (T, 3) int32");
                 if (edges.ndim() != 2 || edges.shape(1) != 4) throw py::value_error("edge_indices must be (E, 4) int32");
                 check(chysx_vbd_build_cloth_coloring(s.h(), tris.data(), (int)tris.shape(0), edges.data(),
                                                      (int)edges.shape(0), n));
             },
             py::arg("tri_indices"), py::arg("edge_indices"), py::arg("n_particles"),
             "Build graph coloring from triangle + bending edge topology.")
        .def("set_coloring",
             [](PyVbd& s, I32 colors) {
                 check(chysx_vbd_set_coloring(s.h(), colors.data(), (int)colors.size()));
             },
             py::arg("colors"), "Use an externally computed colour per particle.")
        .def("build_tri_adjacency",
             [](PyVbd& s, I32 tris, int n) {
                 if (tris.ndim() != 2 || tris.shape(1) != 3) throw py::value_error("tri_indices must be (T, 3) int32");
                 check(chysx_vbd_build_tri_adjacency(s.h(), tris.data(), (int)tris.shape(0), n));
             },
             py::arg("tri_indices"), py::arg("n_particles"), "Build per-vertex triangle adjacency (CSR).")
        .def("build_edge_adjacency",
             [](PyVbd& s, I32 edges, int n) {
                 if (edges.ndim() != 2 || edges.shape(1) != 4) throw py::value_error("edge_indices must be (E, 4) int32");
                 check(chysx_vbd_build_edge_adjacency(s.h(), edges.data(), (int)edges.shape(0), n));
             },
             py::arg("edge_indices"), py::arg("n_particles"), "Build per-vertex bending-edge adjacency (CSR).")
        .def("step_cloth",
             [](PyVbd& s, std::uintptr_t pos, std::uintptr_t vel, std::uintptr_t inv_mass, int n, std::uintptr_t tri,
                std::uintptr_t poses, std::uintptr_t areas, std::uintptr_t mats, int n_tris, std::uintptr_t edges,
                std::uintptr_t rest_angle, std::uintptr_t rest_length, std::uintptr_t props, int n_edges, float gx,
                float gy, float gz, float dt, int iterations, std::uintptr_t stream) {
                 check(chysx_vbd_step_cloth(s.h(), pos, vel, inv_mass, n, tri, poses, areas, mats, n_tris, edges,
                                            rest_angle, rest_length, props, n_edges, gx, gy, gz, dt, iterations,
                                            stream));
             },
             py::arg("pos_ptr"), py::arg("vel_ptr"), py::arg("inv_mass_ptr"), py::arg("n_particles"),
             py::arg("tri_indices_ptr"), py::arg("tri_poses_ptr"), py::arg("tri_areas_ptr"),
             py::arg("tri_materials_ptr"), py::arg("n_tris"), py::arg("edge_indices_ptr"),
             py::arg("edge_rest_angle_ptr"), py::arg("edge_rest_length_ptr"), py::arg("edge_bending_props_ptr"),
             py::arg("n_edges"), py::arg("gx"), py::arg("gy"), py::arg("gz"), py::arg("dt"), py::arg("iterations"),
             py::arg("cuda_stream") = 0, "Run one cloth VBD substep.")
        .def("num_colors",
             [](const PyVbd& s) {
                 int c = 0;
                 check(chysx_vbd_num_colors(s.h(), &c));
                 return c;
             })
        .def("colors", [](const PyVbd& s, int n) {
            py::array_t<int32_t> out(n);
            check(chysx_vbd_colors(s.h(), out.mutable_data(), n));
            return out;
        }, py::arg("n_particles"));
}
