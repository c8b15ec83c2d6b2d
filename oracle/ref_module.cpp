// TEST INFRASTRUCTURE ONLY: a minimal pybind11 module over the reference's
// chysx::cloth::ClothSimulator (compiled from the reference sources by
// oracle/build_ref.sh).  It binds only the cloth step and the calls the
// parity harness needs, with the reference's own method semantics; the
// reference's full bindings.cpp pulls in rigid/IK/coupled subsystems that
// are not part of this path.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>

#include "cloth/cloth_material.h"
#include "cloth/cloth_simulator.h"
#include "solver/vbd_solver.h"
#include "math/vec.cuh"

#ifndef REF_MODULE_NAME
#define REF_MODULE_NAME _chysx_ref
#endif

namespace py = pybind11;
using chysx::cloth::ClothSimulator;

PYBIND11_MODULE(REF_MODULE_NAME, m) {
    py::class_<ClothSimulator>(m, "ClothSimulator", py::module_local())
        .def(py::init<>())
        .def("set_material",
             [](ClothSimulator& s, float density, float damping, float gx, float gy, float gz) {
                 chysx::cloth::ClothMaterial mat;
                 mat.density = density;
                 mat.damping = damping;
                 mat.gx = gx;
                 mat.gy = gy;
                 mat.gz = gz;
                 s.set_material(mat);
             })
        .def("set_external_buffers", &ClothSimulator::set_external_buffers, py::arg("pos_ptr"),
             py::arg("vel_ptr"), py::arg("particle_count"), py::arg("inv_mass_ptr") = 0, py::arg("force_ptr") = 0)
        .def("set_mesh",
             [](ClothSimulator& s, py::array_t<int, py::array::c_style | py::array::forcecast> tris) {
                 s.set_mesh(reinterpret_cast<const chysx::math::Vec3i*>(tris.data()), (int)tris.shape(0));
             })
        .def("set_pins",
             [](ClothSimulator& s, py::array_t<int, py::array::c_style | py::array::forcecast> idx,
                py::array_t<float, py::array::c_style | py::array::forcecast> tgt, float k) {
                 s.set_pins(idx.data(), reinterpret_cast<const chysx::math::Vec3f*>(tgt.data()),
                            (int)idx.shape(0), k);
             })
        .def("build_springs_from_current_positions", &ClothSimulator::build_springs_from_current_positions,
             py::arg("stiffness"), py::arg("cuda_stream") = 0)
        .def("build_fem_stretch_from_current_positions",
             &ClothSimulator::build_fem_stretch_from_current_positions, py::arg("stiffness"),
             py::arg("cuda_stream") = 0)
        .def("build_fem_shear_from_current_positions",
             &ClothSimulator::build_fem_shear_from_current_positions, py::arg("stiffness"),
             py::arg("cuda_stream") = 0)
        .def("build_bending_from_current_positions",
             &ClothSimulator::build_bending_from_current_positions, py::arg("stiffness"),
             py::arg("cuda_stream") = 0)
        .def("redistribute_mass_area_weighted", &ClothSimulator::redistribute_mass_area_weighted,
             py::arg("surface_density"), py::arg("inv_mass_ptr"), py::arg("particle_count"),
             py::arg("cuda_stream") = 0)
        .def("set_pcg_iterations", &ClothSimulator::set_pcg_iterations)
        // static-shape contact (cloth_simulator.h:383-452)
        .def("add_static_plane",
             [](ClothSimulator& s, float nx, float ny, float nz, float d) {
                 chysx::collision::PlaneShape p;
                 p.n = chysx::math::Vec3f(nx, ny, nz);
                 p.d = d;
                 s.add_static_plane(p);
             })
        .def("add_static_box",
             [](ClothSimulator& s, py::array_t<float, py::array::c_style | py::array::forcecast> v15) {
                 if (v15.size() != 15) throw std::invalid_argument("add_static_box: 15 floats");
                 const float* f = v15.data();
                 chysx::collision::BoxShape b;
                 b.center = chysx::math::Vec3f(f[0], f[1], f[2]);
                 b.half_ext = chysx::math::Vec3f(f[3], f[4], f[5]);
                 b.ex = chysx::math::Vec3f(f[6], f[7], f[8]);
                 b.ey = chysx::math::Vec3f(f[9], f[10], f[11]);
                 b.ez = chysx::math::Vec3f(f[12], f[13], f[14]);
                 s.add_static_box(b);
             })
        .def("set_static_contact",
             [](ClothSimulator& s, float t, float k, float mu, float eps) {
                 s.set_static_contact_thickness(t);
                 s.set_static_contact_stiffness(k);
                 s.set_static_contact_friction(mu);
                 s.set_static_contact_friction_epsilon(eps);
             })
        // self-collision (cloth_simulator.h:238-325)
        .def("set_self_collision",
             [](ClothSimulator& s, float thickness, float k, float mu, float eps, int max_contacts) {
                 s.set_self_collision_max_contacts(max_contacts);
                 s.set_self_collision_thickness(thickness);
                 s.set_self_collision_stiffness(k);
                 s.set_self_collision_friction(mu);
                 s.set_self_collision_friction_epsilon(eps);
                 s.set_self_collision_enabled(true);
             })
        // The detector's contact list of the last step (pairs, weights,
        // slips; slips empty when the detector keeps none).
        .def("self_collision_contacts", [](ClothSimulator& s) {
            auto& det = s.self_collision_detector();
            const int cnt = std::min(det.count(0), det.max_contacts());
            const int c = std::max(cnt, 0);
            py::array_t<int> pairs({c, 4});
            py::array_t<float> weights({c, 8});
            const bool has_slip = det.slips().gpu_size() == (size_t)det.max_contacts() && c > 0;
            py::array_t<float> slips({has_slip ? c : 0, 4});
            if (c > 0) {
                cudaMemcpy(pairs.mutable_data(), det.pairs().gpu_data(), (size_t)c * 16, cudaMemcpyDeviceToHost);
                cudaMemcpy(weights.mutable_data(), det.weights().gpu_data(), (size_t)c * 32, cudaMemcpyDeviceToHost);
                if (has_slip)
                    cudaMemcpy(slips.mutable_data(), det.slips().gpu_data(), (size_t)c * 16, cudaMemcpyDeviceToHost);
            }
            return py::make_tuple(pairs, weights, slips);
        })
        .def("step", &ClothSimulator::step, py::arg("dt"), py::arg("cuda_stream") = 0)
        .def("debug_dump_last_solve", [](const ClothSimulator& s) {
            const int n = s.num_particles();
            const int nnz = s.num_off_diag_blocks();
            py::array_t<float> diag({n, 3, 3});
            py::array_t<int> rp({n + 1});
            py::array_t<int> col({nnz});
            py::array_t<float> vals({nnz, 3, 3});
            py::array_t<float> rhs({n, 3});
            py::array_t<float> dx({n, 3});
            if (n > 0) {
                s.debug_copy_hessian_diag(diag.mutable_data());
                s.debug_copy_hessian_csr(rp.mutable_data(), nnz > 0 ? col.mutable_data() : nullptr,
                                         nnz > 0 ? vals.mutable_data() : nullptr);
                s.debug_copy_last_rhs(rhs.mutable_data());
                s.debug_copy_last_dx(dx.mutable_data());
            }
            return py::make_tuple(diag, rp, col, vals, rhs, dx);
        });

    // the reference's cloth VBD solver (src/bindings.cpp:1868-1957), plus a
    // read-back of its colouring
    using chysx::solver::VBDSolver;
    py::class_<VBDSolver>(m, "ClothVBDSolver", py::module_local())
        .def(py::init<>())
        .def("build_cloth_coloring",
             [](VBDSolver& s, py::array_t<int, py::array::c_style | py::array::forcecast> tris,
                py::array_t<int, py::array::c_style | py::array::forcecast> edges, int n) {
                 s.build_cloth_coloring(reinterpret_cast<const chysx::math::Vec3i*>(tris.data()), (int)tris.shape(0),
                                        reinterpret_cast<const chysx::math::Vec4i*>(edges.data()),
                                        (int)edges.shape(0), n);
             })
        .def("build_tri_adjacency",
             [](VBDSolver& s, py::array_t<int, py::array::c_style | py::array::forcecast> tris, int n) {
                 s.build_tri_adjacency(reinterpret_cast<const chysx::math::Vec3i*>(tris.data()), (int)tris.shape(0), n);
             })
        .def("build_edge_adjacency",
             [](VBDSolver& s, py::array_t<int, py::array::c_style | py::array::forcecast> edges, int n) {
                 s.build_edge_adjacency(reinterpret_cast<const chysx::math::Vec4i*>(edges.data()), (int)edges.shape(0),
                                        n);
             })
        .def("step_cloth",
             [](VBDSolver& s, std::uintptr_t pos, std::uintptr_t vel, std::uintptr_t inv_mass, int n, std::uintptr_t tri,
                std::uintptr_t poses, std::uintptr_t areas, std::uintptr_t mats, int n_tris, std::uintptr_t edges,
                std::uintptr_t ra, std::uintptr_t rl, std::uintptr_t props, int n_edges, float gx, float gy, float gz,
                float dt, int iterations) {
                 using namespace chysx::math;
                 chysx::DeviceSpan<Vec3f> p(reinterpret_cast<Vec3f*>(pos), n), v(reinterpret_cast<Vec3f*>(vel), n);
                 chysx::DeviceSpan<float> w(reinterpret_cast<float*>(inv_mass), n);
                 s.step_cloth(p, v, w, reinterpret_cast<const Vec3i*>(tri), n_tris, reinterpret_cast<const Mat2f*>(poses),
                              reinterpret_cast<const float*>(areas), reinterpret_cast<const float*>(mats),
                              reinterpret_cast<const Vec4i*>(edges), n_edges, reinterpret_cast<const float*>(ra),
                              reinterpret_cast<const float*>(rl), reinterpret_cast<const float*>(props),
                              Vec3f(gx, gy, gz), dt, iterations, 0);
             })
        .def("num_colors", &VBDSolver::num_colors)
        .def("colors", [](const VBDSolver& s) {
            const int n = s.num_particles();
            py::array_t<int> out(n);
            if (n > 0) cudaMemcpy(out.mutable_data(), s.particle_colors_ptr(), (size_t)n * sizeof(int),
                                  cudaMemcpyDeviceToHost);
            return out;
        });
}
