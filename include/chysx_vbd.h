/*
 * chysx_vbd.h — C ABI of the B200-native cloth Vertex Block Descent solver.
 *
 * Drop-in for the reference's ClothVBDSolver (caixiao-0725/Ai-Phyiscs,
 * src/bindings.cpp:1868-1957 over solver::VBDSolver, src/solver/
 * vbd_solver.h:134-176): graph colouring, per-vertex element adjacency and
 * one cloth step of VBD (Chen et al. 2024) with a Stable Neo-Hookean
 * membrane and discrete-shell hinge bending.  Status codes and
 * chysx_last_error() are those of chysx_cloth.h.  Device arrays are passed
 * as uintptr_t addresses, host arrays as pointers, streams as uintptr_t.
 */
#ifndef CHYSX_VBD_H_
#define CHYSX_VBD_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct chysx_vbd chysx_vbd; /* opaque solver handle */

/* VBDSolver() / ~VBDSolver(). */
int chysx_vbd_create(chysx_vbd** out);
int chysx_vbd_destroy(chysx_vbd* h);

/* VBDSolver::build_cloth_coloring (vbd_solver.cu:724-811): greedy colouring
 * of the conflict graph of the triangles (host int32 (T, 3)) and of every
 * pair of a bending edge's vertices (host int32 (E, 4): o0, o1, v2, v3; -1
 * where a boundary edge has no opposite vertex), vertices taken by
 * decreasing degree (ties by index). */
int chysx_vbd_build_cloth_coloring(chysx_vbd* h, const int32_t* tris, int n_tris, const int32_t* edges,
                                   int n_edges, int n_particles);
/* VBDSolver::set_coloring (vbd_solver.cu:490-520): a colour per particle. */
int chysx_vbd_set_coloring(chysx_vbd* h, const int32_t* colors, int n_particles);
/* VBDSolver::build_tri_adjacency / build_edge_adjacency
 * (vbd_solver.cu:813-895): per-vertex (element, local vertex) lists. */
int chysx_vbd_build_tri_adjacency(chysx_vbd* h, const int32_t* tris, int n_tris, int n_particles);
int chysx_vbd_build_edge_adjacency(chysx_vbd* h, const int32_t* edges, int n_edges, int n_particles);
int chysx_vbd_num_colors(const chysx_vbd* h, int* out);
/* The colour of every particle (n_particles entries). */
int chysx_vbd_colors(const chysx_vbd* h, int32_t* out, int n_particles);

/* VBDSolver::step_cloth (vbd_solver.cu:897-979): one implicit-Euler step of
 * `iterations` colour sweeps.  pos / vel (float3), inv_mass (float) are
 * advanced in place; per triangle (int32 x3) Dm^-1 (float x4, row-major),
 * rest area, material (mu, lambda, damping); per bending edge (int32 x4) rest
 * angle, rest length, (stiffness, damping).  n_tris / n_edges = 0 leave that
 * energy out.  The step is one CUDA-graph launch on `stream`. */
int chysx_vbd_step_cloth(chysx_vbd* h, uintptr_t pos, uintptr_t vel, uintptr_t inv_mass, int n_particles,
                         uintptr_t tri_indices, uintptr_t tri_poses, uintptr_t tri_areas, uintptr_t tri_materials,
                         int n_tris, uintptr_t edge_indices, uintptr_t edge_rest_angle, uintptr_t edge_rest_length,
                         uintptr_t edge_bending_props, int n_edges, float gx, float gy, float gz, float dt,
                         int iterations, uintptr_t stream);

#ifdef __cplusplus
}
#endif

#endif /* CHYSX_VBD_H_ */
