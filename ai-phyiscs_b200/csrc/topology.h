// Host-side sparsity and gather-list construction for the cloth system.
//
// The global system keeps the reference's split storage (per-row diagonal
// 3x3 block + off-diagonal block rows with sorted, unique columns,
// src/sparse/block_csr.cu:91-147), laid out as a sliced ELLPACK matrix with
// slices of kSlice = 32 consecutive rows (one warp): entry (row, k) of slice
// s lives at slice_off[s] + k*32 + (row & 31), so a warp reading entry k of
// its 32 rows issues one coalesced 128-byte load per component.  Rows shorter
// than the slice width are padded with col = row and zero blocks.
//
// Assembly is row-owned instead of element-scatter: each row gets the list
// of elements incident to it (triangle + its local vertex, spring + its
// end), together with the slot in that row of every other element vertex,
// so one thread writes its row's blocks exactly once with no atomics and no
// zero-fill pass (replaces BlockCSR3::set_zero + resolve_slots + atomic
// scatter, src/sparse/block_csr.cu:149-204, block_csr_atomic.cuh:33-45).
#pragma once

#include <cstdint>
#include <vector>

namespace chysx_b200 {

constexpr int kSlice = 32;
constexpr unsigned kDiagSlot = 0xFFu;   // "other vertex is this row": goes to the diagonal
constexpr int kMaxRowWidth = 254;       // slots are stored in 8 bits

struct HostTopology {
    int n = 0;          // internal rows: particles, plus padding rows that
                        // start every instance on a fresh 32-row slice
    int n_ext = 0;      // particles in the caller's buffers
    int n_slices = 0;
    int n_pad = 0;      // n_slices * 32
    int max_width = 0;  // widest off-diagonal slice
    // reference-format adjacency (row_offsets / col_indices)
    std::vector<int> csr_ptr, csr_col;
    // sliced ELL matrix pattern
    std::vector<int> slice_off;  // [n_slices + 1], in entries (multiples of 32)
    std::vector<int> col;        // [slice_off.back()]
    std::vector<int> csr_to_ell; // ELL entry of each CSR entry (debug dump)
    // triangle incidence: tri id, meta = local | slot_next << 8 | slot_prev << 16
    std::vector<int> tinc_off, tinc;
    std::vector<uint32_t> tinc_meta;
    // spring incidence: edge id, meta = end | slot_other << 8
    std::vector<int> sinc_off, sinc;
    std::vector<uint32_t> sinc_meta;
    // dihedral (bending) incidence: dihedral id, meta = local vertex |
    // slot of local (l+1)%4 << 8 | of (l+2)%4 << 16 | of (l+3)%4 << 24
    std::vector<int> dinc_off, dinc;
    std::vector<uint32_t> dinc_meta;
    // pins sorted by row; pin_perm[sorted] = caller's index
    std::vector<int> pin_off, pin_row, pin_perm;
    // instances: internal rows <-> particles (empty when they coincide)
    std::vector<int> row_to_ext, ext_to_row;
    std::vector<int> inst_slice;  // [n_inst + 1] slice range of every instance
    long long nnz() const { return (long long)csr_col.size(); }
    long long ell_entries() const { return slice_off.empty() ? 0 : slice_off.back(); }
};

// Builds the pattern from triangles (if use_tris), spring edges (if
// use_springs) and pins over n particles.  inst_offsets (empty, or n_inst+1
// increasing particle offsets from 0 to n) splits the particles into
// independent instances; every instance then starts on its own slice and no
// element may connect two instances.  Throws std::out_of_range for a vertex
// index outside [0, n), std::invalid_argument for an element spanning two
// instances, std::runtime_error when a row exceeds kMaxRowWidth neighbours.
// Bending dihedrals (4 vertices each: v0, v1 = the shared edge, v2 = the
// third vertex of the face containing the directed edge v0 -> v1, v3 = that
// of the face containing v1 -> v0) add every pair of their vertices to the
// pattern when use_bending.
// `order` (empty: the caller's order) lists the particles in internal row
// order; within every instance it must be a permutation of that instance's
// particle range.
void build_topology(int n, const std::vector<int>& tris, bool use_tris,
                    const std::vector<int>& edges, bool use_springs,
                    const std::vector<int>& pins, const std::vector<int>& inst_offsets,
                    HostTopology& out, const std::vector<int>& dihedrals = {},
                    bool use_bending = false, const std::vector<int>& order = {});

// A spatially compact row order: recursive coordinate bisection of each
// instance's positions (xyz per particle) at the median of the longest box
// side, with split sizes that are multiples of `block` rows (512) while a
// part spans more than two blocks and of 32 rows below, so every 32-row slice
// and every aligned block of rows is a compact patch.  Deterministic.
void spatial_order(const float* pos, int n, const std::vector<int>& inst_offsets, std::vector<int>& order,
                   int block = 512);

// Dihedrals of a consistently oriented triangle mesh as the reference finds
// them (src/cloth/cloth_simulator.cu:467-506): every interior edge v0 < v1
// whose two directions both occur gives (v0, v1, third(v0->v1),
// third(v1->v0)); when a directed edge occurs in several triangles the last
// one wins.  Ordered by (v0, v1).
void build_dihedrals(const std::vector<int>& tris, std::vector<int>& out);

// Work split of the persistent PCG kernel: `grid` CTAs each take a
// contiguous, balanced range of slices; instances own contiguous slice
// ranges.  Each (CTA, instance) pair that overlaps gets one reduction slot;
// an instance's slots are contiguous and ordered by CTA.
struct HostPlan {
    int grid = 0;
    int n_inst = 0;
    int max_slices_per_cta = 0;
    int max_inst_per_cta = 0;
    std::vector<int> slice_inst, inst_slice, cta_slice, cta_inst_lo, cta_inst_hi, inst_cta_lo, inst_slot;
};

// inst_slice: [n_inst + 1] slice offsets (every instance non-empty).
// grid is clamped to [1, n_slices].
void build_plan(const std::vector<int>& inst_slice, int grid, HostPlan& out);

// Per-vertex incident-triangle lists (sorted by triangle id), used by the
// deterministic mass redistribution.
void build_vertex_triangles(int n, const std::vector<int>& tris, std::vector<int>& off,
                            std::vector<int>& list);

}  // namespace chysx_b200
