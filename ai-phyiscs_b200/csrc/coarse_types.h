// Coarse level of the two-level preconditioner: limits and the arguments
// shared by the coarse kernels and the register-resident PCG kernel.
#pragma once

namespace chysx_b200 {

constexpr int kCoarseMaxBlocks = 160;  // CTAs of a two-level plan (one warp's slot pass)
constexpr int kCoarseMaxNbr = 16;      // coarse blocks one block's rows touch, itself included
// The streamed kernel's coarse level (systems too large for the register-
// resident kernel): coarse blocks of about kCoarseStreamRows rows, at most
// kCoarseDenseMax unknowns, A_c inverted densely once per step.  Measured
// on the 1024 x 1024 configuration (10 steps): blocks of 3, 2 and 5 CTAs
// (~5,300, ~3,500 and ~8,900 rows) took 1,383, 1,269 and 1,662 iterations
// per step at 124, 131 and 119 us per iteration with 7.6, 19.4 and 3.7 ms of
// coarse set-up: 5.59, 5.37 and 4.95 steps/s
constexpr int kCoarseStreamRows = 5120;
constexpr int kCoarseDenseMax = 2560;
constexpr int kCoarseInvertThreads = 256;
// CTAs per coarse block of the register-resident kernel's level (1,024 rows
// at 512 rows per CTA).  Measured on the 256 x 256 configuration: 2-CTA
// blocks (768 unknowns) take 253 iterations per step against 325 with 4-CTA
// blocks (384 unknowns) and 376 with 8-CTA blocks, for a dearer inverse
// (0.95 against 0.50 ms of set-up per step) and a dearer coarse row per CTA
// (14.5 against 13.6 us per iteration): 216 against 202 steps/s
constexpr int kCoarseResidentCtas = 2;
// The coarse assembly splits a block's slices over CTAs of about
// kCoarseSplitSlices slices each (at most kCoarseMaxSplits per block): each
// slice costs dependent L2 round trips, so one CTA per block would walk a
// 2048-row block's 64 slices one after another
constexpr int kCoarseSplitSlices = 8;
constexpr int kCoarseMaxSplits = 32;
// Relative diagonal shift of the streamed kernel's coarse matrix: A_c +
// shift diag(A_c) is inverted instead of A_c (the resident kernel's coarse
// matrix, on smaller blocks, is inverted unshifted).  The coarse matrix of a flat,
// unstretched cloth (the first step from rest) has out-of-plane modes held
// only by inertia, with a scaled condition number ~1e7 on the 1024 x 1024
// grid; an FP32 inverse and FP32 restrictions of such a matrix are not a
// usable preconditioner (the solve stalls).  The shift bounds the scaled
// condition number near 3e5 and still leaves an SPD coarse correction.
constexpr double kCoarseShift = 1.0e-5;
// The streamed kernel's coarse level for batches: at most this many coarse
// blocks per instance (each an instance's rows in one CTA, or a run of such
// segments), so an instance's dense inverse has at most 144 unknowns.
constexpr int kBatchMaxBlocks = 12;

// Coarse space: coarse block B is the rows of CTAs [B G, (B + 1) G) of the
// plan; its fields are the translation (weight 1) and, with nq = 4, the
// linear fields s_a = (x_i - c_B).u_a / sd_a along the principal axes u_a of
// the block's positions (variance sd_a^2 per row; axes below 1e-6 of the
// largest variance get weight 0), each times e_x, e_y, e_z: U = 3 nq coarse
// unknowns per block, m = U nb in all, A_c = R^T A R.
struct CoarseArgs {
    int on = 0;
    int nb = 0;                               // coarse blocks
    int g = 1;                                // CTAs per coarse block
    int nq = 1;                               // fields per coarse block (1 or 4)
    int m = 0;                                // coarse unknowns, 3 nq nb
    int max_nbr = 0;                          // block entries per block row of A_c
    const int* slice_cb = nullptr;            // [n_slices] coarse block of every slice
    const int* cb_row0 = nullptr;             // [nb + 1] first internal row of every coarse block
    const int* nbr = nullptr;                 // [nb][max_nbr] sorted column blocks (-1 padded)
    const int* nbr_cnt = nullptr;             // [nb]
    const int* self_idx = nullptr;            // [nb] position of the block itself in its list
    const unsigned char* ell_nbr = nullptr;   // [ELL entries] list position of the entry's column block
    float4* w = nullptr;                      // [rows] linear-field weights s_1, s_2, s_3 (nq = 4)
    float* ac = nullptr;                      // [nb][max_nbr][U][U] A_c, row-major U x U blocks
    // the assembly's partial sums: a block's slices are split over `splits`
    // CTAs (slice s to split (s - first) % splits), each writing its sums
    // in double to acp[split][nb][max_nbr][U][U]; the inversion adds the
    // splits in order and rounds once into ac
    double* acp = nullptr;
    int splits = 1;
    float* ainv = nullptr;                    // [m][m] A_c^-1 (row-major)
    // A_c^-1 is formed by coarse_invert_kernel in the FP64 workspace
    // (padded m * m + m + 2048 doubles) from A_c + shift diag(A_c); fail != 0
    // after a step whose inversion met a non-positive pivot or a failed wait
    // (the coarse level then adds nothing in that step's solve); dense = 1:
    // the streamed kernel's level (its CTAs read their rows from L2)
    int dense = 0;
    // batched = 1: the streamed kernel's level for several instances.  Its
    // coarse blocks are runs of an instance's segment slots (the rows one
    // CTA holds of it), at most kBatchMaxBlocks per instance, so A_c is
    // block-diagonal by instance; ainv holds each instance's dense inverse
    // (m_b x m_b, m_b = U x its blocks) at inst_aoff[b]
    int batched = 0;
    const int* blk_slot = nullptr;            // [nb + 1] first segment slot of every coarse block
    const int* inst_blk = nullptr;            // [n_inst + 1] first coarse block of every instance
    const int* inst_aoff = nullptr;           // [n_inst + 1] offset of every instance's inverse in ainv
    const int* slot_cb = nullptr;             // [n_slots] coarse block of every segment slot
    double shift = 0.0;
    double* work = nullptr;
    int* fail = nullptr;
};

}  // namespace chysx_b200
