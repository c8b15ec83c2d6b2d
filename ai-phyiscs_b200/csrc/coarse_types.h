// Coarse level of the two-level preconditioner: limits and the arguments
// shared by the coarse kernels and the register-resident PCG kernel.
#pragma once

namespace chysx_b200 {

constexpr int kCoarseMaxBlocks = 160;  // CTAs (3 unknowns each) of a two-level plan
constexpr int kCoarseMaxNbr = 16;      // blocks one block's rows touch, itself included
constexpr int kCoarseThreads = 512;    // >= 3 * kCoarseMaxBlocks: one thread per coarse unknown
constexpr int kCoarseMaxIts = 1000;    // CG iterations for the rows of A_c^-1 (bounded)
constexpr double kCoarseTol = 1e-6;    // relative residual of those solves

struct CoarseArgs {
    int on = 0;
    int nb = 0;                               // blocks (= CTAs of the plan)
    int max_nbr = 0;                          // entries per block row of A_c
    const int* slice_cta = nullptr;           // [n_slices] CTA (block) of every slice
    const int* nbr = nullptr;                 // [nb][max_nbr] sorted column blocks (-1 padded)
    const int* nbr_cnt = nullptr;             // [nb]
    const int* self_idx = nullptr;            // [nb] position of the block itself in its list
    const unsigned char* ell_nbr = nullptr;   // [ELL entries] list position of the entry's column block
    float* ac = nullptr;                      // [nb][max_nbr][9] A_c = R^T A R, row-major 3x3 blocks
    float* ainv = nullptr;                    // [3 nb][3 nb] rows of A_c^-1 (row 3B + c by CTA B)
};

}  // namespace chysx_b200
