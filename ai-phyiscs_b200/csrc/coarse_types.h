// Coarse level of the two-level preconditioner: limits and the arguments
// shared by the coarse kernels and the register-resident PCG kernel.
#pragma once

namespace chysx_b200 {

constexpr int kCoarseMaxBlocks = 160;  // CTAs of a two-level plan (one warp's slot pass)
constexpr int kCoarseMaxNbr = 16;      // coarse blocks one block's rows touch, itself included
constexpr int kCoarseThreads = 512;    // threads of the coarse direct solve; also the bound on the coarse unknowns
constexpr int kCoarseMaxRhs = 4;       // rows of A_c^-1 one CTA computes

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
    int rpc = 0;                              // rows of A_c^-1 per CTA (ceil(m / CTAs))
    int max_nbr = 0;                          // block entries per block row of A_c
    const int* slice_cb = nullptr;            // [n_slices] coarse block of every slice
    const int* cb_row0 = nullptr;             // [nb + 1] first internal row of every coarse block
    const int* nbr = nullptr;                 // [nb][max_nbr] sorted column blocks (-1 padded)
    const int* nbr_cnt = nullptr;             // [nb]
    const int* self_idx = nullptr;            // [nb] position of the block itself in its list
    const unsigned char* ell_nbr = nullptr;   // [ELL entries] list position of the entry's column block
    const int* perm = nullptr;                // [nb] band position of every block (reverse Cuthill-McKee)
    int bw = 0;                               // band half-width of A_c in unknowns, block order perm
    float4* w = nullptr;                      // [rows] linear-field weights s_1, s_2, s_3 (nq = 4)
    float* ac = nullptr;                      // [nb][max_nbr][U][U] A_c, row-major U x U blocks
    float* ainv = nullptr;                    // [m][m] rows of A_c^-1 (rows r..r+rpc by CTA r / rpc)
};

}  // namespace chysx_b200
