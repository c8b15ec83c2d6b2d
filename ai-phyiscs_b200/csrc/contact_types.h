// Contact data passed to the step's kernels (see contact_kernels.cuh).
#pragma once

#include <cuda_runtime.h>

namespace chysx_b200 {

// One prepared contact, 64 B: the rows of its four slots (-1 when the
// weight is zero), the weights, the normal with k - alpha, and the
// per-unit-weight gradient -k depth n - alpha u_t with alpha.
struct __align__(16) PrepContact {
    int4 rows;
    float4 w;
    float4 nk;  // nx, ny, nz, k - alpha
    float4 ga;  // gradient xyz, alpha
};

// Per-row lists of the contact operator, built every step.
struct ContactOp {
    const int* __restrict__ off;  // [n + 1] row offsets into ent
    int* ent;                     // (contact << 2) | slot, sorted per row by the assembly kernel
    const PrepContact* __restrict__ rec;
    int active;
    int residual;  // the warm-start residual subtracts the off-diagonal part
};

// Static shapes: planes (n.xyz, d: 4 floats) then boxes (center, half
// extents, ex, ey, ez: 15 floats), and the contact parameters.
struct StaticContacts {
    const float* __restrict__ shapes;
    int n_planes, n_boxes;
    float thickness, k, mu, eps;
    int active;
};

// The caller's contact list as the step reads it.
struct ContactInput {
    const int4* __restrict__ pairs;
    const float4* __restrict__ weights;  // 2 float4 per contact
    const int* __restrict__ count;
    const float* __restrict__ stiffnesses;  // optional
    const float4* __restrict__ slips;       // optional: u_t xyz, |u_t|
    const int* __restrict__ ext_to_row;     // particle -> internal row (null: identity)
    int max_contacts;
    float stiffness, mu, eps;
};

constexpr int kScanChunk = 4096;  // rows per block of the contact-list scan

}  // namespace chysx_b200
