// Host-side preparation of a U1 model (the argument list of
// sys_linmat_lindef_static) into per-patch device arrays, shared by the
// assembly and the shape-gradient kernels.
#pragma once
#include <vector>

#include "common.cuh"

namespace yeti {

struct U1Patch {
    int p[3] = {0, 0, 0};
    int nkv[3] = {0, 0, 0};
    int nn = 0;              // nodes per element
    int nq = 0;              // Gauss points per element (NBINT)
    int ng = 0;              // Gauss points per direction
    double E = 0, nu = 0, rho = 0;
    int64_t elem_begin = 0;  // global index (0-based) of the first element
    int64_t nelem = 0;
    int64_t nactive = 0;
    int64_t nb_data_elem = 0;
    std::vector<int64_t> act;   // global ids (0-based) of active elements
    std::vector<int64_t> slot;  // COO slot offset of each active element
    DevBuf knots;   // U_1 | U_2 | U_3
    DevBuf gauss;   // 4 * nq  (weight, t1, t2, t3)
    DevBuf ien;     // nactive * nn, int32 0-based CP index
    DevBuf w;       // nactive * nn element weights
    DevBuf span;    // nactive * 3, int32 1-based knot span
    DevBuf slotd;   // nactive, int64 slot offsets
    DevBuf gid;     // nactive, int32 global element ids
};

struct U1Model {
    std::vector<U1Patch> patches;
    DevBuf coords;           // 3 * nb_cp
    int64_t nb_cp = 0;
    int64_t nb_data = 0;     // slots needed (sum over active elements)
};

// Validate the model, compute slot offsets (compacted over active
// elements, build_system_elemStorage.f90:156-293) and upload the geometry.
int u1_prepare(yeti_ctx *ctx, const yeti_u1_model *m, U1Model &out);

// Element stiffness of one patch's active elements by the sum-factorised
// kernel (stiff_sf.cu), written into the COO slots of the pair kernel.
int launch_u1_stiffness_sf(yeti_ctx *ctx, const U1Patch &P, const double *coords,
                           double lam, double mu, double *kdata, int32_t *krow,
                           int32_t *kcol, size_t smem_cap);

}  // namespace yeti
