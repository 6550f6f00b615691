// Compiles the MFEM adapter against the mock and exercises its error path:
// without a GPU, constructing the operator must throw with the library's
// status instead of aborting.
#include <cstdio>
#include <vector>

#include "mfem_mock.hpp"
#include "prandtl_b200_mfem.hpp"

int main()
{
    pdg_params p;
    pdg_default_params(&p);
    std::vector<int32_t> nbr(4 * 2, 0);
    pdg_mesh m{2, 3, 2, {1.0, 1.0, 1.0}, nbr.data()};
    for (int e = 0; e < 2; e++) {
        nbr[e * 4 + 0] = nbr[e * 4 + 1] = 1 - e;
        nbr[e * 4 + 2] = nbr[e * 4 + 3] = e;
    }
    try {
        prandtl_b200::GpuDGSEMOperator op(m, p);
        double pout[1] = {2.0};
        mfem::Vector bdata(pout, 1);
        op.SetBoundary(0, PDG_BC_SUBSONIC_OUTFLOW_P, bdata);  // compiles the boundary setter
        prandtl_b200::GpuRK3SSPSolver ode;
        ode.Init(op);
        std::printf("constructed %d\n", op.Height());
    } catch (const std::exception &e) {
        std::printf("error: %s\n", e.what());
    }
    return 0;
}
