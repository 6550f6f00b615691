// prandtl_b200_mfem.hpp — header-only adapter that plugs the B200 operator
// into an MFEM time loop in place of Prandtl's CPU DGSEMOperator.
//
//   Prandtl                                      this adapter
//   DGSEMOperator : TimeDependentOperator        GpuDGSEMOperator : TimeDependentOperator
//     (src/Operators/DGSEMOperator.hpp:15)         Mult -> pdg_rhs_host
//   RK3SSPSolver (Simulation.cpp:186-188, 1010)  GpuRK3SSPSolver : ODESolver
//                                                  Step -> pdg_rk3_step_host (three fused stages)
//
// Vectors are MFEM host vectors in Ordering::byNODES (Simulation.hpp:64), as
// the reference passes them.  Errors are thrown as std::runtime_error with the
// library's message (the reference aborts through MFEM_ABORT instead).
#ifndef PRANDTL_B200_MFEM_HPP
#define PRANDTL_B200_MFEM_HPP

#include <stdexcept>
#include <string>

#include "prandtl_b200.h"

namespace prandtl_b200 {

inline void check_status(int code, pdg_ctx *ctx, const char *what)
{
    if (code != PDG_OK) {
        std::string msg = std::string(what) + " failed (status " + std::to_string(code) + ")";
        if (ctx) msg += std::string(": ") + pdg_last_error(ctx);
        throw std::runtime_error(msg);
    }
}

inline pdg_ctx *create_context(const pdg_mesh &mesh, const pdg_params &params)
{
    pdg_ctx *ctx = nullptr;
    check_status(pdg_create(&mesh, &params, &ctx), nullptr, "pdg_create");
    return ctx;
}

class GpuDGSEMOperator : public mfem::TimeDependentOperator {
public:
    GpuDGSEMOperator(const pdg_mesh &mesh, const pdg_params &params)
        : GpuDGSEMOperator(create_context(mesh, params))
    {
    }
    ~GpuDGSEMOperator() override { pdg_destroy(ctx_); }
    GpuDGSEMOperator(const GpuDGSEMOperator &) = delete;
    GpuDGSEMOperator &operator=(const GpuDGSEMOperator &) = delete;

    // DGSEMOperator::Mult (DGSEMOperator.cpp:537-591), host vectors
    void Mult(const mfem::Vector &u, mfem::Vector &dudt) const override
    {
        if (u.Size() != Height() || dudt.Size() != Height()) throw std::runtime_error("GpuDGSEMOperator::Mult: size");
        check_status(pdg_rhs_host(ctx_, u.GetData(), dudt.GetData()), ctx_, "pdg_rhs_host");
    }
    // DGSEMOperator::GetMaxCharSpeed (DGSEMOperator.hpp:106-109)
    double GetMaxCharSpeed() const
    {
        double lam = 0.0;
        check_status(pdg_max_char_speed(ctx_, &lam), ctx_, "pdg_max_char_speed");
        return lam;
    }
    // DGSEMOperator::AddBdrFaceIntegrator (DGSEMOperator.cpp:593) for the
    // faces marked -1 - index in the neighbour table; `data` as
    // pdg_set_boundary takes it (may be empty for types without data)
    void SetBoundary(int index, int type, const mfem::Vector &data)
    {
        check_status(pdg_set_boundary(ctx_, index, type, data.Size() ? data.GetData() : nullptr), ctx_,
                     "pdg_set_boundary");
    }
    // The mesh's general geometry (skewed, graded, curved or unstructured
    // elements): `nodes` holds the DG nodes' coordinates in the state's
    // byNODES layout (dim components; e.g. an L2 Gauss-Lobatto vector space
    // of the operator's order with the identity projected onto it),
    // `face_orient` one code per element face as pdg_set_geometry takes them
    // (null: opposite faces, aligned axes).  Euler only; before the first Mult.
    void SetGeometry(const mfem::Vector &nodes, const int32_t *face_orient)
    {
        check_status(pdg_set_geometry(ctx_, nodes.GetData(), face_orient), ctx_, "pdg_set_geometry");
    }
    pdg_ctx *context() const { return ctx_; }

private:
    explicit GpuDGSEMOperator(pdg_ctx *ctx) : mfem::TimeDependentOperator((int)pdg_size(ctx)), ctx_(ctx) {}
    pdg_ctx *ctx_;
};

// MFEM's RK3SSPSolver with each stage's right-hand side fused into its axpy.
class GpuRK3SSPSolver : public mfem::ODESolver {
public:
    void Init(mfem::TimeDependentOperator &f) override
    {
        mfem::ODESolver::Init(f);
        op_ = dynamic_cast<GpuDGSEMOperator *>(&f);
        if (!op_) throw std::runtime_error("GpuRK3SSPSolver needs a GpuDGSEMOperator");
    }
    void Step(mfem::Vector &x, double &t, double &dt) override
    {
        check_status(pdg_rk3_step_host(op_->context(), dt, x.GetData()), op_->context(), "pdg_rk3_step_host");
        t += dt;
    }

private:
    GpuDGSEMOperator *op_ = nullptr;
};

}  // namespace prandtl_b200

#endif
