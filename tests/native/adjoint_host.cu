// adjoint_host.cu — host-side entry points to the pointwise forward and
// reverse-mode physics (physics.cuh, adjoint_physics.cuh), so the CPU tests
// can compare each reverse-mode function with torch autograd of the same
// forward formula.  Test-only: built by tests/test_adjoint_pointwise.py.
#include <cstring>

#include "../../prandtl_b200/csrc/adjoint_physics.cuh"

using namespace pdg;

namespace {
template <int DIM> Prim<DIM> prim(const double *s, double gamma) { return make_prim<DIM>(s, gamma, gamma - 1.0); }

template <int DIM> void vol(double gamma, const double *sa, const double *sb, int dir, double metric, double *F)
{
    volume_flux_rt<DIM>(prim<DIM>(sa, gamma), prim<DIM>(sb, gamma), dir, metric, 1.0 / (gamma - 1.0), F);
}
template <int DIM>
void vol_vjp(double gamma, const double *sa, const double *sb, int dir, double metric, const double *Fb, double *ga,
             double *gb)
{
    PBar<DIM> a, b;
    pbar_zero(a);
    pbar_zero(b);
    volume_flux_vjp<DIM>(prim<DIM>(sa, gamma), prim<DIM>(sb, gamma), dir, metric, 1.0 / (gamma - 1.0), Fb, a, b);
    std::memset(ga, 0, sizeof(double) * (DIM + 2));
    std::memset(gb, 0, sizeof(double) * (DIM + 2));
    pbar_to_cons<DIM>(sa, a, nullptr, gamma - 1.0, ga);
    pbar_to_cons<DIM>(sb, b, nullptr, gamma - 1.0, gb);
}
template <int DIM, int D>
void face_d(double gamma, double diss, const double *sa, const double *sb, double nrm, double *F)
{
    face_flux<DIM, D>(prim<DIM>(sa, gamma), prim<DIM>(sb, gamma), sa + 1, sb + 1, nrm, 1.0 / (gamma - 1.0), false,
                      diss, F);
}
template <int DIM>
void face_vjp(double gamma, double diss, const double *sa, const double *sb, int dir, double nrm, const double *Fb,
              double *ga, double *gb)
{
    PBar<DIM> a, b;
    pbar_zero(a);
    pbar_zero(b);
    double ma[DIM] = {0}, mb[DIM] = {0};
    face_flux_vjp<DIM>(prim<DIM>(sa, gamma), prim<DIM>(sb, gamma), sa + 1, sb + 1, dir, nrm, gamma,
                       1.0 / (gamma - 1.0), diss, Fb, a, b, ma, mb);
    std::memset(ga, 0, sizeof(double) * (DIM + 2));
    std::memset(gb, 0, sizeof(double) * (DIM + 2));
    pbar_to_cons<DIM>(sa, a, ma, gamma - 1.0, ga);
    pbar_to_cons<DIM>(sb, b, mb, gamma - 1.0, gb);
}
template <int DIM> struct GradView {
    const double *dq;
    PDG_FN double operator()(int d, int v) const { return dq[d * (DIM + 2) + v]; }
};
template <int DIM> void visc(double gamma, double mu, double lk, const double *s, const double *dq, double *cols)
{
    const Prim<DIM> q = prim<DIM>(s, gamma);
    const GradView<DIM> G{dq};
    for (int d = 0; d < DIM; d++) viscous_col<DIM>(q, G, d, 1.0 / (gamma - 1.0), mu, lk, cols + d * (DIM + 1));
}
template <int DIM>
void visc_vjp(double gamma, double mu, double lk, const double *s, const double *dq, const double *cb, double *sb,
              double *dqb)
{
    const Prim<DIM> q = prim<DIM>(s, gamma);
    double G[DIM][DIM + 2], gb[DIM][DIM + 2];
    for (int d = 0; d < DIM; d++)
        for (int v = 0; v < DIM + 2; v++) {
            G[d][v] = dq[d * (DIM + 2) + v];
            gb[d][v] = 0.0;
        }
    PBar<DIM> qb;
    pbar_zero(qb);
    for (int d = 0; d < DIM; d++)
        viscous_col_vjp<DIM>(q, G, d, 1.0 / (gamma - 1.0), mu, lk, cb + d * (DIM + 1), qb, gb);
    std::memset(sb, 0, sizeof(double) * (DIM + 2));
    pbar_to_cons<DIM>(s, qb, nullptr, gamma - 1.0, sb);
    for (int d = 0; d < DIM; d++)
        for (int v = 0; v < DIM + 2; v++) dqb[d * (DIM + 2) + v] = gb[d][v];
}
}  // namespace

extern "C" {
void h_volume_flux(int dim, double gamma, const double *sa, const double *sb, int dir, double metric, double *F)
{
    if (dim == 2) vol<2>(gamma, sa, sb, dir, metric, F);
    else vol<3>(gamma, sa, sb, dir, metric, F);
}
void h_volume_flux_vjp(int dim, double gamma, const double *sa, const double *sb, int dir, double metric,
                       const double *Fb, double *ga, double *gb)
{
    if (dim == 2) vol_vjp<2>(gamma, sa, sb, dir, metric, Fb, ga, gb);
    else vol_vjp<3>(gamma, sa, sb, dir, metric, Fb, ga, gb);
}
void h_face_flux(int dim, double gamma, double diss, const double *sa, const double *sb, int dir, double nrm,
                 double *F)
{
    if (dim == 2) {
        if (dir == 0) face_d<2, 0>(gamma, diss, sa, sb, nrm, F);
        else face_d<2, 1>(gamma, diss, sa, sb, nrm, F);
    } else {
        if (dir == 0) face_d<3, 0>(gamma, diss, sa, sb, nrm, F);
        else if (dir == 1) face_d<3, 1>(gamma, diss, sa, sb, nrm, F);
        else face_d<3, 2>(gamma, diss, sa, sb, nrm, F);
    }
}
void h_face_flux_vjp(int dim, double gamma, double diss, const double *sa, const double *sb, int dir, double nrm,
                     const double *Fb, double *ga, double *gb)
{
    if (dim == 2) face_vjp<2>(gamma, diss, sa, sb, dir, nrm, Fb, ga, gb);
    else face_vjp<3>(gamma, diss, sa, sb, dir, nrm, Fb, ga, gb);
}
void h_entropy_vars(int dim, double gamma, const double *s, double *w)
{
    const double gm1 = gamma - 1.0;
    if (dim == 2) entropy_vars<2>(s, gamma, gm1, 1.0 / gm1, w);
    else entropy_vars<3>(s, gamma, gm1, 1.0 / gm1, w);
}
void h_entropy_vars_vjp(int dim, double gamma, const double *s, const double *wb, double *sb)
{
    const double gm1 = gamma - 1.0;
    std::memset(sb, 0, sizeof(double) * (dim + 2));
    if (dim == 2) entropy_vars_vjp<2>(s, wb, gamma, gm1, 1.0 / gm1, sb);
    else entropy_vars_vjp<3>(s, wb, gamma, gm1, 1.0 / gm1, sb);
}
void h_entgrad(int dim, double gamma, const double *s, double *g)
{
    const double gm1 = gamma - 1.0;
    if (dim == 2) entgrad_to_primgrad<2>(s, gm1, 1.0 / gm1, false, g);
    else entgrad_to_primgrad<3>(s, gm1, 1.0 / gm1, false, g);
}
void h_entgrad_vjp(int dim, double gamma, const double *s, const double *g, const double *ob, double *gb, double *sb)
{
    const double gm1 = gamma - 1.0;
    std::memset(sb, 0, sizeof(double) * (dim + 2));
    if (dim == 2) entgrad_vjp<2>(s, g, ob, gm1, 1.0 / gm1, gb, sb);
    else entgrad_vjp<3>(s, g, ob, gm1, 1.0 / gm1, gb, sb);
}
void h_viscous_cols(int dim, double gamma, double mu, double lk, const double *s, const double *dq, double *cols)
{
    if (dim == 2) visc<2>(gamma, mu, lk, s, dq, cols);
    else visc<3>(gamma, mu, lk, s, dq, cols);
}
void h_viscous_cols_vjp(int dim, double gamma, double mu, double lk, const double *s, const double *dq,
                        const double *cb, double *sb, double *dqb)
{
    if (dim == 2) visc_vjp<2>(gamma, mu, lk, s, dq, cb, sb, dqb);
    else visc_vjp<3>(gamma, mu, lk, s, dq, cb, sb, dqb);
}
}
