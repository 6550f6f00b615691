// Drives the MFEM adapter (include/prandtl_b200_mfem.hpp) on a GPU the way
// the reference's time loop drives its operator: GpuDGSEMOperator::Mult on
// host vectors (the initial-dt probe, Simulation.cpp:903) and
// GpuRK3SSPSolver::Step (Simulation.cpp:1010), here twice.
//
// Input file (binary): int32 dim, order, parabolic, compat; int64 ne;
// double h[3], mu, Pr, dt; int32 nbr[ne * 2 * dim]; double u[size].
// Output file: double dudt[size], double lam, double t, double x[size]
// (the state after two steps).
#include <cstdint>
#include <cstdio>
#include <vector>

#include "mfem_mock.hpp"
#include "prandtl_b200_mfem.hpp"

namespace {
template <typename T> bool get(std::FILE *f, T *p, size_t n) { return std::fread(p, sizeof(T), n, f) == n; }
}  // namespace

int main(int argc, char **argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s input output\n", argv[0]);
        return 2;
    }
    std::FILE *in = std::fopen(argv[1], "rb");
    if (!in) return 2;
    int32_t hdr[4];
    int64_t ne = 0;
    double h[3], mu, Pr, dt;
    if (!get(in, hdr, 4) || !get(in, &ne, 1) || !get(in, h, 3) || !get(in, &mu, 1) || !get(in, &Pr, 1) ||
        !get(in, &dt, 1))
        return 3;
    const int dim = hdr[0], order = hdr[1];
    std::vector<int32_t> nbr((size_t)ne * 2 * dim);
    if (!get(in, nbr.data(), nbr.size())) return 3;
    int64_t ndof = 1;
    for (int d = 0; d < dim; d++) ndof *= order + 1;
    const int64_t size = ne * ndof * (dim + 2);
    std::vector<double> u((size_t)size), dudt((size_t)size, 0.0);
    if (!get(in, u.data(), u.size())) return 3;
    std::fclose(in);

    pdg_params p;
    pdg_default_params(&p);
    p.parabolic = hdr[2];
    p.compat = hdr[3];
    p.mu = mu;
    p.Pr = Pr;
    pdg_mesh m{dim, order, ne, {h[0], h[1], h[2]}, nbr.data()};
    try {
        prandtl_b200::GpuDGSEMOperator op(m, p);
        if (op.Height() != size) {
            std::fprintf(stderr, "height %d, expected %lld\n", op.Height(), (long long)size);
            return 4;
        }
        mfem::Vector U(u.data(), (int)size), K(dudt.data(), (int)size);
        op.Mult(U, K);
        const double lam = op.GetMaxCharSpeed();
        prandtl_b200::GpuRK3SSPSolver ode;
        ode.Init(op);
        double t = 0.0;
        ode.Step(U, t, dt);
        ode.Step(U, t, dt);
        std::FILE *out = std::fopen(argv[2], "wb");
        if (!out) return 2;
        std::fwrite(dudt.data(), sizeof(double), dudt.size(), out);
        std::fwrite(&lam, sizeof(double), 1, out);
        std::fwrite(&t, sizeof(double), 1, out);
        std::fwrite(u.data(), sizeof(double), u.size(), out);
        std::fclose(out);
        std::printf("ok %lld\n", (long long)size);
    } catch (const std::exception &e) {
        std::printf("error: %s\n", e.what());
        return 5;
    }
    return 0;
}
