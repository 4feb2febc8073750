// Drives include/nereus_b200_solver.hpp the way a NEREUS build would: one pressure step + projection on a MAC grid
// read from a case file, written back to a result file. Built and run by tests/test_gpu_cpp_shim.py.
//
// case:   int32 dim, Nx, Ny, Nz, nonUniform; double dh, rho, dt, tol; uint8 types[cells];
//         3 x (double width[N+2]); 3 x (double gap[N+1]); double u[], v[], w[] (3D), p[cells]
// result: int32 status, n, iters; double rel_res; double p[cells], u[], v[], w[]
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "nereus_b200_solver.hpp"

template <class T> static void Read(FILE *f, std::vector<T> &v, size_t n)
{
    v.resize(n);
    if (n && std::fread(v.data(), sizeof(T), n, f) != n) { std::fprintf(stderr, "short read\n"); std::exit(3); }
}

int main(int argc, char **argv)
{
    if (argc != 3) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t h[5];
    double d[4];
    if (std::fread(h, 4, 5, f) != 5 || std::fread(d, 8, 4, f) != 4) return 3;
    const int dim = h[0], Nx = h[1], Ny = h[2], Nz = h[3];
    const size_t cells = (size_t)Nx * Ny * Nz;
    std::vector<uint8_t> types;
    Read(f, types, cells);
    std::vector<double> w[3], g[3];
    const int N[3] = {Nx, Ny, dim == 3 ? Nz : 1};
    for (int a = 0; a < 3; a++) Read(f, w[a], N[a] + 2);
    for (int a = 0; a < 3; a++) Read(f, g[a], N[a] + 1);
    std::vector<double> u, v, ww, p;
    Read(f, u, (size_t)(Nx + 1) * Ny * Nz);
    Read(f, v, (size_t)Nx * (Ny + 1) * Nz);
    Read(f, ww, dim == 3 ? (size_t)Nx * Ny * (Nz + 1) : 0);
    Read(f, p, cells);
    std::fclose(f);

    nereus_b200::GridView gv;
    gv.dim = dim;
    gv.Nx = Nx;
    gv.Ny = Ny;
    gv.Nz = Nz;
    gv.nonUniform = h[4] != 0;
    gv.dh = d[0];
    gv.cellTypes = types.data();
    for (int a = 0; a < 3; a++) { gv.width[a] = w[a].data(); gv.gap[a] = g[a].data(); }
    gv.u = u.data();
    gv.v = v.data();
    gv.w = dim == 3 ? ww.data() : nullptr;
    gv.p = p.data();

    nb_result r{};
    try
    {
        nereus_b200::PressureSolver solver(NB_PRECISION_MIXED, 0);
        solver.InitializePressureSolver(gv);
        r = solver.SolvePressure(gv, d[1], d[2], false, d[3]);
        if (solver.LastIterations() != r.iters_inner) return 5;
    }
    catch (const nereus_b200::Error &e)
    {
        std::fprintf(stderr, "nereus_b200 error %d: %s\n", e.status, e.what());
        return 4;
    }
    FILE *o = std::fopen(argv[2], "wb");
    const int32_t oh[3] = {r.status, r.n, r.iters_inner};
    std::fwrite(oh, 4, 3, o);
    std::fwrite(&r.rel_res, 8, 1, o);
    std::fwrite(p.data(), 8, p.size(), o);
    std::fwrite(u.data(), 8, u.size(), o);
    std::fwrite(v.data(), 8, v.size(), o);
    std::fwrite(ww.data(), 8, ww.size(), o);
    std::fclose(o);
    return 0;
}
