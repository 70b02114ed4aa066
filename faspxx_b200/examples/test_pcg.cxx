// test_pcg.cxx -- a FASP++ driver in the shape of example/TestPCG.cxx, switched to the B200
// backend by its includes: weighted-Jacobi (0.8) preconditioned CG on a 2D 5-point Poisson
// matrix, then the same system through Krylov() with BiCGStab, GMRES and FGMRES.
//   test_pcg [grid] [maxIter]      prints "<solver> <code> <iterations> <norm2>" per line
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "faspxx_b200.hxx"

using namespace fasp_b200;

static void poisson2d(USI m, std::vector<USI>& rp, std::vector<USI>& ci, std::vector<DBL>& va)
{
    const USI n = m * m;
    rp.assign(1, 0);
    for (USI i = 0; i < n; ++i) {
        const USI x = i % m, y = i / m;
        if (y > 0) { ci.push_back(i - m); va.push_back(-1.0); }
        if (x > 0) { ci.push_back(i - 1); va.push_back(-1.0); }
        ci.push_back(i); va.push_back(4.0);
        if (x + 1 < m) { ci.push_back(i + 1); va.push_back(-1.0); }
        if (y + 1 < m) { ci.push_back(i + m); va.push_back(-1.0); }
        rp.push_back((USI)ci.size());
    }
}

int main(int argc, char** argv)
{
    const USI m = argc > 1 ? (USI)std::atoi(argv[1]) : 64;
    const USI maxIter = argc > 2 ? (USI)std::atoi(argv[2]) : 2000;
    if (fasp_gpu_init(0) != 0) {
        std::printf("no sm_100 device\n");
        return 2;
    }
    std::vector<USI> rp, ci;
    std::vector<DBL> va;
    poisson2d(m, rp, ci, va);
    const USI n = m * m;
    MAT mat(n, n, (USI)ci.size(), va, ci, rp);
    if (mat.Status() != 0) return 3;

    VEC b(n, 1.0), x(n, 0.0);

    Jacobi pcd;                 // TestPCG.cxx:71-76
    pcd.SetWeight(0.8);
    pcd.SetMaxIter(1);
    pcd.SetMinIter(1);
    pcd.Setup(mat);

    CG solver;                  // TestPCG.cxx:79-88
    solver.SetMaxIter(maxIter);
    solver.SetMinIter(0);
    solver.SetRelTol(1e-8);
    solver.SetAbsTol(0.0);
    solver.SetupPCD(pcd);
    solver.Setup(mat);
    FaspRetCode code = solver.Solve(b, x);
    std::printf("pcg %d %u %.6e\n", (int)code, solver.GetIterations(), solver.GetNorm2());

    Identity id;                // TestKrylov.cxx:76
    for (const char* name : {"bicgstab", "gmres", "fgmres"}) {
        SOLParams p;
        p.algName = name;
        p.maxIter = maxIter;
        p.relTol = 1e-8;
        p.absTol = 0.0;
        VEC y(n, 0.0);
        code = Krylov(mat, b, y, id, p);
        double err = 0;
        for (USI i = 0; i < n; ++i) err = std::max(err, std::abs(y[i] - x[i]));
        std::printf("%s %d %.3e\n", name, (int)code, err);
    }
    return 0;
}
