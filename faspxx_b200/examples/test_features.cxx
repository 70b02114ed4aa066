// A driver in the reference's style for the B200 additions of the façade: a matrix-free
// operator (example/TestMatFree.cxx's 5-point Laplacian as a StencilLOP), MAT::Mult and
// MAT::Add, ReadMat of a MatrixMarket file, and CG preconditioned by MG with bilinear
// transfers and Galerkin coarse operators. Prints one line per check: name code value.
#include <cmath>
#include <cstdio>
#include <vector>

#include "faspxx_b200.hxx"

using namespace fasp_b200;

// 5-point Laplacian (4 on the diagonal, -1 off) on an n x n grid, x fastest
static MAT laplace2d(USI n)
{
    std::vector<USI> rp{0}, ci;
    std::vector<DBL> va;
    for (USI j = 0; j < n; ++j)
        for (USI i = 0; i < n; ++i) {
            const USI r = i + n * j;
            if (j > 0) ci.push_back(r - n), va.push_back(-1.0);
            if (i > 0) ci.push_back(r - 1), va.push_back(-1.0);
            ci.push_back(r), va.push_back(4.0);
            if (i + 1 < n) ci.push_back(r + 1), va.push_back(-1.0);
            if (j + 1 < n) ci.push_back(r + n), va.push_back(-1.0);
            rp.push_back((USI)ci.size());
        }
    return MAT(n * n, n * n, (USI)va.size(), va, ci, rp);
}

// bilinear prolongation from the ((nf-1)/2)^2 grid to nf^2
static MAT bilinear(USI nf)
{
    const USI nc = (nf - 1) / 2;
    auto one = [&](USI i, std::vector<std::pair<USI, DBL>>& t) {
        t.clear();
        if (i % 2 == 1) t.push_back({(i - 1) / 2, 1.0});
        else {
            if (i / 2 >= 1) t.push_back({i / 2 - 1, 0.5});
            if (i / 2 < nc) t.push_back({i / 2, 0.5});
        }
    };
    std::vector<USI> rp{0}, ci;
    std::vector<DBL> va;
    std::vector<std::pair<USI, DBL>> tx, ty;
    for (USI j = 0; j < nf; ++j)
        for (USI i = 0; i < nf; ++i) {
            one(i, tx);
            one(j, ty);
            for (auto& y : ty)
                for (auto& x : tx) ci.push_back(x.first + nc * y.first), va.push_back(x.second * y.second);
            rp.push_back((USI)ci.size());
        }
    return MAT(nf * nf, nc * nc, (USI)va.size(), va, ci, rp);
}

int main()
{
    // 1. the matrix-free example's operator and problem at dim 64 (TestMatFree.cxx)
    {
        const int dim = 64, d1 = dim - 1;
        StencilLOP A(d1, d1, 1, {0, -1, 0, 1, 0}, {-1, 0, 0, 0, 1}, {0, 0, 0, 0, 0},
                     {-1.0, -1.0, 4.0, -1.0, -1.0});
        const double pi = 3.14159265358979323846, h = 1.0 / dim;
        VEC b(d1 * d1, 0.0), x(d1 * d1, 0.25);
        for (int k = 1; k <= d1; ++k)
            for (int j = 1; j <= d1; ++j)
                b.values[(k - 1) * d1 + j - 1] =
                    h * h * (2 * pi * pi * std::sin(pi * k * h) * std::sin(pi * j * h));
        CG cg;
        cg.SetMaxIter(10000);
        cg.SetRestart(20);
        cg.SetAbsTol(1e-12);
        cg.SetRelTol(1e-8);
        Identity pcd;
        cg.SetupPCD(pcd);
        cg.Setup(A);
        const FaspRetCode code = cg.Solve(b, x);
        double err = 0.0;
        for (int j = 1; j <= d1; ++j)
            for (int k = 1; k <= d1; ++k) {
                const double e = x.values[(j - 1) * d1 + k - 1] - std::sin(pi * j * h) * std::sin(pi * k * h);
                err += e * e;
            }
        std::printf("matfree_cg %d %u %.4e\n", (int)code, cg.GetIterations(), std::sqrt(err * h * h));
    }
    // 2. MAT::Mult and MAT::Add
    {
        MAT A = laplace2d(6), C, S;
        C.Mult(A, A);
        S.Add(2.0, A, -1.0, A);
        std::printf("mult %d %u %u\n", C.Status(), C.GetNNZ(), C.GetRowSize());
        std::printf("add %d %u %u\n", S.Status(), S.GetNNZ(), S.GetRowSize());
        // MAT::MultTransposeAdd on the symmetric Laplacian: A^T 1 + 1 = A 1 + 1
        VEC ones(A.GetRowSize(), 1.0), out;
        DVEC d1(ones), d2(ones), dv(A.GetRowSize()), da(A.GetRowSize());
        A.MultTransposeAdd(d1, d2, dv);
        A.Apply(d1, da);
        da.AXPY(1.0, d2);
        da.AXPY(-1.0, dv);
        std::printf("mta %.3e %.3e\n", dv.Norm2(), da.NormInf());
    }
    // 3. ReadMat of a MatrixMarket file (unsorted triplets, 1-based)
    {
        const char* path = "features_tmp.mtx";
        if (FILE* f = std::fopen(path, "w")) {
            std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n3 3 5\n");
            std::fprintf(f, "3 3 2.0\n1 2 -1.0\n2 2 2.0\n1 1 2.0\n3 1 -1.0\n");
            std::fclose(f);
        }
        MAT M;
        const FaspRetCode code = ReadMat(path, M);
        std::remove(path);
        std::printf("readmat %d %u %u\n", (int)code, M.GetRowSize(), M.GetNNZ());
    }
    // 4. CG preconditioned by MG: bilinear transfers, Galerkin coarse operators on the GPU
    {
        const USI nf = 63;
        MAT A = laplace2d(nf), P0 = bilinear(63), P1 = bilinear(31), P2 = bilinear(15),
            P3 = bilinear(7);
        MG<MAT> mg;
        mg.SetNumLevels(4);
        mg.SetMaxIter(1);
        mg.SetMinIter(1);
        Jacobi smoother(2.0 / 3.0), coarse(2.0 / 3.0);
        smoother.SetMaxIter(2);
        smoother.SetMinIter(2);
        coarse.SetMaxIter(40);
        coarse.SetMinIter(40);
        mg.SetupLevel(A, 0, nullptr, smoother, coarse);
        mg.SetTransfer(0, P0);
        mg.SetTransfer(1, P1);
        mg.SetTransfer(2, P2);
        mg.SetTransfer(3, P3);
        CG cg;
        cg.SetMaxIter(200);
        cg.SetRelTol(1e-10);
        cg.SetAbsTol(0.0);
        cg.SetupPCD(mg);
        cg.Setup(A);
        VEC b(nf * nf, 1.0), x(nf * nf, 0.0);
        const FaspRetCode code = cg.Solve(b, x);
        std::printf("mg_pcg %d %u %.3e\n", (int)code, cg.GetIterations(), cg.GetNorm2());
    }
    return 0;
}
