// ref_cuda_bench.cu -- measurement-only driver of the reference's own CUDA
// implementation: its classes and kernels (src/**/*.cu, compiled from the
// reference tree as it lies by oracle/build_oracle.py) run through the loop of
// src/main.cpp:319-357, timed with CUDA events.  It is the "reference CUDA
// build on the same B200" beside bench.py's numbers, never part of the
// product.  The set-up follows src/main.cpp:200-290 with the parameters given
// on the command line (the unit-conversion bookkeeping of main.cpp is left
// out): obstacle mask from a raw uint8 file (x fastest), BGK (obstacle
// bounce-back) or porous BGK, the NEQ velocity inlet and the pressure outlet,
// ADDirichlet(1) + ADNeumannOutlet, a uniform tau field, a Langmuir or linear
// LDF on the obstacle region, coupling on.
//
// Usage: ref_cuda_bench mask.bin nx ny nz steps warmup bgk|porous langmuir|linear
//                       tau tau_ad u_in a b k [fields.bin]
// (a, b, k: q_max, K_L, k for Langmuir; K_henry, -, k for linear).
// Prints one JSON line.  With fields.bin, also writes the fields after all
// warmup + steps steps as float64 arrays of N values each, in the order rho,
// ux, uy, uz, phi, q (the reference's own downloads: Lattice::downloadMacroscopic,
// ADLattice::downloadPhi, AdsorbedField::download), for the parity tests.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "boundary/ad/ADDirichlet.hpp"
#include "boundary/ad/ADNeumannOutlet.hpp"
#include "boundary/ns/PressureDirichlet.hpp"
#include "boundary/ns/VelocityDirichletNEQ.hpp"
#include "collision/ADBGKCollision.hpp"
#include "collision/BGKCollision.hpp"
#include "collision/PorousBGKCollision.hpp"
#include "core/descriptors/D3Q19.hpp"
#include "core/descriptors/D3Q7.hpp"
#include "core/helpers/helpers.hpp"
#include "core/lattice/ADLattice.hpp"
#include "core/lattice/NSLattice.hpp"
#include "reaction/AdsorbedField.hpp"
#include "reaction/LangmuirLDF.hpp"
#include "reaction/LinearLDF.hpp"

int main(int argc, char** argv)
{
    if (argc < 15) {
        std::fprintf(stderr, "usage: ref_cuda_bench mask nx ny nz steps warmup bgk|porous langmuir|linear "
                             "tau tau_ad u_in a b k\n");
        return 2;
    }
    const int nx = std::atoi(argv[2]), ny = std::atoi(argv[3]), nz = std::atoi(argv[4]);
    const int steps = std::atoi(argv[5]), warmup = std::atoi(argv[6]);
    const bool porous = std::string(argv[7]) == "porous";
    const bool langmuir = std::string(argv[8]) == "langmuir";
    const double tau = std::atof(argv[9]), tau_ad = std::atof(argv[10]), u_in = std::atof(argv[11]);
    const double ia = std::atof(argv[12]), ib = std::atof(argv[13]), ik = std::atof(argv[14]);
    const int n = nx * ny * nz;
    std::vector<std::uint8_t> mask((size_t)n);
    {
        FILE* f = std::fopen(argv[1], "rb");
        if (!f || std::fread(mask.data(), 1, mask.size(), f) != mask.size()) {
            std::fprintf(stderr, "cannot read %s\n", argv[1]);
            return 2;
        }
        std::fclose(f);
    }
    try {
        // the lattice velocity and weight tables in __constant__ memory, as
        // src/main.cpp:127-128 uploads them before any lattice is built
        uploadD3Q19Constants();
        uploadD3Q7Constants();
        LBMParams p{};
        p.Nx = nx; p.Ny = ny; p.Nz = nz;
        p.rho0 = DATA_TYPE(1); p.tau = DATA_TYPE(tau); p.tau_ad = DATA_TYPE(tau_ad); p.phi0 = DATA_TYPE(0);
        p.periodicX = false; p.periodicY = true; p.periodicZ = true;
        p.enableAdsorption = true;
        p.qMax = DATA_TYPE(ia); p.bLangmuir = DATA_TYPE(ib); p.kLDF = DATA_TYPE(ik);
        p.KHenry = DATA_TYPE(ia); p.kA = DATA_TYPE(ik);

        Lattice<D3Q19> NS(p);
        ADLattice<D3Q7> AD(p);
        if (porous) NS.setCollisionOperator(std::make_shared<PorousBGKCollision<D3Q19>>(p));
        else NS.setCollisionOperator(std::make_shared<BGKCollision<D3Q19>>(p));
        AD.setCollisionOperator(std::make_shared<ADBGKCollision<D3Q7>>(p));
        auto inlet = buildXPlaneMask(nx, ny, nz, 0);
        auto outlet = buildXPlaneMask(nx, ny, nz, nx - 1);
        NS.setObstacleMask(mask);
        if (porous) NS.setPorosityFromMask(mask, DATA_TYPE(0.67), DATA_TYPE(1.0));
        NS.addBoundary<VelocityDirichletNEQ<D3Q19>>(p, inlet, DATA_TYPE(u_in), DATA_TYPE(0), DATA_TYPE(0));
        NS.addBoundary<PressureDirichlet<D3Q19>>(p, outlet, p.rho0);
        AD.setTauField(std::vector<DATA_TYPE>((size_t)n, DATA_TYPE(tau_ad)));
        AdsorbedField q(p);
        LinearLDF<D3Q7> lin(p);
        LangmuirLDF<D3Q7> lang(p);
        AD.addBoundary<ADDirichlet<D3Q7>>(p, inlet, DATA_TYPE(1.0));
        AD.addBoundary<ADNeumannOutlet<D3Q7>>(p, outlet);
        NS.initEquilibrium();
        AD.initEquilibrium();

        auto body = [&](int s) {   // src/main.cpp:321-336
            NS.step(s);
            NS.computeMacroscopicDevice();
            AD.setAdvectionFromFluidDevice(NS);
            AD.zeroSource();
            if (langmuir) lang.computeSource(AD, q, NS.d_obstacle_ptr());
            else lin.computeSource(AD, q, NS.d_obstacle_ptr());
            AD.step(s);
        };
        int s = 1;
        for (; s <= warmup; ++s) body(s);
        cudaDeviceSynchronize();
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        for (int i = 0; i < steps; ++i, ++s) body(s);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        AD.downloadPhi();
        double cout = 0.0;
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y) cout += (double)AD.phiHost()[(size_t)(nx - 1) + (size_t)nx * (y + (size_t)ny * z)];
        cout /= (double)ny * nz;
        if (argc > 15) {
            NS.downloadMacroscopic();
            q.download();
            FILE* fo = std::fopen(argv[15], "wb");
            if (!fo) {
                std::fprintf(stderr, "cannot write %s\n", argv[15]);
                return 2;
            }
            const std::vector<DATA_TYPE>* fields[6] = {&NS.rhoHost(), &NS.uxHost(), &NS.uyHost(), &NS.uzHost(),
                                                       &AD.phiHost(), &q.host()};
            std::vector<double> buf((size_t)n);
            for (const std::vector<DATA_TYPE>* v : fields) {
                for (size_t i = 0; i < (size_t)n; ++i) buf[i] = (double)(*v)[i];
                std::fwrite(buf.data(), sizeof(double), buf.size(), fo);
            }
            std::fclose(fo);
        }
        std::printf("{\"impl\": \"reference-cuda\", \"precision\": \"%s\", \"cells\": %d, \"steps\": %d, "
                    "\"warmup\": %d, \"ms_per_step\": %.6f, \"mlups\": %.3f, \"c_out\": %.9g}\n",
                    sizeof(DATA_TYPE) == 8 ? "f64" : "f32", n, steps, warmup, ms / steps,
                    (double)n * steps / (ms / 1e3) / 1e6, cout);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "reference error: %s\n", e.what());
        return 1;
    }
    return 0;
}
