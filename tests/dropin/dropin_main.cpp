// The reference's set-up and time loop (src/main.cpp:131-357) written against
// include/fm_dropin.hpp: geometry from geometry.vti, BGK NS with the NEQ
// inlet and the pressure outlet, ADDirichlet + ADNeumannOutlet, a uniform tau
// field, the linear LDF on the obstacle region, coupling on, the outlet CSV, and
// one boundary of each lattice written against the reference's interface that
// counts the apply() calls it gets.
// Usage: dropin_main <dir> <steps> <csvEvery> [f32]; writes <dir>/outlet.csv
// and <dir>/fields.bin (rho, ux, uy, uz, phi, q as float64, N each).
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "fm_dropin.hpp"

using namespace fm_dropin;

struct UnitConverter {
    double dt;
    double timeLatticeToPhys(int step) const { return dt * step; }
};

// A boundary written against the reference's interface
// (include/core/interfaces/{NS,AD}Interfaces.hpp): it only counts the calls
// the lattices make, per phase, and checks the step index it is given.
template <typename LatticeT, typename Base>
struct CountingBoundary : Base {
    int pre = 0, post = 0, bad_step = 0, last = 0;
    void apply(LatticeT&, BoundaryPhase phase, int step) override
    {
        if (phase == BoundaryPhase::PreCollision) {
            ++pre;
            if (step != last + 1) ++bad_step;
            last = step;
        } else {
            ++post;
            if (step != last) ++bad_step;
        }
    }
};
using NSCount = CountingBoundary<Lattice<D3Q19>, NSBoundaryCondition<D3Q19>>;
using ADCount = CountingBoundary<ADLattice<D3Q7>, ADBoundaryCondition<D3Q7>>;

int main(int argc, char** argv)
{
    if (argc < 4) return 2;
    const std::string dir = argv[1];
    const int steps = std::atoi(argv[2]);
    const int csvEvery = std::atoi(argv[3]);
    if (argc > 4 && std::string(argv[4]) == "f32") set_precision(FM_F32);
    try {
        VTIResult geom = readVTI(dir + "/geometry.vti", 0.5);
        LBMParams p{};
        p.Nx = geom.Nx; p.Ny = geom.Ny; p.Nz = geom.Nz;
        p.rho0 = 1.0; p.tau = 0.8; p.tau_ad = 0.7; p.phi0 = 0.0;
        p.periodicX = false; p.periodicY = true; p.periodicZ = true;
        p.KHenry = 2.0; p.kA = 0.01;
        const int n = p.Nx * p.Ny * p.Nz;

        Lattice<D3Q19> Lattice_NS(p);
        ADLattice<D3Q7> Lattice_AD(p);
        AdsorbedField qField(p);
        auto inlet = buildXPlaneMask(p.Nx, p.Ny, p.Nz, 0);
        auto outlet = buildXPlaneMask(p.Nx, p.Ny, p.Nz, p.Nx - 1);
        Lattice_NS.setObstacleMask(geom.mask);
        Lattice_NS.setCollisionOperator(std::make_shared<BGKCollision<D3Q19>>(p));
        Lattice_NS.addBoundary<VelocityDirichletNEQ<D3Q19>>(p, inlet, 0.01, 0.0, 0.0);
        Lattice_NS.addBoundary<PressureDirichlet<D3Q19>>(p, outlet, 1.0);
        Lattice_AD.setCollisionOperator(std::make_shared<ADBGKCollision<D3Q7>>(p));
        Lattice_AD.setTauField(std::vector<DATA_TYPE>((size_t)n, 0.7));
        Lattice_AD.addBoundary<ADDirichlet<D3Q7>>(p, inlet, 1.0);
        Lattice_AD.addBoundary<ADNeumannOutlet<D3Q7>>(p, outlet);
        NSCount& nsCount = Lattice_NS.addBoundary<NSCount>();
        ADCount& adCount = Lattice_AD.addBoundary<ADCount>();
        LinearLDF<D3Q7> LinearIsothermAdsorption(p);
        Lattice_NS.initEquilibrium();
        Lattice_AD.initEquilibrium();
        UnitConverter uc{0.5};
        OutletCSV<ADLattice<D3Q7>, UnitConverter> outletCsv((dir + "/outlet.csv").c_str(), uc, outlet, Lattice_AD);
        outletCsv.log(0);
        for (int s = 1; s <= steps; ++s) {
            Lattice_NS.step(s);
            Lattice_NS.computeMacroscopicDevice();
            Lattice_AD.setAdvectionFromFluidDevice(Lattice_NS);
            Lattice_AD.zeroSource();
            LinearIsothermAdsorption.computeSource(Lattice_AD, qField, Lattice_NS.d_obstacle_ptr());
            Lattice_AD.step(s);
            if (s % csvEvery == 0) outletCsv.log(s);
        }
        outletCsv.flush();
        Lattice_NS.downloadMacroscopic();
        Lattice_AD.downloadPhi();
        qField.download();
        FILE* f = std::fopen((dir + "/fields.bin").c_str(), "wb");
        if (!f) return 3;
        const std::vector<DATA_TYPE>& q = qField.host();
        const std::vector<const std::vector<DATA_TYPE>*> out = {&Lattice_NS.rhoHost(), &Lattice_NS.uxHost(),
                                                               &Lattice_NS.uyHost(), &Lattice_NS.uzHost(),
                                                               &Lattice_AD.phiHost(), &q};
        for (const std::vector<DATA_TYPE>* v : out) std::fwrite(v->data(), sizeof(double), v->size(), f);
        std::fclose(f);
        std::printf("apply ns %d %d %d ad %d %d %d\n", nsCount.pre, nsCount.post, nsCount.bad_step, adCount.pre,
                    adCount.post, adCount.bad_step);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
