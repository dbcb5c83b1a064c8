// Operators written against the reference's plug-in contract
// (include/core/interfaces/NSInterfaces.hpp:9-22, ADInterfaces.hpp:9-22), the
// way a user of the reference subclasses it, compiled against
// include/fm_dropin.hpp unchanged: the signatures, the registration calls
// (setCollisionOperator, addBoundary<T>(args...)) and the BoundaryPhase enum
// are the reference's.  Built by tests/test_dropin.py (compile and link only).
#include <memory>
#include <vector>

#include "fm_dropin.hpp"

using namespace fm_dropin;

template <typename Descriptor>
class MyCollision : public NSCollisionOperator<Descriptor> {
public:
    explicit MyCollision(const LBMParams& p) : p_(p) {}
    void initEq(Lattice<Descriptor>& lat) override { n_ = lat.Size(); }
    void collideStream(Lattice<Descriptor>& lat) override { n_ = lat.Size(); }

private:
    LBMParams p_;
    int n_ = 0;
};

template <typename Descriptor>
class MyWall : public NSBoundaryCondition<Descriptor> {
public:
    MyWall(const LBMParams&, std::vector<std::uint8_t> mask) : mask_(std::move(mask)) {}
    void apply(Lattice<Descriptor>& lat, BoundaryPhase phase, int step) override
    {
        if (phase == BoundaryPhase::PostStreaming && step > 0) seen_ = lat.Size();
    }

private:
    std::vector<std::uint8_t> mask_;
    int seen_ = 0;
};

template <typename Descriptor>
class MyADCollision : public ADCollisionOperator<Descriptor> {
public:
    void initEq(ADLattice<Descriptor>&) override {}
    void collideStream(ADLattice<Descriptor>&) override {}
};

template <typename Descriptor>
class MySource : public ADBoundaryCondition<Descriptor> {
public:
    explicit MySource(double v) : v_(v) {}
    void apply(ADLattice<Descriptor>& lat, BoundaryPhase phase, int) override
    {
        if (phase == BoundaryPhase::PreCollision) v_ += lat.Size();
    }

private:
    double v_;
};

// Builds the set-up on a lattice; not run by the test (it needs a GPU).
int wire(const LBMParams& p)
{
    Lattice<D3Q19> ns(p);
    ADLattice<D3Q7> ad(p);
    std::shared_ptr<NSCollisionOperator<D3Q19>> builtin = std::make_shared<BGKCollision<D3Q19>>(p);
    ns.setCollisionOperator(builtin);
    std::shared_ptr<NSCollisionOperator<D3Q19>> mine = std::make_shared<MyCollision<D3Q19>>(p);
    (void)mine;   // setCollisionOperator(mine) throws: the fused step runs only the built-in operators
    ad.setCollisionOperator(std::make_shared<ADBGKCollision<D3Q7>>(p));
    std::shared_ptr<ADCollisionOperator<D3Q7>> myad = std::make_shared<MyADCollision<D3Q7>>();
    (void)myad;
    MyWall<D3Q19>& wall = ns.addBoundary<MyWall<D3Q19>>(p, std::vector<std::uint8_t>((size_t)ns.Size(), 0));
    (void)wall;
    ad.addBoundary<MySource<D3Q7>>(0.5);
    ns.initEquilibrium();
    ad.initEquilibrium();
    ns.step(1);
    ad.step(1);
    return ns.Size();
}

int main(int argc, char**)
{
    LBMParams p{};
    p.Nx = 8; p.Ny = 4; p.Nz = 4; p.rho0 = 1.0; p.tau = 0.8; p.tau_ad = 0.7;
    return argc > 5 ? wire(p) : 0;
}
