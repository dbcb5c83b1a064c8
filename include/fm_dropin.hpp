// fm_dropin.hpp -- the reference's lattice / operator / boundary / reaction /
// I/O classes, re-expressed over the C ABI of fm.h (header-only C++17).
//
// A program written against the reference (src/main.cpp:101-357) compiles
// against these classes by replacing its includes with this header and adding
// `using namespace fm_dropin;`.  The class names, constructor arguments and
// method names are the reference's:
//   Lattice<D3Q19>            include/core/lattice/NSLattice.hpp:14-265
//   ADLattice<D3Q7>           include/core/lattice/ADLattice.hpp:18-190
//   AdsorbedField             include/reaction/AdsorbedField.hpp:7-60
//   BGKCollision, PorousBGKCollision, ADBGKCollision (include/collision/*.hpp)
//   VelocityDirichletNEQ, VelocityDirichletEq, PressureDirichlet, BounceBack
//                             (include/boundary/ns/*.hpp)
//   ADDirichlet, ADDirichletTanhPulse, ADNeumannOutlet (include/boundary/ad/*.hpp)
//   LinearLDF, LangmuirLDF    include/reaction/{LinearLDF,LangmuirLDF}.hpp
//   OutletCSV                 include/core/io/OutletCSV.hpp:13-67
//   readVTI / VTIResult       include/vti/VTIReader.hpp:14-160
//   ADUnitConverter           include/core/io/ADUnitConverter.hpp:17-104
//   the operator interfaces   include/core/interfaces/{NS,AD}Interfaces.hpp:9-22
// Errors are std::runtime_error with the reference's messages, as there.
//
// One fm_lattice holds the NS lattice, the AD lattice and the adsorbed field,
// and one fused launch runs the whole loop body of src/main.cpp:319-357.  So:
//   * construct Lattice<D3Q19> first; ADLattice and AdsorbedField constructed
//     afterwards on the same thread attach to it;
//   * Lattice::step(s) marks the NS half; the coupled step runs at
//     ADLattice::step(s), by which time LinearLDF / LangmuirLDF::computeSource
//     has named the isotherm and setAdvectionFromFluidDevice the coupling (a
//     step without that call runs uncoupled, as the reference's --coupling off);
//   * computeMacroscopicDevice and zeroSource are part of the fused step
//     (no-ops here); Lattice::initEquilibrium initialises both lattices.
// The storage precision is FP64 by default (the reference's DATA_TYPE as
// shipped, bit-identical results); set_precision(FM_F32) before constructing
// the lattice for the FP32 form.
#pragma once

#include <cstdint>
#include <fstream>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "fm.h"

namespace fm_dropin {

using DATA_TYPE = double;

// include/core/Params.hpp:6-37
struct LBMParams {
    int Nx, Ny, Nz;
    DATA_TYPE rho0;
    DATA_TYPE tau;
    DATA_TYPE tau_ad;
    DATA_TYPE phi0;
    DATA_TYPE minConcentration = 1e-8;
    bool periodicX = true;
    bool periodicY = true;
    bool periodicZ = true;
    bool enableAdsorption = false;
    DATA_TYPE KHenry;
    DATA_TYPE kA;
    DATA_TYPE qMax;
    DATA_TYPE bLangmuir;
    DATA_TYPE kLDF;
    DATA_TYPE porosityValue = 0.67;
    DATA_TYPE betaPorous = 1;
};

enum class BoundaryPhase { PreCollision, PostStreaming };

// include/core/descriptors/D3Q19.hpp:10-11, D3Q7.hpp:10-11 (the velocity sets
// themselves live in the fused kernel)
struct D3Q19 {
    static constexpr DATA_TYPE cs2 = DATA_TYPE(1) / DATA_TYPE(3);
    static constexpr DATA_TYPE inv_cs2 = DATA_TYPE(3);
};
struct D3Q7 {
    static constexpr DATA_TYPE cs2 = DATA_TYPE(1) / DATA_TYPE(4);
    static constexpr DATA_TYPE inv_cs2 = DATA_TYPE(4);
};

inline void check(int rc)
{
    if (rc != FM_OK) throw std::runtime_error(fm_last_error());
}

namespace detail {
struct Shared {
    fm_lattice* lat = nullptr;
    LBMParams p{};
    int n = 0;
    std::vector<std::uint8_t> obstacle;   // host copy; d_obstacle_ptr() hands out its address
    bool ns_pending = false;
    int ns_step = 0;                       // step index of the pending NS step
    bool coupled = false;                  // setAdvectionFromFluidDevice seen for the pending step
    int coupling_set = -1;
    // the NS lattice's boundaries at a phase of a step (set while it lives)
    std::function<void(BoundaryPhase, int)> ns_apply;
    ~Shared()
    {
        if (lat) fm_lattice_destroy(lat);
    }
    void run_step()
    {
        const int c = coupled ? 1 : 0;
        if (c != coupling_set) {
            check(fm_set_coupling(lat, c));
            coupling_set = c;
        }
        check(fm_step(lat, 1));
        ns_pending = false;
        coupled = false;
    }
};
inline std::shared_ptr<Shared>& current()
{
    static thread_local std::shared_ptr<Shared> s;
    return s;
}
inline int& precision()
{
    static int p = FM_F64;
    return p;
}
inline std::shared_ptr<Shared> attach(const char* who)
{
    auto s = current();
    if (!s) throw std::runtime_error(std::string(who) + ": construct Lattice<D3Q19> first");
    return s;
}
inline void fetch(fm_lattice* lat, int field, std::vector<DATA_TYPE>& out, int n)
{
    out.resize((size_t)n);
    check(fm_get_field(lat, field, out.data(), (size_t)n));
}
}  // namespace detail

// Storage precision of lattices constructed afterwards (FM_F64 by default).
inline void set_precision(int precision) { detail::precision() = precision; }

template <typename Descriptor> class Lattice;
template <typename Descriptor> class ADLattice;

// ---- operator interfaces (include/core/interfaces/{NS,AD}Interfaces.hpp:9-22) ----
// The reference's plug-in contract, with its signatures: code that subclasses
// these compiles against this header unchanged.
template <typename Descriptor>
class NSCollisionOperator {
public:
    virtual ~NSCollisionOperator() = default;
    virtual void initEq(Lattice<Descriptor>& lat) = 0;
    virtual void collideStream(Lattice<Descriptor>& lat) = 0;   // f -> f_new
};
template <typename Descriptor>
class NSBoundaryCondition {
public:
    virtual ~NSBoundaryCondition() = default;
    virtual void apply(Lattice<Descriptor>& lat, BoundaryPhase phase, int step) = 0;
};
template <typename Descriptor>
class ADCollisionOperator {
public:
    virtual ~ADCollisionOperator() = default;
    virtual void initEq(ADLattice<Descriptor>& lat) = 0;
    virtual void collideStream(ADLattice<Descriptor>& lat) = 0;  // g -> g_new
};
template <typename Descriptor>
class ADBoundaryCondition {
public:
    virtual ~ADBoundaryCondition() = default;
    virtual void apply(ADLattice<Descriptor>& lat, BoundaryPhase phase, int step) = 0;
};

// How the operators of this header implement that contract.  One fused
// launch per time step does the collision, streaming and every boundary of
// both lattices, so the operators below register with the fm_lattice instead
// of launching anything:
//   * a collision operator names its kind when setCollisionOperator receives it
//     (fused_kind); its initEq / collideStream are empty;
//   * a boundary registers its mask when addBoundary constructs it (attach);
//     its apply is empty.
// The lattices call every registered boundary's apply at the reference's
// points of the step (NS pre-collision in Lattice::step; AD pre-collision,
// then NS and AD post-streaming around the fused step in ADLattice::step), so
// a boundary written against the reference's interface runs there.  It sees
// the lattice through this header's API (field downloads, handle()), not the
// reference's array-of-structures device arrays.  A collision operator that
// is not one of this header's is rejected by setCollisionOperator: the fused
// step has no place for a separate collide-and-stream kernel.
namespace detail {
struct FusedCollision {
    virtual ~FusedCollision() = default;
    virtual int fused_kind() const = 0;
};
struct FusedBoundary {
    virtual ~FusedBoundary() = default;
    virtual void attach(fm_lattice* lat) = 0;
};
}  // namespace detail

template <typename Descriptor>
class BGKCollision : public NSCollisionOperator<Descriptor>, public detail::FusedCollision {
public:
    explicit BGKCollision(const LBMParams&) {}
    void initEq(Lattice<Descriptor>&) override {}
    void collideStream(Lattice<Descriptor>&) override {}
    int fused_kind() const override { return FM_COLL_BGK; }
};
template <typename Descriptor>
class PorousBGKCollision : public NSCollisionOperator<Descriptor>, public detail::FusedCollision {
public:
    explicit PorousBGKCollision(const LBMParams&) {}
    void initEq(Lattice<Descriptor>&) override {}
    void collideStream(Lattice<Descriptor>&) override {}
    int fused_kind() const override { return FM_COLL_POROUS; }
};
template <typename Descriptor>
class ADBGKCollision : public ADCollisionOperator<Descriptor>, public detail::FusedCollision {
public:
    explicit ADBGKCollision(const LBMParams&) {}
    void initEq(ADLattice<Descriptor>&) override {}
    void collideStream(ADLattice<Descriptor>&) override {}
    int fused_kind() const override { return 0; }
};

// ---- NS boundaries --------------------------------------------------------
template <typename Descriptor>
class VelocityDirichletNEQ : public NSBoundaryCondition<Descriptor>, public detail::FusedBoundary {
public:
    VelocityDirichletNEQ(const LBMParams&, std::vector<std::uint8_t> mask, DATA_TYPE ux, DATA_TYPE uy, DATA_TYPE uz)
        : m_(std::move(mask)), u_{ux, uy, uz} {}
    void attach(fm_lattice* lat) override { check(fm_add_ns_velocity_neq(lat, m_.data(), m_.size(), u_[0], u_[1], u_[2])); }
    void apply(Lattice<Descriptor>&, BoundaryPhase, int) override {}

private:
    std::vector<std::uint8_t> m_;
    DATA_TYPE u_[3];
};
template <typename Descriptor>
class VelocityDirichletEq : public NSBoundaryCondition<Descriptor>, public detail::FusedBoundary {
public:
    VelocityDirichletEq(const LBMParams&, std::vector<std::uint8_t> mask, DATA_TYPE ux, DATA_TYPE uy, DATA_TYPE uz)
        : m_(std::move(mask)), u_{ux, uy, uz} {}
    void attach(fm_lattice* lat) override { check(fm_add_ns_velocity_eq(lat, m_.data(), m_.size(), u_[0], u_[1], u_[2])); }
    void apply(Lattice<Descriptor>&, BoundaryPhase, int) override {}

private:
    std::vector<std::uint8_t> m_;
    DATA_TYPE u_[3];
};
template <typename Descriptor>
class PressureDirichlet : public NSBoundaryCondition<Descriptor>, public detail::FusedBoundary {
public:
    PressureDirichlet(const LBMParams&, std::vector<std::uint8_t> mask, DATA_TYPE rho_out)
        : m_(std::move(mask)), rho_(rho_out) {}
    void attach(fm_lattice* lat) override { check(fm_add_ns_pressure(lat, m_.data(), m_.size(), rho_)); }
    void apply(Lattice<Descriptor>&, BoundaryPhase, int) override {}

private:
    std::vector<std::uint8_t> m_;
    DATA_TYPE rho_;
};
template <typename Descriptor>
class BounceBack : public NSBoundaryCondition<Descriptor>, public detail::FusedBoundary {
public:
    BounceBack(const LBMParams&, std::vector<std::uint8_t> mask) : m_(std::move(mask)) {}
    void attach(fm_lattice* lat) override { check(fm_add_ns_bounceback(lat, m_.data(), m_.size())); }
    void apply(Lattice<Descriptor>&, BoundaryPhase, int) override {}

private:
    std::vector<std::uint8_t> m_;
};

// ---- AD boundaries --------------------------------------------------------
template <typename Descriptor>
class ADDirichlet : public ADBoundaryCondition<Descriptor>, public detail::FusedBoundary {
public:
    ADDirichlet(const LBMParams&, std::vector<std::uint8_t> mask, DATA_TYPE phi) : m_(std::move(mask)), phi_(phi) {}
    void attach(fm_lattice* lat) override { check(fm_add_ad_dirichlet(lat, m_.data(), m_.size(), phi_)); }
    void apply(ADLattice<Descriptor>&, BoundaryPhase, int) override {}

private:
    std::vector<std::uint8_t> m_;
    DATA_TYPE phi_;
};
template <typename Descriptor>
class ADDirichletTanhPulse : public ADBoundaryCondition<Descriptor>, public detail::FusedBoundary {
public:
    ADDirichletTanhPulse(const LBMParams&, std::vector<std::uint8_t> mask, DATA_TYPE phi_base, DATA_TYPE phi_amp,
                         int t_on_step, int t_off_step, DATA_TYPE k_step)
        : m_(std::move(mask)), base_(phi_base), amp_(phi_amp), on_(t_on_step), off_(t_off_step), k_(k_step) {}
    void attach(fm_lattice* lat) override
    {
        check(fm_add_ad_tanh_pulse(lat, m_.data(), m_.size(), base_, amp_, on_, off_, k_));
    }
    void apply(ADLattice<Descriptor>&, BoundaryPhase, int) override {}

private:
    std::vector<std::uint8_t> m_;
    DATA_TYPE base_, amp_;
    int on_, off_;
    DATA_TYPE k_;
};
template <typename Descriptor>
class ADNeumannOutlet : public ADBoundaryCondition<Descriptor>, public detail::FusedBoundary {
public:
    ADNeumannOutlet(const LBMParams&, std::vector<std::uint8_t> mask) : m_(std::move(mask)) {}
    void attach(fm_lattice* lat) override { check(fm_add_ad_neumann(lat, m_.data(), m_.size())); }
    void apply(ADLattice<Descriptor>&, BoundaryPhase, int) override {}

private:
    std::vector<std::uint8_t> m_;
};

// ---- the NS lattice ---------------------------------------------------------
template <>
class Lattice<D3Q19> {
public:
    explicit Lattice(const LBMParams& p) : s_(std::make_shared<detail::Shared>())
    {
        s_->p = p;
        s_->n = p.Nx * p.Ny * p.Nz;
        fm_params fp{p.Nx, p.Ny, p.Nz, p.rho0, p.tau, p.tau_ad, p.phi0, p.minConcentration,
                     p.periodicX ? 1 : 0, p.periodicY ? 1 : 0, p.periodicZ ? 1 : 0};
        check(fm_lattice_create(&fp, detail::precision(), nullptr, &s_->lat));
        s_->ns_apply = [this](BoundaryPhase ph, int step) {
            for (auto& bc : bcs_) bc->apply(*this, ph, step);
        };
        detail::current() = s_;
    }
    ~Lattice()
    {
        s_->ns_apply = nullptr;
        if (detail::current() == s_) detail::current().reset();
    }
    Lattice(const Lattice&) = delete;
    Lattice& operator=(const Lattice&) = delete;

    int Size() const { return s_->n; }
    const LBMParams& P() const { return s_->p; }
    fm_lattice* handle() const { return s_->lat; }

    void setObstacleMask(const std::vector<std::uint8_t>& mask)
    {
        check(fm_set_obstacle_mask(s_->lat, mask.data(), mask.size()));
        s_->obstacle = mask;
    }
    void setPorosityFromMask(const std::vector<std::uint8_t>& mask, DATA_TYPE phi_masked, DATA_TYPE phi_else)
    {
        check(fm_set_porosity_from_mask(s_->lat, mask.data(), mask.size(), phi_masked, phi_else));
    }
    void setCollisionOperator(std::shared_ptr<NSCollisionOperator<D3Q19>> op)
    {
        if (!op) throw std::runtime_error("NSLattice::setCollisionOperator: null operator");
        const auto* fused = dynamic_cast<const detail::FusedCollision*>(op.get());
        if (!fused)
            throw std::runtime_error("NSLattice::setCollisionOperator: only BGKCollision and PorousBGKCollision "
                                     "run inside the fused step");
        check(fm_set_collision(s_->lat, fused->fused_kind()));
        collision_ = std::move(op);
    }
    // NSLattice.hpp:165-174
    template <typename TBoundary, typename... Args>
    TBoundary& addBoundary(Args&&... args)
    {
        static_assert(std::is_base_of_v<NSBoundaryCondition<D3Q19>, TBoundary>,
                      "addBoundary: TBoundary must derive from NSBoundaryCondition<Descriptor>");
        auto b = std::make_unique<TBoundary>(std::forward<Args>(args)...);
        if (auto* fused = dynamic_cast<detail::FusedBoundary*>(b.get())) fused->attach(s_->lat);
        TBoundary& ref = *b;
        bcs_.emplace_back(std::move(b));
        return ref;
    }
    void initEquilibrium()
    {
        if (!collision_) throw std::runtime_error("NSLattice::initEquilibrium: collision operator not set");
        collision_->initEq(*this);
        check(fm_init_equilibrium(s_->lat));
    }
    // NSLattice.hpp:188-209: pre-collision boundaries now; the collision, the
    // streaming and the post-streaming boundaries run with ADLattice::step
    void step(int stepIndex)
    {
        if (!collision_) throw std::runtime_error("NSLattice: collision operator not set, could not step()!");
        if (s_->ns_pending) {   // an NS step whose AD step never came
            s_->run_step();
            s_->ns_apply(BoundaryPhase::PostStreaming, s_->ns_step);
        }
        s_->ns_apply(BoundaryPhase::PreCollision, stepIndex);
        collision_->collideStream(*this);
        s_->ns_pending = true;
        s_->ns_step = stepIndex;
    }
    void computeMacroscopicDevice() {}
    // rho and u in one call: one macroscopic pass and one synchronisation
    void downloadMacroscopic()
    {
        const size_t n = (size_t)s_->n;
        h_rho_.resize(n); h_ux_.resize(n); h_uy_.resize(n); h_uz_.resize(n);
        double* const out[6] = {h_rho_.data(), h_ux_.data(), h_uy_.data(), h_uz_.data(), nullptr, nullptr};
        check(fm_get_fields(s_->lat, out, n));
    }
    const std::vector<DATA_TYPE>& rhoHost() const { return h_rho_; }
    const std::vector<DATA_TYPE>& uxHost() const { return h_ux_; }
    const std::vector<DATA_TYPE>& uyHost() const { return h_uy_; }
    const std::vector<DATA_TYPE>& uzHost() const { return h_uz_; }
    const std::vector<std::uint8_t>& obstacleHost() const { return s_->obstacle; }
    // The reference passes this device pointer as the LDF region
    // (src/main.cpp:333); here it is a token that computeSource recognises.
    const std::uint8_t* d_obstacle_ptr() const { return s_->obstacle.data(); }

private:
    std::shared_ptr<detail::Shared> s_;
    std::shared_ptr<NSCollisionOperator<D3Q19>> collision_;
    std::vector<std::unique_ptr<NSBoundaryCondition<D3Q19>>> bcs_;
    std::vector<DATA_TYPE> h_rho_, h_ux_, h_uy_, h_uz_;
};

// ---- the AD lattice ---------------------------------------------------------
template <>
class ADLattice<D3Q7> {
public:
    explicit ADLattice(const LBMParams& p) : s_(detail::attach("ADLattice")), p_(p) {}
    const LBMParams& P() const { return p_; }
    int Size() const { return s_->n; }
    void setTauField(const std::vector<DATA_TYPE>& tau) { check(fm_set_tau_field(s_->lat, tau.data(), tau.size())); }
    void setCollisionOperator(std::shared_ptr<ADCollisionOperator<D3Q7>> op)
    {
        if (!op) throw std::runtime_error("ADLattice::setCollisionOperator: null operator");
        if (!dynamic_cast<const detail::FusedCollision*>(op.get()))
            throw std::runtime_error("ADLattice::setCollisionOperator: only ADBGKCollision runs inside the fused step");
        collision_ = std::move(op);
    }
    // ADLattice.hpp:115-130
    template <typename TBoundary, typename... Args>
    TBoundary& addBoundary(Args&&... args)
    {
        static_assert(std::is_base_of_v<ADBoundaryCondition<D3Q7>, TBoundary>,
                      "AD boundary must derive from ADBoundaryCondition");
        auto b = std::make_unique<TBoundary>(std::forward<Args>(args)...);
        if (auto* fused = dynamic_cast<detail::FusedBoundary*>(b.get())) fused->attach(s_->lat);
        TBoundary& ref = *b;
        bcs_.emplace_back(std::move(b));
        return ref;
    }
    // ADLattice.hpp:134-141 (both lattices are initialised by Lattice::initEquilibrium)
    void initEquilibrium()
    {
        if (!collision_) throw std::runtime_error("ADLattice: collision operator not set, could not initEq()!");
        collision_->initEq(*this);
    }
    void zeroSource() {}
    void setAdvectionFromFluidDevice(const Lattice<D3Q19>&) { s_->coupled = true; }
    // ADLattice.hpp:144-162, with the pending NS step fused into the same launch
    void step(int stepIndex)
    {
        if (!collision_) throw std::runtime_error("ADLattice: collision operator not set, could not step()!");
        for (auto& bc : bcs_) bc->apply(*this, BoundaryPhase::PreCollision, stepIndex);
        collision_->collideStream(*this);
        const bool ns = s_->ns_pending;
        const int ns_step = s_->ns_step;
        s_->run_step();
        if (ns && s_->ns_apply) s_->ns_apply(BoundaryPhase::PostStreaming, ns_step);
        for (auto& bc : bcs_) bc->apply(*this, BoundaryPhase::PostStreaming, stepIndex);
    }
    void downloadPhi() { detail::fetch(s_->lat, FM_FIELD_C, h_phi_, s_->n); }
    const std::vector<DATA_TYPE>& phiHost() const { return h_phi_; }
    fm_lattice* handle() const { return s_->lat; }

private:
    std::shared_ptr<detail::Shared> s_;
    LBMParams p_;
    std::shared_ptr<ADCollisionOperator<D3Q7>> collision_;
    std::vector<std::unique_ptr<ADBoundaryCondition<D3Q7>>> bcs_;
    std::vector<DATA_TYPE> h_phi_;
};

// ---- adsorbed loading ---------------------------------------------------------
class AdsorbedField {
public:
    explicit AdsorbedField(const LBMParams&) : s_(detail::attach("AdsorbedField")), h_q_((size_t)s_->n, 0.0) {}
    void download() { detail::fetch(s_->lat, FM_FIELD_Q, h_q_, s_->n); }
    void upload() { check(fm_set_state(s_->lat, nullptr, nullptr, nullptr, h_q_.data())); }
    std::vector<DATA_TYPE>& host() { return h_q_; }
    const std::vector<DATA_TYPE>& host() const { return h_q_; }

private:
    std::shared_ptr<detail::Shared> s_;
    std::vector<DATA_TYPE> h_q_;
};

// ---- LDF sources: name the isotherm of the fused step ----------------------
namespace detail {
inline const std::uint8_t* region_of(const Shared& s, const std::uint8_t* region)
{
    // the token handed out by Lattice::d_obstacle_ptr, else a host mask of n bytes
    return region == s.obstacle.data() ? s.obstacle.data() : region;
}
}  // namespace detail

template <typename ADDesc>
class LinearLDF {
public:
    explicit LinearLDF(const LBMParams& p) : p_(p) {}
    void computeSource(ADLattice<ADDesc>& ad, AdsorbedField&, const std::uint8_t* regionMask)
    {
        if (set_ == regionMask) return;
        auto s = detail::attach("LinearLDF");
        check(fm_set_isotherm_linear(ad.handle(), detail::region_of(*s, regionMask), (size_t)s->n, p_.KHenry, p_.kA));
        set_ = regionMask;
    }

private:
    LBMParams p_;
    const std::uint8_t* set_ = nullptr;
};

template <typename ADDesc>
class LangmuirLDF {
public:
    explicit LangmuirLDF(const LBMParams& p) : p_(p) {}
    void computeSource(ADLattice<ADDesc>& ad, AdsorbedField&, const std::uint8_t* regionMask)
    {
        if (set_ == regionMask) return;
        auto s = detail::attach("LangmuirLDF");
        check(fm_set_isotherm_langmuir(ad.handle(), detail::region_of(*s, regionMask), (size_t)s->n, p_.qMax,
                                       p_.bLangmuir, p_.kLDF));
        set_ = regionMask;
    }

private:
    LBMParams p_;
    const std::uint8_t* set_ = nullptr;
};

// ---- outlet log: the device reduction instead of a full phi download -------
template <typename ADLat, typename UnitConv>
class OutletCSV {
public:
    OutletCSV(const char* path, const UnitConv& uc, const std::vector<std::uint8_t>& outletMask, ADLat& adLat)
        : uc_(uc), ad_(adLat), out_(path)
    {
        if (!out_) throw std::runtime_error("Could not open outlet csv");
        check(fm_set_outlet_probe(adLat.handle(), outletMask.data(), outletMask.size(), 0));
        out_ << "step,time_s,phi_out_avg,phi_out_min,phi_out_max\n";
    }
    void log(int step)
    {
        double st[3];
        check(fm_outlet_stats(ad_.handle(), st));
        out_ << step << "," << uc_.timeLatticeToPhys(step) << "," << st[0] << "," << st[1] << "," << st[2] << "\n";
    }
    void flush() { out_.flush(); }

private:
    const UnitConv& uc_;
    ADLat& ad_;
    std::ofstream out_;
};

// ---- geometry ---------------------------------------------------------------
struct VTIResult {
    int Nx = 0;
    int Ny = 0;
    int Nz = 0;
    std::vector<std::uint8_t> mask;
};

inline VTIResult readVTI(const std::string& filename, double threshold = 0.5)
{
    VTIResult r;
    long long nv = 0;
    check(fm_vti_info(filename.c_str(), &r.Nx, &r.Ny, &r.Nz, &nv));
    const size_t n = (size_t)r.Nx * (size_t)r.Ny * (size_t)r.Nz;
    r.mask.assign(n, 0);
    check(fm_vti_read(filename.c_str(), threshold, r.mask.data(), nullptr, n));
    return r;
}

// the per-cell values of the first DataArray (a continuous solid fraction)
inline std::vector<double> readVTIValues(const std::string& filename, int* nx = nullptr, int* ny = nullptr,
                                         int* nz = nullptr)
{
    int x = 0, y = 0, z = 0;
    long long nv = 0;
    check(fm_vti_info(filename.c_str(), &x, &y, &z, &nv));
    std::vector<double> v((size_t)x * y * z);
    check(fm_vti_read(filename.c_str(), 0.5, nullptr, v.data(), v.size()));
    if (nx) *nx = x;
    if (ny) *ny = y;
    if (nz) *nz = z;
    return v;
}

// helpers.hpp:7-14
inline std::vector<std::uint8_t> buildXPlaneMask(int Nx, int Ny, int Nz, int x)
{
    std::vector<std::uint8_t> m((size_t)Nx * Ny * Nz, 0);
    for (int z = 0; z < Nz; ++z)
        for (int y = 0; y < Ny; ++y) m[(size_t)x + (size_t)Nx * ((size_t)y + (size_t)Ny * z)] = 1;
    return m;
}

// include/core/io/ADUnitConverter.hpp:17-104: the AD relaxation time from a
// physical diffusivity; buildTauField is fm_build_tau_field (D3Q7, cs2 = 1/4).
template <typename Descriptor>
struct ADUnitConverter {
    int Nx, Ny, Nz;
    double dx_phys;
    double dt_phys;
    static constexpr double cs2_lbm = static_cast<double>(Descriptor::cs2);

    ADUnitConverter(int Nx_, int Ny_, int Nz_, double dx_phys_, double dt_phys_)
        : Nx(Nx_), Ny(Ny_), Nz(Nz_), dx_phys(dx_phys_), dt_phys(dt_phys_)
    {
        if (Nx < 2) throw std::runtime_error("ADUnitConverter: Nx must be >= 2");
        if (dx_phys <= 0.0) throw std::runtime_error("ADUnitConverter: dx_phys must be > 0");
        if (dt_phys <= 0.0) throw std::runtime_error("ADUnitConverter: dt_phys must be > 0");
        if (cs2_lbm <= 0.0) throw std::runtime_error("ADUnitConverter: Descriptor::cs2 must be > 0");
    }
    double diffusivityPhysToLattice(double D_phys) const { return D_phys * dt_phys / (dx_phys * dx_phys); }
    double tauFromDiffusivityPhys(double D_phys) const
    {
        const double tau = diffusivityPhysToLattice(D_phys) / cs2_lbm + 0.5;
        if (tau <= 0.5) throw std::runtime_error("ADUnitConverter: tau_ad <= 0.5 (unstable)");
        return tau;
    }
    std::vector<DATA_TYPE> buildTauField(const std::vector<std::uint8_t>& mask, double D_fluid_phys,
                                         double D_solid_phys) const
    {
        static_assert(std::is_same_v<Descriptor, D3Q7>, "buildTauField: the AD lattice is D3Q7");
        std::vector<double> t(mask.size());
        check(fm_build_tau_field(Nx, Ny, Nz, dx_phys, dt_phys, mask.data(), mask.size(), D_fluid_phys, D_solid_phys,
                                 t.data()));
        return std::vector<DATA_TYPE>(t.begin(), t.end());
    }
};

}  // namespace fm_dropin
