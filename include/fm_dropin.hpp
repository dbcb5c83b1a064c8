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
#include <memory>
#include <stdexcept>
#include <string>
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

struct D3Q19 {};
struct D3Q7 {};

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
    bool coupled = false;                  // setAdvectionFromFluidDevice seen for the pending step
    int coupling_set = -1;
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

// ---- operator interfaces (include/core/interfaces/{NS,AD}Interfaces.hpp) ----
template <typename Descriptor>
class NSCollisionOperator {
public:
    virtual ~NSCollisionOperator() = default;
    virtual int fm_collision() const = 0;
};
template <typename Descriptor>
class NSBoundaryCondition {
public:
    virtual ~NSBoundaryCondition() = default;
    virtual void attach(fm_lattice* lat) = 0;
};
template <typename Descriptor>
class ADCollisionOperator {
public:
    virtual ~ADCollisionOperator() = default;
};
template <typename Descriptor>
class ADBoundaryCondition {
public:
    virtual ~ADBoundaryCondition() = default;
    virtual void attach(fm_lattice* lat) = 0;
};

template <typename Descriptor>
class BGKCollision : public NSCollisionOperator<Descriptor> {
public:
    explicit BGKCollision(const LBMParams&) {}
    int fm_collision() const override { return FM_COLL_BGK; }
};
template <typename Descriptor>
class PorousBGKCollision : public NSCollisionOperator<Descriptor> {
public:
    explicit PorousBGKCollision(const LBMParams&) {}
    int fm_collision() const override { return FM_COLL_POROUS; }
};
template <typename Descriptor>
class ADBGKCollision : public ADCollisionOperator<Descriptor> {
public:
    explicit ADBGKCollision(const LBMParams&) {}
};

// ---- NS boundaries --------------------------------------------------------
template <typename Descriptor>
class VelocityDirichletNEQ : public NSBoundaryCondition<Descriptor> {
public:
    VelocityDirichletNEQ(const LBMParams&, std::vector<std::uint8_t> mask, DATA_TYPE ux, DATA_TYPE uy, DATA_TYPE uz)
        : m_(std::move(mask)), u_{ux, uy, uz} {}
    void attach(fm_lattice* lat) override { check(fm_add_ns_velocity_neq(lat, m_.data(), m_.size(), u_[0], u_[1], u_[2])); }

private:
    std::vector<std::uint8_t> m_;
    DATA_TYPE u_[3];
};
template <typename Descriptor>
class VelocityDirichletEq : public NSBoundaryCondition<Descriptor> {
public:
    VelocityDirichletEq(const LBMParams&, std::vector<std::uint8_t> mask, DATA_TYPE ux, DATA_TYPE uy, DATA_TYPE uz)
        : m_(std::move(mask)), u_{ux, uy, uz} {}
    void attach(fm_lattice* lat) override { check(fm_add_ns_velocity_eq(lat, m_.data(), m_.size(), u_[0], u_[1], u_[2])); }

private:
    std::vector<std::uint8_t> m_;
    DATA_TYPE u_[3];
};
template <typename Descriptor>
class PressureDirichlet : public NSBoundaryCondition<Descriptor> {
public:
    PressureDirichlet(const LBMParams&, std::vector<std::uint8_t> mask, DATA_TYPE rho_out)
        : m_(std::move(mask)), rho_(rho_out) {}
    void attach(fm_lattice* lat) override { check(fm_add_ns_pressure(lat, m_.data(), m_.size(), rho_)); }

private:
    std::vector<std::uint8_t> m_;
    DATA_TYPE rho_;
};
template <typename Descriptor>
class BounceBack : public NSBoundaryCondition<Descriptor> {
public:
    BounceBack(const LBMParams&, std::vector<std::uint8_t> mask) : m_(std::move(mask)) {}
    void attach(fm_lattice* lat) override { check(fm_add_ns_bounceback(lat, m_.data(), m_.size())); }

private:
    std::vector<std::uint8_t> m_;
};

// ---- AD boundaries --------------------------------------------------------
template <typename Descriptor>
class ADDirichlet : public ADBoundaryCondition<Descriptor> {
public:
    ADDirichlet(const LBMParams&, std::vector<std::uint8_t> mask, DATA_TYPE phi) : m_(std::move(mask)), phi_(phi) {}
    void attach(fm_lattice* lat) override { check(fm_add_ad_dirichlet(lat, m_.data(), m_.size(), phi_)); }

private:
    std::vector<std::uint8_t> m_;
    DATA_TYPE phi_;
};
template <typename Descriptor>
class ADDirichletTanhPulse : public ADBoundaryCondition<Descriptor> {
public:
    ADDirichletTanhPulse(const LBMParams&, std::vector<std::uint8_t> mask, DATA_TYPE phi_base, DATA_TYPE phi_amp,
                         int t_on_step, int t_off_step, DATA_TYPE k_step)
        : m_(std::move(mask)), base_(phi_base), amp_(phi_amp), on_(t_on_step), off_(t_off_step), k_(k_step) {}
    void attach(fm_lattice* lat) override
    {
        check(fm_add_ad_tanh_pulse(lat, m_.data(), m_.size(), base_, amp_, on_, off_, k_));
    }

private:
    std::vector<std::uint8_t> m_;
    DATA_TYPE base_, amp_;
    int on_, off_;
    DATA_TYPE k_;
};
template <typename Descriptor>
class ADNeumannOutlet : public ADBoundaryCondition<Descriptor> {
public:
    ADNeumannOutlet(const LBMParams&, std::vector<std::uint8_t> mask) : m_(std::move(mask)) {}
    void attach(fm_lattice* lat) override { check(fm_add_ad_neumann(lat, m_.data(), m_.size())); }

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
        detail::current() = s_;
    }
    ~Lattice()
    {
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
        check(fm_set_collision(s_->lat, op->fm_collision()));
    }
    template <typename TBoundary, typename... Args>
    TBoundary& addBoundary(Args&&... args)
    {
        auto b = std::make_unique<TBoundary>(std::forward<Args>(args)...);
        b->attach(s_->lat);
        TBoundary& ref = *b;
        bcs_.emplace_back(std::move(b));
        return ref;
    }
    void initEquilibrium() { check(fm_init_equilibrium(s_->lat)); }
    void step(int)
    {
        if (s_->ns_pending) s_->run_step();   // an NS step whose AD step never came
        s_->ns_pending = true;
    }
    void computeMacroscopicDevice() {}
    void downloadMacroscopic()
    {
        detail::fetch(s_->lat, FM_FIELD_RHO, h_rho_, s_->n);
        detail::fetch(s_->lat, FM_FIELD_UX, h_ux_, s_->n);
        detail::fetch(s_->lat, FM_FIELD_UY, h_uy_, s_->n);
        detail::fetch(s_->lat, FM_FIELD_UZ, h_uz_, s_->n);
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
    }
    template <typename TBoundary, typename... Args>
    TBoundary& addBoundary(Args&&... args)
    {
        auto b = std::make_unique<TBoundary>(std::forward<Args>(args)...);
        b->attach(s_->lat);
        TBoundary& ref = *b;
        bcs_.emplace_back(std::move(b));
        return ref;
    }
    void initEquilibrium() {}
    void zeroSource() {}
    void setAdvectionFromFluidDevice(const Lattice<D3Q19>&) { s_->coupled = true; }
    void step(int) { s_->run_step(); }
    void downloadPhi() { detail::fetch(s_->lat, FM_FIELD_C, h_phi_, s_->n); }
    const std::vector<DATA_TYPE>& phiHost() const { return h_phi_; }
    fm_lattice* handle() const { return s_->lat; }

private:
    std::shared_ptr<detail::Shared> s_;
    LBMParams p_;
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

}  // namespace fm_dropin
