// sphgpu.hpp — C++ host mirror of the reference's per-step module surface
// over the C ABI of include/sphgpu.h.
//
// Same class names and call shapes as the reference (include/module.hpp:10-14,
// include/bhtree.hpp:76-81, include/simulation.hpp:24-45):
//
//   auto sim = std::make_shared<sph::gpu::Simulation>(param);  // Simulation(param)
//   sim->set_particles(particles);                             // SPHParticle vector
//   sph::gpu::PreInteraction pre;  pre.initialize(param);  pre.calculation(sim);
//   sph::gpu::FluidForce fforce;   ...                     fforce.calculation(sim);
//   sph::gpu::GravityForce gforce; ...                     gforce.calculation(sim);
//   sph::gpu::TimeStep ts;         ...                     ts.calculation(sim);
//   sim->make_tree();  sim->get_tree()->neighbor_search(i, list, is_ij);
//
// A fatal status code throws sph::gpu::SPHException carrying the library's
// message, as THROW_ERROR does in the reference (include/exception.hpp:9-14).
// Particle arrays stay on the device between module calls; get_particles()
// downloads them.
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "sphgpu.h"

namespace sph {
namespace gpu {

class SPHException : public std::runtime_error {
public:
    explicit SPHException(const std::string& m) : std::runtime_error(m) {}
};

// Host particle record with the reference's field names (include/particle.hpp:8-43).
struct SPHParticle {
    double pos[3] = {0, 0, 0}, vel[3] = {0, 0, 0}, vel_p[3] = {0, 0, 0}, acc[3] = {0, 0, 0};
    double mass = 0, dens = 0, pres = 0, ene = 0, ene_p = 0, dene = 0, sml = 0, sound = 0;
    double balsara = 0, alpha = 0, gradh = 0, phi = 0;
    int id = 0, neighbor = 0;
};

inline sphgpu_params default_parameters()
{
    sphgpu_params p;
    sphgpu_default_params(&p);
    return p;
}

class BHTree;

class Simulation : public std::enable_shared_from_this<Simulation> {
    sphgpu_ctx* m_ctx = nullptr;
    std::shared_ptr<BHTree> m_tree;
    int m_num = 0;

public:
    explicit Simulation(const sphgpu_params& p)
    {
        const int rc = sphgpu_create(&p, &m_ctx);
        if(rc < 0) {
            const std::string msg = m_ctx ? sphgpu_last_error(m_ctx) : "sphgpu_create failed";
            sphgpu_destroy(m_ctx);
            m_ctx = nullptr;
            throw SPHException(msg);
        }
    }
    ~Simulation() { sphgpu_destroy(m_ctx); }
    Simulation(const Simulation&) = delete;
    Simulation& operator=(const Simulation&) = delete;

    sphgpu_ctx* ctx() const { return m_ctx; }
    int check(int rc) const
    {
        if(rc < 0) throw SPHException(sphgpu_last_error(m_ctx));
        return rc;
    }

    void set_particles(const std::vector<SPHParticle>& ps)
    {
        const size_t n = ps.size();
        std::vector<std::vector<double>> cols(SPHGPU_NFIELDS, std::vector<double>(n));
        for(size_t i = 0; i < n; ++i) {
            const SPHParticle& p = ps[i];
            for(int k = 0; k < 3; ++k) {
                cols[SPHGPU_F_POS_X + k][i] = p.pos[k];
                cols[SPHGPU_F_VEL_X + k][i] = p.vel[k];
                cols[SPHGPU_F_VELP_X + k][i] = p.vel_p[k];
                cols[SPHGPU_F_ACC_X + k][i] = p.acc[k];
            }
            cols[SPHGPU_F_MASS][i] = p.mass;
            cols[SPHGPU_F_DENS][i] = p.dens;
            cols[SPHGPU_F_PRES][i] = p.pres;
            cols[SPHGPU_F_ENE][i] = p.ene;
            cols[SPHGPU_F_ENE_P][i] = p.ene_p;
            cols[SPHGPU_F_DENE][i] = p.dene;
            cols[SPHGPU_F_SML][i] = p.sml;
            cols[SPHGPU_F_SOUND][i] = p.sound;
            cols[SPHGPU_F_BALSARA][i] = p.balsara;
            cols[SPHGPU_F_ALPHA][i] = p.alpha;
            cols[SPHGPU_F_GRADH][i] = p.gradh;
            cols[SPHGPU_F_PHI][i] = p.phi;
            cols[SPHGPU_F_NEIGHBOR][i] = p.neighbor;
        }
        std::vector<const double*> ptrs(SPHGPU_NFIELDS, nullptr);
        for(int k = 0; k < SPHGPU_NFIELDS; ++k) ptrs[k] = cols[k].data();
        check(sphgpu_upload(m_ctx, (int64_t)n, ptrs.data()));
        m_num = (int)n;
    }

    std::vector<SPHParticle> get_particles() const
    {
        const size_t n = (size_t)m_num;
        std::vector<std::vector<double>> cols(SPHGPU_NFIELDS, std::vector<double>(n));
        std::vector<double*> ptrs(SPHGPU_NFIELDS);
        for(int k = 0; k < SPHGPU_NFIELDS; ++k) ptrs[k] = cols[k].data();
        check(sphgpu_download(m_ctx, ptrs.data()));
        std::vector<SPHParticle> ps(n);
        for(size_t i = 0; i < n; ++i) {
            SPHParticle& p = ps[i];
            for(int k = 0; k < 3; ++k) {
                p.pos[k] = cols[SPHGPU_F_POS_X + k][i];
                p.vel[k] = cols[SPHGPU_F_VEL_X + k][i];
                p.vel_p[k] = cols[SPHGPU_F_VELP_X + k][i];
                p.acc[k] = cols[SPHGPU_F_ACC_X + k][i];
            }
            p.mass = cols[SPHGPU_F_MASS][i];
            p.dens = cols[SPHGPU_F_DENS][i];
            p.pres = cols[SPHGPU_F_PRES][i];
            p.ene = cols[SPHGPU_F_ENE][i];
            p.ene_p = cols[SPHGPU_F_ENE_P][i];
            p.dene = cols[SPHGPU_F_DENE][i];
            p.sml = cols[SPHGPU_F_SML][i];
            p.sound = cols[SPHGPU_F_SOUND][i];
            p.balsara = cols[SPHGPU_F_BALSARA][i];
            p.alpha = cols[SPHGPU_F_ALPHA][i];
            p.gradh = cols[SPHGPU_F_GRADH][i];
            p.phi = cols[SPHGPU_F_PHI][i];
            p.neighbor = (int)cols[SPHGPU_F_NEIGHBOR][i];
            p.id = (int)i;
        }
        return ps;
    }

    int get_particle_num() const { return m_num; }
    double get_time() const
    {
        double t = 0;
        check(sphgpu_get_time(m_ctx, &t, nullptr));
        return t;
    }
    double get_dt() const
    {
        double dt = 0;
        check(sphgpu_get_time(m_ctx, nullptr, &dt));
        return dt;
    }
    void set_dt(double dt) { check(sphgpu_set_dt(m_ctx, dt)); }
    double get_h_per_v_sig() const
    {
        double v = 0;
        check(sphgpu_get_h_per_v_sig(m_ctx, &v));
        return v;
    }
    void make_tree() { check(sphgpu_tree_make(m_ctx)); }
    // OutputManager::write_snapshot / load_for_resume in the CSV v1 format
    void write_csv(const std::string& path, int step, int precision = 16)
    {
        check(sphgpu_write_csv(m_ctx, path.c_str(), step, precision));
    }
    int read_csv(const std::string& path)
    {
        int step = 0;
        check(sphgpu_read_csv(m_ctx, path.c_str(), &step));
        return step;
    }
    // one step of Solver's Lane-Emden relaxation loop; returns dt_relax
    double relax_step(const sphgpu_lane_emden& le, bool first)
    {
        double d = 0.0;
        check(sphgpu_relax_step(m_ctx, &le, first ? 1 : 0, &d));
        return d;
    }
    std::shared_ptr<BHTree> get_tree();
};

// BHTree (include/bhtree.hpp:76-81); the tree lives in the Simulation's context.
class BHTree {
    Simulation* m_sim;
    std::vector<int64_t> m_off[2];
    std::vector<int32_t> m_ids[2];

public:
    explicit BHTree(Simulation* s) : m_sim(s) {}
    void make() { m_sim->make_tree(); }
    void set_kernel() { m_sim->check(sphgpu_tree_set_kernel(m_sim->ctx())); }
    // Lists of every particle in one batched walk; neighbor_search(i, ...)
    // then reads particle i's list (walk order, not distance-sorted).
    void search_all(bool is_ij)
    {
        const int n = m_sim->get_particle_num();
        auto& off = m_off[is_ij ? 1 : 0];
        auto& ids = m_ids[is_ij ? 1 : 0];
        off.assign((size_t)n + 1, 0);
        m_sim->check(sphgpu_neighbor_search(m_sim->ctx(), is_ij ? 1 : 0, off.data(), nullptr, 0));
        ids.assign((size_t)off[n] + 1, 0);
        m_sim->check(sphgpu_neighbor_search(m_sim->ctx(), is_ij ? 1 : 0, off.data(), ids.data(), off[n]));
    }
    int neighbor_search(int i, std::vector<int>& neighbor_list, bool is_ij = false)
    {
        auto& off = m_off[is_ij ? 1 : 0];
        if(off.empty()) search_all(is_ij);
        const int64_t b = off[(size_t)i], e = off[(size_t)i + 1];
        const auto& ids = m_ids[is_ij ? 1 : 0];
        neighbor_list.assign(ids.begin() + b, ids.begin() + e);
        return (int)(e - b);
    }
};

inline std::shared_ptr<BHTree> Simulation::get_tree()
{
    if(!m_tree) m_tree = std::make_shared<BHTree>(this);
    return m_tree;
}

// Module (include/module.hpp:10-14)
class Module {
public:
    virtual ~Module() = default;
    virtual void initialize(const sphgpu_params&) {}
    virtual void calculation(const std::shared_ptr<Simulation>& sim) = 0;
};

class PreInteraction : public Module {
public:
    void calculation(const std::shared_ptr<Simulation>& sim) override
    {
        sim->check(sphgpu_pre_interaction(sim->ctx()));
    }
};

class FluidForce : public Module {
public:
    void calculation(const std::shared_ptr<Simulation>& sim) override { sim->check(sphgpu_fluid_force(sim->ctx())); }
};

class GravityForce : public Module {
public:
    void calculation(const std::shared_ptr<Simulation>& sim) override
    {
        sim->check(sphgpu_gravity_force(sim->ctx()));
    }
};

class TimeStep : public Module {
public:
    void calculation(const std::shared_ptr<Simulation>& sim) override
    {
        double dt = 0;
        sim->check(sphgpu_timestep(sim->ctx(), &dt));
    }
};

// Solver::initialize tail / Solver::integrate (src/solver.cpp:941-978).
inline void initialize(const std::shared_ptr<Simulation>& sim) { sim->check(sphgpu_initialize(sim->ctx())); }
inline void integrate(const std::shared_ptr<Simulation>& sim) { sim->check(sphgpu_integrate(sim->ctx())); }

}  // namespace gpu
}  // namespace sph
