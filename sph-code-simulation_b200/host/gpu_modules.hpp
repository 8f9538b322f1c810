// gpu_modules.hpp — the reference-side binding: Module subclasses that run the
// per-step modules of Guo-astro/sph-code-simulation on the GPU through the C
// ABI of include/sphgpu.h.
//
// A maintainer adds this header beside src/solver.cpp and constructs these
// modules where Solver::initialize constructs its own (src/solver.cpp:686-723);
// it includes the reference's headers (include/module.hpp, simulation.hpp,
// parameters.hpp, particle.hpp, exception.hpp), so it compiles only inside the
// reference's tree (or with its include/ on the path) and links libsphgpu.so.
//
//   auto gpu = std::make_shared<sph::GpuContext>(*param, sph::GpuContext::MIRROR);
//   timestep = std::make_shared<sph::GpuTimeStep>(gpu);       // TimeStep
//   pre      = std::make_shared<sph::GpuPreInteraction>(gpu); // (disph/gsph/...)::PreInteraction
//   fforce   = std::make_shared<sph::GpuFluidForce>(gpu);     // (disph/gsph/...)::FluidForce
//   gforce   = std::make_shared<sph::GpuGravityForce>(gpu);   // GravityForce
//   ... Simulation::make_tree()  ->  gpu->make_tree(*sim)
//
// Particle sync.  The reference keeps its particles in the AoS
// Simulation::particles (include/particle.hpp); the library keeps them on the
// device in octree order.  Two ways to keep both sides consistent:
//
//   MIRROR    Solver::predict / correct stay on the host, unchanged.  The
//             device state is refreshed from the host particles at the first
//             GPU call after host code changed them (make_tree, right after
//             predict), and GpuGravityForce, the last module before correct,
//             copies the modules' outputs back into the particles.  One upload
//             and one download per step; the host copy is current whenever
//             host code runs.
//   RESIDENT  predict / correct run on the device too (gpu->predict(*sim),
//             gpu->correct(*sim) in place of Solver::predict / correct); the
//             particles stay on the device and are copied back only when the
//             host asks (gpu->to_host(*sim): snapshots, energies, output).
//
// In both modes the first GPU call uploads the initial conditions; the
// smoothing-length initialisation of the first PreInteraction call
// (PreInteraction::m_first, src/pre_interaction.cpp:41-44) runs once per
// context, not once per upload.  Fatal status codes throw SPHException through
// THROW_ERROR, as the reference's modules do (include/exception.hpp:9-14).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include <omp.h>

#include "exception.hpp"
#include "module.hpp"
#include "parameters.hpp"
#include "particle.hpp"
#include "simulation.hpp"
#include "sphgpu.h"

namespace sph {

class GpuContext {
public:
    enum Mode { MIRROR, RESIDENT };

    GpuContext(const SPHParameters& p, Mode mode)
        : m_mode(mode),
          m_grad(p.type == SPHType::GSPH || p.type == SPHType::GDISPH || p.type == SPHType::SRGSPH),
          m_sr(p.type == SPHType::SRGSPH)
    {
        const sphgpu_params g = params(p);
        const int rc = sphgpu_create(&g, &m_ctx);
        if(rc < 0) {
            const std::string msg = m_ctx ? sphgpu_last_error(m_ctx) : "sphgpu_create failed";
            sphgpu_destroy(m_ctx);
            m_ctx = nullptr;
            THROW_ERROR(msg);
        }
    }
    ~GpuContext() { sphgpu_destroy(m_ctx); }
    GpuContext(const GpuContext&) = delete;
    GpuContext& operator=(const GpuContext&) = delete;

    sphgpu_ctx* ctx() const { return m_ctx; }
    Mode mode() const { return m_mode; }

    // SPHParameters (include/parameters.hpp:33-91) -> sphgpu_params.
    static sphgpu_params params(const SPHParameters& p)
    {
        sphgpu_params g;
        sphgpu_default_params(&g);
        g.sph_type = p.type == SPHType::DISPH    ? SPHGPU_DISPH
                   : p.type == SPHType::GSPH     ? SPHGPU_GSPH
                   : p.type == SPHType::GDISPH   ? SPHGPU_GDISPH
                   : p.type == SPHType::SRGSPH   ? SPHGPU_SRGSPH : SPHGPU_SSPH;
        g.kernel = p.kernel == KernelType::WENDLAND ? SPHGPU_WENDLAND
                 : p.kernel == KernelType::GAUSSIAN ? SPHGPU_GAUSSIAN : SPHGPU_CUBIC_SPLINE;
        g.neighbor_number = p.physics.neighbor_number;
        g.gamma = p.physics.gamma;
        g.iterative_sml = p.iterative_sml;
        g.cfl_sound = p.cfl.sound;
        g.cfl_force = p.cfl.force;
        g.av_alpha = p.av.alpha;
        g.use_balsara_switch = p.av.use_balsara_switch;
        g.use_time_dependent_av = p.av.use_time_dependent_av;
        g.alpha_max = p.av.alpha_max;
        g.alpha_min = p.av.alpha_min;
        g.epsilon_av = p.av.epsilon;
        g.use_ac = p.ac.is_valid;
        g.alpha_ac = p.ac.alpha;
        g.max_tree_level = p.tree.max_level;
        g.leaf_particle_num = p.tree.leaf_particle_num;
        g.periodic = p.periodic.is_valid;
        for(int k = 0; k < 3; ++k) {
            g.range_min[k] = p.periodic.range_min[k];
            g.range_max[k] = p.periodic.range_max[k];
        }
        g.use_gravity = p.gravity.is_valid;
        g.g_constant = p.gravity.constant;
        g.theta = p.gravity.theta;
        g.gsph_2nd_order = p.gsph.is_2nd_order;
        g.riemann_solver = p.gsph.riemann_solver == RiemannSolverType::ITERATIVE ? SPHGPU_RIEMANN_ITERATIVE
                                                                                   : SPHGPU_RIEMANN_HLL;
        g.sr_2nd_order = p.srgsph.is_2nd_order;
        g.sr_c_speed = p.srgsph.c_speed;
        g.sr_c_shock = p.srgsph.c_shock;
        g.sr_c_cd = p.srgsph.c_cd;
        g.sr_eta = p.srgsph.eta;
        g.sr_c_smooth = p.srgsph.c_smooth;
        // BHTree::make's non-periodic root box covers the origin when OpenMP
        // runs more than one thread (src/bhtree.cpp:68-91): keep the tree the
        // CPU build would make with this process's team size
        g.tree_root_origin = omp_get_max_threads() > 1 ? 1 : 0;
        return g;
    }

    void check(int rc) const
    {
        if(rc < 0) THROW_ERROR(std::string(sphgpu_last_error(m_ctx)));
    }

    // Host particles (and the GSPH gradient arrays, src/solver.cpp:707-719)
    // -> device.  Resets nothing the reference keeps across steps: the
    // smoothing-length initialisation stays done once it has run.
    void to_device(Simulation& sim)
    {
        auto& ps = sim.get_particles();
        const int n = sim.get_particle_num();
        const std::vector<int> up = fields();
        std::vector<double> buf((size_t)n * (up.size() + (m_grad ? 15 : 0)));
        const double* cols[SPHGPU_NFIELDS] = {};
        size_t k = 0;
        for(const int f : up) {
            double* col = buf.data() + k++ * (size_t)n;
            for(int i = 0; i < n; ++i) col[i] = get(ps[i], f);
            cols[f] = col;
        }
        if(m_grad) {
            for(int a = 0; a < 5; ++a) {
                const auto& v = sim.get_vector_array(grad_name(a));
                for(int c = 0; c < 3; ++c) {
                    double* col = buf.data() + k++ * (size_t)n;
                    for(int i = 0; i < n; ++i) col[i] = v[i][c];
                    cols[SPHGPU_F_GRAD_D_X + 3 * a + c] = col;
                }
            }
        }
        check(sphgpu_upload(m_ctx, n, cols));
        check(sphgpu_set_initial_smoothing(m_ctx, m_first ? 1 : 0));
        m_host_newer = false;
        m_uploaded = true;
    }

    // Device -> host particles: every field a module or predict / correct
    // writes (the GSPH gradient arrays too).
    void to_host(Simulation& sim)
    {
        auto& ps = sim.get_particles();
        const int n = sim.get_particle_num();
        const std::vector<int> down = fields();
        std::vector<double> buf((size_t)n * (down.size() + (m_grad ? 15 : 0)));
        double* cols[SPHGPU_NFIELDS] = {};
        size_t k = 0;
        for(const int f : down) cols[f] = buf.data() + k++ * (size_t)n;
        if(m_grad) {
            for(int g = 0; g < 15; ++g) cols[SPHGPU_F_GRAD_D_X + g] = buf.data() + k++ * (size_t)n;
        }
        check(sphgpu_download(m_ctx, cols));
        for(const int f : down) {
            const double* col = cols[f];
            for(int i = 0; i < n; ++i) set(ps[i], f, col[i]);
        }
        if(m_grad) {
            for(int a = 0; a < 5; ++a) {
                auto& v = sim.get_vector_array(grad_name(a));
                for(int c = 0; c < 3; ++c) {
                    const double* col = cols[SPHGPU_F_GRAD_D_X + 3 * a + c];
                    for(int i = 0; i < n; ++i) v[i][c] = col[i];
                }
            }
        }
        m_host_newer = m_mode == MIRROR;  // host code runs next and changes them
    }

    // The device state is current before a module runs.
    void before_module(Simulation& sim)
    {
        if(!m_uploaded || m_host_newer) to_device(sim);
    }

    // Simulation::make_tree (src/simulation.cpp; BHTree::make, src/bhtree.cpp:59-115).
    void make_tree(Simulation& sim)
    {
        before_module(sim);
        check(sphgpu_tree_make(m_ctx));
    }

    // Solver::predict / correct on the device (RESIDENT; src/solver.cpp:1046-1061,
    // 1104-1112), with the dt of the last GpuTimeStep.
    void predict(Simulation& sim)
    {
        before_module(sim);
        check(sphgpu_set_dt(m_ctx, sim.get_dt()));
        check(sphgpu_predict(m_ctx));
    }
    void correct(Simulation& sim)
    {
        before_module(sim);
        check(sphgpu_correct(m_ctx));
    }

    void first_pre_done() { m_first = false; }

private:
    // Fields sent to the device and read back: every per-particle field the
    // modules and predict / correct read or write (SRGSPH state too for
    // SRGSPH contexts).
    std::vector<int> fields() const
    {
        std::vector<int> f = {SPHGPU_F_POS_X, SPHGPU_F_POS_Y, SPHGPU_F_POS_Z, SPHGPU_F_VEL_X, SPHGPU_F_VEL_Y,
                              SPHGPU_F_VEL_Z, SPHGPU_F_VELP_X, SPHGPU_F_VELP_Y, SPHGPU_F_VELP_Z, SPHGPU_F_ACC_X,
                              SPHGPU_F_ACC_Y, SPHGPU_F_ACC_Z, SPHGPU_F_MASS, SPHGPU_F_DENS, SPHGPU_F_PRES,
                              SPHGPU_F_ENE, SPHGPU_F_ENE_P, SPHGPU_F_DENE, SPHGPU_F_SML, SPHGPU_F_SOUND,
                              SPHGPU_F_BALSARA, SPHGPU_F_ALPHA, SPHGPU_F_GRADH, SPHGPU_F_PHI, SPHGPU_F_NEIGHBOR};
        if(m_sr) {
            for(int k = SPHGPU_F_SR_S_X; k <= SPHGPU_F_SR_DE; ++k) f.push_back(k);
        }
        return f;
    }
    static const char* grad_name(int a)
    {
        static const char* names[5] = {"grad_density", "grad_pressure", "grad_velocity_0", "grad_velocity_1",
                                       "grad_velocity_2"};
        return names[a];
    }

    static double get(const SPHParticle& p, int f)
    {
        switch(f) {
        case SPHGPU_F_POS_X: return p.pos[0];
        case SPHGPU_F_POS_Y: return p.pos[1];
        case SPHGPU_F_POS_Z: return p.pos[2];
        case SPHGPU_F_VEL_X: return p.vel[0];
        case SPHGPU_F_VEL_Y: return p.vel[1];
        case SPHGPU_F_VEL_Z: return p.vel[2];
        case SPHGPU_F_VELP_X: return p.vel_p[0];
        case SPHGPU_F_VELP_Y: return p.vel_p[1];
        case SPHGPU_F_VELP_Z: return p.vel_p[2];
        case SPHGPU_F_ACC_X: return p.acc[0];
        case SPHGPU_F_ACC_Y: return p.acc[1];
        case SPHGPU_F_ACC_Z: return p.acc[2];
        case SPHGPU_F_MASS: return p.mass;
        case SPHGPU_F_DENS: return p.dens;
        case SPHGPU_F_PRES: return p.pres;
        case SPHGPU_F_ENE: return p.ene;
        case SPHGPU_F_ENE_P: return p.ene_p;
        case SPHGPU_F_DENE: return p.dene;
        case SPHGPU_F_SML: return p.sml;
        case SPHGPU_F_SOUND: return p.sound;
        case SPHGPU_F_BALSARA: return p.balsara;
        case SPHGPU_F_ALPHA: return p.alpha;
        case SPHGPU_F_GRADH: return p.gradh;
        case SPHGPU_F_PHI: return p.phi;
        case SPHGPU_F_NEIGHBOR: return (double)p.neighbor;
        case SPHGPU_F_SR_S_X: return p.S[0];
        case SPHGPU_F_SR_S_Y: return p.S[1];
        case SPHGPU_F_SR_S_Z: return p.S[2];
        case SPHGPU_F_SR_E: return p.e;
        case SPHGPU_F_SR_N: return p.N;
        case SPHGPU_F_SR_NU: return p.nu;
        case SPHGPU_F_SR_GAMMA_LOR: return p.gamma_lor;
        case SPHGPU_F_SR_ENTHALPY: return p.enthalpy;
        case SPHGPU_F_SR_DS_X: return p.dS[0];
        case SPHGPU_F_SR_DS_Y: return p.dS[1];
        case SPHGPU_F_SR_DS_Z: return p.dS[2];
        case SPHGPU_F_SR_DE: return p.de;
        default: return 0.0;
        }
    }
    static void set(SPHParticle& p, int f, double v)
    {
        switch(f) {
        case SPHGPU_F_POS_X: p.pos[0] = v; break;
        case SPHGPU_F_POS_Y: p.pos[1] = v; break;
        case SPHGPU_F_POS_Z: p.pos[2] = v; break;
        case SPHGPU_F_VEL_X: p.vel[0] = v; break;
        case SPHGPU_F_VEL_Y: p.vel[1] = v; break;
        case SPHGPU_F_VEL_Z: p.vel[2] = v; break;
        case SPHGPU_F_VELP_X: p.vel_p[0] = v; break;
        case SPHGPU_F_VELP_Y: p.vel_p[1] = v; break;
        case SPHGPU_F_VELP_Z: p.vel_p[2] = v; break;
        case SPHGPU_F_ACC_X: p.acc[0] = v; break;
        case SPHGPU_F_ACC_Y: p.acc[1] = v; break;
        case SPHGPU_F_ACC_Z: p.acc[2] = v; break;
        case SPHGPU_F_MASS: p.mass = v; break;
        case SPHGPU_F_DENS: p.dens = v; break;
        case SPHGPU_F_PRES: p.pres = v; break;
        case SPHGPU_F_ENE: p.ene = v; break;
        case SPHGPU_F_ENE_P: p.ene_p = v; break;
        case SPHGPU_F_DENE: p.dene = v; break;
        case SPHGPU_F_SML: p.sml = v; break;
        case SPHGPU_F_SOUND: p.sound = v; break;
        case SPHGPU_F_BALSARA: p.balsara = v; break;
        case SPHGPU_F_ALPHA: p.alpha = v; break;
        case SPHGPU_F_GRADH: p.gradh = v; break;
        case SPHGPU_F_PHI: p.phi = v; break;
        case SPHGPU_F_NEIGHBOR: p.neighbor = (int)v; break;
        case SPHGPU_F_SR_S_X: p.S[0] = v; break;
        case SPHGPU_F_SR_S_Y: p.S[1] = v; break;
        case SPHGPU_F_SR_S_Z: p.S[2] = v; break;
        case SPHGPU_F_SR_E: p.e = v; break;
        case SPHGPU_F_SR_N: p.N = v; break;
        case SPHGPU_F_SR_NU: p.nu = v; break;
        case SPHGPU_F_SR_GAMMA_LOR: p.gamma_lor = v; break;
        case SPHGPU_F_SR_ENTHALPY: p.enthalpy = v; break;
        case SPHGPU_F_SR_DS_X: p.dS[0] = v; break;
        case SPHGPU_F_SR_DS_Y: p.dS[1] = v; break;
        case SPHGPU_F_SR_DS_Z: p.dS[2] = v; break;
        case SPHGPU_F_SR_DE: p.de = v; break;
        default: break;
        }
    }

    sphgpu_ctx* m_ctx = nullptr;
    Mode m_mode;
    bool m_first = true;       // the next PreInteraction call is the first
    bool m_uploaded = false;   // the device holds the particles
    bool m_host_newer = false; // host code may have changed them since
    bool m_grad;               // the Simulation carries the GSPH gradient arrays (src/solver.cpp:707-719)
    bool m_sr;                 // SRGSPH particle state travels too
};

// TimeStep::calculation (src/timestep.cpp:18-38): dt from the acceleration
// and h_per_v_sig the device holds, written to Simulation::dt.
class GpuTimeStep : public Module {
    std::shared_ptr<GpuContext> m_g;

public:
    explicit GpuTimeStep(std::shared_ptr<GpuContext> g) : m_g(std::move(g)) {}
    void initialize(std::shared_ptr<SPHParameters>) override {}
    void calculation(std::shared_ptr<Simulation> sim) override
    {
        // MIRROR: acc, sml and h_per_v_sig are unchanged by correct, so the
        // device copy from the last step is current; no upload here
        if(m_g->mode() == GpuContext::RESIDENT) m_g->before_module(*sim);
        double dt = 0.0;
        m_g->check(sphgpu_timestep(m_g->ctx(), &dt));
        sim->set_dt(dt);
    }
};

// PreInteraction::calculation for the context's SPH type
// (src/pre_interaction.cpp:39-169, src/disph/d_pre_interaction.cpp:21-162,
// src/gsph/g_pre_interaction.cpp:27-144, src/gdisph/gd_pre_interaction.cpp:29-280),
// including BHTree::set_kernel and Simulation::h_per_v_sig.
class GpuPreInteraction : public Module {
    std::shared_ptr<GpuContext> m_g;

public:
    explicit GpuPreInteraction(std::shared_ptr<GpuContext> g) : m_g(std::move(g)) {}
    void initialize(std::shared_ptr<SPHParameters>) override {}
    void calculation(std::shared_ptr<Simulation> sim) override
    {
        m_g->before_module(*sim);
        m_g->check(sphgpu_pre_interaction(m_g->ctx()));
        m_g->first_pre_done();
        double hv = 0.0;
        m_g->check(sphgpu_get_h_per_v_sig(m_g->ctx(), &hv));
        sim->set_h_per_v_sig(hv);
    }
};

// FluidForce::calculation for the context's SPH type (src/fluid_force.cpp:26-116,
// src/disph/d_fluid_force.cpp:26-86, src/gsph/g_fluid_force.cpp:32-304,
// src/gdisph/gd_fluid_force.cpp:45-228): overwrites acc and dene.
class GpuFluidForce : public Module {
    std::shared_ptr<GpuContext> m_g;

public:
    explicit GpuFluidForce(std::shared_ptr<GpuContext> g) : m_g(std::move(g)) {}
    void initialize(std::shared_ptr<SPHParameters>) override {}
    void calculation(std::shared_ptr<Simulation> sim) override
    {
        m_g->before_module(*sim);
        m_g->check(sphgpu_fluid_force(m_g->ctx()));
    }
};

// GravityForce::calculation (src/gravity_force.cpp:52-89): adds the Barnes-Hut
// acceleration and sets phi.  The last module of a step: in MIRROR mode it
// copies the step's results back into the host particles for Solver::correct.
class GpuGravityForce : public Module {
    std::shared_ptr<GpuContext> m_g;

public:
    explicit GpuGravityForce(std::shared_ptr<GpuContext> g) : m_g(std::move(g)) {}
    void initialize(std::shared_ptr<SPHParameters>) override {}
    void calculation(std::shared_ptr<Simulation> sim) override
    {
        m_g->before_module(*sim);
        m_g->check(sphgpu_gravity_force(m_g->ctx()));
        if(m_g->mode() == GpuContext::MIRROR) m_g->to_host(*sim);
    }
};

}  // namespace sph
