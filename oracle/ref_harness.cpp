// ref_harness.cpp — C ABI around the reference's own hot-path modules.
//
// Test and baseline infrastructure only: this file is compiled together with
// the reference's unmodified sources (src/bhtree.cpp, src/pre_interaction.cpp,
// src/fluid_force.cpp, src/gravity_force.cpp, src/timestep.cpp,
// src/simulation.cpp, src/exhaustive_search.cpp, src/disph/*.cpp,
// src/gsph/*.cpp, src/gdisph/*.cpp, src/relaxation/*.cpp) by oracle/Makefile into oracle/_ref/libsphref.so (tree
// search) and oracle/_ref/libsphref_exh.so (-DEXHAUSTIVE_SEARCH).  It is the
// checker the CPU restatement (oracle/sph_oracle.cpp) and the GPU path are
// compared with, and the CPU baseline that bench.py --impl reference times.
//
// Solver.cpp needs boost and HDF5, which this image lacks, so the few lines of
// Solver::initialize / integrate / predict / correct / compute_total_energies
// that drive the modules are restated here (src/solver.cpp:941-978,
// 1046-1061, 1104-1112, 1149-1175).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "parameters.hpp"
#include "simulation.hpp"
#include "particle.hpp"
#include "periodic.hpp"
#include "bhtree.hpp"
#include "pre_interaction.hpp"
#include "fluid_force.hpp"
#include "gravity_force.hpp"
#include "timestep.hpp"
#include "disph/d_pre_interaction.hpp"
#include "disph/d_fluid_force.hpp"
#include "gsph/g_pre_interaction.hpp"
#include "gsph/g_fluid_force.hpp"
#include "gdisph/gd_pre_interaction.hpp"
#include "gdisph/gd_fluid_force.hpp"
#include "exhaustive_search.hpp"
#include "exception.hpp"
#include "relaxation/lane_emden_relaxation.hpp"
#include "srgsph/sr_pre_interaction.hpp"
#include "srgsph/sr_fluid_force.hpp"
#include "srgsph/sr_timestep.hpp"
#include "srgsph/sr_primitive_recovery.hpp"
#include <omp.h>

#include <unistd.h>

#include "sphgpu.h"
#ifdef SPHGPU_SWAP
// libsphref_gpu.so: the same Solver sequence with the GPU modules of
// sph-code-simulation_b200/host/gpu_modules.hpp swapped in for TimeStep,
// PreInteraction, FluidForce, GravityForce and Simulation::make_tree
#include "gpu_modules.hpp"
#endif

using namespace sph;

namespace {

struct RefCtx {
    std::shared_ptr<SPHParameters> param;
    std::shared_ptr<Simulation> sim;
    std::shared_ptr<Module> timestep, pre, fforce, gforce;
    std::shared_ptr<LaneEmdenRelaxation> relax;
    std::string err;
    double t_module[8] = {0};  // seconds: timestep, predict, tree, pre, force, gravity, correct, total
#ifdef SPHGPU_SWAP
    std::shared_ptr<GpuContext> gpu;
#endif
};

#ifdef SPHGPU_SWAP
int g_swap_resident = 0;  // 0: MIRROR (host predict / correct), 1: RESIDENT

void make_tree(RefCtx& c) { c.gpu->make_tree(*c.sim); }
#else
void make_tree(RefCtx& c) { c.sim->make_tree(); }
#endif

std::shared_ptr<SPHParameters> to_param(const sphgpu_params* p)
{
    auto q = std::make_shared<SPHParameters>();
    std::memset(q.get(), 0, sizeof(SPHParameters));
    q->time.start = 0.0;
    q->time.end = 1.0;
    q->type = p->sph_type == SPHGPU_DISPH  ? SPHType::DISPH
            : p->sph_type == SPHGPU_GSPH   ? SPHType::GSPH
            : p->sph_type == SPHGPU_GDISPH ? SPHType::GDISPH
            : p->sph_type == SPHGPU_SRGSPH ? SPHType::SRGSPH : SPHType::SSPH;
    q->cfl.sound = p->cfl_sound;
    q->cfl.force = p->cfl_force;
    q->av.alpha = p->av_alpha;
    q->av.use_balsara_switch = p->use_balsara_switch != 0;
    q->av.use_time_dependent_av = p->use_time_dependent_av != 0;
    q->av.alpha_max = p->alpha_max;
    q->av.alpha_min = p->alpha_min;
    q->av.epsilon = p->epsilon_av;
    q->ac.is_valid = p->use_ac != 0;
    q->ac.alpha = p->alpha_ac;
    q->tree.max_level = p->max_tree_level;
    q->tree.leaf_particle_num = p->leaf_particle_num;
    q->physics.neighbor_number = p->neighbor_number;
    q->physics.gamma = p->gamma;
    q->kernel = p->kernel == SPHGPU_WENDLAND ? KernelType::WENDLAND
              : p->kernel == SPHGPU_GAUSSIAN ? KernelType::GAUSSIAN : KernelType::CUBIC_SPLINE;
    q->iterative_sml = p->iterative_sml != 0;
    q->periodic.is_valid = p->periodic != 0;
    for(int k = 0; k < DIM; ++k) {
        q->periodic.range_min[k] = p->range_min[k];
        q->periodic.range_max[k] = p->range_max[k];
    }
    q->gravity.is_valid = p->use_gravity != 0;
    q->gravity.constant = p->g_constant;
    q->gravity.theta = p->theta;
    q->gsph.is_2nd_order = p->gsph_2nd_order != 0;
    q->gsph.riemann_solver = p->riemann_solver == SPHGPU_RIEMANN_ITERATIVE
        ? RiemannSolverType::ITERATIVE : RiemannSolverType::HLL;
    q->srgsph.is_2nd_order = p->sr_2nd_order != 0;
    q->srgsph.c_speed = p->sr_c_speed;
    q->srgsph.c_shock = p->sr_c_shock;
    q->srgsph.c_cd = p->sr_c_cd;
    q->srgsph.eta = p->sr_eta;
    q->srgsph.c_smooth = p->sr_c_smooth;
    return q;
}

double now()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void store_prim(const RefCtx& c, SPHParticle& p, const srgsph::PrimitiveVariables& q)
{
    const real gamma = c.param->physics.gamma;
    p.vel = q.vel;
    p.ene = q.pressure / ((gamma - 1.0) * q.density);
    p.pres = q.pressure;
    p.dens = q.density;
    p.sound = q.sound_speed;
    p.gamma_lor = q.gamma_lor;
    p.enthalpy = q.enthalpy;
}

// Solver::predict, SRGSPH branch (src/solver.cpp:992-1043; diagnostics left out).
void predict_sr(RefCtx& c)
{
    auto& p = c.sim->get_particles();
    const int num = c.sim->get_particle_num();
    auto* periodic = c.sim->get_periodic().get();
    const real dt = c.sim->get_dt();
    const real gamma = c.param->physics.gamma;
    const real c_speed = c.param->srgsph.c_speed;
    for(int i = 0; i < num; ++i) {
        vec_t S_half = p[i].S + p[i].dS * (0.5 * dt);
        real e_half = p[i].e + p[i].de * (0.5 * dt);
        p[i].S += p[i].dS * dt;
        p[i].e += p[i].de * dt;
        auto prim_half = srgsph::PrimitiveRecovery::conserved_to_primitive(S_half, e_half, p[i].N, gamma, c_speed);
        p[i].pos += prim_half.vel * dt;
        periodic->apply(p[i].pos);
        auto prim_full = srgsph::PrimitiveRecovery::conserved_to_primitive(p[i].S, p[i].e, p[i].N, gamma, c_speed);
        store_prim(c, p[i], prim_full);
        p[i].vel_p = prim_half.vel;
        p[i].ene_p = prim_half.pressure / ((gamma - 1.0) * prim_half.density);
    }
}

// Solver::correct, SRGSPH branch (src/solver.cpp:1075-1102).
void correct_sr(RefCtx& c)
{
    auto& p = c.sim->get_particles();
    const int num = c.sim->get_particle_num();
    const real dt = c.sim->get_dt();
    const real gamma = c.param->physics.gamma;
    const real c_speed = c.param->srgsph.c_speed;
    for(int i = 0; i < num; ++i) {
        vec_t S_half = p[i].S - p[i].dS * (0.5 * dt);
        real e_half = p[i].e - p[i].de * (0.5 * dt);
        p[i].S = S_half + p[i].dS * (0.5 * dt);
        p[i].e = e_half + p[i].de * (0.5 * dt);
        auto prim = srgsph::PrimitiveRecovery::conserved_to_primitive(p[i].S, p[i].e, p[i].N, gamma, c_speed);
        store_prim(c, p[i], prim);
    }
}

// Solver::predict (src/solver.cpp:1046-1061), non-relativistic branch.
void predict(RefCtx& c)
{
    if(c.param->type == SPHType::SRGSPH) return predict_sr(c);
    auto& p = c.sim->get_particles();
    const int num = c.sim->get_particle_num();
    auto* periodic = c.sim->get_periodic().get();
    const real dt = c.sim->get_dt();
    const real gamma = c.param->physics.gamma;
    const real c_sound = gamma * (gamma - 1.0);
#pragma omp parallel for
    for(int i = 0; i < num; ++i) {
        p[i].vel_p = p[i].vel + p[i].acc * (0.5 * dt);
        p[i].ene_p = p[i].ene + p[i].dene * (0.5 * dt);
        p[i].pos += p[i].vel_p * dt;
        p[i].vel += p[i].acc * dt;
        p[i].ene += p[i].dene * dt;
        p[i].sound = std::sqrt(c_sound * p[i].ene);
        periodic->apply(p[i].pos);
    }
}

// Solver::correct (src/solver.cpp:1104-1112), non-relativistic branch.
void correct(RefCtx& c)
{
    if(c.param->type == SPHType::SRGSPH) return correct_sr(c);
    auto& p = c.sim->get_particles();
    const int num = c.sim->get_particle_num();
    const real dt = c.sim->get_dt();
    const real gamma = c.param->physics.gamma;
    const real c_sound = gamma * (gamma - 1.0);
#pragma omp parallel for
    for(int i = 0; i < num; ++i) {
        p[i].vel = p[i].vel_p + p[i].acc * (0.5 * dt);
        p[i].ene = p[i].ene_p + p[i].dene * (0.5 * dt);
        p[i].sound = std::sqrt(c_sound * p[i].ene);
    }
}

// Solver::predict / correct as the swapped-in binding runs them: on the host
// (MIRROR) or on the device (RESIDENT).
void step_predict(RefCtx& c)
{
#ifdef SPHGPU_SWAP
    if(g_swap_resident) return c.gpu->predict(*c.sim);
#endif
    predict(c);
}

void step_correct(RefCtx& c)
{
#ifdef SPHGPU_SWAP
    if(g_swap_resident) return c.gpu->correct(*c.sim);
#endif
    correct(c);
}

// The host particles are current (RESIDENT keeps them on the device).
void host_current(RefCtx& c)
{
#ifdef SPHGPU_SWAP
    if(g_swap_resident) c.gpu->to_host(*c.sim);
#else
    (void)c;
#endif
}

template <typename F>
int guarded(RefCtx* c, F&& f)
{
    try {
        f();
        return 0;
    } catch(SPHException& e) {
        c->err = e.what();
        return -1;
    } catch(std::exception& e) {
        c->err = e.what();
        return -1;
    }
}

double* field_ptr(SPHParticle& p, int k)
{
    switch(k) {
    case SPHGPU_F_POS_X: return &p.pos[0];
    case SPHGPU_F_POS_Y: return &p.pos[1];
    case SPHGPU_F_POS_Z: return &p.pos[2];
    case SPHGPU_F_VEL_X: return &p.vel[0];
    case SPHGPU_F_VEL_Y: return &p.vel[1];
    case SPHGPU_F_VEL_Z: return &p.vel[2];
    case SPHGPU_F_VELP_X: return &p.vel_p[0];
    case SPHGPU_F_VELP_Y: return &p.vel_p[1];
    case SPHGPU_F_VELP_Z: return &p.vel_p[2];
    case SPHGPU_F_ACC_X: return &p.acc[0];
    case SPHGPU_F_ACC_Y: return &p.acc[1];
    case SPHGPU_F_ACC_Z: return &p.acc[2];
    case SPHGPU_F_MASS: return &p.mass;
    case SPHGPU_F_DENS: return &p.dens;
    case SPHGPU_F_PRES: return &p.pres;
    case SPHGPU_F_ENE: return &p.ene;
    case SPHGPU_F_ENE_P: return &p.ene_p;
    case SPHGPU_F_DENE: return &p.dene;
    case SPHGPU_F_SML: return &p.sml;
    case SPHGPU_F_SOUND: return &p.sound;
    case SPHGPU_F_BALSARA: return &p.balsara;
    case SPHGPU_F_ALPHA: return &p.alpha;
    case SPHGPU_F_GRADH: return &p.gradh;
    case SPHGPU_F_PHI: return &p.phi;
    case SPHGPU_F_SR_S_X: return &p.S[0];
    case SPHGPU_F_SR_S_Y: return &p.S[1];
    case SPHGPU_F_SR_S_Z: return &p.S[2];
    case SPHGPU_F_SR_E: return &p.e;
    case SPHGPU_F_SR_N: return &p.N;
    case SPHGPU_F_SR_NU: return &p.nu;
    case SPHGPU_F_SR_GAMMA_LOR: return &p.gamma_lor;
    case SPHGPU_F_SR_ENTHALPY: return &p.enthalpy;
    case SPHGPU_F_SR_DS_X: return &p.dS[0];
    case SPHGPU_F_SR_DS_Y: return &p.dS[1];
    case SPHGPU_F_SR_DS_Z: return &p.dS[2];
    case SPHGPU_F_SR_DE: return &p.de;
    default: return nullptr;
    }
}

const char* grad_names[5] = {"grad_density", "grad_pressure", "grad_velocity_0",
                             "grad_velocity_1", "grad_velocity_2"};

}  // namespace

extern "C" {

// Simulation(param) + module construction (src/solver.cpp:686-723).
void* ref_create(const sphgpu_params* p, int64_t n, const double* const* fields)
{
    auto* c = new RefCtx;
    c->param = to_param(p);
    c->sim = std::make_shared<Simulation>(c->param);
    std::vector<SPHParticle> parts(n);
    for(int64_t i = 0; i < n; ++i) {
        for(int k = 0; k < SPHGPU_NFIELDS; ++k) {
            double* d = field_ptr(parts[i], k);
            if(d) *d = fields && fields[k] ? fields[k][i] : 0.0;
        }
        parts[i].neighbor = 0;
        parts[i].id = (int)i;
    }
    c->sim->set_particles(parts);
    c->sim->set_particle_num((int)n);
    c->timestep = std::make_shared<TimeStep>();
    if(c->param->type == SPHType::DISPH) {
        c->pre = std::make_shared<disph::PreInteraction>();
        c->fforce = std::make_shared<disph::FluidForce>();
    } else if(c->param->type == SPHType::GSPH) {
        c->pre = std::make_shared<gsph::PreInteraction>();
        c->fforce = std::make_shared<gsph::FluidForce>();
        std::vector<std::string> names(grad_names, grad_names + 5);
        c->sim->add_vector_array(names);
    } else if(c->param->type == SPHType::GDISPH) {
        c->pre = std::make_shared<gdisph::PreInteraction>();
        c->fforce = std::make_shared<gdisph::FluidForce>();
        std::vector<std::string> names(grad_names, grad_names + 5);
        c->sim->add_vector_array(names);
    } else if(c->param->type == SPHType::SRGSPH) {
        // src/solver.cpp:699-719; the pre-interaction's particle loop reads
        // neighbours' N while it updates its own, so the harness runs it on
        // one thread (index order)
        c->timestep = std::make_shared<srgsph::TimeStep>();
        c->pre = std::make_shared<srgsph::PreInteraction>();
        c->fforce = std::make_shared<srgsph::FluidForce>();
        std::vector<std::string> names(grad_names, grad_names + 5);
        c->sim->add_vector_array(names);
        omp_set_num_threads(1);
    } else {
        c->pre = std::make_shared<PreInteraction>();
        c->fforce = std::make_shared<FluidForce>();
    }
    c->gforce = std::make_shared<GravityForce>();
#ifdef SPHGPU_SWAP
    try {
        c->gpu = std::make_shared<GpuContext>(*c->param, g_swap_resident ? GpuContext::RESIDENT : GpuContext::MIRROR);
    } catch(SPHException&) {  // no usable device
        delete c;
        return nullptr;
    }
    c->timestep = std::make_shared<GpuTimeStep>(c->gpu);
    c->pre = std::make_shared<GpuPreInteraction>(c->gpu);
    c->fforce = std::make_shared<GpuFluidForce>(c->gpu);
    c->gforce = std::make_shared<GpuGravityForce>(c->gpu);
#endif
    c->timestep->initialize(c->param);
    c->pre->initialize(c->param);
    c->fforce->initialize(c->param);
    c->gforce->initialize(c->param);
    c->sim->get_tree()->resize((int)n);
    return c;
}

void ref_destroy(void* h) { delete static_cast<RefCtx*>(h); }

// OpenMP team size of the modules.  BHTree::make's bounding box depends on it
// (more than one thread: the box also covers the origin), and the SRGSPH
// context sets it to 1 for the whole process.
void ref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
// libsphref_gpu.so: how the swapped-in GPU modules keep the particles
// (0 = MIRROR, 1 = RESIDENT); returns -1 in the CPU-only builds.
int ref_set_swap_mode(int resident)
{
#ifdef SPHGPU_SWAP
    g_swap_resident = resident ? 1 : 0;
    return 0;
#else
    (void)resident;
    return -1;
#endif
}
int ref_max_threads(void) { return omp_get_max_threads(); }

const char* ref_last_error(void* h) { return static_cast<RefCtx*>(h)->err.c_str(); }

int ref_get(void* h, double* const* fields)
{
    auto* c = static_cast<RefCtx*>(h);
    auto& parts = c->sim->get_particles();
    const int n = c->sim->get_particle_num();
    for(int i = 0; i < n; ++i) {
        for(int k = 0; k < SPHGPU_F_NEIGHBOR; ++k) {
            if(fields[k]) fields[k][i] = *field_ptr(parts[i], k);
        }
        if(fields[SPHGPU_F_NEIGHBOR]) fields[SPHGPU_F_NEIGHBOR][i] = parts[i].neighbor;
    }
    for(int k = SPHGPU_F_SR_S_X; k < SPHGPU_NFIELDS; ++k) {
        if(!fields[k]) continue;
        for(int i = 0; i < n; ++i) fields[k][i] = *field_ptr(parts[i], k);
    }
    if(c->param->type == SPHType::GSPH || c->param->type == SPHType::GDISPH || c->param->type == SPHType::SRGSPH) {
        for(int g = 0; g < 5; ++g) {
            auto& arr = c->sim->get_vector_array(grad_names[g]);
            for(int d = 0; d < 3; ++d) {
                double* out = fields[SPHGPU_F_GRAD_D_X + 3 * g + d];
                if(!out) continue;
                for(int i = 0; i < n; ++i) out[i] = arr[i][d];
            }
        }
    }
    return 0;
}

int ref_set(void* h, const double* const* fields)
{
    auto* c = static_cast<RefCtx*>(h);
    auto& parts = c->sim->get_particles();
    const int n = c->sim->get_particle_num();
    for(int i = 0; i < n; ++i) {
        for(int k = 0; k < SPHGPU_NFIELDS; ++k) {
            double* d = field_ptr(parts[i], k);
            if(d && fields[k]) *d = fields[k][i];
        }
    }
    return 0;
}

double ref_get_dt(void* h) { return static_cast<RefCtx*>(h)->sim->get_dt(); }
double ref_get_time(void* h) { return static_cast<RefCtx*>(h)->sim->get_time(); }
void ref_set_dt(void* h, double dt) { static_cast<RefCtx*>(h)->sim->set_dt(dt); }
double ref_get_h_per_v_sig(void* h) { return static_cast<RefCtx*>(h)->sim->get_h_per_v_sig(); }

int ref_tree_make(void* h)
{
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&] { c->sim->make_tree(); });
}
int ref_set_kernel(void* h)
{
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&] { c->sim->get_tree()->set_kernel(); });
}
int ref_pre(void* h)
{
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&] { c->pre->calculation(c->sim); });
}
int ref_force(void* h)
{
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&] { c->fforce->calculation(c->sim); });
}
int ref_gravity(void* h)
{
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&] { c->gforce->calculation(c->sim); });
}
int ref_timestep(void* h)
{
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&] { c->timestep->calculation(c->sim); });
}
int ref_predict(void* h)
{
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&] { predict(*c); });
}
int ref_correct(void* h)
{
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&] { correct(*c); });
}

// Tail of Solver::initialize (src/solver.cpp:941-964).
int ref_initialize(void* h)
{
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&] {
        auto& p = c->sim->get_particles();
        const int num = c->sim->get_particle_num();
        const real gamma = c->param->physics.gamma;
        const real c_sound = gamma * (gamma - 1.0);
        const real alpha = c->param->av.alpha;
        for(int i = 0; i < num; ++i) {
            p[i].alpha = alpha;
            p[i].balsara = 1.0;
            p[i].sound = std::sqrt(c_sound * p[i].ene);
        }
#ifndef EXHAUSTIVE_SEARCH
        make_tree(*c);
#endif
        c->pre->calculation(c->sim);
        c->fforce->calculation(c->sim);
        c->gforce->calculation(c->sim);
        host_current(*c);
    });
}

// Solver::integrate (src/solver.cpp:966-978) + Simulation::update_time,
// timing each module.
int ref_integrate(void* h)
{
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&] {
        double t0 = now(), t1;
        c->timestep->calculation(c->sim);
        t1 = now(); c->t_module[0] += t1 - t0; t0 = t1;
        step_predict(*c);
        t1 = now(); c->t_module[1] += t1 - t0; t0 = t1;
#ifndef EXHAUSTIVE_SEARCH
        make_tree(*c);
#endif
        t1 = now(); c->t_module[2] += t1 - t0; t0 = t1;
        c->pre->calculation(c->sim);
        t1 = now(); c->t_module[3] += t1 - t0; t0 = t1;
        c->fforce->calculation(c->sim);
        t1 = now(); c->t_module[4] += t1 - t0; t0 = t1;
        c->gforce->calculation(c->sim);
        t1 = now(); c->t_module[5] += t1 - t0; t0 = t1;
        step_correct(*c);
        host_current(*c);
        t1 = now(); c->t_module[6] += t1 - t0;
        c->sim->update_time();
    });
}

// One step of Solver's Lane-Emden relaxation loop (src/solver.cpp:779-829;
// progress bar and snapshots left out).  The first call sets up
// LaneEmdenRelaxation (it reads data/lane_emden/n1.5_3d.dat relative to the
// working directory, so the call switches into `refdir` for that) and the
// sound speeds, as src/solver.cpp:726-756 does before the loop.
int ref_relax_step(void* h, const char* refdir, double alpha, double rho_c, double K, double R, double M,
                   double* dt_relax)
{
    auto* c = static_cast<RefCtx*>(h);
    return guarded(c, [&] {
        auto& particles = c->sim->get_particles();
        const int num = c->sim->get_particle_num();
        if(!c->relax) {
            c->relax = std::make_shared<LaneEmdenRelaxation>();
            LaneEmdenRelaxationParams rp;
            rp.alpha_scaling = alpha;
            rp.rho_center = rho_c;
            rp.K = K;
            rp.R = R;
            rp.M_total = M;
            rp.G = c->param->gravity.constant;
            rp.gamma = c->param->physics.gamma;
            char cwd[4096];
            if(!getcwd(cwd, sizeof(cwd)) || chdir(refdir) != 0) THROW_ERROR("cannot enter the reference tree");
            c->relax->initialize(rp);
            if(chdir(cwd) != 0) THROW_ERROR("cannot return to the working directory");
            const real gamma = c->param->physics.gamma;
            const real c_sound_factor = gamma * (gamma - 1.0);
            for(int i = 0; i < num; ++i) particles[i].sound = std::sqrt(c_sound_factor * particles[i].ene);
        }
        c->sim->make_tree();
        c->pre->calculation(c->sim);
        c->fforce->calculation(c->sim);
        if(c->param->gravity.is_valid) c->gforce->calculation(c->sim);
        c->relax->apply_relaxation(c->sim, 0.0);
        c->timestep->calculation(c->sim);
        real dt = c->sim->get_dt();
        dt *= 0.1;
        auto* periodic = c->sim->get_periodic().get();
        for(int i = 0; i < num; ++i) {
            particles[i].vel[0] = 0.0;
            particles[i].vel[1] = 0.0;
            particles[i].vel[2] = 0.0;
            particles[i].pos[0] += 0.5 * particles[i].acc[0] * dt * dt;
            particles[i].pos[1] += 0.5 * particles[i].acc[1] * dt * dt;
            particles[i].pos[2] += 0.5 * particles[i].acc[2] * dt * dt;
            periodic->apply(particles[i].pos);
        }
        *dt_relax = dt;
    });
}

void ref_module_times(void* h, double* out /* [7] */)
{
    auto* c = static_cast<RefCtx*>(h);
    for(int k = 0; k < 7; ++k) out[k] = c->t_module[k];
}

// Solver::compute_total_energies (src/solver.cpp:1149-1175).
void ref_energies(void* h, double* kinetic, double* thermal, double* potential)
{
    auto* c = static_cast<RefCtx*>(h);
    const auto& particles = c->sim->get_particles();
    const int num = c->sim->get_particle_num();
    const bool use_gravity = c->param->gravity.is_valid;
    real k = 0, t = 0, w = 0;
    for(int i = 0; i < num; ++i) {
        const auto& p = particles[i];
        k += 0.5 * p.mass * inner_product(p.vel, p.vel);
        t += p.mass * p.ene;
        if(use_gravity) w += 0.5 * p.mass * p.phi;
    }
    *kinetic = k;
    *thermal = t;
    *potential = w;
}

// Per-particle neighbour lists exactly as the modules obtain them: the tree
// walk of BHTree::neighbor_search (or exhaustive_search in the
// -DEXHAUSTIVE_SEARCH build), distance-sorted, with radius p.sml.
// offsets[n+1]; ids may be NULL to size.  Returns 0 or -1 (capacity).
int ref_neighbor_lists(void* h, int is_ij, int64_t* offsets, int32_t* ids, int64_t cap)
{
    auto* c = static_cast<RefCtx*>(h);
    auto& parts = c->sim->get_particles();
    const int n = c->sim->get_particle_num();
    const int nngb = c->param->physics.neighbor_number;
    std::vector<std::vector<int>> lists(n);
    int rc = guarded(c, [&] {
#pragma omp parallel for
        for(int i = 0; i < n; ++i) {
            std::vector<int> nl(nngb * neighbor_list_size);
#ifdef EXHAUSTIVE_SEARCH
            const int cnt = exhaustive_search(parts[i], parts[i].sml, parts, n, nl,
                                              nngb * neighbor_list_size,
                                              c->sim->get_periodic().get(), is_ij != 0);
#else
            const int cnt = c->sim->get_tree()->neighbor_search(parts[i], nl, parts, is_ij != 0);
#endif
            lists[i].assign(nl.begin(), nl.begin() + cnt);
        }
    });
    if(rc) return rc;
    offsets[0] = 0;
    for(int i = 0; i < n; ++i) offsets[i + 1] = offsets[i] + (int64_t)lists[i].size();
    if(!ids) return 0;
    if(offsets[n] > cap) return -1;
    for(int i = 0; i < n; ++i) {
        std::copy(lists[i].begin(), lists[i].end(), ids + offsets[i]);
    }
    return 0;
}

int ref_is_exhaustive(void)
{
#ifdef EXHAUSTIVE_SEARCH
    return 1;
#else
    return 0;
#endif
}

}  // extern "C"
