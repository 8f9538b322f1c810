// Drives the C++ host mirror (sph::gpu, host/sphgpu.hpp) the way the
// reference's Solver drives its modules: Evrard sphere, initialize, two
// integrate steps, energies.  Exit code 0 on success; without a device the
// Simulation constructor must throw (exit code 3).
#include <cmath>
#include <cstdio>
#include <vector>

#include "sphgpu.hpp"

int main()
{
    using namespace sph::gpu;
    sphgpu_params p = default_parameters();
    p.use_gravity = 1;
    p.neighbor_number = 50;
    std::shared_ptr<Simulation> sim;
    try {
        sim = std::make_shared<Simulation>(p);
    } catch(const SPHException& e) {
        std::printf("no device: %s\n", e.what());
        return 3;
    }
    const int64_t n = sphgpu_sample_evrard(12, 1.0, p.gamma, nullptr);
    std::vector<std::vector<double>> cols(SPHGPU_NFIELDS, std::vector<double>((size_t)n));
    std::vector<double*> ptrs(SPHGPU_NFIELDS);
    for(int k = 0; k < SPHGPU_NFIELDS; ++k) ptrs[k] = cols[k].data();
    sphgpu_sample_evrard(12, 1.0, p.gamma, ptrs.data());
    std::vector<SPHParticle> ps((size_t)n);
    for(int64_t i = 0; i < n; ++i) {
        for(int k = 0; k < 3; ++k) ps[i].pos[k] = cols[SPHGPU_F_POS_X + k][i];
        ps[i].mass = cols[SPHGPU_F_MASS][i];
        ps[i].dens = cols[SPHGPU_F_DENS][i];
        ps[i].ene = cols[SPHGPU_F_ENE][i];
        ps[i].pres = cols[SPHGPU_F_PRES][i];
    }
    sim->set_particles(ps);
    initialize(sim);
    TimeStep ts;
    PreInteraction pre;
    FluidForce ff;
    GravityForce gf;
    for(int s = 0; s < 2; ++s) {  // Solver::integrate through the modules
        ts.calculation(sim);
        sim->check(sphgpu_predict(sim->ctx()));
        sim->make_tree();
        pre.calculation(sim);
        ff.calculation(sim);
        gf.calculation(sim);
        sim->check(sphgpu_correct(sim->ctx()));
    }
    std::vector<int> list;
    const int cnt = sim->get_tree()->neighbor_search(0, list, false);
    const auto out = sim->get_particles();
    double k = 0, u = 0, w = 0;
    sim->check(sphgpu_energies(sim->ctx(), &k, &u, &w, nullptr));
    std::printf("n=%lld neighbours(0)=%d E=%.9f dens0=%.6f\n", (long long)n, cnt, k + u + w, out[0].dens);
    return (cnt > 0 && std::isfinite(k + u + w) && out[0].dens > 0) ? 0 : 1;
}
