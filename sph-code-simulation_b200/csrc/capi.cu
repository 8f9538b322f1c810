// capi.cu — the extern "C" boundary declared in include/sphgpu.h.
//
// Owns the context lifetime, device allocations, host <-> device transfer
// (caller order <-> octree order) and the module sequencing of
// Solver::initialize / Solver::integrate (src/solver.cpp:941-978).
#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "context.cuh"
#include "mlp.cuh"

namespace sphgpu {

int fail(sphgpu_ctx* c, int code, const std::string& msg)
{
    if(c) c->err = msg;
    return code;
}

int cuda_fail(sphgpu_ctx* c, cudaError_t e, const char* where)
{
    std::string m = std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e);
    return fail(c, SPHGPU_ERR_CUDA, m);
}

int check_pass_guard(sphgpu_ctx* c)
{
    const int bits = c->h_status.pass_guard;
    if(!bits) return SPHGPU_OK;
    c->h_status.pass_guard = 0;
    SPHGPU_CUDA(c, cudaMemsetAsync(&c->d_status->pass_guard, 0, sizeof(int), c->stream));
    std::string m = "a bounded device pass hit its limit (corrupt tree):";
    if(bits & PASS_GUARD_MASS) m += " mass / centre of mass";
    if(bits & PASS_GUARD_KSIZE) m += " set_kernel";
    if(bits & PASS_GUARD_GRAVITY) m += " gravity walk";
    if(bits & PASS_GUARD_GRAVITY32) m += " mixed gravity walk";
    return fail(c, SPHGPU_ERR_STATE, m);
}

int sync_and_check(sphgpu_ctx* c)
{
    if(c->d_status)
        SPHGPU_CUDA(c, cudaMemcpyAsync(&c->h_status.pass_guard, &c->d_status->pass_guard, sizeof(int),
                                       cudaMemcpyDeviceToHost, c->stream));
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    return c->d_status ? check_pass_guard(c) : SPHGPU_OK;
}

static cudaEvent_t take_event(sphgpu_ctx* c)
{
    if(c->ev_pool.empty()) {
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
}

void stage_begin(sphgpu_ctx* c, int stage)
{
    if(!c->timing) return;
    c->open_ev[stage] = take_event(c);
    cudaEventRecord(c->open_ev[stage], c->stream);
}

void stage_end(sphgpu_ctx* c, int stage, int launches)
{
    c->stage_launch[stage] += launches;
    c->launches += launches;
    if(!c->timing || !c->open_ev[stage]) return;
    cudaEvent_t b = take_event(c);
    cudaEventRecord(b, c->stream);
    c->pending.push_back({stage, c->open_ev[stage], b});
    c->open_ev[stage] = nullptr;
}

void stage_flush(sphgpu_ctx* c)
{
    for(auto& p : c->pending) {
        float ms = 0.f;
        if(cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) c->stage_ms[p.stage] += ms;
        c->ev_pool.push_back(p.a);
        c->ev_pool.push_back(p.b);
    }
    c->pending.clear();
}

int ensure_list_capacity(sphgpu_ctx* c, int which, int64_t cap)
{
    int*& list = which == 0 ? c->d_glist : c->d_plist;
    int64_t& cur = which == 0 ? c->gcap : c->pcap;
    if(cap <= cur && list) return SPHGPU_OK;
    if(which == 0) c->skin_valid = false;  // the skin buffers no longer match
    if(list) {
        SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
        SPHGPU_CUDA(c, cudaFree(list));
        list = nullptr;
    }
    const size_t bytes = sizeof(int) * (size_t)c->n * (size_t)cap;
    SPHGPU_CUDA(c, cudaMalloc(&list, std::max<size_t>(bytes, 4)));
    cur = cap;
    return SPHGPU_OK;
}

namespace {

void set_dev_params(sphgpu_ctx* c)
{
    const sphgpu_params& p = c->prm;
    DevParams& d = c->dp;
    d.sph_type = p.sph_type;
    d.kernel = p.kernel;
    d.nngb = p.neighbor_number;
    d.iterative = p.iterative_sml;
    d.gamma = p.gamma;
    d.cfl_sound = p.cfl_sound;
    d.cfl_force = p.cfl_force;
    d.sr_2nd = p.sr_2nd_order;
    d.sr_c = p.sr_c_speed;
    d.sr_c_shock = p.sr_c_shock;
    d.sr_c_cd = p.sr_c_cd;
    d.sr_eta = p.sr_eta;
    d.sr_c_smooth = p.sr_c_smooth;
    d.mixed_acc_tol = p.mixed_acc_tol;
    d.riemann_tol = p.riemann_tol;
    d.gather_skin = p.gather_skin;
    d.av_alpha = p.av_alpha;
    d.balsara = p.use_balsara_switch;
    d.td_av = p.use_time_dependent_av;
    d.alpha_max = p.alpha_max;
    d.alpha_min = p.alpha_min;
    d.eps_av = p.epsilon_av;
    d.use_ac = p.use_ac;
    d.alpha_ac = p.alpha_ac;
    d.max_level = p.max_tree_level;
    d.leaf_num = p.leaf_particle_num;
    d.periodic = p.periodic;
    d.root_origin = p.tree_root_origin;
    for(int k = 0; k < 3; ++k) {
        d.lo[k] = p.range_min[k];
        d.hi[k] = p.range_max[k];
        d.range[k] = p.range_max[k] - p.range_min[k];
    }
    d.gravity = p.use_gravity;
    d.G = p.g_constant;
    d.theta = p.theta;
    d.theta2 = p.theta * p.theta;
    d.gsph2 = p.gsph_2nd_order;
    d.riemann = p.riemann_solver;
    d.precision = p.precision;
    d.guess = p.riemann_guess;
    d.mlp_max_newton = p.mlp_max_newton;
    d.ratio = p.iterative_sml ? 1.2 : 1.0;
}

void free_all(sphgpu_ctx* c)
{
    for(void* p : c->state_allocs) cudaFree(p);
    c->state_allocs.clear();
    if(c->d_glist) cudaFree(c->d_glist);
    if(c->d_plist) cudaFree(c->d_plist);
    c->d_glist = c->d_plist = nullptr;
    c->gcap = c->pcap = 0;
    if(c->d_stage) cudaFree(c->d_stage);
    c->d_stage = nullptr;
    c->stage_cap = 0;
    if(c->d_glist_alt) cudaFree(c->d_glist_alt);
    if(c->d_skin) cudaFree(c->d_skin);
    c->d_glist_alt = nullptr;
    c->d_skin = nullptr;
    c->skin_n = 0;
    c->skin_cap = 0;
    c->skin_valid = false;
    c->skin_map_pending = false;
    c->skin_built = false;
    c->skin_since_build = c->skin_idle = c->skin_off = 0;
    c->skin_scale = 1.0;
    c->skin_short = 0;
    c->skin_factor = 1.0;
    c->skin_need = -1.0;
}

template <typename T>
int dalloc(sphgpu_ctx* c, T*& p, size_t count)
{
    void* q = nullptr;
    SPHGPU_CUDA(c, cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 16)));
    c->state_allocs.push_back(q);
    p = static_cast<T*>(q);
    return SPHGPU_OK;
}

int alloc_state(sphgpu_ctx* c, DevState& s, int n)
{
    s.n = n;
    int rc = 0;
    if((rc = dalloc(c, s.pos, n)) || (rc = dalloc(c, s.vel, n)) || (rc = dalloc(c, s.acc, n))
       || (rc = dalloc(c, s.velp, n)) || (rc = dalloc(c, s.thermo, n)) || (rc = dalloc(c, s.visc, n))
       || (rc = dalloc(c, s.grad, 4 * (size_t)n)) || (rc = dalloc(c, s.id, n)) || (rc = dalloc(c, s.nbr, n)))
        return rc;
    s.sr = nullptr;
    if(c->prm.sph_type == SPHGPU_SRGSPH && (rc = dalloc(c, s.sr, 4 * (size_t)n))) return rc;
    return SPHGPU_OK;
}

int alloc_all(sphgpu_ctx* c, int n)
{
    free_all(c);
    c->n = n;
    int rc = 0;
    if((rc = alloc_state(c, c->s, n)) || (rc = alloc_state(c, c->alt, n))) return rc;
    c->node_cap = 5 * n + 2;
    const int nc = c->node_cap;
    if((rc = dalloc(c, c->t.geo, nc)) || (rc = dalloc(c, c->t.mass, nc)) || (rc = dalloc(c, c->t.ksize, nc))
       || (rc = dalloc(c, c->t.link, nc)) || (rc = dalloc(c, c->t.parent, nc)) || (rc = dalloc(c, c->t.nchild, nc))
       || (rc = dalloc(c, c->t.child, 8 * (size_t)nc))
       || (rc = dalloc(c, c->t.counter, nc)) || (rc = dalloc(c, c->t.nnodes, 4))
       || (rc = dalloc(c, c->t.leaf_of, n)) || (rc = dalloc(c, c->t.pks, n)))
        return rc;
    if((rc = dalloc(c, c->d_root, 1)) || (rc = dalloc(c, c->d_bbox_part, 6 * 1024)) || (rc = dalloc(c, c->d_keys, n))
       || (rc = dalloc(c, c->d_keys_alt, n)) || (rc = dalloc(c, c->d_vals, n)) || (rc = dalloc(c, c->d_vals_alt, n))
       || (rc = dalloc(c, c->d_nstart, n)) || (rc = dalloc(c, c->d_base, n)) || (rc = dalloc(c, c->d_lvl, n))
       || (rc = dalloc(c, c->d_leaf_of_start, n)) || (rc = dalloc(c, c->d_inv, n)) || (rc = dalloc(c, c->d_gcount, n))
       || (rc = dalloc(c, c->d_pcount, n)) || (rc = dalloc(c, c->d_dt, 1)) || (rc = dalloc(c, c->d_hvs, 1))
       || (rc = dalloc(c, c->d_red, 8 + 6 * 1024 + 64)) || (rc = dalloc(c, c->d_status, 1)))
        return rc;
    char* rs = nullptr;
    if((rc = dalloc(c, rs, radix_scratch_bytes(n)))) return rc;
    c->d_radix_scratch = rs;
    char* ss = nullptr;
    if((rc = dalloc(c, ss, scan_scratch_bytes(2LL * n + 2)))) return rc;
    c->d_scan_scratch = ss;
    scan_scratch_init(c->scan, ss, 2LL * n + 2);
    const int64_t cap0 = ((int64_t)3 * c->prm.neighbor_number + 31) / 32 * 32;
    if((rc = ensure_list_capacity(c, 0, cap0)) || (rc = ensure_list_capacity(c, 1, cap0))) return rc;
    SPHGPU_CUDA(c, cudaMemsetAsync(c->d_status, 0, sizeof(DevStatus), c->stream));
    const double zero = 0.0, big = DBL_MAX;
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_dt, &zero, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_hvs, &big, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    return SPHGPU_OK;
}

// field -> (array, component); component 4 = int array (nbr)
struct FieldRef {
    double4* arr;
    int comp;
};

FieldRef field_ref(const DevState& s, int f)
{
    const size_t n = (size_t)s.n;
    switch(f) {
    case SPHGPU_F_POS_X: return {s.pos, 0};
    case SPHGPU_F_POS_Y: return {s.pos, 1};
    case SPHGPU_F_POS_Z: return {s.pos, 2};
    case SPHGPU_F_MASS: return {s.pos, 3};
    case SPHGPU_F_VEL_X: return {s.vel, 0};
    case SPHGPU_F_VEL_Y: return {s.vel, 1};
    case SPHGPU_F_VEL_Z: return {s.vel, 2};
    case SPHGPU_F_SML: return {s.vel, 3};
    case SPHGPU_F_ACC_X: return {s.acc, 0};
    case SPHGPU_F_ACC_Y: return {s.acc, 1};
    case SPHGPU_F_ACC_Z: return {s.acc, 2};
    case SPHGPU_F_DENE: return {s.acc, 3};
    case SPHGPU_F_VELP_X: return {s.velp, 0};
    case SPHGPU_F_VELP_Y: return {s.velp, 1};
    case SPHGPU_F_VELP_Z: return {s.velp, 2};
    case SPHGPU_F_ENE_P: return {s.velp, 3};
    case SPHGPU_F_DENS: return {s.thermo, 0};
    case SPHGPU_F_PRES: return {s.thermo, 1};
    case SPHGPU_F_ENE: return {s.thermo, 2};
    case SPHGPU_F_SOUND: return {s.thermo, 3};
    case SPHGPU_F_ALPHA: return {s.visc, 0};
    case SPHGPU_F_BALSARA: return {s.visc, 1};
    case SPHGPU_F_GRADH: return {s.visc, 2};
    case SPHGPU_F_PHI: return {s.visc, 3};
    case SPHGPU_F_NEIGHBOR: return {nullptr, 4};
    case SPHGPU_F_SR_S_X: case SPHGPU_F_SR_S_Y: case SPHGPU_F_SR_S_Z: case SPHGPU_F_SR_E:
        return {s.sr, f - SPHGPU_F_SR_S_X};
    case SPHGPU_F_SR_N: case SPHGPU_F_SR_NU: case SPHGPU_F_SR_GAMMA_LOR: case SPHGPU_F_SR_ENTHALPY:
        return {s.sr ? s.sr + n : nullptr, f - SPHGPU_F_SR_N};
    case SPHGPU_F_SR_DS_X: case SPHGPU_F_SR_DS_Y: case SPHGPU_F_SR_DS_Z: case SPHGPU_F_SR_DE:
        return {s.sr ? s.sr + 2 * n : nullptr, f - SPHGPU_F_SR_DS_X};
    default: {
        const int g = f - SPHGPU_F_GRAD_D_X;
        return {s.grad + (size_t)(g / 4) * n, g % 4};
    }
    }
}

// Device sources of one upload / destinations of one download: a staging slot
// per field, or null (upload: the field is set to 0; download: not read).
struct FieldSlots {
    double* p[SPHGPU_NFIELDS];
};

// Upload: every record of particle i (caller order = octree order until the
// next tree_make) written whole from the staged fields, in one pass.
__global__ void k_put_all(DevState S, FieldSlots F, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    auto g = [&](int f) { return F.p[f] ? F.p[f][i] : 0.0; };
    S.pos[i] = make_double4(g(SPHGPU_F_POS_X), g(SPHGPU_F_POS_Y), g(SPHGPU_F_POS_Z), g(SPHGPU_F_MASS));
    S.vel[i] = make_double4(g(SPHGPU_F_VEL_X), g(SPHGPU_F_VEL_Y), g(SPHGPU_F_VEL_Z), g(SPHGPU_F_SML));
    S.acc[i] = make_double4(g(SPHGPU_F_ACC_X), g(SPHGPU_F_ACC_Y), g(SPHGPU_F_ACC_Z), g(SPHGPU_F_DENE));
    S.velp[i] = make_double4(g(SPHGPU_F_VELP_X), g(SPHGPU_F_VELP_Y), g(SPHGPU_F_VELP_Z), g(SPHGPU_F_ENE_P));
    S.thermo[i] = make_double4(g(SPHGPU_F_DENS), g(SPHGPU_F_PRES), g(SPHGPU_F_ENE), g(SPHGPU_F_SOUND));
    S.visc[i] = make_double4(g(SPHGPU_F_ALPHA), g(SPHGPU_F_BALSARA), g(SPHGPU_F_GRADH), g(SPHGPU_F_PHI));
    S.nbr[i] = (int)g(SPHGPU_F_NEIGHBOR);
    S.id[i] = i;
    const size_t m = (size_t)n;
    for(int q = 0; q < 4; ++q) {
        const int f = SPHGPU_F_GRAD_D_X + 4 * q;
        S.grad[q * m + i] = make_double4(g(f), g(f + 1), g(f + 2), q < 3 ? g(f + 3) : 0.0);
    }
    if(S.sr) {
        for(int q = 0; q < 3; ++q) {
            const int f = SPHGPU_F_SR_S_X + 4 * q;
            S.sr[q * m + i] = make_double4(g(f), g(f + 1), g(f + 2), g(f + 3));
        }
    }
}

// Download: each requested field of particle i into its slot at the caller's
// index id[i], in one pass.
__global__ void k_get_all(DevState S, FieldSlots F, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const int dst = S.id[i];
    auto put1 = [&](int f, double v) {
        if(F.p[f]) F.p[f][dst] = v;
    };
    // a record is read only when one of its fields is requested, so a
    // download of some fields may overlap kernels that write the others
    auto want = [&](int f0, int k) {
        for(int f = f0; f < f0 + k; ++f)
            if(F.p[f]) return true;
        return false;
    };
    auto put4 = [&](int f0, const double4* rec, int fw) {
        if(!want(f0, 3) && !F.p[fw]) return;
        const double4 v = rec[i];
        put1(f0, v.x);
        put1(f0 + 1, v.y);
        put1(f0 + 2, v.z);
        put1(fw, v.w);
    };
    put4(SPHGPU_F_POS_X, S.pos, SPHGPU_F_MASS);
    put4(SPHGPU_F_VEL_X, S.vel, SPHGPU_F_SML);
    put4(SPHGPU_F_ACC_X, S.acc, SPHGPU_F_DENE);
    put4(SPHGPU_F_VELP_X, S.velp, SPHGPU_F_ENE_P);
    if(want(SPHGPU_F_DENS, 1) || want(SPHGPU_F_PRES, 1) || want(SPHGPU_F_ENE, 1) || want(SPHGPU_F_SOUND, 1)) {
        const double4 th = S.thermo[i];
        put1(SPHGPU_F_DENS, th.x);
        put1(SPHGPU_F_PRES, th.y);
        put1(SPHGPU_F_ENE, th.z);
        put1(SPHGPU_F_SOUND, th.w);
    }
    if(want(SPHGPU_F_ALPHA, 1) || want(SPHGPU_F_BALSARA, 1) || want(SPHGPU_F_GRADH, 1) || want(SPHGPU_F_PHI, 1)) {
        const double4 vs = S.visc[i];
        put1(SPHGPU_F_ALPHA, vs.x);
        put1(SPHGPU_F_BALSARA, vs.y);
        put1(SPHGPU_F_GRADH, vs.z);
        put1(SPHGPU_F_PHI, vs.w);
    }
    if(F.p[SPHGPU_F_NEIGHBOR]) put1(SPHGPU_F_NEIGHBOR, (double)S.nbr[i]);
    const size_t m = (size_t)n;
    for(int q = 0; q < 4; ++q) {
        const int f = SPHGPU_F_GRAD_D_X + 4 * q;
        if(!want(f, q < 3 ? 4 : 3)) continue;
        const double4 v = S.grad[q * m + i];
        put1(f, v.x);
        put1(f + 1, v.y);
        put1(f + 2, v.z);
        if(q < 3) put1(f + 3, v.w);
    }
    if(S.sr) {
        for(int q = 0; q < 3; ++q) {
            const int f = SPHGPU_F_SR_S_X + 4 * q;
            if(!want(f, 4)) continue;
            const double4 v = S.sr[q * m + i];
            put1(f, v.x);
            put1(f + 1, v.y);
            put1(f + 2, v.z);
            put1(f + 3, v.w);
        }
    }
}

// sphgpu_integrate_host: the alpha / Balsara / grad-h and density / pressure
// fields uploaded beside the tree build, written once the particles are in
// tree order (slot by the caller index each particle carries)
__global__ void k_put_late(DevState S, FieldSlots F, int n)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const int k = S.id[p];
    double4 v = S.visc[p];
    if(F.p[SPHGPU_F_ALPHA]) v.x = F.p[SPHGPU_F_ALPHA][k];
    if(F.p[SPHGPU_F_BALSARA]) v.y = F.p[SPHGPU_F_BALSARA][k];
    if(F.p[SPHGPU_F_GRADH]) v.z = F.p[SPHGPU_F_GRADH][k];
    S.visc[p] = v;
    if(F.p[SPHGPU_F_DENS] || F.p[SPHGPU_F_PRES]) {
        double4 t = S.thermo[p];
        if(F.p[SPHGPU_F_DENS]) t.x = F.p[SPHGPU_F_DENS][k];
        if(F.p[SPHGPU_F_PRES]) t.y = F.p[SPHGPU_F_PRES][k];
        S.thermo[p] = t;
    }
}

// Staging for `slots` fields of n doubles, grown on demand and kept.
int ensure_stage(sphgpu_ctx* c, int slots)
{
    const int64_t want = (int64_t)slots * c->n;
    if(want <= c->stage_cap && c->d_stage) return SPHGPU_OK;
    if(c->d_stage) {
        SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
        SPHGPU_CUDA(c, cudaFree(c->d_stage));
        c->d_stage = nullptr;
        c->stage_cap = 0;
    }
    SPHGPU_CUDA(c, cudaMalloc(&c->d_stage, sizeof(double) * (size_t)std::max<int64_t>(want, 1)));
    c->stage_cap = want;
    return SPHGPU_OK;
}

// Solver::initialize (src/solver.cpp:941-953)
__global__ void k_init_state(DevState S, int n, double alpha, double cs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    double4 v = S.visc[i];
    v.x = alpha;
    v.y = 1.0;
    S.visc[i] = v;
    double4 t = S.thermo[i];
    t.w = sqrt(cs * t.z);
    S.thermo[i] = t;
}

__global__ void k_iota(int* __restrict__ id, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n) id[i] = i;
}

int check_params(const sphgpu_params* p, std::string& why)
{
    if(p->sph_type < SPHGPU_SSPH || p->sph_type > SPHGPU_SRGSPH)
        return why = "SPH type must be ssph, disph, gsph, gdisph or srgsph", -1;
    if(p->sph_type == SPHGPU_SRGSPH && p->precision != SPHGPU_FP64)
        return why = "srgsph runs in the FP64 form only", -1;
    if(p->sph_type == SPHGPU_SRGSPH && !(p->sr_c_speed > 0.0 && p->sr_eta > 0.0 && p->sr_c_smooth > 0.0))
        return why = "srgsph needs cSpeed, etaSmoothingLength and cSmoothGradient > 0", -1;
    if(p->kernel != SPHGPU_CUBIC_SPLINE && p->kernel != SPHGPU_WENDLAND && p->kernel != SPHGPU_GAUSSIAN)
        return why = "kernel is unknown.", -1;
    if(p->neighbor_number <= 0) return why = "neighborNumber must be positive", -1;
    if(p->max_tree_level < 1 || p->max_tree_level > 21) return why = "maxTreeLevel must be in 1..21", -1;
    if(p->leaf_particle_num < 1) return why = "leafParticleNumber must be >= 1", -1;
    if(p->tree_root_origin != 0 && p->tree_root_origin != 1) return why = "tree_root_origin must be 0 or 1", -1;
    if(p->periodic) {
        for(int k = 0; k < 3; ++k) {
            if(!(p->range_max[k] > p->range_min[k])) return why = "rangeMax must exceed rangeMin", -1;
        }
    }
    if(p->use_time_dependent_av && p->alpha_max < p->alpha_min) return why = "alphaMax < alphaMin", -1;
    if(p->precision != SPHGPU_FP64 && p->precision != SPHGPU_MIXED) return why = "precision must be fp64 or mixed", -1;
    if(!(p->mixed_acc_tol >= 0.0)) return why = "mixed_acc_tol must be >= 0", -1;
    if(!(p->riemann_tol > 0.0 && p->riemann_tol < 1.0)) return why = "riemann_tol must be in (0, 1)", -1;
    if(!(p->gather_skin >= 0.0 && p->gather_skin <= 1.0)) return why = "gather_skin must be in [0, 1]", -1;
    return 0;
}

}  // namespace
}  // namespace sphgpu

using namespace sphgpu;

extern "C" {

void sphgpu_default_params(sphgpu_params* p)
{
    std::memset(p, 0, sizeof(*p));
    p->sph_type = SPHGPU_SSPH;
    p->kernel = SPHGPU_CUBIC_SPLINE;
    p->neighbor_number = 50;
    p->iterative_sml = 1;
    p->gamma = 1.6666666666666667;
    p->cfl_sound = 0.3;
    p->cfl_force = 0.125;
    p->av_alpha = 1.0;
    p->use_balsara_switch = 1;
    p->use_time_dependent_av = 0;
    p->alpha_max = 2.0;
    p->alpha_min = 0.1;
    p->epsilon_av = 0.2;
    p->use_ac = 0;
    p->alpha_ac = 1.0;
    p->max_tree_level = 20;
    p->leaf_particle_num = 1;
    p->periodic = 0;
    p->use_gravity = 0;
    p->g_constant = 1.0;
    p->theta = 0.5;
    p->gsph_2nd_order = 1;
    p->riemann_solver = SPHGPU_RIEMANN_HLL;
    p->precision = SPHGPU_FP64;
    p->riemann_guess = SPHGPU_GUESS_NONE;
    p->mlp_max_newton = 4;
    p->sr_2nd_order = 1;
    p->tree_root_origin = 1;
    p->sr_c_speed = 1.0;
    p->sr_c_shock = 3.0;
    p->sr_c_cd = 1.0;
    p->sr_eta = 1.0;
    p->sr_c_smooth = 2.0;
    p->mixed_acc_tol = 0.0;
    p->riemann_tol = 1e-6;
    p->gather_skin = 0.02;
}

int sphgpu_device_ok(void)
{
    int count = 0;
    if(cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) return 0;
    int dev = 0, major = 0;
    if(cudaGetDevice(&dev) != cudaSuccess) return 0;
    if(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) return 0;
    return major == 10 ? 1 : 0;
}

int sphgpu_create(const sphgpu_params* p, sphgpu_ctx** out)
{
    if(!p || !out) return SPHGPU_ERR_ARG;
    *out = nullptr;
    auto* c = new sphgpu_ctx;
    c->prm = *p;
    std::string why;
    if(check_params(p, why)) {
        c->err = why;
        *out = c;
        return SPHGPU_ERR_ARG;
    }
    set_dev_params(c);
    *out = c;
    if(!sphgpu_device_ok()) return fail(c, SPHGPU_ERR_CUDA, "no usable sm_100 CUDA device");
    SPHGPU_CUDA(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    for(int k = 0; k < 2; ++k) SPHGPU_CUDA(c, cudaEventCreate(&c->user_ev[k]));
    return SPHGPU_OK;
}

int sphgpu_destroy(sphgpu_ctx* c)
{
    if(!c) return SPHGPU_OK;
    if(c->stream) cudaStreamSynchronize(c->stream);
    if(c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
        for(cudaEvent_t e : c->copy_ev) {
            if(e) cudaEventDestroy(e);
        }
    }
    free_all(c);
    if(c->d_mlp) cudaFree(c->d_mlp);
    if(c->d_mlp_master) cudaFree(c->d_mlp_master);
    if(c->d_relax) cudaFree(c->d_relax);
    if(c->d_tcount) cudaFree(c->d_tcount);
    if(c->d_flist_flags) cudaFree(c->d_flist_flags);
    if(c->d_rsearch) cudaFree(c->d_rsearch);
    if(c->d_gnode) cudaFree(c->d_gnode);
    if(c->d_mlp_defer) cudaFree(c->d_mlp_defer);
    if(c->d_harvest) cudaFree(c->d_harvest);
    if(c->d_harvest_count) cudaFree(c->d_harvest_count);
    if(c->d_recheck) cudaFree(c->d_recheck);
    stage_flush(c);
    for(cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    for(cudaEvent_t e : c->user_ev) {
        if(e) cudaEventDestroy(e);
    }
    if(c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return SPHGPU_OK;
}

const char* sphgpu_last_error(const sphgpu_ctx* c) { return c ? c->err.c_str() : "null context"; }

namespace {

// sphgpu_upload; step = true (sphgpu_integrate_host) keeps the simulation
// time and the initial-smoothing flag: the fields continue a run
int upload_impl(sphgpu_ctx* c, int64_t n, const double* const* fields, bool step)
{
    if(!c || n <= 0 || n > SPHGPU_MAX_PARTICLES)
        return fail(c, SPHGPU_ERR_ARG, "particle count out of range (1 .. SPHGPU_MAX_PARTICLES)");
    if(!c->stream) return fail(c, SPHGPU_ERR_CUDA, "context has no device");
    if((int)n != c->n || !c->s.pos) {
        int rc = alloc_all(c, (int)n);
        if(rc) return rc;
    }
    // every given field to its own staging slot (back-to-back copies on the
    // stream: DMA at the link rate from pinned buffers), then one pass that
    // writes every particle record whole
    // (srgsph fields are kept only by srgsph contexts)
    auto wanted = [&](int f) { return fields && fields[f] && (f < SPHGPU_F_SR_S_X || c->s.sr); };
    int slots = 0;
    for(int f = 0; f < SPHGPU_NFIELDS; ++f) slots += wanted(f) ? 1 : 0;
    int rc = ensure_stage(c, slots);
    if(rc) return rc;
    FieldSlots F{};
    int k = 0;
    for(int f = 0; f < SPHGPU_NFIELDS; ++f) {
        if(!wanted(f)) continue;
        F.p[f] = c->d_stage + (size_t)k++ * (size_t)n;
        SPHGPU_CUDA(c, cudaMemcpyAsync(F.p[f], fields[f], sizeof(double) * (size_t)n, cudaMemcpyHostToDevice,
                                       c->stream));
    }
    k_put_all<<<grid_for(n, 256), 256, 0, c->stream>>>(c->s, F, (int)n);
    SPHGPU_LAUNCH_CHECK(c, "upload");
    // skin lists stay valid across an upload of the same particle count:
    // their rows follow the particles into caller order at the next tree
    // build, and the displacement check against their build positions holds
    // whatever the uploaded positions are
    if((rc = skin_upload(c)) < 0) return rc;
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    c->have_tree = false;
    c->flist_ready = false;
    if(!step) {
        c->first_pre = true;
        c->time = 0.0;
    }
    return SPHGPU_OK;
}

}  // namespace

int sphgpu_upload(sphgpu_ctx* c, int64_t n, const double* const* fields)
{
    return upload_impl(c, n, fields, false);
}

int sphgpu_download(sphgpu_ctx* c, double* const* fields)
{
    if(!c || !fields) return SPHGPU_ERR_ARG;
    if(c->n <= 0) return fail(c, SPHGPU_ERR_STATE, "no particles uploaded");
    const int n = c->n;
    int slots = 0;
    for(int f = 0; f < SPHGPU_NFIELDS; ++f) {
        if(!fields[f]) continue;
        if(f >= SPHGPU_F_SR_S_X && !c->s.sr) {  // srgsph fields of another SPH type: zeros
            std::fill(fields[f], fields[f] + n, 0.0);
            continue;
        }
        ++slots;
    }
    int rc = ensure_stage(c, slots);
    if(rc) return rc;
    FieldSlots F{};
    int k = 0;
    for(int f = 0; f < SPHGPU_NFIELDS; ++f) {
        if(!fields[f] || (f >= SPHGPU_F_SR_S_X && !c->s.sr)) continue;
        F.p[f] = c->d_stage + (size_t)k++ * (size_t)n;
    }
    // one pass fills every requested slot in caller order, then the slots go
    // back to back over the link; one wait at the end
    k_get_all<<<grid_for(n, 256), 256, 0, c->stream>>>(c->s, F, n);
    SPHGPU_LAUNCH_CHECK(c, "download");
    for(int f = 0; f < SPHGPU_NFIELDS; ++f) {
        if(!F.p[f]) continue;
        SPHGPU_CUDA(c, cudaMemcpyAsync(fields[f], F.p[f], sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost,
                                       c->stream));
    }
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    return SPHGPU_OK;
}

int64_t sphgpu_particle_num(const sphgpu_ctx* c) { return c ? c->n : 0; }

int sphgpu_get_time(const sphgpu_ctx* c, double* time, double* dt)
{
    if(!c) return SPHGPU_ERR_ARG;
    if(time) *time = c->time;
    if(dt) {
        if(!c->d_dt) {
            *dt = 0.0;
        } else {
            cudaStreamSynchronize(c->stream);
            if(cudaMemcpy(dt, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return SPHGPU_ERR_CUDA;
        }
    }
    return SPHGPU_OK;
}

int sphgpu_set_dt(sphgpu_ctx* c, double dt)
{
    if(!c || !c->d_dt) return SPHGPU_ERR_ARG;
    SPHGPU_CUDA(c, cudaMemcpyAsync(c->d_dt, &dt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    return SPHGPU_OK;
}

int sphgpu_get_h_per_v_sig(const sphgpu_ctx* c, double* v)
{
    if(!c || !v || !c->d_hvs) return SPHGPU_ERR_ARG;
    cudaStreamSynchronize(c->stream);
    if(cudaMemcpy(v, c->d_hvs, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return SPHGPU_ERR_CUDA;
    return SPHGPU_OK;
}

#define SPHGPU_NEED_STATE(c)                                                              \
    do {                                                                                  \
        if(!(c)) return SPHGPU_ERR_ARG;                                                   \
        if((c)->n <= 0) return sphgpu::fail((c), SPHGPU_ERR_STATE, "no particles uploaded"); \
    } while(0)

int sphgpu_tree_make(sphgpu_ctx* c)
{
    SPHGPU_NEED_STATE(c);
    return tree_make(c);
}

int sphgpu_tree_set_kernel(sphgpu_ctx* c)
{
    SPHGPU_NEED_STATE(c);
    return tree_set_kernel(c);
}

int sphgpu_neighbor_search(sphgpu_ctx* c, int is_ij, int64_t* offsets, int32_t* ids, int64_t cap)
{
    SPHGPU_NEED_STATE(c);
    if(!offsets) return SPHGPU_ERR_ARG;
    const int rc = is_ij ? pair_walk(c) : gather_walk(c, false, 1.0);
    if(rc < 0) return rc;
    return export_lists(c, is_ij ? 1 : 0, offsets, ids, cap);
}

int sphgpu_force_pairs(sphgpu_ctx* c, int64_t* offsets, int32_t* ids, int64_t cap)
{
    SPHGPU_NEED_STATE(c);
    if(!offsets) return SPHGPU_ERR_ARG;
    if(!c->have_tree) return fail(c, SPHGPU_ERR_STATE, "force pairs before tree make");
    const int rc = symmetric_lists(c);
    if(rc < 0) return rc;
    return export_lists(c, 1, offsets, ids, cap);
}

int sphgpu_exhaustive_search(sphgpu_ctx* c, int is_ij, int64_t* offsets, int32_t* ids, int64_t cap)
{
    SPHGPU_NEED_STATE(c);
    if(!offsets) return SPHGPU_ERR_ARG;
    return exhaustive_lists(c, is_ij, offsets, ids, cap);
}

int sphgpu_pre_interaction(sphgpu_ctx* c)
{
    SPHGPU_NEED_STATE(c);
    return pre_interaction(c);
}

int sphgpu_fluid_force(sphgpu_ctx* c)
{
    SPHGPU_NEED_STATE(c);
    return fluid_force(c);
}

int sphgpu_gravity_force(sphgpu_ctx* c)
{
    SPHGPU_NEED_STATE(c);
    return gravity(c, false);
}

int sphgpu_gravity_direct(sphgpu_ctx* c)
{
    SPHGPU_NEED_STATE(c);
    return gravity(c, true);
}

int sphgpu_timestep(sphgpu_ctx* c, double* dt)
{
    SPHGPU_NEED_STATE(c);
    int rc = timestep(c);
    if(rc < 0) return rc;
    if(dt) {
        SPHGPU_CUDA(c, cudaMemcpyAsync(dt, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return SPHGPU_OK;
}

int sphgpu_predict(sphgpu_ctx* c)
{
    SPHGPU_NEED_STATE(c);
    return predict(c);
}

int sphgpu_correct(sphgpu_ctx* c)
{
    SPHGPU_NEED_STATE(c);
    return correct(c);
}

int sphgpu_initialize(sphgpu_ctx* c)
{
    SPHGPU_NEED_STATE(c);
    // alpha = avAlpha, balsara = 1, sound = sqrt(gamma (gamma - 1) u)
    k_init_state<<<grid_for(c->n, 256), 256, 0, c->stream>>>(c->s, c->n, c->prm.av_alpha,
                                                             c->prm.gamma * (c->prm.gamma - 1.0));
    SPHGPU_LAUNCH_CHECK(c, "initialize");
    int rc = tree_make(c);
    if(rc < 0) return rc;
    rc = pre_interaction(c);
    if(rc < 0) return rc;
    rc = fluid_force(c);
    if(rc < 0) return rc;
    rc = gravity(c, false);
    if(rc < 0) return rc;
    return sync_and_check(c);
}

int sphgpu_integrate(sphgpu_ctx* c)
{
    SPHGPU_NEED_STATE(c);
    int rc;
    if((rc = timestep(c)) < 0) return rc;
    double dt_h = 0.0;
    SPHGPU_CUDA(c, cudaMemcpyAsync(&dt_h, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if((rc = predict(c)) < 0) return rc;
    if((rc = tree_make(c)) < 0) return rc;
    if((rc = pre_interaction(c)) < 0) return rc;
    if((rc = fluid_force(c)) < 0) return rc;
    if((rc = gravity(c, false)) < 0) return rc;
    if((rc = correct(c)) < 0) return rc;
    rc = sync_and_check(c);
    stage_flush(c);
    if(rc < 0) return rc;
    c->time += dt_h;
    return SPHGPU_OK;
}

namespace {

// Fields of `out` in group g (0: final after tree_make: positions and mass,
// which only predict moves; 1: final after PreInteraction; 2: the rest, final
// after correct) packed into staging slots from *slot on, and copied to the
// host on stream st.
int download_group(sphgpu_ctx* c, double* const* out, int g, int* slot, cudaStream_t st)
{
    auto group_of = [](int f) {
        if(f == SPHGPU_F_POS_X || f == SPHGPU_F_POS_Y || f == SPHGPU_F_POS_Z || f == SPHGPU_F_MASS) return 0;
        if(f == SPHGPU_F_DENS || f == SPHGPU_F_PRES || f == SPHGPU_F_SML || f == SPHGPU_F_GRADH ||
           f == SPHGPU_F_BALSARA || f == SPHGPU_F_ALPHA || f == SPHGPU_F_NEIGHBOR)
            return 1;
        return 2;
    };
    const int n = c->n;
    FieldSlots F{};
    bool any = false;
    for(int f = 0; f < SPHGPU_NFIELDS; ++f) {
        if(!out[f] || group_of(f) != g || (f >= SPHGPU_F_SR_S_X && !c->s.sr)) continue;
        F.p[f] = c->d_stage + (size_t)(*slot)++ * (size_t)n;
        any = true;
    }
    if(!any) return SPHGPU_OK;
    k_get_all<<<grid_for(n, 256), 256, 0, st>>>(c->s, F, n);
    SPHGPU_LAUNCH_CHECK(c, "integrate_host download");
    for(int f = 0; f < SPHGPU_NFIELDS; ++f) {
        if(!F.p[f]) continue;
        SPHGPU_CUDA(c, cudaMemcpyAsync(out[f], F.p[f], sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, st));
    }
    return SPHGPU_OK;
}

// After event ev on the step's stream, the group's download on the copy stream.
int download_group_after(sphgpu_ctx* c, double* const* out, int g, int* slot, cudaEvent_t ev)
{
    SPHGPU_CUDA(c, cudaEventRecord(ev, c->stream));
    SPHGPU_CUDA(c, cudaStreamWaitEvent(c->copy_stream, ev, 0));
    return download_group(c, out, g, slot, c->copy_stream);
}

int integrate_host_step(sphgpu_ctx* c, double* const* out, double* dt_h, const FieldSlots& late, bool has_late)
{
    int rc, slot = 0;
    if((rc = timestep(c)) < 0) return rc;
    SPHGPU_CUDA(c, cudaMemcpyAsync(dt_h, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if((rc = predict(c)) < 0) return rc;
    if((rc = tree_make(c)) < 0) return rc;
    if(has_late) {
        // the fields PreInteraction reads first arrived beside the tree build
        SPHGPU_CUDA(c, cudaStreamWaitEvent(c->stream, c->copy_ev[2], 0));
        k_put_late<<<grid_for(c->n, 256), 256, 0, c->stream>>>(c->s, late, c->n);
        SPHGPU_LAUNCH_CHECK(c, "integrate_host late fields");
    }
    if((rc = download_group_after(c, out, 0, &slot, c->copy_ev[0])) < 0) return rc;
    if((rc = pre_interaction(c)) < 0) return rc;
    if((rc = download_group_after(c, out, 1, &slot, c->copy_ev[1])) < 0) return rc;
    if((rc = fluid_force(c)) < 0) return rc;
    if((rc = gravity(c, false)) < 0) return rc;
    if((rc = correct(c)) < 0) return rc;
    return download_group(c, out, 2, &slot, c->stream);
}

}  // namespace

int sphgpu_integrate_host(sphgpu_ctx* c, const double* const* in_fields, double* const* out_fields)
{
    SPHGPU_NEED_STATE(c);
    if(!in_fields || !out_fields) return fail(c, SPHGPU_ERR_ARG, "integrate_host: field tables required");
    if(!c->copy_stream) {
        SPHGPU_CUDA(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        for(cudaEvent_t& e : c->copy_ev) SPHGPU_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    int in_slots = 0, out_slots = 0;
    for(int f = 0; f < SPHGPU_NFIELDS; ++f) {
        const bool kept = f < SPHGPU_F_SR_S_X || c->s.sr;
        in_slots += in_fields[f] && kept ? 1 : 0;
        out_slots += out_fields[f] && kept ? 1 : 0;
    }
    int rc = ensure_stage(c, std::max(in_slots, out_slots));
    if(rc) return rc;
    // alpha, Balsara, grad-h, density and pressure are first read by
    // PreInteraction (its gather walk guesses h from the density; TimeStep
    // does not read them and predict carries them unchanged): they go up on
    // the copy stream while the step's first modules run (srgsph contexts
    // take every field before the step)
    const int late_f[5] = {SPHGPU_F_ALPHA, SPHGPU_F_BALSARA, SPHGPU_F_GRADH, SPHGPU_F_DENS, SPHGPU_F_PRES};
    const bool split = c->prm.sph_type != SPHGPU_SRGSPH;
    const double* early[SPHGPU_NFIELDS];
    for(int f = 0; f < SPHGPU_NFIELDS; ++f) early[f] = in_fields[f];
    int n_late = 0;
    if(split) {
        for(int f : late_f) {
            if(in_fields[f]) ++n_late;
            early[f] = nullptr;
        }
    }
    if((rc = upload_impl(c, c->n, early, true)) < 0) return rc;
    FieldSlots late{};
    if(n_late > 0) {
        int k = in_slots - n_late;  // the slots after the early fields'
        for(int f : late_f) {
            if(!in_fields[f]) continue;
            late.p[f] = c->d_stage + (size_t)k++ * (size_t)c->n;
            SPHGPU_CUDA(c, cudaMemcpyAsync(late.p[f], in_fields[f], sizeof(double) * (size_t)c->n,
                                           cudaMemcpyHostToDevice, c->copy_stream));
        }
        SPHGPU_CUDA(c, cudaEventRecord(c->copy_ev[2], c->copy_stream));
    }
    double dt_h = 0.0;
    rc = integrate_host_step(c, out_fields, &dt_h, late, n_late > 0);
    // both streams drain on every path: no copy into the caller's buffers
    // outlives the call
    const cudaError_t e1 = cudaStreamSynchronize(c->copy_stream);
    const int rs = sync_and_check(c);
    stage_flush(c);
    if(rc < 0) return rc;
    if(rs < 0) return rs;
    if(e1 != cudaSuccess) return fail(c, SPHGPU_ERR_CUDA, cudaGetErrorString(e1));
    for(int f = SPHGPU_F_SR_S_X; f < SPHGPU_NFIELDS; ++f)
        if(out_fields[f] && !c->s.sr) std::fill(out_fields[f], out_fields[f] + c->n, 0.0);
    c->time += dt_h;
    return SPHGPU_OK;
}

int sphgpu_write_csv(sphgpu_ctx* c, const char* path, int step, int precision)
{
    SPHGPU_NEED_STATE(c);
    if(!path) return fail(c, SPHGPU_ERR_ARG, "write_csv: no path");
    if(precision < 1 || precision > 30) return fail(c, SPHGPU_ERR_ARG, "write_csv: precision must be 1..30");
    static const int cols[20] = {SPHGPU_F_POS_X, SPHGPU_F_POS_Y, SPHGPU_F_POS_Z, SPHGPU_F_VEL_X, SPHGPU_F_VEL_Y,
                                 SPHGPU_F_VEL_Z, SPHGPU_F_ACC_X, SPHGPU_F_ACC_Y, SPHGPU_F_ACC_Z, SPHGPU_F_MASS,
                                 SPHGPU_F_DENS, SPHGPU_F_PRES, SPHGPU_F_ENE, SPHGPU_F_SML, SPHGPU_F_SOUND,
                                 SPHGPU_F_ALPHA, SPHGPU_F_BALSARA, SPHGPU_F_GRADH, SPHGPU_F_PHI, SPHGPU_F_NEIGHBOR};
    const int n = c->n;
    std::vector<double> host((size_t)n * 20);
    double* ptrs[SPHGPU_NFIELDS] = {};
    for(int k = 0; k < 20; ++k) ptrs[cols[k]] = host.data() + (size_t)k * n;
    int rc = sphgpu_download(c, ptrs);
    if(rc < 0) return rc;
    double e[6];
    rc = energies(c, e);
    if(rc < 0) return rc;
    sphgpu_csv_meta m{};
    m.step = step;
    m.time = c->time;
    m.sph_type = c->prm.sph_type;
    m.kernel = c->prm.kernel;
    m.gamma = c->prm.gamma;
    m.g_constant = c->prm.g_constant;
    m.neighbor_number = c->prm.neighbor_number;
    m.use_gravity = c->prm.use_gravity;
    m.use_balsara = c->prm.use_balsara_switch;
    m.use_time_dependent_av = c->prm.use_time_dependent_av;
    m.kinetic = e[0];
    m.thermal = e[1];
    m.potential = e[2];
    m.precision = precision;
    m.timestamp = nullptr;
    rc = sphgpu_csv_write_host(path, n, ptrs, nullptr, &m);
    if(rc < 0) return fail(c, SPHGPU_ERR_ARG, "write_csv: cannot write the file");
    return SPHGPU_OK;
}

int sphgpu_read_csv(sphgpu_ctx* c, const char* path, int* step)
{
    if(!c || !path) return SPHGPU_ERR_ARG;
    int64_t n = 0;
    if(sphgpu_csv_read_host(path, &n, 0, nullptr, nullptr, nullptr) < 0 || n <= 0)
        return fail(c, SPHGPU_ERR_ARG, "read_csv: not a CSV v1 snapshot with particles");
    std::vector<double> host((size_t)n * SPHGPU_NFIELDS, 0.0);
    double* ptrs[SPHGPU_NFIELDS] = {};
    for(int k = 0; k < SPHGPU_NFIELDS; ++k) ptrs[k] = host.data() + (size_t)k * n;
    sphgpu_csv_meta m{};
    if(sphgpu_csv_read_host(path, &n, n, ptrs, nullptr, &m) < 0) return fail(c, SPHGPU_ERR_ARG, "read_csv: bad row");
    const int rc = sphgpu_upload(c, n, ptrs);
    if(rc < 0) return rc;
    c->time = m.time;
    if(step) *step = m.step;
    return SPHGPU_OK;
}

int sphgpu_energies(sphgpu_ctx* c, double* K, double* U, double* W, double* mom)
{
    SPHGPU_NEED_STATE(c);
    double out[6];
    const int rc = energies(c, out);
    if(rc < 0) return rc;
    if(K) *K = out[0];
    if(U) *U = out[1];
    if(W) *W = out[2];
    if(mom) {
        mom[0] = out[3];
        mom[1] = out[4];
        mom[2] = out[5];
    }
    return SPHGPU_OK;
}

int sphgpu_set_walk_mode(sphgpu_ctx* c, int mode)
{
    if(!c || mode < 0 || mode > 1) return SPHGPU_ERR_ARG;
    c->walk_mode = mode;
    c->skin_valid = false;
    return SPHGPU_OK;
}

int sphgpu_set_initial_smoothing(sphgpu_ctx* c, int on)
{
    if(!c) return SPHGPU_ERR_ARG;
    c->first_pre = on != 0;
    if(c->first_pre) c->skin_valid = false;
    return SPHGPU_OK;
}

int64_t sphgpu_tree_nodes(sphgpu_ctx* c, int32_t* ints, double* dbl, int64_t cap)
{
    if(!c) return SPHGPU_ERR_ARG;
    if(!c->have_tree) return fail(c, SPHGPU_ERR_STATE, "no tree");
    const int64_t nn = c->node_count;
    if(!ints || !dbl) return nn;
    if(cap < nn) return fail(c, SPHGPU_ERR_ARG, "node buffer too small");
    std::vector<int4> link((size_t)nn);
    std::vector<double4> geo((size_t)nn), mass((size_t)nn);
    std::vector<double> ks((size_t)nn);
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    SPHGPU_CUDA(c, cudaMemcpy(link.data(), c->t.link, sizeof(int4) * nn, cudaMemcpyDeviceToHost));
    SPHGPU_CUDA(c, cudaMemcpy(geo.data(), c->t.geo, sizeof(double4) * nn, cudaMemcpyDeviceToHost));
    SPHGPU_CUDA(c, cudaMemcpy(mass.data(), c->t.mass, sizeof(double4) * nn, cudaMemcpyDeviceToHost));
    SPHGPU_CUDA(c, cudaMemcpy(ks.data(), c->t.ksize, sizeof(double) * nn, cudaMemcpyDeviceToHost));
    for(int64_t k = 0; k < nn; ++k) {
        ints[3 * k] = link[k].w & 0xff;
        ints[3 * k + 1] = (link[k].w >> 8) & 1;
        ints[3 * k + 2] = link[k].y - link[k].x;
        double* d = dbl + 9 * k;
        d[0] = geo[k].x;
        d[1] = geo[k].y;
        d[2] = geo[k].z;
        d[3] = geo[k].w;
        d[4] = mass[k].w;
        d[5] = mass[k].x;
        d[6] = mass[k].y;
        d[7] = mass[k].z;
        d[8] = ks[k];
    }
    return nn;
}

int sphgpu_get_counters(sphgpu_ctx* c, sphgpu_counters* o)
{
    if(!c || !o) return SPHGPU_ERR_ARG;
    std::memset(o, 0, sizeof(*o));
    if(c->d_status) {
        SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
        SPHGPU_CUDA(c, cudaMemcpy(&c->h_status, c->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost));
    }
    o->newton_nonconverged = (int64_t)c->h_status.newton_nonconv;
    o->riemann_solves = (int64_t)c->h_status.riemann_solves;
    o->riemann_iterations = (int64_t)c->h_status.riemann_iters;
    o->riemann_fallbacks = (int64_t)c->h_status.riemann_fallbacks;
    o->gather_capacity = c->gcap;
    o->max_gather = c->max_gather;
    o->max_pair = c->max_pair;
    o->node_count = c->node_count;
    o->retries = c->retries;
    o->walk_group_warps = (int64_t)c->h_status.walk_group_warps;
    o->walk_split_warps = (int64_t)c->h_status.walk_split_warps;
    o->walk_fallbacks = c->walk_fallbacks;
    o->mlp_guesses = (int64_t)c->h_status.mlp_guesses;
    o->force_list_builds = c->flist_uses;
    o->pre_candidates = (int64_t)c->h_status.pre_cand;
    o->pre_newton_pairs = (int64_t)c->h_status.pre_newton_pairs;
    o->pre_pairs = (int64_t)c->h_status.pre_pairs;
    o->pre_list_entries = (int64_t)c->h_status.pre_list;
    o->force_candidates = (int64_t)c->h_status.force_cand;
    o->force_pairs = (int64_t)c->h_status.force_pairs;
    o->gravity_nodes = (int64_t)c->h_status.grav_nodes;
    o->gravity_monopoles = (int64_t)c->h_status.grav_mono;
    o->gravity_leaf_pairs = (int64_t)c->h_status.grav_leaf_pairs;
    o->mixed_rechecks = c->mixed_rechecks;
    o->skin_builds = c->skin_builds;
    o->skin_reuses = c->skin_reuses;
    return SPHGPU_OK;
}

int sphgpu_reset_counters(sphgpu_ctx* c)
{
    if(!c) return SPHGPU_ERR_ARG;
    if(c->d_status) {
        SPHGPU_CUDA(c, cudaMemsetAsync(c->d_status, 0, sizeof(DevStatus), c->stream));
        SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    std::memset(&c->h_status, 0, sizeof(c->h_status));
    c->retries = 0;
    c->mixed_rechecks = 0;
    c->skin_builds = 0;
    c->skin_reuses = 0;
    return SPHGPU_OK;
}

int sphgpu_enable_timing(sphgpu_ctx* c, int on)
{
    if(!c) return SPHGPU_ERR_ARG;
    if(c->stream) SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    stage_flush(c);
    c->timing = on != 0;
    c->launches = 0;
    for(int k = 0; k < SPHGPU_NSTAGES; ++k) {
        c->stage_ms[k] = 0.0;
        c->stage_launch[k] = 0;
    }
    return SPHGPU_OK;
}

int sphgpu_get_stage_times(sphgpu_ctx* c, double* ms, int64_t* launches)
{
    if(!c || !ms) return SPHGPU_ERR_ARG;
    if(c->stream) SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    stage_flush(c);
    for(int k = 0; k < SPHGPU_NSTAGES; ++k) {
        ms[k] = c->stage_ms[k];
        if(launches) launches[k] = c->stage_launch[k];
    }
    return SPHGPU_OK;
}

int sphgpu_timer_start(sphgpu_ctx* c)
{
    if(!c || !c->stream) return SPHGPU_ERR_ARG;
    SPHGPU_CUDA(c, cudaEventRecord(c->user_ev[0], c->stream));
    return SPHGPU_OK;
}

int sphgpu_timer_stop(sphgpu_ctx* c, double* ms)
{
    if(!c || !c->stream || !ms) return SPHGPU_ERR_ARG;
    SPHGPU_CUDA(c, cudaEventRecord(c->user_ev[1], c->stream));
    SPHGPU_CUDA(c, cudaEventSynchronize(c->user_ev[1]));
    float f = 0.f;
    SPHGPU_CUDA(c, cudaEventElapsedTime(&f, c->user_ev[0], c->user_ev[1]));
    *ms = f;
    return SPHGPU_OK;
}

int64_t sphgpu_launch_count(const sphgpu_ctx* c) { return c ? c->launches : 0; }

int sphgpu_synchronize(sphgpu_ctx* c)
{
    if(!c || !c->stream) return SPHGPU_ERR_ARG;
    return sync_and_check(c);
}

int sphgpu_test_flag_pass_guard(sphgpu_ctx* c, int bits)
{
    if(!c || !c->d_status || bits <= 0 || bits > 15) return SPHGPU_ERR_ARG;
    SPHGPU_CUDA(c, cudaMemcpyAsync(&c->d_status->pass_guard, &bits, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    return SPHGPU_OK;
}

}  // extern "C"
