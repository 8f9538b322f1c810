// context.cuh — the state behind one sphgpu_ctx: parameters, device arrays,
// octree, neighbour lists, counters and stage timers.  One CUDA stream per
// context; every module enqueues on it.
#pragma once

#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "common.cuh"
#include "scan_sort.cuh"

struct sphgpu_ctx {
    sphgpu_params prm{};
    sphgpu::DevParams dp{};
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // sphgpu_integrate_host: downloads beside the step
    cudaEvent_t copy_ev[3] = {};
    std::string err;
    int n = 0;
    bool have_tree = false;     // octree valid for the current positions
    bool first_pre = true;      // PreInteraction::m_first (src/pre_interaction.cpp:41-44)
    double time = 0.0;

    // particle state (octree order) and its ping-pong copy for permutation
    sphgpu::DevState s{}, alt{};
    std::vector<void*> state_allocs;

    // octree
    sphgpu::DevTree t{};
    int node_cap = 0;
    double4* d_root = nullptr;       // root center x, y, z, edge
    double* d_bbox_part = nullptr;   // per-block bbox partials
    uint64_t *d_keys = nullptr, *d_keys_alt = nullptr;
    uint32_t *d_vals = nullptr, *d_vals_alt = nullptr;
    int* d_nstart = nullptr;         // nodes starting at particle p
    int* d_base = nullptr;           // exclusive scan of d_nstart
    int* d_lvl = nullptr;            // lfirst | leaf_level << 8
    int* d_leaf_of_start = nullptr;  // leaf node index for node-starting particles, else -1
    int* d_inv = nullptr;            // particle id -> octree position
    void* d_radix_scratch = nullptr;
    void* d_scan_scratch = nullptr;
    sphgpu::ScanScratch scan{};

    // neighbour lists (ELL: capacity slots per particle, row-major)
    int* d_glist = nullptr;          // gather list (PreInteraction)
    int* d_gcount = nullptr;
    int64_t gcap = 0;
    int* d_plist = nullptr;          // symmetric list (FluidForce)
    int* d_pcount = nullptr;
    int64_t pcap = 0;
    // skin (Verlet) gather lists (walk.cu): a second list buffer, and per
    // particle the walk radius and position of the build
    int* d_glist_alt = nullptr;      // own allocation; trades places with d_glist
    void* d_skin = nullptr;          // the rest, one allocation
    int* d_gcount_alt = nullptr;
    double *d_skin_r = nullptr, *d_skin_r_alt = nullptr;
    double4 *d_skin_x = nullptr, *d_skin_x_alt = nullptr;
    int* d_skin_new = nullptr;       // old position -> new position of the last permutation
    double* d_skin_scal = nullptr;   // largest displacement, failed-check flag
    int skin_n = 0;
    int64_t skin_cap = 0;
    bool skin_valid = false;         // d_glist holds skin lists of the current order
    double skin_delta_now = 0.0;     // the walk's safety margin for the current tree
    int64_t skin_builds = 0, skin_reuses = 0;
    uint32_t* d_skin_map = nullptr;  // after an upload: caller index -> list row
    uint32_t* d_skin_src = nullptr;  // composed permutation (scratch)
    bool skin_map_pending = false;   // d_skin_map applies at the next permutation
    bool skin_built = false;         // a skin build happened since the buffers were made
    int skin_since_build = 0;        // reuses of the current skin lists
    int skin_idle = 0;               // consecutive builds that were never reused
    int skin_off = 0;                // steps left of exact walks (skin paused)
    double skin_scale = 1.0;         // the next build's skin, in units of gather_skin
    int skin_short = 0;              // consecutive builds whose lists served < 2 steps
    double skin_factor = 1.0;        // 1 + the skin of the current lists
    double skin_need = -1.0;         // skin the last failed check needed (< 0: none)
    // pair lists built from the gather lists (flist.cu)
    int* d_tcount = nullptr;         // entries appended to each row from the back
    int* d_flist_flags = nullptr;    // {incomplete, longest list, over neighborNumber * 1000}
    double* d_rsearch = nullptr;     // radius of each particle's gather list
    int flist_n = 0;
    bool flist_ready = false;        // built for the current tree and h
    int64_t flist_uses = 0;

    // mixed form's FP64 re-evaluation (recheck.cu): per particle the sum of
    // |FP32 acceleration terms|, the flags, their scan, the list and its length
    void* d_recheck = nullptr;
    float* d_accabs = nullptr;
    int *d_rflag = nullptr, *d_rpos = nullptr, *d_ridx = nullptr, *d_rcount = nullptr;
    int recheck_n = 0;
    bool accabs_valid = false;       // FluidForce filled accabs for the current tree
    int64_t mixed_rechecks = 0;      // particles re-evaluated in FP64

    // host transfer staging (upload / download): one slot of n doubles per
    // field moved, kept across calls
    double* d_stage = nullptr;
    int64_t stage_cap = 0;           // doubles d_stage holds

    // scalars
    double* d_dt = nullptr;          // Simulation::dt
    double* d_hvs = nullptr;         // Simulation::h_per_v_sig
    double* d_red = nullptr;         // reduction scratch
    double* d_relax = nullptr;       // Lane-Emden table (xi, theta, dtheta) + dt_relax
    int64_t relax_cap = 0;
    sphgpu::DevStatus* d_status = nullptr;
    sphgpu::DevStatus h_status{};

    // learned Riemann guess (BF16 weights + FP32 biases on device)
    void* d_mlp = nullptr;            // BF16 / FP32 image read by the kernels
    float* d_mlp_master = nullptr;    // FP32 master parameters + Adam moments
    // deferred pairs of the learned path: rows (features, pair keys, network
    // output, sort buffers) and per-particle row ranges, in one allocation
    void* d_mlp_defer = nullptr;
    int64_t mlp_rcap = 0;             // rows the allocation holds
    int64_t mlp_ncap = 0;             // particles the allocation holds
    int64_t mlp_rows_demand = 0;      // rows the last learned force pass asked for
    // mixed-precision gravity: 32-byte FP32 node records of the current tree
    void* d_gnode = nullptr;
    int gnode_cap = 0;
    bool have_mlp = false;
    std::vector<float> mlp_master;
    // pair-state harvesting (training data from the plain solver's own runs)
    double* d_harvest = nullptr;
    unsigned long long* d_harvest_count = nullptr;
    int64_t harvest_cap = 0;
    unsigned harvest_mod = 0;

    // counters kept on the host
    int64_t retries = 0;
    int64_t walk_fallbacks = 0;     // group walks redone by the per-lane walk
    int walk_mode = 0;              // 0 = group walk, 1 = per-lane walk only
    int64_t max_gather = 0, max_pair = 0, node_count = 0;

    // timing: event pairs recorded around each stage and read back at the
    // next point where the host waits on the stream anyway
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    struct Pending {
        int stage;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    cudaEvent_t open_ev[SPHGPU_NSTAGES] = {};
    double stage_ms[SPHGPU_NSTAGES] = {};
    int64_t stage_launch[SPHGPU_NSTAGES] = {};
    int64_t launches = 0;          // kernels launched by this context
    cudaEvent_t user_ev[2] = {};   // sphgpu_timer_start / stop
};

namespace sphgpu {

// errors
int fail(sphgpu_ctx* c, int code, const std::string& msg);
int cuda_fail(sphgpu_ctx* c, cudaError_t e, const char* where);

#define SPHGPU_CUDA(c, call)                                   \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if(e_ != cudaSuccess) return cuda_fail((c), e_, #call); \
    } while(0)

#define SPHGPU_LAUNCH_CHECK(c, where)                             \
    do {                                                          \
        cudaError_t e_ = cudaGetLastError();                      \
        if(e_ != cudaSuccess) return cuda_fail((c), e_, (where)); \
    } while(0)

// Device temporaries of one call, released on every return path (error
// returns included): stream-ordered with cudaFreeAsync when taken with
// cudaMallocAsync on the stream, else with cudaFree.
class DevTemps {
public:
    explicit DevTemps(cudaStream_t s) : s_(s) {}
    ~DevTemps()
    {
        for(const Item& a : items_) {
            if(a.async) cudaFreeAsync(a.p, s_);
            else cudaFree(a.p);
        }
    }
    DevTemps(const DevTemps&) = delete;
    DevTemps& operator=(const DevTemps&) = delete;
    template <typename T>
    cudaError_t get(T** p, size_t bytes, bool async = true)
    {
        void* q = nullptr;
        const cudaError_t e = async ? cudaMallocAsync(&q, bytes, s_) : cudaMalloc(&q, bytes);
        if(e == cudaSuccess) items_.push_back({q, async});
        *p = static_cast<T*>(q);
        return e;
    }

private:
    struct Item {
        void* p;
        bool async;
    };
    cudaStream_t s_;
    std::vector<Item> items_;
};

// stage timers
void stage_begin(sphgpu_ctx* c, int stage);
void stage_end(sphgpu_ctx* c, int stage, int launches);
void stage_flush(sphgpu_ctx* c);   // call only after the stream is idle

// module implementations (each returns an sphgpu_status)
int tree_make(sphgpu_ctx* c);
int tree_set_kernel(sphgpu_ctx* c);
int gather_walk(sphgpu_ctx* c, bool compute_guess, double ratio);
// The step's gather lists: skin lists reused when still valid, else built
// (gather_skin > 0), or the exact walk (walk.cu).
int gather_lists(sphgpu_ctx* c, double ratio);
// Move valid skin lists to the order of a new tree (src: old position of the
// particle now at each position).
int skin_permute(sphgpu_ctx* c, const uint32_t* src);
int skin_upload(sphgpu_ctx* c);
int pair_walk(sphgpu_ctx* c);
int export_lists(sphgpu_ctx* c, int which, int64_t* offsets, int32_t* ids, int64_t cap);
int exhaustive_lists(sphgpu_ctx* c, int is_ij, int64_t* offsets, int32_t* ids, int64_t cap);
int pre_interaction(sphgpu_ctx* c);
int fluid_force(sphgpu_ctx* c);
int gravity(sphgpu_ctx* c, bool direct);
// Mixed-precision Barnes-Hut walk: FP32 node records of the current tree,
// then the walk (one launch each).
int gravity_nodes_mixed(sphgpu_ctx* c);
// FluidForce's pair lists from the gather lists (flist.cu): save the gather
// radius before the pre-interaction overwrites h, build after it; the force
// takes them, or the symmetric tree walk when they are incomplete.
int save_gather_radius(sphgpu_ctx* c);
int build_force_lists(sphgpu_ctx* c);
int symmetric_lists(sphgpu_ctx* c);
// SRGSPH modules (srgsph.cu), dispatched from the generic ones.
int sr_pre_interaction(sphgpu_ctx* c);
int sr_fluid_force(sphgpu_ctx* c);
int sr_timestep(sphgpu_ctx* c);
int sr_predict(sphgpu_ctx* c);
int sr_correct(sphgpu_ctx* c);
int gravity_walk_mixed(sphgpu_ctx* c);
// Mixed form: FluidForce / GravityForce in FP64 for the listed particles
// (device list of nsub indices), and the pass that lists them (recheck.cu).
int fluid_force_subset64(sphgpu_ctx* c, const int* idx, int nsub);
int gravity_subset64(sphgpu_ctx* c, const int* idx, int nsub);
int ensure_recheck(sphgpu_ctx* c);
int mixed_recheck(sphgpu_ctx* c);
int timestep(sphgpu_ctx* c);
int predict(sphgpu_ctx* c);
int correct(sphgpu_ctx* c);
int energies(sphgpu_ctx* c, double* out5 /* K, U, W, px.. */);
// Report a bound hit by a pass that ran without a host wait after it (mass,
// set_kernel, gravity): call after a wait that copied DevStatus::pass_guard
// into h_status.  Clears the word on the device and returns SPHGPU_ERR_STATE
// when a bit is set, SPHGPU_OK otherwise.
int check_pass_guard(sphgpu_ctx* c);
// Copy DevStatus::pass_guard to the host, wait on the stream, then
// check_pass_guard.
int sync_and_check(sphgpu_ctx* c);
int ensure_list_capacity(sphgpu_ctx* c, int which, int64_t cap);

}  // namespace sphgpu
