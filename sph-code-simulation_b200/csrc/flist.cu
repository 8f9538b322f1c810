// flist.cu — FluidForce's pair lists built from the gather lists, without a
// second tree walk.
//
// FluidForce sums over the pairs with r < max(h_i, h_j) (src/fluid_force.cpp:
// 53-60 and the gsph / disph / gdisph forces: the is_ij neighbour search of
// src/bhtree.cpp:277-316, then the pair test in the force loop).  After the
// pre-interaction every h is final and, when h_k <= R_k for every particle
// (R_k the radius of its gather list), those pairs are exactly
//   own(i)        = { j in gather(i) : r_ij < h_i }
//   transposed(i) = { j : i in gather(j), r_ij < h_j, not r_ij < h_i }
// because r < h <= R implies r^2 < R^2 for correctly rounded r = sqrt(r^2),
// and r_ij = r_ji bit for bit (exact negation, antisymmetric minimum image).
// From a skin list (built at a wider radius, reused over steps: a superset of
// the gather list) own(i) keeps the gather list's members only: every r < h_i
// when h_i < R_i - delta (delta = the walk's margin), else those that pass the
// exact membership test (gather_member).
// Each particle scans its gather list once: own entries go to the front of its
// row in gather-list order (group ballot compaction), and each pair that only
// the neighbour's kernel reaches is appended to the neighbour's row from the
// back (atomic slot).  A finalise pass sorts each row's appended entries by
// index (a deterministic summation order) and moves them behind the own
// entries.  If some h_k > R_k, or a row does not fit, the step falls back to
// the symmetric tree walk, which gives the same pair sets.
// Building the rows inside the pre-interaction's fused pass instead (pre split
// into a smoothing-length launch and a fused launch, ballots and atomics in its
// loop) was measured slower: shear 1 M pre + lists 7.1 ms against 4.8 + 1.7 ms.
// So was letting the fused pass write only the own part (ballot compaction,
// lanes kept in step for it) and this pass only the appended part: on the
// 8.78 M sphere lists 15.9 -> 10.1 ms but pre 31.7 -> 44.8 ms.  Scanning the
// candidates PreInteraction's last sweep kept within (1 + 4e-4) h (about
// half the list) instead of the list: 14.4 -> 14.6 ms, no gain; the scan is
// not what bounds this pass.
#include <cuda_runtime.h>

#include "context.cuh"

namespace sphgpu {

namespace {

constexpr int LBLK = 256;
constexpr int LG = 8;  // lanes per particle (8: 1.57 ms vs 1.71 ms with 4, shear 1 M)

__global__ void k_save_radius(const DevState S, int n, double* __restrict__ rs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n) rs[i] = S.vel[i].w;
}

// 5 resident blocks (48 registers): 15.8 -> 14.5 ms against 6 on the 8.78 M
// sphere, 1.81 -> 1.69 ms on the 1 M shear layer (4 is slower)
template <int G>
__global__ void __launch_bounds__(LBLK, 5) k_flist(DevParams P, DevState S, int n, const int* __restrict__ glist,
                                                const int* __restrict__ gcount, int gcap,
                                                const double* __restrict__ rs, int* __restrict__ plist,
                                                int* __restrict__ pcount, int* __restrict__ tcount, int pcap,
                                                int* __restrict__ flags, DevTree Tr, double skin_delta)
{
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & (G - 1);
    const unsigned gbase = (threadIdx.x & 31) & ~(unsigned)(G - 1);
    const unsigned gmask = group_mask<G>();
    const long long warp = ((long long)blockIdx.x * LBLK + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * LBLK) >> 5;
    for(long long wb = warp * GPW; wb < n; wb += nwarps * GPW) {
        const int i = (int)(wb + ((threadIdx.x & 31) / G));
        if(i >= n) continue;  // whole groups drop out together
        const double4 pi = S.pos[i];
        const double hi = S.vel[i].w;
        // the gather list may miss r < h_i; from a skin list (a superset) the
        // pairs r < h_i are the gather list's when h_i < R_i - delta, and
        // otherwise those that pass the exact membership test
        const double ri = rs[i];
        if(!(hi <= ri) && lane == 0) flags[0] = 1;
        const bool exact = skin_delta > 0.0 && !(hi < ri - skin_delta);
        const int cnt = min(gcount[i], gcap);
        const int* li = glist + (size_t)i * (size_t)gcap;
        int* row = plist + (size_t)i * (size_t)pcap;
        int oc = 0;
        // r < h_i (an own pair) and, for an own pair j's kernel not reaching
        // i, the entry appended to j's row
        auto test = [&](int j, const double4& pj) {
            const Vec3d d = rij(P, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z);
            const double r2 = abs2x(d);
            const double r = sqrt(r2);
            if(!(r < hi && (!exact || gather_member(P, Tr, pi.x, pi.y, pi.z, ri, skin_delta, j, r2)))) return false;
            if(!(r < __ldg(&S.vel[j].w))) {
                const int t = atomicAdd(&tcount[j], 1);
                if(t < pcap) plist[(size_t)j * (size_t)pcap + (pcap - 1 - t)] = i;
            }
            return true;
        };
        auto compact = [&](bool own, int j) {
            const unsigned m = (__ballot_sync(gmask, own) >> gbase) & ((1u << G) - 1u);
            if(own) {
                const int pos = oc + __popc(m & ((1u << lane) - 1u));
                if(pos < pcap) row[pos] = j;
            }
            oc += __popc(m);
        };
        // two chunks of G entries per iteration, their indices fetched an
        // iteration ahead: two position loads per lane in flight (8.78 M
        // sphere 16.6 -> 15.9 ms; 1 M shear layer 1.73 -> 1.81 ms)
        int ja = lane < cnt ? __ldg(&li[lane]) : 0;
        int jb = G + lane < cnt ? __ldg(&li[G + lane]) : 0;
        for(int kk = 0; kk < cnt; kk += 2 * G) {
            const int ca = ja, cb = jb;  // valid indices even past the list end
            const bool ina = kk + lane < cnt, inb = kk + G + lane < cnt;
            if(kk + 2 * G + lane < cnt) ja = __ldg(&li[kk + 2 * G + lane]);
            if(kk + 3 * G + lane < cnt) jb = __ldg(&li[kk + 3 * G + lane]);
            const double4 pa = ldg4(&S.pos[ca]);
            const double4 pb = ldg4(&S.pos[cb]);
            compact(ina && test(ca, pa), ca);
            compact(inb && test(cb, pb), cb);
        }
        if(lane == 0) pcount[i] = oc;
    }
}

// Appended entries: sorted by index and moved behind the own entries.
__global__ void k_flist_finalize(int n, int* __restrict__ plist, int* __restrict__ pcount,
                                 const int* __restrict__ tcount, int pcap, int fatal_limit,
                                 int* __restrict__ flags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const int oc = pcount[i], tc = tcount[i];
    const long long tot = (long long)oc + tc;
    if(tot > pcap) {
        flags[0] = 1;
        return;
    }
    if(tot > fatal_limit) flags[2] = 1;
    int* row = plist + (size_t)i * (size_t)pcap;
    const int b0 = pcap - tc;
    for(int a = b0 + 1; a < pcap; ++a) {
        const int v = row[a];
        int b = a - 1;
        while(b >= b0 && row[b] > v) {
            row[b + 1] = row[b];
            --b;
        }
        row[b + 1] = v;
    }
    for(int t = 0; t < tc; ++t) row[oc + t] = row[b0 + t];
    pcount[i] = (int)tot;
    atomicMax(&flags[1], (int)tot);
}

}  // namespace

int build_force_lists(sphgpu_ctx* c)
{
    c->flist_ready = false;
    const int n = c->n;
    if(n <= 0) return SPHGPU_OK;
    cudaStream_t st = c->stream;
    if(c->flist_n < n) return fail(c, SPHGPU_ERR_STATE, "force lists before the gather radius was saved");
    if(c->pcap < c->gcap) {
        const int rc = ensure_list_capacity(c, 1, c->gcap);
        if(rc < 0) return rc;
    }
    stage_begin(c, SPHGPU_T_PAIR_WALK);
    SPHGPU_CUDA(c, cudaMemsetAsync(c->d_tcount, 0, sizeof(int) * (size_t)n, st));
    SPHGPU_CUDA(c, cudaMemsetAsync(c->d_flist_flags, 0, 3 * sizeof(int), st));
    const long long gpb = LBLK / LG;
    const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>((n + gpb - 1) / gpb, 148LL * 8 * 4));
    k_flist<LG><<<grid, LBLK, 0, st>>>(c->dp, c->s, n, c->d_glist, c->d_gcount, (int)c->gcap, c->d_rsearch,
                                       c->d_plist, c->d_pcount, c->d_tcount, (int)c->pcap, c->d_flist_flags,
                                       c->t, c->skin_valid ? c->skin_delta_now : 0.0);
    k_flist_finalize<<<grid_for(n, 256), 256, 0, st>>>(n, c->d_plist, c->d_pcount, c->d_tcount, (int)c->pcap,
                                                        c->prm.neighbor_number * 1000, c->d_flist_flags);
    SPHGPU_LAUNCH_CHECK(c, "force lists");
    stage_end(c, SPHGPU_T_PAIR_WALK, 2);
    c->flist_ready = true;
    return SPHGPU_OK;
}

int save_gather_radius(sphgpu_ctx* c)
{
    if(c->flist_n < c->n) {
        if(c->d_tcount) cudaFree(c->d_tcount);
        if(c->d_rsearch) cudaFree(c->d_rsearch);
        c->d_tcount = nullptr;
        c->d_rsearch = nullptr;
        c->flist_n = 0;
        if(!c->d_flist_flags) SPHGPU_CUDA(c, cudaMalloc(&c->d_flist_flags, 3 * sizeof(int)));
        SPHGPU_CUDA(c, cudaMalloc(&c->d_tcount, sizeof(int) * (size_t)c->n));
        SPHGPU_CUDA(c, cudaMalloc(&c->d_rsearch, sizeof(double) * (size_t)c->n));
        c->flist_n = c->n;
    }
    k_save_radius<<<grid_for(c->n, 256), 256, 0, c->stream>>>(c->s, c->n, c->d_rsearch);
    SPHGPU_LAUNCH_CHECK(c, "gather radius");
    ++c->launches;  // a copy of n doubles, left out of the stage timers
    return SPHGPU_OK;
}

// The pair lists FluidForce sums over: the ones built after the
// pre-interaction when they are complete (they stay valid until the next tree
// make), else the symmetric tree walk.
int symmetric_lists(sphgpu_ctx* c)
{
    if(c->flist_ready) {
        int flags[3] = {0, 0, 0};  // incomplete, longest list, over the limit
        SPHGPU_CUDA(c, cudaMemcpyAsync(flags, c->d_flist_flags, 3 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        SPHGPU_CUDA(c, cudaStreamSynchronize(c->stream));
        if(flags[2]) {
            return fail(c, SPHGPU_ERR_NEIGHBOR_OVERFLOW,
                        "Neighbor list overflow: more than neighborNumber * 1000 neighbours");
        }
        if(!flags[0]) {
            c->max_pair = flags[1];
            ++c->flist_uses;
            return SPHGPU_OK;
        }
        c->flist_ready = false;
    }
    return pair_walk(c);
}

}  // namespace sphgpu
