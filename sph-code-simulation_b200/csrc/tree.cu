// tree.cu — BHTree::make and BHTree::set_kernel on the device.
//
// Reference: src/bhtree.cpp:59-115 (make), :154-204 (create_tree), :206-247
// (assign), :117-120 and :249-275 (set_kernel).  The reference builds a
// geometric octree by serial recursion over linked lists.  Here:
//
//  1. root cube: bbox (two-stage min/max reduction) or the periodic box;
//  2. key pass: each particle replays the reference's `pos > center` choice
//     at levels 1..max_level with the same centre arithmetic
//     (center + (+-1) * edge * 0.25, edge * 0.5 per level), so its 3-bit
//     digits are exactly the child indices the recursion would take;
//  3. stable LSD radix sort of the keys (scan_sort.cu);
//  4. node pass: from adjacent-key common prefixes each particle knows how
//     many preorder nodes start at it and at which level its leaf sits
//     (a node at level L >= 2 is internal iff it holds more than
//     leafParticleNumber particles and L <= maxTreeLevel, the rule of
//     create_tree; the root is always internal).  One scan gives every node
//     its preorder index; the node arrays (centre, edge, particle range,
//     skip pointer, parent) are written in one pass;
//  5. leaf order: particles inside a leaf are put in the order of the
//     reference's linked list (ascending particle index at odd levels,
//     descending at even levels, because assign() prepends), so walks visit
//     leaf particles in the reference's order;
//  6. state arrays are gathered into the new order;
//  7. mass and centre of mass bottom-up: leaves accumulate in the order
//     assign() did (reverse of the list order), internal nodes sum children
//     in index order, exactly as create_tree; the last child to finish
//     (atomic counter) computes its parent.
// Every step is FP64 with unfused arithmetic (this file builds with
// -fmad=false), so node geometry, mass and centre of mass are bit-identical
// to the reference's.
#include <cfloat>
#include <cstddef>
#include <cuda_runtime.h>

#include "context.cuh"

namespace sphgpu {

namespace {

constexpr int BLK = 256;

// ---------------------------------------------------------------- bbox
__global__ void k_bbox_partial(const double4* __restrict__ pos, int n, double* __restrict__ part,
                               DevStatus* __restrict__ st)
{
    __shared__ double smin[3][BLK], smax[3][BLK];
    double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for(int i = blockIdx.x * BLK + threadIdx.x; i < n; i += gridDim.x * BLK) {
        const double4 p = pos[i];
        const double v[3] = {p.x, p.y, p.z};
        // a non-finite coordinate would collapse every key onto one path
        if(!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) st->nonfinite = 1;
        for(int k = 0; k < 3; ++k) {
            if(mn[k] > v[k]) mn[k] = v[k];
            if(mx[k] < v[k]) mx[k] = v[k];
        }
    }
    for(int k = 0; k < 3; ++k) {
        smin[k][threadIdx.x] = mn[k];
        smax[k][threadIdx.x] = mx[k];
    }
    __syncthreads();
    for(int s = BLK / 2; s > 0; s >>= 1) {
        if(threadIdx.x < s) {
            for(int k = 0; k < 3; ++k) {
                smin[k][threadIdx.x] = fmin(smin[k][threadIdx.x], smin[k][threadIdx.x + s]);
                smax[k][threadIdx.x] = fmax(smax[k][threadIdx.x], smax[k][threadIdx.x + s]);
            }
        }
        __syncthreads();
    }
    if(threadIdx.x == 0) {
        for(int k = 0; k < 3; ++k) {
            part[blockIdx.x * 6 + k] = smin[k][0];
            part[blockIdx.x * 6 + 3 + k] = smax[k][0];
        }
    }
}

// Root cube of BHTree::make (src/bhtree.cpp:67-103) or BHTree::initialize
// (src/bhtree.cpp:19-32) for periodic runs.
__global__ void k_root(const double* __restrict__ part, int nparts, DevParams P, double4* __restrict__ root)
{
    if(threadIdx.x != 0) return;
    double lo[3], hi[3];
    if(P.periodic) {
        for(int k = 0; k < 3; ++k) {
            lo[k] = P.lo[k];
            hi[k] = P.hi[k];
        }
    } else {
        for(int k = 0; k < 3; ++k) {
            lo[k] = DBL_MAX;
            hi[k] = -DBL_MAX;
        }
        for(int b = 0; b < nparts; ++b) {
            for(int k = 0; k < 3; ++k) {
                lo[k] = fmin(lo[k], part[b * 6 + k]);
                hi[k] = fmax(hi[k], part[b * 6 + 3 + k]);
            }
        }
        // BHTree::make under more than one OpenMP thread: the min / max
        // slots of threads other than the first start at 0.0, so the box
        // reduced from them also covers the origin (src/bhtree.cpp:68-91)
        if(P.root_origin) {
            for(int k = 0; k < 3; ++k) {
                if(lo[k] > 0.0) lo[k] = 0.0;
                if(hi[k] < 0.0) hi[k] = 0.0;
            }
        }
    }
    double c[3], l = 0.0;
    for(int k = 0; k < 3; ++k) {
        c[k] = __dmul_rn(__dadd_rn(hi[k], lo[k]), 0.5);
        const double r = __dsub_rn(hi[k], lo[k]);
        if(l < r) l = r;
    }
    *root = make_double4(c[0], c[1], c[2], l);
}

// ---------------------------------------------------------------- keys
__device__ __forceinline__ int digit_at(double x, double y, double z, double cx, double cy, double cz)
{
    return (x > cx ? 1 : 0) | (y > cy ? 2 : 0) | (z > cz ? 4 : 0);
}

// child centre: center + ((index & a) * b - 1.0) * edge * 0.25 (src/bhtree.cpp:236-241)
__device__ __forceinline__ double child_center(double c, int bit, double e)
{
    const double s = bit ? 1.0 : -1.0;
    return __dadd_rn(c, __dmul_rn(__dmul_rn(s, e), 0.25));
}

__global__ void k_keys(const double4* __restrict__ pos, int n, const double4* __restrict__ root, int depth,
                       uint64_t* __restrict__ keys, uint32_t* __restrict__ vals)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const double4 p = pos[i];
    const double4 r = *root;
    double cx = r.x, cy = r.y, cz = r.z, e = r.w;
    uint64_t key = 0;
    for(int l = 0; l < depth; ++l) {
        const int d = digit_at(p.x, p.y, p.z, cx, cy, cz);
        key = (key << 3) | (uint64_t)d;
        cx = child_center(cx, d & 1, e);
        cy = child_center(cy, d & 2, e);
        cz = child_center(cz, d & 4, e);
        e = __dmul_rn(e, 0.5);
    }
    keys[i] = key;
    vals[i] = (uint32_t)i;
}

// ---------------------------------------------------------------- nodes
__device__ __forceinline__ int common_digits(uint64_t a, uint64_t b, int D)
{
    const uint64_t x = a ^ b;
    if(x == 0) return D;
    return (__clzll((long long)x) - (64 - 3 * D)) / 3;
}

__global__ void k_levels(const uint64_t* __restrict__ keys, int n, int D, int M, int* __restrict__ nstart,
                         int* __restrict__ lvl)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    int cstar = -1;
    const int qlo = max(0, p - M), qhi = min(p, n - 1 - M);
    const uint64_t kp = keys[p];
    for(int q = qlo; q <= qhi; ++q) {
        const int c = common_digits(keys[q], keys[q + M], D);
        if(c > cstar) cstar = c;
    }
    int leaf = cstar + 2;
    if(leaf < 2) leaf = 2;
    if(leaf > D + 1) leaf = D + 1;
    const int lfirst = p == 0 ? 2 : common_digits(keys[p - 1], kp, D) + 2;
    const int ns = leaf - lfirst + 1;
    nstart[p] = ns > 0 ? ns : 0;
    lvl[p] = lfirst | (leaf << 8);
}

__device__ __forceinline__ int lfirst_at(const uint64_t* keys, int s, int D)
{
    return s == 0 ? 2 : common_digits(keys[s - 1], keys[s], D) + 2;
}

// first q >= lo (all q < lo share >= need digits with kp) that shares fewer
__device__ int subtree_end(const uint64_t* keys, int n, int D, uint64_t kp, int need, int lo)
{
    int hi = lo, step = 1;
    while(hi < n && common_digits(keys[hi], kp, D) >= need) {
        lo = hi + 1;
        hi = lo + step;
        step <<= 1;
    }
    if(hi > n) hi = n;
    while(lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if(common_digits(keys[mid], kp, D) >= need) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// smallest s <= hi (hi shares >= need digits with kp) that shares >= need
__device__ int subtree_start(const uint64_t* keys, int D, uint64_t kp, int need, int hi)
{
    int step = 1, lo = hi - 1;
    while(lo >= 0 && common_digits(keys[lo], kp, D) >= need) {
        hi = lo;
        step <<= 1;
        lo = hi - step;
    }
    if(lo < -1) lo = -1;
    while(hi - lo > 1) {
        const int mid = lo + ((hi - lo) >> 1);
        if(common_digits(keys[mid], kp, D) >= need) hi = mid;
        else lo = mid;
    }
    return hi;
}

__global__ void k_nodes(const uint64_t* __restrict__ keys, int n, int D, const int* __restrict__ nstart,
                        const int* __restrict__ base, const int* __restrict__ lvl, const double4* __restrict__ root,
                        int cap, DevTree T, int* __restrict__ leaf_of_start, DevStatus* __restrict__ st)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const double4 r = *root;
    if(p == 0) {
        const int total = base[n - 1] + nstart[n - 1] + 1;
        *T.nnodes = total;
        if(total > cap) st->node_pool = 1;
        T.geo[0] = r;
        T.link[0] = make_int4(0, n, total, 1);
        T.parent[0] = -1;
        T.ksize[0] = 0.0;
    }
    const int ns = nstart[p];
    if(ns == 0) {
        leaf_of_start[p] = -1;
        return;
    }
    const int lv = lvl[p];
    const int lfirst = lv & 0xff, leaf = lv >> 8;
    const int b = 1 + base[p];
    const uint64_t kp = keys[p];
    if(b + ns > cap) {
        st->node_pool = 1;
        leaf_of_start[p] = -1;
        return;
    }
    const int total = base[n - 1] + nstart[n - 1] + 1;
    // centre / edge at level lfirst by replaying digits 1..lfirst-1
    double cx = r.x, cy = r.y, cz = r.z, e = r.w;
    for(int l = 1; l < lfirst; ++l) {
        const int d = (int)((kp >> (3 * (D - l))) & 7);
        cx = child_center(cx, d & 1, e);
        cy = child_center(cy, d & 2, e);
        cz = child_center(cz, d & 4, e);
        e = __dmul_rn(e, 0.5);
    }
    // subtree ends, deepest level first (nested ranges)
    int ends[24];
    int lo = p + 1;
    for(int L = leaf; L >= lfirst; --L) {
        lo = subtree_end(keys, n, D, kp, L - 1, lo);
        ends[L - lfirst] = lo;
    }
    for(int L = lfirst; L <= leaf; ++L) {
        const int idx = b + (L - lfirst);
        const int end = ends[L - lfirst];
        const int skip = end < n ? 1 + base[end] : total;
        T.geo[idx] = make_double4(cx, cy, cz, e);
        T.link[idx] = make_int4(p, end, skip, L | ((L == leaf) ? 256 : 0));
        T.ksize[idx] = 0.0;
        int par;
        if(L > lfirst) {
            par = idx - 1;
        } else if(L - 1 == 1) {
            par = 0;
        } else {
            const int s = subtree_start(keys, D, kp, L - 2, p - 1);
            par = 1 + base[s] + (L - 1 - lfirst_at(keys, s, D));
        }
        T.parent[idx] = par;
        atomicAdd(&T.nchild[par], 1);
        // octant of this node in its parent = the key digit taken at level L-1
        T.child[(size_t)par * 8 + (int)((kp >> (3 * (D - (L - 1)))) & 7)] = idx;
        if(L < leaf) {
            const int d = (int)((kp >> (3 * (D - L))) & 7);
            cx = child_center(cx, d & 1, e);
            cy = child_center(cy, d & 2, e);
            cz = child_center(cz, d & 4, e);
            e = __dmul_rn(e, 0.5);
        }
    }
    leaf_of_start[p] = b + (leaf - lfirst);
}

// Reorder each leaf's particles into the reference's list order.  Small
// leaves use insertion sort; large ones (coincident particles at the maximum
// level) a heap sort, so the cost stays O(L log L) per leaf.
__device__ __forceinline__ bool leaf_before(int a, int b, bool ascending) { return ascending ? a < b : a > b; }

__global__ void k_leaf_order(int n, const int* __restrict__ leaf_of_start, const int4* __restrict__ link,
                             const int* __restrict__ old_id, uint32_t* __restrict__ vals)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const int lf = leaf_of_start[p];
    if(lf < 0) return;
    const int4 lk = link[lf];
    const int cnt = lk.y - lk.x;
    if(cnt <= 1) return;
    const bool ascending = ((lk.w & 0xff) & 1) != 0;
    uint32_t* v = vals + lk.x;
    if(cnt <= 32) {
        for(int a = 1; a < cnt; ++a) {
            const uint32_t x = v[a];
            const int key = old_id[x];
            int b = a - 1;
            while(b >= 0 && leaf_before(key, old_id[v[b]], ascending)) {
                v[b + 1] = v[b];
                --b;
            }
            v[b + 1] = x;
        }
        return;
    }
    // heap sort (ids are unique, so stability is not needed)
    auto sift = [&](int root, int end) {
        while(true) {
            int child = 2 * root + 1;
            if(child >= end) break;
            if(child + 1 < end && leaf_before(old_id[v[child]], old_id[v[child + 1]], ascending)) ++child;
            if(!leaf_before(old_id[v[root]], old_id[v[child]], ascending)) break;
            const uint32_t t = v[root];
            v[root] = v[child];
            v[child] = t;
            root = child;
        }
    };
    for(int r = cnt / 2 - 1; r >= 0; --r) sift(r, cnt);
    for(int end = cnt - 1; end > 0; --end) {
        const uint32_t t = v[0];
        v[0] = v[end];
        v[end] = t;
        sift(0, end);
    }
}

__global__ void k_permute(int n, const uint32_t* __restrict__ src, DevState a, DevState b, int with_grad,
                          int* __restrict__ inv)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const int q = (int)src[p];
    b.pos[p] = a.pos[q];
    b.vel[p] = a.vel[q];
    b.acc[p] = a.acc[q];
    b.velp[p] = a.velp[q];
    b.thermo[p] = a.thermo[q];
    b.visc[p] = a.visc[q];
    const int id = a.id[q];
    b.id[p] = id;
    b.nbr[p] = a.nbr[q];
    inv[id] = p;
    if(with_grad) {
        for(int g = 0; g < 4; ++g) b.grad[(size_t)g * n + p] = a.grad[(size_t)g * n + q];
    }
    if(a.sr) {
        for(int g = 0; g < 4; ++g) b.sr[(size_t)g * n + p] = a.sr[(size_t)g * n + q];
    }
}

// Bottom-up mass / centre of mass (src/bhtree.cpp:154-204, 206-247).
__global__ void k_mass_up(int n, const int* __restrict__ leaf_of_start, DevTree T, const double4* __restrict__ pos,
                          DevStatus* __restrict__ st)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    int node = leaf_of_start[p];
    if(node < 0) return;
    {
        const int4 lk = T.link[node];
        double m = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
        // assign() accumulated in the parent's list order = reverse of ours
        for(int q = lk.y - 1; q >= lk.x; --q) {
            T.leaf_of[q] = node;
            const double4 pq = pos[q];
            m = __dadd_rn(m, pq.w);
            cx = __dadd_rn(cx, __dmul_rn(pq.x, pq.w));
            cy = __dadd_rn(cy, __dmul_rn(pq.y, pq.w));
            cz = __dadd_rn(cz, __dmul_rn(pq.z, pq.w));
        }
        if(m > 0.0) {
            cx = __ddiv_rn(cx, m);
            cy = __ddiv_rn(cy, m);
            cz = __ddiv_rn(cz, m);
        }
        T.mass[node] = make_double4(cx, cy, cz, m);
    }
    // at most 22 levels up, at most 8 children per node: bounded loops
    for(int up = 0; node != 0; ++up) {
        if(up > 64) {
            atomicOr(&st->pass_guard, PASS_GUARD_MASS);
            return;
        }
        const int par = T.parent[node];
        __threadfence();
        const int done = atomicAdd(&T.counter[par], 1);
        if(done != T.nchild[par] - 1) return;
        __threadfence();
        const int stop = T.link[par].z;
        double m = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
        int nch = 0;
        for(int ch = par + 1; ch != stop && nch < 8; ch = T.link[ch].z, ++nch) {
            const double2* q2 = reinterpret_cast<const double2*>(&T.mass[ch]);
            const double2 lo = __ldcg(q2), hi = __ldcg(q2 + 1);
            const double4 mc = make_double4(lo.x, lo.y, hi.x, hi.y);
            m = __dadd_rn(m, mc.w);
            cx = __dadd_rn(cx, __dmul_rn(mc.x, mc.w));
            cy = __dadd_rn(cy, __dmul_rn(mc.y, mc.w));
            cz = __dadd_rn(cz, __dmul_rn(mc.z, mc.w));
        }
        if(m > 0.0) {
            cx = __ddiv_rn(cx, m);
            cy = __ddiv_rn(cy, m);
            cz = __ddiv_rn(cz, m);
        }
        T.mass[par] = make_double4(cx, cy, cz, m);
        node = par;
    }
}

// BHNode::set_kernel (src/bhtree.cpp:249-275): max sml over the subtree.
__global__ void k_ksize_up(int n, const int* __restrict__ leaf_of_start, DevTree T, const double4* __restrict__ vel,
                           DevStatus* __restrict__ st)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    int node = leaf_of_start[p];
    if(node < 0) return;
    {
        const int4 lk = T.link[node];
        double k = 0.0;
        for(int q = lk.x; q < lk.y; ++q) {
            const double h = vel[q].w;
            if(h > k) k = h;
        }
        T.ksize[node] = k;
        for(int q = lk.x; q < lk.y; ++q) T.pks[q] = k;
    }
    for(int up = 0; node != 0; ++up) {
        if(up > 64) {
            atomicOr(&st->pass_guard, PASS_GUARD_KSIZE);
            return;
        }
        const int par = T.parent[node];
        __threadfence();
        const int done = atomicAdd(&T.counter[par], 1);
        if(done != T.nchild[par] - 1) return;
        __threadfence();
        const int stop = T.link[par].z;
        double k = 0.0;
        int nch = 0;
        for(int ch = par + 1; ch != stop && nch < 8; ch = T.link[ch].z, ++nch) {
            const double h = __ldcg(&T.ksize[ch]);
            if(h > k) k = h;
        }
        T.ksize[par] = k;
        node = par;
    }
}

}  // namespace

int tree_make(sphgpu_ctx* c)
{
    c->flist_ready = false;
    c->accabs_valid = false;
    const int n = c->n;
    cudaStream_t st = c->stream;
    if(n <= 0) return fail(c, SPHGPU_ERR_STATE, "tree_make: no particles");
    stage_begin(c, SPHGPU_T_TREE);
    const int D = c->prm.max_tree_level;
    // root cube
    const int nb = (int)std::min<long long>(grid_for(n, BLK), 1024);
    int launches = 3;  // root, keys, levels
    // node_pool, guard and nonfinite are adjacent words: clear all three, so an
    // earlier "no free node" does not outlive a new upload
    static_assert(offsetof(DevStatus, nonfinite) == offsetof(DevStatus, node_pool) + 2 * sizeof(int),
                  "status word layout");
    SPHGPU_CUDA(c, cudaMemsetAsync(&c->d_status->node_pool, 0, 3 * sizeof(int), st));
    k_bbox_partial<<<nb, BLK, 0, st>>>(c->s.pos, n, c->d_bbox_part, c->d_status);
    ++launches;
    k_root<<<1, 32, 0, st>>>(c->d_bbox_part, nb, c->dp, c->d_root);
    // keys + sort
    k_keys<<<grid_for(n, BLK), BLK, 0, st>>>(c->s.pos, n, c->d_root, D, c->d_keys, c->d_vals);
    launches += radix_sort(c->d_keys, c->d_vals, c->d_keys_alt, c->d_vals_alt, n, 3 * D, c->d_radix_scratch, st);
    // nodes
    k_levels<<<grid_for(n, BLK), BLK, 0, st>>>(c->d_keys, n, D, c->prm.leaf_particle_num, c->d_nstart, c->d_lvl);
    launches += exclusive_scan(c->d_nstart, c->d_base, n, (int*)nullptr, c->scan, st);
    SPHGPU_CUDA(c, cudaMemsetAsync(c->t.nchild, 0, sizeof(int) * (size_t)c->node_cap, st));
    SPHGPU_CUDA(c, cudaMemsetAsync(c->t.child, 0xff, sizeof(int) * 8 * (size_t)c->node_cap, st));
    k_nodes<<<grid_for(n, BLK), BLK, 0, st>>>(c->d_keys, n, D, c->d_nstart, c->d_base, c->d_lvl, c->d_root,
                                              c->node_cap, c->t, c->d_leaf_of_start, c->d_status);
    SPHGPU_LAUNCH_CHECK(c, "tree_make: node pass");
    SPHGPU_CUDA(c, cudaMemcpyAsync(&c->h_status, c->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost, st));
    int nnodes = 0;
    SPHGPU_CUDA(c, cudaMemcpyAsync(&nnodes, c->t.nnodes, sizeof(int), cudaMemcpyDeviceToHost, st));
    SPHGPU_CUDA(c, cudaStreamSynchronize(st));
    {
        // a bound hit by set_kernel or gravity since the last wait
        const int rcg = check_pass_guard(c);
        if(rcg < 0) {
            c->have_tree = false;
            return rcg;
        }
    }
    if(c->h_status.nonfinite) {
        c->have_tree = false;
        return fail(c, SPHGPU_ERR_STATE, "non-finite particle position");
    }
    if(c->h_status.node_pool) {
        c->have_tree = false;
        return fail(c, SPHGPU_ERR_NODE_POOL, "There is no free node.");
    }
    c->node_count = nnodes;
    // leaf order + permutation of the particle state
    k_leaf_order<<<grid_for(n, BLK), BLK, 0, st>>>(n, c->d_leaf_of_start, c->t.link, c->s.id, c->d_vals);
    k_permute<<<grid_for(n, BLK), BLK, 0, st>>>(n, c->d_vals, c->s, c->alt, c->prm.sph_type == SPHGPU_GSPH || c->prm.sph_type == SPHGPU_GDISPH ||
                                                    c->prm.sph_type == SPHGPU_SRGSPH,
                                                c->d_inv);
    std::swap(c->s, c->alt);
    {
        const int rcs = skin_permute(c, c->d_vals);  // skin lists follow the particles
        if(rcs < 0) return rcs;
    }
    // mass and centre of mass
    SPHGPU_CUDA(c, cudaMemsetAsync(c->t.counter, 0, sizeof(int) * (size_t)nnodes, st));
    k_mass_up<<<grid_for(n, BLK), BLK, 0, st>>>(n, c->d_leaf_of_start, c->t, c->s.pos, c->d_status);
    SPHGPU_LAUNCH_CHECK(c, "tree_make");
    launches += 4;  // nodes, leaf order, permute, mass
    stage_end(c, SPHGPU_T_TREE, launches);
    c->have_tree = true;
    return SPHGPU_OK;
}

int tree_set_kernel(sphgpu_ctx* c)
{
    if(!c->have_tree) return fail(c, SPHGPU_ERR_STATE, "set_kernel before tree make");
    cudaStream_t st = c->stream;
    stage_begin(c, SPHGPU_T_SET_KERNEL);
    SPHGPU_CUDA(c, cudaMemsetAsync(c->t.counter, 0, sizeof(int) * (size_t)c->node_count, st));
    k_ksize_up<<<grid_for(c->n, BLK), BLK, 0, st>>>(c->n, c->d_leaf_of_start, c->t, c->s.vel, c->d_status);
    SPHGPU_LAUNCH_CHECK(c, "set_kernel");
    stage_end(c, SPHGPU_T_SET_KERNEL, 1);
    return SPHGPU_OK;
}

}  // namespace sphgpu
