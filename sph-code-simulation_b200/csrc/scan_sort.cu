// scan_sort.cu — device-wide exclusive scan and stable LSD radix sort.
//
// The octree build sorts particles by their Morton-path keys (BHTree::make
// replacement, src/bhtree.cpp:59-115).  The sort is a classic three-kernel LSD
// radix sort with 8-bit digits:
//   1. histogram of each 2048-key tile (digit-major [256][tiles] layout),
//   2. exclusive scan of the histograms = global digit offsets per tile,
//   3. scatter: keys are ranked stably inside the tile (warp match + per-warp
//      counts), staged digit-contiguously in shared memory, then written out
//      so that consecutive threads store consecutive addresses.
// All traffic is streaming and HBM-bound: per pass each key/value is read
// twice and written once.
#include <cstdint>
#include <cuda_runtime.h>

#include "scan_sort.cuh"

namespace sphgpu {

namespace {

constexpr int SCAN_BLOCK = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for(int o = 1; o < 32; o <<= 1) {
        const T u = __shfl_up_sync(0xffffffffu, v, o);
        if(lane >= o) v += u;
    }
    return v;
}

// Exclusive scan of one value per thread across the block; returns the
// block total in *total.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* smem /* >= 32 */, T* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const T incl = warp_incl_scan(v);
    if(lane == 31) smem[warp] = incl;
    __syncthreads();
    if(warp == 0) {
        T s = lane < nwarps ? smem[lane] : T(0);
        const T si = warp_incl_scan(s);
        if(lane < nwarps) smem[lane] = si - s;
        if(lane == nwarps - 1) smem[32] = si;
    }
    __syncthreads();
    const T r = incl - v + smem[warp];
    *total = smem[32];
    __syncthreads();
    return r;
}

template <typename T>
__global__ void k_tile_reduce(const T* __restrict__ in, long long n, T* __restrict__ sums)
{
    __shared__ T sm[33];
    const long long base = (long long)blockIdx.x * SCAN_TILE;
    T acc = 0;
#pragma unroll
    for(int k = 0; k < SCAN_ITEMS; ++k) {
        const long long i = base + (long long)k * SCAN_BLOCK + threadIdx.x;
        if(i < n) acc += in[i];
    }
    T tot;
    block_excl_scan(acc, sm, &tot);
    if(threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Exclusive scan of one tile, plus an optional per-tile offset.
template <typename T>
__global__ void k_tile_scan(const T* __restrict__ in, long long n, T* __restrict__ out,
                            const T* __restrict__ offsets, T* __restrict__ total)
{
    __shared__ T sm[33];
    const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    T v[SCAN_ITEMS];
    T acc = 0;
#pragma unroll
    for(int k = 0; k < SCAN_ITEMS; ++k) {
        const long long i = base + k;
        v[k] = i < n ? in[i] : T(0);
        acc += v[k];
    }
    T tot;
    T run = block_excl_scan(acc, sm, &tot);
    if(offsets) run += offsets[blockIdx.x];
#pragma unroll
    for(int k = 0; k < SCAN_ITEMS; ++k) {
        const long long i = base + k;
        if(i < n) out[i] = run;
        run += v[k];
    }
    if(total && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) *total = run;
}

// returns the number of kernels launched
template <typename T>
int scan_rec(const T* in, T* out, long long n, T* total, ScanScratch& s, int depth, cudaStream_t st)
{
    const long long tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if(tiles <= 1) {
        k_tile_scan<T><<<1, SCAN_BLOCK, 0, st>>>(in, n, out, (const T*)nullptr, total);
        return 1;
    }
    T* sums = reinterpret_cast<T*>(s.level[depth]);
    T* sums_scanned = sums + tiles;
    k_tile_reduce<T><<<(unsigned)tiles, SCAN_BLOCK, 0, st>>>(in, n, sums);
    const int inner = scan_rec<T>(sums, sums_scanned, tiles, (T*)nullptr, s, depth + 1, st);
    k_tile_scan<T><<<(unsigned)tiles, SCAN_BLOCK, 0, st>>>(in, n, out, sums_scanned, total);
    return inner + 2;
}

// ------------------------------------------------------------------ radix
constexpr int RS_BLOCK = 256;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_BLOCK * RS_ITEMS;
constexpr int RS_WARPS = RS_BLOCK / 32;

__global__ void k_rs_hist(const uint64_t* __restrict__ keys, int n, int shift, unsigned* __restrict__ hist,
                          int ntiles)
{
    __shared__ unsigned h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * RS_TILE;
#pragma unroll
    for(int k = 0; k < RS_ITEMS; ++k) {
        const long long i = base + (long long)k * RS_BLOCK + threadIdx.x;
        if(i < n) atomicAdd(&h[(keys[i] >> shift) & 0xff], 1u);
    }
    __syncthreads();
    hist[(long long)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_BLOCK) k_rs_scatter(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                         uint64_t* __restrict__ kout, uint32_t* __restrict__ vout, int n,
                                                         int shift, const unsigned* __restrict__ hist_local,
                                                         const unsigned* __restrict__ hist_scanned, int ntiles)
{
    __shared__ unsigned s_goff[256];       // global offset of digit d for this tile
    __shared__ unsigned s_loff[256];       // tile-local start of digit d
    __shared__ unsigned s_run[256];        // keys of digit d already placed
    __shared__ unsigned s_wcnt[RS_WARPS][256];
    __shared__ unsigned s_scan[33];
    __shared__ uint64_t s_key[RS_TILE];
    __shared__ uint32_t s_val[RS_TILE];

    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const long long base = (long long)blockIdx.x * RS_TILE;
    const unsigned cnt = hist_local[(long long)t * ntiles + blockIdx.x];
    s_goff[t] = hist_scanned[(long long)t * ntiles + blockIdx.x];
    unsigned tot;
    s_loff[t] = block_excl_scan(cnt, s_scan, &tot);
    s_run[t] = 0;
    for(int w = 0; w < RS_WARPS; ++w) s_wcnt[w][t] = 0;
    __syncthreads();

    const unsigned lt_mask = (1u << lane) - 1u;
    for(int r = 0; r < RS_ITEMS; ++r) {
        const long long i = base + (long long)r * RS_BLOCK + t;
        const bool valid = i < n;
        uint64_t key = 0;
        uint32_t val = 0;
        unsigned d = 256;  // sentinel for the tail
        if(valid) {
            key = kin[i];
            val = vin[i];
            d = (unsigned)((key >> shift) & 0xff);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned rank = __popc(peers & lt_mask);
        const int leader = __ffs(peers) - 1;
        if(valid && lane == leader) s_wcnt[warp][d] = __popc(peers);
        __syncthreads();
        // per digit: prefix over warps (warp order = key order in the round)
        {
            unsigned run = s_run[t];
            for(int w = 0; w < RS_WARPS; ++w) {
                const unsigned c = s_wcnt[w][t];
                s_wcnt[w][t] = run;
                run += c;
            }
            s_run[t] = run;
        }
        __syncthreads();
        if(valid) {
            const unsigned lp = s_loff[d] + s_wcnt[warp][d] + rank;
            s_key[lp] = key;
            s_val[lp] = val;
        }
        __syncthreads();
        for(int w = 0; w < RS_WARPS; ++w) s_wcnt[w][t] = 0;
        __syncthreads();
    }
    const int count = (int)min((long long)RS_TILE, (long long)n - base);
    for(int k = t; k < count; k += RS_BLOCK) {
        const uint64_t key = s_key[k];
        const unsigned d = (unsigned)((key >> shift) & 0xff);
        const unsigned o = s_goff[d] + (unsigned)k - s_loff[d];
        kout[o] = key;
        vout[o] = s_val[k];
    }
}

}  // namespace

size_t scan_scratch_bytes(long long n)
{
    // geometric series of per-level tile sums (x2 for scanned copies), padded
    size_t total = 0;
    long long m = n;
    while(m > SCAN_TILE) {
        m = (m + SCAN_TILE - 1) / SCAN_TILE;
        total += (size_t)(2 * m + 64) * 8;
    }
    return total + 1024;
}

void scan_scratch_init(ScanScratch& s, void* buf, long long n)
{
    char* p = static_cast<char*>(buf);
    long long m = n;
    int d = 0;
    while(m > SCAN_TILE && d < ScanScratch::MAXLEV) {
        m = (m + SCAN_TILE - 1) / SCAN_TILE;
        s.level[d++] = p;
        p += (size_t)(2 * m + 64) * 8;
    }
}

int exclusive_scan(const int* in, int* out, long long n, int* total, ScanScratch& s, cudaStream_t st)
{
    return scan_rec<int>(in, out, n, total, s, 0, st);
}
int exclusive_scan(const unsigned* in, unsigned* out, long long n, unsigned* total, ScanScratch& s, cudaStream_t st)
{
    return scan_rec<unsigned>(in, out, n, total, s, 0, st);
}
int exclusive_scan(const unsigned long long* in, unsigned long long* out, long long n, unsigned long long* total,
                   ScanScratch& s, cudaStream_t st)
{
    return scan_rec<unsigned long long>(in, out, n, total, s, 0, st);
}

size_t radix_scratch_bytes(int n)
{
    const long long ntiles = (n + RS_TILE - 1) / RS_TILE;
    return (size_t)(2 * 256 * ntiles) * sizeof(unsigned) + scan_scratch_bytes(256 * ntiles) + 1024;
}

// Sorts (keys, vals) by the low `bits` bits of the keys; results end up in
// (keys, vals) again (the alternate buffers are used as ping-pong).
int radix_sort(uint64_t*& keys, uint32_t*& vals, uint64_t*& keys_alt, uint32_t*& vals_alt, int n, int bits,
               void* scratch, cudaStream_t st)
{
    if(n <= 1) return 0;
    int launches = 0;
    const int ntiles = (n + RS_TILE - 1) / RS_TILE;
    unsigned* hist = static_cast<unsigned*>(scratch);
    unsigned* hscan = hist + (size_t)256 * ntiles;
    ScanScratch ss;
    scan_scratch_init(ss, hscan + (size_t)256 * ntiles, 256LL * ntiles);
    for(int shift = 0; shift < bits; shift += 8) {
        k_rs_hist<<<ntiles, RS_BLOCK, 0, st>>>(keys, n, shift, hist, ntiles);
        launches += 2 + exclusive_scan(hist, hscan, 256LL * ntiles, (unsigned*)nullptr, ss, st);
        k_rs_scatter<<<ntiles, RS_BLOCK, 0, st>>>(keys, vals, keys_alt, vals_alt, n, shift, hist, hscan, ntiles);
        uint64_t* tk = keys;
        keys = keys_alt;
        keys_alt = tk;
        uint32_t* tv = vals;
        vals = vals_alt;
        vals_alt = tv;
    }
    return launches;
}

}  // namespace sphgpu
