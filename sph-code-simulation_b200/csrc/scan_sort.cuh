// scan_sort.cuh — device-wide exclusive scan and stable LSD radix sort.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace sphgpu {

struct ScanScratch {
    static constexpr int MAXLEV = 8;
    void* level[MAXLEV] = {nullptr};
};

size_t scan_scratch_bytes(long long n);
void scan_scratch_init(ScanScratch& s, void* buf, long long n);
// out[i] = sum(in[0..i)); *total (device pointer, may be null) = sum(in).
// Each returns the number of kernels it launched.
int exclusive_scan(const int* in, int* out, long long n, int* total, ScanScratch& s, cudaStream_t st);
int exclusive_scan(const unsigned* in, unsigned* out, long long n, unsigned* total, ScanScratch& s, cudaStream_t st);
int exclusive_scan(const unsigned long long* in, unsigned long long* out, long long n, unsigned long long* total,
                    ScanScratch& s, cudaStream_t st);

size_t radix_scratch_bytes(int n);
int radix_sort(uint64_t*& keys, uint32_t*& vals, uint64_t*& keys_alt, uint32_t*& vals_alt, int n, int bits,
                void* scratch, cudaStream_t st);

}  // namespace sphgpu
