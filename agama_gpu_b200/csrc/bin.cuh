// bin.cuh -- per-call counting sort of the points by radial interval.
//
// The Multipole hot loop reads, for each harmonic, the six quintic
// coefficients of the point's radial interval.  With points in random order
// the 32 lanes of a warp read from up to 32 different intervals (32 cache
// lines per load).  Sorting the points by the interval of the heaviest
// Multipole leaf makes a warp's lanes share one interval, so every
// coefficient load is a single broadcast served from L1.
//
// Three launches, all stream-ordered:
//   1. bin_count:   key per point -> keys[], block-local shared-memory
//                   histogram, one global atomic per (block, bin)
//   2. bin_scan:    one block, exclusive scan of the bin counts -> offsets
//   3. bin_scatter: the same tiles as pass 1; each block reserves its range
//                   in every bin with one global atomic, then places its
//                   points: perm[pos] = i, keys[i] = pos (overwriting the
//                   key) and a sorted AoS copy of xyz
// Within a bin the order is not deterministic; each point's result does not
// depend on it.
#pragma once
#include "agb_dev.cuh"

#define AGB_BIN_TILE_MAX 4096      // points per block in passes 1 and 3 (at most)
#define AGB_MAX_BINS 8192

struct BinKey {
    double sigma, g0, g1, g2;     // frame of the keyed Multipole leaf
    const DevLeaf* leaf;          // or, when set, that leaf in device memory
    double logr_min, inv_dlogr;
    int n_int;
    // Output blocks: the key of point i is (i >> log_block) * (n_int + 2) + its
    // interval, so the sorted order runs through the points block by block.  A
    // kernel that walks the sorted order then writes its (permuted) outputs into
    // one block-sized window at a time, which L2 holds and merges, instead of
    // scattering partial-sector writes over the whole output array.
    int log_block;
    int comp;                     // batches: the keyed leaf's component (-1: none)
};

// in-grid interval k in [0, n_int), n_int for the inner region (and the
// origin / NaN), n_int + 1 beyond the grid
__device__ __forceinline__ int bin_of(const BinKey& b, double x, double y, double z)
{
    const double lx = b.sigma * x - b.g0, ly = b.sigma * y - b.g1, lz = b.sigma * z - b.g2;
    const double r = sqrt(lx * lx + ly * ly + lz * lz);
    if (!(r >= 1.0e-300)) return b.n_int;
    const double t = (log(r) - b.logr_min) * b.inv_dlogr;
    if (t < 0.0) return b.n_int;
    if (t >= (double)b.n_int) return b.n_int + 1;
    return (int)t;
}

__global__ void __launch_bounds__(256)
bin_count(const double* __restrict__ xyz, long long n, int tile, BinKey b, int n_bins,
          int* __restrict__ keys, int* __restrict__ counts)
{
    extern __shared__ int hist[];
    if (b.leaf) {                 // the leaf's frame at this call's time (agb_eval_timed)
        b.sigma = b.leaf->sigma;
        b.g0 = b.leaf->g0; b.g1 = b.leaf->g1; b.g2 = b.leaf->g2;
    }
    for (int q = threadIdx.x; q < n_bins; q += blockDim.x) hist[q] = 0;
    __syncthreads();
    const long long lo = (long long)blockIdx.x * tile;
    const long long hi = min(lo + (long long)tile, n);
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const int k = bin_of(b, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]) +
                      (int)(i >> b.log_block) * (b.n_int + 2);
        keys[i] = k;
        atomicAdd(&hist[k], 1);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n_bins; q += blockDim.x)
        if (hist[q]) atomicAdd(&counts[q], hist[q]);
}

// single block: cursor[q] = sum_{p<q} counts[p]
__global__ void __launch_bounds__(1024)
bin_scan(const int* __restrict__ counts, int* __restrict__ cursor, int n_bins)
{
    __shared__ int part[1024];
    const int per = (n_bins + blockDim.x - 1) / blockDim.x;
    const int q0 = threadIdx.x * per;
    int s = 0;
    for (int q = q0; q < min(q0 + per, n_bins); ++q) s += counts[q];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {     // Hillis-Steele inclusive scan
        const int v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int base = part[threadIdx.x] - s;
    for (int q = q0; q < min(q0 + per, n_bins); ++q) {
        cursor[q] = base;
        base += counts[q];
    }
}

__global__ void __launch_bounds__(256)
bin_scatter(const double* __restrict__ xyz, long long n, int tile, int n_bins,
            int* __restrict__ keys, int* __restrict__ cursor,
            int* __restrict__ perm, double* __restrict__ xyz_sorted)
{
    extern __shared__ int sm[];
    int* hist = sm;              // local counts, then local cursors
    int* base = sm + n_bins;     // this block's reserved start in each bin
    for (int q = threadIdx.x; q < n_bins; q += blockDim.x) hist[q] = 0;
    __syncthreads();
    const long long lo = (long long)blockIdx.x * tile;
    const long long hi = min(lo + (long long)tile, n);
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&hist[keys[i]], 1);
    __syncthreads();
    for (int q = threadIdx.x; q < n_bins; q += blockDim.x) {
        const int c = hist[q];
        base[q] = c ? atomicAdd(&cursor[q], c) : 0;
        hist[q] = 0;
    }
    __syncthreads();
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const int k = keys[i];
        const long long pos = (long long)base[k] + atomicAdd(&hist[k], 1);
        if (perm) perm[pos] = (int)i;
        keys[i] = (int)pos;          // from here on: where point i went (the inverse of perm)
        xyz_sorted[3 * pos] = xyz[3 * i];
        xyz_sorted[3 * pos + 1] = xyz[3 * i + 1];
        xyz_sorted[3 * pos + 2] = xyz[3 * i + 2];
    }
}
