// Row-dictionary build on the GPU.
//
// Every row of an operator given as coefficient planes (planes[o*n + i]) gets
// the class id of its first bit-identical occurrence, ids in first-seen order,
// and the distinct rows are gathered into a table (row-major, noff values per
// row).  Steps:
//   1. k_dict_insert: each row hashes its noff coefficient bit patterns and
//      claims a slot of an open-addressing table (capacity >= 2n, linear
//      probing, atomicCAS on the 64-bit key); the slot keeps the smallest row
//      index with that hash (atomicMin) as the representative;
//   2. k_dict_lookup: each row finds its slot again, compares itself with the
//      representative value by value (two different rows with one hash set a
//      flag and the caller falls back to the host build), and marks whether
//      it is its own representative;
//   3. tile counts, one-block scan of the counts, and a per-tile block scan
//      number the representatives in row order; every row then takes its
//      representative's number and the representatives copy their rows into
//      the table.
// The result equals a serial first-seen dedup bit for bit.
#pragma once

#include <climits>
#include <cstdint>

#include "lsg_kernels.cuh"

namespace lsg {

constexpr unsigned long long kDictEmpty = ~0ull;
constexpr int kDictTile = 1024;

__device__ __forceinline__ unsigned long long dict_row_hash(const double* __restrict__ planes, int noff,
                                                            long long n, long long i)
{
    unsigned long long x = 0x9E3779B97F4A7C15ull;
    for (int o = 0; o < noff; o++) {
        const unsigned long long w = (unsigned long long)__double_as_longlong(planes[(size_t)o * n + i]);
        x ^= w + 0x9E3779B97F4A7C15ull + (x << 6) + (x >> 2);
        x *= 0xBF58476D1CE4E5B9ull;
        x ^= x >> 31;
    }
    return x == kDictEmpty ? x - 1 : x;                    // the empty key stays reserved
}

__global__ void k_dict_insert(int noff, long long n, const double* __restrict__ planes, unsigned long long* keys,
                              int* rep, unsigned long long mask)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long h = dict_row_hash(planes, noff, n, i);
        unsigned long long q = h & mask;
        // capacity >= 2n: a free or matching slot exists within mask + 1 probes
        for (unsigned long long probe = 0; probe <= mask; probe++) {
            const unsigned long long prev = atomicCAS(keys + q, kDictEmpty, h);
            if (prev == kDictEmpty || prev == h) {
                atomicMin(rep + q, (int)i);
                break;
            }
            q = (q + 1) & mask;
        }
    }
}

// repidx[i] = the representative of row i; first[i] = 1 if row i is one.
__global__ void k_dict_lookup(int noff, long long n, const double* __restrict__ planes,
                              const unsigned long long* __restrict__ keys, const int* __restrict__ rep,
                              unsigned long long mask, int* __restrict__ repidx, int* __restrict__ first, int* flag)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long h = dict_row_hash(planes, noff, n, i);
        unsigned long long q = h & mask;
        int r = -1;
        for (unsigned long long probe = 0; probe <= mask; probe++) {
            const unsigned long long k = keys[q];
            if (k == h) {
                r = rep[q];
                break;
            }
            if (k == kDictEmpty) break;
            q = (q + 1) & mask;
        }
        bool same = r >= 0 && r < n;
        for (int o = 0; same && o < noff; o++)
            same = __double_as_longlong(planes[(size_t)o * n + i]) == __double_as_longlong(planes[(size_t)o * n + r]);
        if (!same) {
            atomicOr(flag, 1);
            r = (int)i;
        }
        repidx[i] = r;
        first[i] = (r == (int)i) ? 1 : 0;
    }
}

// Block-wide exclusive scan of one int per thread (blockDim.x == kDictTile).
__device__ __forceinline__ int dict_block_scan(int v, int* warp_sums, int& total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;                               // inclusive sums of the warps
    }
    __syncthreads();
    total = warp_sums[(blockDim.x >> 5) - 1];
    const int before = wid > 0 ? warp_sums[wid - 1] : 0;
    __syncthreads();
    return before + x - v;
}

// tile_sum[t] = number of representatives in tile t (kDictTile rows).
__global__ void __launch_bounds__(kDictTile) k_dict_tile_count(long long n, const int* __restrict__ first,
                                                              int* __restrict__ tile_sum)
{
    __shared__ int ws[32];
    const long long i = blockIdx.x * (long long)kDictTile + threadIdx.x;
    int total;
    dict_block_scan(i < n ? first[i] : 0, ws, total);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// In-place exclusive scan of the tile counts by one block; *nclass = total.
__global__ void __launch_bounds__(kDictTile) k_dict_scan_tiles(int ntiles, int* tile_sum, int* nclass)
{
    __shared__ int ws[32];
    int carry = 0;
    for (int base = 0; base < ntiles; base += kDictTile) {
        const int t = base + (int)threadIdx.x;
        const int v = t < ntiles ? tile_sum[t] : 0;
        int total;
        const int ex = dict_block_scan(v, ws, total);
        if (t < ntiles) tile_sum[t] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) *nclass = carry;
}

// Class numbers of the representatives (in row order) and their rows into
// the table; first[i] <- the class number of representative i.
__global__ void __launch_bounds__(kDictTile) k_dict_number(int noff, long long n, const double* __restrict__ planes,
                                                          const int* __restrict__ tile_off, int* __restrict__ first,
                                                          double* __restrict__ dict)
{
    __shared__ int ws[32];
    const long long i = blockIdx.x * (long long)kDictTile + threadIdx.x;
    const int f = i < n ? first[i] : 0;
    int total;
    const int id = tile_off[blockIdx.x] + dict_block_scan(f, ws, total);
    if (i < n && f) {
        first[i] = id;
        for (int o = 0; o < noff; o++) dict[(size_t)id * noff + o] = planes[(size_t)o * n + i];
    }
}

__global__ void k_dict_classes(long long n, const int* __restrict__ repidx, const int* __restrict__ number,
                               int* __restrict__ cls)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        cls[i] = number[repidx[i]];
}

}  // namespace lsg
