// translate_tiled.cuh -- tiled fast path of the pair translation pass.
#pragma once
#include "common.cuh"

#define TILE_B 4   // spheres per block: a tile holds the pairs of two blocks

template <typename T> struct TiledArgs {
    int ntiles;
    const int4* tiles;       // (pair start, pair count, (i0<<16)|j0 -- grouped tiles: the row of tsph --, diagonal)
    const int2* pairs;       // tile-ordered pairs, i < j
    const T* ops;            // records in pair order, op_record_units(L,L) each
    const cpx<T>* x;         // ld x nrhs
    cpx<T>* y;               // ld x nrhs, accumulated
    int ld, nrhs, nsph;      // nrhs: columns per chunk (the kernel's NR)
    int nchunk;              // chunks of nrhs columns: x and y hold nrhs * nchunk columns
    unsigned contran;        // bit r: column r of every chunk is a conjugate-transpose product
    int ctas_per_sm;         // 0: as many as shared memory and the register budget allow
    int* err;
    // grouped tiles (null for block tiles): tile t's spheres by slot,
    // tsph[t * 2B + slot] (-1: none), and each pair's (slot of i, slot of j)
    const int* tsph = nullptr;
    const short2* pslot = nullptr;
    int pairs_per_step = 0;  // 2: two slot-disjoint pairs a step (FP32, one or two columns); otherwise one
    // sphere i's block at soff[i] (complex units; null: i * 2L(L+2), the
    // layout of a cluster of one order; set with host spheres, whose internal
    // blocks sit between the others')
    const int* soff = nullptr;
};
// start of sphere i's block in a vector of the tiled path; SO (per-sphere
// offsets) is a template argument of the kernels, so the clusters of one
// order pay no branch on a.soff in their inner loops
template <bool SO, typename T> __device__ __forceinline__ size_t tile_sphere_base(const TiledArgs<T>& a, int i, int NB)
{
    if constexpr (SO) return (size_t)a.soff[i];
    else return (size_t)i * NB;
}

bool tiled_supported(int L, int nrhs);
// one CTA runs the kernels' bounded mbarrier wait on a barrier no copy completes
int launch_wait_selftest(int limit, int* err, cudaStream_t st);
template <typename T> int launch_translate_tiled(const TiledArgs<T>& a, int L, int nsm, cudaStream_t st);
