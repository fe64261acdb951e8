// tcpass.cuh -- the translation pass of many columns on the tensor cores
// (tcpass.cu): tcgen05 kind::tf32 with the three-product split, dense pair
// operators.
#pragma once
#include "common.cuh"
#include "gentran.cuh"

#define TC_M 128   // columns per M tile (the MMA's M)
#define TC_KC 8    // sources per chunk (one kind::tf32 MMA K step)

// Geometry of the tensor-core operators of a cluster whose spheres all have
// order L: a mode block holds nb = L(L+2) coefficients, padded to NP (a
// multiple of 16) rows and columns; NKC = NP/8 chunks of TC_KC = 8 sources
// (one MMA K step of TF32).
struct TcGeom {
    int L, nb, NP, NKC;
};
__host__ __device__ inline TcGeom tc_geom(int L)
{
    TcGeom g;
    g.L = L;
    g.nb = L * (L + 2);
    g.NP = (g.nb + 15) / 16 * 16;
    g.NKC = g.NP / TC_KC;
    return g;
}
// floats of the dense operator images of one ordered pair: 2 modes x NKC
// chunks x (hi, lo) x 2NP rows x TC_KC sources
__host__ __device__ inline size_t tc_himg_floats(const TcGeom& g) { return (size_t)2 * g.NKC * 2 * 2 * g.NP * TC_KC; }
// floats of the column images of one source sphere and M tile: 2 modes x NKC
// chunks x 4 planes (re hi, re lo, im hi, im lo) x 128 rows x TC_KC sources
__host__ __device__ inline size_t tc_aimg_floats(const TcGeom& g) { return (size_t)2 * g.NKC * 4 * TC_M * TC_KC; }
// M tiles one CTA of the pass carries (the operator chunks are loaded once
// for all of them): 2 when both accumulators fit the 512 tensor-memory columns
__host__ __device__ inline int tc_tiles_per_cta(const TcGeom& g, int nmt) { return nmt >= 2 && 4 * g.NP <= 512 ? 2 : 1; }

struct TcGenArgs {
    int nent;
    const int2* ent;       // (target, source) of each ordered pair
    const double* pos;
    TcGeom geo;
    double rimed_re, rimed_im;
    GtConst g;
    float* himg;           // nent x tc_himg_floats, zeroed by the caller
};
void launch_tc_gen(const TcGenArgs& a, cudaStream_t st);

struct TcPassArgs {
    int nsph;
    TcGeom geo;
    int ld, ncols, nmt;    // x, y: ld x ncols (FP32 complex); nmt = ceil(ncols / 128)
    const int* rstart;     // ordered pairs of target i: entries rstart[i] .. rstart[i+1]-1
    const int* rsrc;       // source sphere of each entry
    int nent;
    const float* himg;
    float* aimg;           // round_up(nmt, tiles per CTA) x nsph x tc_aimg_floats (written by the pass)
    const zf* x;
    zf* y;                 // accumulated into (zeroed by the caller)
    int* err;
};
// 0 on success, -1 when the geometry is not supported (NP > 128)
int launch_tc_pass(const TcPassArgs& a, int nsm, cudaStream_t st);
