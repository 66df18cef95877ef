// Shared device-side definitions for the fmmx engine: complex arithmetic,
// the per-order constant tables, and launch helpers.
//
// Expansion basis and index layout follow the reference FMM's solid harmonics
// (crates/fmm/src/harmonic.rs:76-86): coefficient (n, m), -n <= m <= n, lives at
// idx(n, m) = n(n+1) + m, and an order-p expansion holds dim(p) = (p+1)^2
// complex coefficients.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fmmx.h"

#define FMMX_MAXP 20
#define FMMX_MAXDIM ((FMMX_MAXP + 1) * (FMMX_MAXP + 1))
#define FMMX_BITS 21     // bits per axis of a Morton key (tree.rs:16)
#define FMMX_MAXLEVEL 21 // a cell at this level is always a leaf (tree.rs:414)
#define FMMX_NLEVELS (FMMX_MAXLEVEL + 1)

namespace fmmx {

__host__ __device__ __forceinline__ int dimp(int p) { return (p + 1) * (p + 1); }
__host__ __device__ __forceinline__ int cidx(int n, int m) { return n * (n + 1) + m; }

template <typename T>
struct cplx {
    T re, im;
};
typedef cplx<double> zd;
typedef cplx<float> zf;

template <typename T>
__host__ __device__ __forceinline__ cplx<T> mk(T r, T i) {
    cplx<T> z;
    z.re = r;
    z.im = i;
    return z;
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> zadd(cplx<T> a, cplx<T> b) {
    return mk<T>(a.re + b.re, a.im + b.im);
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> zsub(cplx<T> a, cplx<T> b) {
    return mk<T>(a.re - b.re, a.im - b.im);
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> zmul(cplx<T> a, cplx<T> b) {
    return mk<T>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> zscale(cplx<T> a, T s) {
    return mk<T>(a.re * s, a.im * s);
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> zconj(cplx<T> a) {
    return mk<T>(a.re, -a.im);
}

// Per-order constants, uploaded once per context (engine.cu).
// The tables cover every order up to FMMX_MAXP, so they are the same for all
// contexts: a context created with another p re-uploads identical contents
// and never changes the tables under a live context.
// Cell stride of the mixed form's half-layout expansions: (p+1)(p+2)/2 entries
// rounded up to even, so every cell starts on 16 bytes (FP32 complex) and the
// M2L can load entry pairs as float4. The padding entry is never read.
__host__ __device__ constexpr int half_stride(int p) {
    return (p + 1) * (p + 2) / 2 + (((p + 1) * (p + 2) / 2) & 1);
}

struct OrderTables {
    double fact[2 * FMMX_MAXP + 1];             // j!, j = 0..2 FMMX_MAXP (moments.rs:11-17)
    double binom[FMMX_MAXP + 1][FMMX_MAXP + 1]; // binom[p][k] = C(p, k) as p!/(k!(p-k)!) (moments.rs:20-27)
    double inv2m[FMMX_MAXP + 1];                // 1/(2m) (harmonic.rs:150)
    double invc[FMMX_MAXP + 1][FMMX_MAXP + 1];  // 1/(n^2 - m^2) (harmonic.rs:156,162)
};

// Morton-tree description shared by the build and walk kernels. All arrays are
// in depth-first pre-order cell numbering (parents before children, children
// in octant order), the numbering of the reference's build_rec (tree.rs:404).
struct CellsView {
    const uint32_t* first;
    const uint32_t* count;
    const int32_t* child;  // 8 per cell, -1 if absent
    const uint8_t* leaf;
    const uint8_t* level;
    const double* cx;
    const double* cy;
    const double* cz;
    const double* mass;
    const double* rho;
    const double4* geo;  // cx, cy, cz, rho of each cell in one 32-byte record (the walk's loads)
};

// SM count of the device, read when a context is created (grid sizes of the
// grid-stride and persistent kernels are multiples of it)
inline int g_nsm = 148;

// blocks for n items at `block` threads, at most cap (default 32 per SM; the
// kernels stride over the rest)
static inline unsigned grid_for(size_t n, int block, unsigned cap = 0) {
    if (cap == 0) cap = 32u * (unsigned)g_nsm;
    size_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

}  // namespace fmmx
