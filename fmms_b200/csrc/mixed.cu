// Mixed-precision form: FP32 expansions and P2P, FP64 only where the reference
// needs it (centre-relative coordinates, the MAC, M2M/L2L on the top three
// tree levels).
//
// Expansions are stored for m >= 0 only (a real field has
// v_{-m} = (-1)^m conj(v_m)) and normalised by a per-cell length l (the cell's
// radius rho, or a small fraction of its box size when rho = 0):
//     M^_n^m = M_n^m / l^n,      F^_n^m = F_n^m l^{n+1}.
// Every translation then works on O(1) quantities, so FP32 neither overflows
// nor underflows at p = 12 for cells down to the level-21 cut:
//   P2M: M^_n^m  = sum_b m_b Υ_n^m((x_b - s)/l)
//   M2M: M^_p[n][m] = sum_k sum_l Υ_k^l((s_c - s_p)/l_p) M^_c[n-k][m-l] (l_c/l_p)^{n-k}
//   L2L: F^_c[n][m] = (l_c/l_p)^{n+1} sum_{k,l} conj(Υ_k^l((s_p - s_c)/l_p)) F^_p[n+k][m+l]
//   L2P: Ψ_0^0 = (1/l) sum conj(Υ_k^l(r^)) F^_k^l,  Ψ_1^m = (1/l^2) sum conj(Υ_k^l(r^)) F^_{k+1}^{m+l}
// (the unnormalised forms are moments.rs:30-90 and translate.rs:175-309).
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace fmmx {

// The order tables in global memory: the kernels read them with lane-
// dependent indices (a lane per order m or per degree), which the constant
// cache would serialise over the distinct addresses; global loads are served
// from L1 in parallel.
static __device__ OrderTables g_tab;

void upload_tables_mixed(const OrderTables& t, cudaStream_t s) {
    cudaMemcpyToSymbolAsync(g_tab, &t, sizeof(t), 0, cudaMemcpyHostToDevice, s);
}

__host__ __device__ constexpr int hx(int n, int m) { return n * (n + 1) / 2 + m; }

__device__ __forceinline__ void split_h(int e, int& n, int& m) {
    int q = (int)((sqrtf(8.0f * e + 1.0f) - 1.0f) * 0.5f);
    while (q * (q + 1) / 2 > e) --q;
    while ((q + 1) * (q + 2) / 2 <= e) ++q;
    n = q;
    m = e - q * (q + 1) / 2;
}

// v_{n,m} for any m from the half store (m >= 0)
template <typename T>
__device__ __forceinline__ cplx<T> half_get(const cplx<T>* v, int n, int m) {
    if (m >= 0) return v[hx(n, m)];
    const cplx<T> w = v[hx(n, -m)];
    return ((-m) & 1) ? mk<T>(-w.re, w.im) : mk<T>(w.re, -w.im);
}

// Υ column m (harmonic.rs:141-173) of r into u (half layout), precision A.
template <typename A>
__device__ __forceinline__ void ups_column(A x, A y, A z, A r2, int p, int m, cplx<A>* u) {
    cplx<A> d = mk<A>(A(1), A(0));
    for (int j = 1; j <= m; ++j) d = zmul(zscale(mk<A>(x, y), (A)g_tab.inv2m[j]), d);
    u[hx(m, m)] = d;
    cplx<A> u1 = d, u2 = mk<A>(A(0), A(0));
    for (int n = m + 1; n <= p; ++n) {
        const A a = (A)(2 * n - 1) * z;
        cplx<A> un = zscale(zsub(zscale(u1, a), zscale(u2, r2)), (A)g_tab.invc[n][m]);
        u[hx(n, m)] = un;
        u2 = u1;
        u1 = un;
    }
}

// Normalising length of every cell: rho, or the cell's box size h when rho = 0
// (a single body, or coincident bodies: then every moment above the monopole
// is exactly zero and any positive length works), kept >= 1e-30 so that it is
// a normal FP32 number (a system of coincident bodies has box size DBL_MIN).
__global__ void k_cell_scale(int nc, const double* __restrict__ rho, const double* __restrict__ h,
                             double* __restrict__ ell, float* __restrict__ ellf) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        double l = rho[c];
        if (!(l > 0.0)) l = h[c];
        l = fmax(l, 1e-30);
        ell[c] = l;
        ellf[c] = (float)l;
    }
}

// Cell radii about the build's centres for the current positions, on a
// reused tree: the bodies have drifted since the build, and a cell whose built
// radius is tiny (a tight pair) would otherwise normalise its moments by a
// length far below the bodies' distances from its centre, overflowing FP32
// (M_n / l^n). Never below the built radius. Leaves from their bodies (an
// atomic max on the bit pattern, which orders like the value for
// non-negative doubles), internal cells from their children, deepest level
// first (the construction of tree.rs:152-227 with the centres held fixed).
__global__ void k_rho_bodies(size_t n, const int32_t* __restrict__ body_leaf, CellsView cv,
                             const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, unsigned long long* __restrict__ rho_bits) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int c = body_leaf[k];
        const double dx = x[k] - cv.cx[c], dy = y[k] - cv.cy[c], dz = z[k] - cv.cz[c];
        const double d = sqrt(dx * dx + dy * dy + dz * dz);
        atomicMax(rho_bits + c, (unsigned long long)__double_as_longlong(d));
    }
}
__global__ void k_rho_level(const int32_t* __restrict__ level_cells, int lstart, int lcnt, CellsView cv,
                            unsigned long long* __restrict__ rho_bits) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lcnt; j += gridDim.x * blockDim.x) {
        const int c = level_cells[lstart + j];
        double r = fmax(cv.rho[c], __longlong_as_double((long long)rho_bits[c]));
        if (!cv.leaf[c]) {
            for (int o = 0; o < 8; ++o) {
                const int ch = cv.child[8 * c + o];
                if (ch < 0) continue;
                const double dx = cv.cx[ch] - cv.cx[c], dy = cv.cy[ch] - cv.cy[c], dz = cv.cz[ch] - cv.cz[c];
                r = fmax(r, __longlong_as_double((long long)rho_bits[ch]) + sqrt(dx * dx + dy * dy + dz * dz));
            }
        }
        rho_bits[c] = (unsigned long long)__double_as_longlong(r);
    }
}

// FP64 full-layout moments (the exact upward pass) -> normalised FP32 half layout.
__global__ void k_moments_to_mixed(int nc, int p, const zd* __restrict__ full, const double* __restrict__ ell,
                                   zf* __restrict__ half) {
    const int H = (p + 1) * (p + 2) / 2, D = (p + 1) * (p + 1), HS = half_stride(p);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)nc * H;
         i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i / H), e = (int)(i % H);
        int n, m;
        split_h(e, n, m);
        const double s = pow(ell[c], -n);
        const zd v = full[(size_t)c * D + n * (n + 1) + m];
        half[(size_t)c * HS + e] = mk<float>((float)(v.re * s), (float)(v.im * s));
    }
}

// P2M / M2M for one level, one 128-thread CTA per cell. A = accumulation type
// (double on the top three levels, float below). Output FP32 half layout.
//  - leaf (P2M): thread t takes column m = t % (p+1) of the bodies
//    g, g+G, g+2G, ... (g = t / (p+1), G <= 8 groups), accumulating the column
//    in its own shared-memory entries; the group partials are then summed in a
//    fixed order;
//  - internal (M2M): first the Υ tables of the eight child offsets (one thread
//    per child and column), then one thread per (child, entry) computes that
//    child's contribution, and the children are summed in octant order.
#define UPM_BLOCK 128
template <typename A>
__global__ void __launch_bounds__(UPM_BLOCK) k_upward_mixed(const int32_t* __restrict__ level_cells, int lstart,
                                                            int lcnt, CellsView cv, const double* __restrict__ ell,
                                                            const double* __restrict__ x,
                                                            const double* __restrict__ y,
                                                            const double* __restrict__ z,
                                                            const double* __restrict__ m, int p,
                                                            zf* __restrict__ mom) {
    extern __shared__ unsigned char smem_raw[];
    const int H = (p + 1) * (p + 2) / 2;
    const int P1 = p + 1;
    cplx<A>* u = reinterpret_cast<cplx<A>*>(smem_raw);  // 8 x H: Υ of the child offsets
    cplx<A>* part = u + 8 * H;                          // 8 x H: partial sums
    zf* cm = reinterpret_cast<zf*>(part + 8 * H);       // 8 x H: the children's moments
    A* bod = reinterpret_cast<A*>(cm + 8 * H);          // 4 x UPM_BLOCK: a chunk of the leaf's bodies
    const int tid = threadIdx.x;
    const int G = min(8, UPM_BLOCK / P1);
    for (int j = blockIdx.x; j < lcnt; j += gridDim.x) {
        const int c = level_cells[lstart + j];
        const double sx = cv.cx[c], sy = cv.cy[c], sz = cv.cz[c];
        const double il = 1.0 / ell[c];
        int nparts;
        if (cv.leaf[c]) {
            nparts = G;
            const int mc = tid % P1, g = tid / P1;
            cplx<A>* acc = part + g * H;  // this thread's entries hx(n, mc), n >= mc
            if (g < G)
                for (int n = mc; n <= p; ++n) acc[hx(n, mc)] = mk<A>(A(0), A(0));
            const uint32_t f = cv.first[c], cnt = cv.count[c];
            for (uint32_t b0 = 0; b0 < cnt; b0 += UPM_BLOCK) {
                // the chunk's bodies, relative and scaled, loaded by all threads at once
                const uint32_t nb = min((uint32_t)UPM_BLOCK, cnt - b0);
                __syncthreads();
                if ((uint32_t)tid < nb) {
                    const uint32_t q = f + b0 + tid;
                    bod[tid] = (A)((x[q] - sx) * il);
                    bod[UPM_BLOCK + tid] = (A)((y[q] - sy) * il);
                    bod[2 * UPM_BLOCK + tid] = (A)((z[q] - sz) * il);
                    bod[3 * UPM_BLOCK + tid] = (A)m[q];
                }
                __syncthreads();
                if (g >= G) continue;
                for (uint32_t b = g; b < nb; b += G) {
                    const A rx = bod[b], ry = bod[UPM_BLOCK + b], rz = bod[2 * UPM_BLOCK + b];
                    const A mb = bod[3 * UPM_BLOCK + b];
                    const A r2 = rx * rx + ry * ry + rz * rz;
                    cplx<A> d = mk<A>(A(1), A(0));
                    for (int q = 1; q <= mc; ++q) d = zmul(zscale(mk<A>(rx, ry), (A)g_tab.inv2m[q]), d);
                    cplx<A> u1 = d, u2 = mk<A>(A(0), A(0));
                    acc[hx(mc, mc)].re += d.re * mb;
                    acc[hx(mc, mc)].im += d.im * mb;
                    for (int n = mc + 1; n <= p; ++n) {
                        const A a = (A)(2 * n - 1) * rz;
                        const cplx<A> un = zscale(zsub(zscale(u1, a), zscale(u2, r2)), (A)g_tab.invc[n][mc]);
                        u2 = u1;
                        u1 = un;
                        acc[hx(n, mc)].re += un.re * mb;
                        acc[hx(n, mc)].im += un.im * mb;
                    }
                }
            }
        } else {
            nparts = 8;
            for (int w = tid; w < 8 * P1; w += UPM_BLOCK) {
                const int o = w / P1, mc = w % P1;
                const int ch = cv.child[8 * c + o];
                if (ch < 0) continue;
                const A dx = (A)((cv.cx[ch] - sx) * il), dy = (A)((cv.cy[ch] - sy) * il),
                        dz = (A)((cv.cz[ch] - sz) * il);
                ups_column<A>(dx, dy, dz, dx * dx + dy * dy + dz * dz, p, mc, u + o * H);
            }
            for (int w = tid; w < 8 * H; w += UPM_BLOCK) {  // stage the children's moments
                const int o = w / H, e = w % H;
                const int ch = cv.child[8 * c + o];
                if (ch >= 0) cm[w] = mom[(size_t)ch * half_stride(p) + e];
            }
            __syncthreads();
            for (int w = tid; w < 8 * H; w += UPM_BLOCK) {
                const int o = w / H, e = w % H;
                const int ch = cv.child[8 * c + o];
                A sr = 0, si = 0;
                if (ch >= 0) {
                    int n, mm;
                    split_h(e, n, mm);
                    const cplx<A>* uo = u + o * H;
                    const A ratio = (A)(ell[ch] * il);
                    const zf* mcv = cm + o * H;
                    A rpow = 1;  // ratio^{n-k}, built from k = n down
                    for (int k = n; k >= 0; --k) {
                        const int nk = n - k;
                        const int lo = max(-k, mm - nk), hi = min(k, mm + nk);
                        A tr = 0, ti = 0;
                        for (int l = lo; l <= hi; ++l) {
                            const cplx<A> uu = half_get<A>(uo, k, l);
                            const zf mv = half_get<float>(mcv, nk, mm - l);
                            tr += uu.re * (A)mv.re - uu.im * (A)mv.im;
                            ti += uu.re * (A)mv.im + uu.im * (A)mv.re;
                        }
                        sr += tr * rpow;
                        si += ti * rpow;
                        rpow *= ratio;
                    }
                }
                part[o * H + e] = mk<A>(sr, si);
            }
        }
        __syncthreads();
        zf* out = mom + (size_t)c * half_stride(p);
        for (int e = tid; e < H; e += UPM_BLOCK) {
            A sr = 0, si = 0;
            for (int q = 0; q < nparts; ++q) {
                sr += part[q * H + e].re;
                si += part[q * H + e].im;
            }
            out[e] = mk<float>((float)sr, (float)si);
        }
        __syncthreads();
    }
}

template <typename A>
static size_t upward_smem(int H) {
    return (size_t)16 * H * sizeof(cplx<A>) + (size_t)8 * H * sizeof(zf) + (size_t)4 * UPM_BLOCK * sizeof(A);
}

void launch_upward_mixed(bool fp64, unsigned grid, int warps, cudaStream_t s, const int32_t* level_cells,
                         int lstart, int lcnt, CellsView cv, const double* ell, const double* x, const double* y,
                         const double* z, const double* m, int p, zf* mom) {
    (void)warps;
    const int H = (p + 1) * (p + 2) / 2;
    // above 48 KB (FP64 levels from p = 14) the kernel must opt in to more shared memory
    if (fp64) {
        const size_t sm = upward_smem<double>(H);
        if (sm > 48 * 1024)
            cudaFuncSetAttribute(k_upward_mixed<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_upward_mixed<double><<<grid, UPM_BLOCK, sm, s>>>(level_cells, lstart, lcnt, cv, ell, x, y, z, m, p, mom);
    } else {
        const size_t sm = upward_smem<float>(H);
        if (sm > 48 * 1024)
            cudaFuncSetAttribute(k_upward_mixed<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_upward_mixed<float><<<grid, UPM_BLOCK, sm, s>>>(level_cells, lstart, lcnt, cv, ell, x, y, z, m, p, mom);
    }
}

// Υ column m as ups_column computes it, stored in the full layout (entry
// (n, m) at n(n+1) + m for |m| <= n), with v_{n,-m} = (-1)^m conj(v_{n,m}).
template <typename A>
__device__ __forceinline__ void ups_column_full(A x, A y, A z, A r2, int p, int m, cplx<A>* u) {
    auto put = [&](int n, cplx<A> v) {
        u[n * (n + 1) + m] = v;
        if (m) u[n * (n + 1) - m] = (m & 1) ? mk<A>(-v.re, v.im) : mk<A>(v.re, -v.im);
    };
    cplx<A> d = mk<A>(A(1), A(0));
    for (int j = 1; j <= m; ++j) d = zmul(zscale(mk<A>(x, y), (A)g_tab.inv2m[j]), d);
    put(m, d);
    cplx<A> u1 = d, u2 = mk<A>(A(0), A(0));
    for (int n = m + 1; n <= p; ++n) {
        const A a = (A)(2 * n - 1) * z;
        const cplx<A> un = zscale(zsub(zscale(u1, a), zscale(u2, r2)), (A)g_tab.invc[n][m]);
        put(n, un);
        u2 = u1;
        u1 = un;
    }
}

// L2L for the cells of one level (L >= 1), one warp per cell; A as above.
//
// Output (n, m) of the child's locals is ratio^{n+1} sum_{k <= p-n, |l| <= k}
// conj(Υ_{k,l}(r)) L_{n+k, m+l} of the parent: (p-n+1)^2 products, 121 for
// the monopole and 1 for degree p at p = 10. A thread per output leaves most
// lanes idle behind the low degrees, so the products of all outputs are laid
// out as one list ("items": output by output, k then l) of
// T = q (q+1)^2 (q+2) / 12 entries (q = p + 1; 1,716 at p = 10) and every lane
// takes an equal contiguous run of it. An output that lies inside one lane's
// run is finished there; one that crosses runs leaves a partial sum in each
// (slot 0: the output the run starts in, slot 1: the one it ends in), added
// afterwards, in lane order, by the lane holding its first product -- a fixed
// order, so the result bits do not depend on scheduling. The list is built
// by every block at its start (item: Υ index, parent index, output, and a
// last-product flag); Υ and the parent's locals sit in shared memory in the
// full layout (both signs of m), so a product is two loads and four FMAs.
#define L2LB_WARPS 4

__host__ __device__ constexpr int l2l_items(int p) {
    return (p + 1) * (p + 2) * (p + 2) * (p + 3) / 12;
}

template <typename A>
static size_t l2l_smem(int p) {
    const int P1 = p + 1, H = P1 * (P1 + 1) / 2, F2 = P1 * P1;
    return (size_t)L2LB_WARPS * (F2 + 64 + H) * sizeof(cplx<A>) + (size_t)L2LB_WARPS * F2 * sizeof(zf) +
           (size_t)(H + 1 + l2l_items(p)) * sizeof(uint32_t);
}

template <typename A>
__global__ void __launch_bounds__(L2LB_WARPS * 32) k_l2l_mixed(const int32_t* __restrict__ level_cells, int lstart,
                                                              int lcnt, CellsView cv,
                                                              const int32_t* __restrict__ parent,
                                                              const double* __restrict__ ell, int p,
                                                              zf* __restrict__ loc) {
    extern __shared__ __align__(16) unsigned char lsm[];
    const int P1 = p + 1, H = P1 * (P1 + 1) / 2, F2 = P1 * P1, T = l2l_items(p);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    cplx<A>* U = reinterpret_cast<cplx<A>*>(lsm) + wid * F2;                      // Υ(r), full layout
    cplx<A>* Pp = reinterpret_cast<cplx<A>*>(lsm) + L2LB_WARPS * F2 + wid * 64;  // [lane][2] partials
    cplx<A>* R = reinterpret_cast<cplx<A>*>(lsm) + L2LB_WARPS * (F2 + 64) + wid * H;  // sums per output
    zf* F = reinterpret_cast<zf*>(reinterpret_cast<cplx<A>*>(lsm) + L2LB_WARPS * (F2 + 64 + H)) + wid * F2;
    uint32_t* einfo = reinterpret_cast<uint32_t*>(reinterpret_cast<zf*>(reinterpret_cast<cplx<A>*>(lsm) +
                                                                        L2LB_WARPS * (F2 + 64 + H)) +
                                                  L2LB_WARPS * F2);  // first item | n << 16
    uint32_t* items = einfo + H + 1;

    for (int e = threadIdx.x; e < H; e += blockDim.x) {
        int n, m;
        split_h(e, n, m);
        int s = 0;
        for (int q = 0; q < n; ++q) s += (q + 1) * (p - q + 1) * (p - q + 1);
        const int w = p - n + 1;
        s += m * w * w;
        einfo[e] = (uint32_t)s | ((uint32_t)n << 16);
        for (int k = 0; k <= p - n; ++k)
            for (int l = -k; l <= k; ++l, ++s)
                items[s] = (uint32_t)(k * (k + 1) + l) | ((uint32_t)((n + k) * (n + k + 1) + m + l) << 9) |
                           ((uint32_t)e << 18) | (k == p - n && l == k ? 0x80000000u : 0u);
    }
    if (threadIdx.x == 0) einfo[H] = (uint32_t)T;
    __syncthreads();

    const int W = ((T + 31) / 32) | 1;  // an odd stride keeps the lanes' item reads on distinct banks
    const int r0 = min(T, lane * W), r1 = min(T, r0 + W);
    for (int j = blockIdx.x * L2LB_WARPS + wid; j < lcnt; j += gridDim.x * L2LB_WARPS) {
        const int c = level_cells[lstart + j];
        const int par = parent[c];
        if (par < 0) continue;
        const double il = 1.0 / ell[par];
        const A rx = (A)((cv.cx[par] - cv.cx[c]) * il), ry = (A)((cv.cy[par] - cv.cy[c]) * il),
                rz = (A)((cv.cz[par] - cv.cz[c]) * il);
        if (lane <= p) ups_column_full<A>(rx, ry, rz, rx * rx + ry * ry + rz * rz, p, lane, U);
        const zf* lp = loc + (size_t)par * half_stride(p);
        for (int e = lane; e < H; e += 32) {
            const int n = (int)(einfo[e] >> 16), m = e - n * (n + 1) / 2;
            const zf v = lp[e];
            F[n * (n + 1) + m] = v;
            if (m) F[n * (n + 1) - m] = (m & 1) ? mk<float>(-v.re, v.im) : mk<float>(v.re, -v.im);
        }
        __syncwarp();
        A sr = 0, si = 0;
        uint32_t it = 0;
        for (int i = r0; i < r1; ++i) {
            it = items[i];
            const cplx<A> a = U[it & 511u];
            const zf b = F[(it >> 9) & 511u];
            sr += a.re * (A)b.re + a.im * (A)b.im;  // conj(a) * b
            si += a.re * (A)b.im - a.im * (A)b.re;
            if (it & 0x80000000u) {
                const int e = (int)((it >> 18) & 255u);
                if ((int)(einfo[e] & 0xffffu) >= r0) R[e] = mk<A>(sr, si);  // the whole output is in this run
                else Pp[2 * lane] = mk<A>(sr, si);                          // it started in an earlier run
                sr = 0;
                si = 0;
            }
        }
        if (r1 > r0 && !(it & 0x80000000u)) {  // the run ends inside an output
            const int e = (int)((it >> 18) & 255u);
            Pp[2 * lane + ((int)(einfo[e] & 0xffffu) <= r0 ? 0 : 1)] = mk<A>(sr, si);
        }
        __syncwarp();
        if (r1 > r0) {
            const int e = (int)((items[r1 - 1] >> 18) & 255u);
            const int s0 = (int)(einfo[e] & 0xffffu), s1 = (int)(einfo[e + 1] & 0xffffu);
            if (s0 >= r0 && s1 > r1) {  // an output that starts in this run and crosses into the next ones
                cplx<A> acc = Pp[2 * lane + (s0 == r0 ? 0 : 1)];
                for (int q = lane + 1; q * W < s1; ++q) {
                    acc.re += Pp[2 * q].re;
                    acc.im += Pp[2 * q].im;
                }
                R[e] = acc;
            }
        }
        __syncwarp();
        const A ratio = (A)(ell[c] * il);
        zf* lc = loc + (size_t)c * half_stride(p);
        for (int e = lane; e < H; e += 32) {
            const int n = (int)(einfo[e] >> 16);
            A sc = ratio;
            for (int q = 0; q < n; ++q) sc *= ratio;
            const zf cur = lc[e];
            const cplx<A> v = R[e];
            lc[e] = mk<float>((float)((A)cur.re + v.re * sc), (float)((A)cur.im + v.im * sc));
        }
        __syncwarp();
    }
}

void launch_l2l_mixed(bool fp64, unsigned grid, cudaStream_t s, const int32_t* level_cells, int lstart, int lcnt,
                      CellsView cv, const int32_t* parent, const double* ell, int p, zf* loc) {
    const unsigned blocks = std::max(1u, std::min(grid, (unsigned)((lcnt + L2LB_WARPS - 1) / L2LB_WARPS)));
    if (fp64) {
        const size_t sm = l2l_smem<double>(p);
        if (sm > 48 * 1024)
            cudaFuncSetAttribute(k_l2l_mixed<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_l2l_mixed<double><<<blocks, L2LB_WARPS * 32, sm, s>>>(level_cells, lstart, lcnt, cv, parent, ell, p, loc);
    } else {
        const size_t sm = l2l_smem<float>(p);
        if (sm > 48 * 1024)
            cudaFuncSetAttribute(k_l2l_mixed<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_l2l_mixed<float><<<blocks, L2LB_WARPS * 32, sm, s>>>(level_cells, lstart, lcnt, cv, parent, ell, p, loc);
    }
}

// L2P at every body plus the near field, scattered to particle-id order.
__global__ void k_l2p_mixed(size_t n, const int32_t* __restrict__ body_leaf, const uint32_t* __restrict__ order,
                            CellsView cv, const double* __restrict__ ell, int p, const zf* __restrict__ loc,
                            const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const double* __restrict__ nax,
                            const double* __restrict__ nay, const double* __restrict__ naz,
                            const double* __restrict__ npot, double* __restrict__ acc, double* __restrict__ pot) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int c = body_leaf[k];
        const double l = ell[c], il = 1.0 / l;
        const float rx = (float)((cv.cx[c] - x[k]) * il), ry = (float)((cv.cy[c] - y[k]) * il),
                    rz = (float)((cv.cz[c] - z[k]) * il);
        const float r2 = rx * rx + ry * ry + rz * rz;
        const zf* L = loc + (size_t)c * half_stride(p);
        float p00 = 0, p11r = 0, p11i = 0, p10 = 0;
        zf d = mk<float>(1.f, 0.f);
        for (int lm = 0; lm <= p; ++lm) {
            if (lm > 0) d = zmul(zscale(mk<float>(rx, ry), (float)g_tab.inv2m[lm]), d);
            zf u1 = d, u2 = mk<float>(0.f, 0.f);
            const float sgn = (lm & 1) ? -1.f : 1.f;
            for (int kk = lm; kk <= p; ++kk) {
                zf uk;
                if (kk == lm) {
                    uk = d;
                } else {
                    const float a = (float)(2 * kk - 1) * rz;
                    uk = zscale(zsub(zscale(u1, a), zscale(u2, r2)), (float)g_tab.invc[kk][lm]);
                    u2 = u1;
                    u1 = uk;
                }
                const zf f0 = L[hx(kk, lm)];
                p00 += uk.re * f0.re + uk.im * f0.im;
                if (kk < p) {
                    const zf f11 = half_get<float>(L, kk + 1, lm + 1);
                    const zf f10 = L[hx(kk + 1, lm)];
                    p11r += uk.re * f11.re + uk.im * f11.im;
                    p11i += uk.re * f11.im - uk.im * f11.re;
                    p10 += uk.re * f10.re + uk.im * f10.im;
                }
                if (lm > 0) {
                    const zf g0 = half_get<float>(L, kk, -lm);
                    p00 += sgn * (uk.re * g0.re - uk.im * g0.im);
                    if (kk < p) {
                        const zf g11 = half_get<float>(L, kk + 1, 1 - lm);
                        const zf g10 = half_get<float>(L, kk + 1, -lm);
                        p11r += sgn * (uk.re * g11.re - uk.im * g11.im);
                        p11i += sgn * (uk.re * g11.im + uk.im * g11.re);
                        p10 += sgn * (uk.re * g10.re - uk.im * g10.im);
                    }
                }
            }
        }
        const uint32_t id = order[k];
        acc[3 * (size_t)id + 0] = nax[k] - ((double)p11r * il) * il;
        acc[3 * (size_t)id + 1] = nay[k] - ((double)p11i * il) * il;
        acc[3 * (size_t)id + 2] = naz[k] - ((double)p10 * il) * il;
        pot[id] = npot[k] + (double)p00 * il;
    }
}

// ------------------------------------------------------------------ P2P
// FP32 P2P with compensated accumulation. Source bodies are staged in shared
// memory relative to the target leaf's centre (the FP64 subtraction), so the
// FP32 differences d = x_j - x_i keep their relative precision; each thread
// sums at least P2PM_FLUSH source pairs (two partial sums per component) in
// FP32 and adds them into a double-single (hi, lo) accumulator with an
// error-free TwoSum. 1/r by the hardware rsqrt.
#define P2PM_BLOCK 128
#define P2PM_SRC_CHUNK 256

struct DS {
    float hi, lo;
};
__device__ __forceinline__ void ds_add(DS& a, float b) {
    const float s = a.hi + b;
    const float bb = s - a.hi;
    const float err = (a.hi - (s - bb)) + (b - bb);
    a.hi = s;
    a.lo += err;
}

// The hardware reciprocal square root (about 2^-22 relative error), flushing
// subnormal inputs: r2 is a squared distance plus the squared softening, far
// above the subnormal range whenever it is positive. No Newton step: its
// error is of the order of the FP32 rounding of the per-tile partial sums,
// which dominates the near-field error. Measured at N = 2^20 (uniform cube,
// p = 10, theta 0.5, 4096 targets against the FP64 direct sum): p99 relative
// force error 1.3787e-6 with a Newton step, 1.3773e-6 without, P2P 2.96 ->
// 2.58 ms; theta 0.3, p = 12: 6.42e-7 and 6.49e-7, 12.64 -> 10.98 ms.
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// One source body against one target, FP32, d relative to the target leaf's
// centre.
__device__ __forceinline__ void p2p_term(const float4 s, float xi, float yi, float zi, float soft2, float& ax,
                                         float& ay, float& az, float& pt) {
    const float dx = s.x - xi, dy = s.y - yi, dz = s.z - zi;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, soft2)));
    const float inv = rsqrt_approx(r2);
    const float mi = s.w * inv;
    const float f = mi * inv * inv;
    ax = fmaf(f, dx, ax);
    ay = fmaf(f, dy, ay);
    az = fmaf(f, dz, az);
    pt += mi;
}

// Work units of the near field: the sources of leaf c are cut into units of
// P2P_UNIT_SRC source leaves, units[c] = ceil(len / P2P_UNIT_SRC), so a leaf
// in a dense cluster core with thousands of neighbours spreads over many
// blocks instead of holding one block to the end of the launch (the
// load-balancing aim of the reference's split_fat, crates/visual/src/
// gpufmm.rs:1350-1414). A leaf with one unit writes its bodies' sums
// directly; the units of a leaf with several write partial sums, which
// k_p2p_combine adds per body in unit order (a fixed order: the results do
// not depend on which block ran which unit).
__global__ void k_p2p_plan(int ncells, DirList L, const uint32_t* __restrict__ count, uint32_t* __restrict__ units,
                           uint32_t* __restrict__ units_s, uint32_t* __restrict__ units_b,
                           uint32_t* __restrict__ scratch) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= ncells; c += gridDim.x * blockDim.x) {
        uint32_t nu = 0;
        bool small = false;
        if (c < ncells) {
            const uint32_t len = L.seg_end[c] - L.seg_begin[c];
            nu = (len + P2P_UNIT_SRC - 1) / P2P_UNIT_SRC;
            small = count[c] <= P2P_SMALL_NT;
        }
        units[c] = nu;
        units_s[c] = small ? nu : 0;
        units_b[c] = small ? 0 : nu;
        scratch[c] = nu > 1 ? nu * count[c] : 0;
    }
}

__device__ __forceinline__ int unit_cell(const uint32_t* __restrict__ uoff, int ncells, uint32_t u) {
    int lo = 0, hi = ncells;  // the last c with uoff[c] <= u
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (uoff[mid] <= u) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Body coordinates relative to their own leaf's centre, FP32, with the mass:
// computed once per evaluation (the FP64 subtraction), so that staging a
// source body for the near field is one 16-byte load plus its leaf's offset
// from the target leaf's centre (c_s - c_t, FP64 rounded to FP32 once per
// source leaf). The difference d = x_j - x_i then carries three FP32
// roundings of quantities no larger than the pair's leaf separation instead
// of one: the same order of absolute error.
__global__ void k_local_coords(size_t n, const int32_t* __restrict__ body_leaf, CellsView cv,
                               const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, const double* __restrict__ m,
                               float4* __restrict__ loc) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int c = body_leaf[k];
        loc[k] = make_float4((float)(x[k] - cv.cx[c]), (float)(y[k] - cv.cy[c]), (float)(z[k] - cv.cz[c]),
                             (float)m[k]);
    }
}

// One pair of source bodies (j, j+1) against one target, on packed FP32x2
// arithmetic (sm_100's two-wide FP32 instructions: one issue slot for two
// lanes of work): -x is the target's coordinate negated in both halves.
// The pair's two partial sums stay apart in the two halves of each
// accumulator until the tile ends.
__device__ __forceinline__ void p2p_pair(const float4 a, const float4 b, float2 nx, float2 ny, float2 nz,
                                         float2 soft2, float2& ax, float2& ay, float2& az, float2& pt) {
    const float2 dx = __fadd2_rn(make_float2(a.x, a.y), nx);
    const float2 dy = __fadd2_rn(make_float2(a.z, a.w), ny);
    const float2 dz = __fadd2_rn(make_float2(b.x, b.y), nz);
    float2 r2 = __ffma2_rn(dz, dz, soft2);
    r2 = __ffma2_rn(dy, dy, r2);
    r2 = __ffma2_rn(dx, dx, r2);
    const float2 inv = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
    const float2 mi = __fmul2_rn(make_float2(b.z, b.w), inv);
    const float2 f = __fmul2_rn(mi, __fmul2_rn(inv, inv));
    ax = __ffma2_rn(f, dx, ax);
    ay = __ffma2_rn(f, dy, ay);
    az = __ffma2_rn(f, dz, az);
    pt = __fadd2_rn(pt, mi);
}

// The pair with the target's own body at half h (0 or 1) of it: that half
// becomes a massless body one unit away (no term).
__device__ __forceinline__ void mask_self(float4& a, float4& b, int h, float x, float y, float z) {
    if (h == 0) {
        a.x = x + 1.f; a.z = y; b.x = z; b.z = 0.f;
    } else {
        a.y = x + 1.f; a.w = y; b.y = z; b.w = 0.f;
    }
}

// TILE: source bodies staged per shared-memory tile (the tile shape the
// autotuner picks), as pairs: ta[q] = (x_2q, x_2q+1, y_2q, y_2q+1),
// tz[q] = (z_2q, z_2q+1, m_2q, m_2q+1), an odd tile padded with a massless
// body far away. Each thread carries two targets, so every staged pair feeds
// four interactions; groups of G threads cover the leaf's targets and
// R = BLOCK / G groups split each tile's pairs. The target's own body is
// masked only in the tiles that overlap the target leaf itself. Blocks are
// persistent and take units from a counter.
//
// The sources are taken in chunks of at most P2PM_SRC_CHUNK source leaves and
// P2PM_MAP bodies: a chunk's bodies are numbered consecutively and own[]
// gives each body's leaf in the chunk, so staging a body is a table lookup
// (a leaf of more than P2PM_MAP bodies is a chunk of its own, without the
// table). A target chunk's sums over the R groups are reduced by all threads,
// S threads per output in fixed strips and a fixed shuffle tree.
#define P2PM_MAP 4096
#define P2PM_FLUSH 16

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Start copying the bodies of the tile [b0, b0 + nb) of a chunk to raw[]:
// thread tid takes pairs tid, tid + BLOCK, ...; lq[] keeps each body's leaf
// in the chunk (-1: padding past the tile's end).
template <int PPT>
__device__ __forceinline__ void stage_issue(uint32_t b0, uint32_t nb, int tid, bool mapped,
                                            const uint8_t* own, const uint32_t* sbase,
                                            const float4* __restrict__ loc, float4* raw, int* lq) {
    const int npair = (int)(nb + 1) >> 1;
#pragma unroll
    for (int e = 0; e < PPT; ++e) {
        const int q = tid + e * P2PM_BLOCK;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t gg = b0 + 2u * (uint32_t)q + (uint32_t)h;
            lq[2 * e + h] = -1;
            if (q < npair && gg < b0 + nb) {
                const int l = mapped ? (int)own[gg] : 0;
                lq[2 * e + h] = l;
                cp_async16(raw + 2 * q + h, loc + (gg + sbase[l]));
            }
        }
    }
    cp_async_commit();
}

// Finish the bodies this thread copied: wait for its copies, add the leaf
// offsets and write the pair layout.
template <int PPT>
__device__ __forceinline__ void stage_finish(int npair, int tid, const float4* raw, const float4* soff,
                                             const int* lq, float4* ta, float4* tz) {
    cp_async_wait_all();
#pragma unroll
    for (int e = 0; e < PPT; ++e) {
        const int q = tid + e * P2PM_BLOCK;
        if (q < npair) {
            float4 s2[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int l = lq[2 * e + h];
                if (l >= 0) {
                    const float4 v = raw[2 * q + h];
                    const float4 o = soff[l];
                    s2[h] = make_float4(v.x + o.x, v.y + o.y, v.z + o.z, v.w);
                } else {
                    s2[h] = make_float4(1e18f, 0.f, 0.f, 0.f);  // massless padding
                }
            }
            ta[q] = make_float4(s2[0].x, s2[1].x, s2[0].y, s2[1].y);
            tz[q] = make_float4(s2[0].z, s2[1].z, s2[0].w, s2[1].w);
        }
    }
}
template <int P2PM_TILE>
__global__ void __launch_bounds__(P2PM_BLOCK, 5) k_p2p_mixed(DirList L, int ncells, CellsView cv, P2pUnits U,
                                                         const float4* __restrict__ loc, float soft2_1,
                                                         double* __restrict__ ax, double* __restrict__ ay,
                                                         double* __restrict__ az, double* __restrict__ pot) {
    constexpr int NPAIR = P2PM_TILE / 2;
    constexpr int PPT = (NPAIR + P2PM_BLOCK - 1) / P2PM_BLOCK;  // pairs staged per thread
    __shared__ float4 ta[NPAIR];
    __shared__ float4 tz[NPAIR];
    // the next tile's bodies as copied (leaf-relative); also the per-group
    // sums at the end of a target chunk, when no copy is in flight
    __shared__ float4 raw[P2PM_TILE > 512 ? P2PM_TILE : 512];
    float(*red)[P2PM_BLOCK] = reinterpret_cast<float(*)[P2PM_BLOCK]>(raw);
    static_assert(sizeof(raw) >= 16 * P2PM_BLOCK * sizeof(float), "the group sums alias the copy buffer");
    __shared__ uint32_t pre[P2PM_SRC_CHUNK + 1];
    __shared__ uint32_t sbase[P2PM_SRC_CHUNK];  // first slot of the leaf - its first position in the chunk
    __shared__ float4 soff[P2PM_SRC_CHUNK];     // source leaf centre - target leaf centre
    __shared__ uint8_t own[P2PM_MAP];
    __shared__ uint32_t wsum[P2PM_BLOCK / 32];
    __shared__ int self_pos, nuse_sh;
    __shared__ uint32_t unit_sh;
    const int tid = threadIdx.x;
    const int lane = tid & 31, wid = tid >> 5;
    const uint32_t nunits = U.uoff_b[ncells];
    const float2 soft2 = make_float2(soft2_1, soft2_1);
    for (;;) {
        if (tid == 0) unit_sh = atomicAdd(U.next + 1, 1u);
        __syncthreads();
        const uint32_t u = unit_sh;
        __syncthreads();
        if (u >= nunits) break;
        const int c = unit_cell(U.uoff_b, ncells, u);
        const uint32_t k = u - U.uoff_b[c], nu = U.uoff[c + 1] - U.uoff[c];
        const uint32_t beg = L.seg_begin[c] + k * P2P_UNIT_SRC;
        const uint32_t end = min(L.seg_end[c], beg + P2P_UNIT_SRC);
        const double cx = cv.cx[c], cy = cv.cy[c], cz = cv.cz[c];
        const uint32_t tf = cv.first[c], tn = cv.count[c];
        for (uint32_t t0 = 0; t0 < tn; t0 += 2 * P2PM_BLOCK) {
            const int nt = (int)min((uint32_t)(2 * P2PM_BLOCK), tn - t0);
            const int G = (nt + 1) >> 1;
            const int R = P2PM_BLOCK / G;
            const int g = tid % G, rep = tid / G;
            const bool active = rep < R;
            const int i0 = g, i1 = g + G;
            const bool has1 = active && i1 < nt;
            float x0 = 0, y0 = 0, z0 = 0, x1 = 0, y1 = 0, z1 = 0;
            if (active) {
                const float4 v = loc[tf + t0 + i0];
                x0 = v.x; y0 = v.y; z0 = v.z;
            }
            if (has1) {
                const float4 v = loc[tf + t0 + i1];
                x1 = v.x; y1 = v.y; z1 = v.z;
            }
            const float2 nx0 = make_float2(-x0, -x0), ny0 = make_float2(-y0, -y0), nz0 = make_float2(-z0, -z0);
            const float2 nx1 = make_float2(-x1, -x1), ny1 = make_float2(-y1, -y1), nz1 = make_float2(-z1, -z1);
            DS a0x{0, 0}, a0y{0, 0}, a0z{0, 0}, p0{0, 0}, a1x{0, 0}, a1y{0, 0}, a1z{0, 0}, p1{0, 0};
            // FP32 partial sums, added into the double-single sums once they
            // hold P2PM_FLUSH source pairs (and at the end)
            float2 q0x{0, 0}, q0y{0, 0}, q0z{0, 0}, q0p{0, 0}, q1x{0, 0}, q1y{0, 0}, q1z{0, 0}, q1p{0, 0};
            int held = 0;
            auto flush = [&]() {
                ds_add(a0x, q0x.x + q0x.y);
                ds_add(a0y, q0y.x + q0y.y);
                ds_add(a0z, q0z.x + q0z.y);
                ds_add(p0, q0p.x + q0p.y);
                ds_add(a1x, q1x.x + q1x.y);
                ds_add(a1y, q1y.x + q1y.y);
                ds_add(a1z, q1z.x + q1z.y);
                ds_add(p1, q1p.x + q1p.y);
                q0x = q0y = q0z = q0p = q1x = q1y = q1z = q1p = make_float2(0.f, 0.f);
                held = 0;
            };
            for (uint32_t sc = beg; sc < end;) {
                const int ns = (int)min((uint32_t)P2PM_SRC_CHUNK, end - sc);
                __syncthreads();
                if (tid == 0) self_pos = -1;
                // exclusive prefix of source leaf sizes (warp scans, then warp totals)
                int myq[2] = {-1, -1};
                for (int q0 = 0, h = 0; q0 < ns; q0 += P2PM_BLOCK, ++h) {
                    const int q = q0 + tid;
                    uint32_t v = 0;
                    int src = -1;
                    if (q < ns) {
                        src = (int)L.src(L.key(sc + q));
                        v = cv.count[src];
                        soff[q] = make_float4((float)(cv.cx[src] - cx), (float)(cv.cy[src] - cy),
                                              (float)(cv.cz[src] - cz), 0.f);
                        myq[h] = src;
                    }
                    uint32_t incl = v;
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane >= o) incl += t;
                    }
                    if (lane == 31) wsum[wid] = incl;
                    __syncthreads();
                    uint32_t base = q0 == 0 ? 0 : pre[q0];
                    for (int w = 0; w < wid; ++w) base += wsum[w];
                    if (q < ns) {
                        pre[q + 1] = base + incl;
                        sbase[q] = cv.first[src] - (base + incl - v);
                    }
                    if (q0 == 0 && tid == 0) pre[0] = 0;
                    __syncthreads();
                }
                // the leaves whose bodies fit in the table (at least one)
                int fit = 0;
                for (int q = tid; q < ns; q += P2PM_BLOCK) fit += pre[q + 1] <= P2PM_MAP ? 1 : 0;
                if (tid == 0) nuse_sh = 0;
                __syncthreads();
                if (fit) atomicAdd(&nuse_sh, fit);
                __syncthreads();
                const int nl = max(1, nuse_sh);
                const bool mapped = pre[nl] <= P2PM_MAP;
                for (int h = 0; h < 2; ++h) {
                    const int q = tid + h * P2PM_BLOCK;
                    if (q < nl) {
                        if (myq[h] == c) self_pos = (int)pre[q];
                        if (mapped)
                            for (uint32_t e = pre[q]; e < pre[q + 1]; ++e) own[e] = (uint8_t)q;
                    }
                }
                __syncthreads();
                const uint32_t total = pre[nl];
                const int sp = self_pos;  // position of the target leaf in this chunk's sources, or -1
                sc += nl;
                // tile k + 1's bodies are copied to raw[] (cp.async) while tile k
                // is computed; each thread later finishes the bodies it copied
                // (its leaf's offset added, pair layout), so only the tile
                // hand-over needs a block barrier
                int lq_cur[2 * PPT], lq_nxt[2 * PPT];
                stage_issue<PPT>(0, min((uint32_t)P2PM_TILE, total), tid, mapped, own, sbase, loc, raw, lq_cur);
                for (uint32_t b0 = 0; b0 < total; b0 += P2PM_TILE) {
                    const uint32_t nb = min((uint32_t)P2PM_TILE, total - b0);
                    const int npair = (int)(nb + 1) >> 1;
                    stage_finish<PPT>(npair, tid, raw, soff, lq_cur, ta, tz);
                    __syncthreads();
                    if (b0 + P2PM_TILE < total)
                        stage_issue<PPT>(b0 + P2PM_TILE, min((uint32_t)P2PM_TILE, total - b0 - P2PM_TILE), tid,
                                         mapped, own, sbase, loc, raw, lq_nxt);
                    if (active) {
                        const bool overlaps = sp >= 0 && (uint32_t)sp < b0 + nb && (uint32_t)sp + tn > b0;
                        if (!overlaps) {
#pragma unroll 2
                            for (int j = rep; j < npair; j += R) {
                                const float4 a = ta[j], b = tz[j];
                                p2p_pair(a, b, nx0, ny0, nz0, soft2, q0x, q0y, q0z, q0p);
                                p2p_pair(a, b, nx1, ny1, nz1, soft2, q1x, q1y, q1z, q1p);
                            }
                        } else {
                            // the target's own body sits at position sp + t0 + i in the sources
                            const int s0 = sp + (int)t0 + i0 - (int)b0, s1 = sp + (int)t0 + i1 - (int)b0;
                            for (int j = rep; j < npair; j += R) {
                                const float4 a = ta[j], b = tz[j];
                                float4 a0 = a, b0v = b, a1 = a, b1v = b;
                                if (s0 >= 0 && j == (s0 >> 1)) mask_self(a0, b0v, s0 & 1, x0, y0, z0);
                                if (s1 >= 0 && j == (s1 >> 1)) mask_self(a1, b1v, s1 & 1, x1, y1, z1);
                                p2p_pair(a0, b0v, nx0, ny0, nz0, soft2, q0x, q0y, q0z, q0p);
                                p2p_pair(a1, b1v, nx1, ny1, nz1, soft2, q1x, q1y, q1z, q1p);
                            }
                        }
                        held += (npair - rep + R - 1) / R;
                        if (held >= P2PM_FLUSH) flush();
                    }
                    __syncthreads();
#pragma unroll
                    for (int e = 0; e < 2 * PPT; ++e) lq_cur[e] = lq_nxt[e];
                }
            }
            flush();
            red[0][tid] = a0x.hi; red[1][tid] = a0x.lo; red[2][tid] = a0y.hi; red[3][tid] = a0y.lo;
            red[4][tid] = a0z.hi; red[5][tid] = a0z.lo; red[6][tid] = p0.hi; red[7][tid] = p0.lo;
            red[8][tid] = a1x.hi; red[9][tid] = a1x.lo; red[10][tid] = a1y.hi; red[11][tid] = a1y.lo;
            red[12][tid] = a1z.hi; red[13][tid] = a1z.lo; red[14][tid] = p1.hi; red[15][tid] = p1.lo;
            __syncthreads();
            // outputs: nt targets x 4 components; S threads per output (a power
            // of two up to 32, so an output's threads share a warp)
            const int nout = 4 * nt;
            int S = 1;
            while (S < 32 && 2 * S * nout <= P2PM_BLOCK) S <<= 1;
            for (int o0 = 0; o0 < nout; o0 += P2PM_BLOCK / S) {
                const int o = o0 + tid / S, st = tid % S;
                double v = 0.0;
                if (o < nout) {
                    const int t = o >> 2, comp = o & 3;
                    const int gi = t % G, half = t / G;  // target t = gi + half * G
                    const int row = 8 * half + 2 * comp;
                    for (int r = st; r < R; r += S) {
                        const int q = r * G + gi;
                        v += (double)red[row][q] + (double)red[row + 1][q];
                    }
                }
                for (int w = S >> 1; w > 0; w >>= 1) v += __shfl_down_sync(0xffffffffu, v, w, S);
                if (o < nout && st == 0) {
                    const int t = o >> 2, comp = o & 3;
                    if (nu == 1) {
                        double* out = comp == 0 ? ax : comp == 1 ? ay : comp == 2 ? az : pot;
                        out[tf + t0 + t] = v;
                    } else {
                        reinterpret_cast<double*>(U.part + U.soff[c] + k * tn + t0 + t)[comp] = v;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Small target leaves (at most P2P_SMALL_NT bodies): a warp per work unit,
// four independent warps per block, warp-synchronous (no block barriers).
// With a few targets per leaf, a block per unit spends most of its
// instructions on what every thread repeats per tile and per unit (the loop
// setup, the barriers, the group reduction, finding the unit's leaf); a warp
// pays them over a quarter of the threads. Same arithmetic as the block
// kernel: two targets per lane, groups of G = ceil(nt / 2) lanes, R = 32 / G
// groups over each tile's source pairs, packed FP32x2 interactions,
// double-single sums, the leaf table for staging (chunks of at most
// P2PW_CHUNK leaves and P2PW_MAP bodies), the target's own body masked.
#define P2PW_TILE 128
#define P2PW_CHUNK 128
#define P2PW_MAP 2048
#define P2PW_WARPS 4
struct P2pWarpSmem {
    float4 ta[P2PW_TILE / 2];
    float4 tz[P2PW_TILE / 2];
    float4 soff[P2PW_CHUNK];
    uint32_t pre[P2PW_CHUNK + 1];
    uint32_t sbase[P2PW_CHUNK];
    float red[16][32];
    uint8_t own[P2PW_MAP];
};

__global__ void __launch_bounds__(32 * P2PW_WARPS) k_p2p_mixed_small(DirList L, int ncells, CellsView cv, P2pUnits U,
                                                                     const float4* __restrict__ loc, float soft2_1,
                                                                     double* __restrict__ ax, double* __restrict__ ay,
                                                                     double* __restrict__ az,
                                                                     double* __restrict__ pot) {
    __shared__ P2pWarpSmem smem_w[P2PW_WARPS];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    P2pWarpSmem& S = smem_w[threadIdx.x >> 5];
    const uint32_t nunits = U.uoff_s[ncells];
    const float2 soft2 = make_float2(soft2_1, soft2_1);
    for (;;) {
        uint32_t u = 0;
        if (lane == 0) u = atomicAdd(U.next, 1u);
        u = __shfl_sync(FULL, u, 0);
        if (u >= nunits) break;
        const int c = unit_cell(U.uoff_s, ncells, u);
        const uint32_t k = u - U.uoff_s[c], nu = U.uoff[c + 1] - U.uoff[c];
        const uint32_t beg = L.seg_begin[c] + k * P2P_UNIT_SRC;
        const uint32_t end = min(L.seg_end[c], beg + P2P_UNIT_SRC);
        const double cx = cv.cx[c], cy = cv.cy[c], cz = cv.cz[c];
        const uint32_t tf = cv.first[c];
        const int nt = (int)cv.count[c];  // <= P2P_SMALL_NT (32) by the plan
        const int G = (nt + 1) >> 1;
        const int R = 32 / G;
        const int g = lane % G, rep = lane / G;
        const bool active = rep < R;
        const int i0 = g, i1 = g + G;
        const bool has1 = active && i1 < nt;
        float x0 = 0, y0 = 0, z0 = 0, x1 = 0, y1 = 0, z1 = 0;
        if (active) {
            const float4 v = loc[tf + i0];
            x0 = v.x; y0 = v.y; z0 = v.z;
        }
        if (has1) {
            const float4 v = loc[tf + i1];
            x1 = v.x; y1 = v.y; z1 = v.z;
        }
        const float2 nx0 = make_float2(-x0, -x0), ny0 = make_float2(-y0, -y0), nz0 = make_float2(-z0, -z0);
        const float2 nx1 = make_float2(-x1, -x1), ny1 = make_float2(-y1, -y1), nz1 = make_float2(-z1, -z1);
        DS a0x{0, 0}, a0y{0, 0}, a0z{0, 0}, p0{0, 0}, a1x{0, 0}, a1y{0, 0}, a1z{0, 0}, p1{0, 0};
        float2 q0x{0, 0}, q0y{0, 0}, q0z{0, 0}, q0p{0, 0}, q1x{0, 0}, q1y{0, 0}, q1z{0, 0}, q1p{0, 0};
        int held = 0;
        auto flush = [&]() {
            ds_add(a0x, q0x.x + q0x.y);
            ds_add(a0y, q0y.x + q0y.y);
            ds_add(a0z, q0z.x + q0z.y);
            ds_add(p0, q0p.x + q0p.y);
            ds_add(a1x, q1x.x + q1x.y);
            ds_add(a1y, q1y.x + q1y.y);
            ds_add(a1z, q1z.x + q1z.y);
            ds_add(p1, q1p.x + q1p.y);
            q0x = q0y = q0z = q0p = q1x = q1y = q1z = q1p = make_float2(0.f, 0.f);
            held = 0;
        };
        for (uint32_t sc = beg; sc < end;) {
            const int ns = (int)min((uint32_t)P2PW_CHUNK, end - sc);
            __syncwarp();
            // exclusive prefix of the chunk's source leaf sizes (one warp scan
            // per 32 leaves, carried over); each lane remembers where the
            // target leaf itself lies, if it holds it
            uint32_t base = 0;
            int self_q = P2PW_CHUNK, self_at = -1;
            for (int q0 = 0; q0 < ns; q0 += 32) {
                const int q = q0 + lane;
                uint32_t v = 0;
                int src = -1;
                if (q < ns) {
                    src = (int)L.src(L.key(sc + q));
                    v = cv.count[src];
                    S.soff[q] = make_float4((float)(cv.cx[src] - cx), (float)(cv.cy[src] - cy),
                                            (float)(cv.cz[src] - cz), 0.f);
                }
                uint32_t incl = v;
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += t;
                }
                if (q < ns) {
                    const uint32_t excl = base + incl - v;
                    S.pre[q + 1] = excl + v;
                    S.sbase[q] = cv.first[src] - excl;
                    if (src == c) {
                        self_q = q;
                        self_at = (int)excl;
                    }
                }
                base += __shfl_sync(FULL, incl, 31);
            }
            if (lane == 0) S.pre[0] = 0;
            __syncwarp();
            // the leaves whose bodies fit in the table (at least one)
            unsigned fit = 0;
            for (int q = lane; q < ns; q += 32) fit += S.pre[q + 1] <= P2PW_MAP ? 1u : 0u;
            const int nl = max(1, (int)__reduce_add_sync(FULL, fit));
            const bool mapped = S.pre[nl] <= P2PW_MAP;
            const int sp = __reduce_max_sync(FULL, self_q < nl ? self_at : -1);
            if (mapped)
                for (int q = lane; q < nl; q += 32)
                    for (uint32_t e = S.pre[q]; e < S.pre[q + 1]; ++e) S.own[e] = (uint8_t)q;
            __syncwarp();
            const uint32_t total = S.pre[nl];
            sc += nl;
            for (uint32_t b0 = 0; b0 < total; b0 += P2PW_TILE) {
                const uint32_t nb = min((uint32_t)P2PW_TILE, total - b0);
                const int npair = (int)(nb + 1) >> 1;
                for (int q = lane; q < npair; q += 32) {
                    float4 s2[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const uint32_t gg = b0 + 2u * (uint32_t)q + (uint32_t)h;
                        if (gg < b0 + nb) {
                            const int l = mapped ? (int)S.own[gg] : 0;
                            const float4 v = loc[gg + S.sbase[l]];
                            const float4 o = S.soff[l];
                            s2[h] = make_float4(v.x + o.x, v.y + o.y, v.z + o.z, v.w);
                        } else {
                            s2[h] = make_float4(1e18f, 0.f, 0.f, 0.f);  // massless padding
                        }
                    }
                    S.ta[q] = make_float4(s2[0].x, s2[1].x, s2[0].y, s2[1].y);
                    S.tz[q] = make_float4(s2[0].z, s2[1].z, s2[0].w, s2[1].w);
                }
                __syncwarp();
                if (active) {
                    const bool overlaps = sp >= 0 && (uint32_t)sp < b0 + nb && (uint32_t)sp + (uint32_t)nt > b0;
                    if (!overlaps) {
#pragma unroll 2
                        for (int j = rep; j < npair; j += R) {
                            const float4 a = S.ta[j], b = S.tz[j];
                            p2p_pair(a, b, nx0, ny0, nz0, soft2, q0x, q0y, q0z, q0p);
                            p2p_pair(a, b, nx1, ny1, nz1, soft2, q1x, q1y, q1z, q1p);
                        }
                    } else {
                        // the target's own body sits at position sp + i in the sources
                        const int s0 = sp + i0 - (int)b0, s1 = sp + i1 - (int)b0;
                        for (int j = rep; j < npair; j += R) {
                            const float4 a = S.ta[j], b = S.tz[j];
                            float4 a0 = a, b0v = b, a1 = a, b1v = b;
                            if (s0 >= 0 && j == (s0 >> 1)) mask_self(a0, b0v, s0 & 1, x0, y0, z0);
                            if (s1 >= 0 && j == (s1 >> 1)) mask_self(a1, b1v, s1 & 1, x1, y1, z1);
                            p2p_pair(a0, b0v, nx0, ny0, nz0, soft2, q0x, q0y, q0z, q0p);
                            p2p_pair(a1, b1v, nx1, ny1, nz1, soft2, q1x, q1y, q1z, q1p);
                        }
                    }
                    held += (npair - rep + R - 1) / R;
                    if (held >= P2PM_FLUSH) flush();
                }
                __syncwarp();
            }
        }
        flush();
        S.red[0][lane] = a0x.hi; S.red[1][lane] = a0x.lo; S.red[2][lane] = a0y.hi; S.red[3][lane] = a0y.lo;
        S.red[4][lane] = a0z.hi; S.red[5][lane] = a0z.lo; S.red[6][lane] = p0.hi; S.red[7][lane] = p0.lo;
        S.red[8][lane] = a1x.hi; S.red[9][lane] = a1x.lo; S.red[10][lane] = a1y.hi; S.red[11][lane] = a1y.lo;
        S.red[12][lane] = a1z.hi; S.red[13][lane] = a1z.lo; S.red[14][lane] = p1.hi; S.red[15][lane] = p1.lo;
        __syncwarp();
        // outputs: nt targets x 4 components, each the sum over the R groups
        // in group order
        for (int o = lane; o < 4 * nt; o += 32) {
            const int t = o >> 2, comp = o & 3;
            const int gi = t % G, half = t / G;  // target t = gi + half * G
            const int row = 8 * half + 2 * comp;
            double v = 0.0;
            for (int r = 0; r < R; ++r) v += (double)S.red[row][r * G + gi] + (double)S.red[row + 1][r * G + gi];
            if (nu == 1) {
                double* out = comp == 0 ? ax : comp == 1 ? ay : comp == 2 ? az : pot;
                out[tf + t] = v;
            } else {
                reinterpret_cast<double*>(U.part + U.soff[c] + k * (uint32_t)nt + t)[comp] = v;
            }
        }
        __syncwarp();
    }
}

// The bodies of the leaves with several units: the units' partial sums, in
// unit order (one warp per leaf).
__global__ void k_p2p_combine(int ncells, CellsView cv, P2pUnits U, double* __restrict__ ax, double* __restrict__ ay,
                              double* __restrict__ az, double* __restrict__ pot) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells; c += warps) {
        const uint32_t nu = U.uoff[c + 1] - U.uoff[c];
        if (nu <= 1) continue;
        const uint32_t tn = cv.count[c], tf = cv.first[c];
        const double4* pp = U.part + U.soff[c];
        for (uint32_t i = lane; i < tn; i += 32) {
            double4 s = pp[i];
            for (uint32_t k = 1; k < nu; ++k) {
                const double4 v = pp[k * tn + i];
                s.x += v.x;
                s.y += v.y;
                s.z += v.z;
                s.w += v.w;
            }
            ax[tf + i] = s.x;
            ay[tf + i] = s.y;
            az[tf + i] = s.z;
            pot[tf + i] = s.w;
        }
    }
}

void launch_p2p_plan(unsigned grid, cudaStream_t s, int ncells, DirList L, const uint32_t* count, uint32_t* units,
                     uint32_t* units_s, uint32_t* units_b, uint32_t* scratch) {
    k_p2p_plan<<<grid, 256, 0, s>>>(ncells, L, count, units, units_s, units_b, scratch);
}

template <int TILE>
static void launch_tile(int nsm, cudaStream_t s, DirList L, int ncells, CellsView cv, P2pUnits U, const float4* loc,
                        float soft2, double* ax, double* ay, double* az, double* pot) {
    // persistent blocks: as many as fit on an SM at once (capping them at four
    // to leave room for the far field's list kernels beside the P2P was
    // measured: the P2P lost more, 31.5 -> 35.8 ms at the clustered
    // N = 2^22 workload, than the lists gained)
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_p2p_mixed<TILE>, P2PM_BLOCK, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    k_p2p_mixed<TILE><<<nsm * per_sm, P2PM_BLOCK, 0, s>>>(L, ncells, cv, U, loc, soft2, ax, ay, az, pot);
}

void launch_p2p_mixed(int tile, int nsm, cudaStream_t s, DirList L, int ncells, CellsView cv, P2pUnits U, size_t n,
                      const int32_t* body_leaf, const double* x, const double* y, const double* z, const double* m,
                      float4* loc, float soft2, double* ax, double* ay, double* az, double* pot) {
    k_local_coords<<<grid_for(n, 256), 256, 0, s>>>(n, body_leaf, cv, x, y, z, m, loc);
    {  // the small leaves' units, a warp each, persistent
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_p2p_mixed_small, 32 * P2PW_WARPS, 0) !=
                cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
        k_p2p_mixed_small<<<nsm * per_sm, 32 * P2PW_WARPS, 0, s>>>(L, ncells, cv, U, loc, soft2, ax, ay, az, pot);
    }
    if (tile <= 128) launch_tile<128>(nsm, s, L, ncells, cv, U, loc, soft2, ax, ay, az, pot);
    else if (tile <= 256) launch_tile<256>(nsm, s, L, ncells, cv, U, loc, soft2, ax, ay, az, pot);
    else if (tile <= 512) launch_tile<512>(nsm, s, L, ncells, cv, U, loc, soft2, ax, ay, az, pot);
    else launch_tile<1024>(nsm, s, L, ncells, cv, U, loc, soft2, ax, ay, az, pot);
    k_p2p_combine<<<grid_for((size_t)ncells * 32, 256), 256, 0, s>>>(ncells, cv, U, ax, ay, az, pot);
}

}  // namespace fmmx
