// Downward sweep: L2L (parent local -> child local) level by level from the
// top, and L2P at every body combined with the near field and scattered back
// to particle-id order.
//
//   L2L (translate.rs:175-218): F_c[n,m] += sum_{k,l} conj(Υ_k^l(s - s')) F_p[n+k, m+l]
//   L2P (translate.rs:271-346): Ψ_n^m(x) = sum conj(Υ_k^l(s - x)) F[n+k, m+l],
//       pot += Re Ψ_0^0, a -= (Re Ψ_1^1, Im Ψ_1^1, Ψ_1^0).
#include "common.cuh"
#include "kernels.h"

namespace fmmx {

// The order tables in global memory: the kernels read them with lane-
// dependent indices (a lane per order m or per degree), which the constant
// cache would serialise over the distinct addresses; global loads are served
// from L1 in parallel.
static __device__ OrderTables g_tab;

void upload_tables_sweeps(const OrderTables& t, cudaStream_t s) {
    cudaMemcpyToSymbolAsync(g_tab, &t, sizeof(t), 0, cudaMemcpyHostToDevice, s);
}

#define SW_BLOCK 128
#define SW_OUT ((FMMX_MAXDIM + SW_BLOCK - 1) / SW_BLOCK)

__device__ __forceinline__ void split_e2(int e, int& n, int& m) {
    int q = (int)sqrtf((float)e);
    while (q * q > e) --q;
    while ((q + 1) * (q + 1) <= e) ++q;
    n = q;
    m = e - q * (q + 1);
}

// Υ column m (upsilon_table_into, harmonic.rs:141-173) with negative orders.
__device__ __forceinline__ void upsilon_column_f64(double x, double y, double z, double r2, int p, int m, zd* u) {
    zd d = mk(1.0, 0.0);
    for (int j = 1; j <= m; ++j) d = zmul(zscale(mk(x, y), g_tab.inv2m[j]), d);
    u[cidx(m, m)] = d;
    zd u1 = d, u2 = mk(0.0, 0.0);
    for (int n = m + 1; n <= p; ++n) {
        const double a = (double)(2 * n - 1) * z;
        zd un = zscale(zsub(zscale(u1, a), zscale(u2, r2)), g_tab.invc[n][m]);
        u[cidx(n, m)] = un;
        u2 = u1;
        u1 = un;
    }
    if (m > 0) {
        const double sgn = (m & 1) ? -1.0 : 1.0;
        for (int n = m; n <= p; ++n) u[cidx(n, -m)] = zscale(zconj(u[cidx(n, m)]), sgn);
    }
}

// One CTA per cell of level L (L >= 1): its parent (level L-1) is final.
__global__ void __launch_bounds__(SW_BLOCK) k_l2l_f64(const int32_t* __restrict__ level_cells, int lstart, int lcnt,
                                                     CellsView cv, const int32_t* __restrict__ parent, int p,
                                                     zd* __restrict__ locals) {
    extern __shared__ unsigned char smem_raw[];
    const int dim = dimp(p);
    zd* u = reinterpret_cast<zd*>(smem_raw);
    zd* fp = u + dim;
    const int tid = threadIdx.x;
    for (int j = blockIdx.x; j < lcnt; j += gridDim.x) {
        const int c = level_cells[lstart + j];
        const int par = parent[c];
        if (par < 0) continue;
        const double rx = cv.cx[par] - cv.cx[c], ry = cv.cy[par] - cv.cy[c], rz = cv.cz[par] - cv.cz[c];
        if (tid <= p) upsilon_column_f64(rx, ry, rz, rx * rx + ry * ry + rz * rz, p, tid, u);
        const zd* lp = locals + (size_t)par * dim;
        for (int e = tid; e < dim; e += SW_BLOCK) fp[e] = lp[e];
        __syncthreads();
        zd* lc = locals + (size_t)c * dim;
        for (int e = tid; e < dim; e += SW_BLOCK) {
            int n, m;
            split_e2(e, n, m);
            double sr = 0.0, si = 0.0;
            for (int k = 0; k <= p - n; ++k) {
                const zd* uk = u + cidx(k, 0);
                const zd* fk = fp + cidx(n + k, m);
                for (int l = -k; l <= k; ++l) {
                    const zd a = uk[l], b = fk[l];  // conj(a) * b
                    sr += a.re * b.re + a.im * b.im;
                    si += a.re * b.im - a.im * b.re;
                }
            }
            lc[e] = zadd(lc[e], mk(sr, si));
        }
        __syncthreads();
    }
}

// One thread per body (slot order). The Υ table of s - x is generated column
// by column (two-term recursion in n) and contracted on the fly, so no table
// is stored.
__global__ void k_l2p_f64(size_t n, const int32_t* __restrict__ body_leaf, const uint32_t* __restrict__ order,
                          CellsView cv, int p, const zd* __restrict__ locals, const double* __restrict__ x,
                          const double* __restrict__ y, const double* __restrict__ z, const double* __restrict__ nax,
                          const double* __restrict__ nay, const double* __restrict__ naz,
                          const double* __restrict__ npot, double* __restrict__ acc, double* __restrict__ pot) {
    const int dim = dimp(p);
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int c = body_leaf[k];
        const double rx = cv.cx[c] - x[k], ry = cv.cy[c] - y[k], rz = cv.cz[c] - z[k];
        const double r2 = rx * rx + ry * ry + rz * rz;
        const zd* L = locals + (size_t)c * dim;
        double p00 = 0.0, p11r = 0.0, p11i = 0.0, p10 = 0.0;
        zd d = mk(1.0, 0.0);
        for (int l = 0; l <= p; ++l) {
            if (l > 0) d = zmul(zscale(mk(rx, ry), g_tab.inv2m[l]), d);
            zd u1 = d, u2 = mk(0.0, 0.0);
            const double sgn = (l & 1) ? -1.0 : 1.0;
            for (int kk = l; kk <= p; ++kk) {
                zd uk;
                if (kk == l) {
                    uk = d;
                } else {
                    const double a = (double)(2 * kk - 1) * rz;
                    uk = zscale(zsub(zscale(u1, a), zscale(u2, r2)), g_tab.invc[kk][l]);
                    u2 = u1;
                    u1 = uk;
                }
                // conj(u) * F for +l; conj(u_{k,-l}) = (-1)^l u_{k,l} for -l
                const zd f0 = L[cidx(kk, l)];
                p00 += uk.re * f0.re + uk.im * f0.im;
                if (kk < p) {
                    const zd f11 = L[cidx(kk + 1, l + 1)];
                    const zd f10 = L[cidx(kk + 1, l)];
                    p11r += uk.re * f11.re + uk.im * f11.im;
                    p11i += uk.re * f11.im - uk.im * f11.re;
                    p10 += uk.re * f10.re + uk.im * f10.im;
                }
                if (l > 0) {
                    const zd g0 = L[cidx(kk, -l)];
                    p00 += sgn * (uk.re * g0.re - uk.im * g0.im);
                    if (kk < p) {
                        const zd g11 = L[cidx(kk + 1, 1 - l)];
                        const zd g10 = L[cidx(kk + 1, -l)];
                        p11r += sgn * (uk.re * g11.re - uk.im * g11.im);
                        p11i += sgn * (uk.re * g11.im + uk.im * g11.re);
                        p10 += sgn * (uk.re * g10.re - uk.im * g10.im);
                    }
                }
            }
        }
        const uint32_t id = order[k];
        acc[3 * (size_t)id + 0] = nax[k] + (0.0 - p11r);
        acc[3 * (size_t)id + 1] = nay[k] + (0.0 - p11i);
        acc[3 * (size_t)id + 2] = naz[k] + (0.0 - p10);
        pot[id] = npot[k] + p00;
    }
}

}  // namespace fmmx
