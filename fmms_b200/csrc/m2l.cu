// M2L: multipole-to-local translation over the directed M2L list.
//
// Each CTA owns one destination cell, walks its sources in ascending order and
// keeps the destination's local expansion in registers, so locals are written
// once and without atomics, and results are bit-reproducible.
//
// Two kernels:
//  - naive: F_B[n,m] += sum_{k,l} conj(M_A[k,l]) Θ_{n+k}^{m+l}(s_B - z_A)
//    (translate.rs:47-136, one direction at a time);
//  - rotation: rotate the source multipole so the translation vector lies on
//    z, translate along z with the diagonal kernel
//    F~_n^m = sum_k b_k^{-m} (n+k)! / R^{n+k+1}, rotate back
//    (rotation.rs:262-435, Dehnen 2014 A.6.1 swap decomposition
//    D = Z(α+π/2)·B·Z(-β)·B·Z(-π/2)), O(p^3) per translation.
#include "common.cuh"
#include "kernels.h"

namespace fmmx {

// The order tables in global memory: the kernels read them with lane-
// dependent indices (a lane per order m or per degree), which the constant
// cache would serialise over the distinct addresses; global loads are served
// from L1 in parallel.
static __device__ OrderTables g_tab;

#define M2L_BLOCK 128
#define M2L_OUT ((FMMX_MAXDIM + M2L_BLOCK - 1) / M2L_BLOCK)

void upload_tables_m2l(const OrderTables& t, cudaStream_t s) {
    cudaMemcpyToSymbolAsync(g_tab, &t, sizeof(t), 0, cudaMemcpyHostToDevice, s);
}

__device__ __forceinline__ void split_e(int e, int& n, int& m) {
    int q = (int)sqrtf((float)e);
    while (q * q > e) --q;
    while ((q + 1) * (q + 1) <= e) ++q;
    n = q;
    m = e - q * (q + 1);
}

// Θ column m of r (theta_table_into, harmonic.rs:91-129) into t, negative
// orders by Θ_n^{-m} = (-1)^m conj(Θ_n^m).
__device__ __forceinline__ void theta_column_f64(double x, double y, double z, double r2i, double ir, int p, int m,
                                                 zd* t) {
    zd d = mk(ir, 0.0);
    for (int j = 1; j <= m; ++j) d = zmul(zscale(mk(x, y), (double)(2 * j - 1) * r2i), d);
    t[cidx(m, m)] = d;
    zd u1 = d, u2 = mk(0.0, 0.0);
    for (int n = m + 1; n <= p; ++n) {
        const double a = (double)(2 * n - 1) * z;
        const double b = (double)((n - 1) * (n - 1) - m * m);
        zd un = zscale(zsub(zscale(u1, a), zscale(u2, b)), r2i);
        t[cidx(n, m)] = un;
        u2 = u1;
        u1 = un;
    }
    if (m > 0) {
        const double sgn = (m & 1) ? -1.0 : 1.0;
        for (int n = m; n <= p; ++n) t[cidx(n, -m)] = zscale(zconj(t[cidx(n, m)]), sgn);
    }
}

__global__ void __launch_bounds__(M2L_BLOCK) k_m2l_naive_f64(DirList L, int ncells, CellsView cv, int p,
                                                            const zd* __restrict__ moments, zd* __restrict__ locals) {
    extern __shared__ unsigned char smem_raw[];
    const int dim = dimp(p);
    zd* th = reinterpret_cast<zd*>(smem_raw);
    zd* cm = th + dim;
    const int tid = threadIdx.x;
    int on[M2L_OUT], om[M2L_OUT];
#pragma unroll
    for (int j = 0; j < M2L_OUT; ++j) {
        int e = tid + j * M2L_BLOCK;
        if (e < dim) split_e(e, on[j], om[j]);
        else on[j] = -1;
    }
    for (int c = blockIdx.x; c < ncells; c += gridDim.x) {
        const uint32_t beg = L.seg_begin[c], end = L.seg_end[c];
        if (beg >= end) continue;
        const double bx = cv.cx[c], by = cv.cy[c], bz = cv.cz[c];
        double fr[M2L_OUT], fi[M2L_OUT];
#pragma unroll
        for (int j = 0; j < M2L_OUT; ++j) fr[j] = fi[j] = 0.0;
        for (uint32_t s = beg; s < end; ++s) {
            const int src = (int)L.src(L.key(s));
            const double rx = bx - cv.cx[src], ry = by - cv.cy[src], rz = bz - cv.cz[src];
            if (tid <= p) {
                const double r2 = rx * rx + ry * ry + rz * rz;
                const double r2i = 1.0 / r2;
                theta_column_f64(rx, ry, rz, r2i, rsqrt(r2), p, tid, th);
            }
            const zd* ms = moments + (size_t)src * dim;
            for (int e = tid; e < dim; e += M2L_BLOCK) cm[e] = zconj(ms[e]);
            __syncthreads();
#pragma unroll
            for (int j = 0; j < M2L_OUT; ++j) {
                const int n = on[j];
                if (n < 0) continue;
                const int m = om[j];
                double ar = 0.0, ai = 0.0;
                for (int k = 0; k <= p - n; ++k) {
                    const zd* tk = th + cidx(n + k, m);
                    const zd* mk_ = cm + cidx(k, 0);
                    for (int l = -k; l <= k; ++l) {
                        const zd a = mk_[l], t = tk[l];
                        ar += a.re * t.re - a.im * t.im;
                        ai += a.re * t.im + a.im * t.re;
                    }
                }
                fr[j] += ar;
                fi[j] += ai;
            }
            __syncthreads();
        }
        zd* out = locals + (size_t)c * dim;
#pragma unroll
        for (int j = 0; j < M2L_OUT; ++j) {
            int e = tid + j * M2L_BLOCK;
            if (e < dim) out[e] = mk(fr[j], fi[j]);
        }
    }
}

// ------------------------------------------------------------ rotation M2L
// Block layout of the swap matrices: degree j occupies (2j+1)^2 reals from
// block_off(j) = j(4j^2-1)/3 (rotation.rs:49-61).
__device__ __forceinline__ int block_off(int j) { return j == 0 ? 0 : j * (4 * j * j - 1) / 3; }

// Folded diagonals of RotCtx::new (rotation.rs:212-235): with
// ei = e^{-imπ/2} and fm = (n-|m|)!(n+|m|)!,
// in = ei·fm, out = conj(ei)/fm, fin = ei/fm, fout = conj(ei)·fm.
__device__ __forceinline__ zd ei_of(int m) {
    switch (m & 3) {
        case 0: return mk(1.0, 0.0);
        case 1: return mk(0.0, -1.0);
        case 2: return mk(-1.0, 0.0);
        default: return mk(0.0, 1.0);
    }
}

__global__ void __launch_bounds__(M2L_BLOCK) k_m2l_rot_f64(DirList L, int ncells, CellsView cv, int p,
                                                          const zd* __restrict__ moments, zd* __restrict__ locals,
                                                          const double* __restrict__ swap_g) {
    extern __shared__ unsigned char smem_raw[];
    const int dim = dimp(p);
    const int bs = (p + 1) * (4 * p * p + 8 * p + 3) / 3;
    double* sw = reinterpret_cast<double*>(smem_raw);
    zd* A = reinterpret_cast<zd*>(sw + bs);
    zd* B = A + dim;
    zd* pha = B + dim;       // e^{imα}, index m + p
    zd* phb = pha + 2 * p + 1;  // e^{imβ}
    double* facr = reinterpret_cast<double*>(phb + 2 * p + 1);  // j!/R^{j+1}
    const int tid = threadIdx.x;
    for (int i = tid; i < bs; i += M2L_BLOCK) sw[i] = swap_g[i];
    int on[M2L_OUT], om[M2L_OUT];
    double fmv[M2L_OUT];
#pragma unroll
    for (int j = 0; j < M2L_OUT; ++j) {
        int e = tid + j * M2L_BLOCK;
        if (e < dim) {
            split_e(e, on[j], om[j]);
            int am = om[j] < 0 ? -om[j] : om[j];
            fmv[j] = g_tab.fact[on[j] - am] * g_tab.fact[on[j] + am];
        } else {
            on[j] = -1;
        }
    }
    __syncthreads();
    for (int c = blockIdx.x; c < ncells; c += gridDim.x) {
        const uint32_t beg = L.seg_begin[c], end = L.seg_end[c];
        if (beg >= end) continue;
        const double bx = cv.cx[c], by = cv.cy[c], bz = cv.cz[c];
        double fr[M2L_OUT], fi[M2L_OUT];
#pragma unroll
        for (int j = 0; j < M2L_OUT; ++j) fr[j] = fi[j] = 0.0;
        for (uint32_t s = beg; s < end; ++s) {
            const int src = (int)L.src(L.key(s));
            const double rx = bx - cv.cx[src], ry = by - cv.cy[src], rz = bz - cv.cz[src];
            const double r2 = rx * rx + ry * ry + rz * rz;
            const double alpha = atan2(ry, rx);
            const double beta = atan2(sqrt(rx * rx + ry * ry), rz);
            for (int i = tid; i <= 2 * p; i += M2L_BLOCK) {
                const int m = i - p;
                double sa, ca, sb, cb;
                sincos((double)m * alpha, &sa, &ca);
                sincos((double)m * beta, &sb, &cb);
                pha[i] = mk(ca, sa);
                phb[i] = mk(cb, sb);
            }
            if (tid <= p) {
                const double rinv = rsqrt(r2);
                double irp = rinv;
                for (int j = 0; j < tid; ++j) irp *= rinv;
                facr[tid] = g_tab.fact[tid] * irp;
            }
            __syncthreads();
            // 1) back-rotate, u = in·pha·conj(M)
            const zd* ms = moments + (size_t)src * dim;
#pragma unroll
            for (int j = 0; j < M2L_OUT; ++j) {
                const int n = on[j];
                if (n < 0) continue;
                const int m = om[j];
                const zd mv = ms[cidx(n, m)];
                const zd ph = pha[m + p];
                const double vr = mv.re * ph.re + mv.im * ph.im;
                const double vi = mv.re * ph.im - mv.im * ph.re;
                const zd iv = zscale(ei_of(m), fmv[j]);
                A[cidx(n, m)] = mk(vr * iv.re - vi * iv.im, vr * iv.im + vi * iv.re);
            }
            __syncthreads();
            // s = B_k u, q = phb·s
#pragma unroll
            for (int j = 0; j < M2L_OUT; ++j) {
                const int k = on[j];
                if (k < 0) continue;
                const int r = om[j] + k, nb = 2 * k + 1;
                const double* row = sw + block_off(k) + r * nb;
                const zd* v = A + k * k;
                double sr = 0.0, si = 0.0;
                for (int q = 0; q < nb; ++q) {
                    sr += row[q] * v[q].re;
                    si += row[q] * v[q].im;
                }
                B[k * k + r] = zmul(mk(sr, si), phb[om[j] + p]);
            }
            __syncthreads();
            // r = B_k q, b = out·r
#pragma unroll
            for (int j = 0; j < M2L_OUT; ++j) {
                const int k = on[j];
                if (k < 0) continue;
                const int r = om[j] + k, nb = 2 * k + 1;
                const double* row = sw + block_off(k) + r * nb;
                const zd* v = B + k * k;
                double sr = 0.0, si = 0.0;
                for (int q = 0; q < nb; ++q) {
                    sr += row[q] * v[q].re;
                    si += row[q] * v[q].im;
                }
                const zd ov = zscale(zconj(ei_of(om[j])), 1.0 / fmv[j]);
                A[k * k + r] = zmul(mk(sr, si), ov);
            }
            __syncthreads();
            // 2) axial translation, F~[n][m] = sum_{k=|m|}^{p-n} b[k,-m] facr[n+k]; then g = fin·F~
#pragma unroll
            for (int j = 0; j < M2L_OUT; ++j) {
                const int n = on[j];
                if (n < 0) continue;
                const int m = om[j];
                const int am = m < 0 ? -m : m;
                double sr = 0.0, si = 0.0;
                for (int k = am; k <= p - n; ++k) {
                    const zd bv = A[k * k + (k - m)];
                    const double fv = facr[n + k];
                    sr += bv.re * fv;
                    si += bv.im * fv;
                }
                B[cidx(n, m)] = zmul(mk(sr, si), zscale(ei_of(m), 1.0 / fmv[j]));
            }
            __syncthreads();
            // 3) forward: s = B_n^T g, q = conj(phb)·s
#pragma unroll
            for (int j = 0; j < M2L_OUT; ++j) {
                const int n = on[j];
                if (n < 0) continue;
                const int r = om[j] + n, nb = 2 * n + 1;
                const double* col = sw + block_off(n) + r;
                const zd* v = B + n * n;
                double sr = 0.0, si = 0.0;
                for (int q = 0; q < nb; ++q) {
                    const double w = col[q * nb];
                    sr += w * v[q].re;
                    si += w * v[q].im;
                }
                A[n * n + r] = zmul(mk(sr, si), zconj(phb[om[j] + p]));
            }
            __syncthreads();
            // r = B_n^T q, locals += fout·pha·r
#pragma unroll
            for (int j = 0; j < M2L_OUT; ++j) {
                const int n = on[j];
                if (n < 0) continue;
                const int r = om[j] + n, nb = 2 * n + 1;
                const double* col = sw + block_off(n) + r;
                const zd* v = A + n * n;
                double sr = 0.0, si = 0.0;
                for (int q = 0; q < nb; ++q) {
                    const double w = col[q * nb];
                    sr += w * v[q].re;
                    si += w * v[q].im;
                }
                const zd acc = zmul(mk(sr, si), zscale(zconj(ei_of(om[j])), fmv[j]));
                const zd add = zmul(acc, pha[om[j] + p]);
                fr[j] += add.re;
                fi[j] += add.im;
            }
            __syncthreads();
        }
        zd* out = locals + (size_t)c * dim;
#pragma unroll
        for (int j = 0; j < M2L_OUT; ++j) {
            int e = tid + j * M2L_BLOCK;
            if (e < dim) out[e] = mk(fr[j], fi[j]);
        }
    }
}

size_t m2l_rot_smem_bytes(int p) {
    const int dim = dimp(p);
    const int bs = (p + 1) * (4 * p * p + 8 * p + 3) / 3;
    return (size_t)bs * 8 + 2 * (size_t)dim * 16 + 2 * (2 * p + 1) * 16 + (p + 1) * 8;
}

}  // namespace fmmx
