// Rotation M2L, one lane per directed translation, templated on the
// arithmetic type T (double for the plain form, float for the mixed form) and
// the expansion order P.
//
// Algorithm (the reference's RotCtx::m2l_pair/apply, rotation.rs:262-435,
// Dehnen 2014 A.6.1): back-rotate the source multipole with two x<->z swaps
// B_k around a z-rotation by -β, translate along z with the diagonal kernel
// F~_n^m = sum_k b_k^{-m} (n+k)!/R^{n+k+1}, rotate forward with B_n^T, and add
// into the destination's local expansion.
//
// B200 structure:
//  - A warp owns one destination cell; each lane takes one of its sources, so
//    32 translations run side by side and the destination sum is a reduction
//    across lanes through shared memory (no atomics, fixed order).
//  - Expansions of a real field satisfy v_{-m} = (-1)^m conj(v_m); so do all
//    intermediate vectors (rotations map real fields to real fields). Only
//    m >= 0 is stored, and each swap matvec splits into two real
//    (k+1)x(k+1) products: Re(s) = P_k Re(u), Im(s) = Q_k Im(u) with
//    P_k[r][c] = B_k[r][c] + (-1)^c B_k[r][-c], Q_k[r][c] = B_k[r][c] - (-1)^c B_k[r][-c].
//  - P_k, Q_k (and those of B_k^T) are pair independent and live in constant
//    memory; with P fixed at compile time every matrix element is a constant-
//    bank operand of the FMA that uses it, uniform across the warp.
//  - Phases e^{imα}, e^{imβ} come from powers of (x + iy)/ρ_xy and
//    (z + iρ_xy)/R: no trigonometric calls.
//  - SCALED expansions (mixed form) carry M^_k = M_k / l_a^k and
//    F^_n = F_n l_b^{n+1}, l the cell's radius, so FP32 never overflows at
//    high order: the axial kernel becomes (n+k)! (l_a/R)^k (l_b/R)^{n+1}.
//
// The including file defines ROTW_T (the element type of the constant tables)
// before including this header, once per translation unit.
#pragma once

#include <type_traits>
#include <utility>

#include "common.cuh"
#include "kernels.h"

namespace fmmx {

__host__ __device__ constexpr int rot_hx(int n, int m) { return n * (n + 1) / 2 + m; }
// offset of degree k's four matrices (P, Q, PT, QT), each (k+1)^2
__host__ __device__ constexpr int rot_moff(int k) { return 4 * (k * (k + 1) * (2 * k + 1) / 6); }
#define ROTW_MAXP 16
#define ROTW_MATS (rot_moff(ROTW_MAXP + 1))
#define ROTW_NH (rot_hx(ROTW_MAXP, ROTW_MAXP) + 1)
#ifndef ROTW_AXR_MAXP
#define ROTW_AXR_MAXP 10
#endif
#define ROTW_LD 33  // entry stride of the per-lane columns (conflict-free both ways)

static __constant__ ROTW_T c_rot[ROTW_MATS];            // P_k, Q_k, P_k^T, Q_k^T per degree
static __constant__ ROTW_T c_fm[ROTW_NH];               // (n-m)!(n+m)!, half index
static __constant__ ROTW_T c_ifm[ROTW_NH];              // 1/((n-m)!(n+m)!)
static __constant__ ROTW_T c_fact[2 * ROTW_MAXP + 1];   // j!


// Pair phases e^{imα}, e^{imβ} (m = 0..P): in the lane's shared-memory
// column (FP64: registers are too few) or in registers (FP32).
template <typename T>
struct PhSmem {
    const cplx<T>* a;
    const cplx<T>* b;
    __device__ __forceinline__ cplx<T> A(int m) const { return a[ROTW_LD * m]; }
    __device__ __forceinline__ cplx<T> B(int m) const { return b[ROTW_LD * m]; }
};
template <typename T, int P>
struct PhRegs {
    cplx<T> a[P + 1], b[P + 1];
    __device__ __forceinline__ cplx<T> A(int m) const { return a[m]; }
    __device__ __forceinline__ cplx<T> B(int m) const { return b[m]; }
};

// The per-degree (per-column) bodies below take the degree as a template
// parameter and are expanded over 0..P with an index_sequence fold, so every
// matrix offset, loop bound and array index is a compile-time constant and the
// swap-matrix elements reach the FMAs as constant-bank operands.

// (-i)^m * (ur + i ui) for m mod 4, and i^m * (...)
template <int M, typename T>
__device__ __forceinline__ void mul_mi_pow(T& r, T& i) {
    const T a = r, b = i;
    if constexpr ((M & 3) == 1) { r = b; i = -a; }
    else if constexpr ((M & 3) == 2) { r = -a; i = -b; }
    else if constexpr ((M & 3) == 3) { r = -b; i = a; }
}
template <int M, typename T>
__device__ __forceinline__ void mul_i_pow(T& r, T& i) {
    const T a = r, b = i;
    if constexpr ((M & 3) == 1) { r = -b; i = a; }
    else if constexpr ((M & 3) == 2) { r = -a; i = -b; }
    else if constexpr ((M & 3) == 3) { r = b; i = -a; }
}

// Compiler barrier between degrees: it bounds the live registers. FP32 up to
// p = 10 fits without it, and the scheduler then overlaps neighbouring degrees
// (measured: p = 8 9 % and p = 10 3 % faster without; p = 12 spills and runs
// 8 % slower without); FP64 and higher orders keep it.
template <typename T, int P>
__device__ __forceinline__ void degree_fence() {
    if constexpr (sizeof(T) != 4 || P > 10) asm volatile("" ::: "memory");
}

// Where the back-rotated expansion b goes: the lane's shared-memory column,
// from which the axial step reads it by order, or registers (FP32 at low
// order), from which the forward rotation reads it directly.
template <typename T>
struct ColOut {
    cplx<T>* col;
    template <int E>
    __device__ __forceinline__ void put(T re, T im) { col[ROTW_LD * E] = mk<T>(re, im); }
};
template <typename T, int H>
struct RegOut {
    T re[H], im[H];
    template <int E>
    __device__ __forceinline__ void put(T r, T i) { re[E] = r; im[E] = i; }
};

template <int M, typename T, int N>
struct Unroll {  // compile-time loop helper: f(integral_constant<m>) for m = M..N-1
    template <class F>
    __device__ __forceinline__ static void run(F&& f) {
        if constexpr (M < N) {
            f(std::integral_constant<int, M>{});
            Unroll<M + 1, T, N>::run(f);
        }
    }
};

// Real half-basis swap matvec: Re(s) = Pm Re(v), Im(s) = Qm Im(v), degree
// K = N - 1. The half-basis swap matrices are zero in a parity pattern:
// Pm[r][q] = 0 unless r + q + K is even, Qm[r][q] = 0 unless r, q >= 1 and
// r + q + K is odd, and the same for the matrices of B_K^T (rotw_tables_check
// verifies this on the host for every degree when a context is created). The
// zero terms, about half of each product, are left out at compile time; the
// others are added in the same order as in the full product.
template <typename T, int N, int OFF>
__device__ __forceinline__ void swap_matvec(const T (&vr)[N], const T (&vi)[N], T (&sr)[N], T (&si)[N]) {
    Unroll<0, T, N>::run([&](auto rc) {
        constexpr int r = decltype(rc)::value;
        T a = T(0), b = T(0);
        Unroll<0, T, N>::run([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            if constexpr (((r + q + N - 1) & 1) == 0) a += c_rot[OFF + r * N + q] * vr[q];
            if constexpr (r >= 1 && q >= 1 && ((r + q + N - 1) & 1) == 1) b += c_rot[OFF + N * N + r * N + q] * vi[q];
        });
        sr[r] = a;
        si[r] = b;
    });
}

template <typename T, int P, int K, bool FULL_LAYOUT, class PH, class OUT>
__device__ __forceinline__ void back_degree(const cplx<T>* __restrict__ ms, const PH& ph_, OUT& out, T sa,
                                            T& sak, T cap) {
    typedef cplx<T> Z;
    constexpr int N = K + 1;
    T vr[N], vi[N];
    // FP32 half layout: every cell starts on 16 bytes (the cell stride is
    // half_stride(P), even), so entry pairs that start on an even index load
    // as one float4
    Z Mv[N];
    constexpr bool PAIRS = sizeof(T) == 4 && !FULL_LAYOUT;
    constexpr int B0 = rot_hx(K, 0);
    Unroll<0, T, N>::run([&](auto jc) {
        constexpr int j = decltype(jc)::value;
        if constexpr (PAIRS && ((B0 + j) & 1) == 0 && j + 1 < N) {
            const float4 v = *reinterpret_cast<const float4*>(ms + B0 + j);
            Mv[j] = mk<T>(v.x, v.y);
            Mv[j + 1] = mk<T>(v.z, v.w);
        } else if constexpr (!PAIRS || ((B0 + j) & 1) == 0 || j == 0) {
            Mv[j] = ms[FULL_LAYOUT ? (K * (K + 1) + j) : rot_hx(K, j)];
        }
    });
    Unroll<0, T, N>::run([&](auto mc) {
        constexpr int m = decltype(mc)::value;
        const Z M = Mv[m];
        const Z ph = ph_.A(m);
        T ur = ph.re * M.re + ph.im * M.im;  // ph * conj(M)
        T ui = ph.im * M.re - ph.re * M.im;
        mul_mi_pow<m>(ur, ui);
        const T f = c_fm[rot_hx(K, m)];
        vr[m] = ur * f;
        vi[m] = ui * f;
    });
    T sr[N], si[N];
    swap_matvec<T, N, rot_moff(K)>(vr, vi, sr, si);
    Unroll<0, T, N>::run([&](auto rc) {  // q = phb * s
        constexpr int r = decltype(rc)::value;
        const Z pb = ph_.B(r);
        const T a = sr[r], b = si[r];
        vr[r] = a * pb.re - b * pb.im;
        vi[r] = a * pb.im + b * pb.re;
    });
    swap_matvec<T, N, rot_moff(K)>(vr, vi, sr, si);
    Unroll<0, T, N>::run([&](auto rc) {  // b = i^r / fm * t * sa^k
        constexpr int r = decltype(rc)::value;
        T orr = sr[r], oii = si[r];
        mul_i_pow<r>(orr, oii);
        const T g = c_ifm[rot_hx(K, r)] * sak;
        out.template put<rot_hx(K, r)>(orr * g, oii * g);
    });
    sak = min(sak * sa, cap);
    degree_fence<T, P>();
}

template <typename T, int P, bool FULL_LAYOUT, class PH, class OUT, int... Ks>
__device__ __forceinline__ void back_all(const cplx<T>* __restrict__ ms, const PH& ph_, OUT& out, T sa, T cap,
                                         std::integer_sequence<int, Ks...>) {
    T sak = T(1);
    (back_degree<T, P, Ks, FULL_LAYOUT, PH, OUT>(ms, ph_, out, sa, sak, cap), ...);
}

// `cap` bounds the scale powers of the normalised (mixed) form: a power only
// exceeds 1 where the moments it multiplies are exactly zero (a cell of radius
// 0), and the cap keeps that product 0 instead of 0 * inf.
template <typename T, int P, bool FULL_LAYOUT, class PH, class OUT>
__device__ __forceinline__ void rotw_back(const cplx<T>* __restrict__ ms, const PH& ph_, OUT& out, T sa, T cap) {
    back_all<T, P, FULL_LAYOUT, PH, OUT>(ms, ph_, out, sa, cap, std::make_integer_sequence<int, P + 1>{});
}

// axial translation of column m, in place:
// F~[n][m] = (-1)^m conj(sum_{k=m}^{P-n} b[k][m] (n+k)!) sb^{n+1}
template <typename T, int P, int M>
__device__ __forceinline__ void axial_col(cplx<T>* col, T sb, T cap) {
    constexpr int L = P - M + 1;  // entries k = M..P
    T br[L], bi[L];
    Unroll<0, T, L>::run([&](auto jc) {
        constexpr int j = decltype(jc)::value;
        const cplx<T> v = col[ROTW_LD * rot_hx(M + j, M)];
        br[j] = v.re;
        bi[j] = v.im;
    });
    T sbn = sb;
#pragma unroll
    for (int n = 0; n < M; ++n) sbn = min(sbn * sb, cap);
    constexpr T sg = (M & 1) ? T(-1) : T(1);
    Unroll<M, T, P + 1>::run([&](auto nc) {
        constexpr int n = decltype(nc)::value;
        T ar = T(0), ai = T(0);
        Unroll<M, T, P - n + 1>::run([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            ar += br[k - M] * c_fact[n + k];
            ai += bi[k - M] * c_fact[n + k];
        });
        col[ROTW_LD * rot_hx(n, M)] = mk<T>(sg * ar * sbn, -sg * ai * sbn);
        sbn = min(sbn * sb, cap);
    });
    degree_fence<T, P>();
}

template <typename T, int P, int... Ms>
__device__ __forceinline__ void axial_all(cplx<T>* col, T sb, T cap, std::integer_sequence<int, Ms...>) {
    (axial_col<T, P, Ms>(col, sb, cap), ...);
}

template <typename T, int P>
__device__ __forceinline__ void rotw_axial(cplx<T>* col, T sb, T cap) {
    axial_all<T, P>(col, sb, cap, std::make_integer_sequence<int, P + 1>{});
}

// forward rotation of degree K from g = (-i)^m F / fm, result into the column
template <typename T, int P, int K, class PH>
__device__ __forceinline__ void fwd_rotate(T (&vr)[K + 1], T (&vi)[K + 1], cplx<T>* col, const PH& ph_) {
    typedef cplx<T> Z;
    constexpr int N = K + 1;
    T sr[N], si[N];
    swap_matvec<T, N, rot_moff(K) + 2 * N * N>(vr, vi, sr, si);
    Unroll<0, T, N>::run([&](auto rc) {  // q = conj(phb) * s
        constexpr int r = decltype(rc)::value;
        const Z pb = ph_.B(r);
        const T a = sr[r], b = si[r];
        vr[r] = a * pb.re + b * pb.im;
        vi[r] = b * pb.re - a * pb.im;
    });
    swap_matvec<T, N, rot_moff(K) + 2 * N * N>(vr, vi, sr, si);
    Unroll<0, T, N>::run([&](auto rc) {  // out = i^r fm * pha * t
        constexpr int r = decltype(rc)::value;
        T orr = sr[r], oii = si[r];
        mul_i_pow<r>(orr, oii);
        const T f = c_fm[rot_hx(K, r)];
        orr *= f;
        oii *= f;
        const Z pa = ph_.A(r);
        col[ROTW_LD * rot_hx(K, r)] = mk<T>(orr * pa.re - oii * pa.im, orr * pa.im + oii * pa.re);
    });
    degree_fence<T, P>();
}

template <typename T, int P, int K, class PH>
__device__ __forceinline__ void fwd_degree(cplx<T>* col, const PH& ph_) {
    typedef cplx<T> Z;
    constexpr int N = K + 1;
    T vr[N], vi[N];
    Unroll<0, T, N>::run([&](auto mc) {  // g = (-i)^m F / fm
        constexpr int m = decltype(mc)::value;
        const Z F = col[ROTW_LD * rot_hx(K, m)];
        T ur = F.re, ui = F.im;
        mul_mi_pow<m>(ur, ui);
        const T g = c_ifm[rot_hx(K, m)];
        vr[m] = ur * g;
        vi[m] = ui * g;
    });
    fwd_rotate<T, P, K, PH>(vr, vi, col, ph_);
}

// Axial translation fused into the forward rotation, b in registers: degree K
// of the translated expansion is
// F[K][m] = (-1)^m conj(sum_{k=m}^{P-K} b[k][m] (K+k)!) sb^{K+1}, formed right
// where the forward rotation needs it (no shared-memory round trip).
template <typename T, int P, int K, int H, class PH>
__device__ __forceinline__ void axfwd_degree(const RegOut<T, H>& b, cplx<T>* col, const PH& ph_, T& sbn, T sb,
                                             T cap) {
    constexpr int N = K + 1;
    T vr[N], vi[N];
    Unroll<0, T, N>::run([&](auto mc) {  // g = (-i)^m F / fm
        constexpr int m = decltype(mc)::value;
        T ar = T(0), ai = T(0);
        Unroll<m, T, P - K + 1>::run([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            ar += b.re[rot_hx(k, m)] * c_fact[K + k];
            ai += b.im[rot_hx(k, m)] * c_fact[K + k];
        });
        constexpr T sg = (m & 1) ? T(-1) : T(1);
        T ur = sg * ar * sbn, ui = -sg * ai * sbn;
        mul_mi_pow<m>(ur, ui);
        const T g = c_ifm[rot_hx(K, m)];
        vr[m] = ur * g;
        vi[m] = ui * g;
    });
    sbn = min(sbn * sb, cap);
    fwd_rotate<T, P, K, PH>(vr, vi, col, ph_);
}

template <typename T, int P, int H, class PH, int... Ks>
__device__ __forceinline__ void axfwd_all(const RegOut<T, H>& b, cplx<T>* col, const PH& ph_, T sb, T cap,
                                          std::integer_sequence<int, Ks...>) {
    T sbn = sb;
    (axfwd_degree<T, P, Ks, H, PH>(b, col, ph_, sbn, sb, cap), ...);
}

template <typename T, int P, class PH, int... Ks>
__device__ __forceinline__ void fwd_all(cplx<T>* col, const PH& ph_, std::integer_sequence<int, Ks...>) {
    (fwd_degree<T, P, Ks, PH>(col, ph_), ...);
}

template <typename T, int P, class PH>
__device__ __forceinline__ void rotw_fwd(cplx<T>* col, const PH& ph_) {
    fwd_all<T, P, PH>(col, ph_, std::make_integer_sequence<int, P + 1>{});
}

// FP64: the three phases are separate non-inlined functions so that each is
// register-allocated on its own (all three unrolled at once overflow the
// register file and spill).
template <typename T, int P, bool FULL_LAYOUT>
__device__ __noinline__ void rotw_back_ni(const cplx<T>* __restrict__ ms, const cplx<T>* pa, const cplx<T>* pb,
                                          cplx<T>* col, T sa, T cap) {
    ColOut<T> out{col};
    rotw_back<T, P, FULL_LAYOUT>(ms, PhSmem<T>{pa, pb}, out, sa, cap);
}
template <typename T, int P>
__device__ __noinline__ void rotw_axial_ni(cplx<T>* col, T sb, T cap) {
    rotw_axial<T, P>(col, sb, cap);
}
template <typename T, int P>
__device__ __noinline__ void rotw_fwd_ni(cplx<T>* col, const cplx<T>* pa, const cplx<T>* pb) {
    rotw_fwd<T, P>(col, PhSmem<T>{pa, pb});
}

template <typename T, int P, bool SCALED, bool FULL_LAYOUT>
__device__ __forceinline__ void rotw_body(int c, uint32_t beg, uint32_t end, const DirList& L,
                                          const CellsView& cv, const T* __restrict__ scale,
                                          const cplx<T>* __restrict__ mom, cplx<T>* __restrict__ loc,
                                          cplx<T>* __restrict__ sbuf, int lane) {
    constexpr int H = (P + 1) * (P + 2) / 2;
    constexpr int NA = (H + 31) / 32;
    constexpr int DIM = (P + 1) * (P + 1);
    typedef cplx<T> Z;
    constexpr bool PH_REGS = sizeof(T) == 4;
    // FP32 up to ROTW_AXR_MAXP: b stays in registers through the axial step
    constexpr bool AXR = PH_REGS && P <= ROTW_AXR_MAXP;
    Z* col = sbuf + lane;                    // this lane's column: entry e at col[LD e]
    Z* pha = sbuf + ROTW_LD * H + lane;      // e^{imα}, m = 0..P (FP64 only)
    Z* phb = pha + ROTW_LD * (P + 1);        // e^{imβ}
    T acc_re[NA], acc_im[NA];
#pragma unroll
    for (int t = 0; t < NA; ++t) acc_re[t] = acc_im[t] = T(0);
    const double bx = cv.cx[c], by = cv.cy[c], bz = cv.cz[c];
    for (uint32_t chunk = beg; chunk < end; chunk += 32) {
        const int nact = (int)min(32u, end - chunk);
        if (lane < nact) {
            const int src = (int)L.src(L.key(chunk + lane));
            // geometry in FP64: r = s_B - z_A
            const double rx = bx - cv.cx[src], ry = by - cv.cy[src], rz = bz - cv.cz[src];
            const double rxy2 = rx * rx + ry * ry;
            const double rxy = sqrt(rxy2);
            const double R = sqrt(rxy2 + rz * rz);
            const double iR = 1.0 / R;
            double ear = 1.0, eai = 0.0;
            if (rxy > 0.0) {
                const double ir = 1.0 / rxy;
                ear = rx * ir;
                eai = ry * ir;
            }
            const T ebr = (T)(rz * iR), ebi = (T)(rxy * iR);
            PhRegs<T, P> phr;
            {
                Z a = mk<T>(T(1), T(0)), b = mk<T>(T(1), T(0));
                const Z ea = mk<T>((T)ear, (T)eai), eb = mk<T>(ebr, ebi);
#pragma unroll
                for (int m = 0; m <= P; ++m) {
                    if (PH_REGS) {
                        phr.a[m] = a;
                        phr.b[m] = b;
                    } else {
                        pha[ROTW_LD * m] = a;
                        phb[ROTW_LD * m] = b;
                    }
                    a = zmul(a, ea);
                    b = zmul(b, eb);
                }
            }
            T sa, sb;  // per-degree scale factors of the axial kernel
            if (SCALED) {
                sa = (T)((double)scale[src] * iR);
                sb = (T)((double)scale[c] * iR);
            } else {
                sa = (T)iR;
                sb = (T)iR;
            }
            const Z* ms = mom + (size_t)src * (FULL_LAYOUT ? DIM : half_stride(P));
            const T cap = SCALED ? T(1e30) : T(INFINITY);
            if constexpr (AXR) {
                RegOut<T, H> b;
                rotw_back<T, P, FULL_LAYOUT>(ms, phr, b, sa, cap);
                axfwd_all<T, P, H>(b, col, phr, sb, cap, std::make_integer_sequence<int, P + 1>{});
            } else if constexpr (PH_REGS) {
                ColOut<T> out{col};
                rotw_back<T, P, FULL_LAYOUT>(ms, phr, out, sa, cap);
                rotw_axial<T, P>(col, sb, cap);
                rotw_fwd<T, P>(col, phr);
            } else {
                rotw_back_ni<T, P, FULL_LAYOUT>(ms, pha, phb, col, sa, cap);
                rotw_axial_ni<T, P>(col, sb, cap);
                rotw_fwd_ni<T, P>(col, pha, phb);
            }
        }
        __syncwarp();
        // ---- 4) destination sum over the chunk's lanes, fixed order
#pragma unroll
        for (int t = 0; t < NA; ++t) {
            const int e = lane + 32 * t;
            if (e < H) {
                T sr = T(0), si = T(0);
                const Z* row = sbuf + ROTW_LD * e;
                for (int l = 0; l < nact; ++l) {
                    sr += row[l].re;
                    si += row[l].im;
                }
                acc_re[t] += sr;
                acc_im[t] += si;
            }
        }
        __syncwarp();
    }
    // write the destination's local expansion
#pragma unroll
    for (int t = 0; t < NA; ++t) {
        const int e = lane + 32 * t;
        if (e < H) {
            int n = 0;
            while ((n + 1) * (n + 2) / 2 <= e) ++n;
            const int m = e - n * (n + 1) / 2;
            if (FULL_LAYOUT) {
                cplx<T>* out = loc + (size_t)c * DIM;
                out[n * (n + 1) + m] = mk<T>(acc_re[t], acc_im[t]);
                if (m > 0) {
                    const T sg = (m & 1) ? T(-1) : T(1);
                    out[n * (n + 1) - m] = mk<T>(sg * acc_re[t], -sg * acc_im[t]);
                }
            } else {
                loc[(size_t)c * half_stride(P) + e] = mk<T>(acc_re[t], acc_im[t]);
            }
        }
    }
}

template <typename T, int P>
constexpr size_t rotw_smem_per_warp() {
    return (size_t)ROTW_LD * ((P + 1) * (P + 2) / 2 + (sizeof(T) == 4 ? 0 : 2 * (P + 1))) * sizeof(cplx<T>);
}

// One warp per block. With a work counter the warps are persistent and pull
// destination cells from it; without one (work == nullptr) block b handles
// destination cell b, so every block is short-lived and the block scheduler can
// interleave kernels of higher-priority streams between them.
template <typename T, int P, bool SCALED, bool FULL_LAYOUT>
__global__ void __launch_bounds__(32) k_m2l_rotw(DirList L, int ncells, CellsView cv, const T* __restrict__ scale,
                                                const cplx<T>* __restrict__ mom, cplx<T>* __restrict__ loc,
                                                int* __restrict__ work) {
    extern __shared__ unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    cplx<T>* sbuf = reinterpret_cast<cplx<T>*>(smem_raw) + (size_t)wib * (rotw_smem_per_warp<T, P>() / sizeof(cplx<T>));
    if (!work) {
        const int c = blockIdx.x;
        if (c >= ncells) return;
        const uint32_t beg = L.seg_begin[c], end = L.seg_end[c];
        if (beg < end) rotw_body<T, P, SCALED, FULL_LAYOUT>(c, beg, end, L, cv, scale, mom, loc, sbuf, lane);
        return;
    }
    for (;;) {
        int c = 0;
        if (lane == 0) c = atomicAdd(work, 1);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= ncells) break;
        const uint32_t beg = L.seg_begin[c], end = L.seg_end[c];
        if (beg >= end) continue;
        rotw_body<T, P, SCALED, FULL_LAYOUT>(c, beg, end, L, cv, scale, mom, loc, sbuf, lane);
    }
}


}  // namespace fmmx
