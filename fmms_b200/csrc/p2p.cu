// P2P: direct near-field interactions over the directed leaf list.
//
// One CTA per target leaf. The leaf's source leaves (its own included) are
// streamed through shared memory in tiles of bodies; each target body is held
// by R = BLOCK / targets threads that split the tile's bodies and are reduced
// in a fixed order at the end, so results are deterministic and every thread
// works even for small leaves. A target skips its own slot (the i != j of the
// reference's self kernel, p2p.rs:13-46).
//
// Interaction (p2p.rs:24-39, with optional Plummer softening s^2):
//   d = x_j - x_i, r2 = |d|^2 + s^2, inv = 1/sqrt(r2),
//   a_i += m_j inv^3 d, pot_i += m_j inv.
#include "common.cuh"
#include "kernels.h"

namespace fmmx {

#define P2P_BLOCK 128
#define P2P_TILE 128
#define P2P_SRC_CHUNK 256

__global__ void __launch_bounds__(P2P_BLOCK) k_p2p_f64(DirList L, int ncells, CellsView cv,
                                                      const double* __restrict__ x, const double* __restrict__ y,
                                                      const double* __restrict__ z, const double* __restrict__ m,
                                                      double soft2, double* __restrict__ ax, double* __restrict__ ay,
                                                      double* __restrict__ az, double* __restrict__ pot) {
    __shared__ double tx[P2P_TILE], ty[P2P_TILE], tz[P2P_TILE], tm[P2P_TILE];
    __shared__ uint32_t tslot[P2P_TILE];
    __shared__ uint32_t pre[P2P_SRC_CHUNK + 1];
    __shared__ uint32_t sfirst[P2P_SRC_CHUNK];
    __shared__ double red[4][P2P_BLOCK];
    const int tid = threadIdx.x;
    for (int c = blockIdx.x; c < ncells; c += gridDim.x) {
        const uint32_t beg = L.seg_begin[c], end = L.seg_end[c];
        if (beg >= end) continue;
        const uint32_t tf = cv.first[c], tn = cv.count[c];
        for (uint32_t t0 = 0; t0 < tn; t0 += P2P_BLOCK) {
            const int nt = (int)min((uint32_t)P2P_BLOCK, tn - t0);
            const int R = P2P_BLOCK / nt;
            const int it = tid % nt, rep = tid / nt;
            const bool active = rep < R;
            const uint32_t islot = tf + t0 + it;
            double xi = 0, yi = 0, zi = 0;
            if (active) {
                xi = x[islot];
                yi = y[islot];
                zi = z[islot];
            }
            double sax = 0.0, say = 0.0, saz = 0.0, sp = 0.0;
            for (uint32_t sc = beg; sc < end; sc += P2P_SRC_CHUNK) {
                const int ns = (int)min((uint32_t)P2P_SRC_CHUNK, end - sc);
                __syncthreads();
                // exclusive prefix of the chunk's source leaf sizes
                for (int q = tid; q < ns; q += P2P_BLOCK) {
                    const int src = (int)L.src(L.key(sc + q));
                    pre[q + 1] = cv.count[src];
                    sfirst[q] = cv.first[src];
                }
                if (tid == 0) pre[0] = 0;
                __syncthreads();
                if (tid == 0)
                    for (int q = 1; q <= ns; ++q) pre[q] += pre[q - 1];
                __syncthreads();
                const uint32_t total = pre[ns];
                for (uint32_t b0 = 0; b0 < total; b0 += P2P_TILE) {
                    const uint32_t nb = min((uint32_t)P2P_TILE, total - b0);
                    if ((uint32_t)tid < nb) {
                        const uint32_t g = b0 + tid;
                        int lo = 0, hi = ns;  // last q with pre[q] <= g
                        while (hi - lo > 1) {
                            int mid = (lo + hi) >> 1;
                            if (pre[mid] <= g) lo = mid;
                            else hi = mid;
                        }
                        const uint32_t slot = sfirst[lo] + (g - pre[lo]);
                        tx[tid] = x[slot];
                        ty[tid] = y[slot];
                        tz[tid] = z[slot];
                        tm[tid] = m[slot];
                        tslot[tid] = slot;
                    }
                    __syncthreads();
                    if (active) {
                        for (uint32_t j = rep; j < nb; j += R) {
                            if (tslot[j] == islot) continue;
                            const double dx = tx[j] - xi, dy = ty[j] - yi, dz = tz[j] - zi;
                            const double r2 = dx * dx + dy * dy + dz * dz + soft2;
                            const double inv = rsqrt(r2);
                            const double mj = tm[j];
                            const double inv3 = inv * inv * inv;
                            const double f = mj * inv3;
                            sax += f * dx;
                            say += f * dy;
                            saz += f * dz;
                            sp += mj * inv;
                        }
                    }
                    __syncthreads();
                }
            }
            red[0][tid] = sax;
            red[1][tid] = say;
            red[2][tid] = saz;
            red[3][tid] = sp;
            __syncthreads();
            if (tid < nt) {
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                for (int r = 0; r < R; ++r) {
                    const int q = r * nt + tid;
                    s0 += red[0][q];
                    s1 += red[1][q];
                    s2 += red[2][q];
                    s3 += red[3][q];
                }
                const uint32_t slot = tf + t0 + tid;
                ax[slot] = s0;
                ay[slot] = s1;
                az[slot] = s2;
                pot[slot] = s3;
            }
            __syncthreads();
        }
    }
}

}  // namespace fmmx
