// Seeded input generators (host side).
//
// fmmx_gen_plummer and fmmx_gen_hernquist reproduce the reference samplers
// models::plummer and models::hernquist (crates/fmm/src/models.rs:35-82) bit
// for bit: the same SplitMix64 stream (models.rs:13-31), the same draw order
// and the same libm calls.
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/fmmx.h"

namespace {
struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ULL;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double unit() { return (double)(next() >> 11) / (double)(1ULL << 53); }
};
}  // namespace

extern "C" {

void fmmx_gen_plummer(size_t n, double cx, double cy, double cz, uint64_t seed, double* mass, double* pos) {
    SplitMix64 rng(seed);
    const double m = 1.0 / (double)n;
    for (size_t i = 0; i < n; ++i) {
        const double u = rng.unit();
        const double w = std::pow(u, 2.0 / 3.0);
        const double r = std::sqrt(w / (1.0 - w));
        const double z = 2.0 * rng.unit() - 1.0;
        const double phi = 2.0 * M_PI * rng.unit();
        const double s = std::sqrt(1.0 - z * z);
        mass[i] = m;
        pos[3 * i] = cx + r * s * std::cos(phi);
        pos[3 * i + 1] = cy + r * s * std::sin(phi);
        pos[3 * i + 2] = cz + r * z;
    }
}

void fmmx_gen_hernquist(size_t n, double cx, double cy, double cz, uint64_t seed, double* mass, double* pos) {
    SplitMix64 rng(seed);
    const double m = 1.0 / (double)n;
    for (size_t i = 0; i < n; ++i) {
        const double s = std::sqrt(rng.unit());
        const double r = s / (1.0 - s);
        const double z = 2.0 * rng.unit() - 1.0;
        const double phi = 2.0 * M_PI * rng.unit();
        const double sp = std::sqrt(1.0 - z * z);
        mass[i] = m;
        pos[3 * i] = cx + r * sp * std::cos(phi);
        pos[3 * i + 1] = cy + r * sp * std::sin(phi);
        pos[3 * i + 2] = cz + r * z;
    }
}

// ---------------------------------------------------------------------------
// Generators of the benchmark workloads (extensions; no reference
// counterpart). All draw from the same SplitMix64 stream.

// Standard normal by Box-Muller, as the reference's energy test does
// (crates/fmm/tests/energy_gate.rs:31-35).
static double gaussian(SplitMix64& r) {
    double u1 = r.unit();
    if (u1 < 1e-15) u1 = 1e-15;
    const double u2 = r.unit();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
}

// Plummer sphere of total mass mtot and scale radius a, truncated at r <= rmax*a
// (rejection-resampled), centred at c, with isotropic velocities from the
// Plummer distribution function (Aarseth, Henon & Wielen 1974: q by rejection
// from g(q) = q^2 (1-q^2)^{7/2}, v = q v_esc, v_esc = sqrt(2 G M / sqrt(r^2+a^2))).
static void plummer_ic(SplitMix64& rng, size_t n, double mtot, double a, double rmax, const double c[3],
                       double* mass, double* pos, double* vel) {
    const double m = mtot / (double)n;
    for (size_t i = 0; i < n; ++i) {
        double r;
        do {
            const double u = rng.unit();
            const double w = std::pow(u, 2.0 / 3.0);
            r = std::sqrt(w / (1.0 - w));
        } while (!(r <= rmax));
        const double z = 2.0 * rng.unit() - 1.0;
        const double phi = 2.0 * M_PI * rng.unit();
        const double s = std::sqrt(1.0 - z * z);
        mass[i] = m;
        pos[3 * i] = c[0] + a * r * s * std::cos(phi);
        pos[3 * i + 1] = c[1] + a * r * s * std::sin(phi);
        pos[3 * i + 2] = c[2] + a * r * z;
        if (vel) {
            double q, g;
            do {
                q = rng.unit();
                g = 0.1 * rng.unit();
            } while (g > q * q * std::pow(1.0 - q * q, 3.5));
            const double vesc = std::sqrt(2.0 * mtot / (a * std::sqrt(1.0 + r * r)));
            const double v = q * vesc;
            const double vz = 2.0 * rng.unit() - 1.0;
            const double vphi = 2.0 * M_PI * rng.unit();
            const double vs = std::sqrt(1.0 - vz * vz);
            vel[3 * i] = v * vs * std::cos(vphi);
            vel[3 * i + 1] = v * vs * std::sin(vphi);
            vel[3 * i + 2] = v * vz;
        }
    }
}

void fmmx_gen_plummer_ic(size_t n, double mtot, double a, double rmax, uint64_t seed, double* mass, double* pos,
                         double* vel) {
    SplitMix64 rng(seed);
    const double c[3] = {0.0, 0.0, 0.0};
    plummer_ic(rng, n, mtot, a, rmax, c, mass, pos, vel);
}

// Uniform in the unit cube, masses exp(N(0, sigma^2)) normalised to sum 1.
void fmmx_gen_uniform_lognormal(size_t n, double sigma, uint64_t seed, double* mass, double* pos) {
    SplitMix64 rng(seed);
    double tot = 0.0;
    for (size_t i = 0; i < n; ++i) {
        pos[3 * i] = rng.unit();
        pos[3 * i + 1] = rng.unit();
        pos[3 * i + 2] = rng.unit();
        mass[i] = std::exp(sigma * gaussian(rng));
        tot += mass[i];
    }
    for (size_t i = 0; i < n; ++i) mass[i] /= tot;
}

// nclust Plummer spheres (truncated at 20 scale radii) with scale radii
// log-uniform in [amin, amax], centres uniform in the unit cube and sizes a
// Dirichlet(1) split of n (normalised Exp(1) draws, rounded to sum n); equal
// masses summing to 1; Plummer-DF velocities of each sphere when vel != NULL.
void fmmx_gen_clusters(size_t n, int nclust, double amin, double amax, uint64_t seed, double* mass, double* pos,
                       double* vel) {
    SplitMix64 rng(seed);
    std::vector<double> e(nclust), a(nclust), cen(3 * (size_t)nclust);
    double tot = 0.0;
    for (int k = 0; k < nclust; ++k) {
        e[k] = -std::log(1.0 - rng.unit());
        tot += e[k];
        a[k] = amin * std::exp(std::log(amax / amin) * rng.unit());
        for (int d = 0; d < 3; ++d) cen[3 * k + d] = rng.unit();
    }
    std::vector<size_t> cnt(nclust);
    size_t used = 0;
    for (int k = 0; k < nclust; ++k) {
        cnt[k] = (size_t)std::floor((double)n * e[k] / tot);
        used += cnt[k];
    }
    for (size_t r = 0; used < n; ++r, ++used) cnt[r % nclust]++;  // remainder, round robin
    const double mb = 1.0 / (double)n;
    size_t off = 0;
    for (int k = 0; k < nclust; ++k) {
        if (cnt[k] == 0) continue;
        plummer_ic(rng, cnt[k], mb * (double)cnt[k], a[k], 20.0, &cen[3 * k], mass + off, pos + 3 * off,
                   vel ? vel + 3 * off : nullptr);
        off += cnt[k];
    }
}

}  // extern "C"
