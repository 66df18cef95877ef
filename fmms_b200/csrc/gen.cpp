// Seeded input generators (host side).
//
// fmmx_gen_plummer and fmmx_gen_hernquist reproduce the reference samplers
// models::plummer and models::hernquist (crates/fmm/src/models.rs:35-82) bit
// for bit: the same SplitMix64 stream (models.rs:13-31), the same draw order
// and the same libm calls.
#include <cmath>
#include <cstdint>

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

}  // extern "C"
