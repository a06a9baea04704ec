// synth.cpp -- deterministic synthetic path vertices and training targets (host).
//
// Stands in for the wavefront queues the reference's OptiX closest-hit program fills
// (src/render/nrrs/device.cu:87-110); the reference scenes are not used. Every vertex draws a
// fixed number of 64-bit words from std::mt19937_64, so vertex i has the same values whichever
// range is generated. Vertices are generated in blocks of 65536 with one engine per block,
// seeded from splitmix64(seed, block), so blocks run in parallel.
//   pos      U[0,1)^3                        wi, normal  normalised Gaussian triples
//   roughness U[0,1)    albedo U[0,1)^3      thp         exp(-1 + z) per channel
//   depth    floor(6u)  rnd U[0,1)           ref_mean    exp(-1 + z)
//   target   exp(0 + 2z) per channel, times 100 on all channels with probability 0.01
// u = (word >> 11) * 2^-53; z = sqrt(-2 ln(1-u1)) cos(2 pi u2) (one Box-Muller draw).
#include <cmath>
#include <cstdint>
#include <random>

#include "../../include/nrrs.h"

namespace {

constexpr uint64_t kBlock = 65536;

uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct Draw {
    std::mt19937_64 e;
    double u() { return (double)(e() >> 11) * (1.0 / 9007199254740992.0); }
    double z() {
        const double u1 = u(), u2 = u();
        return std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(6.283185307179586 * u2);
    }
};

void unit3(Draw& d, float* o) {
    double x = d.z(), y = d.z(), z = d.z();
    double n = std::sqrt(x * x + y * y + z * z);
    if (n < 1e-300) { x = 0; y = 0; z = 1; n = 1; }
    o[0] = (float)(x / n);
    o[1] = (float)(y / n);
    o[2] = (float)(z / n);
}

}  // namespace

extern "C" void nrrs_synth_vertices(uint64_t seed, uint64_t first, uint64_t n, float* pos,
                                    float* wi, float* normal, float* roughness, float* albedo,
                                    float* thp, uint32_t* depth, float* rnd, float* ref_mean,
                                    float* target) {
    if (n == 0) return;
    const uint64_t b0 = first / kBlock, b1 = (first + n - 1) / kBlock;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t bb = (int64_t)b0; bb <= (int64_t)b1; ++bb) {
        const uint64_t b = (uint64_t)bb;
        Draw d{std::mt19937_64(splitmix64(seed ^ splitmix64(b + 1)))};
        const uint64_t start = b * kBlock;
        const uint64_t lo = first > start ? first : start;
        const uint64_t hi_all = first + n;
        const uint64_t hi = hi_all < start + kBlock ? hi_all : start + kBlock;
        for (uint64_t g = start; g < hi; ++g) {
            float p[3], w[3], nm[3], a[3], t[3], tg[3];
            for (int k = 0; k < 3; ++k) p[k] = (float)d.u();
            unit3(d, w);
            unit3(d, nm);
            const float r = (float)d.u();
            for (int k = 0; k < 3; ++k) a[k] = (float)d.u();
            for (int k = 0; k < 3; ++k) t[k] = (float)std::exp(-1.0 + d.z());
            const uint32_t dep = (uint32_t)std::floor(d.u() * 6.0);
            const float rn = (float)d.u();
            const float rm = (float)std::exp(-1.0 + d.z());
            for (int k = 0; k < 3; ++k) tg[k] = (float)std::exp(0.0 + 2.0 * d.z());
            const bool firefly = d.u() < 0.01;
            if (firefly)
                for (int k = 0; k < 3; ++k) tg[k] *= 100.0f;
            if (g < lo) continue;
            const uint64_t i = g - first;
            if (pos) for (int k = 0; k < 3; ++k) pos[3 * i + k] = p[k];
            if (wi) for (int k = 0; k < 3; ++k) wi[3 * i + k] = w[k];
            if (normal) for (int k = 0; k < 3; ++k) normal[3 * i + k] = nm[k];
            if (roughness) roughness[i] = r;
            if (albedo) for (int k = 0; k < 3; ++k) albedo[3 * i + k] = a[k];
            if (thp) for (int k = 0; k < 3; ++k) thp[3 * i + k] = t[k];
            if (depth) depth[i] = dep > 5 ? 5 : dep;
            if (rnd) rnd[i] = rn < 1.0f ? rn : 0.99999994f;
            if (ref_mean) ref_mean[i] = rm;
            if (target) for (int k = 0; k < 3; ++k) target[3 * i + k] = tg[k];
        }
    }
}
