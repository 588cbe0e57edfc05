// Photon-recoil kicks shared by the trajectory kernels: Philox4x32-10
// counters keyed by the run's seed, indexed by (particle, absolute step), so a
// run split at any step and resumed draws the same numbers.
#pragma once
#include "common.cuh"

namespace {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): 10 rounds of
// (hi(M0 c0) ^ c1 ^ k0, lo(M1 c2), hi(M1 c2) ^ c3 ^ k1, lo(M0 c0)) with Weyl key bumps.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
    const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int i = 0; i < 10; i++) {
        const unsigned hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        const unsigned hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += W0;
        k.y += W1;
    }
    return c;
}

__device__ __forceinline__ double u01(unsigned x) { return ((double)x + 0.5) * 2.3283064365386963e-10; }

// Recoil kick of one step: N ~ Poisson(lam) events by sequential inversion
// of one uniform draw, then 2N isotropic unit vectors (absorption and
// emission) times v_rec, from the Philox counters (particle, step, draw, 0).
__device__ int recoil_kick(unsigned long long seed, unsigned particle, unsigned step, double lam,
                           double v_rec, double kick[3])
{
    const uint2 key = make_uint2((unsigned)(seed & 0xffffffffu), (unsigned)(seed >> 32));
    const uint4 u0 = philox4x32_10(make_uint4(particle, step, 0u, 0u), key);
    const double u = u01(u0.x);
    double p = exp(-lam), F = p;
    int n = 0;
    while (u > F && n < 256) {
        n++;
        p *= lam / n;
        F += p;
    }
    kick[0] = kick[1] = kick[2] = 0.0;
    for (int i = 0; i < 2 * n; i += 2) {
        const uint4 w = philox4x32_10(make_uint4(particle, step, 1u + (unsigned)(i / 2), 0u), key);
        const double a[2] = {u01(w.x), u01(w.z)}, b[2] = {u01(w.y), u01(w.w)};
        for (int h = 0; h < 2; h++) {
            const double cz = 2.0 * a[h] - 1.0, phi = 2.0 * MM_PI * b[h];
            const double sp = sqrt(fmax(0.0, 1.0 - cz * cz));
            kick[0] += v_rec * (sp * cos(phi));
            kick[1] += v_rec * (sp * sin(phi));
            kick[2] += v_rec * cz;
        }
    }
    return n;
}

}  // namespace
