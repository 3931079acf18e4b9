// integrate.cuh -- device steps of MD and Monte Carlo walkers, shared by the
// server (server.cu) and resident plans (plan.cu).
//
// Velocity Verlet with momenta as in the reference's MD example
// (src/potentials/hdnnpExample.f90:61-64):
//   x += p/m dt + F/(2m) dt^2 ; F_prev = F ; evaluate F ; p += dt/2 (F + F_prev)
// Monte Carlo trial moves displace every coordinate by N(0, sigma).
#pragma once

#include <cuda_runtime.h>

namespace hdnnp {

// Internal linkage (static): each translation unit that includes this header
// gets its own copy.

// SplitMix64 finaliser (Steele, Lea, Flood, OOPSLA 2014): counter-based draws.
static __device__ __host__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Trial move: keep pos and force, pos += sigma * N(0,1) per coordinate
// (Box-Muller transform of two 53-bit uniforms drawn from (key, coordinate)).
static __global__ void k_mc_trial(double* __restrict__ pos, double* __restrict__ pos_keep, const double* __restrict__ force,
                           double* __restrict__ force_keep, int n3, double sigma, unsigned long long key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const double x = pos[i];
    pos_keep[i] = x;
    force_keep[i] = force[i];
    const unsigned long long a = mix64(key + 2ull * (unsigned long long)i);
    const unsigned long long b = mix64(key + 2ull * (unsigned long long)i + 1ull);
    const double u1 = ((double)(a >> 11) + 1.0) * (1.0 / 9007199254740992.0);  // (0, 1]
    const double u2 = (double)(b >> 11) * (1.0 / 9007199254740992.0);          // [0, 1)
    pos[i] = x + sigma * sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

static __global__ void k_mc_reject(double* __restrict__ pos, const double* __restrict__ pos_keep, double* __restrict__ force,
                            const double* __restrict__ force_keep, int n3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    pos[i] = pos_keep[i];
    force[i] = force_keep[i];
}

// Velocity Verlet, first half: x += p/m dt + F/(2m) dt^2, keep F as F_prev.
static __global__ void k_md_drift(double* __restrict__ pos, const double* __restrict__ mom, const double* __restrict__ mass,
                           const double* __restrict__ force, double* __restrict__ force_prev, int n3, double dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const double m = mass[i / 3];
    pos[i] += mom[i] / m * dt + 0.5 * force[i] / m * dt * dt;
    force_prev[i] = force[i];
}

// Second half: p += dt/2 (F_new + F_prev); F = F_new (f_new may alias force).
static __global__ void k_md_kick(double* __restrict__ mom, const double* f_new, const double* __restrict__ force_prev,
                          double* force, int n3, double dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const double f = f_new[i];
    mom[i] += 0.5 * dt * (f + force_prev[i]);
    force[i] = f;
}

}  // namespace hdnnp
