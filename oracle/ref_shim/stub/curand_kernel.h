/* Test infrastructure (oracle only).
 *
 * Stand-in for the cuRAND device header when the reference's kernel header
 * (src/particles_kernel.cuh) is compiled as plain host C++.  Only the scene
 * initialisation kernels (createRectanglesD, particles_kernel.cuh:43-74) use
 * cuRAND, and the oracle harness never calls them; these declarations only
 * let the header compile.
 */
#ifndef DEMSO_ORACLE_CURAND_STUB_H
#define DEMSO_ORACLE_CURAND_STUB_H
struct curandState { unsigned long long s; };
static inline void curand_init(unsigned long long, unsigned long long,
                               unsigned long long, curandState* st) { st->s = 0; }
static inline float curand_normal(curandState*) { return 0.0f; }
#endif
