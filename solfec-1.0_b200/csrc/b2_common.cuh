// b2_common.cuh -- shared device definitions of the B200 contact-solve path.
//
// Conventions (kept from the reference so results compare entry by entry):
//  * 3x3 matrices are column-major, A[3*j+i] = A(i,j) (alg.h:948-953);
//  * the local frame of a contact is [t1 t2 n] with the normal third
//    (dom.c:133-151), so U[2] / R[2] are normal components;
//  * MIN/MAX are the reference's ternaries (alg.h:44-48), not fmin/fmax, so
//    NaN propagation matches.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define B2_MIN(v, w) ((v) < (w) ? (v) : (w))
#define B2_MAX(v, w) ((v) > (w) ? (v) : (w))

namespace b2 {

constexpr int kWarp = 32;

// Diagonal solver kinds (dbs.h:27-33) and failure actions (bgs.h:39-44).
enum { DS_PROJECTED_GRADIENT = 0, DS_DE_SAXCE_FENG = 1, DS_SEMISMOOTH_NEWTON = 2, DS_PROJECTED_NEWTON = 3 };
enum { FAIL_CONTINUE = 0, FAIL_EXIT = 1, FAIL_CALLBACK = 2 };

// D = C + A*b (NVADDMUL, alg.h:948-953)
__device__ __forceinline__ void nvaddmul(const double* C, const double* A, const double* b, double* D) {
  double d0 = C[0] + (A[0] * b[0] + A[3] * b[1] + A[6] * b[2]);
  double d1 = C[1] + (A[1] * b[0] + A[4] * b[1] + A[7] * b[2]);
  double d2 = C[2] + (A[2] * b[0] + A[5] * b[1] + A[8] * b[2]);
  D[0] = d0; D[1] = d1; D[2] = d2;
}

__device__ __forceinline__ double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Counter-based priority of row i for the Jones-Plassmann colouring:
// splitmix64 finaliser of (seed + golden * (i+1)), high 32 bits, with the row
// index in the low 32 bits so priorities are unique. The host colouring in the
// test oracle uses the same definition.
// Priority of row i in the list-order mode: rows earlier in the list win, so
// Jones-Plassmann reproduces the sequential greedy colouring in list order.
__host__ __device__ __forceinline__ uint64_t jp_list_priority(int i) { return ~(uint64_t)(uint32_t)i; }

__host__ __device__ __forceinline__ uint64_t jp_priority(uint64_t seed, int i) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * ((uint64_t)i + 1ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (z & 0xFFFFFFFF00000000ull) | (uint64_t)(uint32_t)i;
}

}  // namespace b2
