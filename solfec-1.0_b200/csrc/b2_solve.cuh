// b2_solve.cuh -- colour-by-colour block Gauss-Seidel with the merit pass fused
// into the next sweep.
//
// Reference loop (bgs.c:913-1069): every iteration sweeps the rows in list
// order (each row: B' = B + sum_j W_ij R_j, diagonal solve, error sums), then
// MERIT_Function (mrf.c:35-185) recomputes U = B + W_ii R_i + sum_j W_ij R_j for
// every row and the merit; the loop stops when error <= epsilon and merit <=
// meritval, or at maxiter.
//
// Here the rows are stored sorted by colour (rows of one colour share no
// non-obstacle body, so W_ij = 0 inside a colour) and processed colour after
// colour, which is the reference loop run on the colour-permuted list. The
// merit of iterate s is evaluated inside sweep s+1: R is double-buffered, so
// while row i gathers R_j for its Gauss-Seidel sum (the new value for rows of
// colours already swept, the old one otherwise) it also gathers the old value
// of every neighbour and forms U_merit = B + W_ii R_i^s + sum_j W_ij R_j^s. The
// merit row term, the U handed to the diagonal solver (the reference starts
// iteration s+1 from the U the merit pass wrote) and the stopping decision for
// iterate s are therefore exactly the reference's, while W is streamed once per
// iteration instead of twice. The sweep after the final iterate is discarded;
// the final R and U are those of the iterate that met the rule.
#pragma once

#include <cuda_runtime.h>
#include "b2_common.cuh"
#include "b2_diag.cuh"

namespace b2 {

constexpr int kSolveThreads = 256;
constexpr int kSolveWarps = kSolveThreads / kWarp;
constexpr int kChunkUnroll = 4;           // 32-block chunks whose loads are issued together
constexpr uint64_t kBarrierLimitNs = 2000000000ull;  // 2 s per grid barrier wait

// Device-side control block of one solve launch (zeroed before launch).
struct SolveControl {
  unsigned bar_count;       // monotone arrival counter of the grid barrier
  int timeout;              // a barrier wait gave up (device error)
  int final_iter;           // launch-local index of the returned iterate
  int iters;                // iterations completed in this launch
  int thrown;               // FAILURE_EXIT raised
  int sweeps;               // sweeps executed (including the discarded one)
  double merit;             // merit of the returned iterate (0 with nomerit)
  double error;             // relative error of the returned iterate
  double merit_input;       // merit of the input iterate (merit mode)
};

struct SolveArgs {
  int n, ncolours;
  const int* colptr;        // [ncolours+1] colour offsets in sorted order
  const int* rowptr;        // [n+1]
  const int* col;           // [K] neighbour (sorted index)
  const double* W64;        // 9 planes of K doubles (plane stride kstride)
  const float* W32;         // 9 planes of K floats (mixed precision)
  long long kstride;
  const double* Wd;         // 9 planes of n: diagonal block W_ii
  const double* Ad;         // 9 planes of n: A = W_ii^-1
  const double* Bv;         // 3 planes of n: free velocity B
  const double* Vv;         // 3 planes of n: previous velocity V
  const double* rho;        // [n]
  const double* gap;        // [n]
  const double* fric;       // [n]
  const double* rest;       // [n]
  const double* coh;        // [n]
  double4* R64[2];          // double-buffered reactions
  float4* R32[2];           // float shadows (mixed precision)
  double4* Us;              // U state (input U; diagonal-solver output without merit)
  double4* Um;              // U of the merit pass (final U with merit)
  double* conmerit;         // per-row merit numerator of the last merit pass (may be null)
  double* part;             // [2][gridDim][4] per-block partial sums
  double* rerhist;          // global history arrays (indexed by iter0 + k)
  double* merhist;
  unsigned long long* failkey;  // per sweep: max (order position + 1) << 2 | kind of a diagonal failure
  unsigned* failcount;          // per sweep: number of diagonal failures
  SolveControl* ctrl;
  double epsilon, meritval, diagepsilon, step, merit_denom;
  int maxiter, diagmaxiter, diagsolver, failure, dynamic, reverse, nomerit;
  int iter0;                // global index of this launch's first iteration
  int in_parity;            // R64/R32 buffer holding the input iterate
  int u0_from_merit;        // sweep 0 hands the merit U (not Us) to the diagonal solver
  double* trace;            // per-row diagonal-solve record of one sweep (null: off)
  int trace_sweep;          // launch-local sweep whose rows are recorded
};

// trace record per row: B'[3], U in[3], R in[3], U out[3], R out[3], kind
constexpr int kTraceStride = 16;

__device__ __forceinline__ bool grid_barrier(SolveControl* ctrl, unsigned nblocks, unsigned& epoch) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    epoch++;
    __threadfence();
    atomicAdd(&ctrl->bar_count, 1u);
    const unsigned target = nblocks * epoch;
    volatile unsigned* cnt = &ctrl->bar_count;
    volatile int* to = &ctrl->timeout;
    uint64_t t0 = globaltimer_ns();
    while (*cnt < target) {
      if (*to) { ok = 0; break; }
      if (globaltimer_ns() - t0 > kBarrierLimitNs) { *to = 1; ok = 0; break; }
      __nanosleep(32);
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

template <typename T>
__device__ __forceinline__ T shfl_down(T v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }

// 32-byte load that bypasses L1 (the R buffers are rewritten by other SMs
// between grid barriers, so a line cached in L1 could be stale).
__device__ __forceinline__ double4 ldcg4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  const double2 lo = __ldcg(q), hi = __ldcg(q + 1);
  return make_double4(lo.x, lo.y, hi.x, hi.y);
}

// Per-sweep flags shared by the tile routine.
struct SweepFlags {
  bool gs;        // Gauss-Seidel update of this sweep (false: merit-only pass)
  bool merit;     // evaluate the merit of the input iterate
  bool u_merit;   // hand the merit U to the diagonal solver
  bool backward;  // colours in reverse order
};

// One tile of up to 32 consecutive rows of one colour, owned by one warp.
// Lanes stride over the tile's contiguous CSR range (lane per block, coalesced
// plane loads) and form the W_ij R_j products, which are staged in shared
// memory; lane r then adds the products of row r0 + r in list order onto its
// running sums, which start from B (Gauss-Seidel, bgs.c:957-963) and from
// B + W_ii R_i (merit U, mrf.c:61-68). Together with the build's disabled
// multiply-add contraction this reproduces the reference's NVADDMUL chains
// operation for operation in FP64. Lane r then solves its row (diagonal
// solve and merit term in FP64).
template <bool MIXED>
__device__ __forceinline__ void solve_tile(const SolveArgs& a, const SweepFlags& f, int r0, int nr, int cs, int ce,
                                           int s, int rin, int rout, void* stage_raw, int* tp, double& errup,
                                           double& errlo, double& mnum) {
  typedef typename std::conditional<MIXED, float, double>::type real;
  constexpr int kSlots = kWarp * kChunkUnroll;
  real(*stage)[kSlots] = reinterpret_cast<real(*)[kSlots]>(stage_raw);  // [6][kSlots]
  const int lane = threadIdx.x & (kWarp - 1);
  const int n = a.n;
  const bool own = lane < nr;
  const int p = r0 + lane;
  if (lane <= nr) tp[lane] = __ldg(a.rowptr + r0 + lane);
  if (lane == 0 && nr == kWarp) tp[kWarp] = __ldg(a.rowptr + r0 + kWarp);

  double B[3] = {0.0, 0.0, 0.0}, W[9], Rold[3] = {0.0, 0.0, 0.0}, ag[3], am[3] = {0.0, 0.0, 0.0};
  if (own) {
#pragma unroll
    for (int q = 0; q < 3; q++) B[q] = __ldg(a.Bv + (size_t)q * n + p);
    const double4 ro = ldcg4(a.R64[rin] + p);
    Rold[0] = ro.x; Rold[1] = ro.y; Rold[2] = ro.z;
#pragma unroll
    for (int q = 0; q < 9; q++) W[q] = __ldg(a.Wd + (size_t)q * n + p);
    if (f.merit) nvaddmul(B, W, Rold, am);
  }
  ag[0] = B[0]; ag[1] = B[1]; ag[2] = B[2];
  __syncwarp();
  const int kb = tp[0], ke = tp[nr];
  const int mb = own ? tp[lane] : 0, me = own ? tp[lane + 1] : 0;

  for (int base = kb; base < ke; base += kSlots) {
    int jj[kChunkUnroll];
    real w[kChunkUnroll][9];
#pragma unroll
    for (int u = 0; u < kChunkUnroll; u++) {
      const int k = base + u * kWarp + lane;
      jj[u] = k < ke ? __ldg(a.col + k) : -1;
    }
#pragma unroll
    for (int u = 0; u < kChunkUnroll; u++) {
      const int k = base + u * kWarp + lane;
#pragma unroll
      for (int q = 0; q < 9; q++) {
        if (k < ke) {
          if constexpr (MIXED) w[u][q] = __ldg(a.W32 + q * a.kstride + k);
          else w[u][q] = __ldg(a.W64 + q * a.kstride + k);
        } else {
          w[u][q] = real(0);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kChunkUnroll; u++) {
      const int j = jj[u];
      const int slot = u * kWarp + lane;
      if (j >= 0) {
        const bool earlier = f.backward ? (j >= ce) : (j < cs);
        real ro0, ro1, ro2;
        if constexpr (MIXED) {
          const float4 v = __ldcg(a.R32[rin] + j);
          ro0 = v.x; ro1 = v.y; ro2 = v.z;
        } else {
          const double4 v = ldcg4(a.R64[rin] + j);
          ro0 = v.x; ro1 = v.y; ro2 = v.z;
        }
        const real* Wk = w[u];
        real m0 = 0, m1 = 0, m2 = 0;
        if (f.merit) {
          m0 = Wk[0] * ro0 + Wk[3] * ro1 + Wk[6] * ro2;
          m1 = Wk[1] * ro0 + Wk[4] * ro1 + Wk[7] * ro2;
          m2 = Wk[2] * ro0 + Wk[5] * ro1 + Wk[8] * ro2;
          stage[3][slot] = m0; stage[4][slot] = m1; stage[5][slot] = m2;
        }
        if (f.gs) {
          real g0, g1, g2;
          if (earlier) {
            real rn0, rn1, rn2;
            if constexpr (MIXED) {
              const float4 v = __ldcg(a.R32[rout] + j);
              rn0 = v.x; rn1 = v.y; rn2 = v.z;
            } else {
              const double4 v = ldcg4(a.R64[rout] + j);
              rn0 = v.x; rn1 = v.y; rn2 = v.z;
            }
            g0 = Wk[0] * rn0 + Wk[3] * rn1 + Wk[6] * rn2;
            g1 = Wk[1] * rn0 + Wk[4] * rn1 + Wk[7] * rn2;
            g2 = Wk[2] * rn0 + Wk[5] * rn1 + Wk[8] * rn2;
          } else if (f.merit) {
            g0 = m0; g1 = m1; g2 = m2;
          } else {
            g0 = Wk[0] * ro0 + Wk[3] * ro1 + Wk[6] * ro2;
            g1 = Wk[1] * ro0 + Wk[4] * ro1 + Wk[7] * ro2;
            g2 = Wk[2] * ro0 + Wk[5] * ro1 + Wk[8] * ro2;
          }
          stage[0][slot] = g0; stage[1][slot] = g1; stage[2][slot] = g2;
        }
      }
    }
    __syncwarp();
    // each row adds its own products, in list order
    const int lo = mb > base ? mb : base;
    const int hi = me < base + kSlots ? me : base + kSlots;
    for (int k = lo; k < hi; k++) {
      const int slot = k - base;
      if (f.gs) {
        ag[0] = ag[0] + (double)stage[0][slot];
        ag[1] = ag[1] + (double)stage[1][slot];
        ag[2] = ag[2] + (double)stage[2][slot];
      }
      if (f.merit) {
        am[0] = am[0] + (double)stage[3][slot];
        am[1] = am[1] + (double)stage[4][slot];
        am[2] = am[2] + (double)stage[5][slot];
      }
    }
    __syncwarp();
  }

  // ---- lane per row: merit term and diagonal solve
  if (own) {
    ContactParams cp;
    cp.friction = __ldg(a.fric + p);
    cp.restitution = __ldg(a.rest + p);
    cp.cohesion = __ldg(a.coh + p);
    cp.gap = __ldg(a.gap + p);
    cp.step = a.step;
    cp.dynamic = a.dynamic;
    double V[3];
#pragma unroll
    for (int q = 0; q < 3; q++) V[q] = __ldg(a.Vv + (size_t)q * n + p);
    if (f.merit) {
      double A[9];
#pragma unroll
      for (int q = 0; q < 9; q++) A[q] = __ldg(a.Ad + (size_t)q * n + p);
      const double up = merit_row(cp, A, V, am, Rold);
      mnum += up;
      a.Um[p] = make_double4(am[0], am[1], am[2], 0.0);
      if (a.conmerit) a.conmerit[p] = up;
    }
    if (f.gs) {
      double R[3] = {Rold[0], Rold[1], Rold[2]};
      double U[3];
      if (f.u_merit) { U[0] = am[0]; U[1] = am[1]; U[2] = am[2]; }
      else { const double4 us = ldcg4(a.Us + p); U[0] = us.x; U[1] = us.y; U[2] = us.z; }
      double* tr = (a.trace && s == a.trace_sweep) ? a.trace + (size_t)kTraceStride * p : nullptr;
      if (tr) {
#pragma unroll
        for (int q = 0; q < 3; q++) { tr[q] = ag[q]; tr[3 + q] = U[q]; tr[6 + q] = R[q]; }
      }
      const int kind = diagonal_solve_row(a.diagsolver, a.failure, cp, a.diagepsilon, a.diagmaxiter, __ldg(a.rho + p),
                                          W, ag, V, U, R);
      if (tr) {
#pragma unroll
        for (int q = 0; q < 3; q++) { tr[9 + q] = U[q]; tr[12 + q] = R[q]; }
        tr[15] = (double)kind;
      }
      if (kind) {
        const unsigned long long pos = f.backward ? (unsigned long long)(n - 1 - p) : (unsigned long long)p;
        atomicMax(a.failkey + a.iter0 + s, ((pos + 1ull) << 2) | (unsigned long long)kind);
        atomicAdd(a.failcount + a.iter0 + s, 1u);
      }
      a.R64[rout][p] = make_double4(R[0], R[1], R[2], 0.0);
      if constexpr (MIXED) a.R32[rout][p] = make_float4((float)R[0], (float)R[1], (float)R[2], 0.f);
      if (a.nomerit) a.Us[p] = make_double4(U[0], U[1], U[2], 0.0);
      const double d0 = R[0] - Rold[0], d1 = R[1] - Rold[1], d2 = R[2] - Rold[2];
      errup += d0 * d0 + d1 * d1 + d2 * d2;
      errlo += R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
    }
  }
  __syncwarp();
}

// Deterministic block reduction of three per-thread values (fixed shuffle
// tree, then warps in order). Result valid in thread 0.
__device__ __forceinline__ void block_sum3(double& x, double& y, double& z, double (*red)[3]) {
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) {
    x += __shfl_down_sync(0xffffffffu, x, d);
    y += __shfl_down_sync(0xffffffffu, y, d);
    z += __shfl_down_sync(0xffffffffu, z, d);
  }
  const int warp = threadIdx.x / kWarp, lane = threadIdx.x & (kWarp - 1);
  if (lane == 0) { red[warp][0] = x; red[warp][1] = y; red[warp][2] = z; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sx = 0, sy = 0, sz = 0;
    for (int w = 0; w < (int)(blockDim.x / kWarp); w++) { sx += red[w][0]; sy += red[w][1]; sz += red[w][2]; }
    x = sx; y = sy; z = sz;
  }
}

// dynamic shared memory of k_solve: per warp 6 x (32 * kChunkUnroll) staged products
template <bool MIXED>
__host__ __device__ constexpr size_t solve_smem_bytes() {
  return (size_t)kSolveWarps * 6 * kWarp * kChunkUnroll * (MIXED ? sizeof(float) : sizeof(double));
}

template <bool MIXED>
__global__ void __launch_bounds__(kSolveThreads, 1) k_solve(SolveArgs a) {
  extern __shared__ __align__(16) unsigned char solve_smem[];
  __shared__ int tp[kSolveWarps][kWarp + 1];
  __shared__ double red[kSolveWarps][3];
  const int warp = threadIdx.x / kWarp;
  const int gwarp = blockIdx.x * kSolveWarps + warp;
  const int nwarps = gridDim.x * kSolveWarps;
  const unsigned nblocks = gridDim.x;
  unsigned epoch = 0;
  double prev_error = 0.0;
  const bool merit_mode = !a.nomerit;

  for (int s = 0;; s++) {
    SweepFlags f;
    f.gs = !(merit_mode && s == a.maxiter);
    f.merit = merit_mode;
    f.u_merit = merit_mode && (s >= 1 || a.u0_from_merit);
    f.backward = a.reverse && ((a.iter0 + s) & 1);
    const int rin = (a.in_parity + s) & 1;        // iterate s-1
    const int rout = (a.in_parity + s + 1) & 1;   // iterate s
    double errup = 0.0, errlo = 0.0, mnum = 0.0;

    for (int cc = 0; cc < a.ncolours; cc++) {
      const int c = f.backward ? a.ncolours - 1 - cc : cc;
      const int cs = __ldg(a.colptr + c), ce = __ldg(a.colptr + c + 1);
      const int ntiles = (ce - cs + kWarp - 1) / kWarp;
      for (int t = gwarp; t < ntiles; t += nwarps) {
        const int r0 = cs + t * kWarp;
        const int nr = min(kWarp, ce - r0);
        void* stage = solve_smem + (size_t)warp * (solve_smem_bytes<MIXED>() / kSolveWarps);
        solve_tile<MIXED>(a, f, r0, nr, cs, ce, s, rin, rout, stage, tp[warp], errup, errlo, mnum);
      }
      if (cc == a.ncolours - 1) {
        block_sum3(errup, errlo, mnum, red);
        if (threadIdx.x == 0) {
          double* pp = a.part + ((size_t)(s & 1) * nblocks + blockIdx.x) * 4;
          pp[0] = errup; pp[1] = errlo; pp[2] = mnum;
        }
      }
      if (!grid_barrier(a.ctrl, nblocks, epoch)) return;
    }
    if (a.ncolours == 0) {
      if (threadIdx.x == 0) {
        double* pp = a.part + ((size_t)(s & 1) * nblocks + blockIdx.x) * 4;
        pp[0] = pp[1] = pp[2] = 0.0;
      }
      if (!grid_barrier(a.ctrl, nblocks, epoch)) return;
    }

    // every block sums the partials in the same order and takes the same decision
    double su = 0.0, sl = 0.0, sm = 0.0;
    for (unsigned b = 0; b < nblocks; b++) {
      const double* pp = a.part + ((size_t)(s & 1) * nblocks + b) * 4;
      su += __ldcg(pp); sl += __ldcg(pp + 1); sm += __ldcg(pp + 2);
    }
    const double error = sqrt(su) / sqrt(sl == 0.0 ? 1.0 : sl);  // bgs.c:1028
    const double merit_prev = merit_mode ? (0.5 * sm) / a.merit_denom : 0.0;  // mrf.c:176-184
    const bool failed = __ldcg(a.failkey + a.iter0 + s) != 0ull;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    int final_iter = -2, thrown = 0;
    double final_merit = 0.0, final_error = 0.0;

    if (merit_mode) {
      if (s == 0 && lead) a.ctrl->merit_input = merit_prev;
      if (s >= 1) {
        if (lead) { a.rerhist[a.iter0 + s - 1] = prev_error; a.merhist[a.iter0 + s - 1] = merit_prev; }
        const bool meets = !(prev_error > a.epsilon || merit_prev > a.meritval);  // bgs.c:1036
        if (meets || s == a.maxiter) {
          final_iter = s - 1; final_merit = merit_prev; final_error = prev_error;
        } else if (f.gs && failed && a.failure == FAIL_EXIT) {
          final_iter = s; thrown = 1; final_merit = merit_prev; final_error = error;
        }
      } else if (f.gs && failed && a.failure == FAIL_EXIT) {
        final_iter = 0; thrown = 1; final_merit = 0.0; final_error = error;
      }
    } else {
      if (lead) { a.rerhist[a.iter0 + s] = error; a.merhist[a.iter0 + s] = 0.0; }
      if (failed && a.failure == FAIL_EXIT) {
        final_iter = s; thrown = 1; final_error = error;
      } else if (!(error > a.epsilon) || s + 1 >= a.maxiter) {
        final_iter = s; final_error = error;
      }
    }
    prev_error = error;
    if (final_iter >= -1) {
      if (lead) {
        a.ctrl->final_iter = final_iter;
        a.ctrl->iters = thrown ? final_iter : final_iter + 1;
        a.ctrl->thrown = thrown;
        a.ctrl->sweeps = s + 1;
        a.ctrl->merit = final_merit;
        a.ctrl->error = final_error;
      }
      return;
    }
  }
}

}  // namespace b2
