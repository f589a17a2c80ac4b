// b2_colour.cuh -- contact-graph colouring and the colour-sorted layout.
//
// The reference sweeps rows in list order (bgs.c:950). Rows that share no
// non-obstacle body are uncoupled (W_ij = 0), so any colouring of the contact
// graph gives an order whose colours can be swept in parallel. The colouring
// is Jones-Plassmann with smallest-available colour: in every round each
// uncoloured row whose priority beats all uncoloured neighbours takes the
// smallest colour no coloured neighbour holds. Priorities come from
// jp_priority(seed, row) (seeded hash) or, in the list-order mode, from the
// row index (earlier rows win); either way the result equals the sequential
// greedy colouring in decreasing priority order and is reproducible bit for
// bit on the host. The list order needs more rounds (the longest chain of
// neighbours in increasing index) but, on meshes and lattices whose contacts
// are listed in geometric order, reaches the fewest colours (6 instead of 10
// on the hexahedra lattice, where the contact graph is the line graph of a
// bipartite graph of degree 6); on random piles both reach the same count.
#pragma once

#include <cuda_runtime.h>
#include "b2_common.cuh"
#include "b2_solve.cuh"

namespace b2 {

constexpr int kMaxColours = 256;

struct ColourControl {
  unsigned bar_count;
  int timeout;
  int overflow;      // more than kMaxColours colours needed
  int ncolours;
  int rounds;
  unsigned remaining[3];
};

__device__ __forceinline__ bool colour_barrier(ColourControl* ctrl, unsigned nblocks, unsigned& epoch) {
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

// Persistent cooperative Jones-Plassmann colouring of the graph (adjptr,
// adjcol). colour[] must be -1 on entry.
__global__ void k_jp_colour(int n, const int* adjptr, const int* adjcol, unsigned long long seed, int list_order,
                            int* colour, int* sel, ColourControl* ctrl) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthreads = gridDim.x * blockDim.x;
  const unsigned nblocks = gridDim.x;
  unsigned epoch = 0;
  for (int r = 0;; r++) {
    if (tid == 0) ctrl->remaining[(r + 1) % 3] = 0u;
    // phase 1: local maxima among uncoloured neighbours
    for (int i = tid; i < n; i += nthreads) {
      int s = 0;
      if (__ldcg(colour + i) < 0) {
        s = 1;
        const uint64_t pi = list_order ? jp_list_priority(i) : jp_priority(seed, i);
        for (int k = adjptr[i]; k < adjptr[i + 1]; k++) {
          const int j = adjcol[k];
          if (__ldcg(colour + j) < 0 && (list_order ? jp_list_priority(j) : jp_priority(seed, j)) > pi) { s = 0; break; }
        }
      }
      sel[i] = s;
    }
    if (!colour_barrier(ctrl, nblocks, epoch)) return;
    // phase 2: selected rows take the smallest colour unused by coloured neighbours
    unsigned left = 0;
    for (int i = tid; i < n; i += nthreads) {
      if (__ldcg(sel + i)) {
        unsigned long long used[kMaxColours / 64] = {0ull, 0ull, 0ull, 0ull};
        for (int k = adjptr[i]; k < adjptr[i + 1]; k++) {
          const int cj = __ldcg(colour + adjcol[k]);
          if (cj >= 0) used[cj >> 6] |= 1ull << (cj & 63);
        }
        int c = -1;
#pragma unroll
        for (int w = 0; w < kMaxColours / 64; w++) {
          if (c < 0 && ~used[w] != 0ull) c = w * 64 + __ffsll((long long)~used[w]) - 1;
        }
        if (c < 0) { atomicExch(&ctrl->overflow, 1); c = kMaxColours - 1; }
        colour[i] = c;
        atomicMax(&ctrl->ncolours, c + 1);
      } else if (__ldcg(colour + i) < 0) {
        left++;
      }
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) left += __shfl_down_sync(0xffffffffu, left, d);
    if ((threadIdx.x & 31) == 0 && left) atomicAdd(&ctrl->remaining[r % 3], left);
    if (!colour_barrier(ctrl, nblocks, epoch)) return;
    const unsigned rem = *(volatile unsigned*)&ctrl->remaining[r % 3];
    if (rem == 0u || *(volatile int*)&ctrl->overflow) {
      if (tid == 0) ctrl->rounds = r + 1;
      return;
    }
  }
}

// Sets *diff if the graph (adjptr[n+1], adjcol[K]) differs from the copy kept
// with the last colouring.
__global__ void k_graph_diff(int n, long long K, const int* adjptr, const int* adjcol, const int* pptr,
                             const int* pcol, int* diff) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  bool d = false;
  for (long long i = t; i <= n; i += stride) d |= adjptr[i] != pptr[i];
  for (long long k = t; k < K; k += stride) d |= adjcol[k] != pcol[k];
  if (__any_sync(0xffffffffu, d) && (threadIdx.x & 31) == 0) atomicExch(diff, 1);
}

// colour offsets from the colour-sorted keys
__global__ void k_colptr(int n, const int* sorted_colour, int ncolours, int* colptr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > n) return;
  const int cur = p < n ? sorted_colour[p] : ncolours;
  const int prev = p > 0 ? sorted_colour[p - 1] : -1;
  for (int c = prev + 1; c <= cur; c++) colptr[c] = p;
}

__global__ void k_inverse_perm(int n, const int* perm, int* iperm) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) iperm[perm[p]] = p;
}

__global__ void k_sorted_degree(int n, const int* perm, const int* adjptr, int* deg) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) { const int i = perm[p]; deg[p] = adjptr[i + 1] - adjptr[i]; }
}

// Off-diagonal blocks in the colour-sorted CSR computed from the row factors:
// W_ij = h H_i^b M_b^-1 H_j^b^T for j > i (ldy.c:738-794, serial form
// left = H_i, right = M^-1 H_j^T) and the transposed block of the pair for
// j < i (ldy.c:829-844); the transposed block is recomputed with identical
// operands and order, so it is bitwise the transpose. Thread per sorted
// block (coalesced plane writes); the block's sorted row by binary search in
// the sorted row offsets.
__global__ void k_offdiag_assembled(int n, long long K, const int* perm, const int* iperm, const int* adjptr,
                                    const int* adjcol, const int* adjbod, const int* master, const double* factors,
                                    double step, const int* rowptr, const int* brow, int* col, double* W64,
                                    float* W32, long long kstride) {
  const long long qo = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (qo >= K) return;
  int p;
  if (brow) {
    p = brow[qo];
  } else {
    int lo_r = 0, hi_r = n;  // rowptr[lo_r] <= qo < rowptr[hi_r]
    while (hi_r - lo_r > 1) {
      const int mid = (lo_r + hi_r) >> 1;
      if (rowptr[mid] <= qo) lo_r = mid; else hi_r = mid;
    }
    p = lo_r;
  }
  const int i = perm[p];
  const int t = (int)(qo - rowptr[p]);
  {
    const int kb = adjptr[i];
    const int j = adjcol[kb + t], b = adjbod[kb + t];
    const int lo = j > i ? i : j, hi = j > i ? j : i;
    const double* left = factors + (size_t)lo * kFactorStride + (master[lo] == b ? 0 : 36);
    const double* right = factors + (size_t)hi * kFactorStride + (master[hi] == b ? 18 : 54);
    double Lr[18], Pr[18], W[9];
#pragma unroll
    for (int q = 0; q < 18; q += 2) {
      const double2 l = ld2(left + q), p = ld2(right + q);
      Lr[q] = l.x; Lr[q + 1] = l.y; Pr[q] = p.x; Pr[q + 1] = p.y;
    }
#pragma unroll
    for (int q = 0; q < 9; q++) W[q] = 0.0;
    hp_add(Lr, Pr, W);
#pragma unroll
    for (int q = 0; q < 9; q++) W[q] *= step;
    col[qo] = iperm[j];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const double v = j > i ? W[3 * c + r] : W[3 * r + c];  // (r, c) of W_ij
        W64[(3 * c + r) * kstride + qo] = v;
        W32[(3 * c + r) * kstride + qo] = (float)v;
      }
  }
}

// Body-pair table of the off-diagonal blocks, built once per layout while
// the contact topology holds. Every non-obstacle body b with contacts
// c_0 < c_1 < ... < c_{d-1} (its ascending body list) couples each pair
// a < e: the block of row c_a, column c_e through b and its transpose
// (row c_e, column c_a). Row i lists its neighbours through its master body,
// then through its slave body, each ascending (k_adj_fill), so the pair's
// slot in row c_a is that row's offset of body b plus e - 1, and in row c_e
// its offset plus a. A record holds the two factor offsets (lo = c_a's H
// through b, hi = c_e's M^-1 H^T through b) and the two sorted slots.
__device__ __forceinline__ int pair_row_offset(int i, int b, const int* master, const int* obstacle,
                                               const int* bptr) {
  const int m = master[i];
  if (m == b) return 0;
  return (m >= 0 && !obstacle[m]) ? bptr[m + 1] - bptr[m] - 1 : 0;
}

__global__ void k_pair_count(int nbod, const int* obstacle, const int* bptr, long long* cnt) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbod) return;
  const long long d = obstacle[b] ? 0 : (long long)(bptr[b + 1] - bptr[b]);
  cnt[b] = d * (d - 1) / 2;
}

__global__ void k_pair_fill(int nbod, const int* obstacle, const int* master, const int* bptr, const int* brow,
                            const long long* pptr, const int* iperm, const int* rowptr, int4* rec) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbod || obstacle[b]) return;
  const int b0 = bptr[b], d = bptr[b + 1] - b0;
  long long k = pptr[b];
  for (int a = 0; a < d; a++) {
    const int i = brow[b0 + a];
    const int qi = rowptr[iperm[i]] + pair_row_offset(i, b, master, obstacle, bptr);
    const int fl = i * kFactorStride + (master[i] == b ? 0 : 36);
    for (int e = a + 1; e < d; e++) {
      const int j = brow[b0 + e];
      const int qj = rowptr[iperm[j]] + pair_row_offset(j, b, master, obstacle, bptr);
      rec[k++] = make_int4(fl, j * kFactorStride + (master[j] == b ? 18 : 54), qi + e - 1, qj + a);
    }
  }
}

// The off-diagonal blocks from the body-pair table (thread per pair): the
// product of k_offdiag_assembled for the pair (lo, hi) through b, computed
// once and written as the block (lo, hi) and its transpose (hi, lo); bitwise
// the blocks k_offdiag_assembled writes. The pairs of one body are
// neighbours in the table, so their factors are read from L1.
__global__ void k_offdiag_pairs(long long npairs, const int4* __restrict__ rec, const double* __restrict__ factors,
                                double step, double* W64, float* W32, long long kstride) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= npairs) return;
  const int4 r = rec[g];
  const double* left = factors + r.x;
  const double* right = factors + r.y;
  double Lr[18], Pr[18], W[9];
#pragma unroll
  for (int q = 0; q < 18; q += 2) {
    const double2 l = ld2(left + q), p = ld2(right + q);
    Lr[q] = l.x; Lr[q + 1] = l.y; Pr[q] = p.x; Pr[q + 1] = p.y;
  }
#pragma unroll
  for (int q = 0; q < 9; q++) W[q] = 0.0;
  hp_add(Lr, Pr, W);
#pragma unroll
  for (int q = 0; q < 9; q++) W[q] *= step;
#pragma unroll
  for (int rr = 0; rr < 3; rr++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      W64[(3 * c + rr) * kstride + r.z] = W[3 * c + rr];   // row lo, column hi: W as computed
      W32[(3 * c + rr) * kstride + r.z] = (float)W[3 * c + rr];
      W64[(3 * c + rr) * kstride + r.w] = W[3 * rr + c];   // row hi, column lo: the transpose
      W32[(3 * c + rr) * kstride + r.w] = (float)W[3 * rr + c];
    }
}

// The contact's factor through one of its bodies, as k_row_factors forms it:
// side 0 (master) or 1 (slave, H negated, ldy.c:685); P = M^-1 H^T when want_p.
__device__ __forceinline__ void contact_factor(const SceneDev& sc, int i, int slave_side, bool want_p, double* H,
                                               double* P) {
  const int b = slave_side ? sc.slave[i] : sc.master[i];
  double base[9], X[3];
#pragma unroll
  for (int q = 0; q < 9; q++) base[q] = sc.base[(size_t)9 * i + q];
  const double* Xp = slave_side ? sc.spnt : sc.mpnt;
#pragma unroll
  for (int q = 0; q < 3; q++) X[q] = Xp[(size_t)3 * i + q];
  rig_H(sc.rot + (size_t)9 * b, sc.x0 + (size_t)3 * b, base, X, H);
  if (slave_side) {
#pragma unroll
    for (int q = 0; q < 18; q++) H[q] = -H[q];
  }
  if (want_p) minv_ht(sc.jinv + (size_t)9 * b, sc.minv[b], H, P);
}

// k_offdiag_pairs without the stored factors: each pair forms its two
// factors from the bodies (the same operations as k_row_factors, so the
// blocks are bitwise the same), which saves the factor array's write and
// read-back. The pair record's factor offsets give the contacts and sides.
__global__ void k_offdiag_pairs_formed(long long npairs, const int4* __restrict__ rec, SceneDev sc, double step,
                                       double* W64, float* W32, long long kstride) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= npairs) return;
  const int4 r = rec[g];
  const int lo = r.x / kFactorStride, hi = r.y / kFactorStride;
  double Lr[18], Hh[18], Pr[18], W[9];
  contact_factor(sc, lo, r.x - lo * kFactorStride != 0, false, Lr, nullptr);
  contact_factor(sc, hi, r.y - hi * kFactorStride != 18, true, Hh, Pr);
#pragma unroll
  for (int q = 0; q < 9; q++) W[q] = 0.0;
  hp_add(Lr, Pr, W);
#pragma unroll
  for (int q = 0; q < 9; q++) W[q] *= step;
#pragma unroll
  for (int rr = 0; rr < 3; rr++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      W64[(3 * c + rr) * kstride + r.z] = W[3 * c + rr];
      W32[(3 * c + rr) * kstride + r.z] = (float)W[3 * c + rr];
      W64[(3 * c + rr) * kstride + r.w] = W[3 * rr + c];
      W32[(3 * c + rr) * kstride + r.w] = (float)W[3 * rr + c];
    }
}

// Sorted row of every off-diagonal block of the colour-sorted CSR (thread per
// row), kept with the layout so the per-step block kernel needs no search.
__global__ void k_block_rows(int n, const int* rowptr, int* brow) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  for (int k = rowptr[p]; k < rowptr[p + 1]; k++) brow[k] = p;
}

// Sets *diff if the contact topology (master and slave of every contact, the
// obstacle flag of every body) differs from the copy kept with the last
// contact graph.
__global__ void k_topology_diff(int n, int nb, const int* master, const int* slave, const int* obst, const int* pm,
                                const int* ps, const int* po, int* diff) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  bool d = false;
  for (int i = t; i < n; i += stride) d |= master[i] != pm[i] || slave[i] != ps[i];
  for (int b = t; b < nb; b += stride) d |= obst[b] != po[b];
  if (__any_sync(0xffffffffu, d) && (threadIdx.x & 31) == 0) atomicExch(diff, 1);
}

// Tile of every sorted row (forward tile numbering).
__global__ void k_row_tile(int T, const int4* tiles, int* rtile) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const int4 ti = tiles[t];
  for (int r = 0; r < (ti.y & 63); r++) rtile[ti.x + r] = t;
}

// The tiles holding the neighbours of a tile's rows, earlier (side 0) and
// later (side 1) in forward colour order, each tile once: a per-warp hash
// table in shared memory (hcap slots per side, at least twice the tile's
// blocks, so a probe always ends) deduplicates them. With depE null it counts
// (cnt[side * (T + 1) + t]); otherwise it writes the lists at the scanned
// offsets, in arbitrary order (they are sets). Warp per tile.
__global__ void k_tile_deps(int T, const int4* tiles, const int2* tilek, const int* col, const int* rtile, int hcap,
                            int* cnt, const int* ptrE, const int* ptrL, int* depE, int* depL) {
  extern __shared__ int dep_smem[];
  const int wpb = blockDim.x / kWarp, warp = threadIdx.x / kWarp, lane = threadIdx.x & (kWarp - 1);
  const int t = blockIdx.x * wpb + warp;
  if (t >= T) return;  // uniform per warp
  int* tab = dep_smem + (size_t)warp * (2 * hcap + 2);
  int* num = tab + 2 * hcap;
  for (int i = lane; i < 2 * hcap; i += kWarp) tab[i] = -1;
  if (lane < 2) num[lane] = 0;
  __syncwarp();
  const int4 ti = tiles[t];
  const int2 tk = tilek[t];
  const bool fill = depE != nullptr;
  for (int k = tk.x + lane; k < tk.y; k += kWarp) {
    const int j = col[k];
    if (j >= ti.z && j < ti.w) continue;  // a row of the same colour (none: they share no body)
    const int side = j < ti.z ? 0 : 1;
    const int d = rtile[j];
    int* tb = tab + side * hcap;
    unsigned h = ((unsigned)d * 2654435761u) & (unsigned)(hcap - 1);
    while (true) {
      const int old = atomicCAS(tb + h, -1, d);
      if (old == -1) {
        const int pos = atomicAdd(num + side, 1);
        if (fill) {
          if (side == 0) depE[ptrE[t] + pos] = d;
          else depL[ptrL[t] + pos] = d;
        }
        break;
      }
      if (old == d) break;
      h = (h + 1) & (unsigned)(hcap - 1);
    }
  }
  __syncwarp();
  if (!fill && lane < 2) cnt[lane * (T + 1) + t] = num[lane];
}

// Off-diagonal blocks handed in by the caller (AoS, 9 doubles per block in
// caller CSR order) gathered into the colour-sorted plane layout.
__global__ void k_offdiag_copy(int n, const int* perm, const int* iperm, const int* adjptr, const int* adjcol,
                               const double* Woff, const int* rowptr, int* col, double* W64, float* W32,
                               long long kstride) {
  const int p = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
  const int lane = threadIdx.x & (kWarp - 1);
  if (p >= n) return;
  const int i = perm[p];
  const int kb = adjptr[i], d = adjptr[i + 1] - kb, qb = rowptr[p];
  for (int t = lane; t < d; t += kWarp) {
    const long long qo = qb + t;
    col[qo] = iperm[adjcol[kb + t]];
    const double* w = Woff + (size_t)9 * (kb + t);
#pragma unroll
    for (int q = 0; q < 9; q++) {
      const double v = w[q];
      W64[q * kstride + qo] = v;
      W32[q * kstride + qo] = (float)v;
    }
  }
}

// Row quantities (caller order, AoS) into the colour-sorted plane layout.
__global__ void k_rows_permute(int n, const int* perm, const double* Wii, const double* Aii, const double* rho_in,
                               const double* Bi, const double* Vi, const double* gap_in, const double* fric_in,
                               const double* rest_in, const double* coh_in, double* Wd, double* Ad, double* Bv,
                               double* Vv, double* rho, double* gap, double* fric, double* rest, double* coh) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int i = perm[p];
#pragma unroll
  for (int q = 0; q < 9; q++) {
    Wd[(size_t)q * n + p] = Wii[(size_t)9 * i + q];
    Ad[(size_t)q * n + p] = Aii[(size_t)9 * i + q];
  }
#pragma unroll
  for (int q = 0; q < 3; q++) {
    Bv[(size_t)q * n + p] = Bi[(size_t)3 * i + q];
    Vv[(size_t)q * n + p] = Vi[(size_t)3 * i + q];
  }
  rho[p] = rho_in[i];
  gap[p] = gap_in[i];
  fric[p] = fric_in[i];
  rest[p] = rest_in[i];
  coh[p] = coh_in[i];
}

// Initial R and U (caller order, 3 doubles per row) into the sorted buffers.
__global__ void k_state_in(int n, const int* perm, const double* R, const double* U, double4* R64, float4* R32,
                           double4* Us) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int i = perm[p];
  const double r0 = R[3 * (size_t)i], r1 = R[3 * (size_t)i + 1], r2 = R[3 * (size_t)i + 2];
  R64[p] = make_double4(r0, r1, r2, 0.0);
  R32[p] = make_float4((float)r0, (float)r1, (float)r2, 0.f);
  Us[p] = make_double4(U[3 * (size_t)i], U[3 * (size_t)i + 1], U[3 * (size_t)i + 2], 0.0);
}

// Final R, U and per-constraint merit back into caller order.
__global__ void k_state_out(int n, const int* perm, const double4* R64, const double4* Usrc, const double* conmerit,
                            double merit_denom, double* R, double* U, double* cm) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int i = perm[p];
  const double4 r = R64[p], u = Usrc[p];
  R[3 * (size_t)i] = r.x; R[3 * (size_t)i + 1] = r.y; R[3 * (size_t)i + 2] = r.z;
  U[3 * (size_t)i] = u.x; U[3 * (size_t)i + 1] = u.y; U[3 * (size_t)i + 2] = u.z;
  if (cm && conmerit) cm[i] = conmerit[p] / merit_denom;
}

// Shadow copy of a double buffer into its float buffer (start of a mixed solve).
__global__ void k_shadow(int n, const double4* R64, float4* R32) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double4 r = R64[p];
  R32[p] = make_float4((float)r.x, (float)r.y, (float)r.z, 0.f);
}

}  // namespace b2
