// b2_solve.cuh -- block Gauss-Seidel in colour order with dataflow scheduling
// and the merit pass fused into the next sweep.
//
// Reference loop (bgs.c:913-1069): every iteration sweeps the rows in list
// order (each row: B' = B + sum_j W_ij R_j, diagonal solve, error sums), then
// MERIT_Function (mrf.c:35-185) recomputes U = B + W_ii R_i + sum_j W_ij R_j for
// every row and the merit; the loop stops when error <= epsilon and merit <=
// meritval, or at maxiter.
//
// Order. Rows are stored sorted by colour (rows of one colour share no
// non-obstacle body, so W_ij = 0 inside a colour); the sweep is the reference
// loop run on this colour-permuted list (colours in reverse on the backward
// sweeps of the reverse option).
//
// Fused merit. The merit of iterate s is evaluated inside sweep s+1: while a
// row gathers its neighbours' reactions for the Gauss-Seidel sum (the new
// value for rows earlier in the sweep, the previous one otherwise) it also
// forms U_merit = B + W_ii R_i^s + sum_j W_ij R_j^s from the previous values.
// The merit, the U handed to the diagonal solver (the reference starts
// iteration s+1 from the U its merit pass wrote) and the stopping decision for
// iterate s are the reference's, while W is streamed once per iteration.
//
// Scheduling. Instead of a grid-wide barrier per colour, warps claim tiles
// (runs of at most 32 rows of one colour and one problem) from one counter in
// (sweep, colour, tile) order and wait only for the rows a tile reads: for
// sweep s, a neighbour earlier in the sweep must have completed sweep s, a
// later one sweep s-1 (per-row completion counters). Reactions are
// triple-buffered, so a tile of sweep s+1 may run while sweep s is being
// decided; sweep s+2 waits for that decision. Every wait is bounded.
// Progress: a tile only waits for rows of tiles claimed before it, so the
// earliest unfinished tile can always proceed (all blocks are co-resident,
// cooperative launch).
//
// Problems. One launch may solve several independent problems (a batch of
// scenes); each keeps its own decisions, and the tiles of a problem's sweeps
// after its final decision are skipped.
//
// Reductions. Each tile writes its error and merit partial sums; the warp that
// completes a problem's last tile of a sweep adds that problem's partials in
// tile order and takes its stopping decision, decisions being taken in sweep
// order. Results therefore do not depend on which warp ran which tile.
#pragma once

#include <cuda_runtime.h>
#include "b2_common.cuh"
#include "b2_diag.cuh"

namespace b2 {

constexpr int kSolveThreads = 64;
constexpr int kSolveWarps = kSolveThreads / kWarp;
// 32-block chunks whose loads are issued together: 2 in FP64 (more would spill
// under the 168-register cap); 1 in the FP32 sweeps, whose pass 1 reads only
// shared memory (staged W, gathered reactions) -- measured fastest
template <bool MIXED>
__host__ __device__ constexpr int chunk_unroll() { return MIXED ? 1 : 2; }
constexpr int kTileHeader = 256;                     // bytes of per-warp shared memory before the staging
constexpr uint64_t kBarrierLimitNs = 2000000000ull;  // 2 s per bounded wait (default of SolveArgs::wait_ns)

enum { DECIDE_NONE = 0, DECIDE_CONTINUE = 1, DECIDE_STOP = 2 };

// Device-side control block of one solve launch (zeroed before launch).
struct SolveControl {
  unsigned next_tile;       // tile counter in (sweep, colour, tile) order
  int stop;                 // set once every problem has taken its final decision
  int timeout;              // a bounded wait gave up (device error)
  int nstopped;             // problems that have taken their final decision
  int sweeps;               // sweeps started (including discarded speculative ones)
  int pad;
  unsigned long long t_start;  // global timer at launch (ns)
};

// Per-problem control block: one independent GAUSS_SEIDEL_Solve each
// (zeroed before launch).
struct ProblemControl {
  unsigned tiles_done[3];   // completed tiles of sweep s, slot s % 3
  int stop;                 // the final decision is taken
  int final_iter;           // launch-local index of the returned iterate
  int iters;                // iterations completed in this launch
  int thrown;               // FAILURE_EXIT raised
  int pad;
  double merit;             // merit of the returned iterate (0 with nomerit)
  double error;             // relative error of the returned iterate
  double merit_input;       // merit of the input iterate (merit mode)
  double prev_error;        // relative error of the latest iterate, kept between decisions
  unsigned long long t_stop;  // global timer at the final decision (ns)
};

struct SolveArgs {
  int n, ntiles, nprob;
  int nactive;              // problems with at least one row (the launch ends when all have decided)
  const int4* tiles;        // [ntiles] first row, rows | problem << 6, first and end row of its colour (forward order)
  const int2* tilek;        // [ntiles] the tile's off-diagonal blocks [kb, ke)
  const int* ptile_ptr;     // [nprob+1] the tiles of each problem ...
  const int* ptile;         // [ntiles]  ... in ascending order (fixed summation order)
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
  const int* kind;          // [n] constraint kind (dom.h:98), or null: all CONTACT (the KINDS kernels only)
  const double* Zv;         // [4][n] the bilateral rows' Z (b2_diag.cuh), with kind
  const double* gap;        // [n]
  const double* fric;       // [n]
  const double* rest;       // [n]
  const double* coh;        // [n]
  double4* R64[3];          // triple-buffered reactions: iterate k in R64[(in + 1 + k) % 3]
  float4* R32[3];           // float shadows (mixed precision)
  double4* Us[2];           // U state without merit: sweep s reads Us[s%2], writes Us[(s+1)%2]
  double4* Um[2];           // merit U computed in sweep s: Um[s%2]
  double* conmerit[2];      // per-row merit numerator computed in sweep s: conmerit[s%2] (may be null)
  int* done;                // [n] sweeps completed per row (zeroed before launch)
  // per tile (forward numbering), when available: the tiles holding its rows'
  // neighbours in earlier / later colours, and sweeps completed per tile
  // (zeroed before launch); null: the per-row flags above are used instead
  const int* depE_ptr;
  const int* depE;
  const int* depL_ptr;
  const int* depL;
  int* tile_done;
  int* decided;             // [nprob][pstride] decision after each sweep (zeroed before launch)
  double* part;             // [3][ntiles][4] per-tile partial sums
  double* rerhist;          // [nprob][pstride] history arrays (indexed by iter0 + k)
  double* merhist;
  unsigned long long* failkey;  // [nprob][pstride] per sweep: max (order position + 1) << 2 | kind of a diagonal failure
  unsigned* failcount;          // [nprob][pstride] per sweep: number of diagonal failures
  int pstride;              // per-problem stride of the arrays above (>= maxiter + 2)
  const double* free_energy;  // [nprob] free energy of each problem (ldy.c:739)
  SolveControl* ctrl;
  ProblemControl* pctl;     // [nprob]
  double* trace;            // per-row diagonal-solve record of one sweep (null: off)
  int trace_sweep;
  double epsilon, meritval, diagepsilon, step;
  int maxiter, diagmaxiter, diagsolver, failure, dynamic, reverse, nomerit;
  int iter0;                // global index of this launch's first iteration
  int in;                   // R64/R32 buffer holding the input iterate
  int u0_from_merit;        // sweep 0 hands the merit U (not Us) to the diagonal solver
  int gcap;                 // Gauss-Seidel products staged per tile window
  int warp_smem;            // bytes of dynamic shared memory per warp
  unsigned long long wait_ns;  // limit of every wait on a flag another warp sets (ns)
};

// trace record per row: B'[3], U in[3], R in[3], U out[3], R out[3], kind
constexpr int kTraceStride = 16;

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded wait until *p >= need. Returns false when the solve has stopped or
// the wait ran out (the timeout is recorded in ctrl). The first check is
// inlined; only the spin is out of line (a call site saves live registers, so
// the common case must not be a call).
static __device__ __noinline__ bool wait_at_least_spin(const int* p, int need, SolveControl* ctrl, uint64_t limit) {
  const uint64_t t0 = globaltimer_ns();
  volatile int* stop = &ctrl->stop;
  volatile int* to = &ctrl->timeout;
  while (ld_acquire(p) < need) {
    if (*stop || *to) return false;
    if (globaltimer_ns() - t0 > limit) { *to = 1; return false; }
    __nanosleep(64);
  }
  return true;
}
__device__ __forceinline__ bool wait_at_least(const int* p, int need, SolveControl* ctrl, uint64_t limit) {
  if (ld_acquire(p) >= need) return true;
  return wait_at_least_spin(p, need, ctrl, limit);
}

// Gate of a tile of sweep s >= 2 of one problem: 1 = run (the decision after
// sweep s-2 is to continue), 2 = skip (the problem has taken its final
// decision, so later sweeps are discarded), 0 = the solve is ending or the
// bounded wait gave up.
static __device__ __noinline__ int gate_wait_spin(const int* decided_s2, const int* pstop, SolveControl* ctrl, uint64_t limit) {
  const uint64_t t0 = globaltimer_ns();
  volatile int* stop = &ctrl->stop;
  volatile int* to = &ctrl->timeout;
  while (true) {
    const int d = ld_acquire(decided_s2);
    if (d == DECIDE_CONTINUE) return 1;
    if (d == DECIDE_STOP) return 2;
    if (*(volatile const int*)pstop) return 2;
    if (*stop || *to) return 0;
    if (globaltimer_ns() - t0 > limit) { *to = 1; return 0; }
    __nanosleep(64);
  }
}
__device__ __forceinline__ int gate_wait(const int* decided_s2, const int* pstop, SolveControl* ctrl, uint64_t limit) {
  if (ld_acquire(decided_s2) == DECIDE_CONTINUE) return 1;
  return gate_wait_spin(decided_s2, pstop, ctrl, limit);
}

// Bounded wait until every tile of list[lo, hi) has completed `need` sweeps:
// the lanes take the entries in turn (one parallel round for a typical tile),
// and the warp barrier after the waits orders every lane's later loads after
// all of them (each tile publishes its rows with one release after its own
// warp barrier).
__device__ __forceinline__ bool wait_tiles(const int* list, int lo, int hi, const int* tile_done, int need,
                                           SolveControl* ctrl, uint64_t limit, int lane) {
  bool ok = true;
  for (int i = lo + lane; i < hi; i += kWarp) ok = wait_at_least(tile_done + __ldg(list + i), need, ctrl, limit) && ok;
  return ok;
}

// 32-byte load that bypasses L1 (reaction buffers are rewritten by other SMs
// while the kernel runs, so a line cached in L1 could be stale).
__device__ __forceinline__ double4 ldcg4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  const double2 lo = __ldcg(q), hi = __ldcg(q + 1);
  return make_double4(lo.x, lo.y, hi.x, hi.y);
}

// ---- staging of a tile's column indices and FP32 coefficient planes (TMA) --

// Each window of a tile's blocks is copied into the warp's shared memory with
// one-dimensional bulk copies (no cluster, no multicast): the column indices
// always, the nine W planes in the FP32 sweeps (at 72 bytes a block the FP64
// planes would leave windows too small to hold a tile). Passes 1 and 2 read
// them there instead of through L1.
template <bool MIXED>
__host__ __device__ constexpr bool stage_w() { return MIXED; }
constexpr int kStageBar = 192;  // byte offset of the warp's staging barrier in its header
constexpr int kStageSlack = 8;  // window planes hold gcap + slack blocks (16-byte aligned copy ranges)

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void stage_bar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool stage_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the staging copies of the given phase.
static __device__ __noinline__ bool stage_wait_spin(uint32_t bar, uint32_t parity, SolveControl* ctrl) {
  const uint64_t t0 = globaltimer_ns();
  while (!stage_try_wait(bar, parity)) {
    if (globaltimer_ns() - t0 > kBarrierLimitNs) { *(volatile int*)&ctrl->timeout = 1; return false; }
  }
  return true;
}
__device__ __forceinline__ bool stage_wait(uint32_t bar, uint32_t parity, SolveControl* ctrl) {
  if (stage_try_wait(bar, parity)) return true;
  return stage_wait_spin(bar, parity, ctrl);
}

// Blocks [a0, a1) (multiples of 4: every copy starts on a 16-byte boundary and
// is a multiple of 16 bytes) of the column indices and, with WITHW, the nine W
// planes into the warp's window, completion counted on its barrier. One lane
// issues.
template <bool WITHW, typename real>
__device__ __forceinline__ void stage_issue(uint32_t bar, uint32_t col_s, uint32_t w_s, int wstride, const int* col,
                                            const real* W, long long kstride, int a0, int a1) {
  const uint32_t bytes = (uint32_t)(a1 - a0) * 4u;
  const uint32_t wbytes = WITHW ? (uint32_t)(a1 - a0) * (uint32_t)sizeof(real) : 0u;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the window's previous reads are done
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes + 9u * wbytes)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(col_s),
               "l"(col + a0), "r"(bytes), "r"(bar)
               : "memory");
  if constexpr (WITHW)
#pragma unroll
  for (int q = 0; q < 9; q++)
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     w_s + (uint32_t)q * (uint32_t)wstride * (uint32_t)sizeof(real)),
                 "l"(W + q * kstride + a0), "r"(wbytes), "r"(bar)
                 : "memory");
}

template <bool MIXED>
__device__ __forceinline__ auto stage_src(const SolveArgs& a) {
  if constexpr (MIXED) return a.W32;
  else return a.W64;
}

// Per-sweep flags shared by the tile routine.
struct SweepFlags {
  bool gs;        // Gauss-Seidel update of this sweep (false: merit-only pass)
  bool merit;     // evaluate the merit of the input iterate
  bool u_merit;   // hand the merit U to the diagonal solver
  bool backward;  // colours in reverse order
  bool prev_done; // every row of the problem has completed the previous sweep (its decision is taken)
};

// Loads of one 32-block chunk: column indices and the nine coefficients of
// each block (lane per block, coalesced plane loads).
template <bool MIXED, typename real>
__device__ __forceinline__ void load_chunk(const SolveArgs& a, int base, int ke, int lane,
                                           int (&jj)[chunk_unroll<MIXED>()], real (&w)[chunk_unroll<MIXED>()][9],
                                           const int* col_s, const real* w_s, int a0, int wstride) {
  constexpr int kChunkUnroll = chunk_unroll<MIXED>();
#pragma unroll
  for (int u = 0; u < kChunkUnroll; u++) {
    const int k = base + u * kWarp + lane;
    jj[u] = k < ke ? col_s[k - a0] : -1;
  }
#pragma unroll
  for (int u = 0; u < kChunkUnroll; u++) {
    const int k = base + u * kWarp + lane;
#pragma unroll
    for (int q = 0; q < 9; q++) {
      if (k < ke) {
        if constexpr (stage_w<MIXED>()) w[u][q] = w_s[q * wstride + k - a0];
        else if constexpr (MIXED) w[u][q] = __ldg(a.W32 + q * a.kstride + k);
        else w[u][q] = __ldg(a.W64 + q * a.kstride + k);
      } else {
        w[u][q] = real(0);
      }
    }
  }
}

template <bool MIXED, typename real>
__device__ __forceinline__ void load_r(const SolveArgs& a, int buf, int j, real& r0, real& r1, real& r2) {
  if constexpr (MIXED) {
    const float4 v = __ldcg(a.R32[buf] + j);
    r0 = v.x; r1 = v.y; r2 = v.z;
  } else {
    const double4 v = ldcg4(a.R64[buf] + j);
    r0 = v.x; r1 = v.y; r2 = v.z;
  }
}

// 16-byte asynchronous copy global -> shared memory, cached in L2 only (the
// reaction buffers are rewritten by other SMs while the kernel runs, so a line
// cached in L1 could be stale).
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
// Completion of this thread's asynchronous copies (visible to the thread).
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// The FP32 sweeps gather the previous-sweep reactions of a whole window with
// asynchronous copies before pass 1 (one round trip instead of one per
// chunk). The FP64 sweeps load them in pass 1, next to their uncoalesced W
// loads, which set the chain there (measured: gathering first is slower).
template <bool MIXED>
__host__ __device__ constexpr bool gather_r() { return MIXED; }

// Bytes per block of the window's products: FP32 sweeps, one float4 slot that
// first receives the gathered reaction and is then overwritten by the product
// (in place, by the lane that gathered it); FP64 sweeps, three planes of
// doubles (conflict-free row sums; measured faster than 32-byte slots).
template <bool MIXED>
__host__ __device__ constexpr size_t slot_bytes() { return MIXED ? 16 : 24; }

// shared memory of one warp of k_solve: tile row offsets, one slot per block of
// the window, and the staged column indices (and FP32 W)
template <bool MIXED>
__host__ __device__ constexpr size_t solve_warp_smem(int gcap) {
  return (size_t)kTileHeader + (size_t)gcap * slot_bytes<MIXED>() +
         (size_t)(gcap + kStageSlack) * (4 + (stage_w<MIXED>() ? 9 * (MIXED ? sizeof(float) : sizeof(double)) : 0));
}
// shared memory of a warp: fixed part and bytes per staged block
template <bool MIXED>
__host__ __device__ constexpr size_t solve_smem_fixed() { return solve_warp_smem<MIXED>(0); }
template <bool MIXED>
__host__ __device__ constexpr size_t solve_smem_per_block() {
  return slot_bytes<MIXED>() + 4 + (stage_w<MIXED>() ? 9 * (MIXED ? sizeof(float) : sizeof(double)) : 0);
}

// One tile of up to 32 consecutive rows of one colour, owned by one warp.
//
// Pass 1 needs only values of the previous sweep: lanes stride over the
// tile's contiguous CSR range (lane per block, coalesced plane loads), form
// the merit products W_ij R_j^old and the Gauss-Seidel products of neighbours
// later in the sweep, and the merit term of each row is evaluated. Pass 2
// waits for the neighbours earlier in the sweep and forms their products with
// the new reactions. Only pass 2 and the diagonal solves lie on the chain of
// colours, so the streaming of W and the merit overlap the waits.
//
// The products are staged in shared memory and lane r adds those of row
// r0 + r in list order onto its running sums, which start from B
// (Gauss-Seidel, bgs.c:957-963) and from B + W_ii R_i (merit U, mrf.c:61-68);
// with the build's disabled multiply-add contraction this reproduces the
// reference's NVADDMUL chains operation for operation in FP64. Lane r then
// solves its row (diagonal solve in FP64). Tiles with more blocks than the
// staging holds are processed in windows. Returns false if a wait gave up or
// the solve has stopped.
template <bool MIXED, bool KINDS>
__device__ __forceinline__ bool solve_tile(const SolveArgs& a, const SweepFlags& f, int r0, int nr, int cs, int ce,
                                           int s, int rin, int rout, int prob, int kb0, int ke0, int tile,
                                           unsigned char* wsm, uint32_t& phase, double& errup, double& errlo,
                                           double& mnum) {
  typedef typename std::conditional<MIXED, float, double>::type real;
  constexpr int kChunkUnroll = chunk_unroll<MIXED>();
  constexpr int kSlots = kWarp * kChunkUnroll;
  const int gcap = a.gcap;
  const int wstride = gcap + kStageSlack;
  int* tp = reinterpret_cast<int*>(wsm);                        // [kWarp + 1]
  float4* slot = reinterpret_cast<float4*>(wsm + kTileHeader);   // FP32: [gcap] R_j, then W_ij R_j
  real* gst = reinterpret_cast<real*>(wsm + kTileHeader);        // FP64: [3][gcap] W_ij R_j
  int* col_s = reinterpret_cast<int*>(wsm + kTileHeader + (size_t)gcap * slot_bytes<MIXED>());  // [wstride] (staged)
  // product of the window's block g, and its read-back for the row sums
  auto put = [&](int g, real m0, real m1, real m2) {
    if constexpr (MIXED) slot[g] = make_float4(m0, m1, m2, 0.f);
    else { gst[g] = m0; gst[gcap + g] = m1; gst[2 * gcap + g] = m2; }
  };
  auto add = [&](int g, double (&acc)[3]) {
    if constexpr (MIXED) {
      const float4 v = slot[g];
      acc[0] = acc[0] + (double)v.x; acc[1] = acc[1] + (double)v.y; acc[2] = acc[2] + (double)v.z;
    } else {
      acc[0] = acc[0] + (double)gst[g]; acc[1] = acc[1] + (double)gst[gcap + g]; acc[2] = acc[2] + (double)gst[2 * gcap + g];
    }
  };
  real* w_s = reinterpret_cast<real*>(col_s + wstride);                                  // [9][wstride] (staged)
  const uint32_t bar = smem_addr(wsm + kStageBar);
  const int lane = threadIdx.x & (kWarp - 1);
  const int n = a.n;
  const bool own = lane < nr;
  const int p = r0 + lane;
  // window 0 on its way while the row data is read (the tile's block range is
  // in its record, so the copy does not wait for the row offsets)
  if (lane == 0 && ke0 > kb0)
      stage_issue<stage_w<MIXED>()>(bar, smem_addr(col_s), smem_addr(w_s), wstride, a.col, stage_src<MIXED>(a), a.kstride, kb0 & ~3,
                  (min(ke0, kb0 + gcap) + 3) & ~3);
  if constexpr (!stage_w<MIXED>()) {  // FP64 W planes of the tile into L2 ahead of pass 1 (a hint)
    if (lane < 9 && ke0 > kb0) {
      const int p0 = kb0 & ~1, p1 = (ke0 + 1) & ~1;  // 16-byte aligned range of doubles
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a.W64 + lane * a.kstride + p0),
                   "r"((uint32_t)(p1 - p0) * 8u)
                   : "memory");
    }
  }
  if (lane <= nr) tp[lane] = __ldg(a.rowptr + r0 + lane);
  if (lane == 0 && nr == kWarp) tp[kWarp] = __ldg(a.rowptr + r0 + kWarp);
  bool ok = true;
  const bool by_tile = a.tile_done != nullptr;
  if (!f.prev_done) {  // the rows and all neighbours of this tile have completed the previous sweep
    if (by_tile) {
      if (lane == 0) ok = wait_at_least(a.tile_done + tile, s, a.ctrl, a.wait_ns);
      ok = wait_tiles(a.depE, __ldg(a.depE_ptr + tile), __ldg(a.depE_ptr + tile + 1), a.tile_done, s, a.ctrl, a.wait_ns, lane) && ok;
      ok = wait_tiles(a.depL, __ldg(a.depL_ptr + tile), __ldg(a.depL_ptr + tile + 1), a.tile_done, s, a.ctrl, a.wait_ns, lane) && ok;
      __syncwarp();
    } else if (own) {
      ok = wait_at_least(a.done + p, s, a.ctrl, a.wait_ns);
    }
  }

  double B[3] = {0.0, 0.0, 0.0}, W[9], Rold[3] = {0.0, 0.0, 0.0}, ag[3], am[3] = {0.0, 0.0, 0.0};
  double V[3] = {0.0, 0.0, 0.0};
  double rho_row = 0.0;  // the diagonal solver's rho, loaded with the row data
  ContactParams cp;
  cp.step = a.step;
  cp.dynamic = a.dynamic;
  cp.friction = cp.restitution = cp.cohesion = cp.gap = 0.0;
  int ckind = CON_CONTACT;
  double Zr[4] = {0.0, 0.0, 0.0, 0.0};
  if constexpr (KINDS) {
    if (own && ok) {
      ckind = __ldg(a.kind + p);
      if (ckind != CON_CONTACT)
#pragma unroll
        for (int q = 0; q < 4; q++) Zr[q] = __ldg(a.Zv + (size_t)q * n + p);
    }
  }
  if (own && ok) {
#pragma unroll
    for (int q = 0; q < 3; q++) B[q] = __ldg(a.Bv + (size_t)q * n + p);
    const double4 ro = ldcg4(a.R64[rin] + p);
    Rold[0] = ro.x; Rold[1] = ro.y; Rold[2] = ro.z;
#pragma unroll
    for (int q = 0; q < 9; q++) W[q] = __ldg(a.Wd + (size_t)q * n + p);
    cp.friction = __ldg(a.fric + p);
    cp.restitution = __ldg(a.rest + p);
    cp.cohesion = __ldg(a.coh + p);
    cp.gap = __ldg(a.gap + p);
    rho_row = __ldg(a.rho + p);
#pragma unroll
    for (int q = 0; q < 3; q++) V[q] = __ldg(a.Vv + (size_t)q * n + p);
  }
  ag[0] = B[0]; ag[1] = B[1]; ag[2] = B[2];
  __syncwarp();
  const int kb = tp[0], ke = tp[nr];
  const int mb = own ? tp[lane] : 0, me = own ? tp[lane + 1] : 0;
  const int nwin = ke > kb ? (ke - kb + gcap - 1) / gcap : 1;

  for (int win = 0; win < nwin; win++) {
    const int wb = kb + win * gcap, we = min(ke, wb + gcap);
    const int a0 = wb & ~3;
    {
      if (we > wb) {
        if (win > 0 && lane == 0)
          stage_issue<stage_w<MIXED>()>(bar, smem_addr(col_s), smem_addr(w_s), wstride, a.col, stage_src<MIXED>(a), a.kstride, a0, (we + 3) & ~3);
        ok = stage_wait(bar, phase, a.ctrl) && ok;
        phase ^= 1u;
      }
    }
    // ---- gather of the previous-sweep reactions the window needs: 16-byte
    // asynchronous copies into the blocks' slots, all in flight together. Lane
    // l copies the blocks k = wb + l (mod 32), the blocks it computes below.
    if constexpr (gather_r<MIXED>()) {
    for (int k = wb + lane; k < we; k += kWarp) {
      const int j = col_s[k - a0];
      const bool earlier = f.backward ? (j >= ce) : (j < cs);
      if (f.merit || (f.gs && !earlier)) {
        if (!f.prev_done && !by_tile) ok = wait_at_least(a.done + j, s, a.ctrl, a.wait_ns) && ok;
        cp_async16(smem_addr(slot + (k - wb)), a.R32[rin] + j);
      }
    }
    cp_async_wait_all();
    }
    // ---- pass 1: previous-sweep values. W_ij R_j^(s-1) of every block (the
    // merit's products, and the Gauss-Seidel products of later neighbours),
    // written over the block's gathered reaction
    for (int base = wb; base < we; base += kSlots) {
      int jj[kChunkUnroll];
      real w[kChunkUnroll][9];
      load_chunk<MIXED, real>(a, base, we, lane, jj, w, col_s, w_s, a0, wstride);
#pragma unroll
      for (int u = 0; u < kChunkUnroll; u++) {
        const int j = jj[u];
        if (j >= 0) {
          const bool earlier = f.backward ? (j >= ce) : (j < cs);
          if (f.merit || (f.gs && !earlier)) {
            const int g = base + u * kWarp + lane - wb;
            real ro0, ro1, ro2;
            if constexpr (gather_r<MIXED>()) {
              const float4 v = slot[g];
              ro0 = v.x; ro1 = v.y; ro2 = v.z;
            } else {
              if (!f.prev_done && !by_tile) ok = wait_at_least(a.done + j, s, a.ctrl, a.wait_ns) && ok;
              load_r<MIXED, real>(a, rin, j, ro0, ro1, ro2);
            }
            const real* Wk = w[u];
            put(g, Wk[0] * ro0 + Wk[3] * ro1 + Wk[6] * ro2, Wk[1] * ro0 + Wk[4] * ro1 + Wk[7] * ro2,
                Wk[2] * ro0 + Wk[5] * ro1 + Wk[8] * ro2);
          }
        }
      }
    }
    __syncwarp();
    if (f.merit) {  // each row adds its own merit products, in list order
      // the row's own term first (ag still holds B here); set here, not at the
      // row load, so that the load's latency hides behind the window's staging
      if (win == 0 && own) nvaddmul(ag, W, Rold, am);
      const int lo = mb > wb ? mb : wb;
      const int hi = me < we ? me : we;
      for (int k = lo; k < hi; k++) add(k - wb, am);
      __syncwarp();  // pass 2 overwrites the slots of earlier neighbours
    }
    // ---- merit term of each row (mrf.c:81-87), once its U is complete
    if (win == nwin - 1 && f.merit && own) {
      double A[9];
#pragma unroll
      for (int q = 0; q < 9; q++) A[q] = __ldg(a.Ad + (size_t)q * n + p);
      double up;
      if (KINDS && ckind != CON_CONTACT) up = merit_row_bilateral(ckind, Zr, cp.gap, a.step, a.dynamic, A, V, am);
      else up = merit_row<MIXED>(cp, A, V, am, Rold);
      mnum += up;
      a.Um[s & 1][p] = make_double4(am[0], am[1], am[2], 0.0);
      if (a.conmerit[0]) a.conmerit[s & 1][p] = up;
    }
    if (!f.gs) continue;
    if (by_tile && win == 0) {  // every tile holding an earlier neighbour has completed this sweep
      const int* ptr = f.backward ? a.depL_ptr : a.depE_ptr;
      ok = wait_tiles(f.backward ? a.depL : a.depE, __ldg(ptr + tile), __ldg(ptr + tile + 1), a.tile_done, s + 1,
                      a.ctrl, a.wait_ns, lane) && ok;
      __syncwarp();
    }
    // ---- pass 2: neighbours earlier in this sweep (their new reactions)
    bool gathered = false;
    if constexpr (gather_r<MIXED>()) {
      if (by_tile) {  // no wait left per neighbour: all new reactions in one round of asynchronous copies
        auto is_earlier = [&](int j) { return f.backward ? (j >= ce) : (j < cs); };
        for (int k = wb + lane; k < we; k += kWarp) {
          const int j = col_s[k - a0];
          if (is_earlier(j)) cp_async16(smem_addr(slot + (k - wb)), a.R32[rout] + j);
        }
        cp_async_wait_all();
        for (int k = wb + lane; k < we; k += kWarp) {
          const int j = col_s[k - a0];
          if (is_earlier(j)) {
            const float4 v = slot[k - wb];
            real Wk[9];
#pragma unroll
            for (int q = 0; q < 9; q++) Wk[q] = w_s[q * wstride + k - a0];
            put(k - wb, Wk[0] * v.x + Wk[3] * v.y + Wk[6] * v.z, Wk[1] * v.x + Wk[4] * v.y + Wk[7] * v.z,
                Wk[2] * v.x + Wk[5] * v.y + Wk[8] * v.z);
          }
        }
        gathered = true;
      }
    }
    if (!gathered)
    for (int base = wb; base < we; base += kSlots) {
#pragma unroll
      for (int u = 0; u < kChunkUnroll; u++) {
        const int k = base + u * kWarp + lane;
        if (k < we) {
          const int j = col_s[k - a0];
          const bool earlier = f.backward ? (j >= ce) : (j < cs);
          if (earlier) {
            if (!by_tile) ok = wait_at_least(a.done + j, s + 1, a.ctrl, a.wait_ns) && ok;
            real Wk[9];
#pragma unroll
            for (int q = 0; q < 9; q++) {
              if constexpr (stage_w<MIXED>()) Wk[q] = w_s[q * wstride + k - a0];
              else if constexpr (MIXED) Wk[q] = __ldg(a.W32 + q * a.kstride + k);
              else Wk[q] = __ldg(a.W64 + q * a.kstride + k);
            }
            real rn0, rn1, rn2;
            load_r<MIXED, real>(a, rout, j, rn0, rn1, rn2);
            put(k - wb, Wk[0] * rn0 + Wk[3] * rn1 + Wk[6] * rn2, Wk[1] * rn0 + Wk[4] * rn1 + Wk[7] * rn2,
                Wk[2] * rn0 + Wk[5] * rn1 + Wk[8] * rn2);
          }
        }
      }
    }
    __syncwarp();
    {  // each row adds its own Gauss-Seidel products, in list order
      const int lo = mb > wb ? mb : wb;
      const int hi = me < we ? me : we;
      for (int k = lo; k < hi; k++) add(k - wb, ag);
    }
    __syncwarp();
  }
  ok = __all_sync(0xffffffffu, ok);
  if (!ok) return false;

  // ---- lane per row: diagonal solve
  if (own) {
    if (f.gs) {
      double R[3] = {Rold[0], Rold[1], Rold[2]};
      double U[3];
      if (f.u_merit) { U[0] = am[0]; U[1] = am[1]; U[2] = am[2]; }
      else { const double4 us = ldcg4(a.Us[s & 1] + p); U[0] = us.x; U[1] = us.y; U[2] = us.z; }
      double* tr = (a.trace && s == a.trace_sweep) ? a.trace + (size_t)kTraceStride * p : nullptr;
      if (tr) {
#pragma unroll
        for (int q = 0; q < 3; q++) { tr[q] = ag[q]; tr[3 + q] = U[q]; tr[6 + q] = R[q]; }
      }
      int kind;
      if (KINDS && ckind != CON_CONTACT)
        kind = bilateral_solve_row(ckind, Zr, a.step, a.dynamic, a.failure, a.diagepsilon, a.diagmaxiter, W, ag, V, U,
                                   R);
      else
        kind = diagonal_solve_row<MIXED>(a.diagsolver, a.failure, cp, a.diagepsilon, a.diagmaxiter, rho_row, W, ag, V,
                                         U, R);
      if (tr) {
#pragma unroll
        for (int q = 0; q < 3; q++) { tr[9 + q] = U[q]; tr[12 + q] = R[q]; }
        tr[15] = (double)kind;
      }
      if (kind) {
        const unsigned long long pos = f.backward ? (unsigned long long)(n - 1 - p) : (unsigned long long)p;
        const size_t fo = (size_t)prob * a.pstride + a.iter0 + s;
        atomicMax(a.failkey + fo, ((pos + 1ull) << 2) | (unsigned long long)kind);
        atomicAdd(a.failcount + fo, 1u);
      }
      a.R64[rout][p] = make_double4(R[0], R[1], R[2], 0.0);
      if constexpr (MIXED) a.R32[rout][p] = make_float4((float)R[0], (float)R[1], (float)R[2], 0.f);
      if (a.nomerit) a.Us[(s + 1) & 1][p] = make_double4(U[0], U[1], U[2], 0.0);
      const double d0 = R[0] - Rold[0], d1 = R[1] - Rold[1], d2 = R[2] - Rold[2];
      errup += d0 * d0 + d1 * d1 + d2 * d2;
      errlo += R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
    }
    if (!by_tile) st_release(a.done + p, s + 1);  // publishes this row's writes of sweep s
  }
  __syncwarp();
  if (by_tile && lane == 0) st_release(a.tile_done + tile, s + 1);  // publishes the tile's writes of sweep s
  return true;
}

// Decision after sweep s of problem `prob`, taken by the warp that completed
// the problem's last tile of the sweep: sums the problem's tile partials in
// tile order and applies the reference's stopping rule (bgs.c:1028-1036,
// mrf.c:176-184). Decisions of a problem are taken in sweep order.
static __device__ __noinline__ void finalize_sweep(const SolveArgs& a, int prob, int s) {
  const int lane = threadIdx.x & (kWarp - 1);
  ProblemControl* pc = a.pctl + prob;
  volatile int* decided = a.decided + (size_t)prob * a.pstride;
  int prev = DECIDE_CONTINUE;
  if (s >= 1) {
    bool ok = true;
    if (lane == 0) ok = wait_at_least((const int*)decided + s - 1, DECIDE_CONTINUE, a.ctrl, a.wait_ns);
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (!ok) return;
    prev = decided[s - 1];
  }
  if (prev == DECIDE_STOP) {
    if (lane == 0) { pc->tiles_done[s % 3] = 0; __threadfence(); decided[s] = DECIDE_STOP; }
    return;
  }
  double su = 0.0, sl = 0.0, sm = 0.0;
  const double* base = a.part + (size_t)(s % 3) * a.ntiles * 4;
  const int t0 = __ldg(a.ptile_ptr + prob), t1 = __ldg(a.ptile_ptr + prob + 1);
  if (a.nprob == 1) {  // tiles 0 .. ntiles-1
#pragma unroll 8
    for (int t = lane; t < t1; t += kWarp) {
      su += __ldcg(base + 4 * t); sl += __ldcg(base + 4 * t + 1); sm += __ldcg(base + 4 * t + 2);
    }
  } else {
#pragma unroll 8
    for (int i = t0 + lane; i < t1; i += kWarp) {
      const int t = __ldg(a.ptile + i);
      su += __ldcg(base + 4 * t); sl += __ldcg(base + 4 * t + 1); sm += __ldcg(base + 4 * t + 2);
    }
  }
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) {
    su += __shfl_down_sync(0xffffffffu, su, d);
    sl += __shfl_down_sync(0xffffffffu, sl, d);
    sm += __shfl_down_sync(0xffffffffu, sm, d);
  }
  if (lane != 0) return;
  const size_t ho = (size_t)prob * a.pstride + a.iter0;
  const bool merit_mode = !a.nomerit;
  const double error = sqrt(su) / sqrt(sl == 0.0 ? 1.0 : sl);                         // bgs.c:1028
  double lo = __ldg(a.free_energy + prob);
  lo = lo < 2.220446049250313e-16 ? 1.0 : lo;                                           // mrf.c:45
  const double merit_prev = merit_mode ? (0.5 * sm) / (lo == 0.0 ? 1.0 : lo) : 0.0;     // mrf.c:176-184
  const bool gs_sweep = !(merit_mode && s == a.maxiter);
  const bool failed = __ldcg(a.failkey + ho + s) != 0ull;
  volatile double* perr_slot = &pc->prev_error;
  const double perr = *perr_slot;  // error of iterate s-1
  int final_iter = -2, thrown = 0;
  double fm = 0.0, fe = 0.0;
  if (merit_mode) {
    if (s == 0) pc->merit_input = merit_prev;
    if (s >= 1) {
      a.rerhist[ho + s - 1] = perr;
      a.merhist[ho + s - 1] = merit_prev;
      const bool meets = !(perr > a.epsilon || merit_prev > a.meritval);  // bgs.c:1036
      if (meets || s == a.maxiter) { final_iter = s - 1; fm = merit_prev; fe = perr; }
      else if (gs_sweep && failed && a.failure == FAIL_EXIT) { final_iter = s; thrown = 1; fm = merit_prev; fe = error; }
    } else if (failed && a.failure == FAIL_EXIT) {
      final_iter = 0; thrown = 1; fe = error;
    }
  } else {
    a.rerhist[ho + s] = error;
    a.merhist[ho + s] = 0.0;
    if (failed && a.failure == FAIL_EXIT) { final_iter = s; thrown = 1; fe = error; }
    else if (!(error > a.epsilon) || s + 1 >= a.maxiter) { final_iter = s; fe = error; }
  }
  *perr_slot = error;
  pc->tiles_done[s % 3] = 0;
  if (final_iter >= -1) {
    pc->final_iter = final_iter;
    pc->iters = thrown ? final_iter : final_iter + 1;
    pc->thrown = thrown;
    pc->merit = fm;
    pc->error = fe;
    pc->t_stop = globaltimer_ns();
    __threadfence();
    decided[s] = DECIDE_STOP;
    *(volatile int*)&pc->stop = 1;
    if (atomicAdd(&a.ctrl->nstopped, 1) + 1 == a.nactive) *(volatile int*)&a.ctrl->stop = 1;
  } else {
    __threadfence();
    decided[s] = DECIDE_CONTINUE;
  }
}

// Persistent solve of all problems of the layout. Tiles are numbered by
// colour (forward order) and, inside a colour, by problem; every sweep claims
// them in that order (reversed on backward sweeps). A problem's tiles of a
// sweep after its final decision are skipped. The launch ends when every
// problem has decided.
// Six blocks of two warps per SM (at most 168 registers a thread): with the
// list-order colouring a sweep has about six levels of ~1.5k tiles each, so
// 1,776 resident warps hold a whole level in one wave.
template <bool MIXED, bool KINDS>
__device__ __forceinline__ void solve_persistent(const SolveArgs& a) {
  extern __shared__ __align__(16) unsigned char solve_smem[];
  const int warp = threadIdx.x / kWarp;
  const int lane = threadIdx.x & (kWarp - 1);
  unsigned char* wsm = solve_smem + (size_t)warp * a.warp_smem;
  const bool merit_mode = !a.nomerit;
  const int maxsweep = merit_mode ? a.maxiter : a.maxiter - 1;  // last sweep that can run
  volatile int* stop = &a.ctrl->stop;
  const int T = a.ntiles;
  if (blockIdx.x == 0 && threadIdx.x == 0) a.ctrl->t_start = globaltimer_ns();
  uint32_t phase = 0;  // parity of the warp's staging barrier
  if (lane == 0) stage_bar_init(smem_addr(wsm + kStageBar));
  __syncwarp();

  while (true) {
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(&a.ctrl->next_tile, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    const int s = (int)(t / (unsigned)T);
    const int w = (int)(t % (unsigned)T);
    if (s > maxsweep || *stop) break;
    SweepFlags f;
    f.gs = !(merit_mode && s == a.maxiter);
    f.merit = merit_mode;
    f.u_merit = merit_mode && (s >= 1 || a.u0_from_merit);
    f.backward = a.reverse && ((a.iter0 + s) & 1);
    f.prev_done = s == 0;
    const int tile = f.backward ? T - 1 - w : w;
    const int4 ti = __ldg(a.tiles + tile);  // first row, rows | problem << 6, colour bounds
    const int2 tk = __ldg(a.tilek + tile);  // its blocks
    const int prob = ti.y >> 6, nr = ti.y & 63;
    const unsigned ntp = a.nprob == 1 ? (unsigned)T : (unsigned)(__ldg(a.ptile_ptr + prob + 1) - __ldg(a.ptile_ptr + prob));
    volatile int* decided = a.decided + (size_t)prob * a.pstride;
    if (s >= 2) {  // sweep s reuses the buffers of iterate s-3: wait for the decision after sweep s-2
      int gate = 0;
      if (lane == 0) gate = gate_wait((const int*)decided + s - 2, &a.pctl[prob].stop, a.ctrl, a.wait_ns);
      gate = __shfl_sync(0xffffffffu, gate, 0);
      if (gate == 0) break;
      if (gate == 2) continue;  // this problem has finished: its later sweeps are not run
    }
    if (s >= 1) {  // the decision after sweep s-1 is taken only once all its tiles have completed (and
                   // released their rows): then no neighbour needs its own wait in pass 1
      int pd = 0;
      if (lane == 0) pd = ld_acquire((const int*)decided + s - 1) != DECIDE_NONE;
      f.prev_done = __shfl_sync(0xffffffffu, pd, 0) != 0;
    }
    const int rin = (a.in + s) % 3;       // iterate s-1
    const int rout = (a.in + s + 1) % 3;  // iterate s
    double errup = 0.0, errlo = 0.0, mnum = 0.0;
    if (!solve_tile<MIXED, KINDS>(a, f, ti.x, nr, ti.z, ti.w, s, rin, rout, prob, tk.x, tk.y, tile, wsm, phase, errup,
                                  errlo, mnum))
      break;
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
      errup += __shfl_down_sync(0xffffffffu, errup, d);
      errlo += __shfl_down_sync(0xffffffffu, errlo, d);
      mnum += __shfl_down_sync(0xffffffffu, mnum, d);
    }
    unsigned prev = 0;
    if (lane == 0) {
      double* pp = a.part + ((size_t)(s % 3) * T + tile) * 4;
      pp[0] = errup; pp[1] = errlo; pp[2] = mnum;
      __threadfence();
      prev = atomicAdd(&a.pctl[prob].tiles_done[s % 3], 1u);
      if (w == 0) atomicMax(&a.ctrl->sweeps, s + 1);
    }
    prev = __shfl_sync(0xffffffffu, prev, 0);
    if (prev == ntp - 1) {
      __threadfence();
      finalize_sweep(a, prob, s);
    }
  }
}

// FP64 sweeps (bitwise the reference's arithmetic: this translation unit is
// built without fused multiply-adds).
template <bool MIXED>
__global__ void __launch_bounds__(kSolveThreads, 6) k_solve(const __grid_constant__ SolveArgs a) {
  solve_persistent<MIXED, false>(a);
}

// the same with rows of the bilateral kinds (a.kind, a.Zv), used only when a
// problem has such rows, so that the contact kernels keep their registers
template <bool MIXED>
__global__ void __launch_bounds__(kSolveThreads, 6) k_solve_kinds(const __grid_constant__ SolveArgs a) {
  solve_persistent<MIXED, true>(a);
}

// FP32 sweeps of mixed precision, defined in b2_solve_fp32.cu: that
// translation unit is built with fused multiply-adds, which the FP32 products
// and the FP64 diagonal solves and merit of these sweeps may use (their results
// are not bitwise the reference's anyway; the closing FP64 sweep is).
__global__ void __launch_bounds__(kSolveThreads, 6) k_solve_fp32(const __grid_constant__ SolveArgs a);
__global__ void __launch_bounds__(kSolveThreads, 6) k_solve_fp32_kinds(const __grid_constant__ SolveArgs a);

}  // namespace b2
