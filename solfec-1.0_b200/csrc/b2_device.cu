// b2_device.cu -- device layer of the B200 contact-solve path: context, memory,
// kernel orchestration and the thin C ABI declared in include/b2_device.h.
//
// Per step the path is: upload (optional) -> row factors, W_ii, rho, A, B, V,
// free energy -> contact graph through shared bodies -> Jones-Plassmann
// colouring -> colour-sorted CSR of 3x3 blocks in nine coefficient planes ->
// persistent Gauss-Seidel solve with the merit fused into the next sweep ->
// results scattered back to the caller's row order.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cfloat>
#include <climits>
#include <vector>
#include <algorithm>
#include <mutex>

#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include "../../include/b2_device.h"
#include "b2_common.cuh"
#include "b2_diag.cuh"
#include "b2_solve.cuh"
#include "b2_assemble.cuh"
#include "b2_colour.cuh"
#include "b2_rigid.cuh"
#include "b2_detect.cuh"
#include "b2_bilateral.cuh"

using namespace b2;

namespace {

thread_local char g_err[1024] = "";

void set_err(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

#define B2_CK(call)                                                                  \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      set_err("%s failed at %s:%d: %s", #call, __FILE__, __LINE__, cudaGetErrorString(e_)); \
      return B2DEV_ECUDA;                                                            \
    }                                                                                \
  } while (0)

#define B2_TRY(expr)             \
  do {                           \
    int rc_ = (expr);            \
    if (rc_ != B2DEV_OK) return rc_; \
  } while (0)

struct Buf {
  void* p = nullptr;
  size_t cap = 0;
};

// Grow-only device buffer of at least `bytes` (contents not preserved).
int ensure(Buf& b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.cap >= bytes) return B2DEV_OK;
  if (b.p) { cudaFree(b.p); b.p = nullptr; b.cap = 0; }
  size_t want = bytes + bytes / 8;  // headroom for growing problems
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) {
    set_err("cudaMalloc(%zu bytes) failed: %s", want, cudaGetErrorString(e));
    return B2DEV_ECUDA;
  }
  b.cap = want;
  return B2DEV_OK;
}

template <class T>
T* ptr(Buf& b) { return static_cast<T*>(b.p); }

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

inline int blocks_for(long long n, int t) { return (int)std::max<long long>(1, (n + t - 1) / t); }

__global__ void k_iota(int n, int* v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i;
}

// adjptr monotone within [0, K] and every adjcol in [0, n)
__global__ void k_check_graph(int n, long long K, const int* adjptr, const int* adjcol, int* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int a = adjptr[i], b = adjptr[i + 1];
  if (a < 0 || b < a || b > K || (i == 0 && a != 0)) { atomicExch(bad, 1); return; }
  for (int k = a; k < b; k++)
    if (adjcol[k] < 0 || adjcol[k] >= n) { atomicExch(bad, 1); return; }
}

__global__ void k_set_last_zero(int* a, int n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) a[n] = 0;
}

// one diagonal block solve per thread on caller-given rows (unit parity of the
// device diagonal solvers)
__global__ void k_diag_batch(int n, int solver, int failure, double diagepsilon, int diagmaxiter, int dynamic,
                             double step, const double* W, const double* B, const double* V, const double* rho,
                             const double* gap, const double* fric, const double* rest, const double* coh, double* U,
                             double* R, int* kind) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ContactParams cp;
  cp.friction = fric[i]; cp.restitution = rest[i]; cp.cohesion = coh[i]; cp.gap = gap[i]; cp.step = step;
  cp.dynamic = dynamic;
  double w[9], b[3], v[3], u[3], r[3];
  for (int q = 0; q < 9; q++) w[q] = W[9 * (size_t)i + q];
  for (int q = 0; q < 3; q++) { b[q] = B[3 * (size_t)i + q]; v[q] = V[3 * (size_t)i + q]; u[q] = U[3 * (size_t)i + q]; r[q] = R[3 * (size_t)i + q]; }
  kind[i] = diagonal_solve_row(solver, failure, cp, diagepsilon, diagmaxiter, rho[i], w, b, v, u, r);
  for (int q = 0; q < 3; q++) { U[3 * (size_t)i + q] = u[q]; R[3 * (size_t)i + q] = r[q]; }
}

// caller-order blocks back out of the sorted plane layout (introspection)
__global__ void k_offdiag_out(int n, const int* iperm, const int* adjptr, const int* rowptr, const double* W64,
                              long long kstride, double* Woff) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int kb = adjptr[i], d = adjptr[i + 1] - kb, qb = rowptr[iperm[i]];
  for (int t = 0; t < d; t++)
    for (int q = 0; q < 9; q++) Woff[(size_t)9 * (kb + t) + q] = W64[q * kstride + qb + t];
}

}  // namespace

struct b2dev_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sms = 0;

  // scene (caller order)
  int nbod = 0, ncon = 0;
  Buf rot, x0, jinv, minv, velo, velo0, obst, master, slave, mpnt, spnt, base;
  Buf gap_c, fric_c, rest_c, coh_c;
  // constraint kinds of the rows (b2dev_set_kinds): caller order, and the
  // colour-sorted planes the KINDS solve kernels read; none = all CONTACT
  Buf kind_c, Z_c, kind_s, Z_s;
  bool has_kinds = false;
  bool have_scene = false;

  // caller-order row data and graph
  Buf factors, Wii, Aii, rho_c, B_c, V_c, fe_part, fe_dev, bad;
  Buf bdeg, bptr, cursor, brow, deg, adjptr, adjcol, adjbod, Woff_c;
  bool assembled_mode = false;

  // colouring and layout
  Buf colour, sel, cctrl, keys_out, iota, perm, iperm, colptr, sdeg;
  int colour_list = 1;            // 1: greedy order = list order, 0: seeded Jones-Plassmann priorities
  Buf gptr_prev, gcol_prev;       // graph of the last colouring (reused while the graph is unchanged)
  bool colour_valid = false;
  // the colour-sorted layout (perm, rowptr, colptr, tile table) of the last
  // prepare_layout, and what it was built for: reused with the colouring
  bool layout_valid = false;
  int layout_nprob = 0, layout_tile_rows = 0;
  std::vector<int> layout_prob_off;
  int colour_n = -1, colour_mode = -1, ncolours_prev = 0;
  long long colour_K = -1;
  uint64_t colour_seed_prev = 0;
  long long colour_reuse = 0;     // colourings skipped because the graph was unchanged
  Buf rowptr, col, W64, W32, Wd, Ad, Bv, Vv, rho, gap, fric, rest, coh;
  std::vector<int> colptr_h;
  std::vector<int> rowptr_h;   // sorted CSR offsets (host copy, sizes the tiles)
  std::vector<int> rprob_h;    // problem of each sorted row

  // state and solve scratch
  Buf R64[3], R32[3], Us[2], Um[2], conmerit[2], done, decided, part, rer, mer, failkey, failcount, sctrl, io,
      cub_tmp, trace;
  int ntiles = 0;
  int max_tile_blocks = 0;  // most off-diagonal blocks of one tile
  int tile_rows = kWarp;    // rows per tile (at most one warp)
  bool tile_rows_auto = true;  // chosen from the problem size until set (b2dev_set_tile_rows, the autotuner)

  // independent problems solved together (one GAUSS_SEIDEL_Solve each); rows
  // of problem k are caller rows prob_off[k] .. prob_off[k+1]-1
  int nprob = 1;
  std::vector<int> prob_off;
  Buf tiles, tilek, tile_prob, ptile_ptr, ptile, row_prob, pctl, pfe, pvec;
  // per tile: the tiles its rows depend on (earlier / later colours) and its completion flag
  Buf rtile, dcnt, depE_ptr, depL_ptr, depE, depL, tile_done;
  bool deps_valid = false;
  // rigid time integration (b2dev_rigid_*): mass centre, inertia, mass, scheme,
  // external force of the step, NEW2 auxiliary vector, per-step loads
  Buf rb_x, rb_J, rb_mass, rb_scheme, rb_fext, rb_aux, rb_loads, rb_flags, rb_fail;
  bool have_rigid = false;
  bool rb_imp = false;        // some body integrates with NEW3 (its Newton solve can fail)
  bool rb_have_flags = false;
  // sphere contact detection (b2dev_spheres_setup, b2dev_detect_spheres): the
  // spheres, the grid, the pair lists, the contacts before sparsification
  // (st_*), and per contact of the last detection its sphere pair key, role
  // flag, spatial point, new flag and carried R, U
  int nsph = 0, nsurf = 0;
  std::vector<double> sph_mat_h;
  Buf sph_body, sph_ref, sph_rad, sph_surf, sph_mat, sph_cur, sph_cell, sph_hkey, sph_hkey_s, sph_idx, sph_sorted,
      sph_bstart, sph_bend, sph_cnt, sph_off, sph_pi, sph_pj, sph_rmax, sph_total, sph_keep, sph_pos, sph_bcnt, sph_bptr,
      sph_blist, sph_pkey, sph_pslo, sph_pR, sph_pU, sph_ccnt;
  Buf st_master, st_slave, st_point, st_mpnt, st_spnt, st_base, st_gap, st_fric, st_rest, st_coh, st_R0, st_U0,
      st_key, st_slo, st_new, st_area;
  Buf det_point, det_R0, det_U0, det_key, det_slo, det_new, det_area;
  // bilateral constraints listed after the detected contacts by every
  // detection (b2dev_constraints_setup): kind, bodies, points, frame and Z of
  // each; det_ncont counts the contacts among the last detection's rows
  int cn_n = 0, det_ncont = 0;
  Buf cn_kind, cn_master, cn_slave, cn_mpnt, cn_spnt, cn_base, cn_Z;
  // convexes of the detection (b2dev_convexes_setup): their data, the
  // adjacency of convexes of one body, and the convex-convex sweep
  int nconv = 0;
  Buf cvx_body, cvx_vptr, cvx_vert, cvx_fptr, cvx_fac, cvx_sptr, cvx_surf, cvx_ns, cvx_cur, cvx_pla, cvx_box,
      cvx_aptr, cvx_adj;
  bool cvx_have_adj = false;
  Buf cc_lox, cc_idx, cc_sidx, cc_cnt, cc_off, cc_keys, cc_keys_s, cc_cell, cc_hkey, cc_hkey_s, cc_large,
      cc_bstart, cc_bend, cc_misc, cc_keep, cc_cls, cc_order;
  size_t cc_order_off = 0;  // the work order's offset in cc_order
  // CONTACT_SPARSIFY (dom.c:3107-3109 defaults)
  double sp_threshold = 0.01, sp_minarea = 0.0, sp_mindist = kGeomEps;
  // CONTACT_EXCLUDE_BODIES / CONTACT_EXCLUDE_SURFACES / UNPHYSICAL_PENETRATION
  Buf ex_bodies, ex_surf;
  int n_ex_bodies = 0;
  std::vector<int> ex_surf_pairs;  // surface pairs (s1, s2), the table built for nsurf
  int ex_surf_nsurf = -1;
  double depth = -DBL_MAX;
  bool det_valid = false;       // the scene's contacts are those of the last detection
  bool det_assembled = false;   // ... and the local dynamics was assembled from them
  std::vector<int> ptile_count;  // tiles per problem
  int trace_sweep = -1;  // sweep of the next solve whose diagonal solves are recorded
  unsigned long long wait_ns = kBarrierLimitNs;  // limit of the solver's bounded waits
  // the contact topology (master, slave, obstacle flags) of the last contact
  // graph built by b2dev_assemble: an unchanged topology keeps that graph
  Buf topo_m, topo_s, topo_o, topo_flag;
  int topo_n = -1, topo_nb = -1;
  bool topo_valid = false;
  Buf blkrow;  // sorted row of every off-diagonal block (with the layout)
  // body-pair table of the off-diagonal blocks (k_pair_fill), valid for the
  // layout and contact topology it was built on
  Buf pr_cnt, pr_ptr, pr_rec;
  long long npairs = 0;
  bool pairs_valid = false;
  bool factors_stored = true;  // the last row pass wrote the factor array

  int n = 0;
  long long K = 0, kstride = 0;
  int ncolours = 0;
  double free_energy = 0.0, step = 0.0;
  int dynamic = 1;
  bool ready = false;
  int state_r = 0;             // R64 buffer holding the current reactions
  Buf* state_u = nullptr;      // buffer holding the current U (one of Us[], Um[])
  Buf* state_cm = nullptr;     // buffer holding the per-row merit numerators of the last merit pass
  cudaEvent_t ev[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  long long launches = 0;  // kernels of this library launched on this context
  float assemble_ms = 0.f;
  bool assemble_ms_pending = false;  // ev[0], ev[1] of the last assembly not yet read

  // CUDA graph of the batched solve (rebuilt when its captured arguments change)
  cudaGraphExec_t graph = nullptr;
  std::vector<uintptr_t> graph_key;
  void* pinned = nullptr;  // SolveControl + nprob ProblemControl written by the graph
  size_t pinned_cap = 0;
};

namespace {

int scan_exclusive(b2dev_ctx* c, const int* in, int* out, int count) {
  size_t bytes = 0;
  B2_CK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, count, c->stream));
  B2_TRY(ensure(c->cub_tmp, bytes));
  B2_CK(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, bytes, in, out, count, c->stream));
  return B2DEV_OK;
}

int cooperative_grid(const void* func, int threads, int sms, int want, int* grid, size_t smem = 0) {
  int per_sm = 0;
  if (smem > 0) B2_CK(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  B2_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem));
  if (per_sm < 1) {
    set_err("kernel cannot be resident with %d threads per block", threads);
    return B2DEV_ECUDA;
  }
  int cap = per_sm * sms;
  *grid = std::max(1, std::min(cap, want > 0 ? want : cap));
  return B2DEV_OK;
}

// Per tile, the tiles holding its rows' neighbours (in earlier and in later
// colours, each once) and a completion flag per tile: a tile waits for these
// few flags in one parallel round instead of one acquire per neighbour row.
// Without them (tiles too large for the deduplication table) the solve waits
// per row.
int build_deps(b2dev_ctx* c) {
  cudaStream_t st = c->stream;
  c->deps_valid = false;
  const int T = c->ntiles, n = c->n;
  if (T == 0 || c->K == 0) return B2DEV_OK;
  int hcap = 64;
  while (hcap < 2 * c->max_tile_blocks + 2) hcap *= 2;
  const size_t per_warp = sizeof(int) * (2 * (size_t)hcap + 2);
  if (per_warp > 200 * 1024) return B2DEV_OK;
  const int wpb = (int)std::max<size_t>(1, std::min<size_t>(8, (96 * 1024) / per_warp));
  const size_t smem = per_warp * wpb;
  B2_TRY(ensure(c->rtile, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->dcnt, sizeof(int) * 2 * (T + 1)));
  B2_TRY(ensure(c->depE_ptr, sizeof(int) * (T + 1)));
  B2_TRY(ensure(c->depL_ptr, sizeof(int) * (T + 1)));
  B2_TRY(ensure(c->tile_done, sizeof(int) * (T + 1)));
  c->launches++;
  k_row_tile<<<blocks_for(T, 256), 256, 0, st>>>(T, ptr<int4>(c->tiles), ptr<int>(c->rtile));
  B2_CK(cudaMemsetAsync(c->dcnt.p, 0, sizeof(int) * 2 * (T + 1), st));
  B2_CK(cudaFuncSetAttribute((const void*)k_tile_deps, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  c->launches++;
  k_tile_deps<<<blocks_for(T, wpb), wpb * kWarp, smem, st>>>(T, ptr<int4>(c->tiles), ptr<int2>(c->tilek),
                                                             ptr<int>(c->col), ptr<int>(c->rtile), hcap,
                                                             ptr<int>(c->dcnt), nullptr, nullptr, nullptr, nullptr);
  B2_TRY(scan_exclusive(c, ptr<int>(c->dcnt), ptr<int>(c->depE_ptr), T + 1));
  B2_TRY(scan_exclusive(c, ptr<int>(c->dcnt) + T + 1, ptr<int>(c->depL_ptr), T + 1));
  int tot[2] = {0, 0};
  B2_CK(cudaMemcpyAsync(&tot[0], ptr<int>(c->depE_ptr) + T, sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CK(cudaMemcpyAsync(&tot[1], ptr<int>(c->depL_ptr) + T, sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CK(cudaStreamSynchronize(st));
  B2_TRY(ensure(c->depE, sizeof(int) * (tot[0] + 1)));
  B2_TRY(ensure(c->depL, sizeof(int) * (tot[1] + 1)));
  c->launches++;
  k_tile_deps<<<blocks_for(T, wpb), wpb * kWarp, smem, st>>>(
      T, ptr<int4>(c->tiles), ptr<int2>(c->tilek), ptr<int>(c->col), ptr<int>(c->rtile), hcap, ptr<int>(c->dcnt),
      ptr<int>(c->depE_ptr), ptr<int>(c->depL_ptr), ptr<int>(c->depE), ptr<int>(c->depL));
  B2_CK(cudaGetLastError());
  c->deps_valid = true;
  return B2DEV_OK;
}

// Tile table: runs of at most `rows` consecutive sorted rows of one colour and
// one problem, numbered in forward colour order (problems ascending inside a
// colour); per problem, its tiles in ascending order.
int build_tiles(b2dev_ctx* c, int rows) {
  cudaStream_t st = c->stream;
  rows = std::max(1, std::min(kWarp, rows));
  c->tile_rows = rows;
  std::vector<int4> tl;
  std::vector<int2> tk;  // off-diagonal block range of each tile
  std::vector<int> tp;
  int mx = 0;
  for (int k = 0; k < c->ncolours; k++) {
    const int cb = c->colptr_h[k], ce = c->colptr_h[k + 1];
    for (int r = cb; r < ce;) {
      const int pr = c->rprob_h[r];
      int e = r + 1;
      while (e < ce && e - r < rows && c->rprob_h[e] == pr) e++;
      tl.push_back(make_int4(r, (e - r) | (pr << 6), cb, ce));  // rows | problem << 6
      tk.push_back(make_int2(c->rowptr_h[r], c->rowptr_h[e]));
      tp.push_back(pr);
      mx = std::max(mx, c->rowptr_h[e] - c->rowptr_h[r]);
      r = e;
    }
  }
  const int T = (int)tl.size();
  c->ntiles = T;
  c->max_tile_blocks = mx;
  std::vector<int> pptr(c->nprob + 1, 0), plist(std::max(T, 1));
  for (int t = 0; t < T; t++) pptr[tp[t] + 1]++;
  for (int k = 0; k < c->nprob; k++) pptr[k + 1] += pptr[k];
  c->ptile_count.assign(c->nprob, 0);
  for (int k = 0; k < c->nprob; k++) c->ptile_count[k] = pptr[k + 1] - pptr[k];
  {
    std::vector<int> cur(pptr.begin(), pptr.end() - 1);
    for (int t = 0; t < T; t++) plist[cur[tp[t]]++] = t;
  }
  B2_TRY(ensure(c->tiles, sizeof(int4) * (T + 1)));
  B2_TRY(ensure(c->tilek, sizeof(int2) * (T + 1)));
  B2_TRY(ensure(c->tile_prob, sizeof(int) * (T + 1)));
  B2_TRY(ensure(c->ptile_ptr, sizeof(int) * (c->nprob + 1)));
  B2_TRY(ensure(c->ptile, sizeof(int) * (T + 1)));
  if (T > 0) {
    B2_CK(cudaMemcpyAsync(c->tiles.p, tl.data(), sizeof(int4) * T, cudaMemcpyHostToDevice, st));
    B2_CK(cudaMemcpyAsync(c->tilek.p, tk.data(), sizeof(int2) * T, cudaMemcpyHostToDevice, st));
    B2_CK(cudaMemcpyAsync(c->tile_prob.p, tp.data(), sizeof(int) * T, cudaMemcpyHostToDevice, st));
    B2_CK(cudaMemcpyAsync(c->ptile.p, plist.data(), sizeof(int) * T, cudaMemcpyHostToDevice, st));
  }
  B2_CK(cudaMemcpyAsync(c->ptile_ptr.p, pptr.data(), sizeof(int) * (c->nprob + 1), cudaMemcpyHostToDevice, st));
  B2_CK(cudaStreamSynchronize(st));  // the host vectors above go out of scope
  return build_deps(c);
}

// Colour the caller-order graph (adjptr/adjcol) and build the colour-sorted
// layout; row data must already sit in the caller-order buffers.
// same_graph: the caller knows the contact graph is that of the last layout
// (an unchanged contact topology), so the comparison pass is skipped.
// kind and Z of every row into the colour-sorted planes (kind_s[p], Z_s[q n + p])
__global__ void k_kinds_permute(int n, const int* perm, const int* kind_c, const double* Z_c, int* kind_s,
                                double* Z_s) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int i = perm[p];
  kind_s[p] = kind_c[i];
  for (int q = 0; q < 4; q++) Z_s[(size_t)q * n + p] = Z_c[4 * (size_t)i + q];
}

static int permute_kinds(b2dev_ctx* c) {
  const int n = c->n;
  B2_TRY(ensure(c->kind_s, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->Z_s, sizeof(double) * 4 * (n + 1)));
  if (n == 0) return B2DEV_OK;
  c->launches++;
  k_kinds_permute<<<blocks_for(n, 256), 256, 0, c->stream>>>(n, ptr<int>(c->perm), ptr<int>(c->kind_c),
                                                             ptr<double>(c->Z_c), ptr<int>(c->kind_s),
                                                             ptr<double>(c->Z_s));
  B2_CK(cudaGetLastError());
  return B2DEV_OK;
}

// Duration of the last assembly from its events, once they have completed.
static void assemble_time(b2dev_ctx* c) {
  if (!c->assemble_ms_pending) return;
  if (cudaEventSynchronize(c->ev[1]) == cudaSuccess) cudaEventElapsedTime(&c->assemble_ms, c->ev[0], c->ev[1]);
  c->assemble_ms_pending = false;
}

// Device view of the uploaded scene (bodies and contacts) for the assembly kernels.
static SceneDev scene_view(b2dev_ctx* c) {
  SceneDev sc;
  sc.nbod = c->nbod; sc.ncon = c->ncon;
  sc.rot = ptr<double>(c->rot); sc.x0 = ptr<double>(c->x0); sc.jinv = ptr<double>(c->jinv);
  sc.minv = ptr<double>(c->minv); sc.velo = ptr<double>(c->velo); sc.velo0 = ptr<double>(c->velo0);
  sc.obstacle = ptr<int>(c->obst); sc.master = ptr<int>(c->master); sc.slave = ptr<int>(c->slave);
  sc.mpnt = ptr<double>(c->mpnt); sc.spnt = ptr<double>(c->spnt); sc.base = ptr<double>(c->base);
  return sc;
}

// The body-pair table of the current layout and contact topology (body lists
// bptr/brow, sorted rows rowptr/iperm, roles master/obstacle). Left invalid
// (the block kernel then runs) when the pair count or the factor offsets
// would not fit an int.
static int build_pairs(b2dev_ctx* c) {
  const int nb = c->nbod, n = c->n;
  cudaStream_t st = c->stream;
  c->pairs_valid = false;
  if ((long long)n * kFactorStride + kFactorStride > INT_MAX || c->K % 2 != 0) return B2DEV_OK;
  B2_TRY(ensure(c->pr_cnt, sizeof(long long) * (nb + 1)));
  B2_TRY(ensure(c->pr_ptr, sizeof(long long) * (nb + 1)));
  B2_CK(cudaMemsetAsync(c->pr_cnt.p, 0, sizeof(long long) * (nb + 1), st));
  c->launches++;
  k_pair_count<<<blocks_for(nb, 256), 256, 0, st>>>(nb, ptr<int>(c->obst), ptr<int>(c->bptr),
                                                   ptr<long long>(c->pr_cnt));
  size_t bytes = 0;
  B2_CK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, ptr<long long>(c->pr_cnt), ptr<long long>(c->pr_ptr), nb + 1,
                                      st));
  B2_TRY(ensure(c->cub_tmp, bytes));
  B2_CK(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, bytes, ptr<long long>(c->pr_cnt), ptr<long long>(c->pr_ptr),
                                      nb + 1, st));
  long long np = 0;
  B2_CK(cudaMemcpyAsync(&np, ptr<long long>(c->pr_ptr) + nb, sizeof(long long), cudaMemcpyDeviceToHost, st));
  B2_CK(cudaStreamSynchronize(st));
  if (2 * np != c->K) return B2DEV_OK;  // every block is one side of one pair
  B2_TRY(ensure(c->pr_rec, sizeof(int4) * (size_t)(np + 1)));
  c->launches++;
  k_pair_fill<<<blocks_for(nb, 128), 128, 0, st>>>(nb, ptr<int>(c->obst), ptr<int>(c->master), ptr<int>(c->bptr),
                                                  ptr<int>(c->brow), ptr<long long>(c->pr_ptr), ptr<int>(c->iperm),
                                                  ptr<int>(c->rowptr), ptr<int4>(c->pr_rec));
  B2_CK(cudaGetLastError());
  c->npairs = np;
  c->pairs_valid = true;
  return B2DEV_OK;
}

constexpr int kSmallProblemRows = 16384;  // at most this many rows: 8 rows per tile (tile_rows_auto)

int prepare_layout(b2dev_ctx* c, uint64_t seed, bool assembled, bool same_graph) {
  const int n = c->n;
  cudaStream_t st = c->stream;
  const int T = 256;
  B2_TRY(ensure(c->colour, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->sel, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->cctrl, sizeof(ColourControl)));
  B2_TRY(ensure(c->keys_out, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->iota, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->perm, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->iperm, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->colptr, sizeof(int) * (kMaxColours + 2)));
  B2_TRY(ensure(c->sdeg, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->rowptr, sizeof(int) * (n + 1)));

  ColourControl cc;
  memset(&cc, 0, sizeof cc);
  bool reuse = false;
  if (c->colour_valid && c->colour_n == n && c->colour_K == c->K && c->colour_mode == c->colour_list &&
      (c->colour_list || c->colour_seed_prev == seed) && n > 0 && same_graph) {
    reuse = true;
  } else if (c->colour_valid && c->colour_n == n && c->colour_K == c->K && c->colour_mode == c->colour_list &&
      (c->colour_list || c->colour_seed_prev == seed) && n > 0) {  // same graph as the last colouring?
    B2_CK(cudaMemsetAsync(c->bad.p, 0, sizeof(int), st));
    c->launches++;
    k_graph_diff<<<std::max(1, std::min(4 * c->sms, blocks_for(std::max<long long>(c->K, n + 1), T))), T, 0, st>>>(
        n, c->K, ptr<int>(c->adjptr), ptr<int>(c->adjcol), ptr<int>(c->gptr_prev), ptr<int>(c->gcol_prev),
        ptr<int>(c->bad));
    int diff = 1;
    B2_CK(cudaMemcpyAsync(&diff, c->bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaStreamSynchronize(st));
    reuse = diff == 0;
  }
  // rows per tile by size unless set: a small single problem has far fewer
  // tiles per colour level than resident warps, and its sweep is the chain of
  // colour levels, each as long as its slowest tile; 8-row tiles (a tile's
  // diagonal solves wait for the slowest of 8 lanes, not of 32) shortened the
  // sweep of a 2,163-row pile from 91 to 73 us and of a 375-row one from 39 to
  // 36 us, while large problems, whose levels fill the machine, keep 32
  if (c->tile_rows_auto && c->nprob == 1) c->tile_rows = n <= kSmallProblemRows ? 8 : kWarp;
  // same graph, same colours: the sorted layout and the tile table are those of
  // the last layout, unless the problems or the rows per tile changed since
  const bool same_layout = reuse && c->layout_valid && c->layout_nprob == c->nprob &&
                           c->layout_prob_off == c->prob_off && c->layout_tile_rows == c->tile_rows;
  c->layout_valid = false;
  if (reuse) {
    c->colour_reuse++;
    cc.ncolours = c->ncolours_prev;
  } else {
  B2_CK(cudaMemsetAsync(c->colour.p, 0xff, sizeof(int) * (n + 1), st));
  B2_CK(cudaMemsetAsync(c->cctrl.p, 0, sizeof(ColourControl), st));
  if (n > 0) {
    int grid = 0;
    B2_TRY(cooperative_grid((const void*)k_jp_colour, T, c->sms, blocks_for(n, T), &grid));
    int nn = n;
    const int* ap = ptr<int>(c->adjptr);
    const int* ac = ptr<int>(c->adjcol);
    unsigned long long sd = seed;
    int lo = c->colour_list;
    int* colp = ptr<int>(c->colour);
    int* selp = ptr<int>(c->sel);
    ColourControl* ctl = ptr<ColourControl>(c->cctrl);
    void* args[] = {&nn, &ap, &ac, &sd, &lo, &colp, &selp, &ctl};
    c->launches++;
    B2_CK(cudaLaunchCooperativeKernel((const void*)k_jp_colour, grid, T, args, 0, st));
  }
  B2_CK(cudaMemcpyAsync(&cc, c->cctrl.p, sizeof cc, cudaMemcpyDeviceToHost, st));
  B2_CK(cudaStreamSynchronize(st));
  if (cc.timeout) { set_err("colouring: grid barrier wait timed out"); return B2DEV_ETIMEOUT; }
  if (cc.overflow) { set_err("colouring: more than %d colours needed", kMaxColours); return B2DEV_ECOLOURS; }
  // keep the graph this colouring belongs to
  c->colour_valid = false;
  if (n > 0) {
    B2_TRY(ensure(c->gptr_prev, sizeof(int) * (n + 1)));
    B2_TRY(ensure(c->gcol_prev, sizeof(int) * (c->K + 1)));
    B2_CK(cudaMemcpyAsync(c->gptr_prev.p, c->adjptr.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, st));
    if (c->K > 0) B2_CK(cudaMemcpyAsync(c->gcol_prev.p, c->adjcol.p, sizeof(int) * c->K, cudaMemcpyDeviceToDevice, st));
    c->colour_valid = true;
    c->colour_n = n;
    c->colour_K = c->K;
    c->colour_mode = c->colour_list;
    c->colour_seed_prev = seed;
    c->ncolours_prev = cc.ncolours;
  }
  }
  c->ncolours = n > 0 ? cc.ncolours : 0;

  if (!same_layout) {
  // rows sorted by colour, ascending row index inside a colour (stable radix sort)
  c->launches++;
  k_iota<<<blocks_for(n, T), T, 0, st>>>(n, ptr<int>(c->iota));
  if (n > 0) {
    size_t bytes = 0;
    B2_CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, ptr<int>(c->colour), ptr<int>(c->keys_out),
                                          ptr<int>(c->iota), ptr<int>(c->perm), n, 0, 9, st));
    B2_TRY(ensure(c->cub_tmp, bytes));
    B2_CK(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, bytes, ptr<int>(c->colour), ptr<int>(c->keys_out),
                                          ptr<int>(c->iota), ptr<int>(c->perm), n, 0, 9, st));
  }
  c->launches++;
  k_colptr<<<blocks_for(n + 1, T), T, 0, st>>>(n, ptr<int>(c->keys_out), c->ncolours, ptr<int>(c->colptr));
  c->launches++;
  k_inverse_perm<<<blocks_for(n, T), T, 0, st>>>(n, ptr<int>(c->perm), ptr<int>(c->iperm));
  c->launches++;
  k_sorted_degree<<<blocks_for(n, T), T, 0, st>>>(n, ptr<int>(c->perm), ptr<int>(c->adjptr), ptr<int>(c->sdeg));
  c->launches++;
  k_set_last_zero<<<1, 32, 0, st>>>(ptr<int>(c->sdeg), n);
  B2_TRY(scan_exclusive(c, ptr<int>(c->sdeg), ptr<int>(c->rowptr), n + 1));
  B2_TRY(ensure(c->blkrow, sizeof(int) * ((size_t)c->K + 1)));
  if (n > 0 && c->K > 0) {
    c->launches++;
    k_block_rows<<<blocks_for(n, T), T, 0, st>>>(n, ptr<int>(c->rowptr), ptr<int>(c->blkrow));
  }

  c->colptr_h.assign(c->ncolours + 1, 0);
  if (c->ncolours > 0) {
    B2_CK(cudaMemcpyAsync(c->colptr_h.data(), c->colptr.p, sizeof(int) * (c->ncolours + 1), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaStreamSynchronize(st));
  }
  }

  const long long K = c->K;
  c->kstride = ((K + 31) / 32) * 32;
  B2_TRY(ensure(c->col, sizeof(int) * (c->kstride + 32)));
  B2_TRY(ensure(c->W64, sizeof(double) * 9 * (c->kstride + 1)));
  B2_TRY(ensure(c->W32, sizeof(float) * 9 * (c->kstride + 1)));
  const int wpb = 8;
  if (!same_layout || !same_graph) c->pairs_valid = false;
  if (n > 0 && K > 0 && assembled && same_layout && same_graph && !c->pairs_valid)
    B2_TRY(build_pairs(c));  // the second assembly on this layout and topology: the body-pair table
  if (n > 0 && K > 0) {
    if (assembled && c->pairs_valid && !c->factors_stored) {
      c->launches++;
      k_offdiag_pairs_formed<<<(unsigned)((c->npairs + 255) / 256), 256, 0, st>>>(
          c->npairs, ptr<int4>(c->pr_rec), scene_view(c), c->step, ptr<double>(c->W64), ptr<float>(c->W32),
          c->kstride);
    } else if (assembled && c->pairs_valid) {
      c->launches++;
      k_offdiag_pairs<<<(unsigned)((c->npairs + 255) / 256), 256, 0, st>>>(
          c->npairs, ptr<int4>(c->pr_rec), ptr<double>(c->factors), c->step, ptr<double>(c->W64), ptr<float>(c->W32),
          c->kstride);
    } else if (assembled) {
      if (!c->factors_stored) {  // the row pass left the factors out expecting the pair kernel: the same pass with them
        c->launches++;
        k_row_factors<<<blocks_for(n, 256), 256, 0, st>>>(scene_view(c), c->step, ptr<double>(c->factors),
                                                          ptr<double>(c->Wii), ptr<double>(c->Aii),
                                                          ptr<double>(c->rho_c), ptr<double>(c->B_c),
                                                          ptr<double>(c->V_c), ptr<double>(c->fe_part),
                                                          ptr<int>(c->bad), 1);
        c->factors_stored = true;
      }
      c->launches++;
      k_offdiag_assembled<<<blocks_for(K, 256), 256, 0, st>>>(
          n, K, ptr<int>(c->perm), ptr<int>(c->iperm), ptr<int>(c->adjptr), ptr<int>(c->adjcol), ptr<int>(c->adjbod),
          ptr<int>(c->master), ptr<double>(c->factors), c->step, ptr<int>(c->rowptr), ptr<int>(c->blkrow),
          ptr<int>(c->col), ptr<double>(c->W64), ptr<float>(c->W32), c->kstride);
    } else {
      c->launches++;
      k_offdiag_copy<<<blocks_for(n, wpb), wpb * kWarp, 0, st>>>(
          n, ptr<int>(c->perm), ptr<int>(c->iperm), ptr<int>(c->adjptr), ptr<int>(c->adjcol), ptr<double>(c->Woff_c),
          ptr<int>(c->rowptr), ptr<int>(c->col), ptr<double>(c->W64), ptr<float>(c->W32), c->kstride);
    }
  }
  B2_TRY(ensure(c->Wd, sizeof(double) * 9 * (n + 1)));
  B2_TRY(ensure(c->Ad, sizeof(double) * 9 * (n + 1)));
  B2_TRY(ensure(c->Bv, sizeof(double) * 3 * (n + 1)));
  B2_TRY(ensure(c->Vv, sizeof(double) * 3 * (n + 1)));
  B2_TRY(ensure(c->rho, sizeof(double) * (n + 1)));
  B2_TRY(ensure(c->gap, sizeof(double) * (n + 1)));
  B2_TRY(ensure(c->fric, sizeof(double) * (n + 1)));
  B2_TRY(ensure(c->rest, sizeof(double) * (n + 1)));
  B2_TRY(ensure(c->coh, sizeof(double) * (n + 1)));
  c->launches++;
  k_rows_permute<<<blocks_for(n, T), T, 0, st>>>(
      n, ptr<int>(c->perm), ptr<double>(c->Wii), ptr<double>(c->Aii), ptr<double>(c->rho_c), ptr<double>(c->B_c),
      ptr<double>(c->V_c), ptr<double>(c->gap_c), ptr<double>(c->fric_c), ptr<double>(c->rest_c),
      ptr<double>(c->coh_c), ptr<double>(c->Wd), ptr<double>(c->Ad), ptr<double>(c->Bv), ptr<double>(c->Vv),
      ptr<double>(c->rho), ptr<double>(c->gap), ptr<double>(c->fric), ptr<double>(c->rest), ptr<double>(c->coh));

  if (c->has_kinds) B2_TRY(permute_kinds(c));
  for (int b = 0; b < 3; b++) {
    B2_TRY(ensure(c->R64[b], sizeof(double4) * (n + 1)));
    B2_TRY(ensure(c->R32[b], sizeof(float4) * (n + 1)));
  }
  for (int b = 0; b < 2; b++) {
    B2_TRY(ensure(c->Us[b], sizeof(double4) * (n + 1)));
    B2_TRY(ensure(c->Um[b], sizeof(double4) * (n + 1)));
    B2_TRY(ensure(c->conmerit[b], sizeof(double) * (n + 1)));
  }
  B2_TRY(ensure(c->done, sizeof(int) * (n + 1)));
  if (!same_layout) {  // sorted CSR offsets and the problem of every sorted row, kept on the host for the tile table
    c->rowptr_h.assign(n + 1, 0);
    B2_CK(cudaMemcpyAsync(c->rowptr_h.data(), c->rowptr.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, st));
    c->rprob_h.assign(n, 0);
    if (c->nprob > 1 && n > 0) {
      std::vector<int> perm(n);
      B2_CK(cudaMemcpyAsync(perm.data(), c->perm.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
      B2_CK(cudaStreamSynchronize(st));
      for (int q = 0; q < n; q++)
        c->rprob_h[q] = (int)(std::upper_bound(c->prob_off.begin(), c->prob_off.end(), perm[q]) - c->prob_off.begin()) - 1;
    }
    B2_CK(cudaStreamSynchronize(st));
    B2_TRY(ensure(c->row_prob, sizeof(int) * (n + 1)));
    if (n > 0) B2_CK(cudaMemcpyAsync(c->row_prob.p, c->rprob_h.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  }
  if (!same_layout) B2_TRY(build_tiles(c, c->tile_rows));
  // new contacts start from R = U = 0 (MEM_Alloc zeroes, mem.c:64-86)
  B2_CK(cudaMemsetAsync(c->R64[0].p, 0, sizeof(double4) * (n + 1), st));
  B2_CK(cudaMemsetAsync(c->R32[0].p, 0, sizeof(float4) * (n + 1), st));
  B2_CK(cudaMemsetAsync(c->Us[0].p, 0, sizeof(double4) * (n + 1), st));
  B2_CK(cudaMemsetAsync(c->conmerit[0].p, 0, sizeof(double) * (n + 1), st));
  c->state_r = 0;
  c->state_u = &c->Us[0];
  c->state_cm = nullptr;
  B2_CK(cudaGetLastError());
  B2_CK(cudaStreamSynchronize(st));
  c->layout_valid = c->colour_valid;
  c->layout_nprob = c->nprob;
  c->layout_prob_off = c->prob_off;
  c->layout_tile_rows = c->tile_rows;
  c->ready = true;
  return B2DEV_OK;
}

template <class T>
int upload(b2dev_ctx* c, Buf& b, const T* src, size_t count, int on_device) {
  B2_TRY(ensure(b, sizeof(T) * (count + 1)));
  if (count == 0) return B2DEV_OK;
  if (!src) { set_err("null input array"); return B2DEV_EINVAL; }
  B2_CK(cudaMemcpyAsync(b.p, src, sizeof(T) * count, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        c->stream));
  return B2DEV_OK;
}

// Final iterate of every row into the state buffers R64[0], Us[0] and
// conmerit[0] (the problems of a batch return different iterates). Each row is
// read and written by one thread, so the copy may read its own destination.
__global__ void k_state_gather(int n, const int* __restrict__ row_prob, const ProblemControl* __restrict__ pc, int in,
                               int nomerit, double4* R0, double4* R1, double4* R2, double4* Us0, double4* Us1,
                               double4* Um0, double4* Um1, double* cm0, double* cm1) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const ProblemControl& q = pc[row_prob[p]];
  const int f = q.final_iter;
  double4* Rb[3] = {R0, R1, R2};
  const double4 r = Rb[(in + 1 + f) % 3][p];
  double4 u;
  double cm = 0.0;
  if (nomerit) {
    u = ((f + 1) & 1) ? Us1[p] : Us0[p];
  } else {
    const int ms = q.thrown ? f : f + 1;
    u = (ms & 1) ? Um1[p] : Um0[p];
    cm = (ms & 1) ? cm1[p] : cm0[p];
  }
  R0[p] = r;
  Us0[p] = u;
  if (!nomerit) cm0[p] = cm;
}

// Kernel arguments and launch shape of one persistent solve (nothing queued).
int solve_setup(b2dev_ctx* c, bool mixed, const b2dev_solve_opts* o, int maxiter, int iter0, int in,
                int u0_from_merit, int grid_req, SolveArgs* a, int* grid, size_t* smem) {
  const int n = c->n;
  const int P = c->nprob;
  const void* fn = c->has_kinds ? (mixed ? (const void*)k_solve_fp32_kinds : (const void*)k_solve_kinds<false>)
                                 : (mixed ? (const void*)k_solve_fp32 : (const void*)k_solve<false>);
  // enough warps for the tiles of about two sweeps in flight, capped by residency
  const int want = grid_req > 0 ? grid_req : blocks_for(2LL * c->ntiles, kSolveWarps);
  // staging window: the largest tile if the shared memory of the blocks that
  // registers allow per SM holds it, else windows
  int per_sm_regs = 0;
  B2_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_regs, fn, kSolveThreads, 0));
  per_sm_regs = std::max(1, per_sm_regs);
  const int smem_sm = 227 * 1024 - per_sm_regs * 1024;  // per-block reserve of the runtime
  const size_t per_block = mixed ? solve_smem_per_block<true>() : solve_smem_per_block<false>();
  const size_t fixed = mixed ? solve_smem_fixed<true>() : solve_smem_fixed<false>();
  const size_t per_warp = (size_t)smem_sm / per_sm_regs / kSolveWarps;
  const int gfit = per_warp > fixed + 64 * per_block ? (int)((per_warp - fixed) / per_block) & ~3 : 64;
  const int gwant = ((c->max_tile_blocks + 8) + 3) & ~3;
  int gcap = std::max(64, std::min(gwant, gfit));
  if (o->stage_blocks > 0) gcap = std::max(64, std::min(gcap, o->stage_blocks & ~3));
  const size_t wsm = mixed ? solve_warp_smem<true>(gcap) : solve_warp_smem<false>(gcap);
  *smem = wsm * kSolveWarps;
  B2_TRY(cooperative_grid(fn, kSolveThreads, c->sms, want, grid, *smem));
  const int pstride = o->maxiter + 2;
  B2_TRY(ensure(c->part, sizeof(double) * (3 * 4 * (size_t)c->ntiles + 4)));
  B2_TRY(ensure(c->decided, sizeof(int) * (size_t)P * pstride));
  B2_TRY(ensure(c->rer, sizeof(double) * (size_t)P * pstride));
  B2_TRY(ensure(c->mer, sizeof(double) * (size_t)P * pstride));
  B2_TRY(ensure(c->failkey, sizeof(unsigned long long) * (size_t)P * pstride));
  B2_TRY(ensure(c->failcount, sizeof(unsigned) * (size_t)P * pstride));
  B2_TRY(ensure(c->pctl, sizeof(ProblemControl) * P));
  if (c->trace_sweep >= 0 && iter0 == 0) B2_TRY(ensure(c->trace, sizeof(double) * kTraceStride * (n + 1)));

  SolveArgs& A = *a;
  memset(&A, 0, sizeof A);
  A.n = n;
  A.ntiles = c->ntiles;
  A.nprob = P;
  A.nactive = 0;
  for (int k = 0; k < P; k++) A.nactive += c->ptile_count[k] > 0 ? 1 : 0;
  A.tiles = ptr<int4>(c->tiles);
  A.tilek = ptr<int2>(c->tilek);
  A.ptile_ptr = ptr<int>(c->ptile_ptr);
  A.ptile = ptr<int>(c->ptile);
  A.done = ptr<int>(c->done);
  if (c->deps_valid) {
    A.depE_ptr = ptr<int>(c->depE_ptr); A.depE = ptr<int>(c->depE);
    A.depL_ptr = ptr<int>(c->depL_ptr); A.depL = ptr<int>(c->depL);
    A.tile_done = ptr<int>(c->tile_done);
  }
  A.decided = ptr<int>(c->decided);
  A.rowptr = ptr<int>(c->rowptr);
  A.col = ptr<int>(c->col);
  A.W64 = ptr<double>(c->W64);
  A.W32 = ptr<float>(c->W32);
  A.kstride = c->kstride;
  A.Wd = ptr<double>(c->Wd);
  A.Ad = ptr<double>(c->Ad);
  A.Bv = ptr<double>(c->Bv);
  A.Vv = ptr<double>(c->Vv);
  A.rho = ptr<double>(c->rho);
  A.gap = ptr<double>(c->gap);
  A.kind = c->has_kinds ? ptr<int>(c->kind_s) : nullptr;
  A.Zv = c->has_kinds ? ptr<double>(c->Z_s) : nullptr;
  A.fric = ptr<double>(c->fric);
  A.rest = ptr<double>(c->rest);
  A.coh = ptr<double>(c->coh);
  for (int b = 0; b < 3; b++) {
    A.R64[b] = ptr<double4>(c->R64[b]);
    A.R32[b] = ptr<float4>(c->R32[b]);
  }
  for (int b = 0; b < 2; b++) {
    A.Us[b] = ptr<double4>(c->Us[b]);
    A.Um[b] = ptr<double4>(c->Um[b]);
    A.conmerit[b] = ptr<double>(c->conmerit[b]);
  }
  A.part = ptr<double>(c->part);
  A.rerhist = ptr<double>(c->rer);
  A.merhist = ptr<double>(c->mer);
  A.failkey = ptr<unsigned long long>(c->failkey);
  A.failcount = ptr<unsigned>(c->failcount);
  A.pstride = pstride;
  A.free_energy = ptr<double>(c->pfe);
  A.ctrl = ptr<SolveControl>(c->sctrl);
  A.pctl = ptr<ProblemControl>(c->pctl);
  A.epsilon = o->epsilon;
  A.meritval = o->meritval;
  A.diagepsilon = o->diagepsilon;
  A.step = c->step;
  A.maxiter = maxiter;
  A.diagmaxiter = o->diagmaxiter;
  A.diagsolver = o->diagsolver;
  A.failure = o->failure;
  A.dynamic = c->dynamic;
  A.reverse = o->reverse;
  A.nomerit = o->nomerit;
  A.iter0 = iter0;
  A.in = in;
  A.u0_from_merit = u0_from_merit;
  A.gcap = gcap;
  A.warp_smem = (int)wsm;
  A.wait_ns = c->wait_ns;
  if (c->trace_sweep >= 0 && iter0 == 0) {
    A.trace = ptr<double>(c->trace);
    A.trace_sweep = c->trace_sweep;
  }
  return B2DEV_OK;
}

// Queue the control resets and the cooperative launch (no synchronisation,
// so the sequence can be captured into a CUDA graph).
int solve_enqueue(b2dev_ctx* c, bool mixed, const SolveArgs& a, int grid, size_t smem) {
  cudaStream_t st = c->stream;
  const int n = c->n, P = c->nprob;
  B2_CK(cudaMemsetAsync(c->sctrl.p, 0, sizeof(SolveControl), st));
  B2_CK(cudaMemsetAsync(c->pctl.p, 0, sizeof(ProblemControl) * P, st));
  B2_CK(cudaMemsetAsync(c->done.p, 0, sizeof(int) * (n + 1), st));
  if (a.tile_done) B2_CK(cudaMemsetAsync(a.tile_done, 0, sizeof(int) * (a.ntiles + 1), st));
  B2_CK(cudaMemsetAsync(c->decided.p, 0, sizeof(int) * (size_t)P * a.pstride, st));
  if (a.iter0 == 0) {
    B2_CK(cudaMemsetAsync(c->failkey.p, 0, sizeof(unsigned long long) * (size_t)P * a.pstride, st));
    B2_CK(cudaMemsetAsync(c->failcount.p, 0, sizeof(unsigned) * (size_t)P * a.pstride, st));
  } else {  // a continuation launch (one problem): its own sweeps only
    B2_CK(cudaMemsetAsync(ptr<unsigned long long>(c->failkey) + a.iter0, 0,
                          sizeof(unsigned long long) * (a.pstride - a.iter0), st));
    B2_CK(cudaMemsetAsync(ptr<unsigned>(c->failcount) + a.iter0, 0, sizeof(unsigned) * (a.pstride - a.iter0), st));
  }
  if (a.trace) B2_CK(cudaMemsetAsync(a.trace, 0, sizeof(double) * kTraceStride * (n + 1), st));
  const void* fn = c->has_kinds ? (mixed ? (const void*)k_solve_fp32_kinds : (const void*)k_solve_kinds<false>)
                                 : (mixed ? (const void*)k_solve_fp32 : (const void*)k_solve<false>);
  SolveArgs arg = a;
  void* args[] = {&arg};
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kSolveThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  c->launches++;
  B2_CK(cudaLaunchKernelExC(&cfg, fn, args));
  return B2DEV_OK;
}

// Floors of the FP32 sweeps' stopping rule in mixed precision: FP32 products
// carry relative rounding of about 6e-8, so iterate differences (the relative
// error) and merits (quadratic in the velocity residual) below these are not
// resolved by them; a tighter caller rule is met by the FP64 sweeps.
constexpr double kMixedEpsilonFloor = 1e-5;
constexpr double kMixedMeritFloor = 1e-10;

// One persistent solve launch, synchronised: per-problem outcomes in pc.
int solve_launch(b2dev_ctx* c, bool mixed, const b2dev_solve_opts* o, int maxiter, int iter0, int in,
                 int u0_from_merit, int grid_req, SolveControl* g, std::vector<ProblemControl>& pc, float* kernel_ms,
                 int* grid_used) {
  cudaStream_t st = c->stream;
  if (!u0_from_merit && c->state_u != &c->Us[0])  // the first sweep reads its U from Us[0]
    B2_CK(cudaMemcpyAsync(c->Us[0].p, c->state_u->p, sizeof(double4) * c->n, cudaMemcpyDeviceToDevice, st));
  SolveArgs a;
  int grid = 0;
  size_t smem = 0;
  B2_TRY(solve_setup(c, mixed, o, maxiter, iter0, in, u0_from_merit, grid_req, &a, &grid, &smem));
  B2_CK(cudaEventRecord(c->ev[4], st));
  B2_TRY(solve_enqueue(c, mixed, a, grid, smem));
  B2_CK(cudaEventRecord(c->ev[5], st));
  pc.assign(c->nprob, ProblemControl());
  B2_CK(cudaMemcpyAsync(g, c->sctrl.p, sizeof(SolveControl), cudaMemcpyDeviceToHost, st));
  B2_CK(cudaMemcpyAsync(pc.data(), c->pctl.p, sizeof(ProblemControl) * c->nprob, cudaMemcpyDeviceToHost, st));
  B2_CK(cudaStreamSynchronize(st));
  if (kernel_ms) cudaEventElapsedTime(kernel_ms, c->ev[4], c->ev[5]);
  if (grid_used) *grid_used = grid;
  if (g->timeout) { set_err("solve: a bounded device-side wait timed out"); return B2DEV_ETIMEOUT; }
  if (c->nprob == 1) {  // where the returned iterate's R, U and per-row merit live
    const int f = pc[0].final_iter;
    c->state_r = (in + 1 + f) % 3;
    if (o->nomerit) {
      c->state_u = &c->Us[(f + 1) & 1];
      c->state_cm = nullptr;
    } else {
      const int msweep = pc[0].thrown ? f : f + 1;  // sweep that evaluated the merit of the returned iterate
      c->state_u = &c->Um[msweep & 1];
      c->state_cm = &c->conmerit[msweep & 1];
    }
  } else {  // every problem's final iterate into the canonical buffers
    c->launches++;
    k_state_gather<<<blocks_for(c->n, 256), 256, 0, st>>>(
        c->n, ptr<int>(c->row_prob), ptr<ProblemControl>(c->pctl), in, o->nomerit, ptr<double4>(c->R64[0]),
        ptr<double4>(c->R64[1]), ptr<double4>(c->R64[2]), ptr<double4>(c->Us[0]), ptr<double4>(c->Us[1]),
        ptr<double4>(c->Um[0]), ptr<double4>(c->Um[1]), ptr<double>(c->conmerit[0]), ptr<double>(c->conmerit[1]));
    B2_CK(cudaGetLastError());
    c->state_r = 0;
    c->state_u = &c->Us[0];
    c->state_cm = o->nomerit ? nullptr : &c->conmerit[0];
  }
  return B2DEV_OK;
}

}  // namespace

extern "C" {

const char* b2dev_last_error(void) { return g_err; }

b2dev_ctx* b2dev_create(int device, void* stream) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    set_err("no CUDA device %d (found %d)", device, ndev);
    return nullptr;
  }
  DeviceGuard g(device);
  b2dev_ctx* c = new b2dev_ctx();
  c->device = device;
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
  if (!coop) {
    set_err("device %d does not support cooperative launches", device);
    delete c;
    return nullptr;
  }
  if (stream) {
    c->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      set_err("cudaStreamCreate failed");
      delete c;
      return nullptr;
    }
    c->own_stream = true;
  }
  for (int k = 0; k < 8; k++) cudaEventCreate(&c->ev[k]);
  if (ensure(c->sctrl, sizeof(SolveControl)) != B2DEV_OK || ensure(c->fe_dev, sizeof(double)) != B2DEV_OK ||
      ensure(c->bad, sizeof(int)) != B2DEV_OK) {
    b2dev_destroy(c);
    return nullptr;
  }
  return c;
}

void b2dev_destroy(b2dev_ctx* c) {
  if (!c) return;
  DeviceGuard g(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  Buf* all[] = {&c->rot, &c->x0, &c->jinv, &c->minv, &c->velo, &c->velo0, &c->obst, &c->master, &c->slave,
                &c->mpnt, &c->spnt, &c->base, &c->gap_c, &c->fric_c, &c->rest_c, &c->coh_c, &c->kind_c, &c->Z_c,
                &c->kind_s, &c->Z_s, &c->factors, &c->Wii,
                &c->Aii, &c->rho_c, &c->B_c, &c->V_c, &c->fe_part, &c->fe_dev, &c->bad, &c->bdeg, &c->bptr,
                &c->cursor, &c->brow, &c->deg, &c->adjptr, &c->adjcol, &c->adjbod, &c->Woff_c, &c->colour, &c->sel,
                &c->cctrl, &c->keys_out, &c->iota, &c->perm, &c->iperm, &c->colptr, &c->sdeg, &c->rowptr, &c->col,
                &c->W64, &c->W32, &c->Wd, &c->Ad, &c->Bv, &c->Vv, &c->rho, &c->gap, &c->fric, &c->rest, &c->coh,
                &c->R64[0], &c->R64[1], &c->R64[2], &c->R32[0], &c->R32[1], &c->R32[2], &c->Us[0], &c->Us[1],
                &c->Um[0], &c->Um[1], &c->conmerit[0], &c->conmerit[1], &c->done, &c->decided, &c->tiles, &c->tilek, &c->rtile, &c->dcnt, &c->depE_ptr, &c->depL_ptr, &c->depE, &c->depL, &c->tile_done, &c->rb_x, &c->rb_J, &c->rb_mass, &c->rb_scheme, &c->rb_fext, &c->rb_aux, &c->rb_loads, &c->rb_flags, &c->rb_fail, &c->tile_prob, &c->ptile_ptr, &c->ptile, &c->row_prob, &c->pctl, &c->pfe, &c->pvec, &c->gptr_prev, &c->gcol_prev,
                &c->part, &c->rer,
                &c->mer, &c->failkey, &c->failcount, &c->sctrl, &c->io, &c->cub_tmp, &c->trace,
                // contact detection: spheres, grid, pairs, staged and detected contacts, convexes
                &c->sph_body, &c->sph_ref, &c->sph_rad, &c->sph_surf, &c->sph_mat, &c->sph_cur, &c->sph_cell,
                &c->sph_hkey, &c->sph_hkey_s, &c->sph_idx, &c->sph_sorted, &c->sph_bstart, &c->sph_bend,
                &c->sph_cnt, &c->sph_off, &c->sph_pi, &c->sph_pj, &c->sph_rmax, &c->sph_total, &c->sph_keep,
                &c->sph_pos, &c->sph_bcnt, &c->sph_bptr, &c->sph_blist, &c->sph_pkey, &c->sph_pslo, &c->sph_pR,
                &c->sph_pU, &c->sph_ccnt, &c->st_master, &c->st_slave, &c->st_point, &c->st_mpnt, &c->st_spnt,
                &c->st_base, &c->st_gap, &c->st_fric, &c->st_rest, &c->st_coh, &c->st_R0, &c->st_U0, &c->st_key,
                &c->st_slo, &c->st_new, &c->det_point, &c->det_R0, &c->det_U0, &c->det_key, &c->det_slo,
                &c->det_new, &c->cvx_body, &c->cvx_vptr, &c->cvx_vert, &c->cvx_fptr, &c->cvx_fac, &c->cvx_sptr,
                &c->cvx_surf, &c->cvx_ns, &c->cvx_cur, &c->cvx_pla, &c->cvx_box, &c->cvx_aptr, &c->cvx_adj,
                &c->cc_lox, &c->cc_idx, &c->cc_sidx, &c->cc_cnt, &c->cc_off, &c->cc_keys, &c->cc_keys_s,
                &c->cc_cell, &c->cc_hkey, &c->cc_hkey_s, &c->cc_large, &c->cc_bstart, &c->cc_bend, &c->cc_misc, &c->cc_keep, &c->cc_cls, &c->cc_order, &c->ex_bodies, &c->ex_surf,
                &c->st_area, &c->det_area, &c->cn_kind, &c->cn_master, &c->cn_slave, &c->cn_mpnt, &c->cn_spnt,
                &c->cn_base, &c->cn_Z,
                &c->topo_m, &c->topo_s, &c->topo_o, &c->topo_flag, &c->blkrow, &c->pr_cnt, &c->pr_ptr,
                &c->pr_rec};
  for (Buf* b : all)
    if (b->p) cudaFree(b->p);
  if (c->graph) cudaGraphExecDestroy(c->graph);
  if (c->pinned) cudaFreeHost(c->pinned);
  for (int k = 0; k < 8; k++)
    if (c->ev[k]) cudaEventDestroy(c->ev[k]);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  delete c;
}

void* b2dev_stream(b2dev_ctx* c) { return c ? (void*)c->stream : nullptr; }

int b2dev_upload_scene(b2dev_ctx* c, int nbod, const double* rot, const double* x0, const double* jinv,
                       const double* minv, const double* velo, const double* velo0, const int* obstacle, int ncon,
                       const int* master, const int* slave, const double* mpnt, const double* spnt,
                       const double* base, const double* gap, const double* friction, const double* restitution,
                       const double* cohesion, int on_device) {
  if (!c || nbod < 0 || ncon < 0) { set_err("invalid scene sizes"); return B2DEV_EINVAL; }
  DeviceGuard g(c->device);
  c->nbod = nbod;
  c->ncon = ncon;
  B2_TRY(upload(c, c->rot, rot, (size_t)9 * nbod, on_device));
  B2_TRY(upload(c, c->x0, x0, (size_t)3 * nbod, on_device));
  B2_TRY(upload(c, c->jinv, jinv, (size_t)9 * nbod, on_device));
  B2_TRY(upload(c, c->minv, minv, (size_t)nbod, on_device));
  B2_TRY(upload(c, c->velo, velo, (size_t)6 * nbod, on_device));
  B2_TRY(upload(c, c->velo0, velo0, (size_t)6 * nbod, on_device));
  B2_TRY(upload(c, c->obst, obstacle, (size_t)nbod, on_device));
  B2_TRY(upload(c, c->master, master, (size_t)ncon, on_device));
  B2_TRY(upload(c, c->slave, slave, (size_t)ncon, on_device));
  B2_TRY(upload(c, c->mpnt, mpnt, (size_t)3 * ncon, on_device));
  B2_TRY(upload(c, c->spnt, spnt, (size_t)3 * ncon, on_device));
  B2_TRY(upload(c, c->base, base, (size_t)9 * ncon, on_device));
  B2_TRY(upload(c, c->gap_c, gap, (size_t)ncon, on_device));
  B2_TRY(upload(c, c->fric_c, friction, (size_t)ncon, on_device));
  B2_TRY(upload(c, c->rest_c, restitution, (size_t)ncon, on_device));
  B2_TRY(upload(c, c->coh_c, cohesion, (size_t)ncon, on_device));
  c->have_scene = true;
  c->have_rigid = false;  // b2dev_rigid_setup again for the new bodies
  c->det_valid = c->det_assembled = false;
  c->ready = false;
  c->has_kinds = false;   // new constraints: all contacts until b2dev_set_kinds
  c->cn_n = 0;            // constraints kept across detections refer to the old bodies
  c->det_ncont = 0;
  return B2DEV_OK;
}

int b2dev_set_kinds(b2dev_ctx* c, int n, const int* kind, const double* Z, int on_device) {
  if (!c) { set_err("set_kinds: null context"); return B2DEV_EINVAL; }
  const int rows = c->ready ? c->n : c->ncon;
  if (n != rows) { set_err("set_kinds: %d rows given, the problem has %d", n, rows); return B2DEV_EINVAL; }
  DeviceGuard g(c->device);
  if (!kind) { c->has_kinds = false; return B2DEV_OK; }
  std::vector<int> k(n);
  std::vector<double> z(4 * (size_t)n, 0.0);
  if (on_device) {
    if (n) B2_CK(cudaMemcpy(k.data(), kind, sizeof(int) * n, cudaMemcpyDeviceToHost));
    if (n && Z) B2_CK(cudaMemcpy(z.data(), Z, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost));
  } else {
    std::copy(kind, kind + n, k.begin());
    if (Z) std::copy(Z, Z + 4 * (size_t)n, z.begin());
  }
  bool any = false;
  for (int i = 0; i < n; i++) {
    if (k[i] < CON_CONTACT || k[i] > CON_RIGLNK) {
      set_err("set_kinds: row %d: kind %d is not CONTACT, FIXPNT, FIXDIR, VELODIR, VELODIR3 or RIGLNK (0-5)", i, k[i]);
      return B2DEV_EUNSUPPORTED;
    }
    any = any || k[i] != CON_CONTACT;
  }
  B2_TRY(upload(c, c->kind_c, k.data(), (size_t)n, 0));
  B2_TRY(upload(c, c->Z_c, z.data(), z.size(), 0));
  c->has_kinds = any;
  if (any && c->ready) B2_TRY(permute_kinds(c));
  B2_CK(cudaStreamSynchronize(c->stream));
  return B2DEV_OK;
}

int b2dev_assemble(b2dev_ctx* c, double step, int dynamic, uint64_t colour_seed) {
  if (!c || !c->have_scene) { set_err("assemble: no scene uploaded"); return B2DEV_ESTATE; }
  if (!(step > 0.0)) { set_err("assemble: step must be positive"); return B2DEV_EINVAL; }
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  const int T = 256;
  const int n = c->ncon, nb = c->nbod;
  if (c->nprob > 1 && ((int)c->prob_off.size() != c->nprob + 1 || c->prob_off.back() != n)) {
    set_err("assemble: the problem offsets do not cover the %d contacts", n);
    return B2DEV_EINVAL;
  }
  c->n = n;
  c->step = step;
  c->dynamic = dynamic ? 1 : 0;
  c->assembled_mode = true;
  c->det_assembled = c->det_valid;
  assemble_time(c);  // the previous assembly's events before they are recorded again
  B2_CK(cudaEventRecord(c->ev[0], st));

  B2_TRY(ensure(c->factors, sizeof(double) * kFactorStride * (n + 1)));
  B2_TRY(ensure(c->Wii, sizeof(double) * 9 * (n + 1)));
  B2_TRY(ensure(c->Aii, sizeof(double) * 9 * (n + 1)));
  B2_TRY(ensure(c->rho_c, sizeof(double) * (n + 1)));
  B2_TRY(ensure(c->B_c, sizeof(double) * 3 * (n + 1)));
  B2_TRY(ensure(c->V_c, sizeof(double) * 3 * (n + 1)));
  const int rb = blocks_for(n, T);
  B2_TRY(ensure(c->fe_part, sizeof(double) * rb));
  B2_CK(cudaMemsetAsync(c->bad.p, 0, sizeof(int), st));
  // is the contact topology that of the last contact graph? (checked with the
  // body indices below, in one synchronisation)
  const bool topo_cand = c->topo_valid && c->topo_n == n && c->topo_nb == nb && n > 0;
  if (topo_cand) {
    B2_TRY(ensure(c->topo_flag, sizeof(int)));
    B2_CK(cudaMemsetAsync(c->topo_flag.p, 0, sizeof(int), st));
    c->launches++;
    k_topology_diff<<<std::max(1, std::min(4 * c->sms, blocks_for(std::max(n, nb), T))), T, 0, st>>>(
        n, nb, ptr<int>(c->master), ptr<int>(c->slave), ptr<int>(c->obst), ptr<int>(c->topo_m), ptr<int>(c->topo_s),
        ptr<int>(c->topo_o), ptr<int>(c->topo_flag));
  }

  SceneDev sc;
  sc.nbod = nb; sc.ncon = n;
  sc.rot = ptr<double>(c->rot); sc.x0 = ptr<double>(c->x0); sc.jinv = ptr<double>(c->jinv);
  sc.minv = ptr<double>(c->minv); sc.velo = ptr<double>(c->velo); sc.velo0 = ptr<double>(c->velo0);
  sc.obstacle = ptr<int>(c->obst); sc.master = ptr<int>(c->master); sc.slave = ptr<int>(c->slave);
  sc.mpnt = ptr<double>(c->mpnt); sc.spnt = ptr<double>(c->spnt); sc.base = ptr<double>(c->base);
  // a kept layout whose body-pair table is valid forms the factors in the
  // pair kernel: none are stored (if the topology check below fails, the rows
  // are assembled again with the factors)
  const bool formed = c->pairs_valid && topo_cand;
  c->launches++;
  k_row_factors<<<rb, T, 0, st>>>(sc, step, ptr<double>(c->factors), ptr<double>(c->Wii), ptr<double>(c->Aii),
                                  ptr<double>(c->rho_c), ptr<double>(c->B_c), ptr<double>(c->V_c),
                                  ptr<double>(c->fe_part), ptr<int>(c->bad), formed ? 0 : 1);
  c->launches++;
  k_sum_partials<<<1, 1024, 0, st>>>(ptr<double>(c->fe_part), rb, ptr<double>(c->fe_dev));
  B2_TRY(ensure(c->pfe, sizeof(double) * (c->nprob + 1)));
  if (c->nprob == 1) {
    B2_CK(cudaMemcpyAsync(c->pfe.p, c->fe_dev.p, sizeof(double), cudaMemcpyDeviceToDevice, st));
  } else {  // free energy of every problem (rows of each problem in caller order)
    B2_TRY(ensure(c->pvec, sizeof(int) * (c->nprob + 1)));
    B2_CK(cudaMemcpyAsync(c->pvec.p, c->prob_off.data(), sizeof(int) * (c->nprob + 1), cudaMemcpyHostToDevice, st));
    c->launches++;
    k_problem_free_energy<<<c->nprob, 256, 0, st>>>(ptr<int>(c->pvec), ptr<double>(c->Aii), ptr<double>(c->B_c),
                                                    ptr<double>(c->pfe));
  }
  bool same_topo = false;
  {  // body indices are checked before any kernel indexes per-body arrays with them
    int flags[2] = {0, 1};
    B2_CK(cudaMemcpyAsync(&flags[0], c->bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (topo_cand) B2_CK(cudaMemcpyAsync(&flags[1], c->topo_flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaMemcpyAsync(&c->free_energy, c->fe_dev.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaStreamSynchronize(st));
    if (flags[0]) { set_err("assemble: self-contact or invalid body index (outside the rigid contact path)"); return B2DEV_EUNSUPPORTED; }
    same_topo = topo_cand && flags[1] == 0;
  }
  c->factors_stored = !formed;  // prepare_layout writes them after all if the per-block kernel runs
  if (same_topo) {  // the contact graph of the last assembly holds (adjptr, adjcol, adjbod, K)
    B2_TRY(prepare_layout(c, colour_seed, true, true));
    B2_CK(cudaEventRecord(c->ev[1], st));  // read when asked (b2dev_last_assemble_ms): no synchronisation here
    c->assemble_ms_pending = true;
    return B2DEV_OK;
  }
  c->topo_valid = false;

  // contact graph through shared non-obstacle bodies
  B2_TRY(ensure(c->bdeg, sizeof(int) * (nb + 1)));
  B2_TRY(ensure(c->bptr, sizeof(int) * (nb + 1)));
  B2_TRY(ensure(c->cursor, sizeof(int) * (nb + 1)));
  B2_CK(cudaMemsetAsync(c->bdeg.p, 0, sizeof(int) * (nb + 1), st));
  B2_CK(cudaMemsetAsync(c->cursor.p, 0, sizeof(int) * (nb + 1), st));
  c->launches++;
  k_body_count<<<rb, T, 0, st>>>(n, ptr<int>(c->master), ptr<int>(c->slave), ptr<int>(c->obst), ptr<int>(c->bdeg));
  B2_TRY(scan_exclusive(c, ptr<int>(c->bdeg), ptr<int>(c->bptr), nb + 1));
  B2_TRY(ensure(c->brow, sizeof(int) * (2 * (size_t)n + 1)));
  c->launches++;
  k_body_fill<<<rb, T, 0, st>>>(n, ptr<int>(c->master), ptr<int>(c->slave), ptr<int>(c->obst), ptr<int>(c->bptr),
                                ptr<int>(c->cursor), ptr<int>(c->brow));
  c->launches++;
  k_body_sort<<<blocks_for(nb, T), T, 0, st>>>(nb, ptr<int>(c->bptr), ptr<int>(c->brow));
  B2_TRY(ensure(c->deg, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->adjptr, sizeof(int) * (n + 1)));
  c->launches++;
  k_row_degree<<<rb, T, 0, st>>>(n, ptr<int>(c->master), ptr<int>(c->slave), ptr<int>(c->obst), ptr<int>(c->bptr),
                                 ptr<int>(c->deg));
  c->launches++;
  k_set_last_zero<<<1, 32, 0, st>>>(ptr<int>(c->deg), n);
  B2_TRY(scan_exclusive(c, ptr<int>(c->deg), ptr<int>(c->adjptr), n + 1));
  int K = 0, bad = 0;
  B2_CK(cudaMemcpyAsync(&K, ptr<int>(c->adjptr) + n, sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CK(cudaMemcpyAsync(&bad, c->bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CK(cudaMemcpyAsync(&c->free_energy, c->fe_dev.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  B2_CK(cudaStreamSynchronize(st));
  if (bad) { set_err("assemble: self-contact or invalid body index (outside the rigid contact path)"); return B2DEV_EUNSUPPORTED; }
  if (K < 0) { set_err("assemble: block count overflows 32-bit indexing"); return B2DEV_EINVAL; }
  c->K = K;
  B2_TRY(ensure(c->adjcol, sizeof(int) * ((size_t)K + 1)));
  B2_TRY(ensure(c->adjbod, sizeof(int) * ((size_t)K + 1)));
  c->launches++;
  k_adj_fill<<<rb, T, 0, st>>>(n, ptr<int>(c->master), ptr<int>(c->slave), ptr<int>(c->obst), ptr<int>(c->bptr),
                               ptr<int>(c->brow), ptr<int>(c->adjptr), ptr<int>(c->adjcol), ptr<int>(c->adjbod));
  // the topology this graph belongs to
  B2_TRY(ensure(c->topo_m, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->topo_s, sizeof(int) * (n + 1)));
  B2_TRY(ensure(c->topo_o, sizeof(int) * (nb + 1)));
  if (n > 0) {
    B2_CK(cudaMemcpyAsync(c->topo_m.p, c->master.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
    B2_CK(cudaMemcpyAsync(c->topo_s.p, c->slave.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
  }
  if (nb > 0) B2_CK(cudaMemcpyAsync(c->topo_o.p, c->obst.p, sizeof(int) * nb, cudaMemcpyDeviceToDevice, st));
  c->topo_n = n;
  c->topo_nb = nb;
  c->topo_valid = true;
  B2_TRY(prepare_layout(c, colour_seed, true, false));
  B2_CK(cudaEventRecord(c->ev[1], st));
  c->assemble_ms_pending = true;
  return B2DEV_OK;
}

int b2dev_upload_locdyn(b2dev_ctx* c, int n, const double* W, const double* A, const double* rho, const double* B,
                        const double* V, const double* gap, const double* friction, const double* restitution,
                        const double* cohesion, const int* adjptr, const int* adjcol, const double* Woff,
                        double free_energy, double step, int dynamic, uint64_t colour_seed, int on_device) {
  if (!c || n < 0 || !adjptr) { set_err("invalid local dynamics"); return B2DEV_EINVAL; }
  DeviceGuard g(c->device);
  int K = 0;
  if (on_device) {
    if (n > 0) B2_CK(cudaMemcpy(&K, adjptr + n, sizeof(int), cudaMemcpyDeviceToHost));
    if (K < 0) { set_err("adjptr[n] negative"); return B2DEV_EINVAL; }
  } else {
    K = adjptr[n];
    if (adjptr[0] != 0) { set_err("adjptr[0] must be 0"); return B2DEV_EINVAL; }
    for (int i = 0; i < n; i++)
      if (adjptr[i + 1] < adjptr[i]) { set_err("adjptr not monotone at row %d", i); return B2DEV_EINVAL; }
    for (int k = 0; k < K; k++)
      if (adjcol[k] < 0 || adjcol[k] >= n) { set_err("adjcol[%d] = %d out of range", k, adjcol[k]); return B2DEV_EINVAL; }
  }
  c->n = n;
  c->K = K;
  c->step = step;
  c->dynamic = dynamic ? 1 : 0;
  c->free_energy = free_energy;
  c->has_kinds = false;  // new rows: all contacts until b2dev_set_kinds
  B2_TRY(ensure(c->pfe, sizeof(double) * 2));
  B2_CK(cudaMemcpyAsync(c->pfe.p, &c->free_energy, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  c->assembled_mode = false;
  B2_TRY(upload(c, c->Wii, W, (size_t)9 * n, on_device));
  B2_TRY(upload(c, c->Aii, A, (size_t)9 * n, on_device));
  B2_TRY(upload(c, c->rho_c, rho, (size_t)n, on_device));
  B2_TRY(upload(c, c->B_c, B, (size_t)3 * n, on_device));
  B2_TRY(upload(c, c->V_c, V, (size_t)3 * n, on_device));
  B2_TRY(upload(c, c->gap_c, gap, (size_t)n, on_device));
  B2_TRY(upload(c, c->fric_c, friction, (size_t)n, on_device));
  B2_TRY(upload(c, c->rest_c, restitution, (size_t)n, on_device));
  B2_TRY(upload(c, c->coh_c, cohesion, (size_t)n, on_device));
  B2_TRY(upload(c, c->adjptr, adjptr, (size_t)n + 1, on_device));
  B2_TRY(upload(c, c->adjcol, adjcol, (size_t)K, on_device));
  B2_TRY(upload(c, c->Woff_c, Woff, (size_t)9 * K, on_device));
  if (on_device && n > 0) {  // device-resident graph: check it before the colouring walks it
    B2_CK(cudaMemsetAsync(c->bad.p, 0, sizeof(int), c->stream));
    c->launches++;
    k_check_graph<<<blocks_for(n, 256), 256, 0, c->stream>>>(n, K, ptr<int>(c->adjptr), ptr<int>(c->adjcol),
                                                             ptr<int>(c->bad));
    int bad = 0;
    B2_CK(cudaMemcpyAsync(&bad, c->bad.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    B2_CK(cudaStreamSynchronize(c->stream));
    if (bad) { set_err("adjptr/adjcol out of range"); return B2DEV_EINVAL; }
  }
  c->topo_valid = false;  // the contact graph buffers now hold the uploaded one
  return prepare_layout(c, colour_seed, false, false);
}

int b2dev_set_state(b2dev_ctx* c, const double* R, const double* U, int on_device) {
  if (!c || !c->ready) { set_err("set_state: no local dynamics"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  const int n = c->n;
  cudaStream_t st = c->stream;
  B2_TRY(ensure(c->io, sizeof(double) * 6 * (n + 1)));
  double* dR = ptr<double>(c->io);
  double* dU = dR + 3 * (size_t)(n + 1);
  if (n > 0) {
    const cudaMemcpyKind kd = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (R) B2_CK(cudaMemcpyAsync(dR, R, sizeof(double) * 3 * n, kd, st));
    else B2_CK(cudaMemsetAsync(dR, 0, sizeof(double) * 3 * n, st));
    if (U) B2_CK(cudaMemcpyAsync(dU, U, sizeof(double) * 3 * n, kd, st));
    else B2_CK(cudaMemsetAsync(dU, 0, sizeof(double) * 3 * n, st));
    c->launches++;
    k_state_in<<<blocks_for(n, 256), 256, 0, st>>>(n, ptr<int>(c->perm), dR, dU, ptr<double4>(c->R64[0]),
                                                   ptr<float4>(c->R32[0]), ptr<double4>(c->Us[0]));
  }
  c->state_r = 0;
  c->state_u = &c->Us[0];
  c->state_cm = nullptr;
  B2_CK(cudaGetLastError());
  return B2DEV_OK;
}

// ---- rigid time integration (bod.c:1313-1493) ----

static RigidDev rigid_view(b2dev_ctx* c) {
  RigidDev d;
  d.nbod = c->nbod;
  d.rot = ptr<double>(c->rot); d.x = ptr<double>(c->rb_x); d.velo = ptr<double>(c->velo);
  d.velo0 = ptr<double>(c->velo0); d.fext = ptr<double>(c->rb_fext); d.aux = ptr<double>(c->rb_aux);
  d.J = ptr<double>(c->rb_J); d.jinv = ptr<double>(c->jinv); d.mass = ptr<double>(c->rb_mass);
  d.minv = ptr<double>(c->minv); d.scheme = ptr<int>(c->rb_scheme); d.obstacle = ptr<int>(c->obst);
  d.flags = c->rb_have_flags ? ptr<int>(c->rb_flags) : nullptr;
  d.fail = ptr<int>(c->rb_fail);
  return d;
}

// a failed NEW3 Newton solve of an earlier step end (bod.c:196, 206)
static int rigid_failures(b2dev_ctx* c) {
  if (!c->rb_imp) return B2DEV_OK;
  int fail = 0;
  B2_CK(cudaMemcpyAsync(&fail, c->rb_fail.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  B2_CK(cudaStreamSynchronize(c->stream));
  if (fail) {
    set_err("BODY_Dynamic_Step_End: NEW3 (RIG_IMP) %s", (fail & 1) ? "singular Jacobian in the Newton solve"
                                                                   : "Newton solve not converged in 50 steps");
    return B2DEV_EINVAL;
  }
  return B2DEV_OK;
}

int b2dev_rigid_flags(b2dev_ctx* c, const int* flags, int on_device) {
  if (!c || !c->have_rigid) { set_err("rigid_flags: no rigid bodies set up"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  if (!flags) { c->rb_have_flags = false; return B2DEV_OK; }
  B2_TRY(upload(c, c->rb_flags, flags, (size_t)c->nbod, on_device));
  B2_CK(cudaStreamSynchronize(c->stream));
  c->rb_have_flags = true;
  return B2DEV_OK;
}

int b2dev_rigid_setup(b2dev_ctx* c, const double* J, const double* mass, const double* x, const int* scheme,
                      int on_device) {
  if (!c || !c->have_scene) { set_err("rigid_setup: no scene uploaded"); return B2DEV_ESTATE; }
  if (!J || !mass || !x) { set_err("rigid_setup: inertia, mass and mass centre are required"); return B2DEV_EINVAL; }
  DeviceGuard g(c->device);
  const int nb = c->nbod;
  std::vector<int> sch(nb, SCH_RIG_NEG);  // the reference's default (bod.c:1008)
  if (scheme) {
    if (on_device) {
      B2_CK(cudaMemcpy(sch.data(), scheme, sizeof(int) * nb, cudaMemcpyDeviceToHost));
    } else {
      std::copy(scheme, scheme + nb, sch.begin());
    }
    for (int b = 0; b < nb; b++)
      if (sch[b] != SCH_RIG_POS && sch[b] != SCH_RIG_NEG && sch[b] != SCH_RIG_IMP) {
        set_err("rigid_setup: body %d: scheme %d is not RIG_POS (0), RIG_NEG (1) or RIG_IMP (2)", b, sch[b]);
        return B2DEV_EUNSUPPORTED;
      }
  }
  c->rb_imp = std::find(sch.begin(), sch.end(), (int)SCH_RIG_IMP) != sch.end();
  c->rb_have_flags = false;
  B2_TRY(upload(c, c->rb_J, J, (size_t)9 * nb, on_device));
  B2_TRY(upload(c, c->rb_mass, mass, (size_t)nb, on_device));
  B2_TRY(upload(c, c->rb_x, x, (size_t)3 * nb, on_device));
  B2_TRY(upload(c, c->rb_scheme, sch.data(), (size_t)nb, 0));
  B2_TRY(ensure(c->rb_fext, sizeof(double) * 6 * (nb + 1)));
  B2_TRY(ensure(c->rb_aux, sizeof(double) * 3 * (nb + 1)));
  B2_CK(cudaMemsetAsync(c->rb_aux.p, 0, sizeof(double) * 3 * (nb + 1), c->stream));
  B2_TRY(ensure(c->rb_fail, sizeof(int)));
  B2_CK(cudaMemsetAsync(c->rb_fail.p, 0, sizeof(int), c->stream));
  B2_CK(cudaStreamSynchronize(c->stream));
  c->have_rigid = true;
  return B2DEV_OK;
}

int b2dev_rigid_step_begin(b2dev_ctx* c, double step, const double* gravity, const double* loads, int on_device) {
  if (!c || !c->have_rigid) { set_err("rigid_step_begin: no rigid bodies set up"); return B2DEV_ESTATE; }
  if (!(step > 0.0)) { set_err("rigid_step_begin: step must be positive"); return B2DEV_EINVAL; }
  DeviceGuard g(c->device);
  B2_TRY(rigid_failures(c));
  const int nb = c->nbod;
  if (nb == 0) return B2DEV_OK;
  const double* dl = nullptr;
  if (loads) {
    B2_TRY(upload(c, c->rb_loads, loads, (size_t)9 * nb, on_device));
    dl = ptr<double>(c->rb_loads);
  }
  const double g0 = gravity ? gravity[0] : 0.0, g1 = gravity ? gravity[1] : 0.0, g2 = gravity ? gravity[2] : 0.0;
  c->launches++;
  k_rigid_begin<<<blocks_for(nb, 128), 128, 0, c->stream>>>(rigid_view(c), step, g0, g1, g2, dl);
  B2_CK(cudaGetLastError());
  c->ready = false;  // the bodies moved: the local dynamics must be assembled again
  return B2DEV_OK;
}

int b2dev_rigid_step_end(b2dev_ctx* c, double step) {
  if (!c || !c->have_rigid) { set_err("rigid_step_end: no rigid bodies set up"); return B2DEV_ESTATE; }
  const bool contacts = c->ncon > 0;  // without contacts there are no reactions to apply
  if (contacts && (!c->ready || !c->assembled_mode)) {
    set_err("rigid_step_end: no solved local dynamics of these bodies");
    return B2DEV_ESTATE;
  }
  if (!(step > 0.0)) { set_err("rigid_step_end: step must be positive"); return B2DEV_EINVAL; }
  DeviceGuard g(c->device);
  const int nb = c->nbod;
  if (nb == 0) return B2DEV_OK;
  c->launches++;
  k_rigid_end<<<blocks_for(nb, 128), 128, 0, c->stream>>>(
      rigid_view(c), step, ptr<double>(c->x0), contacts ? ptr<int>(c->master) : nullptr,
      contacts ? ptr<double>(c->mpnt) : nullptr, contacts ? ptr<double>(c->spnt) : nullptr,
      contacts ? ptr<double>(c->base) : nullptr, contacts ? ptr<int>(c->bptr) : nullptr,
      contacts ? ptr<int>(c->brow) : nullptr, contacts ? ptr<double4>(c->R64[c->state_r]) : nullptr,
      contacts ? ptr<int>(c->iperm) : nullptr);
  B2_CK(cudaGetLastError());
  return B2DEV_OK;
}

int b2dev_rigid_get(b2dev_ctx* c, double* rot, double* x, double* velo, double* velo0, int on_device) {
  if (!c || !c->have_rigid) { set_err("rigid_get: no rigid bodies set up"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  const int nb = c->nbod;
  cudaStream_t st = c->stream;
  const cudaMemcpyKind kd = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (nb > 0) {
    if (rot) B2_CK(cudaMemcpyAsync(rot, c->rot.p, sizeof(double) * 9 * nb, kd, st));
    if (x) B2_CK(cudaMemcpyAsync(x, c->rb_x.p, sizeof(double) * 3 * nb, kd, st));
    if (velo) B2_CK(cudaMemcpyAsync(velo, c->velo.p, sizeof(double) * 6 * nb, kd, st));
    if (velo0) B2_CK(cudaMemcpyAsync(velo0, c->velo0.p, sizeof(double) * 6 * nb, kd, st));
  }
  B2_CK(cudaStreamSynchronize(st));
  return rigid_failures(c);
}

int b2dev_update_constraints(b2dev_ctx* c) {
  if (!c || !c->have_rigid) { set_err("update_constraints: no rigid bodies set up"); return B2DEV_ESTATE; }
  if (!c->has_kinds || c->ncon == 0) return B2DEV_OK;  // contacts only: nothing to update
  DeviceGuard g(c->device);
  B2_TRY(ensure(c->bad, sizeof(int)));
  B2_CK(cudaMemsetAsync(c->bad.p, 0, sizeof(int), c->stream));
  c->launches++;
  k_constraints_update<<<blocks_for(c->ncon, 128), 128, 0, c->stream>>>(
      c->ncon, c->nbod, ptr<int>(c->kind_c), ptr<int>(c->master), ptr<int>(c->slave), ptr<double>(c->rot),
      ptr<double>(c->rb_x), ptr<double>(c->x0), ptr<double>(c->mpnt), ptr<double>(c->spnt), ptr<double>(c->base),
      ptr<double>(c->gap_c), ptr<double>(c->Z_c), ptr<int>(c->bad));
  B2_CK(cudaGetLastError());
  int bad = 0;
  B2_CK(cudaMemcpyAsync(&bad, c->bad.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  B2_CK(cudaStreamSynchronize(c->stream));
  if (bad) { set_err("update_constraints: a constraint's body index is out of range"); return B2DEV_EINVAL; }
  c->ready = false;  // frames and gaps changed: the local dynamics must be assembled again
  return B2DEV_OK;
}

int b2dev_constraints_setup(b2dev_ctx* c, int n, const int* kind, const int* master, const int* slave,
                            const double* mpnt, const double* spnt, const double* base, const double* Z) {
  if (!c || !c->have_scene) { set_err("constraints_setup: no scene uploaded"); return B2DEV_ESTATE; }
  if (n < 0 || (n > 0 && (!kind || !master || !slave || !mpnt || !spnt || !base || !Z))) {
    set_err("constraints_setup: %d constraints need kind, bodies, points, base and Z", n);
    return B2DEV_EINVAL;
  }
  for (int j = 0; j < n; j++) {
    if (kind[j] < CON_FIXPNT || kind[j] > CON_RIGLNK) {
      set_err("constraints_setup: constraint %d: kind %d is not FIXPNT, FIXDIR, VELODIR, VELODIR3 or RIGLNK (1-5)",
              j, kind[j]);
      return B2DEV_EUNSUPPORTED;
    }
    if (master[j] < 0 || master[j] >= c->nbod || slave[j] < -1 || slave[j] >= c->nbod || slave[j] == master[j]) {
      set_err("constraints_setup: constraint %d: bodies %d, %d out of range or equal", j, master[j], slave[j]);
      return B2DEV_EINVAL;
    }
  }
  DeviceGuard g(c->device);
  B2_TRY(upload(c, c->cn_kind, kind, (size_t)n, 0));
  B2_TRY(upload(c, c->cn_master, master, (size_t)n, 0));
  B2_TRY(upload(c, c->cn_slave, slave, (size_t)n, 0));
  B2_TRY(upload(c, c->cn_mpnt, mpnt, (size_t)3 * n, 0));
  B2_TRY(upload(c, c->cn_spnt, spnt, (size_t)3 * n, 0));
  B2_TRY(upload(c, c->cn_base, base, (size_t)9 * n, 0));
  B2_TRY(upload(c, c->cn_Z, Z, (size_t)4 * n, 0));
  B2_CK(cudaStreamSynchronize(c->stream));
  c->cn_n = n;
  return B2DEV_OK;
}

// ---- contact update and detection between spheres (dom.c:3700-3790) ----

int b2dev_spheres_setup(b2dev_ctx* c, int nsph, const int* body, const double* centre, const double* radius,
                        const int* surface, int nsurf, const double* material, int on_device) {
  if (!c || !c->have_scene) { set_err("spheres_setup: no scene uploaded"); return B2DEV_ESTATE; }
  if (nsph < 0 || (nsph > 0 && (!body || !centre || !radius || !surface)) || nsurf <= 0 || !material) {
    set_err("spheres_setup: invalid arguments");
    return B2DEV_EINVAL;
  }
  if (nsph > (1 << 30)) { set_err("spheres_setup: %d spheres exceed the pair key range", nsph); return B2DEV_EINVAL; }
  for (int a = 0; a < nsurf; a++)
    for (int b = 0; b < nsurf; b++)
      for (int v = 0; v < 2; v++)
        if (material[2 * ((size_t)a * nsurf + b) + v] != material[2 * ((size_t)b * nsurf + a) + v]) {
          set_err("spheres_setup: the material table is not symmetric at surfaces (%d, %d)", a, b);
          return B2DEV_EINVAL;
        }
  DeviceGuard g(c->device);
  c->nsph = nsph;
  c->nsurf = nsurf;
  c->sph_mat_h.assign(material, material + 2 * (size_t)nsurf * nsurf);
  B2_TRY(upload(c, c->sph_body, body, (size_t)nsph, on_device));
  B2_TRY(upload(c, c->sph_ref, centre, (size_t)3 * nsph, on_device));
  B2_TRY(upload(c, c->sph_rad, radius, (size_t)nsph, on_device));
  B2_TRY(upload(c, c->sph_surf, surface, (size_t)nsph, on_device));
  B2_TRY(upload(c, c->sph_mat, c->sph_mat_h.data(), c->sph_mat_h.size(), 0));
  B2_CK(cudaStreamSynchronize(c->stream));
  c->det_valid = c->det_assembled = false;
  return B2DEV_OK;
}

int b2dev_convexes_setup(b2dev_ctx* c, int nconv, const int* body, const int* vptr, const double* vert,
                         const int* fptr, const int* fac, const int* sptr, const int* surf) {
  if (!c || !c->have_scene) { set_err("convexes_setup: no scene uploaded"); return B2DEV_ESTATE; }
  if (nconv < 0 || (nconv > 0 && (!body || !vptr || !vert || !fptr || !fac || !sptr || !surf))) {
    set_err("convexes_setup: invalid arguments");
    return B2DEV_EINVAL;
  }
  std::vector<int> ns(std::max(nconv, 1), 0);
  if (nconv > 0 && (vptr[0] != 0 || fptr[0] != 0 || sptr[0] != 0)) {
    set_err("convexes_setup: offsets must start at 0");
    return B2DEV_EINVAL;
  }
  for (int k = 0; k < nconv; k++) {
    const int nv = vptr[k + 1] - vptr[k], nf = sptr[k + 1] - sptr[k];
    if (body[k] < 0 || body[k] >= c->nbod) { set_err("convexes_setup: convex %d: body out of range", k); return B2DEV_EINVAL; }
    if (nv < 1 || nv > 256 || nf < 1 || fptr[k + 1] < fptr[k]) {  // GJK runs at most 4 nv^2 steps
      set_err("convexes_setup: convex %d: %d vertices and %d faces", k, nv, nf);
      return B2DEV_EINVAL;
    }
    int m = fptr[k];
    for (int f = 0; f < nf; f++) {
      if (m >= fptr[k + 1] || fac[m] < 3 || m + fac[m] >= fptr[k + 1]) {
        set_err("convexes_setup: convex %d: face %d overruns its face list", k, f);
        return B2DEV_EINVAL;
      }
      for (int t = 1; t <= fac[m]; t++)
        if (fac[m + t] < 0 || fac[m + t] >= nv) {
          set_err("convexes_setup: convex %d: face %d: vertex index out of range", k, f);
          return B2DEV_EINVAL;
        }
      m += fac[m] + 1;
    }
    while (ns[k] < nf && surf[sptr[k] + ns[k]] != -INT_MAX) ns[k]++;
    if (ns[k] == 0) { set_err("convexes_setup: convex %d has no surface face", k); return B2DEV_EINVAL; }
  }
  DeviceGuard g(c->device);
  c->nconv = nconv;
  const int nvt = nconv > 0 ? vptr[nconv] : 0, nft = nconv > 0 ? sptr[nconv] : 0, nfac = nconv > 0 ? fptr[nconv] : 0;
  B2_TRY(upload(c, c->cvx_body, body, (size_t)nconv, 0));
  B2_TRY(upload(c, c->cvx_vptr, vptr, (size_t)nconv + (nconv > 0), 0));
  B2_TRY(upload(c, c->cvx_vert, vert, (size_t)3 * nvt, 0));
  B2_TRY(upload(c, c->cvx_fptr, fptr, (size_t)nconv + (nconv > 0), 0));
  B2_TRY(upload(c, c->cvx_fac, fac, (size_t)nfac, 0));
  B2_TRY(upload(c, c->cvx_sptr, sptr, (size_t)nconv + (nconv > 0), 0));
  B2_TRY(upload(c, c->cvx_surf, surf, (size_t)nft, 0));
  B2_TRY(upload(c, c->cvx_ns, ns.data(), (size_t)nconv, 0));
  // adjacency of the convexes of one body: those within GEOMETRIC_EPSILON of
  // each other as set up (the overlap callback of cvx.c:575-589); a rigid
  // body's convexes keep it
  {
    std::vector<std::vector<int>> of_body(c->nbod);
    for (int k = 0; k < nconv; k++) of_body[body[k]].push_back(k);
    std::vector<std::vector<int>> adj(std::max(nconv, 1));
    bool any = false;
    for (const auto& list : of_body)
      for (size_t a = 0; a < list.size(); a++)
        for (size_t b = a + 1; b < list.size(); b++) {
          const int x = list[a], y = list[b];
          double p[3], q[3];
          if (gjk_polytopes(vert + 3 * (size_t)vptr[x], vptr[x + 1] - vptr[x], vert + 3 * (size_t)vptr[y],
                            vptr[y + 1] - vptr[y], p, q) < kGeomEps) {
            adj[x].push_back(y);
            adj[y].push_back(x);
            any = true;
          }
        }
    std::vector<int> aptr(nconv + 1, 0), alist;
    for (int k = 0; k < nconv; k++) {
      aptr[k + 1] = aptr[k] + (int)adj[k].size();
      alist.insert(alist.end(), adj[k].begin(), adj[k].end());
    }
    alist.push_back(0);
    B2_TRY(upload(c, c->cvx_aptr, aptr.data(), aptr.size(), 0));
    B2_TRY(upload(c, c->cvx_adj, alist.data(), alist.size(), 0));
    c->cvx_have_adj = any;
  }
  B2_TRY(ensure(c->cvx_cur, sizeof(double) * 3 * (nvt + 1)));
  B2_TRY(ensure(c->cvx_pla, sizeof(double) * 6 * (nft + 1)));
  B2_TRY(ensure(c->cvx_box, sizeof(double) * 6 * (nconv + 1)));
  B2_CK(cudaStreamSynchronize(c->stream));
  c->det_valid = c->det_assembled = false;
  return B2DEV_OK;
}

static ConvexDev convex_view(b2dev_ctx* c) {
  ConvexDev v;
  v.n = c->nconv;
  v.body = ptr<int>(c->cvx_body); v.vptr = ptr<int>(c->cvx_vptr); v.vert = ptr<double>(c->cvx_vert);
  v.fptr = ptr<int>(c->cvx_fptr); v.fac = ptr<int>(c->cvx_fac); v.sptr = ptr<int>(c->cvx_sptr);
  v.surf = ptr<int>(c->cvx_surf); v.nsurf_face = ptr<int>(c->cvx_ns); v.cur = ptr<double>(c->cvx_cur);
  v.pla = ptr<double>(c->cvx_pla); v.box = ptr<double>(c->cvx_box);
  return v;
}

static const char* detect_bad_text(int bad) {
  if (bad & 16) return "a sphere's body index is out of range";
  if (bad & 1) return "a sphere radius is not positive and finite, or a centre is not finite";
  if (bad & 2) return "a sphere centre is too far from the origin for the detection grid";
  if (bad & 4) return "two sphere centres coincide (no contact normal)";
  if (bad & 32) return "a convex has no finite face plane";
  if (bad & 64) return "a convex pair has more than 32 face planes together (intersection capacity)";
  if (bad & 128) return "a contact gap is at or below the unphysical penetration depth (the reference stops, dom.c:3792)";
  return "a surface id is out of the material table";
}

static ContactOut staged(b2dev_ctx* c) {
  ContactOut o;
  o.master = ptr<int>(c->st_master); o.slave = ptr<int>(c->st_slave); o.point = ptr<double>(c->st_point);
  o.mpnt = ptr<double>(c->st_mpnt); o.spnt = ptr<double>(c->st_spnt); o.base = ptr<double>(c->st_base);
  o.gap = ptr<double>(c->st_gap); o.fric = ptr<double>(c->st_fric); o.rest = ptr<double>(c->st_rest);
  o.coh = ptr<double>(c->st_coh); o.R0 = ptr<double>(c->st_R0); o.U0 = ptr<double>(c->st_U0);
  o.key = ptr<long long>(c->st_key); o.slave_lo = ptr<int>(c->st_slo); o.isnew = ptr<int>(c->st_new);
  o.area = ptr<double>(c->st_area);
  return o;
}

int b2dev_exclude_bodies(b2dev_ctx* c, int npairs, const int* pairs) {
  if (!c || npairs < 0 || (npairs > 0 && !pairs)) { set_err("exclude_bodies: invalid arguments"); return B2DEV_EINVAL; }
  std::vector<long long> keys;
  for (int k = 0; k < npairs; k++) {
    const int a = pairs[2 * k], b = pairs[2 * k + 1];
    if (a < 0 || b < 0 || a >= c->nbod || b >= c->nbod) {
      set_err("exclude_bodies: pair %d: body out of range", k);
      return B2DEV_EINVAL;
    }
    keys.push_back(((long long)std::min(a, b) << 32) | (long long)std::max(a, b));
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  DeviceGuard g(c->device);
  B2_TRY(upload(c, c->ex_bodies, keys.data(), keys.size(), 0));
  B2_CK(cudaStreamSynchronize(c->stream));
  c->n_ex_bodies = (int)keys.size();
  return B2DEV_OK;
}

int b2dev_exclude_surfaces(b2dev_ctx* c, int npairs, const int* pairs) {
  if (!c || npairs < 0 || (npairs > 0 && !pairs)) { set_err("exclude_surfaces: invalid arguments"); return B2DEV_EINVAL; }
  for (int k = 0; k < 2 * npairs; k++)
    if (pairs[k] < 0) { set_err("exclude_surfaces: negative surface id"); return B2DEV_EINVAL; }
  c->ex_surf_pairs.assign(pairs, pairs + 2 * (size_t)npairs);
  c->ex_surf_nsurf = -1;  // the table is built for the material table's surfaces at the next detection
  return B2DEV_OK;
}

int b2dev_unphysical_penetration(b2dev_ctx* c, double depth) {
  if (!c) { set_err("unphysical_penetration: null context"); return B2DEV_EINVAL; }
  if (!(depth > 0.0)) { set_err("unphysical_penetration: depth must be positive"); return B2DEV_EINVAL; }
  c->depth = -depth;  // lng.c:9191
  return B2DEV_OK;
}

// the excluded surface pairs as a symmetric nsurf x nsurf table (ids past the
// material table exclude nothing)
static int exclusion_table(b2dev_ctx* c) {
  if (c->ex_surf_pairs.empty() || c->ex_surf_nsurf == c->nsurf) return B2DEV_OK;
  const int n = c->nsurf;
  std::vector<unsigned char> t((size_t)n * n, 0);
  for (size_t k = 0; k + 1 < c->ex_surf_pairs.size(); k += 2) {
    const int a = c->ex_surf_pairs[k], b = c->ex_surf_pairs[k + 1];
    if (a < n && b < n) t[(size_t)a * n + b] = t[(size_t)b * n + a] = 1;
  }
  B2_TRY(upload(c, c->ex_surf, t.data(), t.size(), 0));
  c->ex_surf_nsurf = n;
  return B2DEV_OK;
}

int b2dev_contact_sparsify(b2dev_ctx* c, double threshold, double minarea, double mindist) {
  if (!c) { set_err("contact_sparsify: null context"); return B2DEV_EINVAL; }
  // lng.c:8875-8899 (CONTACT_SPARSIFY): threshold in [0, 1], minarea and mindist not negative
  if (!(threshold >= 0.0 && threshold <= 1.0) || !(minarea >= 0.0) || !(mindist >= 0.0)) {
    set_err("contact_sparsify: threshold must lie in [0, 1], minarea and mindist must not be negative");
    return B2DEV_EINVAL;
  }
  c->sp_threshold = threshold;
  c->sp_minarea = minarea;
  c->sp_mindist = mindist;
  return B2DEV_OK;
}

int b2dev_detect_spheres(b2dev_ctx* c, int* ncon, int* nnew) {
  if (!c) { set_err("detect: null context"); return B2DEV_EINVAL; }
  if (!c->have_scene || !c->have_rigid) {
    set_err("detect: upload a scene and set up its rigid bodies (mass centres) first");
    return B2DEV_ESTATE;
  }
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  const int T = 256, ns = c->nsph, nb = c->nbod;

  // the previous step's contacts: keys, roles and their R, U (the last solve's
  // state when it was assembled from them, else the values they were given)
  // (rows: the contacts, then the constraints kept across detections; only
  // the contacts' keys are matched, the constraints carry by position)
  const int nrow_prev = c->det_valid ? c->ncon : 0;
  const int nprev = c->det_valid ? c->det_ncont : 0;
  const bool carry_cn = c->cn_n > 0 && c->det_valid && nrow_prev - nprev == c->cn_n;
  B2_TRY(ensure(c->sph_pkey, sizeof(long long) * (nprev + 1)));
  B2_TRY(ensure(c->sph_pslo, sizeof(int) * (nprev + 1)));
  B2_TRY(ensure(c->sph_pR, sizeof(double) * 3 * (nrow_prev + 1)));
  B2_TRY(ensure(c->sph_pU, sizeof(double) * 3 * (nrow_prev + 1)));
  if (nprev > 0) {
    B2_CK(cudaMemcpyAsync(c->sph_pkey.p, c->det_key.p, sizeof(long long) * nprev, cudaMemcpyDeviceToDevice, st));
    B2_CK(cudaMemcpyAsync(c->sph_pslo.p, c->det_slo.p, sizeof(int) * nprev, cudaMemcpyDeviceToDevice, st));
  }
  if (nrow_prev > 0) {
    if (c->det_assembled && c->n == nrow_prev && c->state_u) {
      c->launches++;
      k_state_out<<<blocks_for(nrow_prev, T), T, 0, st>>>(nrow_prev, ptr<int>(c->perm),
                                                           ptr<double4>(c->R64[c->state_r]), ptr<double4>(*c->state_u),
                                                           nullptr, 1.0, ptr<double>(c->sph_pR),
                                                           ptr<double>(c->sph_pU), nullptr);
    } else {
      B2_CK(cudaMemcpyAsync(c->sph_pR.p, c->det_R0.p, sizeof(double) * 3 * nrow_prev, cudaMemcpyDeviceToDevice, st));
      B2_CK(cudaMemcpyAsync(c->sph_pU.p, c->det_U0.p, sizeof(double) * 3 * nrow_prev, cudaMemcpyDeviceToDevice, st));
    }
  }

  // grid: cell edge from the largest radius, 2^k >= 2 n buckets
  unsigned int M = 1024;
  while (M < 2u * (unsigned int)ns) M *= 2;
  int mbits = 0;
  while ((1u << mbits) < M) mbits++;
  B2_TRY(ensure(c->sph_cur, sizeof(double) * 3 * (ns + 1)));
  B2_TRY(ensure(c->sph_cell, sizeof(int4) * (ns + 1)));
  B2_TRY(ensure(c->sph_hkey, sizeof(unsigned int) * (ns + 1)));
  B2_TRY(ensure(c->sph_hkey_s, sizeof(unsigned int) * (ns + 1)));
  B2_TRY(ensure(c->sph_idx, sizeof(int) * (ns + 1)));
  B2_TRY(ensure(c->sph_sorted, sizeof(int) * (ns + 1)));
  B2_TRY(ensure(c->sph_bstart, sizeof(int) * M));
  B2_TRY(ensure(c->sph_bend, sizeof(int) * M));
  B2_TRY(ensure(c->sph_cnt, sizeof(int) * (ns + 1)));
  B2_TRY(ensure(c->sph_off, sizeof(int) * (ns + 1)));
  B2_TRY(ensure(c->sph_rmax, sizeof(unsigned long long)));
  B2_TRY(ensure(c->bad, sizeof(int)));
  B2_CK(cudaMemsetAsync(c->bad.p, 0, sizeof(int), st));
  B2_CK(cudaMemsetAsync(c->sph_rmax.p, 0, sizeof(unsigned long long), st));
  B2_CK(cudaMemsetAsync(c->sph_bstart.p, 0, sizeof(int) * M, st));
  B2_CK(cudaMemsetAsync(c->sph_bend.p, 0, sizeof(int) * M, st));
  B2_CK(cudaMemsetAsync(c->sph_cnt.p, 0, sizeof(int) * (ns + 1), st));
  SphereDev sd;
  sd.nsph = ns;
  sd.nbod = nb;
  sd.body = ptr<int>(c->sph_body); sd.ref = ptr<double>(c->sph_ref); sd.rad = ptr<double>(c->sph_rad);
  sd.surf = ptr<int>(c->sph_surf); sd.cur = ptr<double>(c->sph_cur); sd.cell = ptr<int4>(c->sph_cell);
  sd.hkey = ptr<unsigned int>(c->sph_hkey);
  const ConvexDev cvd = convex_view(c);
  int npair = 0, bad = 0;
  B2_TRY(exclusion_table(c));
  PairFilter pf;
  pf.body_pairs = c->n_ex_bodies ? ptr<long long>(c->ex_bodies) : nullptr;
  pf.n = c->n_ex_bodies;
  ContactRules cr;
  cr.nosurf = c->ex_surf_pairs.empty() ? nullptr : ptr<unsigned char>(c->ex_surf);
  cr.depth = c->depth;
  if (c->nconv > 0) {
    c->launches++;
    k_cvx_update<<<blocks_for(c->nconv, 64), 64, 0, st>>>(cvd, ptr<double>(c->rot), ptr<double>(c->rb_x),
                                                        ptr<double>(c->x0));
  }
  if (ns > 0) {
    c->launches += 2;
    k_sph_centres<<<blocks_for(ns, T), T, 0, st>>>(sd, ptr<double>(c->rot), ptr<double>(c->rb_x),
                                                   ptr<double>(c->x0), ptr<unsigned long long>(c->sph_rmax),
                                                   ptr<int>(c->bad));
    k_sph_cells<<<blocks_for(ns, T), T, 0, st>>>(sd, ptr<unsigned long long>(c->sph_rmax), M - 1,
                                                 ptr<int>(c->sph_idx), ptr<int>(c->bad));
    size_t bytes = 0;
    B2_CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, ptr<unsigned int>(c->sph_hkey),
                                          ptr<unsigned int>(c->sph_hkey_s), ptr<int>(c->sph_idx),
                                          ptr<int>(c->sph_sorted), ns, 0, mbits, st));
    B2_TRY(ensure(c->cub_tmp, bytes));
    B2_CK(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, bytes, ptr<unsigned int>(c->sph_hkey),
                                          ptr<unsigned int>(c->sph_hkey_s), ptr<int>(c->sph_idx),
                                          ptr<int>(c->sph_sorted), ns, 0, mbits, st));
    c->launches += 2;
    k_sph_buckets<<<blocks_for(ns, T), T, 0, st>>>(ns, ptr<unsigned int>(c->sph_hkey_s), ptr<int>(c->sph_bstart),
                                                   ptr<int>(c->sph_bend));
    k_sph_pairs<false><<<blocks_for(ns, T), T, 0, st>>>(sd, ptr<int>(c->obst), pf, ptr<int>(c->sph_sorted),
                                                        ptr<int>(c->sph_bstart), ptr<int>(c->sph_bend), M - 1,
                                                        ptr<int>(c->sph_cnt), nullptr, nullptr);
    const int* pair_count = ptr<int>(c->sph_cnt);
    if (c->nconv > 0) {  // convex partners: counted apart, the totals scanned
      B2_TRY(ensure(c->sph_ccnt, sizeof(int) * (ns + 1)));
      B2_CK(cudaMemsetAsync(c->sph_ccnt.p, 0, sizeof(int) * (ns + 1), st));
      c->launches += 2;
      k_cvx_pairs<false><<<blocks_for(ns, 128), 128, 0, st>>>(sd, cvd, ptr<int>(c->obst), pf, ptr<int>(c->sph_ccnt),
                                                               nullptr, nullptr, nullptr);
      k_add_counts<<<blocks_for(ns, T), T, 0, st>>>(ns, ptr<int>(c->sph_cnt), ptr<int>(c->sph_ccnt));
      pair_count = ptr<int>(c->sph_ccnt);
    }
    // the pair total in 64 bits before the int scan: offsets, pair indices and
    // the body lists (two entries per contact) are int
    unsigned long long total = 0;
    B2_TRY(ensure(c->sph_total, sizeof(unsigned long long)));
    B2_CK(cudaMemsetAsync(c->sph_total.p, 0, sizeof(unsigned long long), st));
    c->launches++;
    k_count_total<<<std::min(blocks_for(ns, T), 4 * c->sms), T, 0, st>>>(ns, pair_count,
                                                                         ptr<unsigned long long>(c->sph_total));
    B2_CK(cudaMemcpyAsync(&total, c->sph_total.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaMemcpyAsync(&bad, c->bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaStreamSynchronize(st));
    if (bad) { set_err("detect: %s", detect_bad_text(bad)); return B2DEV_EINVAL; }
    if (total > (unsigned long long)(INT_MAX / 2 - 1)) {
      set_err("detect: %llu candidate pairs exceed the supported %d", total, INT_MAX / 2 - 1);
      return B2DEV_EINVAL;
    }
    B2_TRY(scan_exclusive(c, pair_count, ptr<int>(c->sph_off), ns + 1));
    B2_CK(cudaMemcpyAsync(&npair, ptr<int>(c->sph_off) + ns, sizeof(int), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaStreamSynchronize(st));
  }
  const int nps = npair;  // pairs with a sphere; the convex-convex candidates follow (their keys are larger)

  // convex-convex candidates: the grid over the box centres of ordinary
  // convexes and the list of large ones, counted, written, the keys sorted
  int ncc = 0;
  const int nv = c->nconv;
  if (nv > 1) {
    unsigned int Mc = 1024;
    while (Mc < 2u * (unsigned int)nv) Mc *= 2;
    int cbits = 0;
    while ((1u << cbits) <= Mc) cbits++;  // keys up to Mc (the large convexes' bucket)
    B2_TRY(ensure(c->cc_lox, sizeof(double) * (nv + 1)));
    B2_TRY(ensure(c->cc_idx, sizeof(int) * (nv + 1)));
    B2_TRY(ensure(c->cc_sidx, sizeof(int) * (nv + 1)));
    B2_TRY(ensure(c->cc_cnt, sizeof(int) * (nv + 1)));
    B2_TRY(ensure(c->cc_off, sizeof(int) * (nv + 1)));
    B2_TRY(ensure(c->cc_cell, sizeof(int4) * (nv + 1)));
    B2_TRY(ensure(c->cc_hkey, sizeof(unsigned int) * (nv + 1)));
    B2_TRY(ensure(c->cc_hkey_s, sizeof(unsigned int) * (nv + 1)));
    B2_TRY(ensure(c->cc_large, sizeof(int) * (nv + 1)));
    B2_TRY(ensure(c->cc_bstart, sizeof(int) * (Mc + 1)));
    B2_TRY(ensure(c->cc_bend, sizeof(int) * (Mc + 1)));
    B2_TRY(ensure(c->cc_misc, 32));  // extent sum, largest ordinary side (bits), large count, selected count
    B2_TRY(ensure(c->sph_total, sizeof(unsigned long long)));
    double* esum = ptr<double>(c->cc_misc);
    unsigned long long* emax = ptr<unsigned long long>(c->cc_misc) + 1;
    int* nlarge_d = reinterpret_cast<int*>(ptr<unsigned long long>(c->cc_misc) + 2);
    B2_CK(cudaMemsetAsync(c->cc_misc.p, 0, 32, st));
    B2_CK(cudaMemsetAsync(c->cc_bstart.p, 0, sizeof(int) * (Mc + 1), st));
    B2_CK(cudaMemsetAsync(c->cc_bend.p, 0, sizeof(int) * (Mc + 1), st));
    c->launches += 3;
    k_cc_extent<<<blocks_for(nv, T), T, 0, st>>>(cvd, ptr<double>(c->cc_lox), esum);
    k_cc_classify<<<blocks_for(nv, T), T, 0, st>>>(nv, ptr<double>(c->cc_lox), esum, emax, ptr<int>(c->cc_large),
                                                   nlarge_d);
    k_cc_cells<<<blocks_for(nv, T), T, 0, st>>>(cvd, ptr<double>(c->cc_lox), esum, emax, Mc - 1,
                                                ptr<int4>(c->cc_cell), ptr<unsigned int>(c->cc_hkey),
                                                ptr<int>(c->cc_idx), ptr<int>(c->bad));
    size_t bytes = 0;
    B2_CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, ptr<unsigned int>(c->cc_hkey),
                                          ptr<unsigned int>(c->cc_hkey_s), ptr<int>(c->cc_idx),
                                          ptr<int>(c->cc_sidx), nv, 0, cbits, st));
    B2_TRY(ensure(c->cub_tmp, bytes));
    B2_CK(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, bytes, ptr<unsigned int>(c->cc_hkey),
                                          ptr<unsigned int>(c->cc_hkey_s), ptr<int>(c->cc_idx),
                                          ptr<int>(c->cc_sidx), nv, 0, cbits, st));
    int nlarge = 0;
    B2_CK(cudaMemcpyAsync(&nlarge, nlarge_d, sizeof(int), cudaMemcpyDeviceToHost, st));
    c->launches++;
    k_sph_buckets<<<blocks_for(nv, T), T, 0, st>>>(nv, ptr<unsigned int>(c->cc_hkey_s), ptr<int>(c->cc_bstart),
                                                   ptr<int>(c->cc_bend));
    B2_CK(cudaStreamSynchronize(st));
    c->launches += 2;
    k_cc_pairs<false><<<blocks_for(nv, 128), 128, 0, st>>>(
        cvd, ptr<int>(c->obst), pf, ns, ptr<int>(c->cc_sidx), ptr<int4>(c->cc_cell), ptr<int>(c->cc_bstart),
        ptr<int>(c->cc_bend), Mc - 1, ptr<int>(c->cc_large), nlarge, ptr<int>(c->cc_cnt), nullptr, nullptr);
    unsigned long long total = 0;
    B2_CK(cudaMemsetAsync(c->sph_total.p, 0, sizeof(unsigned long long), st));
    k_count_total<<<std::min(blocks_for(nv, T), 4 * c->sms), T, 0, st>>>(nv, ptr<int>(c->cc_cnt),
                                                                         ptr<unsigned long long>(c->sph_total));
    B2_CK(cudaMemcpyAsync(&total, c->sph_total.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaMemcpyAsync(&bad, c->bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaStreamSynchronize(st));
    if (bad) { set_err("detect: %s", detect_bad_text(bad)); return B2DEV_EINVAL; }
    if (total + (unsigned long long)nps > (unsigned long long)(INT_MAX / 2 - 1)) {
      set_err("detect: %llu candidate pairs exceed the supported %d", total + nps, INT_MAX / 2 - 1);
      return B2DEV_EINVAL;
    }
    const int nbox = (int)total;  // pairs whose inflated boxes overlap
    if (nbox > 0) {
      B2_TRY(scan_exclusive(c, ptr<int>(c->cc_cnt), ptr<int>(c->cc_off), nv));
      B2_TRY(ensure(c->cc_keys, sizeof(long long) * (nbox + 1)));
      B2_TRY(ensure(c->cc_keys_s, sizeof(long long) * (nbox + 1)));
      B2_TRY(ensure(c->cc_keep, nbox + 1));
      c->launches += 2;
      k_cc_pairs<true><<<blocks_for(nv, 128), 128, 0, st>>>(
          cvd, ptr<int>(c->obst), pf, ns, ptr<int>(c->cc_sidx), ptr<int4>(c->cc_cell), ptr<int>(c->cc_bstart),
          ptr<int>(c->cc_bend), Mc - 1, ptr<int>(c->cc_large), nlarge, nullptr, ptr<int>(c->cc_off),
          ptr<long long>(c->cc_keys));
      B2_TRY(ensure(c->cc_cls, sizeof(unsigned int) * 2 * (nbox + 1)));
      B2_TRY(ensure(c->cc_order, sizeof(int) * 2 * (nbox + 1)));
      unsigned int* cls = ptr<unsigned int>(c->cc_cls);
      unsigned int* cls_s = cls + (nbox + 1);
      int* iota = ptr<int>(c->cc_order);
      int* order = iota + (nbox + 1);
      k_cc_gjk<<<blocks_for(nbox, 128), 128, 0, st>>>(nbox, ns, cvd, ptr<long long>(c->cc_keys),
                                                      ptr<unsigned char>(c->cc_keep), cls);
      // the touching pairs with their work classes, then sorted by key
      int* nsel = reinterpret_cast<int*>(ptr<unsigned long long>(c->cc_misc) + 3);
      bytes = 0;
      B2_CK(cub::DeviceSelect::Flagged(nullptr, bytes, ptr<long long>(c->cc_keys), ptr<unsigned char>(c->cc_keep),
                                       ptr<long long>(c->cc_keys_s), nsel, nbox, st));
      B2_TRY(ensure(c->cub_tmp, bytes));
      B2_CK(cub::DeviceSelect::Flagged(c->cub_tmp.p, bytes, ptr<long long>(c->cc_keys),
                                       ptr<unsigned char>(c->cc_keep), ptr<long long>(c->cc_keys_s), nsel, nbox,
                                       st));
      bytes = 0;
      B2_CK(cub::DeviceSelect::Flagged(nullptr, bytes, cls, ptr<unsigned char>(c->cc_keep), cls_s, nsel, nbox, st));
      B2_TRY(ensure(c->cub_tmp, bytes));
      B2_CK(cub::DeviceSelect::Flagged(c->cub_tmp.p, bytes, cls, ptr<unsigned char>(c->cc_keep), cls_s, nsel, nbox,
                                       st));
      B2_CK(cudaMemcpyAsync(&ncc, nsel, sizeof(int), cudaMemcpyDeviceToHost, st));
      B2_CK(cudaStreamSynchronize(st));
      if (ncc > 0) {
        bytes = 0;
        B2_CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, ptr<unsigned long long>(c->cc_keys_s),
                                              ptr<unsigned long long>(c->cc_keys), cls_s, cls, ncc, 0, 64, st));
        B2_TRY(ensure(c->cub_tmp, bytes));
        B2_CK(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, bytes, ptr<unsigned long long>(c->cc_keys_s),
                                              ptr<unsigned long long>(c->cc_keys), cls_s, cls, ncc, 0, 64, st));
        // work order: the key-order positions sorted (stably) by class
        c->launches++;
        k_iota<<<blocks_for(ncc, T), T, 0, st>>>(ncc, iota);
        bytes = 0;
        B2_CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, cls, cls_s, iota, order, ncc, 0, 32, st));
        B2_TRY(ensure(c->cub_tmp, bytes));
        B2_CK(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, bytes, cls, cls_s, iota, order, ncc, 0, 32, st));
      }
      c->cc_order_off = (size_t)nbox + 1;
    }
  }
  npair = nps + ncc;

  // contacts of the pairs, in pair order (row arrays with room for the
  // constraints that follow them)
  const size_t np1 = (size_t)npair + 1;
  const size_t nr1 = np1 + (size_t)c->cn_n;
  B2_TRY(ensure(c->sph_pi, sizeof(int) * np1));
  B2_TRY(ensure(c->sph_pj, sizeof(int) * np1));
  B2_TRY(ensure(c->st_master, sizeof(int) * nr1));
  B2_TRY(ensure(c->st_slave, sizeof(int) * nr1));
  B2_TRY(ensure(c->st_point, sizeof(double) * 3 * nr1));
  B2_TRY(ensure(c->st_mpnt, sizeof(double) * 3 * nr1));
  B2_TRY(ensure(c->st_spnt, sizeof(double) * 3 * nr1));
  B2_TRY(ensure(c->st_base, sizeof(double) * 9 * nr1));
  B2_TRY(ensure(c->st_gap, sizeof(double) * nr1));
  B2_TRY(ensure(c->st_fric, sizeof(double) * nr1));
  B2_TRY(ensure(c->st_rest, sizeof(double) * nr1));
  B2_TRY(ensure(c->st_coh, sizeof(double) * nr1));
  B2_TRY(ensure(c->st_R0, sizeof(double) * 3 * nr1));
  B2_TRY(ensure(c->st_U0, sizeof(double) * 3 * nr1));
  B2_TRY(ensure(c->st_key, sizeof(long long) * nr1));
  B2_TRY(ensure(c->st_slo, sizeof(int) * nr1));
  B2_TRY(ensure(c->st_new, sizeof(int) * nr1));
  B2_TRY(ensure(c->st_area, sizeof(double) * nr1));
  B2_TRY(ensure(c->sph_keep, sizeof(int) * np1));
  B2_TRY(ensure(c->sph_pos, sizeof(int) * np1));
  B2_TRY(ensure(c->sph_bcnt, sizeof(int) * (nb + 1)));
  B2_TRY(ensure(c->sph_bptr, sizeof(int) * (nb + 1)));
  B2_TRY(ensure(c->sph_blist, sizeof(int) * 2 * np1));
  const ContactOut so = staged(c);
  int nkeep = 0, nfresh = 0;
  if (npair > 0) {
    if (nps > 0) {
      c->launches += 3;
      k_sph_pairs<true><<<blocks_for(ns, T), T, 0, st>>>(sd, ptr<int>(c->obst), pf, ptr<int>(c->sph_sorted),
                                                         ptr<int>(c->sph_bstart), ptr<int>(c->sph_bend), M - 1,
                                                         nullptr, ptr<int>(c->sph_off), ptr<int>(c->sph_pj));
      if (c->nconv > 0) {  // after the sphere partners (sph_cnt still holds their count)
        c->launches++;
        k_cvx_pairs<true><<<blocks_for(ns, 128), 128, 0, st>>>(sd, cvd, ptr<int>(c->obst), pf, nullptr,
                                                                ptr<int>(c->sph_off), ptr<int>(c->sph_cnt),
                                                                ptr<int>(c->sph_pj));
      }
      k_sph_sort_seg<<<blocks_for(ns, T), T, 0, st>>>(ns, ptr<int>(c->sph_off), ptr<int>(c->sph_pj),
                                                      ptr<int>(c->sph_pi));
      k_sph_contacts<<<blocks_for(nps, T), T, 0, st>>>(
          nps, sd, cvd, ptr<int>(c->sph_pi), ptr<int>(c->sph_pj), ptr<double>(c->rot), ptr<double>(c->rb_x),
          ptr<double>(c->x0), c->nsurf, ptr<double>(c->sph_mat), cr, nprev, ptr<long long>(c->sph_pkey),
          ptr<int>(c->sph_pslo), ptr<double>(c->sph_pR), ptr<double>(c->sph_pU), so, ptr<int>(c->bad));
    }
    if (ncc > 0) {
      c->launches++;
      k_cc_contacts<<<blocks_for(ncc, 64), 64, 0, st>>>(
          ncc, nps, ns, ptr<int>(c->cc_order) + c->cc_order_off, cvd, ptr<long long>(c->cc_keys),
          ptr<double>(c->rot), ptr<double>(c->rb_x),
          ptr<double>(c->x0), c->nsurf, ptr<double>(c->sph_mat), cr, nprev, ptr<long long>(c->sph_pkey),
          ptr<double>(c->sph_pR), ptr<double>(c->sph_pU), so, ptr<int>(c->bad));
    }
    // sparsification neighbourhoods: the contacts of each body
    B2_CK(cudaMemsetAsync(c->sph_bcnt.p, 0, sizeof(int) * (nb + 1), st));
    c->launches++;
    k_sph_body_count<<<blocks_for(npair, T), T, 0, st>>>(npair, nb, so.master, so.slave, ptr<int>(c->sph_bcnt),
                                                         ptr<int>(c->bad));
    B2_TRY(scan_exclusive(c, ptr<int>(c->sph_bcnt), ptr<int>(c->sph_bptr), nb + 1));
    B2_CK(cudaMemcpyAsync(c->sph_bcnt.p, c->sph_bptr.p, sizeof(int) * (nb + 1), cudaMemcpyDeviceToDevice, st));
    c->launches += 2;
    k_sph_body_fill<<<blocks_for(npair, T), T, 0, st>>>(npair, nb, so.master, so.slave, ptr<int>(c->sph_bcnt),
                                                        ptr<int>(c->sph_blist));
    k_sph_sparsify<<<blocks_for(npair, T), T, 0, st>>>(
        npair, nb, so.master, so.slave, so.isnew, so.point, so.area, so.key, so.slave_lo, ns,
        c->cvx_have_adj ? ptr<int>(c->cvx_aptr) : nullptr, ptr<int>(c->cvx_adj), ptr<int>(c->sph_bptr),
        ptr<int>(c->sph_blist), 2.0 * c->sp_mindist, c->sp_threshold, c->sp_minarea, ptr<int>(c->sph_keep));
    B2_TRY(scan_exclusive(c, ptr<int>(c->sph_keep), ptr<int>(c->sph_pos), npair));
    int lastpos = 0, lastkeep = 0;
    B2_CK(cudaMemcpyAsync(&lastpos, ptr<int>(c->sph_pos) + npair - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaMemcpyAsync(&lastkeep, ptr<int>(c->sph_keep) + npair - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaMemcpyAsync(&bad, c->bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaStreamSynchronize(st));
    if (bad) { set_err("detect: %s", detect_bad_text(bad)); return B2DEV_EINVAL; }
    nkeep = lastpos + lastkeep;
  }

  // the kept contacts become the scene's contacts: when nothing was removed
  // (the common case) the staged arrays are taken over as they are, else the
  // kept ones are compacted into the scene's arrays
  const size_t nk1 = (size_t)nkeep + 1 + (size_t)c->cn_n;
  if (npair > 0 && nkeep == npair) {
    std::swap(c->master, c->st_master); std::swap(c->slave, c->st_slave); std::swap(c->det_point, c->st_point);
    std::swap(c->mpnt, c->st_mpnt); std::swap(c->spnt, c->st_spnt); std::swap(c->base, c->st_base);
    std::swap(c->gap_c, c->st_gap); std::swap(c->fric_c, c->st_fric); std::swap(c->rest_c, c->st_rest);
    std::swap(c->coh_c, c->st_coh); std::swap(c->det_R0, c->st_R0); std::swap(c->det_U0, c->st_U0);
    std::swap(c->det_key, c->st_key); std::swap(c->det_slo, c->st_slo); std::swap(c->det_new, c->st_new);
    std::swap(c->det_area, c->st_area);
  } else {
    B2_TRY(ensure(c->master, sizeof(int) * nk1));
    B2_TRY(ensure(c->slave, sizeof(int) * nk1));
    B2_TRY(ensure(c->mpnt, sizeof(double) * 3 * nk1));
    B2_TRY(ensure(c->spnt, sizeof(double) * 3 * nk1));
    B2_TRY(ensure(c->base, sizeof(double) * 9 * nk1));
    B2_TRY(ensure(c->gap_c, sizeof(double) * nk1));
    B2_TRY(ensure(c->fric_c, sizeof(double) * nk1));
    B2_TRY(ensure(c->rest_c, sizeof(double) * nk1));
    B2_TRY(ensure(c->coh_c, sizeof(double) * nk1));
    B2_TRY(ensure(c->det_point, sizeof(double) * 3 * nk1));
    B2_TRY(ensure(c->det_R0, sizeof(double) * 3 * nk1));
    B2_TRY(ensure(c->det_U0, sizeof(double) * 3 * nk1));
    B2_TRY(ensure(c->det_key, sizeof(long long) * nk1));
    B2_TRY(ensure(c->det_slo, sizeof(int) * nk1));
    B2_TRY(ensure(c->det_new, sizeof(int) * nk1));
    B2_TRY(ensure(c->det_area, sizeof(double) * nk1));
    if (npair > 0) {
      ContactOut d;
      d.master = ptr<int>(c->master); d.slave = ptr<int>(c->slave); d.point = ptr<double>(c->det_point);
      d.mpnt = ptr<double>(c->mpnt); d.spnt = ptr<double>(c->spnt); d.base = ptr<double>(c->base);
      d.gap = ptr<double>(c->gap_c); d.fric = ptr<double>(c->fric_c); d.rest = ptr<double>(c->rest_c);
      d.coh = ptr<double>(c->coh_c); d.R0 = ptr<double>(c->det_R0); d.U0 = ptr<double>(c->det_U0);
      d.key = ptr<long long>(c->det_key); d.slave_lo = ptr<int>(c->det_slo); d.isnew = ptr<int>(c->det_new);
      d.area = ptr<double>(c->det_area);
      c->launches++;
      k_sph_compact<<<blocks_for(npair, T), T, 0, st>>>(npair, ptr<int>(c->sph_keep), ptr<int>(c->sph_pos), so,
                                                         d);
    }
  }
  if (c->cn_n > 0) {  // the constraints kept across detections follow the contacts
    ContactOut d;
    d.master = ptr<int>(c->master); d.slave = ptr<int>(c->slave); d.point = ptr<double>(c->det_point);
    d.mpnt = ptr<double>(c->mpnt); d.spnt = ptr<double>(c->spnt); d.base = ptr<double>(c->base);
    d.gap = ptr<double>(c->gap_c); d.fric = ptr<double>(c->fric_c); d.rest = ptr<double>(c->rest_c);
    d.coh = ptr<double>(c->coh_c); d.R0 = ptr<double>(c->det_R0); d.U0 = ptr<double>(c->det_U0);
    d.key = ptr<long long>(c->det_key); d.slave_lo = ptr<int>(c->det_slo); d.isnew = ptr<int>(c->det_new);
    d.area = ptr<double>(c->det_area);
    B2_TRY(ensure(c->kind_c, sizeof(int) * nk1));
    B2_TRY(ensure(c->Z_c, sizeof(double) * 4 * nk1));
    if (nkeep > 0) {
      B2_CK(cudaMemsetAsync(c->kind_c.p, 0, sizeof(int) * nkeep, st));
      B2_CK(cudaMemsetAsync(c->Z_c.p, 0, sizeof(double) * 4 * nkeep, st));
    }
    c->launches++;
    k_constraints_append<<<blocks_for(c->cn_n, 128), 128, 0, st>>>(
        nkeep, c->cn_n, ptr<int>(c->cn_kind), ptr<int>(c->cn_master), ptr<int>(c->cn_slave), ptr<double>(c->cn_mpnt),
        ptr<double>(c->cn_spnt), ptr<double>(c->cn_base), ptr<double>(c->cn_Z),
        carry_cn ? ptr<double>(c->sph_pR) + 3 * (size_t)nprev : nullptr,
        carry_cn ? ptr<double>(c->sph_pU) + 3 * (size_t)nprev : nullptr, d, ptr<int>(c->kind_c), ptr<double>(c->Z_c));
  }
  if (npair > 0) {  // new contacts kept
    B2_TRY(ensure(c->sph_cnt, sizeof(int) * nk1));
    size_t bytes = 0;
    B2_CK(cub::DeviceReduce::Sum(nullptr, bytes, ptr<int>(c->det_new), ptr<int>(c->sph_cnt), nkeep, st));
    B2_TRY(ensure(c->cub_tmp, bytes));
    B2_CK(cub::DeviceReduce::Sum(c->cub_tmp.p, bytes, ptr<int>(c->det_new), ptr<int>(c->sph_cnt), nkeep, st));
    B2_CK(cudaMemcpyAsync(&nfresh, c->sph_cnt.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  }
  B2_CK(cudaGetLastError());
  B2_CK(cudaStreamSynchronize(st));
  c->ncon = nkeep + c->cn_n;
  c->det_ncont = nkeep;
  c->has_kinds = c->cn_n > 0;
  c->det_valid = true;
  c->det_assembled = false;
  c->ready = false;  // the local dynamics must be assembled for the new contacts
  if (ncon) *ncon = nkeep;
  if (nnew) *nnew = nfresh;
  return B2DEV_OK;
}

int b2dev_detect_carry_state(b2dev_ctx* c) {
  if (!c || !c->det_valid || !c->det_assembled || !c->ready || c->n != c->ncon) {
    set_err("detect_carry_state: assemble the contacts of the last detection first");
    return B2DEV_ESTATE;
  }
  return b2dev_set_state(c, ptr<double>(c->det_R0), ptr<double>(c->det_U0), 1);
}

int b2dev_get_contacts(b2dev_ctx* c, int* master, int* slave, double* point, double* mpnt, double* spnt,
                       double* base, double* gap, double* friction, double* restitution, long long* key,
                       int* slave_lo, int* isnew, double* R0, double* U0, int on_device) {
  if (!c || !c->det_valid) { set_err("get_contacts: no detection"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  const size_t n = (size_t)c->det_ncont;  // the contacts (constraint rows follow them)
  const cudaMemcpyKind kd = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (n > 0) {
    if (master) B2_CK(cudaMemcpyAsync(master, c->master.p, sizeof(int) * n, kd, st));
    if (slave) B2_CK(cudaMemcpyAsync(slave, c->slave.p, sizeof(int) * n, kd, st));
    if (point) B2_CK(cudaMemcpyAsync(point, c->det_point.p, sizeof(double) * 3 * n, kd, st));
    if (mpnt) B2_CK(cudaMemcpyAsync(mpnt, c->mpnt.p, sizeof(double) * 3 * n, kd, st));
    if (spnt) B2_CK(cudaMemcpyAsync(spnt, c->spnt.p, sizeof(double) * 3 * n, kd, st));
    if (base) B2_CK(cudaMemcpyAsync(base, c->base.p, sizeof(double) * 9 * n, kd, st));
    if (gap) B2_CK(cudaMemcpyAsync(gap, c->gap_c.p, sizeof(double) * n, kd, st));
    if (friction) B2_CK(cudaMemcpyAsync(friction, c->fric_c.p, sizeof(double) * n, kd, st));
    if (restitution) B2_CK(cudaMemcpyAsync(restitution, c->rest_c.p, sizeof(double) * n, kd, st));
    if (key) B2_CK(cudaMemcpyAsync(key, c->det_key.p, sizeof(long long) * n, kd, st));
    if (slave_lo) B2_CK(cudaMemcpyAsync(slave_lo, c->det_slo.p, sizeof(int) * n, kd, st));
    if (isnew) B2_CK(cudaMemcpyAsync(isnew, c->det_new.p, sizeof(int) * n, kd, st));
    if (R0) B2_CK(cudaMemcpyAsync(R0, c->det_R0.p, sizeof(double) * 3 * n, kd, st));
    if (U0) B2_CK(cudaMemcpyAsync(U0, c->det_U0.p, sizeof(double) * 3 * n, kd, st));
  }
  B2_CK(cudaStreamSynchronize(st));
  return B2DEV_OK;
}

int b2dev_get_contact_area(b2dev_ctx* c, double* area, int on_device) {
  if (!c || !c->det_valid) { set_err("get_contact_area: no detection"); return B2DEV_ESTATE; }
  if (!area) { set_err("get_contact_area: null output"); return B2DEV_EINVAL; }
  DeviceGuard g(c->device);
  if (c->det_ncont > 0)
    B2_CK(cudaMemcpyAsync(area, c->det_area.p, sizeof(double) * c->det_ncont,
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
  B2_CK(cudaStreamSynchronize(c->stream));
  return B2DEV_OK;
}

int b2dev_sphere_centres(b2dev_ctx* c, double* cur, int on_device) {
  if (!c || !cur) { set_err("sphere_centres: null argument"); return B2DEV_EINVAL; }
  if (!c->det_valid) { set_err("sphere_centres: no detection"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  if (c->nsph > 0)
    B2_CK(cudaMemcpyAsync(cur, c->sph_cur.p, sizeof(double) * 3 * c->nsph,
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
  B2_CK(cudaStreamSynchronize(c->stream));
  return B2DEV_OK;
}

int b2dev_get_state(b2dev_ctx* c, double* R, double* U, double* conmerit, int on_device) {
  if (!c || !c->ready) { set_err("get_state: no local dynamics"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  const int n = c->n;
  cudaStream_t st = c->stream;
  if (n == 0) return B2DEV_OK;
  B2_TRY(ensure(c->io, sizeof(double) * 7 * (n + 1)));
  double* dR = ptr<double>(c->io);
  double* dU = dR + 3 * (size_t)(n + 1);
  double* dC = dU + 3 * (size_t)(n + 1);
  double lo = c->free_energy < DBL_EPSILON ? 1.0 : c->free_energy;
  lo = lo == 0.0 ? 1.0 : lo;
  c->launches++;
  k_state_out<<<blocks_for(n, 256), 256, 0, st>>>(n, ptr<int>(c->perm), ptr<double4>(c->R64[c->state_r]),
                                                  ptr<double4>(*c->state_u),
                                                  c->state_cm ? ptr<double>(*c->state_cm) : nullptr, lo, dR, dU,
                                                  c->state_cm ? dC : nullptr);
  const cudaMemcpyKind kd = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (R) B2_CK(cudaMemcpyAsync(R, dR, sizeof(double) * 3 * n, kd, st));
  if (U) B2_CK(cudaMemcpyAsync(U, dU, sizeof(double) * 3 * n, kd, st));
  if (conmerit) {
    if (c->state_cm) B2_CK(cudaMemcpyAsync(conmerit, dC, sizeof(double) * n, kd, st));
    else if (on_device) B2_CK(cudaMemsetAsync(conmerit, 0, sizeof(double) * n, st));
    else memset(conmerit, 0, sizeof(double) * n);
  }
  if (!on_device) B2_CK(cudaStreamSynchronize(st));  // device outputs are ordered on the library's stream
  return B2DEV_OK;
}

int b2dev_solve(b2dev_ctx* c, const b2dev_solve_opts* o, b2dev_solve_report* rep, double* rerhist, double* merhist) {
  if (!c || !o || !rep) { set_err("solve: null argument"); return B2DEV_EINVAL; }
  if (!c->ready) { set_err("solve: no local dynamics (assemble or upload first)"); return B2DEV_ESTATE; }
  if (o->maxiter <= 0 || o->diagmaxiter <= 0 || o->diagsolver < 0 || o->diagsolver > 3 || o->failure < 0 ||
      o->failure > 2 || (o->precision != B2DEV_FP64 && o->precision != B2DEV_MIXED)) {
    set_err("solve: invalid options");
    return B2DEV_EINVAL;
  }
  if (o->precision == B2DEV_MIXED && o->maxiter < 2) { set_err("solve: mixed precision needs maxiter >= 2"); return B2DEV_EINVAL; }
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  memset(rep, 0, sizeof *rep);
  const int maxiter = o->maxiter;
  B2_CK(cudaEventRecord(c->ev[2], st));

  if (c->nprob != 1) { set_err("solve: the context holds %d problems (use b2dev_solve_batch)", c->nprob); return B2DEV_ESTATE; }
  SolveControl g1, g2;
  memset(&g1, 0, sizeof g1);
  memset(&g2, 0, sizeof g2);
  std::vector<ProblemControl> q1, q2;
  if (c->n == 0) {  // no rows: one iteration with zero error and merit, as the reference loop does
    rep->iters = 1;
    B2_CK(cudaEventRecord(c->ev[3], st));
    B2_CK(cudaEventSynchronize(c->ev[3]));
    if (rerhist) rerhist[0] = 0.0;
    if (merhist) merhist[0] = 0.0;
    return B2DEV_OK;
  }
  int iters = 0, final_global = 0;
  bool thrown = false;
  double merit = 0.0, error = 0.0;
  std::vector<std::pair<int, int>> ranges;  // [first, last] global sweep indices of returned iterates
  if (o->precision == B2DEV_MIXED) {
    c->launches++;
    k_shadow<<<blocks_for(c->n, 256), 256, 0, st>>>(c->n, ptr<double4>(c->R64[c->state_r]),
                                                    ptr<float4>(c->R32[c->state_r]));
    // The FP32 sweeps stop at the caller's rule or, when that asks for more
    // than FP32 products resolve, at the FP32 floors; the FP64 sweeps that
    // follow continue to the caller's epsilon and meritval.
    b2dev_solve_opts o32 = *o;
    o32.epsilon = std::max(o->epsilon, kMixedEpsilonFloor);
    if (!o->nomerit) o32.meritval = std::max(o->meritval, kMixedMeritFloor);
    B2_TRY(solve_launch(c, true, &o32, maxiter - 1, 0, c->state_r, 0, o->grid, &g1, q1, &rep->ms_kernel[0], &rep->grid));
    const ProblemControl& s1 = q1[0];
    rep->sweeps_launch[0] = g1.sweeps;
    rep->merit_input = s1.merit_input;
    iters = s1.iters;
    thrown = s1.thrown != 0;
    ranges.push_back({0, s1.final_iter});
    merit = s1.merit;
    error = s1.error;
    rep->iters_mixed = iters;
    rep->sweeps = g1.sweeps;
    // closing FP64 refinement, continuing the iteration count: one FP64
    // sweep and the FP64 merit of its iterate (a merit-only pass, no
    // speculative sweeps); if that iterate does not meet the caller's rule,
    // FP64 sweeps continue until it does or maxiter is reached
    for (int pass = 0; !thrown && iters < maxiter; pass++) {
      const int budget = pass == 0 ? 1 : maxiter - iters;
      float ms = 0.f;
      B2_TRY(solve_launch(c, false, o, budget, iters, c->state_r, o->nomerit ? 0 : 1, o->grid, &g2, q2, &ms,
                          &rep->grid));
      const ProblemControl& s2 = q2[0];
      rep->ms_kernel[1] += ms;
      rep->sweeps_launch[1] += g2.sweeps;
      ranges.push_back({iters, iters + s2.final_iter});
      iters += s2.iters;
      thrown = s2.thrown != 0;
      merit = s2.merit;
      error = s2.error;
      rep->sweeps += g2.sweeps;
      const bool meets = o->nomerit ? !(error > o->epsilon) : !(error > o->epsilon || merit > o->meritval);
      if (meets || pass > 0) break;
    }
  } else {
    B2_TRY(solve_launch(c, false, o, maxiter, 0, c->state_r, 0, o->grid, &g1, q1, &rep->ms_kernel[0], &rep->grid));
    const ProblemControl& s1 = q1[0];
    rep->sweeps_launch[0] = g1.sweeps;
    rep->merit_input = s1.merit_input;
    iters = s1.iters;
    thrown = s1.thrown != 0;
    ranges.push_back({0, s1.final_iter});
    merit = s1.merit;
    error = s1.error;
    rep->sweeps = g1.sweeps;
  }
  B2_CK(cudaEventRecord(c->ev[3], st));
  final_global = iters;

  // failure bookkeeping over the sweeps that produced the returned iterates
  std::vector<unsigned long long> fk(maxiter + 2, 0ull);
  std::vector<unsigned> fc(maxiter + 2, 0u);
  B2_CK(cudaMemcpyAsync(fk.data(), c->failkey.p, sizeof(unsigned long long) * (maxiter + 1), cudaMemcpyDeviceToHost, st));
  B2_CK(cudaMemcpyAsync(fc.data(), c->failcount.p, sizeof(unsigned) * (maxiter + 1), cudaMemcpyDeviceToHost, st));
  if (rerhist && iters > 0) B2_CK(cudaMemcpyAsync(rerhist, c->rer.p, sizeof(double) * iters, cudaMemcpyDeviceToHost, st));
  if (merhist && iters > 0) B2_CK(cudaMemcpyAsync(merhist, c->mer.p, sizeof(double) * iters, cudaMemcpyDeviceToHost, st));
  B2_CK(cudaStreamSynchronize(st));
  int last_kind = 0, nfail = 0;
  for (auto& r : ranges)
    for (int s = r.first; s <= r.second && s <= maxiter; s++) {
      if (fk[s]) last_kind = (int)(fk[s] & 3ull);
      nfail += (int)fc[s];
    }
  cudaEventElapsedTime(&rep->ms_device, c->ev[2], c->ev[3]);
  rep->iters = final_global;
  rep->thrown = thrown ? 1 : 0;
  rep->last_fail_kind = last_kind;
  rep->nfailures = nfail;
  rep->merit = o->nomerit ? 0.0 : merit;
  rep->error = error;
  return B2DEV_OK;
}


// ---- batches of independent problems ------------------------------------------

int b2dev_set_colour_order(b2dev_ctx* c, int list_order) {
  if (!c) { set_err("set_colour_order: null context"); return B2DEV_EINVAL; }
  c->colour_list = list_order ? 1 : 0;
  return B2DEV_OK;
}

long long b2dev_colour_reuse_count(b2dev_ctx* c) { return c ? c->colour_reuse : 0; }

int b2dev_set_problems(b2dev_ctx* c, int nprob, const int* row_offsets) {
  if (!c || nprob < 1 || (nprob > 1 && !row_offsets)) { set_err("set_problems: invalid arguments"); return B2DEV_EINVAL; }
  std::vector<int> off(nprob + 1, 0);
  if (nprob > 1) {
    for (int k = 0; k <= nprob; k++) off[k] = row_offsets[k];
    if (off[0] != 0) { set_err("set_problems: offsets must start at 0"); return B2DEV_EINVAL; }
    for (int k = 0; k < nprob; k++)
      if (off[k + 1] < off[k]) { set_err("set_problems: offsets must not decrease"); return B2DEV_EINVAL; }
  }
  c->nprob = nprob;
  c->prob_off = nprob > 1 ? off : std::vector<int>();
  c->ready = false;  // the next assembly lays the problems out
  return B2DEV_OK;
}

int b2dev_problem_free_energy(b2dev_ctx* c, double* out) {
  if (!c || !c->ready || !out) { set_err("problem_free_energy: no local dynamics"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  B2_CK(cudaStreamSynchronize(c->stream));  // the library's work on its stream first
  B2_CK(cudaMemcpy(out, c->pfe.p, sizeof(double) * c->nprob, cudaMemcpyDeviceToHost));
  return B2DEV_OK;
}

int b2dev_set_tile_rows(b2dev_ctx* c, int rows) {
  if (!c || !c->ready || rows < 1 || rows > kWarp) { set_err("set_tile_rows: invalid arguments or no layout"); return B2DEV_EINVAL; }
  DeviceGuard g(c->device);
  c->tile_rows_auto = false;
  return build_tiles(c, rows);
}

int b2dev_tile_rows(b2dev_ctx* c) { return c ? c->tile_rows : 0; }

int b2dev_set_wait_limit(b2dev_ctx* c, double seconds) {
  if (!c || !(seconds >= 0.0) || seconds > 60.0) { set_err("set_wait_limit: 0 <= seconds <= 60"); return B2DEV_EINVAL; }
  c->wait_ns = seconds == 0.0 ? kBarrierLimitNs : std::max(1ull, (unsigned long long)(seconds * 1e9));
  return B2DEV_OK;
}

// Batched solve: one persistent launch over every problem of the context, each
// an independent GAUSS_SEIDEL_Solve with its own stopping decision (FP64
// sweeps). With use_graph the launch sequence (control resets, the
// cooperative solve kernel, the gather of final iterates and the copy of the
// outcomes) is captured once into a CUDA graph and replayed while its
// arguments are unchanged. reps: nprob entries; rerhist/merhist: NULL or
// nprob * opts->maxiter doubles; total: aggregate (may be NULL).
int b2dev_solve_batch(b2dev_ctx* c, const b2dev_solve_opts* o, b2dev_batch_report* reps, double* rerhist,
                      double* merhist, b2dev_solve_report* total, int use_graph) {
  if (!c || !o || !reps) { set_err("solve_batch: null argument"); return B2DEV_EINVAL; }
  if (!c->ready) { set_err("solve_batch: no local dynamics (assemble first)"); return B2DEV_ESTATE; }
  if (o->maxiter <= 0 || o->diagmaxiter <= 0 || o->diagsolver < 0 || o->diagsolver > 3 || o->failure < 0 ||
      o->failure > 2 || o->precision != B2DEV_FP64) {
    set_err("solve_batch: invalid options (batched solves run FP64 sweeps)");
    return B2DEV_EINVAL;
  }
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  const int P = c->nprob, n = c->n;
  memset(reps, 0, sizeof(b2dev_batch_report) * P);
  if (total) memset(total, 0, sizeof *total);
  if (n == 0) {
    for (int k = 0; k < P; k++) reps[k].iters = 1;
    return B2DEV_OK;
  }
  // the canonical state buffers hold the initial iterate
  if (c->state_r != 0) B2_CK(cudaMemcpyAsync(c->R64[0].p, c->R64[c->state_r].p, sizeof(double4) * n, cudaMemcpyDeviceToDevice, st));
  if (c->state_u != &c->Us[0]) B2_CK(cudaMemcpyAsync(c->Us[0].p, c->state_u->p, sizeof(double4) * n, cudaMemcpyDeviceToDevice, st));
  c->state_r = 0;
  c->state_u = &c->Us[0];
  SolveArgs a;
  int grid = 0;
  size_t smem = 0;
  B2_TRY(solve_setup(c, false, o, o->maxiter, 0, 0, 0, o->grid, &a, &grid, &smem));
  const size_t outb = sizeof(SolveControl) + sizeof(ProblemControl) * P;
  if (c->pinned_cap < outb) {
    if (c->pinned) cudaFreeHost(c->pinned);
    c->pinned = nullptr;
    c->pinned_cap = 0;
    B2_CK(cudaMallocHost(&c->pinned, outb));
    c->pinned_cap = outb;
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
  }
  SolveControl* gout = static_cast<SolveControl*>(c->pinned);
  ProblemControl* pout = reinterpret_cast<ProblemControl*>(static_cast<char*>(c->pinned) + sizeof(SolveControl));
  auto enqueue_all = [&]() -> int {
    B2_TRY(solve_enqueue(c, false, a, grid, smem));
    c->launches++;
    k_state_gather<<<blocks_for(n, 256), 256, 0, st>>>(
        n, ptr<int>(c->row_prob), ptr<ProblemControl>(c->pctl), 0, o->nomerit, ptr<double4>(c->R64[0]),
        ptr<double4>(c->R64[1]), ptr<double4>(c->R64[2]), ptr<double4>(c->Us[0]), ptr<double4>(c->Us[1]),
        ptr<double4>(c->Um[0]), ptr<double4>(c->Um[1]), ptr<double>(c->conmerit[0]), ptr<double>(c->conmerit[1]));
    B2_CK(cudaGetLastError());
    B2_CK(cudaMemcpyAsync(gout, c->sctrl.p, sizeof(SolveControl), cudaMemcpyDeviceToHost, st));
    B2_CK(cudaMemcpyAsync(pout, c->pctl.p, sizeof(ProblemControl) * P, cudaMemcpyDeviceToHost, st));
    return B2DEV_OK;
  };
  B2_CK(cudaEventRecord(c->ev[4], st));
  if (use_graph) {
    std::vector<uintptr_t> key;
    const unsigned char* ab = reinterpret_cast<const unsigned char*>(&a);
    for (size_t i = 0; i + sizeof(uintptr_t) <= sizeof a; i += sizeof(uintptr_t)) {
      uintptr_t v;
      memcpy(&v, ab + i, sizeof v);
      key.push_back(v);
    }
    key.push_back((uintptr_t)grid);
    key.push_back((uintptr_t)smem);
    key.push_back((uintptr_t)c->pinned);
    key.push_back((uintptr_t)c->row_prob.p);
    key.push_back((uintptr_t)n);
    key.push_back((uintptr_t)P);
    if (!c->graph || key != c->graph_key) {
      if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
      cudaGraph_t gr = nullptr;
      B2_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      const int rc = enqueue_all();
      const cudaError_t ec = cudaStreamEndCapture(st, &gr);
      if (rc != B2DEV_OK) { if (gr) cudaGraphDestroy(gr); return rc; }
      if (ec != cudaSuccess) { set_err("solve_batch: graph capture failed: %s", cudaGetErrorString(ec)); return B2DEV_ECUDA; }
      const cudaError_t ei = cudaGraphInstantiate(&c->graph, gr, 0);
      cudaGraphDestroy(gr);
      if (ei != cudaSuccess) { c->graph = nullptr; set_err("solve_batch: graph instantiation failed: %s", cudaGetErrorString(ei)); return B2DEV_ECUDA; }
      c->graph_key = key;
    }
    B2_CK(cudaGraphLaunch(c->graph, st));
  } else {
    B2_TRY(enqueue_all());
  }
  B2_CK(cudaEventRecord(c->ev[5], st));
  B2_CK(cudaStreamSynchronize(st));
  c->state_r = 0;
  c->state_u = &c->Us[0];
  c->state_cm = o->nomerit ? nullptr : &c->conmerit[0];
  if (gout->timeout) { set_err("solve_batch: a bounded device-side wait timed out"); return B2DEV_ETIMEOUT; }
  const int pstride = a.pstride, maxiter = o->maxiter;
  std::vector<unsigned long long> fk((size_t)P * pstride);
  std::vector<unsigned> fc((size_t)P * pstride);
  B2_CK(cudaMemcpy(fk.data(), c->failkey.p, sizeof(unsigned long long) * fk.size(), cudaMemcpyDeviceToHost));
  B2_CK(cudaMemcpy(fc.data(), c->failcount.p, sizeof(unsigned) * fc.size(), cudaMemcpyDeviceToHost));
  std::vector<double> rh, mh;
  if (rerhist || merhist) {
    rh.resize((size_t)P * pstride);
    mh.resize((size_t)P * pstride);
    B2_CK(cudaMemcpy(rh.data(), c->rer.p, sizeof(double) * rh.size(), cudaMemcpyDeviceToHost));
    B2_CK(cudaMemcpy(mh.data(), c->mer.p, sizeof(double) * mh.size(), cudaMemcpyDeviceToHost));
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]);
  int maxit = 0, anythrown = 0, nfail_all = 0;
  double mmax = 0.0, emax = 0.0;
  for (int k = 0; k < P; k++) {
    const ProblemControl& q = pout[k];
    b2dev_batch_report& r = reps[k];
    r.iters = q.iters;
    r.thrown = q.thrown;
    r.merit = o->nomerit ? 0.0 : q.merit;
    r.error = q.error;
    r.merit_input = q.merit_input;
    r.ms_to_decision = q.t_stop > gout->t_start ? (double)(q.t_stop - gout->t_start) * 1e-6 : 0.0;
    r.rows = c->prob_off.empty() ? n : c->prob_off[k + 1] - c->prob_off[k];
    if (r.rows == 0) r.iters = 1;  // no rows: one iteration with zero error and merit, as the reference loop does
    int last = 0, nf = 0;
    for (int s = 0; s <= q.final_iter && s <= maxiter; s++) {
      const size_t i = (size_t)k * pstride + s;
      if (fk[i]) last = (int)(fk[i] & 3ull);
      nf += (int)fc[i];
    }
    r.last_fail_kind = last;
    r.nfailures = nf;
    if (rerhist) memcpy(rerhist + (size_t)k * maxiter, rh.data() + (size_t)k * pstride, sizeof(double) * std::min(q.iters, maxiter));
    if (merhist) memcpy(merhist + (size_t)k * maxiter, mh.data() + (size_t)k * pstride, sizeof(double) * std::min(q.iters, maxiter));
    maxit = std::max(maxit, q.iters);
    anythrown |= q.thrown;
    nfail_all += nf;
    mmax = std::max(mmax, r.merit);
    emax = std::max(emax, r.error);
  }
  if (total) {
    total->iters = maxit;
    total->thrown = anythrown;
    total->nfailures = nfail_all;
    total->sweeps = gout->sweeps;
    total->merit = mmax;
    total->error = emax;
    total->ms_device = ms;
    total->ms_kernel[0] = ms;
    total->sweeps_launch[0] = gout->sweeps;
    total->grid = grid;
  }
  return B2DEV_OK;
}

// Autotuner of the batched solve: times one solve of the current problems
// (from the current initial state, restored after every trial) for every
// combination of rows per tile, persistent grid size and staging window, and
// keeps the fastest tile rows in the layout. The chosen grid and staging
// window are returned for the caller's options.
int b2dev_autotune_batch(b2dev_ctx* c, const b2dev_solve_opts* o, b2dev_tune_result* res) {
  if (!c || !o || !res) { set_err("autotune_batch: null argument"); return B2DEV_EINVAL; }
  if (!c->ready) { set_err("autotune_batch: no local dynamics"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  const int n = c->n, P = c->nprob;
  memset(res, 0, sizeof *res);
  if (n == 0) { res->tile_rows = c->tile_rows; return B2DEV_OK; }
  // initial state into a scratch copy
  struct Scratch {  // freed on every return path
    Buf b;
    ~Scratch() { if (b.p) cudaFree(b.p); }
  } scratch;
  Buf& save = scratch.b;
  B2_TRY(ensure(save, sizeof(double4) * 2 * (size_t)n));
  double4* sv = ptr<double4>(save);
  B2_CK(cudaMemcpyAsync(sv, c->R64[c->state_r].p, sizeof(double4) * n, cudaMemcpyDeviceToDevice, st));
  B2_CK(cudaMemcpyAsync(sv + n, c->state_u->p, sizeof(double4) * n, cudaMemcpyDeviceToDevice, st));
  const int rows_c[3] = {32, 16, 8};
  const int stage_c[2] = {0, 128};
  std::vector<b2dev_batch_report> reps(P);
  float best = 1e30f;
  int nt = 0, rc = B2DEV_OK;
  for (int ir = 0; ir < 3 && rc == B2DEV_OK; ir++) {
    rc = build_tiles(c, rows_c[ir]);
    for (int is = 0; is < 2 && rc == B2DEV_OK; is++) {
      b2dev_solve_opts oo = *o;
      oo.stage_blocks = stage_c[is];
      oo.grid = 0;
      SolveArgs a;
      int gmax = 0;
      size_t smem = 0;
      rc = solve_setup(c, false, &oo, oo.maxiter, 0, 0, 0, 0, &a, &gmax, &smem);
      const int grids[3] = {gmax, std::max(1, gmax * 3 / 4), std::max(1, gmax / 2)};
      for (int ig = 0; ig < 3 && rc == B2DEV_OK; ig++) {
        if (ig > 0 && grids[ig] == grids[ig - 1]) continue;
        oo.grid = grids[ig];
        B2_CK(cudaMemcpyAsync(c->R64[0].p, sv, sizeof(double4) * n, cudaMemcpyDeviceToDevice, st));
        B2_CK(cudaMemcpyAsync(c->Us[0].p, sv + n, sizeof(double4) * n, cudaMemcpyDeviceToDevice, st));
        c->state_r = 0;
        c->state_u = &c->Us[0];
        b2dev_solve_report tot;
        rc = b2dev_solve_batch(c, &oo, reps.data(), nullptr, nullptr, &tot, 0);
        if (rc != B2DEV_OK) break;
        if (nt < 32) {
          res->trial_rows[nt] = rows_c[ir];
          res->trial_grid[nt] = oo.grid;
          res->trial_stage[nt] = oo.stage_blocks;
          res->trial_ms[nt] = tot.ms_device;
        }
        nt++;
        if (tot.ms_device < best) {
          best = tot.ms_device;
          res->tile_rows = rows_c[ir];
          res->grid = oo.grid;
          res->stage_blocks = oo.stage_blocks;
          res->ms = tot.ms_device;
        }
      }
    }
  }
  res->ntrials = std::min(nt, 32);
  // the chosen tile rows (kept from now on) and the initial state back in place
  if (rc == B2DEV_OK) {
    c->tile_rows_auto = false;
    rc = build_tiles(c, res->tile_rows);
  }
  cudaMemcpyAsync(c->R64[0].p, sv, sizeof(double4) * n, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(c->Us[0].p, sv + n, sizeof(double4) * n, cudaMemcpyDeviceToDevice, st);
  cudaStreamSynchronize(st);
  c->state_r = 0;
  c->state_u = &c->Us[0];
  c->state_cm = nullptr;
  return rc;
}

int b2dev_sizes(b2dev_ctx* c, int* n, long long* nblocks, int* ncolours, double* free_energy) {
  if (!c) return B2DEV_EINVAL;
  if (n) *n = c->n;
  if (nblocks) *nblocks = c->K;
  if (ncolours) *ncolours = c->ncolours;
  if (free_energy) *free_energy = c->free_energy;
  return B2DEV_OK;
}

int b2dev_get_order(b2dev_ctx* c, int* order) {
  if (!c || !c->ready) { set_err("get_order: no local dynamics"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  B2_CK(cudaStreamSynchronize(c->stream));  // the library's work on its stream first
  if (c->n) B2_CK(cudaMemcpy(order, c->perm.p, sizeof(int) * c->n, cudaMemcpyDeviceToHost));
  return B2DEV_OK;
}

int b2dev_get_colours(b2dev_ctx* c, int* colour) {
  if (!c || !c->ready) { set_err("get_colours: no local dynamics"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  B2_CK(cudaStreamSynchronize(c->stream));  // the library's work on its stream first
  if (c->n) B2_CK(cudaMemcpy(colour, c->colour.p, sizeof(int) * c->n, cudaMemcpyDeviceToHost));
  return B2DEV_OK;
}

int b2dev_get_locdyn(b2dev_ctx* c, double* W, double* A, double* rho, double* B, double* V, int* adjptr, int* adjcol,
                     double* Woff, double* free_energy) {
  if (!c || !c->ready) { set_err("get_locdyn: no local dynamics"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  B2_CK(cudaStreamSynchronize(c->stream));  // the library's work on its stream first
  const int n = c->n;
  const long long K = c->K;
  if (W) B2_CK(cudaMemcpy(W, c->Wii.p, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost));
  if (A) B2_CK(cudaMemcpy(A, c->Aii.p, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost));
  if (rho) B2_CK(cudaMemcpy(rho, c->rho_c.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (B) B2_CK(cudaMemcpy(B, c->B_c.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
  if (V) B2_CK(cudaMemcpy(V, c->V_c.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
  if (adjptr) B2_CK(cudaMemcpy(adjptr, c->adjptr.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
  if (adjcol && K) B2_CK(cudaMemcpy(adjcol, c->adjcol.p, sizeof(int) * K, cudaMemcpyDeviceToHost));
  if (Woff && K) {
    B2_TRY(ensure(c->io, sizeof(double) * 9 * (K + 1)));
    c->launches++;
    k_offdiag_out<<<blocks_for(n, 256), 256, 0, c->stream>>>(n, ptr<int>(c->iperm), ptr<int>(c->adjptr),
                                                             ptr<int>(c->rowptr), ptr<double>(c->W64), c->kstride,
                                                             ptr<double>(c->io));
    B2_CK(cudaMemcpyAsync(Woff, c->io.p, sizeof(double) * 9 * K, cudaMemcpyDeviceToHost, c->stream));
    B2_CK(cudaStreamSynchronize(c->stream));
  }
  if (free_energy) *free_energy = c->free_energy;
  return B2DEV_OK;
}

float b2dev_last_assemble_ms(b2dev_ctx* c) {
  if (!c) return 0.f;
  DeviceGuard g(c->device);
  assemble_time(c);
  return c->assemble_ms;
}

long long b2dev_launch_count(b2dev_ctx* c) { return c ? c->launches : 0; }

// ---- contact-graph colouring for callers that cannot allocate device memory
//
// b2dev_colour_noalloc runs the same Jones-Plassmann kernel as the context
// path, but its scratch (the control block and one selection flag per row)
// lives in this file-scope device array instead of memory obtained with
// cudaMalloc. Every GPU that loads the library keeps the array until exit.
constexpr int kNoAllocMaxRows = 1 << 20;  // rows of the largest graph the entry point accepts
constexpr size_t kNoAllocCtrlBytes = 256;  // control block, padded
static __device__ __align__(256) unsigned char g_colour_scratch[kNoAllocCtrlBytes + sizeof(int) * kNoAllocMaxRows];
static_assert(sizeof(ColourControl) <= kNoAllocCtrlBytes, "colour control block must fit its slot");

namespace {
constexpr int kNoAllocMaxDevices = 64;
struct NoAllocSetup {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_colour_scratch on this device
  int grid = 0;                      // co-resident blocks of the colouring kernel
};
NoAllocSetup g_noalloc[kNoAllocMaxDevices];
std::mutex g_noalloc_mutex;
}  // namespace

int b2dev_trace_sweep(b2dev_ctx* c, int sweep) {
  if (!c) return B2DEV_EINVAL;
  c->trace_sweep = sweep;
  return B2DEV_OK;
}

int b2dev_get_trace(b2dev_ctx* c, double* out) {
  if (!c || !c->ready || !c->trace.p) { set_err("get_trace: no trace recorded"); return B2DEV_ESTATE; }
  DeviceGuard g(c->device);
  B2_CK(cudaStreamSynchronize(c->stream));  // the library's work on its stream first
  const int n = c->n;
  std::vector<double> tmp((size_t)kTraceStride * n);
  std::vector<int> perm(n);
  if (n) {
    B2_CK(cudaMemcpy(tmp.data(), c->trace.p, sizeof(double) * tmp.size(), cudaMemcpyDeviceToHost));
    B2_CK(cudaMemcpy(perm.data(), c->perm.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
  }
  for (int p = 0; p < n; p++)
    memcpy(out + (size_t)kTraceStride * perm[p], tmp.data() + (size_t)kTraceStride * p, sizeof(double) * kTraceStride);
  return B2DEV_OK;
}

int b2dev_colour_noalloc(int device, void* stream, int n, const int* adjptr, const int* adjcol, uint64_t seed,
                         int* colour, int* info) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev || device >= kNoAllocMaxDevices) {
    set_err("colour_noalloc: no CUDA device %d", device);
    return B2DEV_EINVAL;
  }
  if (n < 0 || n > kNoAllocMaxRows) {
    set_err("colour_noalloc: %d rows exceed the fixed scratch of %d rows this entry point holds", n, kNoAllocMaxRows);
    return B2DEV_EINVAL;
  }
  if (n > 0 && (!adjptr || !adjcol || !colour)) {
    set_err("colour_noalloc: null graph or output pointer");
    return B2DEV_EINVAL;
  }
  DeviceGuard g(device);
  cudaStream_t st = (cudaStream_t)stream;
  NoAllocSetup& su = g_noalloc[device];
  {  // set-up, once per device, with the device current
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!su.ready) {
      void* addr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&addr, g_colour_scratch);
      if (e != cudaSuccess) {
        set_err("colour_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return B2DEV_ECUDA;
      }
      int sms = 0, per_sm = 0;
      B2_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
      B2_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_jp_colour, 256, 0));
      if (per_sm < 1) { set_err("colour_noalloc: colouring kernel cannot be resident"); return B2DEV_ECUDA; }
      su.scratch = static_cast<unsigned char*>(addr);
      su.grid = per_sm * sms;
      su.ready = true;
    }
  }
  ColourControl* ctl = reinterpret_cast<ColourControl*>(su.scratch);
  int* sel = reinterpret_cast<int*>(su.scratch + kNoAllocCtrlBytes);
  // the control block starts at zero and every row uncoloured; the selection
  // flags are written before they are read, so the previous call's values are harmless
  B2_CK(cudaMemsetAsync(ctl, 0, sizeof(ColourControl), st));
  if (n > 0) {
    B2_CK(cudaMemsetAsync(colour, 0xff, sizeof(int) * n, st));
    int nn = n;
    unsigned long long sd = seed;
    int lo = 0;  // seeded priorities
    void* args[] = {&nn, (void*)&adjptr, (void*)&adjcol, &sd, &lo, &colour, &sel, &ctl};
    const int grid = std::max(1, std::min(su.grid, blocks_for(n, 256)));
    B2_CK(cudaLaunchCooperativeKernel((const void*)k_jp_colour, grid, 256, args, 0, st));
  }
  if (info)  // timeout flag, overflow flag, number of colours, rounds
    B2_CK(cudaMemcpyAsync(info, &ctl->timeout, 4 * sizeof(int), cudaMemcpyDeviceToDevice, st));
  return B2DEV_OK;
}

int b2dev_diag_solve_batch(b2dev_ctx* c, int n, int solver, int failure, double diagepsilon, int diagmaxiter,
                           int dynamic, double step, const double* W, const double* B, const double* V,
                           const double* rho, const double* gap, const double* friction, const double* restitution,
                           const double* cohesion, double* U, double* R, int* kind) {
  if (!c || n < 0 || solver < 0 || solver > 3 || failure < 0 || failure > 2 || diagmaxiter <= 0) {
    set_err("diag_solve_batch: invalid arguments");
    return B2DEV_EINVAL;
  }
  if (n == 0) return B2DEV_OK;
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  const size_t per = 9 + 3 + 3 + 1 + 1 + 1 + 1 + 1 + 3 + 3;  // doubles per row
  B2_TRY(ensure(c->io, sizeof(double) * per * n + sizeof(int) * (n + 1)));
  double* d = ptr<double>(c->io);
  double *dW = d, *dB = dW + 9 * (size_t)n, *dV = dB + 3 * (size_t)n, *drho = dV + 3 * (size_t)n, *dgap = drho + n;
  double *dfr = dgap + n, *dre = dfr + n, *dco = dre + n, *dU = dco + n, *dR = dU + 3 * (size_t)n;
  int* dk = reinterpret_cast<int*>(dR + 3 * (size_t)n);
  const cudaMemcpyKind h2d = cudaMemcpyHostToDevice, d2h = cudaMemcpyDeviceToHost;
  B2_CK(cudaMemcpyAsync(dW, W, sizeof(double) * 9 * n, h2d, st));
  B2_CK(cudaMemcpyAsync(dB, B, sizeof(double) * 3 * n, h2d, st));
  B2_CK(cudaMemcpyAsync(dV, V, sizeof(double) * 3 * n, h2d, st));
  B2_CK(cudaMemcpyAsync(drho, rho, sizeof(double) * n, h2d, st));
  B2_CK(cudaMemcpyAsync(dgap, gap, sizeof(double) * n, h2d, st));
  B2_CK(cudaMemcpyAsync(dfr, friction, sizeof(double) * n, h2d, st));
  B2_CK(cudaMemcpyAsync(dre, restitution, sizeof(double) * n, h2d, st));
  B2_CK(cudaMemcpyAsync(dco, cohesion, sizeof(double) * n, h2d, st));
  B2_CK(cudaMemcpyAsync(dU, U, sizeof(double) * 3 * n, h2d, st));
  B2_CK(cudaMemcpyAsync(dR, R, sizeof(double) * 3 * n, h2d, st));
  c->launches++;
  k_diag_batch<<<blocks_for(n, 128), 128, 0, st>>>(n, solver, failure, diagepsilon, diagmaxiter, dynamic, step, dW,
                                                   dB, dV, drho, dgap, dfr, dre, dco, dU, dR, dk);
  B2_CK(cudaGetLastError());
  B2_CK(cudaMemcpyAsync(U, dU, sizeof(double) * 3 * n, d2h, st));
  B2_CK(cudaMemcpyAsync(R, dR, sizeof(double) * 3 * n, d2h, st));
  if (kind) B2_CK(cudaMemcpyAsync(kind, dk, sizeof(int) * n, d2h, st));
  B2_CK(cudaStreamSynchronize(st));
  return B2DEV_OK;
}

}  // extern "C"

#include "b2_learn.cuh"
