// b2_learn.cuh -- learned warm start of the contact solve: per-contact
// features, the network's prediction turned into an initial reaction, the
// merit test that keeps the plain start as the fallback, and the C ABI of the
// network (training and inference). Included by b2_device.cu after the
// context definition; the network kernels are in b2_mlp.cuh.
//
// Features of contact row p (dimensionless; v_s = sqrt(|B|^2 + |V|^2 +
// (|R_prev| / rho)^2), rho = 1 / lambda_max(W_ii), h = time step):
//   0      signed log(1 + |gap / (h v_s)|)
//   1-3    V / v_s               relative velocity (local frame: two tangents, normal)
//   4-12   rho W_ii              the diagonal block, column-major
//   13-15  B / v_s               free velocity
//   16-18  R_prev / (rho v_s)    previous-step reaction
//   19     friction coefficient
//   20-21  rho h / m for the master and slave bodies (0 for an obstacle or none)
//   22-24  contact normal in world coordinates (third column of the contact base)
//   25     1 (bias of the first layer)
// The network predicts y = (R - R_prev) / (rho v_s); the initial reaction is
// R_prev + rho v_s y. With the last layer at zero it reproduces the plain
// previous-step start exactly.
#pragma once

#include "b2_mlp.cuh"

namespace {

struct NnRows {
  int n;
  double step;
  const int* perm;
  const double *Wd, *Bv, *Vv, *rho, *gap, *fric;
  const double4* R;  // previous-step reactions (sorted order)
  // scene data (caller order); null when the local dynamics were given directly
  const int *master, *slave, *obst;
  const double *minv, *base;

  __device__ double scale(int p) const {
    const double r = rho[p];
    double b2 = 0.0, v2 = 0.0;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const double bq = Bv[(size_t)q * n + p], vq = Vv[(size_t)q * n + p];
      b2 += bq * bq;
      v2 += vq * vq;
    }
    const double4 rp = R[p];
    const double rl = sqrt(rp.x * rp.x + rp.y * rp.y + rp.z * rp.z) / r;
    return r * (sqrt(b2 + v2 + rl * rl) + 1e-300);
  }

  __device__ void features(int p, float (&x)[b2::mlp::kIn]) const {
    const double r = rho[p];
    const double s = scale(p);  // rho v_s
    const double vs = s / r;
#pragma unroll
    for (int k = 0; k < b2::mlp::kIn; k++) x[k] = 0.f;
    const double g = gap[p] / (step * vs);
    x[0] = (float)copysign(log1p(fabs(g)), g);
#pragma unroll
    for (int q = 0; q < 3; q++) {
      x[1 + q] = (float)(Vv[(size_t)q * n + p] / vs);
      x[13 + q] = (float)(Bv[(size_t)q * n + p] / vs);
    }
#pragma unroll
    for (int q = 0; q < 9; q++) x[4 + q] = (float)(r * Wd[(size_t)q * n + p]);
    const double4 rp = R[p];
    x[16] = (float)(rp.x / s);
    x[17] = (float)(rp.y / s);
    x[18] = (float)(rp.z / s);
    x[19] = (float)fric[p];
    if (master) {
      const int i = perm[p];
      const int m = master[i], sl = slave[i];
      if (m >= 0 && !obst[m]) x[20] = (float)(r * step * minv[m]);
      if (sl >= 0 && !obst[sl]) x[21] = (float)(r * step * minv[sl]);
#pragma unroll
      for (int q = 0; q < 3; q++) x[22 + q] = (float)base[9 * (size_t)i + 6 + q];
    }
    x[b2::mlp::kBiasCol] = 1.f;
  }
};

// features, scale and previous reaction of every row, in caller order (training sets)
__global__ void k_nn_features(NnRows rows, float* __restrict__ feat, double* __restrict__ scale,
                              double* __restrict__ rprev) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= rows.n) return;
  const int i = rows.perm[p];
  float x[b2::mlp::kIn];
  rows.features(p, x);
#pragma unroll
  for (int k = 0; k < b2::mlp::kIn; k++) feat[(size_t)i * b2::mlp::kIn + k] = x[k];
  scale[i] = rows.scale(p);
  const double4 rp = rows.R[p];
  rprev[3 * (size_t)i] = rp.x;
  rprev[3 * (size_t)i + 1] = rp.y;
  rprev[3 * (size_t)i + 2] = rp.z;
}

struct NnSrc {
  NnRows rows;
  __device__ bool operator()(long long row, float (&x)[b2::mlp::kIn]) const {
    if (row >= rows.n) {
#pragma unroll
      for (int k = 0; k < b2::mlp::kIn; k++) x[k] = 0.f;
      return false;
    }
    rows.features((int)row, x);
    return true;
  }
};

// the prediction as an initial reaction (sorted order), both precisions
struct NnDst {
  NnRows rows;
  double4* R64;
  float4* R32;
  __device__ void operator()(long long row, const float (&y)[3]) const {
    const int p = (int)row;
    const double s = rows.scale(p);
    const double4 rp = rows.R[p];
    const double r0 = rp.x + s * (double)y[0], r1 = rp.y + s * (double)y[1], r2 = rp.z + s * (double)y[2];
    R64[p] = make_double4(r0, r1, r2, 0.0);
    R32[p] = make_float4((float)r0, (float)r1, (float)r2, 0.f);
  }
};

// Merit numerators of every row for two sets of reactions Ra and Rb in one
// pass over W (mrf.c:61-87 arithmetic for each: U = B + W_ii R_i + sum_j
// W_ij R_j in list order, up = <A C, C>).
__global__ void k_merit_rows(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                             const double* __restrict__ W64, long long kstride, const double* __restrict__ Wd,
                             const double* __restrict__ Ad, const double* __restrict__ Bv,
                             const double* __restrict__ Vv, const double* __restrict__ gap,
                             const double* __restrict__ fric, const double* __restrict__ rest,
                             const double* __restrict__ coh, double step, int dynamic, const double4* __restrict__ Ra,
                             const double4* __restrict__ Rb, double* __restrict__ upa, double* __restrict__ upb) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  double ua = 0.0, ub = 0.0;
  if (p < n) {
  double B[3], W[9], A[9], V[3], Ua[3], Ub[3];
  const double4 ra = Ra[p], rb = Rb[p];
  const double Rpa[3] = {ra.x, ra.y, ra.z}, Rpb[3] = {rb.x, rb.y, rb.z};
#pragma unroll
  for (int q = 0; q < 3; q++) { B[q] = Bv[(size_t)q * n + p]; V[q] = Vv[(size_t)q * n + p]; }
#pragma unroll
  for (int q = 0; q < 9; q++) { W[q] = Wd[(size_t)q * n + p]; A[q] = Ad[(size_t)q * n + p]; }
  nvaddmul(B, W, Rpa, Ua);
  nvaddmul(B, W, Rpb, Ub);
  for (int k = rowptr[p]; k < rowptr[p + 1]; k++) {
    const int j = col[k];
    const double4 ja = Ra[j], jb = Rb[j];
    double w[9];
#pragma unroll
    for (int q = 0; q < 9; q++) w[q] = W64[q * kstride + k];
    Ua[0] = Ua[0] + (w[0] * ja.x + w[3] * ja.y + w[6] * ja.z);
    Ua[1] = Ua[1] + (w[1] * ja.x + w[4] * ja.y + w[7] * ja.z);
    Ua[2] = Ua[2] + (w[2] * ja.x + w[5] * ja.y + w[8] * ja.z);
    Ub[0] = Ub[0] + (w[0] * jb.x + w[3] * jb.y + w[6] * jb.z);
    Ub[1] = Ub[1] + (w[1] * jb.x + w[4] * jb.y + w[7] * jb.z);
    Ub[2] = Ub[2] + (w[2] * jb.x + w[5] * jb.y + w[8] * jb.z);
  }
  ContactParams cp;
  cp.friction = fric[p]; cp.restitution = rest[p]; cp.cohesion = coh[p]; cp.gap = gap[p]; cp.step = step;
  cp.dynamic = dynamic;
  ua = merit_row(cp, A, V, Ua, Rpa);
  ub = merit_row(cp, A, V, Ub, Rpb);
  }
  // block partials in a fixed order (lanes, then warps): upa[blockIdx.x], upb[blockIdx.x]
  __shared__ double red[2][32];
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) {
    ua += __shfl_down_sync(0xffffffffu, ua, d);
    ub += __shfl_down_sync(0xffffffffu, ub, d);
  }
  if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = ua; red[1][threadIdx.x >> 5] = ub; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sa = 0.0, sb = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) { sa += red[0][w]; sb += red[1][w]; }
    upa[blockIdx.x] = sa;
    upb[blockIdx.x] = sb;
  }
}

}  // namespace

struct b2dev_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sms = 0;
  Buf P, m, v, wpacked, gpart, lpart, err, tiles, loss, gsum;
  long long adam_steps = 0;
};

namespace {

int mlp_check(b2dev_mlp* net) {
  int err = 0;
  B2_CK(cudaMemcpyAsync(&err, net->err.p, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
  B2_CK(cudaStreamSynchronize(net->stream));
  if (err) { set_err("network kernel: a bounded tensor-core wait timed out"); return B2DEV_ETIMEOUT; }
  return B2DEV_OK;
}

// dynamic shared memory limit of the network kernels on the current device
// (set on every call: cheap, and free of shared state between host threads)
int mlp_smem_attr() {
  const int bytes = b2::mlp::kSmemGrad + b2::mlp::kSmemAlign;
  B2_CK(cudaFuncSetAttribute((const void*)b2::mlp::k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  B2_CK(cudaFuncSetAttribute((const void*)b2::mlp::k_mlp_forward<b2::mlp::ArraySrc, b2::mlp::ArrayDst>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  B2_CK(cudaFuncSetAttribute((const void*)b2::mlp::k_mlp_forward<NnSrc, NnDst>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  return B2DEV_OK;
}

// gradient of the loss over the listed tiles (or tiles 0..ntiles-1), one CTA per tile
int mlp_grad_launch(b2dev_mlp* net, int ntiles, const int* tiles, int nrows, const float* feat, const float* target,
                    float inv_n) {
  using namespace b2::mlp;
  B2_TRY(mlp_smem_attr());
  B2_TRY(ensure(net->gpart, sizeof(float) * (size_t)ntiles * kParams));
  B2_TRY(ensure(net->lpart, sizeof(float) * (size_t)(ntiles + 1)));
  k_mlp_grad<<<ntiles, kThreads, kSmemGrad + kSmemAlign, net->stream>>>(
      ptr<unsigned char>(net->wpacked), ptr<float>(net->P), feat, target, tiles, nrows, inv_n, ptr<float>(net->gpart),
      ptr<float>(net->lpart), ptr<int>(net->err));
  B2_CK(cudaGetLastError());
  return B2DEV_OK;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

int b2dev_mlp_nparams(void) { return b2::mlp::kParams; }

int b2dev_mlp_create(int device, void* stream, b2dev_mlp** out) {
  if (!out) { set_err("mlp_create: null output"); return B2DEV_EINVAL; }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    set_err("mlp_create: no CUDA device %d", device);
    return B2DEV_EINVAL;
  }
  DeviceGuard g(device);
  int major = 0, minor = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device);
  if (major != 10 || minor != 0) {
    set_err("mlp_create: the network kernels are built for sm_100a (found sm_%d%d)", major, minor);
    return B2DEV_EUNSUPPORTED;
  }
  b2dev_mlp* net = new b2dev_mlp();
  net->device = device;
  cudaDeviceGetAttribute(&net->sms, cudaDevAttrMultiProcessorCount, device);
  if (stream) {
    net->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) != cudaSuccess) {
      set_err("mlp_create: cudaStreamCreate failed");
      delete net;
      return B2DEV_ECUDA;
    }
    net->own_stream = true;
  }
  using namespace b2::mlp;
  int rc = B2DEV_OK;
  Buf* bufs[] = {&net->P, &net->m, &net->v, &net->gsum};
  for (Buf* b : bufs)
    if (rc == B2DEV_OK) rc = ensure(*b, sizeof(float) * kParams);
  if (rc == B2DEV_OK) rc = ensure(net->wpacked, kPackedBytes);
  if (rc == B2DEV_OK) rc = ensure(net->err, sizeof(int));
  if (rc == B2DEV_OK) rc = ensure(net->loss, sizeof(double) * 4096);
  if (rc == B2DEV_OK) {
    cudaMemsetAsync(net->P.p, 0, sizeof(float) * kParams, net->stream);
    cudaMemsetAsync(net->m.p, 0, sizeof(float) * kParams, net->stream);
    cudaMemsetAsync(net->v.p, 0, sizeof(float) * kParams, net->stream);
    cudaMemsetAsync(net->wpacked.p, 0, kPackedBytes, net->stream);
    cudaMemsetAsync(net->err.p, 0, sizeof(int), net->stream);
    if (cudaStreamSynchronize(net->stream) != cudaSuccess) { set_err("mlp_create: initialisation failed"); rc = B2DEV_ECUDA; }
  }
  if (rc != B2DEV_OK) {
    Buf* all[] = {&net->P, &net->m, &net->v, &net->gsum, &net->wpacked, &net->err, &net->loss};
    for (Buf* b : all)
      if (b->p) cudaFree(b->p);
    if (net->own_stream) cudaStreamDestroy(net->stream);
    delete net;
    return rc;
  }
  *out = net;
  return B2DEV_OK;
}

void b2dev_mlp_destroy(b2dev_mlp* net) {
  if (!net) return;
  DeviceGuard g(net->device);
  cudaStreamSynchronize(net->stream);
  Buf* all[] = {&net->P, &net->m, &net->v, &net->wpacked, &net->gpart, &net->lpart, &net->err, &net->tiles,
                &net->loss, &net->gsum};
  for (Buf* b : all)
    if (b->p) cudaFree(b->p);
  if (net->own_stream) cudaStreamDestroy(net->stream);
  delete net;
}

int b2dev_mlp_set_params(b2dev_mlp* net, const float* params) {
  if (!net || !params) { set_err("mlp_set_params: null argument"); return B2DEV_EINVAL; }
  DeviceGuard g(net->device);
  using namespace b2::mlp;
  B2_CK(cudaMemcpyAsync(net->P.p, params, sizeof(float) * kParams, cudaMemcpyHostToDevice, net->stream));
  B2_CK(cudaMemsetAsync(net->m.p, 0, sizeof(float) * kParams, net->stream));
  B2_CK(cudaMemsetAsync(net->v.p, 0, sizeof(float) * kParams, net->stream));
  net->adam_steps = 0;
  k_mlp_pack<<<blocks_for(kParams, 256), 256, 0, net->stream>>>(ptr<float>(net->P), ptr<unsigned char>(net->wpacked));
  B2_CK(cudaGetLastError());
  B2_CK(cudaStreamSynchronize(net->stream));
  return B2DEV_OK;
}

int b2dev_mlp_get_params(b2dev_mlp* net, float* params) {
  if (!net || !params) { set_err("mlp_get_params: null argument"); return B2DEV_EINVAL; }
  DeviceGuard g(net->device);
  B2_CK(cudaMemcpyAsync(params, net->P.p, sizeof(float) * b2::mlp::kParams, cudaMemcpyDeviceToHost, net->stream));
  B2_CK(cudaStreamSynchronize(net->stream));
  return B2DEV_OK;
}

int b2dev_mlp_grad(b2dev_mlp* net, int nrows, const float* feat, const float* target, float* grad, double* loss) {
  using namespace b2::mlp;
  if (!net || nrows <= 0 || !feat || !target || !grad) { set_err("mlp_grad: invalid arguments"); return B2DEV_EINVAL; }
  DeviceGuard g(net->device);
  const int ntiles = (nrows + kRows - 1) / kRows;
  B2_TRY(mlp_grad_launch(net, ntiles, nullptr, nrows, feat, target, 1.0f / (float)nrows));
  std::vector<float> part((size_t)ntiles * kParams), lp(ntiles);
  B2_CK(cudaMemcpyAsync(part.data(), net->gpart.p, sizeof(float) * part.size(), cudaMemcpyDeviceToHost, net->stream));
  B2_CK(cudaMemcpyAsync(lp.data(), net->lpart.p, sizeof(float) * ntiles, cudaMemcpyDeviceToHost, net->stream));
  B2_TRY(mlp_check(net));
  for (int p = 0; p < kParams; p++) {
    double s = 0.0;
    for (int t = 0; t < ntiles; t++) s += part[(size_t)t * kParams + p];
    grad[p] = (float)s;
  }
  if (loss) {
    double s = 0.0;
    for (int t = 0; t < ntiles; t++) s += lp[t];
    *loss = s / nrows;
  }
  return B2DEV_OK;
}

int b2dev_mlp_train(b2dev_mlp* net, int nrows, const float* feat, const float* target, int epochs, int batch_tiles,
                    double lr, uint64_t seed, double* epoch_loss) {
  using namespace b2::mlp;
  if (!net || nrows <= 0 || !feat || !target || epochs < 0 || batch_tiles <= 0 || !(lr > 0.0)) {
    set_err("mlp_train: invalid arguments");
    return B2DEV_EINVAL;
  }
  DeviceGuard g(net->device);
  const int ntiles = (nrows + kRows - 1) / kRows;
  const int last_rows = nrows - (ntiles - 1) * kRows;
  const int steps_per_epoch = (ntiles + batch_tiles - 1) / batch_tiles;
  B2_TRY(ensure(net->tiles, sizeof(int) * (size_t)ntiles));
  B2_TRY(ensure(net->loss, sizeof(double) * (size_t)std::max(steps_per_epoch, 1)));
  std::vector<int> order(ntiles);
  std::vector<double> losses(steps_per_epoch);
  uint64_t rs = seed;
  const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  for (int e = 0; e < epochs; e++) {
    for (int t = 0; t < ntiles; t++) order[t] = t;
    for (int t = ntiles - 1; t > 0; t--) std::swap(order[t], order[(int)(splitmix(rs) % (uint64_t)(t + 1))]);
    B2_CK(cudaMemcpyAsync(net->tiles.p, order.data(), sizeof(int) * ntiles, cudaMemcpyHostToDevice, net->stream));
    for (int b = 0; b < steps_per_epoch; b++) {
      const int t0 = b * batch_tiles, nt = std::min(batch_tiles, ntiles - t0);
      long long rows = 0;
      for (int t = t0; t < t0 + nt; t++) rows += order[t] == ntiles - 1 ? last_rows : kRows;
      B2_TRY(mlp_grad_launch(net, nt, ptr<int>(net->tiles) + t0, nrows, feat, target, 1.0f / (float)rows));
      net->adam_steps++;
      const float bc1 = 1.0f - powf(beta1, (float)net->adam_steps), bc2 = 1.0f - powf(beta2, (float)net->adam_steps);
      k_mlp_adam<<<blocks_for(kParams, 256), 256, 0, net->stream>>>(
          ptr<float>(net->P), ptr<float>(net->m), ptr<float>(net->v), ptr<float>(net->gpart), nt, (float)lr, beta1,
          beta2, eps, bc1, bc2, ptr<unsigned char>(net->wpacked), ptr<float>(net->lpart), ptr<double>(net->loss) + b);
      B2_CK(cudaGetLastError());
    }
    B2_CK(cudaMemcpyAsync(losses.data(), net->loss.p, sizeof(double) * steps_per_epoch, cudaMemcpyDeviceToHost,
                          net->stream));
    B2_TRY(mlp_check(net));
    if (epoch_loss) {
      double s = 0.0;
      for (double l : losses) s += l;
      epoch_loss[e] = s / nrows;
    }
  }
  return B2DEV_OK;
}

int b2dev_mlp_forward(b2dev_mlp* net, int nrows, const float* feat, float* out) {
  using namespace b2::mlp;
  if (!net || nrows < 0 || (nrows > 0 && (!feat || !out))) { set_err("mlp_forward: invalid arguments"); return B2DEV_EINVAL; }
  if (nrows == 0) return B2DEV_OK;
  DeviceGuard g(net->device);
  B2_TRY(mlp_smem_attr());
  const int ntiles = (nrows + kRows - 1) / kRows;
  const int grid = std::min(ntiles, net->sms);
  ArraySrc src{feat, nrows};
  ArrayDst dst{out};
  k_mlp_forward<ArraySrc, ArrayDst><<<grid, kThreads, kSmemGrad + kSmemAlign, net->stream>>>(
      ptr<unsigned char>(net->wpacked), ptr<float>(net->P), ntiles, src, dst, ptr<int>(net->err));
  B2_CK(cudaGetLastError());
  return mlp_check(net);
}

}  // extern "C"

namespace {

NnRows nn_rows(b2dev_ctx* c) {
  NnRows r;
  r.n = c->n;
  r.step = c->step;
  r.perm = ptr<int>(c->perm);
  r.Wd = ptr<double>(c->Wd); r.Bv = ptr<double>(c->Bv); r.Vv = ptr<double>(c->Vv);
  r.rho = ptr<double>(c->rho); r.gap = ptr<double>(c->gap); r.fric = ptr<double>(c->fric);
  r.R = ptr<double4>(c->R64[c->state_r]);
  const bool scene = c->have_scene && c->assembled_mode;
  r.master = scene ? ptr<int>(c->master) : nullptr;
  r.slave = scene ? ptr<int>(c->slave) : nullptr;
  r.obst = scene ? ptr<int>(c->obst) : nullptr;
  r.minv = scene ? ptr<double>(c->minv) : nullptr;
  r.base = scene ? ptr<double>(c->base) : nullptr;
  return r;
}

// merit of reactions R (sorted order) into *out (host)
// Merits (mrf.c:176-184) of two sets of reactions, one pass over W.
int merit_of2(b2dev_ctx* c, const double4* Ra, const double4* Rb, double* outa, double* outb) {
  const int n = c->n;
  cudaStream_t st = c->stream;
  const int nb = blocks_for(n, 128);
  B2_TRY(ensure(c->fe_part, sizeof(double) * 2 * (nb + 1)));
  double* pa = ptr<double>(c->fe_part);
  double* pb = pa + (nb + 1);
  c->launches++;
  k_merit_rows<<<nb, 128, 0, st>>>(n, ptr<int>(c->rowptr), ptr<int>(c->col), ptr<double>(c->W64),
                                                   c->kstride, ptr<double>(c->Wd), ptr<double>(c->Ad),
                                                   ptr<double>(c->Bv), ptr<double>(c->Vv), ptr<double>(c->gap),
                                                   ptr<double>(c->fric), ptr<double>(c->rest), ptr<double>(c->coh),
                                                   c->step, c->dynamic, Ra, Rb, pa, pb);
  B2_TRY(ensure(c->io, sizeof(double) * 2));
  c->launches += 2;
  k_sum_partials<<<1, 1024, 0, st>>>(pa, nb, ptr<double>(c->io));  // 0.5 sum up
  k_sum_partials<<<1, 1024, 0, st>>>(pb, nb, ptr<double>(c->io) + 1);
  double half[2] = {0.0, 0.0};
  B2_CK(cudaMemcpyAsync(half, c->io.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
  B2_CK(cudaStreamSynchronize(st));
  double lo = c->free_energy < DBL_EPSILON ? 1.0 : c->free_energy;  // mrf.c:45
  lo = lo == 0.0 ? 1.0 : lo;
  *outa = half[0] / lo;
  *outb = half[1] / lo;
  return B2DEV_OK;
}

}  // namespace

extern "C" {

int b2dev_nn_features(b2dev_ctx* c, float* feat, double* scale, double* rprev) {
  if (!c || !c->ready) { set_err("nn_features: no local dynamics"); return B2DEV_ESTATE; }
  if (c->n > 0 && (!feat || !scale || !rprev)) { set_err("nn_features: null output"); return B2DEV_EINVAL; }
  if (c->n == 0) return B2DEV_OK;
  DeviceGuard g(c->device);
  c->launches++;
  k_nn_features<<<blocks_for(c->n, 128), 128, 0, c->stream>>>(nn_rows(c), feat, scale, rprev);
  B2_CK(cudaGetLastError());
  B2_CK(cudaStreamSynchronize(c->stream));
  return B2DEV_OK;
}

int b2dev_nn_warm_start(b2dev_ctx* c, b2dev_mlp* net, double accept_ratio, b2dev_nn_report* rep) {
  if (c && c->has_kinds) {
    set_err("nn_warm_start: the learned start covers contact rows only; this problem has bilateral constraints");
    return B2DEV_EUNSUPPORTED;
  }
  using namespace b2::mlp;
  if (!c || !c->ready || !net || !rep || !(accept_ratio > 0.0 && accept_ratio <= 1.0)) {
    set_err("nn_warm_start: invalid arguments");
    return B2DEV_EINVAL;
  }
  if (net->device != c->device) { set_err("nn_warm_start: network and context on different devices"); return B2DEV_EINVAL; }
  memset(rep, 0, sizeof *rep);
  const int n = c->n;
  if (n == 0) return B2DEV_OK;
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  B2_TRY(mlp_smem_attr());
  // the prediction goes to a reaction buffer the state does not use
  const int cand = (c->state_r + 1) % 3;
  B2_TRY(ensure(c->R64[cand], sizeof(double4) * (n + 1)));
  B2_TRY(ensure(c->R32[cand], sizeof(float4) * (n + 1)));
  B2_CK(cudaEventRecord(c->ev[6], st));
  // the network reads weights written on its own stream
  B2_CK(cudaEventRecord(c->ev[7], net->stream));
  B2_CK(cudaStreamWaitEvent(st, c->ev[7], 0));
  B2_CK(cudaMemsetAsync(net->err.p, 0, sizeof(int), st));
  const int ntiles = (n + kRows - 1) / kRows;
  const int grid = std::min(ntiles, c->sms);
  NnSrc src{nn_rows(c)};
  NnDst dst{nn_rows(c), ptr<double4>(c->R64[cand]), ptr<float4>(c->R32[cand])};
  c->launches++;
  k_mlp_forward<NnSrc, NnDst><<<grid, kThreads, kSmemGrad + kSmemAlign, st>>>(
      ptr<unsigned char>(net->wpacked), ptr<float>(net->P), ntiles, src, dst, ptr<int>(net->err));
  B2_CK(cudaGetLastError());
  int err = 0;
  B2_CK(cudaMemcpyAsync(&err, net->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_TRY(merit_of2(c, ptr<double4>(c->R64[cand]), ptr<double4>(c->R64[c->state_r]), &rep->merit_nn,
                   &rep->merit_plain));
  if (err) { set_err("nn_warm_start: a bounded tensor-core wait timed out"); return B2DEV_ETIMEOUT; }
  // the plain start stays unless the network's reactions have a merit below
  // accept_ratio times the plain start's (1: any improvement)
  rep->used_nn = rep->merit_nn < accept_ratio * rep->merit_plain ? 1 : 0;
  if (rep->used_nn) c->state_r = cand;
  B2_CK(cudaEventRecord(c->ev[7], st));
  B2_CK(cudaEventSynchronize(c->ev[7]));
  cudaEventElapsedTime(&rep->ms, c->ev[6], c->ev[7]);
  return B2DEV_OK;
}

}  // extern "C"
