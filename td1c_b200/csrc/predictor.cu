// predictor.cu -- the learned mean-field predictor's data path: history ring,
// per-unit Gram matrices, the exact judge, network inputs and the predicted
// stage fields.
//
// The RK4 stages of a split2 step (clcrk inside tdse_split2) each form the
// pair potentials W (bas_sph2ang2 of the Poisson solution, hprod_mkv2mf.F90)
// and the integrals int2e from the stage orbitals.  The learned form forms
// them exactly once per step, at the step's start state y_n (W_n, int2e_n),
// and gives the four stages values at the stage times t_n + c dt (c = 0,
// 1/2, 1/2, 1) from the history W_n, W_{n-1}, ...:
//   c = 1:    W = sum_h w_h(u) W_{n-h}, h = 0..3, per unit u,
//             w = (4, -6, 4, -1) (the cubic through the last four steps) + dw(u),
//             dw = 1e-3 x the network's output (per unit, from its Gram matrix);
//   c = 1/2:  the cubic interpolant through n-2, n-1, n and the c = 1 value:
//             W = 15/16 W_n - 5/16 W_{n-1} + 1/16 W_{n-2} + 5/16 W(c = 1);
//   c = 0:    W_n itself.
// A unit is one stored pair and one FEDVR element (all theta points of the
// element's radial points), so the weights may follow the radial structure of
// each pair field; int2e takes the same formulas with the cubic weights.
//
// The exact W_n is also the judge of the prediction made one step earlier:
// per unit, |sum_h w_h W_{n-1-h} - W_n|^2 = w^H G w - 2 Re(w^H g) + t with the
// Gram matrix G of the previous four history values, g_h = <W_{n-1-h}, W_n>
// and t = |W_n|^2, evaluated in FP64; the step's relative error is
// sqrt(sum_u err_u / sum_u t_u), summed in a fixed order.
//
// Ring slot of history value n - h: (n - h) mod 5, n the device step counter.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

constexpr int LP_H = 4;      // history values a prediction combines
constexpr int LP_SLOTS = 5;  // ring slots: the history plus the newest value
constexpr int LP_NF = 32;    // network inputs per unit
// the network's outputs are weight corrections in units of LP_DW (the cubic's
// one-step error is ~1e-4 to 1e-6 of a unit's norm, so useful corrections are
// small); each correction is limited to |dw| <= 1
constexpr double LP_DW = 1e-3;

__device__ __forceinline__ int lp_slot(int n, int h) { return ((n - h) % LP_SLOTS + LP_SLOTS) % LP_SLOTS; }

// unit u = pair * nfe + element; its radial points [e nd, min((e + 1) nd, Nr))
__device__ __forceinline__ void lp_unit(const LpArgs& a, int u, int& p, int& r0, int& nr) {
  p = u / a.nfe;
  const int e = u % a.nfe;
  r0 = e * a.nd;
  nr = min(a.nd, a.Nr - r0);
}

// One CTA per unit: pushes W_n (from a.W) into its ring slot, forms
// <W_{n-h}, W_n> for h = 0..4 (h = 0: t), judges the last prediction, and
// shifts the unit's Gram matrix.  Inner products in FP64 with a fixed-order
// block reduction.
__global__ void __launch_bounds__(256) lp_push_kernel(LpArgs a) {
  __shared__ double red[8][2 * (LP_H + 1)];
  const int u = blockIdx.x, n = *a.counter;
  int p, r0, nr;
  lp_unit(a, u, p, r0, nr);
  const size_t ng = (size_t)a.nlat * a.Nr;
  const cplx* Wn = a.W + (size_t)p * ng;
  cplx* dst = a.ring + (size_t)lp_slot(n, 0) * a.nw + (size_t)p * ng;
  const cplx* prev[LP_H];
#pragma unroll
  for (int h = 0; h < LP_H; ++h) prev[h] = a.ring + (size_t)lp_slot(n, h + 1) * a.nw + (size_t)p * ng;
  double acc[2 * (LP_H + 1)] = {};
  const int npts = a.nlat * nr;
  for (int i = threadIdx.x; i < npts; i += blockDim.x) {
    const size_t off = (size_t)(i / nr) * a.Nr + r0 + i % nr;
    const cplx x = Wn[off];
    dst[off] = x;
    acc[0] += x.x * x.x + x.y * x.y;
#pragma unroll
    for (int h = 0; h < LP_H; ++h) {
      const cplx q = prev[h][off];  // <q, x> = conj(q) x
      acc[2 + 2 * h] += q.x * x.x + q.y * x.y;
      acc[3 + 2 * h] += q.x * x.y - q.y * x.x;
    }
  }
  // fixed-order reduction: warp shuffles, then warp 0 over the warps
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 2 * (LP_H + 1); ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double s[2 * (LP_H + 1)];
  for (int k = 0; k < 2 * (LP_H + 1); ++k) {
    s[k] = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s[k] += red[w][k];
  }
  const double t = s[0];
  cplx g[LP_H];  // g[h] = <W_{n-1-h}, W_n>
  for (int h = 0; h < LP_H; ++h) g[h] = mkc(s[2 + 2 * h], s[3 + 2 * h]);
  // judge the prediction the weights w of the previous step made for W_n
  cplx* G = a.gram + (size_t)u * LP_H * LP_H;  // G[i][j] = <x_i, x_j>, x_0 the newest of the previous history
  const cplx* w = a.weights + (size_t)u * LP_H;
  double err = t;
  for (int i = 0; i < LP_H; ++i) {
    cplx gw = mkc(0.0, 0.0);
    for (int j = 0; j < LP_H; ++j) cfma(gw, G[i * LP_H + j], w[j]);
    const cplx wi = w[i];
    err += wi.x * gw.x + wi.y * gw.y;            // Re(conj(w_i) (G w)_i)
    err -= 2.0 * (wi.x * g[i].x + wi.y * g[i].y);  // - 2 Re(conj(w_i) g_i)
  }
  a.err[u] = err;
  a.tnorm[u] = t;
  if (a.record) {  // training record: the Gram matrix and target of the prediction just judged
    double* rec = a.record + ((size_t)(*a.rec_count) * a.nu + u) * LP_REC;
    for (int k = 0; k < LP_H * LP_H; ++k) { rec[2 * k] = G[k].x; rec[2 * k + 1] = G[k].y; }
    for (int h = 0; h < LP_H; ++h) { rec[32 + 2 * h] = g[h].x; rec[33 + 2 * h] = g[h].y; }
    rec[40] = t;
  }
  // shift: x_0 <- W_n, x_h <- x_{h-1}
  cplx Gn[LP_H * LP_H];
  Gn[0] = mkc(t, 0.0);
  for (int j = 1; j < LP_H; ++j) { Gn[j] = cconj(g[j - 1]); Gn[j * LP_H] = g[j - 1]; }
  for (int i = 1; i < LP_H; ++i)
    for (int j = 1; j < LP_H; ++j) Gn[i * LP_H + j] = G[(i - 1) * LP_H + (j - 1)];
  for (int k = 0; k < LP_H * LP_H; ++k) G[k] = Gn[k];
}

// The step's judge value, sqrt(sum err / sum t) over units in a fixed order;
// the running maximum over the window; the step counter and record count advance.
__global__ void lp_judge_kernel(LpArgs a) {
  __shared__ double se[256], st[256];
  double e = 0.0, t = 0.0;
  for (int u = threadIdx.x; u < a.nu; u += blockDim.x) { e += fmax(a.err[u], 0.0); t += a.tnorm[u]; }
  se[threadIdx.x] = e;
  st[threadIdx.x] = t;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) { se[threadIdx.x] += se[threadIdx.x + o]; st[threadIdx.x] += st[threadIdx.x + o]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double rel = st[0] > 0.0 ? sqrt(se[0] / st[0]) : 0.0;
    a.judge[0] = rel;                    // this step's value
    a.judge[1] = fmax(a.judge[1], rel);  // the window's maximum (reset by the host)
    *a.counter += 1;
    if (a.record) *a.rec_count += 1;
  }
}

// Network inputs of every unit from the Gram matrix of the four history
// values the prediction combines (x_0 newest): in FP64, the Gram matrix of
// the finite differences d_0 = x_0, d_1 = x_0 - x_1, d_2 = x_0 - 2 x_1 + x_2,
// d_3 = x_0 - 3 x_1 + 3 x_2 - x_3 (the history's value, slope, curvature and
// third difference), then log10 |d_1| / |d_0|, log10 |d_2| / |d_1|,
// log10 |d_3| / |d_2| (scaled by 1/4), the correlations of (d_1, d_2),
// (d_2, d_3), (d_1, d_3) (re, im), the element's position and the pair's
// kind; zero padding to 32.
__device__ void lp_feature_row(const cplx* G, int e, int nfe, int kind, float* x) {
  const double D[LP_H][LP_H] = {{1, 0, 0, 0}, {1, -1, 0, 0}, {1, -2, 1, 0}, {1, -3, 3, -1}};
  cplx Gd[LP_H][LP_H];
  for (int a = 0; a < LP_H; ++a)
    for (int b = 0; b < LP_H; ++b) {
      cplx v = mkc(0.0, 0.0);
      for (int i = 0; i < LP_H; ++i)
        for (int j = 0; j < LP_H; ++j) {
          const double c = D[a][i] * D[b][j];
          if (c != 0.0) { v.x += c * G[i * LP_H + j].x; v.y += c * G[i * LP_H + j].y; }
        }
      Gd[a][b] = v;
    }
  double nrm[LP_H];
  for (int a = 0; a < LP_H; ++a) nrm[a] = sqrt(fmax(Gd[a][a].x, 1e-300));
  int k = 0;
  for (int a = 1; a < LP_H; ++a) x[k++] = (float)(0.25 * fmax(log10(nrm[a] / nrm[a - 1]), -40.0));
  const int pr[3][2] = {{1, 2}, {2, 3}, {1, 3}};
  for (int q = 0; q < 3; ++q) {
    const int a = pr[q][0], b = pr[q][1];
    const double sc = 1.0 / (nrm[a] * nrm[b]);
    x[k++] = (float)fmin(fmax(Gd[a][b].x * sc, -1.0), 1.0);
    x[k++] = (float)fmin(fmax(Gd[a][b].y * sc, -1.0), 1.0);
  }
  x[k++] = (float)((e + 0.5) / nfe);
  x[k++] = (float)(kind == 0);
  x[k++] = (float)(kind == 2);
  while (k < LP_NF) x[k++] = 0.f;
}

__global__ void lp_features_kernel(LpArgs a) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= a.nu) return;
  const int p = u / a.nfe, e = u % a.nfe;
  lp_feature_row(a.gram + (size_t)u * LP_H * LP_H, e, a.nfe, a.pair_kind[p], a.feat + (size_t)u * LP_NF);
}

// weights of every unit for c = 1: the cubic's plus LP_DW times the network
// output (re, im per history value), each correction limited to |dw| <= 1
__global__ void lp_weights_kernel(LpArgs a) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= a.nu) return;
  const double cub[LP_H] = {4.0, -6.0, 4.0, -1.0};
  for (int h = 0; h < LP_H; ++h) {
    double dr = a.use_net ? LP_DW * a.net_out[(size_t)u * 2 * LP_H + 2 * h] : 0.0;
    double di = a.use_net ? LP_DW * a.net_out[(size_t)u * 2 * LP_H + 2 * h + 1] : 0.0;
    dr = fmin(fmax(dr, -1.0), 1.0);
    di = fmin(fmax(di, -1.0), 1.0);
    a.weights[(size_t)u * LP_H + h] = mkc(cub[h] + dr, di);
  }
}

// W (stage value at c = 1 or 1/2) into a.W from the ring, per unit weights
__global__ void lp_apply_kernel(LpArgs a, int half) {
  const size_t nw = a.nw;
  const int n = *a.counter - 1;  // the history's newest value (the judge advanced the counter)
  const cplx* x[LP_H];
#pragma unroll
  for (int h = 0; h < LP_H; ++h) x[h] = a.ring + (size_t)lp_slot(n, h) * nw;
  const size_t ng = (size_t)a.nlat * a.Nr;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < nw; t += (size_t)gridDim.x * blockDim.x) {
    const int p = (int)(t / ng);
    const int r = (int)(t % a.Nr);
    const int e = min(r / a.nd, a.nfe - 1);
    const cplx* w = a.weights + ((size_t)p * a.nfe + e) * LP_H;
    cplx v = mkc(0.0, 0.0);
#pragma unroll
    for (int h = 0; h < LP_H; ++h) cfma(v, w[h], x[h][t]);
    if (half) {  // 15/16 W_n - 5/16 W_{n-1} + 1/16 W_{n-2} + 5/16 W(c = 1)
      v = cscale(v, 0.3125);
      const cplx a0 = x[0][t], a1 = x[1][t], a2 = x[2][t];
      v.x += 0.9375 * a0.x - 0.3125 * a1.x + 0.0625 * a2.x;
      v.y += 0.9375 * a0.y - 0.3125 * a1.y + 0.0625 * a2.y;
    }
    a.W[t] = v;
  }
}

// int2e: push the exact value (mode 0), or the stage value at c = 1 (mode 1) or 1/2 (mode 2)
__global__ void lp_int2e_kernel(LpArgs a, int mode) {
  const int n = *a.counter - (mode == 0 ? 0 : 1);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < a.ni; t += gridDim.x * blockDim.x) {
    if (mode == 0) {
      a.iring[(size_t)lp_slot(n, 0) * a.ni + t] = a.int2e[t];
      continue;
    }
    const cplx i0 = a.iring[(size_t)lp_slot(n, 0) * a.ni + t], i1 = a.iring[(size_t)lp_slot(n, 1) * a.ni + t];
    const cplx i2 = a.iring[(size_t)lp_slot(n, 2) * a.ni + t], i3 = a.iring[(size_t)lp_slot(n, 3) * a.ni + t];
    cplx v;
    v.x = 4.0 * i0.x - 6.0 * i1.x + 4.0 * i2.x - i3.x;
    v.y = 4.0 * i0.y - 6.0 * i1.y + 4.0 * i2.y - i3.y;
    if (mode == 2) {
      v.x = 0.3125 * v.x + 0.9375 * i0.x - 0.3125 * i1.x + 0.0625 * i2.x;
      v.y = 0.3125 * v.y + 0.9375 * i0.y - 0.3125 * i1.y + 0.0625 * i2.y;
    }
    a.int2e[t] = v;
  }
}

int launch_lp_push_judge(const LpArgs& a, cudaStream_t st) {
  if (a.ni > 0) lp_int2e_kernel<<<(a.ni + 255) / 256, 256, 0, st>>>(a, 0);  // no active orbitals: no int2e
  lp_push_kernel<<<a.nu, 256, 0, st>>>(a);
  lp_judge_kernel<<<1, 256, 0, st>>>(a);
  return (int)cudaGetLastError();
}
int launch_lp_features(const LpArgs& a, cudaStream_t st) {
  lp_features_kernel<<<(a.nu + 127) / 128, 128, 0, st>>>(a);
  return (int)cudaGetLastError();
}
int launch_lp_weights(const LpArgs& a, cudaStream_t st) {
  lp_weights_kernel<<<(a.nu + 127) / 128, 128, 0, st>>>(a);
  return (int)cudaGetLastError();
}
int launch_lp_stage(const LpArgs& a, int half, cudaStream_t st) {
  lp_apply_kernel<<<148 * 8, 256, 0, st>>>(a, half);
  if (a.ni > 0) lp_int2e_kernel<<<(a.ni + 255) / 256, 256, 0, st>>>(a, half ? 2 : 1);
  return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// training helpers: network inputs of recorded samples and the loss gradient
// ---------------------------------------------------------------------------
// rec: [n][LP_REC] records (G, g, t); unit ids: sample s is unit s % nu
__global__ void lp_rec_features_kernel(int n, const double* __restrict__ rec, const int* __restrict__ idx, int nu, int nfe,
                                       const int* __restrict__ pair_kind, float* __restrict__ x) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const long i = idx ? idx[s] : s;
  const double* r = rec + (size_t)i * LP_REC;
  cplx G[LP_H * LP_H];
  for (int k = 0; k < LP_H * LP_H; ++k) G[k] = mkc(r[2 * k], r[2 * k + 1]);
  const int u = (int)(i % nu);
  lp_feature_row(G, u % nfe, nfe, pair_kind[u / nfe], x + (size_t)s * LP_NF);
}

// relative squared error of each sample's prediction with weights cubic + dw,
// and dL/d(dw) for the mean over the batch (FP64, cast to FP32 for the network)
__global__ void lp_loss_kernel(int n, const double* __restrict__ rec, const int* __restrict__ idx,
                               const float* __restrict__ out, float* __restrict__ dy, double* __restrict__ loss, int use_net) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const long i = idx ? idx[s] : s;
  const double* r = rec + (size_t)i * LP_REC;
  const double cub[LP_H] = {4.0, -6.0, 4.0, -1.0};
  cplx w[LP_H];
  for (int h = 0; h < LP_H; ++h) {
    double dr = use_net ? LP_DW * out[(size_t)s * 2 * LP_H + 2 * h] : 0.0;
    double di = use_net ? LP_DW * out[(size_t)s * 2 * LP_H + 2 * h + 1] : 0.0;
    w[h] = mkc(cub[h] + fmin(fmax(dr, -1.0), 1.0), fmin(fmax(di, -1.0), 1.0));
  }
  const double t = fmax(r[40], 1e-300);
  double err = r[40];
  for (int a = 0; a < LP_H; ++a) {
    cplx gw = mkc(-r[32 + 2 * a], -r[33 + 2 * a]);  // (G w - g)_a
    for (int b = 0; b < LP_H; ++b) cfma(gw, mkc(r[2 * (a * LP_H + b)], r[2 * (a * LP_H + b) + 1]), w[b]);
    // err = w^H G w - 2 Re(w^H g) + t = Re(w^H (G w - g)) - Re(w^H g) + t
    err += w[a].x * gw.x + w[a].y * gw.y - (w[a].x * r[32 + 2 * a] + w[a].y * r[33 + 2 * a]);
    if (dy) {
      // d/d Re w_a = 2 Re (G w - g)_a, d/d Im w_a = 2 Im (G w - g)_a, times LP_DW for the
      // network output; zero where the limit is active
      const double dr = use_net ? LP_DW * out[(size_t)s * 2 * LP_H + 2 * a] : 0.0;
      const double di = use_net ? LP_DW * out[(size_t)s * 2 * LP_H + 2 * a + 1] : 0.0;
      dy[(size_t)s * 2 * LP_H + 2 * a] = fabs(dr) < 1.0 ? (float)(LP_DW * 2.0 * gw.x / t / n) : 0.f;
      dy[(size_t)s * 2 * LP_H + 2 * a + 1] = fabs(di) < 1.0 ? (float)(LP_DW * 2.0 * gw.y / t / n) : 0.f;
    }
  }
  loss[s] = fmax(err, 0.0) / t;
}

}  // namespace td1c

using namespace td1c;

extern "C" {

int td1c_lp_features(int n, const double* rec, const int* idx, int nu, int nfe, const int* pair_kind, float* x, void* stream) {
  if (n < 0 || nu < 1 || nfe < 1 || !rec || !pair_kind || !x) return ST_CONFIG;
  if (n) lp_rec_features_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(n, rec, idx, nu, nfe, pair_kind, x);
  return cudaGetLastError() == cudaSuccess ? 0 : ST_CUDA;
}

int td1c_lp_loss(int n, const double* rec, const int* idx, const float* out, float* dy, double* loss, int use_net, void* stream) {
  if (n < 0 || !rec || !loss || (use_net && !out)) return ST_CONFIG;
  if (n) lp_loss_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(n, rec, idx, out, dy, loss, use_net);
  return cudaGetLastError() == cudaSuccess ? 0 : ST_CUDA;
}

}  // extern "C"
