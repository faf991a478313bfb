// mlp.cu -- the learned mean-field predictor's network on the device: FP32
// training (forward, hand-written backward, Adam) and BF16 inference on the
// fifth-generation tensor cores.
//
// The network is a stack of linear layers with tanh between them,
//   h_0 = x, h_k = tanh(W_k h_{k-1} + b_k) (k < depth), y = W_depth h_{depth-1} + b_depth,
// weights W_k [n_k x n_{k-1}] row-major in FP32 (the master copy the optimiser
// updates).  Training runs in FP32 on the CUDA cores:
//   forward   H_k = act(H_{k-1} W_k^T + b_k)          (mlp_gemm, NT form)
//   backward  dW_k = G_k^T H_{k-1}, db_k = sum_rows G_k  (TN form, column sums)
//             G_{k-1} = (G_k W_k) * (1 - H_{k-1}^2)      (NN form, tanh derivative)
//   Adam      m = b1 m + (1 - b1) g, v = b2 v + (1 - b2) g^2,
//             p -= lr (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps)
// (Kingma and Ba, 2015), the same steps as the CPU reference network the tests
// compare against.  Sums over rows are in a fixed order, so gradients are
// deterministic.
//
// Inference (mlp_infer_bf16_kernel) runs all layers of a 128-row tile in one
// CTA: the layer's weights (BF16, split once per weight update) and the
// tile's activations (BF16) sit in shared memory in the canonical K-major
// layout; one thread issues tcgen05.mma kind::f16 (BF16 x BF16, FP32
// accumulation in tensor memory, M = 128, N = layer width, K = 16 per
// instruction); the epilogue warps read the accumulator rows with tcgen05.ld,
// add the bias, apply tanh and write the next layer's BF16 activations.
// Hidden widths are multiples of 16 up to 256; the input is zero-padded to a
// multiple of 16, the output to 16 columns.  Waits on the MMA's mbarrier are
// bounded (1 s) and report ST_TIMEOUT; the kernel then waits (bounded) for
// its committed MMAs before freeing the tensor memory.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace td1c {

// ---------------------------------------------------------------------------
// FP32 training kernels
// ---------------------------------------------------------------------------
// C[i][j] = alpha * sum_k A(i, k) B(k, j) (+ bias[j]) (tanh), A(i,k) = A[i sai + k sak],
// B(k,j) = B[k sbk + j sbj]; C row-major with pitch ldc.  64 x 64 tiles, 16 x 16
// threads with 4 x 4 outputs each, K in steps of 16 through shared memory.
constexpr int MG_T = 64, MG_K = 16;
__global__ void __launch_bounds__(256) mlp_gemm_kernel(int M, int N, int K, const float* __restrict__ A, long sai, long sak,
                                                       const float* __restrict__ B, long sbk, long sbj, float* __restrict__ C,
                                                       long ldc, const float* __restrict__ bias, int act, float alpha,
                                                       int accumulate) {
  __shared__ float As[MG_K][MG_T + 4];
  __shared__ float Bs[MG_K][MG_T + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i0 = blockIdx.y * MG_T, j0 = blockIdx.x * MG_T;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += MG_K) {
    for (int e = threadIdx.x; e < MG_T * MG_K; e += 256) {
      const int r = e / MG_K, kk = e % MG_K;  // A: row r of the tile, depth kk
      const int gi = i0 + r, gk = k0 + kk;
      As[kk][r] = (gi < M && gk < K) ? A[(long)gi * sai + (long)gk * sak] : 0.f;
      const int cc = e % MG_T, kb = e / MG_T;  // B: column cc, depth kb
      const int gj = j0 + cc, gk2 = k0 + kb;
      Bs[kb][cc] = (gj < N && gk2 < K) ? B[(long)gk2 * sbk + (long)gj * sbj] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < MG_K; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { a[u] = As[kk][ty + 16 * u]; b[u] = Bs[kk][tx + 16 * u]; }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int gi = i0 + ty + 16 * u;
    if (gi >= M) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int gj = j0 + tx + 16 * v;
      if (gj >= N) continue;
      float x = alpha * acc[u][v];
      if (accumulate) x += C[(long)gi * ldc + gj];
      if (bias) x += bias[gj];
      if (act == 1) x = tanhf(x);
      C[(long)gi * ldc + gj] = x;
    }
  }
}

// db[j] = sum_i G[i][j] over rows in a fixed order (one thread per column)
__global__ void mlp_colsum_kernel(int M, int N, const float* __restrict__ G, float* __restrict__ db) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  float s = 0.f;
  for (int i = 0; i < M; ++i) s += G[(long)i * N + j];
  db[j] = s;
}

// G[i][j] *= 1 - H[i][j]^2 (the tanh derivative in terms of the activation)
__global__ void mlp_dtanh_kernel(long n, float* __restrict__ G, const float* __restrict__ H) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float h = H[t];
  G[t] *= 1.f - h * h;
}

__global__ void mlp_adam_kernel(long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t];
  const float mt = b1 * m[t] + (1.f - b1) * gt;
  const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
}

static int mlp_gemm(int M, int N, int K, const float* A, long sai, long sak, const float* B, long sbk, long sbj, float* C,
                    long ldc, const float* bias, int act, float alpha, int accumulate, cudaStream_t st) {
  dim3 grid((N + MG_T - 1) / MG_T, (M + MG_T - 1) / MG_T);
  mlp_gemm_kernel<<<grid, 256, 0, st>>>(M, N, K, A, sai, sak, B, sbk, sbj, C, ldc, bias, act, alpha, accumulate);
  return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// BF16 inference on tcgen05
// ---------------------------------------------------------------------------
constexpr int MI_BM = 128, MI_MAXW = 256, MI_THREADS = 160;  // 4 epilogue warps + 1 MMA warp
__device__ __forceinline__ uint32_t mi_off(int r, int k, int kp) {  // bf16 K-major canonical: 8 rows x 8 elements
  return (uint32_t)((r >> 3) * (kp * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
__device__ __forceinline__ uint64_t mi_desc(uint32_t saddr, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}
__device__ __forceinline__ unsigned short mi_bf16(float x) {  // round to nearest even
  uint32_t u = __float_as_uint(x);
  if ((u & 0x7F800000u) == 0x7F800000u) return (unsigned short)(u >> 16);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (unsigned short)(u >> 16);
}

// weights of one layer as BF16 planes in the K-major canonical layout (np rows x kp depth)
__global__ void mlp_pack_bf16_kernel(const float* __restrict__ W, int n, int k, int np, int kp, unsigned short* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= np * kp) return;
  const int r = e / kp, c = e % kp;
  out[mi_off(r, c, kp) / 2] = (r < n && c < k) ? mi_bf16(W[(long)r * k + c]) : (unsigned short)0;
}

struct MiShared {
  unsigned long long done, drain;
  uint32_t tmem;
  int abort;
};

// One CTA per 128-row tile; every layer: weights -> shared memory, MMAs, epilogue
// into the next layer's activations.  y[rows x nout] FP32.
__global__ void __launch_bounds__(MI_THREADS, 1) mlp_infer_bf16_kernel(MlpInferArgs a) {
  extern __shared__ __align__(1024) unsigned char mi_smem[];
  // weights of one layer (MI_MAXW x MI_MAXW bf16, 128 KB) and the tile's activations (128 x MI_MAXW bf16,
  // 64 KB).  One activation buffer serves every layer: the epilogue of layer L
  // runs after that layer's MMAs have completed (their commit), so it may
  // overwrite the activations they read with the next layer's.
  unsigned char* s_w = mi_smem;
  unsigned char* s_x = mi_smem + MI_MAXW * MI_MAXW * 2;
  MiShared* sh = reinterpret_cast<MiShared*>(mi_smem + MI_MAXW * MI_MAXW * 2 + MI_BM * MI_MAXW * 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row0 = blockIdx.x * MI_BM;
  if (tid == 0) {
    mbar_init(&sh->done, 1);
    mbar_init(&sh->drain, 1);
    sh->abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&sh->tmem)), "r"(256u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // input tile -> activations 0 (bf16, K-major, depth kin padded)
  {
    const int kp = a.kp[0];
    for (int e = tid; e < MI_BM * kp; e += MI_THREADS) {
      const int r = e / kp, c = e % kp, gr = row0 + r;
      const float x = (gr < a.rows && c < a.nin) ? a.x[(long)gr * a.ldx + c] : 0.f;
      *reinterpret_cast<unsigned short*>(s_x + mi_off(r, c, kp)) = mi_bf16(x);
    }
  }
  fence_async_smem();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sh->tmem;
  bool issued = false;
  for (int L = 0; L < a.depth; ++L) {
    const int kp = a.kp[L], np = a.np[L];  // depth and (padded) width of this layer
    // weights of layer L
    {
      const uint4* src = reinterpret_cast<const uint4*>(a.wbf16[L]);
      uint4* dst = reinterpret_cast<uint4*>(s_w);
      for (int i = tid; i < np * kp * 2 / 16; i += MI_THREADS) dst[i] = __ldg(src + i);
    }
    fence_async_smem();
    __syncthreads();
    if (warp == 4 && lane == 0 && !*(volatile int*)&sh->abort) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // kind::f16: D F32 (bits 4-5 = 1), A BF16 (bits 7-9 = 1), B BF16 (bits 10-12 = 1), K-major, N, M = 128
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(np >> 3) << 17) | ((uint32_t)(MI_BM >> 4) << 24);
      const uint32_t xa = su32(s_x), wa = su32(s_w);
      const uint32_t sbo = (uint32_t)(kp * 16);
      for (int ks = 0; ks < kp / 16; ++ks) {
        const uint64_t da = mi_desc(xa + ks * 256, sbo), db = mi_desc(wa + ks * 256, sbo);
        const uint32_t acc = ks ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
      issued = true;
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(&sh->done))
                   : "memory");
    }
    if (warp < 4) {
      if (!*(volatile int*)&sh->abort && mbar_wait(&sh->done, (uint32_t)(L & 1))) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int r = 32 * warp + lane, gr = row0 + r;
        const bool last = L == a.depth - 1;
        const int kpn = last ? 0 : a.kp[L + 1];
        for (int cc = 0; cc < np; cc += 16) {
          uint32_t v[16];
          const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)cc;
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
              "[%16];"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
                "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
              : "r"(taddr));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int c = cc + j;
            const int nl = a.n[L];
            float y = __uint_as_float(v[j]) + (c < nl ? a.b[L][c] : 0.f);
            if (!last) {
              y = c < nl ? tanhf(y) : 0.f;
              if (c < kpn) *reinterpret_cast<unsigned short*>(s_x + mi_off(r, c, kpn)) = mi_bf16(y);
            } else if (gr < a.rows && c < nl) {
              a.y[(long)gr * a.ldy + c] = y;
            }
          }
        }
      } else if (lane == 0) {
        if (!sh->abort) atomicOr(a.status, ST_TIMEOUT);
        sh->abort = 1;
      }
    }
    fence_async_smem();  // the next layer's activations, written by the generic proxy, are MMA operands
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (warp == 4 && lane == 0 && issued) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(&sh->drain))
                 : "memory");
    if (!mbar_wait(&sh->drain, 0)) atomicOr(a.status, ST_TIMEOUT);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u));
  }
}

int mlp_infer_smem() { return MI_MAXW * MI_MAXW * 2 + MI_BM * MI_MAXW * 2 + (int)sizeof(MiShared) + 16; }

// The kernel's shared-memory opt-in, once per device; callers that capture the
// launch into a graph call this before the capture.
int mlp_infer_prepare() {
  static bool attr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ST_CUDA;
  if (dev >= 0 && dev < 64 && attr[dev]) return 0;
  if (cudaFuncSetAttribute(mlp_infer_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp_infer_smem()) !=
      cudaSuccess)
    return ST_CUDA;
  if (dev >= 0 && dev < 64) attr[dev] = true;
  return 0;
}

int launch_mlp_infer_bf16(const MlpInferArgs& a, cudaStream_t st) {
  if (mlp_infer_prepare()) return (int)cudaErrorInvalidValue;
  const int ntile = (a.rows + MI_BM - 1) / MI_BM;
  if (ntile > 0) mlp_infer_bf16_kernel<<<ntile, MI_THREADS, mlp_infer_smem(), st>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace td1c

using namespace td1c;

// ---------------------------------------------------------------------------
// C-ABI of the network kernels (device pointers, library-independent of any
// bound context; asynchronous on the given stream)
// ---------------------------------------------------------------------------
extern "C" {

// sizes[0..depth]: layer widths n_0 (input) .. n_depth (output).  W[k], b[k]
// (k < depth) device pointers to layer k+1's weights [n_{k+1} x n_k] and bias.
// acts: device buffer of sum_{k=1..depth} rows * n_k floats (the activations,
// kept for the backward pass); y points into it (the last layer).
int td1c_mlp_forward(int depth, const int* sizes, const float* const* W, const float* const* b, const float* x, int rows,
                     float* acts, void* stream) {
  if (depth < 1 || depth > MLP_MAXDEPTH || rows < 0 || !sizes || !W || !b || !x || !acts) return ST_CONFIG;
  cudaStream_t st = (cudaStream_t)stream;
  const float* in = x;
  float* out = acts;
  for (int k = 0; k < depth; ++k) {
    const int nin = sizes[k], nout = sizes[k + 1];
    if (mlp_gemm(rows, nout, nin, in, nin, 1, W[k], 1, nin, out, nout, b[k], k < depth - 1 ? 1 : 0, 1.f, 0, st))
      return ST_CUDA;
    in = out;
    out += (long)rows * nout;
  }
  return 0;
}

// Backward pass of td1c_mlp_forward's network for an output gradient dy
// [rows x n_depth] (dL/dy, already divided by whatever the loss averages over):
// dW[k], db[k] (device, same shapes as W, b) are overwritten.  work: device
// scratch of 2 * rows * max_k n_k floats.
int td1c_mlp_backward(int depth, const int* sizes, const float* const* W, const float* x, int rows, const float* acts,
                      const float* dy, float* const* dW, float* const* db, float* work, void* stream) {
  if (depth < 1 || depth > MLP_MAXDEPTH || rows < 1 || !sizes || !W || !x || !acts || !dy || !dW || !db || !work)
    return ST_CONFIG;
  cudaStream_t st = (cudaStream_t)stream;
  int wmax = 0;
  for (int k = 0; k <= depth; ++k) wmax = std::max(wmax, sizes[k]);
  const float* actk[MLP_MAXDEPTH + 1];
  actk[0] = x;
  {
    const float* p = acts;
    for (int k = 1; k <= depth; ++k) { actk[k] = p; p += (long)rows * sizes[k]; }
  }
  float* g = work;
  float* gprev = work + (long)rows * wmax;
  cudaMemcpyAsync(g, dy, (size_t)rows * sizes[depth] * sizeof(float), cudaMemcpyDeviceToDevice, st);
  for (int k = depth - 1; k >= 0; --k) {
    const int nin = sizes[k], nout = sizes[k + 1];
    // dW[k] [nout x nin] = G^T [nout x rows] * H_k [rows x nin]
    if (mlp_gemm(nout, nin, rows, g, 1, nout, actk[k], nin, 1, dW[k], nin, nullptr, 0, 1.f, 0, st)) return ST_CUDA;
    mlp_colsum_kernel<<<(nout + 127) / 128, 128, 0, st>>>(rows, nout, g, db[k]);
    if (k > 0) {
      // G_prev [rows x nin] = G [rows x nout] * W [nout x nin], times the tanh derivative of H_k
      if (mlp_gemm(rows, nin, nout, g, nout, 1, W[k], nin, 1, gprev, nin, nullptr, 0, 1.f, 0, st)) return ST_CUDA;
      const long n = (long)rows * nin;
      mlp_dtanh_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, gprev, actk[k]);
      std::swap(g, gprev);
    }
  }
  return (int)cudaGetLastError() ? ST_CUDA : 0;
}

// One Adam step on n parameters p with gradient g and moments m, v (device);
// step is the 1-based step count of the bias corrections.
int td1c_mlp_adam(long n, float* p, const float* g, float* m, float* v, float lr, float beta1, float beta2, float eps, int step,
                  void* stream) {
  if (n < 0 || step < 1) return ST_CONFIG;
  const float c1 = 1.f - std::pow(beta1, (float)step), c2 = 1.f - std::pow(beta2, (float)step);
  if (n) mlp_adam_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(n, p, g, m, v, lr, beta1, beta2, eps, c1, c2);
  return (int)cudaGetLastError() ? ST_CUDA : 0;
}

// BF16 inference on the tensor cores.  pack: device buffer receiving the
// BF16 weight planes (td1c_mlp_pack_size(depth, sizes) bytes), rebuilt from
// the FP32 weights by this call when repack != 0.  y [rows x n_depth] FP32.
long td1c_mlp_pack_size(int depth, const int* sizes) {
  long tot = 0;
  for (int k = 0; k < depth; ++k) {
    const long np = (sizes[k + 1] + 15) / 16 * 16, kp = (sizes[k] + 15) / 16 * 16;
    tot += np * kp * 2;
  }
  return tot;
}

int td1c_mlp_infer_bf16(int depth, const int* sizes, const float* const* W, const float* const* b, void* pack, int repack,
                        const float* x, int rows, float* y, int* status, void* stream) {
  if (depth < 1 || depth > MLP_MAXDEPTH || rows < 0 || !sizes || !W || !b || !pack || !x || !y || !status) return ST_CONFIG;
  for (int k = 0; k <= depth; ++k)
    if (sizes[k] < 1 || sizes[k] > MI_MAXW) return ST_CONFIG;
  cudaStream_t st = (cudaStream_t)stream;
  MlpInferArgs a{};
  a.depth = depth; a.rows = rows; a.nin = sizes[0]; a.x = x; a.ldx = sizes[0]; a.y = y; a.ldy = sizes[depth]; a.status = status;
  unsigned short* p = (unsigned short*)pack;
  for (int k = 0; k < depth; ++k) {
    const int np = (sizes[k + 1] + 15) / 16 * 16, kp = (sizes[k] + 15) / 16 * 16;
    a.n[k] = sizes[k + 1]; a.np[k] = np; a.kp[k] = kp; a.b[k] = b[k]; a.wbf16[k] = p;
    if (repack) mlp_pack_bf16_kernel<<<(np * kp + 255) / 256, 256, 0, st>>>(W[k], sizes[k + 1], sizes[k], np, kp, p);
    p += (long)np * kp;
  }
  return launch_mlp_infer_bf16(a, st) ? ST_CUDA : 0;
}

}  // extern "C"
