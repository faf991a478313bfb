// legendre_tc.cu -- the mean field's theta <-> l transforms in split TF32 on
// the fifth-generation tensor cores, as a warp-specialised persistent kernel.
//
// Contract (legendre_gemm.cu): C[b](M x N) = T[b](M x K) * B[b](K x N), T a
// real Legendre table, B a complex slab of K rows x N reals (pair mode: B =
// conj(B0) * B1, the pair density, formed in the loader).  These are the
// pair-density multipoles (ang2sph2, bas_ang2sph2.F90:330-482) and the pair
// potentials on the grid (sph2ang2, bas_sph2ang2.F90:334-463) of the
// mixed-precision RHS.  Every FP64 operand x is split into x_hi = tf32(x) and
// x_lo = tf32(x - x_hi), and T B = T_hi B_hi + T_hi B_lo + T_lo B_hi (lo * lo
// dropped): three tcgen05.mma kind::tf32 per depth step accumulating FP32 in
// tensor memory, about 2^-21 relative per product.  C is written in FP64.
//
// The MMA computes the transposed tile D(128 x Np) = S^T T^T: A = 128 slab
// columns x K (K-major), B = the Np table rows x K (K-major), so the table is
// the N operand and one MMA covers all M <= Np <= 128 output rows.
//
// One persistent CTA per SM works through a contiguous range of tiles (128
// slab columns of one batch) whose batches share one table, so the table's
// hi/lo planes -- split once at set-up into the tensor-core layout -- are
// copied into shared memory once per CTA and stay resident.  A tile's depth
// runs in chunks of 16.  Roles:
//   warps 0-3   epilogue: tcgen05.ld of accumulator rows (warp w reads TMEM
//               lanes 32w..32w+31 = slab columns), FP64 stores of C;
//   warps 4-11  converters: read a raw chunk (FP64 rows as they lie in
//               global memory), form the pair product, split hi/lo and store
//               the chunk's tensor-core stage (canonical K-major layout, no
//               swizzle; one thread per stage row, so stores are conflict-free);
//   warp 12     one thread issues the TMA tensor loads (3-d boxes of 128
//               doubles x 16 rows of one slab; rows past K and columns past N
//               read as zero) into a ring of raw slots, several chunks ahead;
//   warp 13     one thread issues the MMAs of a chunk and commits them to the
//               stage's "empty" mbarrier, and each finished tile to the
//               accumulator's "full" mbarrier.
// Two accumulators (TMEM columns 0 and 128) let the epilogue of tile i overlap
// the MMAs of tile i + 1.  The tensor maps cover this GPU's own buffers only
// and no load uses cluster multicast.
//
// Every wait is bounded (mbar_wait, 1 s).  A wait that runs out sets
// ST_TIMEOUT, raises the CTA's abort flag, and every role leaves its loop.
// Before the CTA ends, the TMA thread waits (bounded) for the last load it
// issued into every raw slot, and before the tensor memory is freed the MMA
// thread commits to a drain barrier and waits (bounded) for it, so no copy
// or committed MMA can still be writing when the CTA's resources go; the
// epilogue has waited for its own tcgen05.ld.
#include <algorithm>
#include <map>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"
#include "tma.cuh"

namespace td1c {

constexpr int TC_BM = 128;                   // slab columns per tile (MMA M)
constexpr int TC_BK = 16;                    // depth of one chunk
constexpr int TC_PLANE = TC_BM * TC_BK * 4;  // bytes of one staged hi or lo plane (8 KB)
constexpr int TC_STAGE = 2 * TC_PLANE;       // hi + lo
constexpr int TC_RAWOP = TC_BM * TC_BK * 8;  // one operand's raw box: 16 rows x 128 doubles (16 KB)
constexpr int TC_THREADS = 448;              // 4 epilogue + 8 converter warps + TMA warp + MMA warp
constexpr int TC_NCONV = 256;
constexpr int TC_SMEM_MAX = 227 * 1024;
constexpr int TC_MAXSLOT = 8;

// the table's hi/lo planes in the layout above (np rows x kp depths each, zero padded)
__global__ void tc_presplit_kernel(const double* __restrict__ T, int mt, int k, int lda, int np, int kp,
                                   uint32_t* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= np * kp) return;
  const int r = e / kp, c = e % kp;
  const double x = (r < mt && c < k) ? T[(size_t)r * lda + c] : 0.0;
  uint32_t hi, lo;
  tc_split(x, hi, lo);
  const uint32_t o = tc_off(r, c, kp) / 4;
  out[o] = hi;
  out[(size_t)np * kp + o] = lo;
}

constexpr int TC_MAXB = 16;  // batch descriptors of a CTA's tile range cached in shared memory

struct TcShared {
  unsigned long long raw_full[TC_MAXSLOT], raw_empty[TC_MAXSLOT], st_full[TC_MAXSLOT], st_empty[TC_MAXSLOT];
  unsigned long long acc_full[2], acc_empty[2], drain;
  LegGemmBatch batch[TC_MAXB];  // slots first_slot .. first_slot + TC_MAXB - 1 of the group order
  int2 z[TC_MAXB];              // their tensor-map slab indices (B0, B1)
  uint32_t tmem;
  int abort;
};

__device__ __forceinline__ bool tc_aborted(const TcShared* sh) { return *(volatile const int*)&sh->abort != 0; }
__device__ __forceinline__ void tc_fail(TcShared* sh, int* status) {
  atomicOr(status, ST_TIMEOUT);
  *(volatile int*)&sh->abort = 1;
}

template <bool PAIR>
__global__ void __launch_bounds__(TC_THREADS, 1) legendre_tc_kernel(const __grid_constant__ CUtensorMap tmap, LegTcArgs a) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  constexpr int nops = PAIR ? 2 : 1;
  const int np = a.np, kp = a.kp, S = a.stages, RR = a.raw_slots;
  const int table_bytes = 2 * np * kp * 4;
  unsigned char* s_table = tc_smem;                                   // [hi | lo] table planes
  unsigned char* s_raw = tc_smem + ((table_bytes + 1023) & ~1023);   // RR raw slots of nops boxes
  unsigned char* s_ring = s_raw + RR * nops * TC_RAWOP;               // S stages of [hi | lo] slab chunks
  TcShared* sh = reinterpret_cast<TcShared*>(s_ring + S * TC_STAGE);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int4 work = a.work[blockIdx.x];  // (table, first tile, end tile, -)
  const int t_begin = work.y, t_end = work.z;
  const int nchunk = kp / TC_BK;
  const int total = (t_end - t_begin) * nchunk;  // chunks of this CTA, in order
  const int ntn = a.ntn, first_slot = t_begin / ntn;

  for (int i = tid; i < TC_MAXB; i += TC_THREADS)
    if (first_slot + i <= (t_end - 1) / ntn) {
      const int b = a.order[first_slot + i];
      sh->batch[i] = a.batches[b];
      sh->z[i] = a.zc[b];
    }
  if (tid == 0) {
    for (int r = 0; r < RR; ++r) { mbar_init(&sh->raw_full[r], 1); mbar_init(&sh->raw_empty[r], TC_NCONV); }
    for (int s = 0; s < S; ++s) { mbar_init(&sh->st_full[s], TC_NCONV); mbar_init(&sh->st_empty[s], 1); }
    for (int q = 0; q < 2; ++q) { mbar_init(&sh->acc_full[q], 1); mbar_init(&sh->acc_empty[q], 128); }
    mbar_init(&sh->drain, 1);
    sh->abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&sh->tmem)),
                 "r"((uint32_t)a.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // the table planes: one copy per CTA, read by the tensor cores for every tile
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.tables + (size_t)work.x * 2 * np * kp);
    uint4* dst = reinterpret_cast<uint4*>(s_table);
    for (int i = tid; i < table_bytes / 16; i += TC_THREADS) dst[i] = __ldg(src + i);
  }
  fence_async_smem();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sh->tmem;
  // the batch of tile t (from shared memory when the range is cached)
  auto slot_of = [&](int t) { return t / ntn - first_slot; };

  if (warp == 12) {
    // ---- TMA producer: chunk j of the CTA -> raw slot j % RR
    if (lane == 0) {
      int last[TC_MAXSLOT];
      for (int r = 0; r < TC_MAXSLOT; ++r) last[r] = -1;
      for (int j = 0; j < total; ++j) {
        const int r = j % RR;
        if (tc_aborted(sh) || !mbar_wait(&sh->raw_empty[r], ((j / RR) & 1) ^ 1)) {
          if (!tc_aborted(sh)) tc_fail(sh, a.status);
          break;
        }
        const int t = t_begin + j / nchunk, c = j % nchunk, sl = slot_of(t);
        const int2 z = sl < TC_MAXB ? sh->z[sl] : a.zc[a.order[t / ntn]];
        unsigned char* dst = s_raw + r * nops * TC_RAWOP;
        mbar_expect_tx(&sh->raw_full[r], nops * TC_RAWOP);
        tensor_load_3d(dst, &tmap, (t % ntn) * TC_BM, c * TC_BK, z.x, &sh->raw_full[r]);
        if (PAIR) tensor_load_3d(dst + TC_RAWOP, &tmap, (t % ntn) * TC_BM, c * TC_BK, z.y, &sh->raw_full[r]);
        last[r] = j;
      }
      // no load may land after the CTA is gone: wait for the last one issued into every slot
      for (int r = 0; r < RR; ++r)
        if (last[r] >= 0 && !mbar_wait(&sh->raw_full[r], (last[r] / RR) & 1)) atomicOr(a.status, ST_TIMEOUT);
    }
  } else if (warp >= 4 && warp < 12) {
    // ---- converters: thread = one stage row (slab column n0 + row) and 8 of the chunk's 16 depths
    const int p = tid - 128, row = p & 127, k0 = (p >> 7) * 8;
    const int col = row >> 1, comp = row & 1;  // complex column and its real / imaginary part
    for (int j = 0; j < total; ++j) {
      const int r = j % RR, s = j % S;
      bool ok = !tc_aborted(sh) && mbar_wait(&sh->raw_full[r], (j / RR) & 1);
      ok = ok && !tc_aborted(sh) && mbar_wait(&sh->st_empty[s], ((j / S) & 1) ^ 1);
      if (!ok) {
        if (!tc_aborted(sh)) tc_fail(sh, a.status);
        break;
      }
      const unsigned char* raw = s_raw + r * nops * TC_RAWOP;
      const uint32_t base = su32(s_ring + s * TC_STAGE);
#pragma unroll
      for (int g = 0; g < 2; ++g) {
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int k = k0 + 4 * g + u;
          cplx z = *reinterpret_cast<const cplx*>(raw + k * (TC_BM * 8) + col * 16);
          if (PAIR) z = cmulc(z, *reinterpret_cast<const cplx*>(raw + TC_RAWOP + k * (TC_BM * 8) + col * 16));
          tc_split(comp ? z.y : z.x, hi[u], lo[u]);
        }
        const uint32_t o = tc_off(row, k0 + 4 * g, TC_BK);
        asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(base + o), "r"(hi[0]), "r"(hi[1]), "r"(hi[2]), "r"(hi[3]));
        asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(base + TC_PLANE + o), "r"(lo[0]), "r"(lo[1]), "r"(lo[2]),
                     "r"(lo[3]));
      }
      mbar_arrive(&sh->raw_empty[r]);  // this thread's reads of the raw slot are done
      fence_async_smem();              // generic-proxy stores -> tensor-core reads
      mbar_arrive(&sh->st_full[s]);
    }
  } else if (warp == 13) {
    // ---- MMA issue (one thread)
    if (lane == 0) {
      const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(np >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
      const uint32_t t_hi = su32(s_table), t_lo = t_hi + (uint32_t)(np * kp * 4);
      const uint32_t sbo_t = (uint32_t)(kp * 32), sbo_s = (uint32_t)(TC_BK * 32);
      int j = 0;
      bool issued = false;
      for (int i = 0, t = t_begin; t < t_end; ++t, ++i) {
        const int acc = i & 1;
        if (tc_aborted(sh) || !mbar_wait(&sh->acc_empty[acc], ((i >> 1) & 1) ^ 1)) {
          if (!tc_aborted(sh)) tc_fail(sh, a.status);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(acc * 128);  // accumulators 128 columns apart
        bool ok = true;
        for (int c = 0; c < nchunk; ++c, ++j) {
          const int s = j % S;
          if (tc_aborted(sh) || !mbar_wait(&sh->st_full[s], (j / S) & 1)) { ok = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t sh_hi = su32(s_ring + s * TC_STAGE), sh_lo = sh_hi + TC_PLANE;
#pragma unroll
          for (int ks = 0; ks < TC_BK / 8; ++ks) {
            const uint32_t ko = (uint32_t)((c * (TC_BK / 8) + ks) * 256);
            const uint64_t bh = tc_desc(t_hi + ko, sbo_t), bl = tc_desc(t_lo + ko, sbo_t);
            const uint64_t ah = tc_desc(sh_hi + ks * 256, sbo_s), al = tc_desc(sh_lo + ks * 256, sbo_s);
            tc_mma(d, ah, bh, idesc, (c | ks) != 0);
            tc_mma(d, ah, bl, idesc, 1u);
            tc_mma(d, al, bh, idesc, 1u);
          }
          issued = true;
          tc_commit(&sh->st_empty[s]);  // the stage is free once these MMAs have read it
        }
        if (!ok) {
          if (!tc_aborted(sh)) tc_fail(sh, a.status);
          break;
        }
        tc_commit(&sh->acc_full[acc]);
      }
      // nothing may still write tensor memory when it is freed: wait for every
      // MMA this thread committed (tcgen05.commit tracks all of them)
      if (issued) {
        tc_commit(&sh->drain);
        if (!mbar_wait(&sh->drain, 0)) atomicOr(a.status, ST_TIMEOUT);
      }
    }
  } else {
    // ---- epilogue (warps 0-3): TMEM lanes 32 w .. 32 w + 31 are slab columns n0 + row
    for (int i = 0, t = t_begin; t < t_end; ++t, ++i) {
      const int acc = i & 1;
      if (tc_aborted(sh)) break;
      if (!mbar_wait(&sh->acc_full[acc], (i >> 1) & 1)) {
        if (lane == 0 && !tc_aborted(sh)) tc_fail(sh, a.status);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int sl = slot_of(t);
      double* C = sl < TC_MAXB ? sh->batch[sl].C : a.batches[a.order[t / ntn]].C;
      const int ldc = sl < TC_MAXB ? sh->batch[sl].ldc : a.batches[a.order[t / ntn]].ldc;
      const int gn = (t % ntn) * TC_BM + 32 * warp + lane;
      const bool col_ok = gn < a.N;
      for (int cc = 0; cc < np; cc += 16) {
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(acc * 128 + cc);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
            "[%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
              "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (col_ok) {
#pragma unroll
          for (int q = 0; q < 16; ++q)
            if (cc + q < a.M) C[(size_t)(cc + q) * ldc + gn] = (double)__uint_as_float(r[q]);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(&sh->acc_empty[acc]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)a.tmem_cols));
  }
}

int legendre_tc_smem(int np, int kp, int raw_slots, int stages, int nops) {
  const int table_bytes = 2 * np * kp * 4;
  return ((table_bytes + 1023) & ~1023) + raw_slots * nops * TC_RAWOP + stages * TC_STAGE + (int)sizeof(TcShared) + 16;
}

// Builds the persistent plan of one batch list: split tables, tile order
// grouped by table, each CTA's tile range, and the tensor map of the slab
// array (slab_count slabs of K rows x N doubles from slab_base, in the
// batches' pitch; each batch's B0 / B1 is one of them).  Returns 0, or a
// non-zero status when the shapes are outside the kernel's range (the caller
// then keeps the per-tile split-TF32 kernel).
int legendre_tc_plan(const std::vector<LegGemmBatch>& h_batches, const LegGemmBatch* d_batches, int M, int K, int N, bool pair,
                     const double* slab_base, int slab_count, int nsm, LegTcPlan* out, std::vector<void*>& allocs,
                     cudaStream_t st) {
  const int np = (M + 15) / 16 * 16, kp = (K + TC_BK - 1) / TC_BK * TC_BK;
  const int nops = pair ? 2 : 1;
  if (h_batches.empty() || np > 128 || N % 2 || !slab_base || slab_count < 1) return ST_CONFIG;
  const int ldb = h_batches[0].ldb;
  for (const auto& b : h_batches)
    if (b.ldb != ldb || (ldb * 8) % 16) return ST_CONFIG;
  // stage ring and raw ring in the shared memory the table leaves
  int stages = 4, raw = 0;
  for (; stages >= 2; --stages) {
    const int avail = TC_SMEM_MAX - legendre_tc_smem(np, kp, 0, stages, nops);
    raw = std::min(TC_MAXSLOT, avail / (nops * TC_RAWOP));
    if (raw >= 3 || (stages == 2 && raw >= 2)) break;
  }
  if (stages < 2 || raw < 2) return ST_CONFIG;
  // slab index of every batch operand in the tensor map
  const size_t slab = (size_t)K * ldb;  // doubles per slab
  std::vector<int2> zc;
  for (const auto& b : h_batches) {
    const ptrdiff_t d0 = b.B0 - slab_base, d1 = pair ? b.B1 - slab_base : 0;
    if (d0 < 0 || d1 < 0 || d0 % (ptrdiff_t)slab || d1 % (ptrdiff_t)slab || d0 / (ptrdiff_t)slab >= slab_count ||
        d1 / (ptrdiff_t)slab >= slab_count)
      return ST_CONFIG;
    zc.push_back(make_int2((int)(d0 / (ptrdiff_t)slab), (int)(d1 / (ptrdiff_t)slab)));
  }
  {
    const cuuint64_t dims[3] = {(cuuint64_t)N, (cuuint64_t)K, (cuuint64_t)slab_count};
    const cuuint64_t strides[2] = {(cuuint64_t)ldb * 8, (cuuint64_t)slab * 8};
    const cuuint32_t box[3] = {(cuuint32_t)TC_BM, (cuuint32_t)TC_BK, 1u};
    if (encode_f64_map(&out->tmap, slab_base, 3, dims, strides, box, pair ? "pair-density slabs" : "pair-potential slabs"))
      return ST_CONFIG;
  }
  // distinct tables
  std::map<const double*, int> tix;
  std::vector<const double*> tabs;
  std::vector<int> lda;
  for (const auto& b : h_batches)
    if (!tix.count(b.A)) { tix[b.A] = (int)tabs.size(); tabs.push_back(b.A); lda.push_back(b.lda); }
  const int nt = (int)tabs.size();
  uint32_t* d_tab = nullptr;
  if (cudaMalloc(&d_tab, (size_t)nt * 2 * np * kp * 4) != cudaSuccess) return ST_CUDA;
  allocs.push_back(d_tab);
  for (int i = 0; i < nt; ++i) {
    const int n = np * kp;
    tc_presplit_kernel<<<(n + 255) / 256, 256, 0, st>>>(tabs[i], M, K, lda[i], np, kp, d_tab + (size_t)i * 2 * n);
  }
  // tiles grouped by table; CTAs per group in proportion to its tiles
  const int ntn = (N + TC_BM - 1) / TC_BM;
  std::vector<int> order;
  std::vector<int> g_first(nt), g_count(nt, 0);
  for (int g = 0; g < nt; ++g) {
    g_first[g] = (int)order.size();
    for (int b = 0; b < (int)h_batches.size(); ++b)
      if (tix[h_batches[b].A] == g) { order.push_back(b); ++g_count[g]; }
  }
  const long total = (long)order.size() * ntn;
  std::vector<int4> work;
  for (int g = 0; g < nt; ++g) {
    const long tg = (long)g_count[g] * ntn;
    const int nc = (int)std::max<long>(1, std::min<long>(tg, (long)((double)nsm * tg / total + 0.5)));
    const long t0 = (long)g_first[g] * ntn;
    for (int c = 0; c < nc; ++c)
      work.push_back(make_int4(g, (int)(t0 + tg * c / nc), (int)(t0 + tg * (c + 1) / nc), 0));
  }
  int* d_order = nullptr;
  int4* d_work = nullptr;
  int2* d_zc = nullptr;
  if (cudaMalloc(&d_order, order.size() * sizeof(int)) != cudaSuccess) return ST_CUDA;
  allocs.push_back(d_order);
  if (cudaMalloc(&d_work, work.size() * sizeof(int4)) != cudaSuccess) return ST_CUDA;
  allocs.push_back(d_work);
  if (cudaMalloc(&d_zc, zc.size() * sizeof(int2)) != cudaSuccess) return ST_CUDA;
  allocs.push_back(d_zc);
  cudaMemcpyAsync(d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_work, work.data(), work.size() * sizeof(int4), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_zc, zc.data(), zc.size() * sizeof(int2), cudaMemcpyHostToDevice, st);
  cudaStreamSynchronize(st);
  LegTcArgs& a = out->args;
  a.batches = d_batches; a.order = d_order; a.work = d_work; a.tables = d_tab; a.zc = d_zc;
  a.M = M; a.K = K; a.N = N; a.np = np; a.kp = kp; a.ntn = ntn; a.stages = stages; a.raw_slots = raw;
  a.tmem_cols = 256;  // two accumulators of np <= 128 columns, 128 apart
  out->ncta = (int)work.size();
  out->pair = pair;
  out->smem = legendre_tc_smem(np, kp, raw, stages, nops);
  return (int)cudaGetLastError() == 0 ? 0 : ST_CUDA;
}

int launch_legendre_tc(const LegTcPlan& p, int* status, cudaStream_t st) {
  static bool attr[2] = {false, false};
  LegTcArgs a = p.args;
  a.status = status;
  if (p.pair) {
    if (!attr[1]) { cudaFuncSetAttribute(legendre_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_MAX); attr[1] = true; }
    legendre_tc_kernel<true><<<p.ncta, TC_THREADS, p.smem, st>>>(p.tmap, a);
  } else {
    if (!attr[0]) { cudaFuncSetAttribute(legendre_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_MAX); attr[0] = true; }
    legendre_tc_kernel<false><<<p.ncta, TC_THREADS, p.smem, st>>>(p.tmap, a);
  }
  return (int)cudaGetLastError();
}

}  // namespace td1c
