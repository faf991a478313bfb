// int2e_static.cu -- MO two-electron integrals without any device allocation.
//
// Some callers cannot call cudaMalloc: a host that hands the GPU's memory to
// its own pool allocator and forbids other allocations, a real-time loop that
// must not pay or risk an allocation (cudaMalloc synchronises the device and
// can fail under fragmentation), or an embedding framework that only lends
// its own buffers.  td1c_gpu_int2e_static serves them: the caller passes the
// active-pair densities, the pair potentials and the output buffer, and every
// piece of scratch the computation needs -- the int2e block tables and the
// split-K partial sums of the block GEMM -- lives in one file-scope device
// array of fixed size, I2S_SCRATCH_BYTES (8 MiB).  Each GPU that loads this
// library holds that array until the process exits.
//
// The arithmetic is the library's int2e path (int2e_block_kernel,
// int2e_sum_kernel, int2e_fill_kernel of reductions.cu; hprod_mkint2_sph.F90:
// 2-100): int2e(i,j,k,l) = sum_x rho2_ij[x] v2sph_kl[x] over x in [0, K) for
// i >= j and m_i + m_k = m_j + m_l, the i < j half by conjugate symmetry, and
// zero where the m rule fails.  Only where the scratch comes from differs.
//
// Sharing rules: every call on a device uses the same array, which keeps the
// last call's tables and partial sums.  Calls whose GPU work overlaps in time
// (on different streams, or from different host threads without ordering)
// race on the array and give wrong results; order them on one stream.
// Nothing in the array has to start at zero: each call writes every table
// entry and every partial sum before reading it, and the output is cleared
// by the call itself.
#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"
#include "reductions.cuh"

namespace td1c {

namespace {

constexpr size_t I2S_SCRATCH_BYTES = size_t(8) << 20;  // 8 MiB per device
constexpr int I2S_MAXACT = 16;                          // active orbitals
constexpr int I2S_MAXROW = I2S_MAXACT * (I2S_MAXACT + 1) / 2;  // pairs i >= j
constexpr int I2S_MAXCOL = I2S_MAXACT * I2S_MAXACT;            // ordered pairs kl
constexpr int I2S_MAXBLK = 96;                          // GEMM blocks (checked on every call)
constexpr int I2S_MAXENT = I2S_MAXROW * I2S_MAXCOL;     // block entries
constexpr int I2S_NSPLIT = 128;                         // K split of the library's own int2e
constexpr int I2S_ROWCHUNK = 24, I2S_COLCHUNK = 36;     // int2e_block_kernel CTA tile

// scratch layout (byte offsets, each 256-aligned)
constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t OFF_BLK = 0;
constexpr size_t OFF_ROW = OFF_BLK + align256(sizeof(Int2eBlock) * I2S_MAXBLK);
constexpr size_t OFF_COL = OFF_ROW + align256(sizeof(int) * I2S_MAXROW);
constexpr size_t OFF_DST = OFF_COL + align256(sizeof(int2) * I2S_MAXCOL);
constexpr size_t OFF_PART = OFF_DST + align256(sizeof(int4) * I2S_MAXENT);
static_assert(OFF_PART + sizeof(cplx) * I2S_MAXENT <= I2S_SCRATCH_BYTES,
              "scratch must hold at least one partial sum per block entry");

// In host code this name is only a handle for cudaGetSymbolAddress; kernels
// are given the device address that call returns.
static __device__ __align__(256) unsigned char g_int2e_scratch[I2S_SCRATCH_BYTES];

// One GEMM block: rows row0 .. row0+nrow-1 of the row list, columns col0 ..
// col0+ncol-1 of the column list, entries from ent0 on (row-major).
struct I2sBlk {
  unsigned short row0, col0;
  unsigned char nrow, ncol;
  unsigned short pad;
  int ent0;
};

// The whole block plan, passed by value (about 2 KB of kernel parameters).
struct I2sPlan {
  int nact, nblocks, nrow, ncol, nblkent;
  I2sBlk blk[I2S_MAXBLK];
  unsigned char row_ij[I2S_MAXROW][2];  // (i, j), i >= j, m_i - m_j = delta of the block
  unsigned char col_kl[I2S_MAXCOL][2];  // (k, l), m_l - m_k = delta
};

// Index of the pair (a, b), a >= b, in the packed lower triangle stored by
// columns: (0,0) (1,0) .. (n-1,0) (1,1) (2,1) ..
__device__ __forceinline__ int packed_pair(int a, int b, int n) { return b * n - b * (b - 1) / 2 + (a - b); }

// Expands the plan into the tables int2e_block_kernel reads.
__global__ void i2s_expand_kernel(I2sPlan p, Int2eBlock* __restrict__ blocks, int* __restrict__ row_pair,
                                  int2* __restrict__ col_pair, int4* __restrict__ ent_dst) {
  const int n = p.nact;
  const int span = max(max(p.nblocks, p.nrow), max(p.ncol, p.nblkent));
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < span; t += gridDim.x * blockDim.x) {
    if (t < p.nblocks) {
      Int2eBlock b{};
      b.row0 = p.blk[t].row0; b.nrow = p.blk[t].nrow; b.col0 = p.blk[t].col0; b.ncol = p.blk[t].ncol;
      b.ent0 = p.blk[t].ent0;
      blocks[t] = b;
    }
    if (t < p.nrow) row_pair[t] = packed_pair(p.row_ij[t][0], p.row_ij[t][1], n);
    if (t < p.ncol) {
      // v2sph_kl is the stored pair (k, l) when k > l, else the conjugate of
      // the stored (l, k) -- the same choice as the library's own tables
      const int k = p.col_kl[t][0], l = p.col_kl[t][1];
      col_pair[t] = k > l ? make_int2(packed_pair(k, l, n), 0) : make_int2(packed_pair(l, k, n), 1);
    }
    if (t < p.nblkent) {
      int b = 0;
      while (b + 1 < p.nblocks && p.blk[b + 1].ent0 <= t) ++b;
      const int e = t - p.blk[b].ent0, nc = p.blk[b].ncol;
      const int r = p.blk[b].row0 + e / nc, c = p.blk[b].col0 + e % nc;
      ent_dst[t] = make_int4(p.row_ij[r][0], p.row_ij[r][1], p.col_kl[c][0], p.col_kl[c][1]);
    }
  }
}

std::mutex g_scratch_mu;
void* g_scratch_ptr[64] = {};

// Device address of this device's scratch array, looked up on the first call
// with the device current.  Returns nullptr (and prints why) on failure.
void* scratch_for_current_device() {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    fprintf(stderr, "td1c_gpu_int2e_static: no usable current device (%s)\n", cudaGetErrorString(e));
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_int2e_scratch);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "td1c_gpu_int2e_static: cudaGetSymbolAddress on device %d failed: %s\n", dev,
              cudaGetErrorString(e));
      return nullptr;
    }
    g_scratch_ptr[dev] = p;
  }
  return g_scratch_ptr[dev];
}

}  // namespace

}  // namespace td1c

extern "C" {

int td1c_gpu_int2e_static(int nact, const int* mval, long K, const double* d_rho2, const double* d_v2sph,
                          double* d_int2e, void* stream) {
  using namespace td1c;
  if (nact < 1 || nact > I2S_MAXACT) {
    fprintf(stderr, "td1c_gpu_int2e_static: nact = %d is outside 1..%d (the size of the static scratch)\n", nact,
            I2S_MAXACT);
    return ST_CONFIG;
  }
  if (!mval || K < 1 || !d_rho2 || !d_v2sph || !d_int2e) {
    fprintf(stderr, "td1c_gpu_int2e_static: null pointer or K = %ld < 1\n", K);
    return ST_CONFIG;
  }
  // block plan on the stack: delta = m_i - m_j blocks, rows (i outer, j <= i
  // inner), columns (k outer, l inner), chunked to the kernel's CTA tile as in
  // the library's own int2e tables; chunks of one delta share its row and
  // column lists
  I2sPlan p{};
  p.nact = nact;
  int dmax = 0;
  for (int a = 0; a < nact; ++a)
    for (int b = 0; b < nact; ++b) dmax = std::max(dmax, std::abs(mval[a] - mval[b]));
  for (int d = -dmax; d <= dmax; ++d) {
    const int row0 = p.nrow, col0 = p.ncol;
    for (int i = 0; i < nact; ++i)
      for (int j = 0; j <= i; ++j)
        if (mval[i] - mval[j] == d) { p.row_ij[p.nrow][0] = (unsigned char)i; p.row_ij[p.nrow][1] = (unsigned char)j; ++p.nrow; }
    for (int k = 0; k < nact; ++k)
      for (int l = 0; l < nact; ++l)
        if (mval[l] - mval[k] == d) { p.col_kl[p.ncol][0] = (unsigned char)k; p.col_kl[p.ncol][1] = (unsigned char)l; ++p.ncol; }
    const int nr = p.nrow - row0, nc = p.ncol - col0;
    if (nr == 0 || nc == 0) { p.nrow = row0; p.ncol = col0; continue; }
    const int cchunk = std::min(nc, I2S_COLCHUNK);
    for (int r = 0; r < nr; r += I2S_ROWCHUNK)
      for (int c = 0; c < nc; c += cchunk) {
        if (p.nblocks == I2S_MAXBLK) {
          fprintf(stderr, "td1c_gpu_int2e_static: more than %d int2e blocks\n", I2S_MAXBLK);
          return ST_CONFIG;
        }
        I2sBlk& b = p.blk[p.nblocks++];
        b.row0 = (unsigned short)(row0 + r); b.nrow = (unsigned char)std::min(I2S_ROWCHUNK, nr - r);
        b.col0 = (unsigned short)(col0 + c); b.ncol = (unsigned char)std::min(cchunk, nc - c);
        b.ent0 = p.nblkent;
        p.nblkent += b.nrow * b.ncol;
      }
  }
  // the K split: the library's own 128 where the partial sums fit, fewer
  // (same sums, coarser split) where they do not
  int nsplit = 1;
  if (p.nblkent > 0) {
    const size_t room = (I2S_SCRATCH_BYTES - OFF_PART) / (sizeof(cplx) * (size_t)p.nblkent);
    if (room < 1) {
      fprintf(stderr, "td1c_gpu_int2e_static: %d block entries exceed the %zu-byte scratch\n", p.nblkent,
              I2S_SCRATCH_BYTES);
      return ST_CONFIG;
    }
    nsplit = (int)std::min<size_t>(I2S_NSPLIT, room);
  }
  unsigned char* base = static_cast<unsigned char*>(scratch_for_current_device());
  if (!base) return ST_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Int2eArgs a{};
  a.nact = nact; a.nblocks = p.nblocks; a.nblkent = p.nblkent; a.K = (size_t)K;
  a.blocks = reinterpret_cast<Int2eBlock*>(base + OFF_BLK);
  a.row_pair = reinterpret_cast<int*>(base + OFF_ROW);
  a.col_pair = reinterpret_cast<int2*>(base + OFF_COL);
  a.ent_dst = reinterpret_cast<int4*>(base + OFF_DST);
  a.partial = reinterpret_cast<cplx*>(base + OFF_PART);
  a.rho2 = reinterpret_cast<const cplx*>(d_rho2);
  a.v2sph = reinterpret_cast<const cplx*>(d_v2sph);
  a.int2e = reinterpret_cast<cplx*>(d_int2e);
  if (p.nblocks > 0) {
    i2s_expand_kernel<<<8, 256, 0, st>>>(p, const_cast<Int2eBlock*>(a.blocks), const_cast<int*>(a.row_pair),
                                          const_cast<int2*>(a.col_pair), const_cast<int4*>(a.ent_dst));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      fprintf(stderr, "td1c_gpu_int2e_static: table expansion launch: %s\n", cudaGetErrorString(e));
      return ST_CUDA;
    }
  }
  // clears the output, runs the block GEMM, the fixed-order sum and the fill
  return launch_int2e(a, nsplit, st) == 0 ? 0 : ST_CUDA;
}

}  // extern "C"
