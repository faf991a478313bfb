// reductions.cuh -- argument blocks of the orbital matrix-element and int2e kernels.
#pragma once
#include "common.cuh"

namespace td1c {

struct OrbdotsArgs {
  int nbas, nfun, nent;
  const cplx* orb; const cplx* h0orb; const cplx* h1orb; const cplx* gorb; const cplx* v2orb;
  const int4* ent;   // [nent] (kind, j, i, 0): kind 0 A, 1 B, 2 C, 3 E, 4 GV
  cplx* partial;     // [nchunk][nent]
  cplx* result;      // [nent]
};
int orbdots_nchunk(size_t nbas);  // chunks (CTAs) of the orbdots pass; the partial buffer holds nchunk x nent
int launch_orbdots(const OrbdotsArgs& a, cudaStream_t st);

struct Int2eBlock { int row0, nrow, col0, ncol, ent0, pad0, pad1, pad2; };
struct Int2eArgs {
  int nact, nblocks, nblkent;
  size_t K;                 // Nr * (lmax2 + 1)
  const Int2eBlock* blocks;
  const int* row_pair;      // stored pair index of each block row (ij, i >= j)
  const int2* col_pair;     // (stored pair, conj) of each block column (kl)
  const int4* ent_dst;      // [nblkent] (i, j, k, l) active indices
  const cplx* rho2;         // [npair][K]
  const cplx* v2sph;        // [npair][K]
  cplx* partial;            // [nsplit][nblkent]
  cplx* int2e;              // [nact^4]
};
int launch_int2e(const Int2eArgs& a, int nsplit, cudaStream_t st);

// int2e on the FP64 tensor cores (DMMA m8n8k4), split over K.  Every
// Delta-m block is padded to m-tiles of 8 row pairs (rho2) and n-tiles of 8
// columns (v2sph); a group is one m-tile x up to I2D_NTMAX n-tiles, and the
// host assigns at most I2D_MAXG groups to each warp (-1: none).
constexpr int I2D_NW = 16, I2D_MAXG = 1, I2D_NTMAX = 3;
struct I2dGroup { int arow0, brow0, nnt, pad; };  // 8 A rows x nnt n-tiles (8 B rows each)
struct I2dArgs {
  int nra, nrb, ngroups, nblkent;
  size_t K;
  const int* a_pair;     // [nra] stored pair of the padded A row (-1: padding)
  const int* a_ent;      // [nra] first entry of the row (ent0 + r ncol), -1 for padding
  const int2* b_pair;    // [nrb] (stored pair, conj) of the padded B row ((-1, 0): padding)
  const int* b_col;      // [nrb] column index inside its block, -1 for padding
  const I2dGroup* groups;
  const int* warp_group;  // [nsets][I2D_NW][I2D_MAXG] group of each warp slot, -1: none
  int nsets;
  const cplx* rho2;
  const cplx* v2sph;
  double* partial;       // [nsplit][nblkent][2]
};
int launch_int2e_sum_fill(const Int2eArgs& a, int nsplit, cudaStream_t st);
size_t int2e_dmma_smem(const I2dArgs& a);
bool int2e_dmma_fits(const I2dArgs& a);
int launch_int2e_dmma(const I2dArgs& d, const Int2eArgs& sum, int nsplit, cudaStream_t st);

// int2e in split TF32 on tcgen05 (the mixed-precision form): every product of
// the P stored active pairs in one 128 x 2NB GEMM per K slice, entries formed
// from it per CTA (the same entry list and partial layout as the DMMA plan).
struct I2tArgs {
  int P, NB;             // stored active pairs (<= 64); B rows per part (>= P, multiple of 16)
  size_t K;
  const int* pair;       // [P] stored pair index of compact pair p
  const int4* ent;       // [nent] (row pair, column pair, conjugated column, 0) of each entry
  int nent;
  const cplx* rho2;
  const cplx* v2sph;
  cplx* partial;         // [nsplit][nent]
  int* status;
};
size_t int2e_tc_smem(const I2tArgs& a);
bool int2e_tc_fits(const I2tArgs& a);
int launch_int2e_tc(const I2tArgs& t, const Int2eArgs& sum, int nsplit, cudaStream_t st);

}  // namespace td1c
