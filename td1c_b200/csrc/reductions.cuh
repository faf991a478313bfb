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

}  // namespace td1c
