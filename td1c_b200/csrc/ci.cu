// ci.cu -- CAS CI part of the RHS: 1-/2-RDMs (ormas_mkden1_ras.F90,
// ormas_mkden2_ras.F90) and the sigma vector (ormas_hcic_ras.F90, called via
// ormas_xact2.F90:44-80 with the ormas_phase energy shift).
//
// Formulation (same H, same RDM definitions as the reference, organised for
// the GPU around one-particle coupling vectors):
//   D^s_pq = E^s_pq c   (s = alpha, beta), a vector in the determinant sector
//            of total M = mtot + m_p - m_q, computed by a gather per element.
//   den1(x,y) = <E_yx> = c^H D_yx                (x,y same m)
//   den2(p,q,r,s) = <E_qp E_sr> - d_ps den1(r,q) = D_pq^H D_sr - d_ps den1(r,q)
//   sigma = sum_rs k_rs D_rs + 1/2 sum_rs E_rs T_rs,  T_rs = sum_pq (rs|pq) D_pq,
//           k_rs = h_rs - 1/2 sum_t (rt|ts)
// For singlets with nela = nelb the reference keeps only the beta parts of
// the RDMs and doubles them (ormas_mkden1_ras.F90:28-32,
// ormas_mkden2_ras.F90:77,161,292); spin_sym reproduces that.
// Determinant sectors: beta string blocks of alpha strings of matching M,
// both string lists sorted by (M, bit mask); the CI vector is the sector mtot.
#include "common.cuh"
#include "kernels.cuh"

namespace td1c {

__device__ __forceinline__ unsigned excite_str(unsigned s, int p, int q, int& sg) {
  // a^+_p a_q |s>; returns ~0u when zero
  if (!((s >> q) & 1u)) return ~0u;
  unsigned t = s & ~(1u << q);
  if ((t >> p) & 1u) return ~0u;
  int lo = min(p, q), hi = max(p, q);
  unsigned between = (hi - lo > 1) ? (t & (((1u << hi) - 1u) & ~((1u << (lo + 1)) - 1u))) : 0u;
  sg = (__popc(between) & 1) ? -1 : 1;
  return t | (1u << p);
}

// index of determinant (ia, ib) in sector sec, or -1
__device__ __forceinline__ int det_in_sector(const CiTables& t, int sec, int ia, int ib) {
  if (ia < 0 || ib < 0) return -1;
  int off = t.sec_off[sec * t.nstr_b + ib];
  if (off < 0) return -1;
  int p = ia - t.sec_first[sec * t.nstr_b + ib];
  if (p < 0 || p >= t.sec_cnt[sec * t.nstr_b + ib]) return -1;
  return off + p;
}

// D^s_pq[K] = sum_I <K|E^s_pq|I> c_I : I = E^s_qp K
__global__ void ci_dvec_kernel(CiArgs a) {
  const CiTables& t = a.t;
  const int pq = blockIdx.y;
  const int n = t.nact;
  const int p = pq % n, q = pq / n;  // Fortran-style pq = p + n q
  const int S = t.mtot + t.orb_m[p] - t.orb_m[q];
  const int sec = S - t.smin;
  if (sec < 0 || sec >= t.nsec) return;
  const int size = t.sec_size[sec];
  const int K = blockIdx.x * blockDim.x + threadIdx.x;
  if (K >= size) return;
  const long o = t.dvec_off[pq];
  const int ka = t.sec_detA[t.sec_base[sec] + K], kb = t.sec_detB[t.sec_base[sec] + K];
  const int sec0 = t.mtot - t.smin;
  cplx da = mkc(0, 0), db = mkc(0, 0);
  int sg;
  unsigned ia = excite_str(t.stra[ka], q, p, sg);
  if (ia != ~0u) {
    int I = det_in_sector(t, sec0, t.idx_a[ia], kb);
    if (I >= 0) da = cscale(a.cic[I], (double)sg);
  }
  unsigned ib = excite_str(t.strb[kb], q, p, sg);
  if (ib != ~0u) {
    int I = det_in_sector(t, sec0, ka, t.idx_b[ib]);
    if (I >= 0) db = cscale(a.cic[I], (double)sg);
  }
  a.Da[o + K] = da;
  a.Db[o + K] = db;
}

template <int NT>
__device__ __forceinline__ cplx block_sum(cplx v) {
  __shared__ double sx[NT], sy[NT];
  sx[threadIdx.x] = v.x; sy[threadIdx.x] = v.y;
  __syncthreads();
  for (int s = NT / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) { sx[threadIdx.x] += sx[threadIdx.x + s]; sy[threadIdx.x] += sy[threadIdx.x + s]; }
    __syncthreads();
  }
  return mkc(sx[0], sy[0]);
}

// den1(x, y) = <E_yx>: block per (x, y)
__global__ void __launch_bounds__(256) ci_den1_kernel(CiArgs a) {
  const CiTables& t = a.t;
  const int n = t.nact;
  const int x = blockIdx.x % n, y = blockIdx.x / n;
  if (t.orb_m[x] != t.orb_m[y]) { if (threadIdx.x == 0) a.den1[x + n * y] = mkc(0, 0); return; }
  const int yx = y + n * x;
  const long o = t.dvec_off[yx];
  cplx s = mkc(0, 0);
  for (int J = threadIdx.x; J < t.lcic; J += blockDim.x) {
    cplx c = a.cic[J];
    cplx d = t.spin_sym ? cscale(a.Db[o + J], 2.0) : cadd(a.Da[o + J], a.Db[o + J]);
    s = cadd(s, cmulc(c, d));
  }
  s = block_sum<256>(s);
  if (threadIdx.x == 0) a.den1[x + n * y] = s;
}

// G(p,q,r,s) = D_pq^H D_sr over the common sector; block per m-allowed quadruple
__global__ void __launch_bounds__(256) ci_den2_kernel(CiArgs a) {
  const CiTables& t = a.t;
  const int n = t.nact;
  const int4 qd = t.quads[blockIdx.x];
  const int p = qd.x, q = qd.y, r = qd.z, s_ = qd.w;
  const int pq = p + n * q, sr = s_ + n * r;
  const int S = t.mtot + t.orb_m[p] - t.orb_m[q];
  const int sec = S - t.smin;
  const int size = (sec >= 0 && sec < t.nsec) ? t.sec_size[sec] : 0;
  const long o1 = t.dvec_off[pq], o2 = t.dvec_off[sr];
  cplx acc = mkc(0, 0);
  for (int K = threadIdx.x; K < size; K += blockDim.x) {
    cplx u, v;
    if (t.spin_sym) { u = a.Db[o1 + K]; v = cscale(cadd(a.Da[o2 + K], a.Db[o2 + K]), 2.0); }
    else { u = cadd(a.Da[o1 + K], a.Db[o1 + K]); v = cadd(a.Da[o2 + K], a.Db[o2 + K]); }
    acc = cadd(acc, cmulc(u, v));
  }
  acc = block_sum<256>(acc);
  if (threadIdx.x == 0) a.den2[p + n * (q + n * (r + n * s_))] = acc;
}

__global__ void ci_den2_delta_kernel(CiArgs a) {
  const int n = a.t.nact;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * n * n) return;
  int p = t % n, q = (t / n) % n, r = t / (n * n);
  // den2(p,q,r,p) -= den1(r,q)   (ormas_mkden2_ras.F90:339-346)
  cplx& d = a.den2[p + n * (q + n * (r + n * p))];
  d = csub(d, a.den1[r + n * q]);
}

// T_rs[K] = sum_pq (rs|pq) D_pq[K], D = D^a + D^b
__global__ void ci_tvec_kernel(CiArgs a) {
  const CiTables& t = a.t;
  const int n = t.nact;
  const int rs = blockIdx.y;
  const int r = rs % n, s = rs / n;  // rs = r + n s
  const int S = t.mtot + t.orb_m[s] - t.orb_m[r];
  const int sec = S - t.smin;
  if (sec < 0 || sec >= t.nsec) return;
  const int size = t.sec_size[sec];
  const int K = blockIdx.x * blockDim.x + threadIdx.x;
  if (K >= size) return;
  // pq with m_p - m_q = m_s - m_r: group of that delta
  const int g = (t.orb_m[s] - t.orb_m[r]) - (t.smin - t.mtot);
  cplx acc = mkc(0, 0);
  for (int e = t.dgrp_off[g]; e < t.dgrp_off[g + 1]; ++e) {
    const int pq = t.dgrp[e];
    const int p = pq % n, q = pq / n;
    cplx I2 = a.int2e[r + n * (s + n * (p + n * q))];
    const long o = t.dvec_off[pq];
    cfma(acc, I2, cadd(a.Da[o + K], a.Db[o + K]));
  }
  a.T[t.dvec_off[s + n * r] + K] = acc;  // T_rs shares the sector (and layout) of D_sr
}

// sigma_J = sum_rs k_rs D_rs[J] + 1/2 sum_rs (E_rs T_rs)[J]; then
// hcic = fac (sigma - E_act c)
__global__ void __launch_bounds__(128) ci_sigma_kernel(CiArgs a) {
  // one warp per determinant J, lanes over the (r, s) pairs, fixed-order
  // shuffle reduction
  const CiTables& t = a.t;
  const int n = t.nact;
  __shared__ cplx sk[16 * 16];
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int r = e % n, s = e / n;
    cplx k = a.int1e[r + n * s];
    for (int u = 0; u < n; ++u) k = csub(k, cscale(a.int2e[r + n * (u + n * (u + n * s))], 0.5));
    sk[e] = k;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int J = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (J >= t.lcic) return;
  const int ja = t.det_a[J], jb = t.det_b[J];
  const unsigned sa = t.stra[ja], sbs = t.strb[jb];
  cplx sig = mkc(0, 0);
  for (int rs = lane; rs < n * n; rs += 32) {
    const int r = rs % n, s = rs / n;
    const long o = t.dvec_off[rs];
    if (t.orb_m[r] == t.orb_m[s]) cfma(sig, sk[rs], cadd(a.Da[o + J], a.Db[o + J]));
    const int sec = t.mtot + t.orb_m[s] - t.orb_m[r] - t.smin;
    if (sec < 0 || sec >= t.nsec) continue;
    const long ot = t.dvec_off[s + n * r];
    int sg;
    // K = E_sr J (alpha), then beta
    unsigned ka = excite_str(sa, s, r, sg);
    if (ka != ~0u) {
      int K = det_in_sector(t, sec, t.idx_a[ka], jb);
      if (K >= 0) sig = cadd(sig, cscale(a.T[ot + K], 0.5 * sg));
    }
    unsigned kb = excite_str(sbs, s, r, sg);
    if (kb != ~0u) {
      int K = det_in_sector(t, sec, ja, t.idx_b[kb]);
      if (K >= 0) sig = cadd(sig, cscale(a.T[ot + K], 0.5 * sg));
    }
  }
  for (int o = 16; o > 0; o >>= 1) { sig.x += __shfl_xor_sync(0xffffffff, sig.x, o); sig.y += __shfl_xor_sync(0xffffffff, sig.y, o); }
  if (lane != 0) return;
  const double e = *a.ene_act;
  cplx c = a.cic[J];
  sig = csub(sig, cscale(c, e));
  cplx fac = a.icomp == 1 ? mkc(0.0, -a.dtime) : mkc(-a.dtime, 0.0);
  a.sigma[J] = cmul(sig, fac);
}

int launch_ci_dvec(const CiArgs& a, int maxsec, cudaStream_t st) {
  const int n = a.t.nact;
  dim3 grid((maxsec + 127) / 128, n * n);
  ci_dvec_kernel<<<grid, 128, 0, st>>>(a);
  return (int)cudaGetLastError();
}

int launch_ci_rdm(const CiArgs& a, cudaStream_t st) {
  const int n = a.t.nact;
  ci_den1_kernel<<<n * n, 256, 0, st>>>(a);
  cudaMemsetAsync(a.den2, 0, sizeof(cplx) * (size_t)n * n * n * n, st);
  if (a.t.nquad > 0) ci_den2_kernel<<<a.t.nquad, 256, 0, st>>>(a);
  ci_den2_delta_kernel<<<(n * n * n + 127) / 128, 128, 0, st>>>(a);
  return (int)cudaGetLastError();
}

int launch_ci_tvec(const CiArgs& a, int maxsec, cudaStream_t st) {
  const int n = a.t.nact;
  dim3 grid((maxsec + 127) / 128, n * n);
  ci_tvec_kernel<<<grid, 128, 0, st>>>(a);
  return (int)cudaGetLastError();
}

int launch_ci_sigma(const CiArgs& a, cudaStream_t st) {
  ci_sigma_kernel<<<(a.t.lcic + 3) / 4, 128, 0, st>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace td1c
